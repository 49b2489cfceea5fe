"""Scene description -> pipeline -> frames on the GPU (the reference's Render operator, Src/PiperRenderer.cpp:
306-359): the committed Cornell-box and textured-room descriptions render through scene_json.render / its command
line into PFM frames equal to the directly built scenes' films (within the accumulation rounding of the film's
atomics, 1e-5 relative), every frame of a multi-frame action alike."""
import json
import os
import shutil

import numpy as np
import pytest

from piper2_b200 import api, scene_json, scenes

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
SCENES = os.path.join(HERE, "golden", "scenes")


def _direct(build):
    sd = build(seed=0, width=32, height=32, spp=4)
    with api.Pipeline(sd) as pl:
        film = pl.new_film()
        pl.launch(film)
        return pl.resolve(film).cpu().numpy()


@pytest.mark.parametrize("name,build", [("cornell", scenes.cornell_box), ("textured", scenes.textured_room)])
def test_frames_equal_direct_render(tmp_path, name, build):
    with open(os.path.join(SCENES, name, "scene.json")) as fh:
        desc = json.load(fh)
    desc["Actions"][0]["FrameCount"] = 2
    desc["Actions"].append(dict(desc["Actions"][0], FrameCount=1))
    paths = scene_json.render({"ImageSize": [32, 32], "SceneDesc": desc, "BaseDir": os.path.join(SCENES, name),
                               "OutputDir": str(tmp_path)})
    assert [os.path.relpath(p, tmp_path) for p in paths] == ["Action0/Frame0.pfm", "Action0/Frame1.pfm",
                                                             "Action1/Frame0.pfm"]
    expect = _direct(build)
    for p in paths:
        img = scene_json.read_pfm(p)
        assert img.shape == (32, 32, 3)
        assert np.allclose(img, expect, rtol=1e-5, atol=1e-6), p


def test_command_line(tmp_path):
    folder = tmp_path / "cornell"
    shutil.copytree(os.path.join(SCENES, "cornell"), folder)
    assert scene_json.main([str(folder / "options.json")]) == 0
    img = scene_json.read_pfm(str(folder / "out" / "Action0" / "Frame0.pfm"))
    assert np.allclose(img, _direct(scenes.cornell_box), rtol=1e-5, atol=1e-6)
