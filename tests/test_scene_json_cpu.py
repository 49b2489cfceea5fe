"""The scene-description path (the reference renderer's JSON scenes, Src/PiperRenderer.cpp:150-362) on the CPU:
the committed descriptions of the Cornell box and the textured room (tests/golden/make_scene_json.py) load into
scenes whose every sample, rendered by the oracle, equals the directly built scenes' bit for bit; the OBJ and
image readers; the PFM writer's handling of invalid pixels; and the errors for what the path does not support."""
import copy
import json
import os

import numpy as np
import pytest

from piper2_b200 import scene_json, scenes

HERE = os.path.dirname(os.path.abspath(__file__))
SCENES = os.path.join(HERE, "golden", "scenes")


@pytest.mark.parametrize("name,build", [("cornell", scenes.cornell_box), ("textured", scenes.textured_room)])
def test_description_renders_like_the_built_scene(oracle, name, build):
    ls = scene_json.load(os.path.join(SCENES, name, "scene.json"))
    sd = ls.scene_for("Camera", 32, 32, "Fill")
    ref = build(seed=0, width=32, height=32, spp=4)
    assert bytes(sd.settings) == bytes(ref.settings)
    assert sd.triangle_count == ref.triangle_count and sd.env_radiance == ref.env_radiance
    _, a = oracle.OracleScene(sd, use_bvh=False).render(sd.settings, threads=os.cpu_count())
    _, b = oracle.OracleScene(ref, use_bvh=False).render(ref.settings, threads=os.cpu_count())
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_actions_and_settings():
    ls = scene_json.load(os.path.join(SCENES, "cornell", "scene.json"))
    assert [(a.active_sensor, a.frame_count, a.fit_mode) for a in ls.actions] == [("Camera", 1, "Fill")]
    assert (ls.spp, ls.max_depth, ls.min_rr_depth, ls.filter, ls.scramble) == (4, 8, 3, "box", 0)
    st = ls.settings("Camera", 64, 48, "OverScan")
    assert (st.width, st.height, st.fit_mode) == (64, 48, 1)
    with pytest.raises(scene_json.SceneError, match="Failed to find a node with sensor named \"Nope\""):
        ls.settings("Nope", 8, 8)


def _desc():
    with open(os.path.join(SCENES, "cornell", "scene.json")) as fh:
        return json.load(fh)


def _load(d):
    return scene_json.load(d, base_dir=os.path.join(SCENES, "cornell"))


def test_unsupported_and_invalid_descriptions():
    d = _desc()
    d["Scene"]["Children"][0]["Surface"]["ClassID"] = "Piper.BuiltinComponent.ClassicSurface.Velvet"
    with pytest.raises(scene_json.SceneError, match="Velvet"):
        _load(d)
    d = _desc()
    d["Scene"]["Children"] = [c for c in d["Scene"]["Children"] if "SampledEnvironment" not in c.get("ClassID", "")]
    with pytest.raises(scene_json.SceneError, match="SampledEnvironment"):
        _load(d)
    d = _desc()
    d["Scene"]["Children"][0]["Transform"] = {"Offset": 0.0, "Step": 1.0, "KeyFrames": []}
    with pytest.raises(scene_json.SceneError, match="dynamic"):
        _load(d)
    d = _desc()
    d["Scene"]["Children"][0]["Surface"]["Diffuse"]["Value"] = [0.5, 0.5, 0.5]
    with pytest.raises(scene_json.SceneError, match="Unsupported channel 3"):
        _load(d)
    d = _desc()
    d["Scene"]["Children"][0]["Surface"]["Roughness"]["Value"] = [0.5, 0.5]
    with pytest.raises(scene_json.SceneError, match="Mismatched channel"):
        _load(d)
    d = _desc()
    d["RenderDriver"]["Filter"]["FilterType"] = "mitchell"
    with pytest.raises(scene_json.SceneError, match="mitchell"):
        _load(d)
    d = _desc()
    d["Scene"]["Children"][0]["Type"] = "Mesh"
    with pytest.raises(scene_json.SceneError, match="Invalid scene node"):
        _load(d)
    d = _desc()
    d["Scene"]["Children"].append({"Type": "Instance", "ClassID": "Piper.BuiltinComponent.BasicLight.Point",
                                   "Intensity": [1, 1, 1]})
    with pytest.raises(scene_json.SceneError, match="BasicLight.Point"):
        _load(d)
    d = _desc()
    d["Objects"] = [{"ID": "x", "ClassID": "NoDots"}]
    with pytest.raises(scene_json.SceneError, match="Invalid classID"):
        _load(d)


def test_rotated_instance_and_scramble(oracle):
    """A rotation in a group transform is flattened into world space (the library's divergence from the reference,
    which inverts instance transforms wrongly): the loaded mesh carries the SRT matrix of the transform."""
    d = _desc()
    node = copy.deepcopy(d["Scene"]["Children"][5])
    node["Transform"] = {"Translation": [0.1, 0.0, 0.0], "Rotation": [0.0, 0.3, 0.0], "Scale": 0.9}
    d["Scene"]["Children"][5] = node
    d["Sampler"]["Scramble"] = True
    ls = _load(d)
    m = ls.scene.meshes[5]
    expect = scenes.srt_matrix(translation=(0.1, 0.0, 0.0), scale=(0.9, 0.9, 0.9),
                               quat=scenes.euler_quaternion(0.0, 0.3, 0.0))
    assert m.transform is not None and np.array_equal(m.transform, expect)
    assert ls.scramble == 1


def test_obj_reader(tmp_path):
    p = tmp_path / "quad.obj"
    p.write_text("# a quad and a triangle\nv 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nvt 0 0\nvt 1 0\nvt 1 1\nvt 0 1\n"
                 "f 1/1 2/2 3/3 4/4\nf -4/-4 -2/-2 -1/-1\n")
    v, ix, tc = scene_json.load_obj(str(p))
    assert v.shape == (4, 3) and tc.shape == (4, 2)
    assert ix.tolist() == [[0, 1, 2], [0, 2, 3], [0, 2, 3]]
    p.write_text("v 0 0 0\nv 1 0 0\nf 1 2\n")
    with pytest.raises(scene_json.SceneError, match="fewer than three"):
        scene_json.load_obj(str(p))
    p.write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 9\n")
    with pytest.raises(scene_json.SceneError, match="out of range"):
        scene_json.load_obj(str(p))


def test_image_reader_and_pfm(tmp_path):
    img = np.arange(2 * 3 * 3, dtype=np.uint8).reshape(2, 3, 3)
    p = tmp_path / "a.ppm"
    p.write_bytes(b"P6\n# comment\n3 2\n255\n" + img.tobytes())
    assert np.array_equal(scene_json.load_image(str(p)), img)
    rgb = np.random.default_rng(0).uniform(0, 2, (5, 7, 3)).astype(np.float32)
    bad = rgb.copy()
    bad[1, 2] = (np.nan, 0, 0)
    bad[3, 4] = (0.5, -0.1, 0.2)
    q = str(tmp_path / "f.pfm")
    assert scene_json.write_pfm(q, bad) == 2
    back = scene_json.read_pfm(q)
    expect = rgb.copy()
    expect[1, 2] = expect[3, 4] = (1, 0, 0)
    assert np.array_equal(back, expect)
