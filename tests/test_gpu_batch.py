"""Batched multi-scene rendering on the GPU: scenes of different sizes, spp, depths and materials share one
wavefront whose slots are refilled from every scene's (pixel, sample) space.  Each path is the one a
single-scene launch traces, so every scene's film equals its own single-scene render within accumulation
rounding (1e-5 relative), with and without graph replay and with a wavefront much smaller than the work."""
import numpy as np
import pytest

from piper2_b200 import scenes

pytestmark = pytest.mark.gpu


def _api():
    from piper2_b200 import api

    return api


def _scene_set():
    return [
        scenes.cornell_box(seed=1, width=64, height=48, spp=4),
        scenes.cornell_box(seed=2, width=40, height=40, spp=8, max_depth=5),
        scenes.guiding_room(seed=0, width=48, height=27, spp=2, max_depth=16),
        scenes.cornell_box(seed=3, width=16, height=24, spp=1),
    ]


def _single_films(sds):
    out = []
    for sd in sds:
        with _api().Pipeline(sd) as pl:
            film, _ = pl.render()
        out.append(film)
    return out


@pytest.mark.parametrize("capacity,graph", [(1 << 20, 1), (1024, 1), (3000, 0)])
def test_batch_films_match_single_scene(capacity, graph):
    sds = _scene_set()
    ref = _single_films(sds)
    with _api().Batch(sds) as b:
        b.set_config(capacity=capacity, use_graph=graph)
        b.render()
        for i, r in enumerate(ref):
            np.testing.assert_allclose(b.film(i), r, rtol=1e-5, atol=1e-6)
        ms, total, iters = b.timing()
        assert np.all(ms > 0) and np.all(ms <= total * 1.001 + 0.05) and iters > 0
        st = b.stats()
        assert st.paths == sum(sd.settings.width * sd.settings.height * sd.settings.samples_per_pixel for sd in sds)
        # a second render of the same batch gives the same films (state fully reset)
        b.render()
        for i, r in enumerate(ref):
            np.testing.assert_allclose(b.film(i), r, rtol=1e-5, atol=1e-6)


def test_batch_autotune_and_config_checks():
    from piper2_b200 import capi

    sds = _scene_set()
    with _api().Batch(sds) as b:
        cfg, ms = b.autotune()
        assert cfg.capacity >= 1024 and cfg.shade_block in (64, 128, 256, 512) and ms > 0
        b.render()
        ref = _single_films(sds)
        for i, r in enumerate(ref):
            np.testing.assert_allclose(b.film(i), r, rtol=1e-5, atol=1e-6)
        with pytest.raises(capi.PB2Error):
            b.set_config(capacity=10)
        with pytest.raises(capi.PB2Error):
            b.set_config(shade_block=100)
