"""A scene that reaches the library as Piper component payloads (pb2_builder_*, see test_builder_cpu.py) renders
exactly as the same scene given through the C ABI's scene description: every sample bit-identical."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("name", ["cornell_box", "six_materials_gaussian"])
def test_payload_built_pipeline_renders_identically(name):
    from piper2_b200 import api

    import test_builder_cpu as tb

    sd = tb.SCENES[name]()
    if name == "cornell_box":  # a smaller frame of the same scene
        sd.settings.width = sd.settings.height = 64
        sd.settings.samples_per_pixel = 4
    b, sd = tb.replay(name, sd)
    with api.Pipeline(b) as pl:
        film_b, samples_b = pl.render(samples=True)
    with api.Pipeline(sd) as pl:
        film_d, samples_d = pl.render(samples=True)
    b.close()
    assert np.array_equal(samples_b.view(np.uint32), samples_d.view(np.uint32))
    np.testing.assert_allclose(film_b, film_d, rtol=1e-5, atol=1e-6)
