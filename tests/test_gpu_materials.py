"""GPU parity, against the CPU oracle, for the parts of the render path the Cornell configuration does not
reach: the reference's other surfaces (Surface/Classic/Kernel.cpp), the thin-lens aperture of the camera
(PerspectiveCamera/Kernel.cpp:22-48) and the triangle and gaussian film filters
(RenderDriver/FixedSampler/Kernel.cpp:55-69).

Per-sample radiance must be bit-identical (same Sobol dimensions, same arithmetic order, same traversal);
films agree within accumulation rounding (1e-5 relative + 1e-6 absolute), because the film sums use
atomics in any order, as the reference's CAS loop does (Tracer/Embree/Embree.cpp:420-428)."""
import ctypes as C

import numpy as np
import pytest

from piper2_b200 import capi, scenes

pytestmark = pytest.mark.gpu


def _api():
    from piper2_b200 import api

    return api


def _assert_samples_equal(samples, osamples):
    diff = np.any(samples.view(np.uint32) != osamples.view(np.uint32), axis=-1)
    assert not diff.any(), f"{diff.sum()} of {diff.size} samples differ"


def _render_both(oracle, sd, use_bvh=False):
    with _api().Pipeline(sd) as pl:
        film, samples = pl.render(samples=True)
    ofilm, osamples = oracle.OracleScene(sd, use_bvh=use_bvh).render(sd.settings)
    return film, samples, ofilm, osamples


def _six_material_box(seed, size, spp):
    """The Cornell box with every surface the C ABI accepts from the reference's Classic module:
    Plastic (Lambert + GGX MicrofacetReflection with dielectric Fresnel, Kernel.cpp:384-470), Oren-Nayar
    Matte (:103-109), Substrate (FresnelBlend), smooth Glass (FresnelSpecular, :500-537), rough Glass
    (GGX reflection + MicrofacetTransmission, :539-600) and Mirror (:680-692)."""
    sd = scenes.cornell_box(seed=seed, width=size, height=size, spp=spp)
    sd.materials = [scenes.material("Plastic", (0.4, 0.4, 0.4), (0.5, 0.5, 0.5), (0.3, 0)),
                    scenes.material("Matte", (0.65, 0.05, 0.05), roughness=(0.4, 0)),
                    scenes.material("Substrate", (0.12, 0.45, 0.15), (0.2, 0.2, 0.2), (0.2, 0.3)),
                    scenes.material("Glass", (1, 1, 1), (1, 1, 1), (0, 0)),
                    scenes.material("Glass", (1, 1, 1), (1, 1, 1), (0.2, 0.2)),
                    scenes.material("Mirror", (0.9, 0.9, 0.9))]
    sd.meshes[5].material = 3   # short box: smooth glass
    sd.meshes[6].material = 4   # tall box: rough glass
    sd.meshes[2].material = 5   # back wall: mirror
    return sd


@pytest.mark.parametrize("seed,size,spp", [(6, 24, 8), (7, 48, 16)])
def test_reference_surfaces_samples_bitexact(oracle, seed, size, spp):
    sd = _six_material_box(seed, size, spp)
    film, samples, ofilm, osamples = _render_both(oracle, sd)
    _assert_samples_equal(samples, osamples)
    np.testing.assert_allclose(film, ofilm, rtol=1e-5, atol=1e-6)


def test_reference_surfaces_deep_paths_bitexact(oracle):
    """Depth 16 without Russian roulette, so chains of glossy and specular bounces (glass inside glass,
    mirror to glass) run to the depth limit; uses the oracle's BVH."""
    sd = _six_material_box(8, 32, 4)
    sd.settings.max_depth, sd.settings.min_rr_depth = 16, 16
    _, samples, _, osamples = _render_both(oracle, sd, use_bvh=True)
    _assert_samples_equal(samples, osamples)


def test_second_plastic_and_substrate_parameters_bitexact(oracle):
    """Other roughness values of the microfacet lobes, including anisotropic Substrate and a nearly smooth
    Plastic, on every wall."""
    sd = scenes.cornell_box(seed=9, width=32, height=32, spp=8)
    sd.materials = [scenes.material("Plastic", (0.2, 0.5, 0.3), (0.6, 0.6, 0.6), (0.02, 0)),
                    scenes.material("Substrate", (0.6, 0.2, 0.2), (0.3, 0.3, 0.3), (0.05, 0.6)),
                    scenes.material("Plastic", (0.7, 0.7, 0.7), (0.3, 0.2, 0.1), (0.8, 0)),
                    scenes.material("Matte", (0.5, 0.5, 0.5), roughness=(1.0, 0))]
    for i, m in enumerate(sd.meshes):
        m.material = i % 4
    _, samples, _, osamples = _render_both(oracle, sd)
    _assert_samples_equal(samples, osamples)


def test_thin_lens_camera_rays_bitexact(oracle):
    """A finite aperture (FStop 1.4 at 35 mm: radius 12.5 mm), so the lens-disk sample of dims 3/4 moves
    the ray origin (PerspectiveCamera.cpp:43-44, Src/Kernel/Sampling.hpp:24-29)."""
    sd = scenes.cornell_box(seed=0, width=40, height=24)
    focal_mm = 35.0
    sensor_mm = 2.0 * focal_mm * np.tan(np.radians(20.0))
    sd.settings.camera = scenes.camera_from_config((0.5, 0.5, -1.4), (0.5, 0.5, 0.5), (0.0, 1.0, 0.0),
                                                   (sensor_mm, sensor_mm), focal_mm, 1.4)
    st = sd.settings
    assert st.camera.aperture_radius > 0.01
    with _api().Pipeline(sd) as pl:
        rays, pts = pl.camera_rays(sample=5)
        rect, ndc = pl.rect, pl.ndc
    full = oracle.full_rect(st)
    log2res = int(np.ceil(np.log2(max(full.width, full.height))))
    spread = []
    for k in range(0, rect.width * rect.height, 3):
        px, py = pts[k]
        nx = np.float32(ndc.ox) + np.float32(ndc.sx) * np.float32(px) / np.float32(st.width)
        ny = np.float32(ndc.oy) + np.float32(ndc.sy) * np.float32(py) / np.float32(st.height)
        col, row = k % rect.width, k // rect.width
        oi = C.c_uint64()
        oo = (C.c_float * 2)()
        oracle.oracle().or_sobol_start(1 << log2res, log2res, col, row, 5, C.byref(oi), oo)
        u1 = oracle.oracle().or_sobol_sample(oi.value, 3)
        u2 = oracle.oracle().or_sobol_sample(oi.value, 4)
        r = capi.Ray()
        oracle.oracle().or_camera_ray(C.byref(st.camera), float(nx), float(ny), u1, u2, C.byref(r))
        exp = np.array(list(r.org) + [r.tmin] + list(r.dir) + [r.tmax], dtype=np.float32)
        assert np.array_equal(rays[k].view(np.uint32), exp.view(np.uint32)), k
        spread.append(np.linalg.norm(exp[:3] - np.array(st.camera.position, dtype=np.float32)))
    assert max(spread) > 1e-3  # the aperture really moved the origins


def test_thin_lens_render_bitexact(oracle):
    sd = scenes.cornell_box(seed=3, width=32, height=32, spp=8)
    focal_mm = 35.0
    sensor_mm = 2.0 * focal_mm * np.tan(np.radians(20.0))
    sd.settings.camera = scenes.camera_from_config((0.5, 0.5, -1.4), (0.5, 0.3, 0.3), (0.0, 1.0, 0.0),
                                                   (sensor_mm, sensor_mm), focal_mm, 2.0)
    film, samples, ofilm, osamples = _render_both(oracle, sd)
    _assert_samples_equal(samples, osamples)
    np.testing.assert_allclose(film, ofilm, rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("filt,alpha", [("triangle", 2.0), ("gaussian", 2.0), ("gaussian", 0.5)])
def test_film_filters_match_oracle(oracle, filt, alpha):
    """Each sample is splatted into its 2 x 2 pixels with the filter's weight (FixedSampler/Kernel.cpp:30-69;
    the gaussian goes through exp): the RGBW film, weights included, within accumulation rounding."""
    sd = scenes.cornell_box(seed=4, width=40, height=32, spp=4)
    sd.settings.filter = capi.FILTER[filt]
    sd.settings.gaussian_alpha = alpha
    film, samples, ofilm, osamples = _render_both(oracle, sd)
    _assert_samples_equal(samples, osamples)
    np.testing.assert_allclose(film, ofilm, rtol=1e-5, atol=1e-6)
    # the weights differ from the box filter's (which is 1 per splat)
    assert not np.allclose(film[..., 3], np.round(film[..., 3]))


def test_tiled_overscan_rect_matches_oracle(oracle):
    """A non-square film with the OverScan fit mode (Sensor.hpp:36-75) and a sub-rect launch."""
    sd = scenes.cornell_box(seed=5, width=48, height=20, spp=4)
    sd.settings.fit_mode = capi.FIT["OverScan"]
    film, samples, ofilm, osamples = _render_both(oracle, sd)
    _assert_samples_equal(samples, osamples)
    np.testing.assert_allclose(film, ofilm, rtol=1e-5, atol=1e-6)
