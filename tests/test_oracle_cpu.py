"""CPU checks of the oracle itself: the Sobol tables, the elementary functions, the BVH traversal, and
the render restatement against the reference's own kernels (compiled natively into
oracle/_ref/librefcpu.so when the reference sources are present) or, without them, against the
golden vectors those kernels produced (tests/golden/, made by tests/golden/make_golden.py)."""
import ctypes as C
import math
import os

import numpy as np
import pytest

from piper2_b200 import capi, scenes, sobol_tables

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# The Sobol tables are regenerated from the Joe-Kuo direction numbers; this digest pins them.
SOBOL_DIGEST = None  # filled from tests/golden/sobol_digest.txt


def _golden_digest():
    with open(os.path.join(GOLDEN, "sobol_digest.txt")) as f:
        return f.read().strip()


def test_sobol_tables_digest(oracle):
    mat, vdc, inv = sobol_tables.tables()
    d = sobol_tables.checksum(mat, vdc, inv)
    assert d == _golden_digest()
    assert oracle.oracle().or_sobol_digest().decode() == d


def test_sobol_matches_scipy_gray_code():
    """SciPy's Sobol generator (Joe-Kuo data) visits the points in Gray-code order."""
    from scipy.stats import qmc

    mat = sobol_tables.sobol_matrices32()
    for dims in (range(0, 8), range(1000, 1024)):
        d = len(dims)
        pts = qmc.Sobol(max(dims) + 1, scramble=False, bits=32).random(512)[:, list(dims)]
        for k in range(512):
            g = k ^ (k >> 1)
            for j, dim in enumerate(dims):
                v, i, c = 0, g, 0
                while i:
                    if i & 1:
                        v ^= int(mat[dim * 52 + c])
                    i >>= 1
                    c += 1
                assert v / 2**32 == pts[k, j]


def test_sobol_02_net(oracle):
    """Dimensions 0/1 form a (0,2)-sequence: every 2^(2m) block has one point per 2^-m x 2^-m cell, and
    sobolIntervalToIndex finds, for pixel (px, py) and sample s, the index of block s in that pixel."""
    o = oracle.oracle()
    m = 4
    res = 1 << m
    for s in (0, 1, 5):
        seen = set()
        for px in range(res):
            for py in range(res):
                idx = o.or_sobol_interval_to_index(m, s, px, py)
                assert idx >> (2 * m) == s
                x, y = o.or_sobol_sample(idx, 0), o.or_sobol_sample(idx, 1)
                assert int(x * res) == px and int(y * res) == py
                seen.add(idx)
        assert len(seen) == res * res


def test_elementary_functions_accuracy():
    """pb2_math sin/cos/exp/acos against the C library (through the oracle build): within 2 ulp."""
    import subprocess
    import tempfile

    src = r"""
    #include <stdio.h>
    #include <math.h>
    #include "pb2_math.h"
    int main(void) {
        double worst[4] = {0, 0, 0, 0};
        for (int i = 0; i <= 2000000; ++i) {
            float x = -7.0f + 14.0f * (float)i / 2000000.0f;
            float s, c; pb2_sincosf(x, &s, &c);
            double es = sin((double)x), ec = cos((double)x);
            double us = fabs(s - es) / nextafterf(fabsf((float)es) + 1e-30f, INFINITY) * 0;
            double ds = fabs((double)s - es) / fmax(fabs(es) * 1.1920929e-7, 1.4e-45);
            double dc = fabs((double)c - ec) / fmax(fabs(ec) * 1.1920929e-7, 1.4e-45);
            if (fabs(es) > 1e-6 && ds > worst[0]) worst[0] = ds;
            if (fabs(ec) > 1e-6 && dc > worst[1]) worst[1] = dc;
            float xe = -20.0f + 20.0f * (float)i / 2000000.0f;
            double ee = exp((double)xe);
            double de = fabs((double)pb2_expf(xe) - ee) / (ee * 1.1920929e-7);
            if (de > worst[2]) worst[2] = de;
            float xa = -1.0f + 2.0f * (float)i / 2000000.0f;
            double ea = acos((double)xa);
            double da = ea > 0 ? fabs((double)pb2_acosf(xa) - ea) / (ea * 1.1920929e-7) : 0;
            if (da > worst[3]) worst[3] = da;
            (void)us;
        }
        printf("%g %g %g %g\n", worst[0], worst[1], worst[2], worst[3]);
        return 0;
    }
    """
    root = os.path.dirname(GOLDEN.rstrip("/").rsplit("/", 1)[0] + "/x")
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "piper2_b200", "csrc")
    with tempfile.TemporaryDirectory() as td:
        c = os.path.join(td, "t.c")
        with open(c, "w") as f:
            f.write(src)
        exe = os.path.join(td, "t")
        subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-I", inc, c, "-o", exe, "-lm"], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    worst = [float(v) for v in out]
    # relative error in units of 2^-23 (1 ulp at the bottom of a binade is 2^-23 relative)
    assert worst[0] < 4 and worst[1] < 4, worst
    assert worst[2] < 4 and worst[3] < 4, worst
    del root


def test_plane_make_python_equals_oracle(oracle):
    for origin, u, v in [((0.375, 0.999, 0.375), (0.25, 0, 0), (0, 0, 0.25)),
                         ((1, 2, 3), (0.3, -0.2, 0.7), (0.1, 0.9, -0.4)),
                         ((0, 0, 0), (0, 0, 2), (0, 3, 0))]:
        py = scenes.plane_make(origin, u, v)
        op = capi.Plane()
        f = lambda t: (C.c_float * 3)(*t)  # noqa: E731
        oracle.oracle().or_plane_make(f(origin), f(u), f(v), C.byref(op))
        assert bytes(py) == bytes(op)


def test_bvh_oracle_equals_bruteforce(oracle):
    soup = scenes.triangle_soup(3000, seed=4)
    rays = scenes.soup_rays(3000, seed=5)
    a = oracle.OracleScene(soup, use_bvh=True).trace_closest(rays)
    b = oracle.OracleScene(soup, use_bvh=False).trace_closest(rays)
    assert np.array_equal(a["prim"], b["prim"]) and np.array_equal(a["t"], b["t"])
    srays = scenes.soup_rays(3000, seed=6, kind="any")
    assert np.array_equal(oracle.OracleScene(soup, use_bvh=True).trace_any(srays),
                          oracle.OracleScene(soup, use_bvh=False).trace_any(srays))


def _compare_to_reference(osamp, rsamp):
    assert np.array_equal(osamp[..., :2], rsamp[..., :2]), "film points differ"
    exact = np.all(osamp[..., 2:] == rsamp[..., 2:], axis=-1)
    rel = np.abs(osamp[..., 2:] - rsamp[..., 2:]).max(-1) / (np.abs(rsamp[..., 2:]).max(-1) + 1e-6)
    # differences come only from the C library's sin/cos vs pb2_math's (last-bit) on a few paths
    assert exact.mean() > 0.85, exact.mean()
    assert (rel > 1e-3).mean() < 5e-3, (rel > 1e-3).mean()
    m_o, m_r = osamp[..., 2:].mean(axis=(0, 1, 2)), rsamp[..., 2:].mean(axis=(0, 1, 2))
    np.testing.assert_allclose(m_o, m_r, rtol=2e-3)


def test_oracle_vs_golden_reference_vectors(oracle):
    """Golden per-sample radiance of the reference's own kernels (Cornell box 32x32, 4 spp)."""
    data = np.load(os.path.join(GOLDEN, "cornell_32x32_4spp.npz"))
    sd = scenes.cornell_box(seed=int(data["seed"]), width=32, height=32, spp=4)
    _, osamp = oracle.OracleScene(sd, use_bvh=False).render(sd.settings)
    _compare_to_reference(osamp, data["samples"])
    # Sobol values and camera rays of the reference kernels are reproduced exactly
    o = oracle.oracle()
    for idx, dim, val in data["sobol"]:
        assert np.float32(o.or_sobol_sample(int(idx), int(dim))) == np.float32(val)


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "_ref", "librefcpu.so")),
                    reason="reference harness not built (needs the reference sources)")
def test_oracle_vs_reference_harness(oracle):
    sd = scenes.cornell_box(seed=5, width=48, height=40, spp=8)
    _, osamp = oracle.OracleScene(sd, use_bvh=True).render(sd.settings)
    _, rsamp = oracle.RefScene(sd, use_bvh=True).render(threads=1)
    _compare_to_reference(osamp, rsamp)
    rs = oracle.RefScene(sd)
    r = rs.camera_ray(0.3, 0.7, 0.25, 0.5)
    cr = capi.Ray()
    oracle.oracle().or_camera_ray(C.byref(sd.settings.camera), 0.3, 0.7, 0.25, 0.5, C.byref(cr))
    # identical up to the lens-disk cos/sin, which the pinhole aperture scales to nothing
    assert np.array_equal(r, np.array(list(cr.org) + list(cr.dir), dtype=np.float32))


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "_ref", "librefcpu.so")),
                    reason="reference harness not built (needs the reference sources)")
def test_oracle_vs_reference_materials(oracle):
    """Plastic (GGX + dielectric Fresnel), rough and smooth glass, mirror, substrate, Oren-Nayar."""
    sd = scenes.cornell_box(seed=6, width=24, height=24, spp=8)
    sd.materials = [scenes.material("Plastic", (0.4, 0.4, 0.4), (0.5, 0.5, 0.5), (0.3, 0)),
                    scenes.material("Matte", (0.65, 0.05, 0.05), roughness=(0.4, 0)),
                    scenes.material("Substrate", (0.12, 0.45, 0.15), (0.2, 0.2, 0.2), (0.2, 0.3)),
                    scenes.material("Glass", (1, 1, 1), (1, 1, 1), (0, 0)),
                    scenes.material("Glass", (1, 1, 1), (1, 1, 1), (0.2, 0.2)),
                    scenes.material("Mirror", (0.9, 0.9, 0.9))]
    sd.meshes[5].material = 3
    sd.meshes[6].material = 4
    sd.meshes[2].material = 5
    _, osamp = oracle.OracleScene(sd, use_bvh=False).render(sd.settings)
    _, rsamp = oracle.RefScene(sd, use_bvh=False).render(threads=1)
    _compare_to_reference(osamp, rsamp)


def test_owen_scrambling_keeps_stratification(oracle):
    """Owen-scrambled dimensions (extension: the reference's Scramble is notImplemented) stay stratified:
    the first 2^m indices of every dimension fall one per interval of width 2^-m, as unscrambled Sobol
    points do; the values differ from the unscrambled ones, and seeds give different scrambles."""
    lib = oracle.oracle()
    m = 10
    for dim in (2, 3, 5, 11, 100, 1023):
        for seed in (0, 7):
            v = np.array([lib.or_sobol_sample_scrambled(i, dim, 1, seed) for i in range(1 << m)])
            cells = np.floor(v * (1 << m)).astype(int)
            assert np.array_equal(np.sort(cells), np.arange(1 << m)), (dim, seed)
            plain = np.array([lib.or_sobol_sample(i, dim) for i in range(1 << m)])
            assert np.mean(v != plain) > 0.9
        a = np.array([lib.or_sobol_sample_scrambled(i, dim, 1, 1) for i in range(64)])
        b = np.array([lib.or_sobol_sample_scrambled(i, dim, 1, 2) for i in range(64)])
        assert np.mean(a != b) > 0.9
    # scramble = 0 is the unscrambled sampler
    assert all(lib.or_sobol_sample_scrambled(i, 9, 0, 5) == lib.or_sobol_sample(i, 9) for i in range(200))


def test_pixel_render_equals_film_resolve(oracle):
    """or_render_pixels gathers, per pixel, exactly the samples whose 2x2 splat reaches it: its resolved
    values equal the resolved film of or_render over the same samples (border and interior pixels)."""
    sd = scenes.cornell_box(seed=0, width=32, height=32, spp=4)
    o = oracle.OracleScene(sd, use_bvh=False)
    film, _ = o.render(sd.settings, samples=False)
    pix = np.array([(0, 0), (31, 31), (0, 17), (13, 0), (5, 9), (16, 16), (30, 2), (21, 27)], dtype=np.uint32)
    got = o.render_pixels(pix, 0, 4)
    want = film[pix[:, 1], pix[:, 0], :3] / film[pix[:, 1], pix[:, 0], 3:4]
    np.testing.assert_allclose(got, want, rtol=2e-6, atol=1e-7)


def test_fp64_truth_is_the_same_estimator(oracle):
    """The double-precision build follows the same sample points and branches: per pixel over the same
    samples it agrees with the single-precision oracle to float rounding (rare paths may take another
    branch at a rounding boundary, so the bound is on the median and the mean)."""
    sd = scenes.guiding_room(seed=0, width=64, height=36, spp=4, tess=3)
    rng = np.random.default_rng(5)
    pix = np.stack([rng.integers(0, 64, 96), rng.integers(0, 36, 96)], 1).astype(np.uint32)
    a = oracle.OracleScene(sd).render_pixels(pix, 0, 16)
    b = oracle.TruthScene(sd).render_pixels(pix, 0, 16)
    rel = np.abs(a - b) / (np.abs(b) + 1e-4)
    assert np.median(rel) < 1e-5, np.median(rel)
    assert np.mean(rel) < 1e-3, np.mean(rel)


@pytest.mark.parametrize("name", ["cornell_256x256", "guiding_room_640x360", "guiding_room_1280x720",
                                  "mixed_materials_1920x1080"])
def test_truth_sets_consistent(oracle, name):
    """Each committed ground-truth set (double precision, 4096 spp over a pixel sample) names its sample
    range, holds distinct in-film pixels, and agrees with a fresh 16-spp single-precision render of
    disjoint samples at those pixels in the mean (within five standard errors of the difference)."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("make_truth", os.path.join(GOLDEN, "make_truth.py"))
    mt = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mt)
    pixels, ref = mt.load(name)
    with np.load(mt.path(name)) as z:
        assert int(z["spp"]) == 4096 and int(z["sample_begin"]) == 4096
    sd = mt.SETS[name][0]()
    st = sd.settings
    assert len(np.unique(pixels[:, 1] * st.width + pixels[:, 0])) == len(pixels)
    assert pixels[:, 0].max() < st.width and pixels[:, 1].max() < st.height
    sub = pixels[:: max(1, len(pixels) // 256)]
    refs = ref[:: max(1, len(pixels) // 256)]
    o = oracle.OracleScene(sd)
    est = o.render_pixels(sub, 0, 16)
    d = (est - refs).mean(axis=1)
    se = d.std(ddof=1) / math.sqrt(len(d))
    assert abs(d.mean()) < 5 * se + 1e-6, (d.mean(), se)
