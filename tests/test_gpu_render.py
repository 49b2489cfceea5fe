"""Render-path parity on the GPU against the CPU oracle: Sobol samples and camera rays bit-exact,
per-sample path radiance bit-exact (same Sobol dimensions, same arithmetic order, same traversal),
and the film within accumulation rounding (the film sums use atomics in any order, as the
reference's CAS loop does: tolerance 1e-5 relative + 1e-6 absolute per channel)."""
import numpy as np
import pytest

from piper2_b200 import scenes

pytestmark = pytest.mark.gpu


def _api():
    from piper2_b200 import api

    return api


def test_sobol_generate_bitexact(oracle):
    rng = np.random.default_rng(0)
    idx = rng.integers(0, 1 << 40, size=20000, dtype=np.uint64)
    idx[:5] = [0, 1, 2, (1 << 40) - 1, 12345]
    dim = rng.integers(0, 1024, size=20000, dtype=np.uint32)
    got = _api().sobol_generate(idx, dim)
    exp = np.array([oracle.oracle().or_sobol_sample(int(i), int(d)) for i, d in zip(idx, dim)], dtype=np.float32)
    assert np.array_equal(got.view(np.uint32), exp.view(np.uint32))


def test_sobol_start_bitexact(oracle):
    import ctypes as C

    rng = np.random.default_rng(1)
    for log2res in (1, 8, 11):
        n = 4000
        ps = np.stack([rng.integers(0, 1 << log2res, n), rng.integers(0, 1 << log2res, n), rng.integers(0, 256, n)],
                      axis=1).astype(np.uint32)
        idx, off = _api().sobol_start(log2res, ps)
        for k in range(0, n, 97):
            oi = C.c_uint64()
            oo = (C.c_float * 2)()
            oracle.oracle().or_sobol_start(1 << log2res, log2res, int(ps[k, 0]), int(ps[k, 1]), int(ps[k, 2]),
                                           C.byref(oi), oo)
            assert int(idx[k]) == oi.value
            assert np.float32(oo[0]) == off[k, 0] and np.float32(oo[1]) == off[k, 1]


def test_camera_rays_bitexact(oracle):
    import ctypes as C

    from piper2_b200 import capi

    sd = scenes.cornell_box(seed=0, width=48, height=32)
    st = sd.settings
    with _api().Pipeline(sd) as pl:
        rays, pts = pl.camera_rays(sample=3)
        rect = pl.rect
        ndc = pl.ndc
    for k in range(0, rect.width * rect.height, 7):
        px, py = pts[k]
        nx = np.float32(ndc.ox) + np.float32(ndc.sx) * np.float32(px) / np.float32(st.width)
        ny = np.float32(ndc.oy) + np.float32(ndc.sy) * np.float32(py) / np.float32(st.height)
        # u1/u2 = Sobol dims 3/4 of this pixel's sample index
        col, row = k % rect.width, k // rect.width
        oi = C.c_uint64()
        oo = (C.c_float * 2)()
        full = oracle.full_rect(st)
        log2res = int(np.ceil(np.log2(max(full.width, full.height))))
        oracle.oracle().or_sobol_start(1 << log2res, log2res, col, row, 3, C.byref(oi), oo)
        u1 = oracle.oracle().or_sobol_sample(oi.value, 3)
        u2 = oracle.oracle().or_sobol_sample(oi.value, 4)
        r = capi.Ray()
        oracle.oracle().or_camera_ray(C.byref(st.camera), float(nx), float(ny), u1, u2, C.byref(r))
        exp = np.array(list(r.org) + [r.tmin] + list(r.dir) + [r.tmax], dtype=np.float32)
        assert np.array_equal(rays[k].view(np.uint32), exp.view(np.uint32)), k


@pytest.mark.parametrize("size,spp", [(16, 1), (40, 4)])
def test_cornell_samples_bitexact(oracle, size, spp):
    sd = scenes.cornell_box(seed=1, width=size, height=size, spp=spp)
    with _api().Pipeline(sd) as pl:
        film, samples = pl.render(samples=True)
    ofilm, osamples = oracle.OracleScene(sd, use_bvh=False).render(sd.settings)
    diff = np.any(samples.view(np.uint32) != osamples.view(np.uint32), axis=-1)
    assert not diff.any(), f"{diff.sum()} of {diff.size} samples differ"
    np.testing.assert_allclose(film, ofilm, rtol=1e-5, atol=1e-6)


def test_cornell_full_config(oracle):
    """The full Cornell-box configuration: 256 x 256, 16 spp, max depth 8, NEE + MIS."""
    sd = scenes.cornell_box(seed=0)
    with _api().Pipeline(sd) as pl:
        film, samples = pl.render(samples=True)
        st = pl.stats()
    ofilm, osamples = oracle.OracleScene(sd, use_bvh=True).render(sd.settings)
    diff = np.any(samples.view(np.uint32) != osamples.view(np.uint32), axis=-1)
    assert not diff.any(), f"{diff.sum()} of {diff.size} samples differ"
    np.testing.assert_allclose(film, ofilm, rtol=1e-5, atol=1e-6)
    assert st.paths == 256 * 256 * 16 and st.closest_rays >= st.paths


@pytest.mark.parametrize("sample_begin", [0, 5])
def test_two_material_room_samples_bitexact(oracle, sample_begin):
    """Matte walls and a GGX-conductor floor in one closed room (paths run to the depth limit, light-plane
    pass-through): lanes of one warp append to different material queues; every sample bit-exact,
    including a sample range that does not start at 0."""
    import torch

    sd = scenes.guiding_room(seed=0, width=64, height=36, spp=4, max_depth=16)
    with _api().Pipeline(sd) as pl:
        film = pl.new_film()
        out = torch.zeros((36, 64, 3, 5), dtype=torch.float32, device="cuda")
        pl.launch(film, sample_begin=sample_begin, sample_count=3, sample_out=out)
        torch.cuda.synchronize()
        film, samples = film.cpu().numpy(), out.cpu().numpy()
    ofilm, osamples = oracle.OracleScene(sd, use_bvh=True).render(sd.settings, sample_begin=sample_begin,
                                                                  sample_count=3)
    diff = np.any(samples.view(np.uint32) != osamples.view(np.uint32), axis=-1)
    assert not diff.any(), f"{diff.sum()} of {diff.size} samples differ"
    np.testing.assert_allclose(film, ofilm, rtol=1e-5, atol=1e-6)


def test_mixed_materials_crops_bitexact(oracle):
    """The mixed-materials configuration (3.1M triangles: fBm terrain + 200 icospheres of Lambert, smooth
    dielectric and GGX-conductor materials, environment 0.5 + sun plane, depth 16): two crops of the
    1920 x 1080 frame, every sample bit-exact, including a sample range that does not start at 0."""
    import torch

    from piper2_b200 import capi

    sd = scenes.mixed_materials(seed=0)
    osc = oracle.OracleScene(sd, use_bvh=True)
    with _api().Pipeline(sd) as pl:
        for rect, begin, count in ((capi.Rect(900, 500, 48, 32), 0, 4), (capi.Rect(200, 80, 32, 32), 7, 3)):
            film = pl.new_film()
            out = torch.zeros((rect.height, rect.width, count, 5), dtype=torch.float32, device="cuda")
            pl.launch(film, rect, sample_begin=begin, sample_count=count, sample_out=out)
            torch.cuda.synchronize()
            samples = out.cpu().numpy()
            _, osamples = osc.render(sd.settings, rect=rect, sample_begin=begin, sample_count=count)
            diff = np.any(samples.view(np.uint32) != osamples.view(np.uint32), axis=-1)
            assert not diff.any(), f"{diff.sum()} of {diff.size} samples differ"


def test_owen_scrambled_render_bitexact_and_unbiased(oracle):
    """Owen-scrambled sampling (extension; the reference's Scramble is notImplemented): every sample equals
    the oracle's, and the image mean agrees with the unscrambled render within 4 standard errors."""
    sd = scenes.cornell_box(seed=1, width=48, height=48, spp=8)
    sd.settings.scramble, sd.settings.scramble_seed = 1, 12345
    with _api().Pipeline(sd) as pl:
        film, samples = pl.render(samples=True)
    _, osamples = oracle.OracleScene(sd, use_bvh=False).render(sd.settings)
    diff = np.any(samples.view(np.uint32) != osamples.view(np.uint32), axis=-1)
    assert not diff.any(), f"{diff.sum()} of {diff.size} samples differ"
    big = scenes.cornell_box(seed=1, width=128, height=128, spp=16)
    with _api().Pipeline(big) as pl:
        _, s0 = pl.render(samples=True)
    big.settings.scramble, big.settings.scramble_seed = 1, 99
    with _api().Pipeline(big) as pl:
        _, s1 = pl.render(samples=True)
    r0 = s0[..., 2:5].reshape(-1, 3).astype(np.float64)
    r1 = s1[..., 2:5].reshape(-1, 3).astype(np.float64)
    se = np.sqrt(r0.var(axis=0) / len(r0) + r1.var(axis=0) / len(r1))
    assert np.all(np.abs(r0.mean(axis=0) - r1.mean(axis=0)) <= 4 * se)
    assert not np.array_equal(r0, r1)


def test_tiled_launches_sum_to_full(oracle):
    """Launching 8 x 8 tiles (the reference's FixedSampler launch shape) gives the same film."""
    import torch

    from piper2_b200 import capi

    sd = scenes.cornell_box(seed=2, width=24, height=16, spp=2)
    with _api().Pipeline(sd) as pl:
        film = pl.new_film()
        for ty in range(0, 16, 8):
            for tx in range(0, 24, 8):
                r = capi.Rect(tx, ty, 8, 8)
                pl.launch(film, r)
        torch.cuda.synchronize()
        tiled = film.cpu().numpy()
        full, _ = pl.render()
    np.testing.assert_allclose(tiled, full, rtol=1e-5, atol=1e-6)


def test_invalid_settings_rejected():
    from piper2_b200 import capi

    sd = scenes.cornell_box(seed=0, width=8, height=8)
    st = sd.settings
    st.scramble = 2
    with pytest.raises(capi.PB2Error, match="scramble"):
        _api().Pipeline(sd, st)
    st.scramble = 0
    st.max_depth = 200
    with pytest.raises(capi.PB2Error):
        _api().Pipeline(sd, st)


def test_cornell_converges_to_fp64_truth():
    """The GPU estimator converges to the independent double-precision CPU render (4096 spp of disjoint
    samples, tests/golden/truth_cornell_256x256.npz): at the truth's pixels the relMSE falls with the
    sample count as Monte-Carlo error should (about 1/spp: 16 -> 256 spp must gain at least 8x), and the
    256-spp mean agrees with the truth's mean within 1 %."""
    import os

    with np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                              "truth_cornell_256x256.npz")) as z:
        px, ref = z["pixels"].astype(np.int64), z["rgb"]
    sd = scenes.cornell_box(seed=0)
    errs, means = {}, {}
    with _api().Pipeline(sd) as pl:
        for spp in (16, 256):
            film = pl.new_film()
            for b in range(0, spp, 16):
                pl.launch(film, sample_begin=b, sample_count=16)
            img = pl.resolve(film).cpu().numpy().astype(np.float64)[px[:, 1], px[:, 0]]
            errs[spp] = float(np.mean((img - ref) ** 2 / (ref ** 2 + 1e-2)))
            means[spp] = float(img.mean())
    assert errs[256] * 8 < errs[16], errs
    assert abs(means[256] / ref.mean() - 1) < 0.01, (means, ref.mean())


def test_several_lights_and_environment_bitexact(oracle):
    """Three area lights (one of two planes) and a non-zero environment: every branch of the MIS query
    (the selected light's plane, another light's plane, an occluder, an escape to the environment) is
    taken, and every sample stays bit-exact with the oracle."""
    from piper2_b200 import scenes as sc

    sd = sc.cornell_box(seed=1, width=48, height=48, spp=4)
    sd.planes = list(sd.planes) + [sc.plane_make((0.05, 0.999, 0.70), (0.15, 0.0, 0.0), (0.0, 0.0, 0.15)),
                                   sc.plane_make((0.80, 0.999, 0.05), (0.12, 0.0, 0.0), (0.0, 0.0, 0.12)),
                                   sc.plane_make((0.80, 0.999, 0.80), (0.10, 0.0, 0.0), (0.0, 0.0, 0.10))]
    sd.area_lights = list(sd.area_lights) + [((3.0, 5.0, 8.0), 1, 1, (0.0, 0.0, 0.0)),
                                             ((6.0, 6.0, 2.0), 2, 2, (0.0, 0.0, 0.0))]
    sd.env_radiance = (0.3, 0.4, 0.5)
    with _api().Pipeline(sd) as pl:
        film, samples = pl.render(samples=True)
    ofilm, osamples = oracle.OracleScene(sd, use_bvh=False).render(sd.settings)
    diff = np.any(samples.view(np.uint32) != osamples.view(np.uint32), axis=-1)
    assert not diff.any(), f"{diff.sum()} of {diff.size} samples differ"
    np.testing.assert_allclose(film, ofilm, rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("slots", [256, 1000])
def test_launch_with_slot_refill_bitexact(oracle, slots):
    """A launch with more paths than the pipeline's slot bound refills freed slots with its remaining paths:
    every sample (written at its launch-relative place) and the film are those of the oracle, for a sub-rect
    and a sample range that does not start at 0."""
    import torch

    from piper2_b200 import capi

    sd = scenes.cornell_box(seed=2, width=40, height=24, spp=8)
    rect = capi.Rect(4, 2, 30, 20)
    with _api().Pipeline(sd) as pl:
        pl.set_path_slots(slots)
        film = pl.new_film()
        out = torch.zeros((rect.height, rect.width, 5, 5), dtype=torch.float32, device="cuda")
        pl.launch(film, rect, sample_begin=3, sample_count=5, sample_out=out)
        torch.cuda.synchronize()
        film, samples = film.cpu().numpy(), out.cpu().numpy()
        st = pl.stats()
    ofilm, osamples = oracle.OracleScene(sd, use_bvh=False).render(sd.settings, rect=rect, sample_begin=3,
                                                                   sample_count=5)
    diff = np.any(samples.view(np.uint32) != osamples.view(np.uint32), axis=-1)
    assert not diff.any(), f"{diff.sum()} of {diff.size} samples differ"
    np.testing.assert_allclose(film, ofilm, rtol=1e-5, atol=1e-6)
    assert st.paths == rect.width * rect.height * 5


def test_path_slots_rejects_out_of_range():
    from piper2_b200 import capi

    sd = scenes.cornell_box(seed=0, width=8, height=8)
    with _api().Pipeline(sd) as pl:
        with pytest.raises(capi.PB2Error, match="path slots"):
            pl.set_path_slots(100)


def test_counting_build_counts_and_keeps_results(oracle):
    """The counting build of the render's traversal queries gives the same samples, and counts the rays the
    launch statistics count (closest: extend + MIS; shadow)."""
    sd = scenes.cornell_box(seed=3, width=32, height=32, spp=4)
    with _api().Pipeline(sd) as pl:
        _, s0 = pl.render(samples=True)
        st0 = pl.stats()
        pl.set_counting(True)
        _, s1 = pl.render(samples=True)
        c = pl.trace_counters()
        st1 = pl.stats()
        pl.set_counting(False)
    assert np.array_equal(s0.view(np.uint32), s1.view(np.uint32))
    assert c["extend"][0] + c["mis"][0] == st1.closest_rays - st0.closest_rays
    assert c["shadow"][0] == st1.shadow_rays - st0.shadow_rays
    for k, (rays, visits, tests) in c.items():
        assert rays > 0 and visits >= rays * 0.5 and tests > 0, (k, rays, visits, tests)


def test_two_devices_in_one_process(oracle):
    """Kernel attributes and launch grids are cached per device: a process that switches devices with
    pb2_set_device renders on both, each bit-exact with the oracle (needs two GPUs; skipped otherwise)."""
    import torch

    from piper2_b200 import capi

    if torch.cuda.device_count() < 2:
        pytest.skip("one GPU")
    sd = scenes.cornell_box(seed=1, width=24, height=24, spp=2)
    _, osamples = oracle.OracleScene(sd, use_bvh=False).render(sd.settings)
    for dev in (0, 1, 0):
        torch.cuda.set_device(dev)
        capi.check(capi.lib().pb2_set_device(dev))
        with _api().Pipeline(sd) as pl:
            _, samples = pl.render(samples=True)
        assert np.array_equal(samples.view(np.uint32), osamples.view(np.uint32)), dev
    torch.cuda.set_device(0)
    capi.check(capi.lib().pb2_set_device(0))


def test_bounce_graphs_equal_plain_launches(oracle):
    """The bounce loop replayed as CUDA graphs (the default: every four bounces after the first four) gives the
    samples of plain launches bit for bit, over launches in a row on one pipeline whose parameters change (a
    sub-rect, another sample range, a slot bound that makes the launch refill), so the graphs are updated in
    place from one launch to the next; the first launch is also checked against the oracle."""
    import torch

    from piper2_b200 import capi

    sd = scenes.cornell_box(seed=4, width=48, height=32, spp=8)
    full = capi.Rect(0, 0, 48, 32)
    sub = capi.Rect(5, 3, 30, 20)
    cases = [(full, 0, 8, None), (sub, 3, 5, 300), (full, 2, 6, 1 << 24), (full, 0, 8, None)]

    def run(pl, graphs):
        pl.set_graphs(graphs)
        outs = []
        for rect, begin, count, slots in cases:
            if slots is not None:
                pl.set_path_slots(slots)
            film = pl.new_film()
            out = torch.zeros((rect.height, rect.width, count, 5), dtype=torch.float32, device="cuda")
            pl.launch(film, rect, sample_begin=begin, sample_count=count, sample_out=out)
            torch.cuda.synchronize()
            outs.append(out.cpu().numpy())
        return outs

    with _api().Pipeline(sd) as pl:
        plain = run(pl, False)
        graphed = run(pl, True)
        graphed_again = run(pl, True)
    for k, (a, b, c) in enumerate(zip(plain, graphed, graphed_again)):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), f"launch {k}: graphs differ from plain launches"
        assert np.array_equal(a.view(np.uint32), c.view(np.uint32)), f"launch {k}: updated graphs differ"
    _, osamples = oracle.OracleScene(sd, use_bvh=False).render(sd.settings)
    assert np.array_equal(graphed[0].view(np.uint32), osamples.view(np.uint32))


def test_refill_over_many_bitmap_blocks_bitexact():
    """A refilled launch whose free-slot bitmap spans several 1024-word scan blocks (2^21 slots: 64 blocks) gives
    the samples of the same launch with every path in its own slot, bit for bit."""
    import torch

    sd = scenes.cornell_box(seed=6, width=256, height=256, spp=48)  # 3.1M paths
    outs = []
    with _api().Pipeline(sd) as pl:
        for slots in (1 << 21, 1 << 22):
            pl.set_path_slots(slots)
            film = pl.new_film()
            out = torch.zeros((256, 256, 48, 5), dtype=torch.float32, device="cuda")
            pl.launch(film, pl.rect, 0, 48, sample_out=out)
            torch.cuda.synchronize()
            outs.append(out.cpu().numpy())
            del out
    assert np.array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32))
    assert np.all(outs[0][..., 4] >= 0.0) and np.count_nonzero(outs[0][..., 0]) > 0
