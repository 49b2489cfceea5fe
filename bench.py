"""Benchmark of the traversal stress test (1M triangles; 4M closest-hit + 4M any-hit rays).

A step is one pass of the hot path over one batch: a closest-hit trace of 4M rays and an any-hit trace of
4M shadow rays against the 8-wide BVH of a 1M-triangle soup (centroids U[0,1]^3, lognormal edges with
median 0.01 and sigma 0.5; closest-hit rays from the bounding sphere to uniform interior points;
any-hit rays of length U[0.1, 1]).  Synthetic, seeded data of the configuration's shapes.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value   : Mrays/s over both ray sets, inputs resident in HBM, device time (CUDA events) of the K steps,
          L2 flushed (256 MiB write) before every step; for N > 1 every rank traces its own batch
          (weak scaling) and the time is the max over ranks.
e2e     : the same through the host-buffer C-ABI calls (pinned host rays in, hits out, copies timed).
roofline: the closest-hit kernel's algorithmic bytes per launch (32 B ray + 16 B hit + 80 B per node
          visit + 36 B per triangle test, visits and tests counted by the counting build of the same
          traversal on the same BVH) / its CUDA-event duration, against the measured HBM copy peak.
--impl reference: the CPU port of the path (binned-SAH BVH + the same watertight test; Embree itself is
          not available here) on all host cores, on a bounded sample of the same ray sets.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

N_TRIS = 1 << 20
N_RAYS = 1 << 22
METRIC = "Mrays/s (closest-hit + any-hit) on the traversal stress test; reference: CPU tracer on host cores"
CONFIG = {"workload": "traversal stress test: 1M-triangle soup, 4M closest-hit + 4M any-hit rays",
          "triangles": N_TRIS, "closest_rays": N_RAYS, "anyhit_rays": N_RAYS, "seed": 0,
          "l2": "flushed (256 MiB write) before every step"}
BYTES_RAY, BYTES_HIT, BYTES_NODE, BYTES_TRI = 32, 16, 80, 36


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _bf16_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"]), "measured"
    except Exception:
        return 1590.0, "fallback"


def mlp_bench():
    """The guiding network's kernels against the tensor-pipe peak: one Adam step on 2^16 records (forward +
    backward + update; 3 x 43,008 FLOP per record by the dense-layer count) and one forward pass over 2^20
    vertices (43,008 FLOP each: 2 (96x64 + 3 x 64x64 + 64x48))."""
    import numpy as np
    import torch

    from piper2_b200 import api

    g = api.Guide(seed=0)
    rng = np.random.default_rng(0)
    b = 1 << 16
    rec = np.zeros((b, 16), np.float32)
    rec[:, 0:3] = rng.uniform(0, 1, (b, 3))
    for k in (3, 6, 9):
        v = rng.normal(size=(b, 3))
        rec[:, k:k + 3] = v / np.linalg.norm(v, axis=1, keepdims=True)
    rec[:, 12] = rng.exponential(1.0, b)
    drec = torch.from_numpy(rec).cuda()
    n = 1 << 20
    feat = torch.from_numpy(np.concatenate([rec] * 16)[:, :12].copy()).cuda()
    out = torch.empty((n, 48), device="cuda")
    import ctypes as C

    from piper2_b200 import capi

    lib = capi.lib()
    sp = C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def train():
        capi.check(lib.pb2_guide_train(g.h, C.c_void_p(drec.data_ptr()), b, C.c_float(1e-3), None, sp))

    status = torch.zeros(1, dtype=torch.int32, device="cuda")

    def fwd():  # the kernel alone: the time-out flag goes to a device word, read once after the timing
        capi.check(lib.pb2_guide_forward_async(g.h, C.c_void_p(feat.data_ptr()), n, C.c_void_p(out.data_ptr()),
                                               C.c_void_p(status.data_ptr()), sp))

    def fwd_sync():
        capi.check(lib.pb2_guide_forward(g.h, C.c_void_p(feat.data_ptr()), n, C.c_void_p(out.data_ptr()), sp))

    def fwd_mma():
        capi.check(lib.pb2_guide_forward_mma(g.h, C.c_void_p(feat.data_ptr()), n, C.c_void_p(out.data_ptr()), sp))

    res = {}
    peak, kind = _bf16_peak()
    for name, fn, flops in (("train_step_2^16", train, 3 * 43008 * b), ("forward_tcgen05_2^20", fwd, 43008 * n),
                            ("forward_tcgen05_2^20_synchronising_call", fwd_sync, 43008 * n),
                            ("forward_mma_sync_2^20", fwd_mma, 43008 * n)):
        for _ in range(3):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(20):
            fn()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 20
        tf = flops / (ms * 1e-3) / 1e12
        res[name] = {"ms": round(ms, 4), "tflops": round(tf, 2), "frac": round(tf / peak, 4)}
    if int(status.item()) != 0:
        raise RuntimeError("guide forward: a tensor-core wait timed out")
    res["peak_tflops"] = peak
    res["peak_source"] = kind
    res["note"] = ("forward_tcgen05: tcgen05.mma kind::f16, seven 128-row warp groups per CTA, TMEM accumulators, "
                   "timed through pb2_guide_forward_async (kernel launches back to back); the synchronising call "
                   "pb2_guide_forward adds a flag clear, a flag read and a stream synchronisation per call; training: one fused tcgen05 kernel per batch "
                   "(forward, loss gradient, backward-data and the weight gradients accumulated in TMEM) plus the "
                   "reduction over CTAs and Adam; forward_mma_sync: the mma.sync m16n8k16 cross-check; the "
                   "network is 64 wide")
    return res


def truth_rel_mse(img, name):
    """relMSE of a resolved image (H, W, 3) against a committed ground-truth pixel set
    (tests/golden/truth_<name>.npz: the double-precision CPU render at 4096 spp of a seeded pixel sample,
    made by tests/golden/make_truth.py): mean over those pixels and channels of (I - R)^2 / (R^2 + 0.01).
    None if the set is absent."""
    import numpy as np

    path = os.path.join(ROOT, "tests", "golden", f"truth_{name}.npz")
    if not os.path.exists(path):
        return None
    with np.load(path) as z:
        px, ref = z["pixels"].astype(np.int64), z["rgb"]
    val = np.asarray(img, dtype=np.float64)[px[:, 1], px[:, 0], :3]
    return float(np.mean((val - ref) ** 2 / (ref ** 2 + 1e-2)))


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 7:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_ours(args):
    import ctypes as C

    import numpy as np
    import torch

    from piper2_b200 import api, capi, scenes

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    soup = scenes.triangle_soup(N_TRIS, seed=0)
    crays = scenes.soup_rays(N_RAYS, seed=1 + 2 * rank, kind="closest")
    arays = scenes.soup_rays(N_RAYS, seed=2 + 2 * rank, kind="any")
    acc = api.Accel(soup)
    info = acc.info()
    stream = torch.cuda.current_stream()
    d_c = torch.from_numpy(crays.view(np.float32).reshape(-1, 8)).to(dev)
    d_a = torch.from_numpy(arays.view(np.float32).reshape(-1, 8)).to(dev)
    d_hits = torch.empty((N_RAYS, 4), dtype=torch.float32, device=dev)
    d_occ = torch.empty(N_RAYS, dtype=torch.int32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    # work counters of this traversal on this BVH (for the byte model), outside the timed region
    acc.set_counting(True)
    acc.trace_closest_dev(d_c.data_ptr(), N_RAYS, d_hits.data_ptr())
    nv_c, nt_c = acc.counters()
    acc.trace_any_dev(d_a.data_ptr(), N_RAYS, d_occ.data_ptr())
    nv_a, nt_a = acc.counters()
    acc.set_counting(False)

    def step(ev):
        flush.zero_()
        ev[0].record(stream)
        acc.trace_closest_dev(d_c.data_ptr(), N_RAYS, d_hits.data_ptr())
        ev[1].record(stream)
        acc.trace_any_dev(d_a.data_ptr(), N_RAYS, d_occ.data_ptr())
        ev[2].record(stream)

    mk = lambda: [torch.cuda.Event(enable_timing=True) for _ in range(3)]  # noqa: E731
    for _ in range(args.warmup):
        step(mk())
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    torch.cuda.synchronize()
    evs = [mk() for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        for e in evs:
            step(e)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t_closest = [e[0].elapsed_time(e[1]) for e in evs]
    t_any = [e[1].elapsed_time(e[2]) for e in evs]
    step_ms = [a + b for a, b in zip(t_closest, t_any)]
    total_ms = sum(step_ms)

    # end to end: host buffers through the C ABI (copies in the timed region)
    h_c = torch.from_numpy(crays.view(np.uint8)).pin_memory()
    h_a = torch.from_numpy(arays.view(np.uint8)).pin_memory()
    h_hits = torch.empty(N_RAYS * 16, dtype=torch.uint8).pin_memory()
    h_occ = torch.empty(N_RAYS * 4, dtype=torch.uint8).pin_memory()
    lib = capi.lib()
    sp = C.c_void_p(stream.cuda_stream)

    def e2e_step():
        capi.check(lib.pb2_trace_closest_host(acc.h, C.c_void_p(h_c.data_ptr()), N_RAYS, C.c_void_p(h_hits.data_ptr()), sp))
        capi.check(lib.pb2_trace_any_host(acc.h, C.c_void_p(h_a.data_ptr()), N_RAYS, C.c_void_p(h_occ.data_ptr()), sp))

    for _ in range(max(1, args.warmup)):
        e2e_step()
    torch.cuda.synchronize()
    e2e_ms = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_step()
        e2e_ms.append((time.perf_counter() - t0) * 1e3)

    res = torch.tensor([total_ms, sum(e2e_ms), sum(t_closest)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(res, op=dist.ReduceOp.MAX)
        dist.destroy_process_group()
    total_ms, e2e_total, closest_total = res.tolist()
    if rank != 0:
        return
    rays_all = 2 * N_RAYS * args.steps * world
    value = rays_all / (total_ms * 1e-3) / 1e6
    e2e_value = rays_all / (e2e_total * 1e-3) / 1e6
    # roofline of the closest-hit kernel
    bytes_per_launch = N_RAYS * (BYTES_RAY + BYTES_HIT) + BYTES_NODE * nv_c + BYTES_TRI * nt_c
    avg_closest_s = (sum(t_closest) / len(t_closest)) * 1e-3
    achieved = bytes_per_launch / avg_closest_s / 1e9
    peak, peak_kind = _peaks()
    cpu = cpu_baseline(soup, crays, arays, args) if world == 1 else None
    render = render_bench(args) if world == 1 else None
    line = {
        "metric": METRIC,
        "value": round(value, 2),
        "unit": "Mrays/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(total_ms / args.steps, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded generator of the configuration's shapes)",
        "config": dict(CONFIG, parallelism=f"replicas x{world} (independent ray batches)"),
        "e2e": {"value": round(e2e_value, 2), "unit": "Mrays/s", "h2d_bytes_per_step": 2 * N_RAYS * 32,
                "d2h_bytes_per_step": N_RAYS * 16 + N_RAYS * 4},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": None,
                     "traffic_note": "DRAM bytes need an ncu capture, not taken in this run; see the committed "
                                     "ncu summary of the closest-hit kernel on this workload",
                     "peak_source": peak_kind,
                     "kernel": "k_trace_api<closest>",
                     "bytes_model": {"per_ray": BYTES_RAY + BYTES_HIT, "per_node_visit": BYTES_NODE,
                                     "per_triangle_test": BYTES_TRI,
                                     "node_visits_per_ray": round(nv_c / N_RAYS, 3),
                                     "triangle_tests_per_ray": round(nt_c / N_RAYS, 3)}},
        "cpu_baseline": cpu,
        "gpu_launches": 2 * args.steps,
        "render": render,
        "clocks": clk.summary(),
        "detail": {"closest_mrays_s": round(N_RAYS / (sum(t_closest) / args.steps * 1e-3) / 1e6, 2),
                   "anyhit_mrays_s": round(N_RAYS / (sum(t_any) / args.steps * 1e-3) / 1e6, 2),
                   "anyhit_node_visits_per_ray": round(nv_a / N_RAYS, 3),
                   "anyhit_triangle_tests_per_ray": round(nt_a / N_RAYS, 3),
                   "bvh_nodes": info.node_count, "bvh_build_ms": round(info.build_ms, 3)},
    }
    print(json.dumps(line))


def _render_rate(pl, rect, spp, chunk, frames=1):
    """Device time of `frames` full renders of `rect` at `spp`, launched `chunk` samples at a time."""
    import torch

    film = pl.new_film()
    pl.launch(film, rect, 0, min(chunk, spp))
    torch.cuda.synchronize()
    s0 = pl.stats()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(frames):
        for b in range(0, spp, chunk):
            pl.launch(film, rect, b, min(chunk, spp - b))
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    s1 = pl.stats()
    rays = (s1.closest_rays - s0.closest_rays) + (s1.shadow_rays - s0.shadow_rays)
    samples = rect.width * rect.height * spp * frames
    return {"samples_per_s": round(samples / (ms * 1e-3), 1), "mrays_per_s": round(rays / (ms * 1e-3) / 1e6, 2),
            "ms_per_frame": round(ms / frames, 3), "rays_per_sample": round(rays / samples, 3)}


def render_roofline(pl, rect, spp, chunk, ms_per_frame):
    """Byte model of the render path for one frame, by the counting build of its traversal queries (a separate
    untimed render of the same samples): per traced ray its 32-byte ray, the record it writes (closest hit
    16 B + triangle slot 4 B, MIS record 16 B, occlusion flag 4 B), 80 B per 8-wide node visited and 36 B per
    triangle tested, plus 48 B of queued path state written and read again per ray, plus 16 B x 4 film splats
    per sample; over the timed frame, against the measured HBM copy peak."""
    pl.set_counting(True)
    film = pl.new_film()
    for b in range(0, spp, chunk):
        pl.launch(film, rect, b, min(chunk, spp - b))
    c = pl.trace_counters()
    pl.set_counting(False)
    record = {"extend": 20, "mis": 16, "shadow": 4}
    traversal = sum(r * (32 + record[k]) + 80 * v + 36 * t for k, (r, v, t) in c.items())
    rays = sum(r for r, _, _ in c.values())
    samples = rect.width * rect.height * spp
    total = traversal + 96 * rays + 64 * samples
    achieved = total / (ms_per_frame * 1e-3) / 1e9
    peak, kind = _peaks()
    return {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_source": kind, "bytes_per_frame": int(total),
            "per_query": {k: {"rays": r, "node_visits_per_ray": round(v / max(r, 1), 3),
                              "triangle_tests_per_ray": round(t / max(r, 1), 3)} for k, (r, v, t) in c.items()}}


def batch_bench():
    """64 scenes of uneven size (10k-2M triangles, 128-1024 px film side, 4-64 spp) through one batched
    render: autotuned configuration, aggregate samples/s, per-scene completion percentiles; beside it the
    same scenes rendered one after another through single-scene pipelines (device time of the launches)."""
    import numpy as np
    import torch

    from piper2_b200 import api, scenes

    sds = scenes.batch_workload(seed=0)
    samples = sum(sd.settings.width * sd.settings.height * sd.settings.samples_per_pixel for sd in sds)
    with api.Batch(sds) as b:
        cfg, tune_ms = b.autotune()
        b.render()  # warm-up
        b.render()
        ms, total, iters = b.timing()
        st = b.stats()
    out = {"workload": "64 scenes: mixed-materials generator, triangles log-uniform 10k-2M, film side log-uniform "
                       "128-1024 (16:9), spp uniform 4-64 rounded up to a power of two, depth 16",
           "triangles": sum(sum(len(m.indices) for m in sd.meshes) for sd in sds), "samples": samples,
           "samples_per_s": round(samples / (total * 1e-3), 1), "ms": round(total, 2),
           "mrays_per_s": round((st.closest_rays + st.shadow_rays) / (total * 1e-3) / 1e6, 2),
           "scene_ms_p50": round(float(np.percentile(ms, 50)), 2), "scene_ms_p90": round(float(np.percentile(ms, 90)), 2),
           "scene_ms_p99": round(float(np.percentile(ms, 99)), 2), "iterations": iters,
           "config": {"capacity": cfg.capacity, "shade_block": cfg.shade_block,
                      "trace_blocks_per_sm": cfg.trace_blocks_per_sm, "graph": bool(cfg.use_graph)},
           "autotune_ms": round(tune_ms, 1)}
    seq = 0.0
    for sd in sds:
        with api.Pipeline(sd) as pl:
            spp = sd.settings.samples_per_pixel
            film = pl.new_film()
            pl.launch(film, pl.rect, 0, min(spp, 16))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            for s0 in range(0, spp, 16):
                pl.launch(film, pl.rect, s0, min(16, spp - s0))
            e1.record()
            torch.cuda.synchronize()
            seq += e0.elapsed_time(e1)
        torch.cuda.empty_cache()
    out["sequential_single_scene_ms"] = round(seq, 2)
    out["sequential_samples_per_s"] = round(samples / (seq * 1e-3), 1)
    return out


def render_bench(args):
    """The render path: the Cornell-box configuration (256 x 256, 16 spp, depth 8) against the reference's own
    kernels compiled natively (oracle/_ref) on all host cores over a bounded crop; the mixed-materials
    configuration (3.1M triangles, 1920 x 1080, 64 spp, depth 16); guided vs plain on the hard-indirect room
    at its configuration (1280 x 720, 256 spp).  Every image's relMSE is also taken against the double-precision CPU render at 4096 spp
    (a committed pixel sample, tests/golden/truth_*.npz)."""
    import torch

    import oracle_py

    from piper2_b200 import api, capi, guiding_eval, scenes

    sd = scenes.cornell_box(seed=0)
    st = sd.settings
    with api.Pipeline(sd) as pl:
        out = {"workload": "Cornell box 256x256, 16 spp, max depth 8, NEE+MIS (plain BxDF sampling)"}
        out.update(_render_rate(pl, pl.rect, st.samples_per_pixel, st.samples_per_pixel, frames=max(3, args.steps // 2)))
        out["roofline"] = render_roofline(pl, pl.rect, st.samples_per_pixel, st.samples_per_pixel, out["ms_per_frame"])
        film = pl.new_film()
        pl.launch(film, sample_begin=0, sample_count=st.samples_per_pixel)
        out["relmse_vs_fp64_4096spp"] = truth_rel_mse(pl.resolve(film).cpu().numpy(), "cornell_256x256")
    if oracle_py.ref_available():
        crop = capi.Rect(0, 96, 256, 16)
        rs = oracle_py.RefScene(sd, use_bvh=True)
        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        rs.render(rect=crop, threads=threads, samples=False)
        dt = time.perf_counter() - t0
        n = crop.width * crop.height * st.samples_per_pixel
        out["cpu_baseline"] = {"value": round(n / dt, 1), "unit": "samples/s", "cores": threads, "kind": "reference",
                               "sample": "rows 96-111 of the frame (65,536 samples) through the reference's own "
                                         "kernels compiled natively, CPU BVH in place of Embree"}
    result = {"cornell": out}
    md = scenes.mixed_materials(seed=0)
    with api.Pipeline(md) as pl:
        mm = {"workload": "mixed materials 1920x1080, 64 spp, max depth 16, 3.1M triangles (terrain + 200 "
                          "icospheres: Lambert / smooth dielectric / GGX conductor), env 0.5 + sun"}
        mm.update(_render_rate(pl, pl.rect, md.settings.samples_per_pixel, 8))
        mm["roofline"] = render_roofline(pl, pl.rect, md.settings.samples_per_pixel, 8, mm["ms_per_frame"])
        film = pl.new_film()
        for b in range(0, md.settings.samples_per_pixel, 8):
            pl.launch(film, sample_begin=b, sample_count=8)
        mm["relmse_vs_fp64_4096spp"] = truth_rel_mse(pl.resolve(film).cpu().numpy(), "mixed_materials_1920x1080")
    mm.update(mixed_materials_cpu(md))
    result["mixed_materials"] = mm
    torch.cuda.empty_cache()
    result["batch"] = batch_bench()
    torch.cuda.empty_cache()
    g = guiding_eval.evaluate(width=1280, height=720, spp=256, ref_spp=0, repeats=3,
                              truth=lambda img: truth_rel_mse(img, "guiding_room_1280x720"))
    result["guiding"] = g
    result["guiding_mlp"] = mlp_bench()
    return result


def mixed_materials_cpu(md):
    """CPU baselines of the mixed-materials configuration on a 128 x 64 crop at the frame's 64 spp (524,288
    samples), on all host threads: the reference's own kernels compiled natively (oracle/_ref; the reference
    has no conductor, so the GGX conductors become its Plastic with the conductor's F0 as specular colour,
    no diffuse, and alpha as roughness) and the oracle's port of the same estimator on the exact scene."""
    import copy

    import oracle_py

    from piper2_b200 import capi, scenes

    crop = capi.Rect(896, 480, 128, 64)
    n = crop.width * crop.height * md.settings.samples_per_pixel
    threads = os.cpu_count() or 1
    out = {}
    if oracle_py.ref_available():
        rmd = copy.copy(md)
        rmd.materials = [scenes.material("Plastic", (0, 0, 0, 1), tuple(m.color1), (m.roughness[0], 0))
                         if m.type == 6 else m for m in md.materials]
        rs = oracle_py.RefScene(rmd, use_bvh=True)
        t0 = time.perf_counter()
        rs.render(rect=crop, threads=threads, samples=False)
        dt = time.perf_counter() - t0
        rs.close()
        out["cpu_baseline"] = {"value": round(n / dt, 1), "unit": "samples/s", "cores": threads, "kind": "reference",
                               "sample": "crop x 896-1023, y 480-543 at 64 spp (524,288 samples) through the "
                                         "reference's own kernels compiled natively, CPU BVH in place of Embree; "
                                         "GGX conductors as the reference's Plastic (it has no conductor)"}
    osc = oracle_py.OracleScene(md, use_bvh=True)
    t0 = time.perf_counter()
    osc.render(md.settings, rect=crop, threads=threads, samples=False)
    dt = time.perf_counter() - t0
    osc.close()
    out["cpu_baseline_port"] = {"value": round(n / dt, 1), "unit": "samples/s", "cores": threads, "kind": "port",
                                "sample": "the same crop through the oracle's restatement of the estimator, exact "
                                          "scene"}
    return out


def cpu_baseline(soup, crays, arays, args, sample=None):
    """The CPU port (binned-SAH BVH + watertight test) on all host threads, bounded sample."""
    import oracle_py

    threads = os.cpu_count() or 1
    osc = oracle_py.OracleScene(soup, use_bvh=True)
    n = sample or int(os.environ.get("PB2_CPU_SAMPLE", 1 << 17))
    t0 = time.perf_counter()
    osc.trace_closest(crays[:n], threads=threads)
    osc.trace_any(arays[:n], threads=threads)
    dt = time.perf_counter() - t0
    osc.close()
    return {"value": round(2 * n / dt / 1e6, 3), "unit": "Mrays/s", "cores": threads, "kind": "port",
            "sample": f"{n} closest-hit + {n} any-hit rays of the same sets (1M-triangle BVH built beforehand)"}


def run_reference(args):
    world, rank, _ = _dist()
    if rank != 0:
        return
    import oracle_py  # noqa: F401

    from piper2_b200 import scenes

    soup = scenes.triangle_soup(N_TRIS, seed=0)
    crays = scenes.soup_rays(N_RAYS, seed=1, kind="closest")
    arays = scenes.soup_rays(N_RAYS, seed=2, kind="any")
    import oracle_py as op

    threads = os.cpu_count() or 1
    osc = op.OracleScene(soup, use_bvh=True)
    n = int(os.environ.get("PB2_CPU_SAMPLE", 1 << 16))
    for i in range(args.warmup):
        osc.trace_closest(crays[:n // 4], threads=threads)
    times = []
    for i in range(args.steps):
        lo = (i * n) % (N_RAYS - n)
        t0 = time.perf_counter()
        osc.trace_closest(crays[lo:lo + n], threads=threads)
        osc.trace_any(arays[lo:lo + n], threads=threads)
        times.append(time.perf_counter() - t0)
    value = 2 * n * args.steps / sum(times) / 1e6
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": round(value, 3),
        "unit": "Mrays/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(1e3 * sum(times) / args.steps, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded generator of the configuration's shapes)",
        "config": dict(CONFIG, parallelism="host threads"),
        "cpu_baseline": {"value": round(value, 3), "unit": "Mrays/s", "cores": threads, "kind": "port",
                         "sample": f"{n} closest-hit + {n} any-hit rays per step (Embree 3.12.1 is not installed; "
                                   "the reference's Embree tracer is replaced by its CPU restatement)"},
        "e2e": {"value": round(value, 3), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
