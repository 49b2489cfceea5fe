"""Time-to-equal-error of guided against plain path tracing on the hard-indirect room.

Both integrators render the same frame at the same sample count; the error is the relative MSE against a
plain render of many more samples taken from a disjoint Sobol range,

    relMSE = mean over pixels and channels of (I - R)^2 / (R^2 + 0.01),

and since Monte-Carlo error falls as 1 / time, the time one integrator needs to reach the other's error is
proportional to time x relMSE.  `speedup` = (T_plain relMSE_plain) / (T_guided relMSE_guided); the guided
time includes its online training.  The reference's own noise adds the same amount to both errors, so the
reported speed-up is, if anything, an underestimate.

`truth`, if given, is a second error measure: a function image (H, W, 3) -> relMSE against an independent
ground truth (the bench passes the double-precision CPU render at 4096 spp over a pixel sample); its
errors and speed-up are reported as `relmse_fp64` / `speedup_fp64`.

    python -m piper2_b200.guiding_eval [--width 640 --height 360 --spp 64 --ref-spp 1024]
"""
from __future__ import annotations

import argparse
import json

import numpy as np


def _time(torch, fn):
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    out = fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1), out


def rel_mse(img, ref):
    return float(np.mean((img - ref) ** 2 / (ref ** 2 + 1e-2)))


def evaluate(width=1280, height=720, spp=64, ref_spp=1024, spp_per_pass=8, train_steps=4, batch=1 << 16,
             learning_rate=1e-2, selection_prob=0.5, seed=0, tess=15, max_depth=16, chunk=64, train_passes=None,
             weight_quantile=0.99, spatial_cells=0, truth=None, guided_types=0,
             max_guided_depth=2, repeats=1):
    import torch

    from . import api, scenes

    sd = scenes.guiding_room(seed=seed, width=width, height=height, spp=spp, max_depth=max_depth, tess=tess)
    out = {"workload": f"guiding room {width}x{height}, {spp} spp, max depth {max_depth}",
           "reference": f"plain, {ref_spp} spp from samples [{spp}, {spp + ref_spp})" if ref_spp else None}
    with api.Pipeline(sd) as pl:
        ref = None
        if ref_spp:
            film = pl.new_film()
            for s in range(0, ref_spp, chunk):
                pl.launch(film, sample_begin=spp + s, sample_count=min(chunk, ref_spp - s))
            ref = pl.resolve(film).cpu().numpy().astype(np.float64)
        # plain: its fastest form, one launch of all samples or passes of spp_per_pass samples (timed after a
        # warm-up launch); both render the same samples
        pl.launch(pl.new_film(), sample_begin=0, sample_count=min(spp, 4))
        film = pl.new_film()
        t_one, _ = _time(torch, lambda: pl.launch(film, sample_begin=0, sample_count=spp))
        film_p = pl.new_film()
        t_passes, _ = _time(torch, lambda: [pl.launch(film_p, sample_begin=b, sample_count=min(spp_per_pass, spp - b))
                                           for b in range(0, spp, spp_per_pass)])
        t_plain = min(t_one, t_passes)
        plain = pl.resolve(film).cpu().numpy().astype(np.float64)
        # guided: a fresh network per run, progressive passes with online training.  Online training is not
        # deterministic (records are gathered with atomics), so `repeats` independent runs are made and
        # their errors and times averaged.
        runs = []
        for r in range(max(1, repeats)):
            guide = api.Guide(seed=seed + 1 + r)
            pl.set_guide(guide, selection_prob=selection_prob, record_capacity=1 << 20,
                         weight_quantile=weight_quantile, spatial_cells=spatial_cells, guided_types=guided_types,
                         max_guided_depth=max_guided_depth)
            film = pl.new_film()
            t_g, losses = _time(torch, lambda: pl.render_guided(film, spp, spp_per_pass, train_steps, batch,
                                                                learning_rate, train_passes))
            runs.append((t_g, pl.resolve(film).cpu().numpy().astype(np.float64), losses))
            pl.set_guide(None)
    t_guided = float(np.mean([r[0] for r in runs]))
    guided, losses = runs[-1][1], runs[-1][2]
    e_plain = rel_mse(plain, ref) if ref is not None else None
    e_guided = float(np.mean([rel_mse(r[1], ref) for r in runs])) if ref is not None else None
    out.update({
        "plain": {"ms": round(t_plain, 2), "ms_one_launch": round(t_one, 2), "ms_passes": round(t_passes, 2),
                  "relmse": e_plain, "mean": float(plain.mean())},
        "guided": {"ms": round(t_guided, 2), "relmse": e_guided, "mean": float(guided.mean()),
                   "guided_types": guided_types or "matte", "max_guided_depth": max_guided_depth or None,
                   "passes": spp // spp_per_pass, "train_steps_per_pass": train_steps, "batch": batch,
                   "train_passes": train_passes, "learning_rate": learning_rate, "weight_quantile": weight_quantile,
                   "spatial_cells": spatial_cells,
                   "first_loss": losses[0] if losses else None, "last_loss": losses[-1] if losses else None},
        "reference_mean": float(ref.mean()) if ref is not None else None,
        "relmse_ratio": e_plain / e_guided if e_guided else None,
        "speedup": (t_plain * e_plain) / (t_guided * e_guided) if e_guided else None,
    })
    out["guided"]["runs"] = len(runs)
    out["guided"]["ms_each"] = [round(r[0], 2) for r in runs]
    if truth is not None:
        each = [truth(r[1]) for r in runs]
        f_plain, f_guided = truth(plain), float(np.mean(each))
        out["plain"]["relmse_fp64"] = f_plain
        out["guided"]["relmse_fp64"] = f_guided
        out["guided"]["relmse_fp64_each"] = each
        out["relmse_ratio_fp64"] = f_plain / f_guided if f_guided > 0 else None
        out["speedup_fp64"] = (t_plain * f_plain) / (t_guided * f_guided) if f_guided > 0 else None
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--width", type=int, default=1280)
    ap.add_argument("--height", type=int, default=720)
    ap.add_argument("--spp", type=int, default=64)
    ap.add_argument("--ref-spp", type=int, default=1024)
    ap.add_argument("--spp-per-pass", type=int, default=8)
    ap.add_argument("--train-steps", type=int, default=4)
    ap.add_argument("--train-passes", type=int, default=None)
    ap.add_argument("--batch", type=int, default=1 << 16)
    ap.add_argument("--lr", type=float, default=1e-2)
    ap.add_argument("--selection-prob", type=float, default=0.5)
    ap.add_argument("--weight-quantile", type=float, default=0.99)
    ap.add_argument("--spatial-cells", type=int, default=0)
    ap.add_argument("--tess", type=int, default=15)
    ap.add_argument("--max-guided-depth", type=int, default=2)
    a = ap.parse_args()
    print(json.dumps(evaluate(a.width, a.height, a.spp, a.ref_spp, a.spp_per_pass, a.train_steps, a.batch, a.lr,
                              a.selection_prob, tess=a.tess, train_passes=a.train_passes,
                              weight_quantile=a.weight_quantile, spatial_cells=a.spatial_cells,
                              max_guided_depth=a.max_guided_depth)))


if __name__ == "__main__":
    main()
