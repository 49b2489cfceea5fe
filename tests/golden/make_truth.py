"""Generates the ground-truth pixel sets of tests/golden: double-precision renders at 4096 spp.

The ground truth of every relMSE the bench reports is the oracle's double-precision build
(oracle/_build/liboracle_fp64.so: the same estimator, sample points and constants as the single-precision
oracle, every intermediate in double).  A full frame at 4096 spp is hours of CPU time for the larger
configurations, so the truth is taken on a seeded uniform sample of pixels; relMSE over those pixels is an
unbiased estimate of the full frame's.  The truth uses Sobol samples [4096, 8192), disjoint from every
sample a measured render uses (those start at 0 and stay below 4096).

    python tests/golden/make_truth.py [name ...]      (all sets by default; uses every host core)

Writes truth_<name>.npz with `pixels` (n, 2) uint16 film coordinates (x, y), `rgb` (n, 3) float64
resolved values, and the scene's description (`scene`, `spp`, `sample_begin`).
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import build_oracle  # noqa: E402
import oracle_py  # noqa: E402

from piper2_b200 import scenes  # noqa: E402

TRUTH_SPP = 4096
TRUTH_BEGIN = 4096

# name -> (scene constructor, pixel count)
SETS = {
    "cornell_256x256": (lambda: scenes.cornell_box(seed=0), 4096),
    "guiding_room_640x360": (lambda: scenes.guiding_room(seed=0, width=640, height=360, spp=64), 4096),
    "guiding_room_1280x720": (lambda: scenes.guiding_room(seed=0, width=1280, height=720, spp=256), 2048),
    "mixed_materials_1920x1080": (lambda: scenes.mixed_materials(seed=0), 1024),
}


def pixel_sample(width, height, n, seed=1234):
    """n distinct pixels drawn uniformly from the film (seeded)."""
    rng = np.random.default_rng(seed)
    flat = rng.choice(width * height, size=n, replace=False)
    return np.stack([flat % width, flat // width], axis=1).astype(np.uint16)


def path(name):
    return os.path.join(HERE, f"truth_{name}.npz")


def make(name):
    ctor, n = SETS[name]
    sd = ctor()
    st = sd.settings
    pixels = pixel_sample(st.width, st.height, n)
    t0 = time.time()
    truth = oracle_py.TruthScene(sd)
    rgb = truth.render_pixels(pixels, TRUTH_BEGIN, TRUTH_SPP)
    truth.close()
    np.savez_compressed(path(name), pixels=pixels, rgb=rgb, scene=np.array(sd.name), spp=TRUTH_SPP,
                        sample_begin=TRUTH_BEGIN)
    print(f"{name}: {n} pixels x {TRUTH_SPP} spp in {time.time() - t0:.0f} s", flush=True)


def load(name):
    """(pixels (n, 2) x/y, rgb (n, 3)) of a committed truth set."""
    with np.load(path(name)) as z:
        return z["pixels"].astype(np.int64), z["rgb"]


def rel_mse_at(img, name):
    """relMSE = mean over the truth pixels and channels of (I - R)^2 / (R^2 + 0.01); img is (H, W, 3)."""
    pixels, ref = load(name)
    val = np.asarray(img, dtype=np.float64)[pixels[:, 1], pixels[:, 0], :3]
    return float(np.mean((val - ref) ** 2 / (ref ** 2 + 1e-2)))


if __name__ == "__main__":
    build_oracle.build_oracle()
    for nm in sys.argv[1:] or list(SETS):
        make(nm)
