"""Generates the golden vectors of tests/golden from the reference's own kernels.

Run where the reference sources are available (they are compiled natively into
oracle/_ref/librefcpu.so by oracle/build_oracle.py):

    python tests/golden/make_golden.py /path/to/Piper2     (or PIPER2_REFERENCE=/path/to/Piper2)

Writes:
  sobol_digest.txt          SHA-256 of the regenerated Sobol tables
  cornell_32x32_4spp.npz    per-sample (film point, radiance) of the Cornell-box scene, seed 0, rendered
                            by the reference kernels (single thread), plus sampled Sobol values of the
                            reference's sobolGenerate
  textured_room_32x32_4spp.npz  the same for the textured room (checkerboard and image textures, texcoords)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import build_oracle  # noqa: E402
import oracle_py  # noqa: E402

from piper2_b200 import scenes, sobol_tables  # noqa: E402


def main():
    build_oracle.build_oracle()
    if build_oracle.build_ref(sys.argv[1] if len(sys.argv) > 1 else None) is None:
        raise SystemExit("reference sources not found: pass the Piper2 checkout or set PIPER2_REFERENCE")
    with open(os.path.join(HERE, "sobol_digest.txt"), "w") as f:
        f.write(sobol_tables.checksum(*sobol_tables.tables()) + "\n")
    sd = scenes.cornell_box(seed=0, width=32, height=32, spp=4)
    _, samples = oracle_py.RefScene(sd, use_bvh=False).render(threads=1)
    rng = np.random.default_rng(0)
    idx = rng.integers(0, 1 << 40, size=256, dtype=np.uint64)
    dim = rng.integers(0, 1024, size=256, dtype=np.uint32)
    ref = oracle_py.ref()
    sob = np.array([(float(i), float(d), ref.ref_sobol_generate(int(i), int(d))) for i, d in zip(idx, dim)])
    # store exact integers for the index (float64 holds them exactly below 2^53)
    np.savez_compressed(os.path.join(HERE, "cornell_32x32_4spp.npz"), samples=samples, seed=0, sobol=sob)
    sd = scenes.textured_room(seed=0, width=32, height=32, spp=4)
    _, samples = oracle_py.RefScene(sd, use_bvh=False).render(threads=1)
    np.savez_compressed(os.path.join(HERE, "textured_room_32x32_4spp.npz"), samples=samples, seed=0)
    print("golden vectors written")


if __name__ == "__main__":
    main()
