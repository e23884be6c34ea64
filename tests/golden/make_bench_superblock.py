"""Record the sector structure of the benchmark superblock.

Runs the engine's warm-up (warm_up_point, dmrg_sub.f90:974-1147) on YC4x12
(48 sites, 44 electrons, t1=1, t2=0.3, J1=0.4, J2=0.036) keeping m=1000
multiplets, and stores the descriptor part (ints only, no matrix values) of the
last warm-up superblock, sys=23 + 2 sites + env=23: the sector lists, piece
offsets and operator sub-block shapes that fix the H.psi workload.  bench.py
fills the matrices with seeded random values.  Needs a GPU; run from the repo
root:  python tests/golden/make_bench_superblock.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from tsc_tri_t1t2j1j2_b200 import Context  # noqa: E402


def main(m=1000):
    ctx = Context(12, 4, 1.0, 0.3, 0.4, 0.036)
    steps = ctx.get_ground_state(m, m, [], lanzero=1e-10, seed=1, capture_step=22, warmup_only=True)
    ints, data, sl, el = ctx.capture()
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), f"superblock_yc4x12_m{m}.npz")
    np.savez_compressed(out, ints=ints, sys_len=sl, env_len=el, ncplx=len(data),
                        e0=steps[-1]["e0"], steps=len(steps))
    print("wrote", out, sl, el, len(ints), len(data))


if __name__ == "__main__":
    main(int(sys.argv[1]) if len(sys.argv) > 1 else 1000)
