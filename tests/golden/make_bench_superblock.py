"""Record the sector structure of a benchmark superblock.

Runs the engine's warm-up (warm_up_point, dmrg_sub.f90:974-1147) on a YC4
cylinder (t1=1, t2=0.3, J1=0.4, J2=0.036, one hole per 12 sites) keeping m
multiplets and stores the descriptor part (ints only, no matrix values) of the
last warm-up superblock, sys = N/2-1 sites + 2 sites + env = N/2-1 sites: the
sector lists, piece offsets and operator sub-block shapes that fix the H.psi
workload.  bench.py fills the matrices with seeded random values.

  python tests/golden/make_bench_superblock.py            # YC4x12, m=1000 (lanzero 1e-10)
  python tests/golden/make_bench_superblock.py 24 4000 --reference-schedule --solve
                                                          # YC4x24, m=4000 (warm-up lanzero 1e-3)

With --solve, the real superblock captured there (its operators and start
vector, not random values) is also solved by Lanczos (lanczos_memo_new,
eigen.f90:4-199, lanzero 1e-10) in the plain FP64 and the split-precision
form from the same start vector, and a JSON line reports both energies, their
relative difference, the iteration counts and the seconds of each solve, with
the warm-up's per-step timings and the stored-model spill counters.  Needs a
GPU; run from the repo root.
"""
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from tsc_tri_t1t2j1j2_b200 import Context  # noqa: E402

MODEL = dict(Ny=4, t1=1.0, t2=0.3, J1=0.4, J2=0.036)


def main(Nx=12, m=1000, solve=False, reference_schedule=False):
    N = 4 * Nx
    ctx = Context(Nx=Nx, **MODEL)
    t0 = time.perf_counter()
    # lanzero 1e-10 in every step, or the reference's warm-up tolerance (1e-3, main.f90 schedule)
    steps = ctx.get_ground_state(m, m, [], lanzero=-1.0 if reference_schedule else 1e-10, seed=1,
                                 capture_step=N // 2 - 2, warmup_only=True)
    warm_s = time.perf_counter() - t0
    ints, data, sl, el = ctx.capture()
    spill = ctx.spill_stats()
    ctx.close()
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), f"superblock_yc4x{Nx}_m{m}.npz")
    np.savez_compressed(out, ints=ints, sys_len=sl, env_len=el, ncplx=len(data),
                        e0=steps[-1]["e0"], steps=len(steps))
    print("wrote", out, sl, el, len(ints), len(data), flush=True)
    if not solve:
        return
    res = {"workload": f"YC4x{Nx} warm-up to m={m}, last warm-up superblock sys={sl}|2|env={el}",
           "warmup_seconds": warm_s, "spill": spill,
           "warmup_steps": [{k: s[k] for k in ("sys_len", "num_state", "lanczos_iters", "step_seconds",
                                                "lanczos_seconds", "truncate_seconds", "grow_seconds",
                                                "hpsi_seconds", "set_seconds")} for s in steps]}
    for name, mode in (("fp64", Context.FP64), ("split", Context.SPLIT_BF16)):
        c = Context(Nx=Nx, **MODEL)
        try:
            c.set_precision(mode, 1e-11)
            c.set_superblock_flat(sl, el, ints, data)
            n = c.dim
            psi0 = np.ascontiguousarray(data[len(data) - n:])
            t1 = time.perf_counter()
            vec, e0, iters = c.lanczos_memo_new(psi0, 1e-10)
            res[name] = {"e0": e0, "iters": iters, "seconds": time.perf_counter() - t1, "dim": n}
        finally:
            c.close()
    res["dE_over_E_split_vs_fp64"] = abs(res["split"]["e0"] - res["fp64"]["e0"]) / abs(res["fp64"]["e0"])
    res["solve_speedup_split_over_fp64"] = res["fp64"]["seconds"] / res["split"]["seconds"]
    print(json.dumps(res))


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    main(int(args[0]) if args else 12, int(args[1]) if len(args) > 1 else 1000, "--solve" in sys.argv,
         "--reference-schedule" in sys.argv)
