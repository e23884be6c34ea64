#!/usr/bin/env python
"""Benchmark of the superblock hot path: H.psi (model_wave, get_sys.f90:6915) on
the YC4x24 superblock of the benchmark list's config 3 (96 sites, 88
electrons, t1=1, t2=0.3, J1=0.4, J2=0.036) at the middle of the lattice,
sys=47 | 2 sites | env=47, keeping m=4000 SU(2) multiplets.

The sector structure is the one the engine's own warm-up to m=4000 produces
(tests/golden/superblock_yc4x24_m4000.npz, made by
tests/golden/make_bench_superblock.py); operator and psi values are seeded
random (complex N(0,1), Hermitian diagonal blocks), identical for every arm.  A
step is one H.psi application.  `--config 2` puts the YC4x12 m=1000 superblock
(config 2) in the headline instead; it is always measured as a side leg.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--config 2|3]

Prints one JSON line (rank 0).  value = algorithmic TFLOP/s (flops counted in
the reference's GEMM association order, 8*m*n*k per complex GEMM) of all ranks
in the plain FP64 form; N>1 runs independent replicas (the path does not
shard).  Rank 0 adds the split-precision form on the same superblock
("split", with its speed-up over FP64 and its error), the config-2 superblock
in both forms ("config2_hpsi"), the whole YC4x12 ground-state search in both
forms with per-phase seconds ("sweep"), the reference's CPU-runnable case
whole beside the CPU oracle ("sweep_config1"), parameter points and the
synthetic block-sparse H.psi ("config5").
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
FIXTURE = os.path.join(ROOT, "tests", "golden", "superblock_yc4x12_m1000.npz")
MODEL = dict(Nx=12, Ny=4, t1=1.0, t2=0.3, J1=0.4, J2=0.036, delta=12)
FIXTURE3 = os.path.join(ROOT, "tests", "golden", "superblock_yc4x24_m4000.npz")
MODEL3 = dict(Nx=24, Ny=4, t1=1.0, t2=0.3, J1=0.4, J2=0.036, delta=12)
SEED = 20240601
TARGET_METRIC = "sweep sec & H·psi TFLOP/s: split-prec batched vs FP64 GPU at |dE/E|<=1e-10"
METRIC = "H·psi TFLOP/s (plain complex-FP64 GPU form, algorithmic flops)"
WORKLOAD = ("YC4x12 (48 sites, 44 e-, S=0, t1=1 t2=0.3 J1=0.4 J2=0.036) superblock sys=23|2|env=23 "
            "at m=1000 multiplets; one H.psi (model_wave) per step")
WORKLOAD3 = ("YC4x24 (96 sites, 88 e-, S=0, t1=1 t2=0.3 J1=0.4 J2=0.036) superblock sys=47|2|env=47 "
             "at m=4000 multiplets (structure of the engine's warm-up to m=4000); one H.psi (model_wave) per step")
HEADLINES = {2: (FIXTURE, MODEL, WORKLOAD), 3: (FIXTURE3, MODEL3, WORKLOAD3)}


# ----------------------------------------------------------------------------- workload
def scale_dims(ints, k):
    """The same descriptors with every matrix dimension (block, sector, piece
    offset and width, psi sector) multiplied by k: the sector structure of the
    m=1000 superblock at k^2 the size (k=4: m ~ 4000, the size class of YC4x24 at
    m=4000, 64x the flops per H.psi)."""
    if k == 1:
        return ints
    x = ints.astype(np.int64).copy()
    i = 0

    def block():
        nonlocal i
        num = x[i + 1]
        x[i + 2] *= k
        i += 5
        for _ in range(num):
            x[i + 3] *= k
            x[i + 4] *= k
            i += 5

    def model():
        nonlocal i
        nops = x[i + 1]
        i += 2
        block()
        for _ in range(4 * nops):
            block()

    def basis():
        nonlocal i
        num = x[i + 1]
        x[i + 2] *= k
        i += 3
        npc = 0
        for _ in range(num):
            x[i + 2] *= k
            npc += x[i + 3]
            i += 4
        for _ in range(npc):
            x[i + 4] *= k
            x[i + 5] *= k
            i += 6

    model()
    model()
    basis()
    basis()
    num = x[i + 2]
    x[i + 3] *= k * k
    i += 4
    for _ in range(num):
        x[i + 4] *= k
        x[i + 5] *= k
        i += 6
    assert i == len(x)
    return x.astype(np.int32)


def make_superblock(seed=SEED, scale=1, fixture=FIXTURE):
    """Fixture descriptors + seeded values -> (sys_len, env_len, ints, data, psi_offset, n)."""
    z = np.load(fixture)
    ints = scale_dims(z["ints"].astype(np.int32), scale)
    rng = np.random.default_rng(seed)
    chunks = []
    i = 0

    def block(herm):
        nonlocal i
        _ln, num, _dim, _up, _dn = ints[i:i + 5]
        i += 5
        for _ in range(num):
            _nu, _nd, dd, r, q = ints[i:i + 5]
            i += 5
            a = rng.standard_normal((r, q)) + 1j * rng.standard_normal((r, q))
            if herm and r == q and dd == 0:
                a = 0.5 * (a + a.conj().T)
            chunks.append(np.asarray(a, np.complex128).ravel(order="F"))

    def model():
        nonlocal i
        _ln, nops = ints[i:i + 2]
        i += 2
        block(True)
        for _ in range(nops):
            for herm in (False, False, False, True):
                block(herm)

    def basis():
        nonlocal i
        _ln, num, _dim = ints[i:i + 3]
        i += 3
        npc = int(ints[i:i + 4 * num].reshape(num, 4)[:, 3].sum())
        i += 4 * num + 6 * npc

    model()
    model()
    basis()
    basis()
    _sl, _el, num, _dim = ints[i:i + 4]
    i += 4
    secs = ints[i:i + 6 * num].reshape(num, 6)
    i += 6 * num
    n = int((secs[:, 4].astype(np.int64) * secs[:, 5]).sum())
    psi = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    psi /= np.linalg.norm(psi)
    off = int(sum(len(c) for c in chunks))
    chunks.append(psi.astype(np.complex128))
    assert i == len(ints)
    return int(z["sys_len"]), int(z["env_len"]), ints, np.concatenate(chunks), off, n


# ------------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.out = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=lambda: self.out.extend(self.proc.stdout), daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self):
        rows = [[x.strip() for x in line.split(",")] for line in self.out if line.count(",") >= 8]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------------------ helpers
def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return None, 0, 1, 0
    import torch.distributed as dist
    import datetime
    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    return dist, rank, ws, local


def max_over_ranks(x, dist, device):
    """Max of a per-rank float over the process group (timings are max over ranks)."""
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def fp64_peak_tflops(torch, dev):
    """cuBLAS ZGEMM throughput (8 n^3 flops), best of 5: the FP64 denominator."""
    n = 4096
    a = torch.randn(n, n, dtype=torch.complex128, device=dev)
    b = torch.randn(n, n, dtype=torch.complex128, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = max(best, 8.0 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    return best


def cpu_hpsi(sb, nreps, model=MODEL):
    """Oracle (CPU restatement of the reference) H.psi on the same superblock."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import orc
    sl, el, ints, data, _off, n = sb
    o = orc.Oracle(orc.RunConfig(Nx=model["Nx"], Ny=model["Ny"], t1=model["t1"], t2=model["t2"],
                                 J1=model["J1"], J2=model["J2"], delta=model["delta"], sweeps=[1]))
    t0 = time.perf_counter()
    out, sec, flops = o.hpsi_flat(sl, el, ints, data, n, nreps=nreps)
    wall = time.perf_counter() - t0
    return out, sec, flops, wall


# ---------------------------------------------------------------------------- arms
def run_reference(args):
    dist, rank, ws, _local = dist_setup()
    if rank != 0:
        return 0
    fixture, model, workload = HEADLINES[args.config]
    sb = make_superblock(fixture=fixture)
    # bounded sample: at most ~60 s of CPU work whatever K is
    out, sec1, flops, _ = cpu_hpsi(sb, 1, model)
    per = max(sec1, 1e-6)
    k = max(1, min(args.steps, int(60.0 / per)))
    if k > 1:
        _, sec, flops, wall = cpu_hpsi(sb, k, model)
    else:
        sec = sec1
    value = flops / sec / 1e12
    cores = os.cpu_count()
    line = {
        "impl": "reference", "metric": METRIC, "target_metric": TARGET_METRIC, "value": value,
        "unit": "TFLOP/s", "n_gpus": args.gpus, "steps": k, "warmup": 1, "ms_per_step": sec * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
        "data": "synthetic: engine-recorded sector structure, seeded N(0,1) values",
        "config": {"workload": workload, "parallelism": "cpu threads (OpenBLAS)", "cache": "inputs > L2"},
        "cpu_baseline": {"value": value, "unit": "TFLOP/s", "cores": cores, "kind": "port",
                         "sample": f"{k} of {args.steps} H.psi steps (bounded to ~60 s), OpenBLAS threads={cores}; "
                                   "the reference Fortran cannot be compiled here (no Fortran compiler)"},
        "e2e": {"value": value, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def measured_bf16_peak():
    """Burst cuBLAS bf16 TFLOP/s measured on this pool (MEASURED_PEAKS.json), else the fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"]), "MEASURED_PEAKS.json bf16_tflops (burst)"
    except (OSError, KeyError, ValueError):
        return 1590.0, "fallback 1.59 PFLOP/s"


def split_leg(torch, dev, sb, steps, fp64_out, model=MODEL, fp64_ms=None):
    """The split-precision form (BF16 slices on tcgen05) on the same superblock and psi."""
    from tsc_tri_t1t2j1j2_b200 import Context
    sl, el, ints, data, off, n = sb
    ctx = Context(device=dev.index, **model)
    ctx.set_precision(Context.SPLIT_BF16)
    ctx.set_superblock_flat(sl, el, ints, data)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    psi = torch.from_numpy(data[off:off + n].copy()).to(dev)
    out = torch.empty_like(psi)
    torch.cuda.synchronize()
    for _ in range(3):
        ctx.hpsi_device(psi.data_ptr(), out.data_ptr())
    torch.cuda.synchronize()
    # the split form waits for each call (to read the context's status word), so its
    # device time is the sum of the calls' own event brackets (input slicing + 2 launches)
    ms = 0.0
    for _ in range(steps):
        ctx.hpsi_device(psi.data_ptr(), out.data_ptr())
        ms += ctx.hpsi_stats()["device_ms"]
    ms /= steps
    st = ctx.hpsi_stats()
    views = ctx.split_views()
    ctx.close()
    got = out.cpu().numpy()
    err = float(np.max(np.abs(got - fp64_out)) / np.max(np.abs(fp64_out)))
    # tensor work the kernel executes: 6 slice products x 4 real parts per complex
    # multiply-add, 2 flops each = 6x the complex flops of the task list
    bf16_flops = 6.0 * st["exec_flops"]
    peak, src = measured_bf16_peak()
    achieved = bf16_flops / (ms * 1e-3) / 1e12
    # the same H.psi with the operator views each way (the default picks shared
    # views once the folded ones would pass 4 GiB)
    modes = {}
    for name, shared in (("shared", True), ("folded", False)):
        ctx = Context(device=dev.index, **model)
        ctx.set_precision(Context.SPLIT_BF16)
        ctx.set_split_view_sharing(shared)
        ctx.set_superblock_flat(sl, el, ints, data)
        for _ in range(2):
            ctx.hpsi_device(psi.data_ptr(), out.data_ptr())
        fms = 0.0
        for _ in range(max(3, steps // 2)):
            ctx.hpsi_device(psi.data_ptr(), out.data_ptr())
            fms += ctx.hpsi_stats()["device_ms"]
        fms /= max(3, steps // 2)
        modes[name] = {"ms_per_hpsi": fms, "operator_view_bytes": ctx.split_views()["operators"][0],
                       "max_rel_err_vs_fp64": float(np.max(np.abs(out.cpu().numpy() - fp64_out))
                                                    / np.max(np.abs(fp64_out)))}
        ctx.close()
    chosen = "shared" if views["operators"][0] == modes["shared"]["operator_view_bytes"] else "folded"
    return {"hpsi_tflops": st["ref_flops"] / (ms * 1e-3) / 1e12, "ms_per_hpsi": ms,
            "operator_views": chosen, "view_modes": modes,
            "hpsi_speedup_over_fp64": (fp64_ms / ms) if fp64_ms else None,
            "max_rel_err_vs_fp64": err, "tolerance": 2e-5,
            "sliced_operand_bytes": {k: v[0] for k, v in views.items()},
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "peak_source": src,
                         "note": "BF16 tensor flops executed (6x the task list's complex flops)",
                         "kernel": "grouped_zgemm_split (tcgen05, 2 launches per H.psi)"}}


SWEEP_CONFIG = dict(kept_min=200, kept_warm=200, sweeps=[200, 400, 600, 800, 1000, 1000], lanzero=1e-10)
SWEEP_WORKLOAD = ("YC4x12 t1=1 t2=0.3 J1=0.4 J2=0.036, warm-up m=200, 6 sweeps m=200,400,600,800,1000,1000, "
                  "lanzero 1e-10, random start seed 1")


def sweep_leg(dev):
    """Whole ground-state search of YC4x12 (48 sites, m ramped to 1000 over 6 sweeps)
    on the device in both forms: seconds of the warm-up and of the sweeps, the
    final energies and their relative difference."""
    from tsc_tri_t1t2j1j2_b200 import Context
    res = {"workload": SWEEP_WORKLOAD}
    for name, mode in (("fp64", Context.FP64), ("split", Context.SPLIT_BF16)):
        ctx = Context(device=dev.index, **MODEL)
        ctx.set_precision(mode, 1e-11)
        t0 = time.perf_counter()
        steps = ctx.get_ground_state(**SWEEP_CONFIG)
        wall = time.perf_counter() - t0
        t1 = time.perf_counter()
        dens = ctx.measure_density()
        meas_s = time.perf_counter() - t1
        t1 = time.perf_counter()
        cor = ctx.measure_density_cor(1)   # the wave ends at sys_len 2: site 1 with its leg partners
        cor_s = time.perf_counter() - t1
        tuned = ctx.autotune_table()
        ctx.close()
        sw = [s for s in steps if s["phase"] != 0]
        res[name] = {
            "total_seconds": wall,
            "warmup_seconds": sum(s["step_seconds"] for s in steps if s["phase"] == 0),
            "sweep_seconds": sum(s["step_seconds"] for s in sw),
            "seconds_per_sweep": sum(s["step_seconds"] for s in sw) / (len(SWEEP_CONFIG["sweeps"]) + 1),
            "lanczos_seconds": sum(s["lanczos_seconds"] for s in sw),
            "hpsi_seconds": sum(s["hpsi_seconds"] for s in sw),
            "phase_seconds": {ph: sum(s[ph + "_seconds"] for s in sw)
                              for ph in ("set", "lanczos", "truncate", "grow", "wave")},
            "lanczos_iters": int(sum(s["lanczos_iters"] for s in sw)),
            "split_iters": int(sum(s["split_iters"] for s in sw)),
            "final_e0": steps[-1]["e0"],
            "min_e0": min(s["e0"] for s in steps),
            "density_seconds": meas_s,
            "density": dens,
            "density_cor_seconds": cor_s,
            "density_cor": cor,
            "trun_err": np.array([s["trun_err"] for s in steps]),
            "autotune_ms_per_gflop": {str(k): v for k, v in tuned.items()},
        }
    res["density_max_abs_diff_split_vs_fp64"] = float(np.max(np.abs(res["split"]["density"] - res["fp64"]["density"])))
    res["density_sum_fp64"] = float(res["fp64"]["density"].sum())
    res["density_cor_site1_max_abs_diff_split_vs_fp64"] = float(
        np.max(np.abs(res["split"]["density_cor"] - res["fp64"]["density_cor"])))
    res["density_cor_site1_partners"] = int(np.count_nonzero(res["fp64"]["density_cor"]))
    if len(res["split"]["trun_err"]) == len(res["fp64"]["trun_err"]):
        res["trun_err_max_abs_diff_split_vs_fp64"] = float(
            np.max(np.abs(res["split"]["trun_err"] - res["fp64"]["trun_err"])))
    for name in ("fp64", "split"):
        del res[name]["density"], res[name]["density_cor"], res[name]["trun_err"]
    res["final_dE_over_E_split_vs_fp64"] = abs(res["split"]["final_e0"] - res["fp64"]["final_e0"]) / abs(
        res["fp64"]["final_e0"])
    res["sweep_speedup_split_over_fp64"] = res["fp64"]["sweep_seconds"] / res["split"]["sweep_seconds"]
    return res


CONFIG1 = dict(Nx=6, Ny=4, t1=1.0, t2=0.0, J1=0.4, J2=0.0, delta=12)
CONFIG1_RUN = dict(kept_min=100, kept_warm=100, sweeps=[100, 200, 300, 400], lanzero=1e-10)


def config1_leg(dev, with_cpu):
    """The reference's CPU-runnable case, whole: YC4x6 (24 sites, 22 e-), t1=1, J1=0.4,
    4 sweeps m=100/200/300/400, lanzero 1e-10 -- on the device in both forms and,
    with the CPU leg, the oracle (CPU restatement, OpenBLAS on all host cores)."""
    from tsc_tri_t1t2j1j2_b200 import Context
    res = {"workload": "YC4x6 t1=1 J1=0.4 t2=J2=0, warm-up m=100, 4 sweeps m=100,200,300,400, lanzero 1e-10"}
    dens, cors = {}, {}
    for name, mode in (("fp64", Context.FP64), ("split", Context.SPLIT_BF16)):
        ctx = Context(device=dev.index, **CONFIG1)
        ctx.set_precision(mode, 1e-11)
        t0 = time.perf_counter()
        steps = ctx.get_ground_state(**CONFIG1_RUN)
        res[name] = {"seconds": time.perf_counter() - t0, "steps": len(steps), "final_e0": steps[-1]["e0"]}
        dens[name] = ctx.measure_density()
        cors[name] = ctx.measure_density_cor(1)
        ctx.close()
    if with_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import orc
        cfg = orc.RunConfig(Nx=6, Ny=4, t1=1.0, t2=0.0, J1=0.4, J2=0.0, kept_min=100, kept_warm=100,
                            sweeps=[100, 200, 300, 400], lanzero=1e-10)
        t0 = time.perf_counter()
        o = orc.Oracle(cfg)
        ref = o.run()
        sec = time.perf_counter() - t0
        dref = o.measure_density()
        cref = o.density_cor(1).real
        res["cpu_oracle"] = {"seconds": sec, "cores": os.cpu_count(), "steps": len(ref), "final_e0": ref[-1]["e0"]}
        res["fp64_final_dE_over_E_vs_oracle"] = abs(res["fp64"]["final_e0"] - ref[-1]["e0"]) / abs(ref[-1]["e0"])
        res["speedup_fp64_gpu_over_cpu"] = sec / res["fp64"]["seconds"]
        res["density_max_abs_diff_fp64_vs_oracle"] = float(np.max(np.abs(dens["fp64"] - dref)))
        res["density_max_abs_diff_split_vs_oracle"] = float(np.max(np.abs(dens["split"] - dref)))
        res["density_cor_site1_max_abs_diff_fp64_vs_oracle"] = float(np.max(np.abs(cors["fp64"] - cref)))
        res["density_cor_site1_max_abs_diff_split_vs_oracle"] = float(np.max(np.abs(cors["split"] - cref)))
        res["split_final_dE_over_E_vs_oracle"] = abs(res["split"]["final_e0"] - ref[-1]["e0"]) / abs(ref[-1]["e0"])
    return res


def config5_leg(torch, dev, zgemm_peak, ks=(64,), batch=True):
    """The benchmark list's synthetic block-sparse H.psi (tsc_blocksparse_*): one
    problem of K sectors per K in `ks` (the list names 64, 128, 256, 400),
    dimensions log-uniform in [16, 2048], 8 left and 8 right operator sets with
    sector shifts in -2..2, 200 terms with alpha ~ U[-1,1]; and a batch of 32
    independent problems of uneven size (K in 16..64, dimensions in [16, 256])
    applied in one pair of launches.  FP64 and split forms, the split form's
    largest absolute deviation from the FP64 result."""
    from tsc_tri_t1t2j1j2_b200 import Context
    from tsc_tri_t1t2j1j2_b200.blocksparse import pack, random_psi, synthetic, synthetic_packed
    out = {"workload": "synthetic block-sparse H.psi: entries re/im N(0,1), shift-0 blocks Hermitian; "
                       "single (K=64; K<n> for other K): dims log-uniform [16,2048] 8+8 sets 200 terms; "
                       "batch32: 32 problems K in 16..64 dims [16,256] 8+8 sets 200 terms each, one launch pair"}
    rng = np.random.default_rng(SEED + 5)

    def single(k):   # K = 64 keeps the generator state of the default leg
        r = rng if k == 64 else np.random.default_rng(SEED + 5 + k)
        P, ints, data = synthetic_packed(r, k, 16, 2048)
        return [P], (1, ints, data), r

    cases = [("single" if k == 64 else f"K{k}", lambda k=k: single(k)) for k in ks]
    if batch:
        cases.append(("batch32", lambda: (lambda pr: (pr, pack(pr), rng))(
            [synthetic(rng, int(k), 16, 256) for k in rng.integers(16, 65, 32)])))
    for name, make in cases:
        probs, packed, prng = make()
        ctx = Context(device=dev.index, **MODEL)
        n, flops, xflops = ctx.blocksparse_set_packed(*packed)
        del packed
        x = torch.from_numpy(random_psi(prng, probs)).to(dev)
        ys = {}
        res = {"problems": len(probs), "psi_amplitudes": n, "gflop_per_application": flops / 1e9,
               "gflop_executed": xflops / 1e9}
        stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
        for form, mode in (("fp64", Context.FP64), ("split", Context.SPLIT_BF16)):
            y = torch.empty_like(x)
            torch.cuda.synchronize()
            for _ in range(2):
                ctx.blocksparse_apply(x.data_ptr(), y.data_ptr(), mode)
            torch.cuda.synchronize()
            reps = 5
            ms = 0.0
            for _ in range(reps):   # each call's own event bracket (the split form waits per call)
                ctx.blocksparse_apply(x.data_ptr(), y.data_ptr(), mode)
                ms += ctx.hpsi_stats()["device_ms"]
            ms /= reps
            res[form] = {"ms": ms, "tflops": flops / (ms * 1e-3) / 1e12,
                         "executed_tflops": xflops / (ms * 1e-3) / 1e12}
            ys[form] = y.cpu().numpy()
        res["fp64"]["frac_of_zgemm"] = res["fp64"]["executed_tflops"] / zgemm_peak
        bf16, _ = measured_bf16_peak()
        res["split"]["frac_of_bf16"] = 6.0 * res["split"]["executed_tflops"] / bf16
        res["split_max_abs_err"] = float(np.max(np.abs(ys["split"] - ys["fp64"])))
        res["split_max_rel_err"] = res["split_max_abs_err"] / float(np.max(np.abs(ys["fp64"])))
        res["split_speedup"] = res["fp64"]["ms"] / res["split"]["ms"]
        res["split_operator_view_bytes"] = ctx.split_views()["operators"][0]
        out[name] = res
        ctx.close()
    return out


def points_leg(dev):
    """Eight parameter points of the reference's CPU-runnable case (YC4x6, 4 sweeps
    m=100..400), t2 = 0, 0.05, ..., 0.35 with J2 = J1 (t2/t1)^2: run one after the
    other, then all at once (run_parameter_points: a context and host thread per
    point).  Seconds of both and the final energies' largest difference."""
    from tsc_tri_t1t2j1j2_b200 import Context, run_parameter_points
    pts = [dict(Nx=6, Ny=4, t1=1.0, t2=0.05 * k, J1=0.4, J2=0.4 * (0.05 * k) ** 2) for k in range(8)]
    t0 = time.perf_counter()
    seq = []
    for p in pts:
        ctx = Context(device=dev.index, **p)
        seq.append(ctx.get_ground_state(**CONFIG1_RUN)[-1]["e0"])
        ctx.close()
    t_seq = time.perf_counter() - t0
    t0 = time.perf_counter()
    par = [st[-1]["e0"] for st in run_parameter_points(pts, CONFIG1_RUN, device=dev.index)]
    t_par = time.perf_counter() - t0
    return {"workload": "8 x YC4x6 (t2 = 0..0.35, J2 = J1 t2^2), 4 sweeps m=100..400, lanzero 1e-10",
            "sequential_seconds": t_seq, "concurrent_seconds": t_par, "throughput_gain": t_seq / t_par,
            "final_e0_max_rel_diff": max(abs(a - b) / abs(b) for a, b in zip(par, seq))}


def fp64_hpsi(torch, dev, sb, model, steps, warmup, dist=None, clocks=None):
    """The plain FP64 form on one superblock: the autotuner's schedule, `steps`
    H.psi timed back to back by CUDA events on the engine stream (one barrier and
    synchronisation on each side), and the mean device time of one H.psi's
    grouped-GEMM launches.  Returns (ctx, psi, out, result dict)."""
    from tsc_tri_t1t2j1j2_b200 import Context
    sl, el, ints, data, off, n = sb
    ctx = Context(device=dev.index, **model)
    ctx.set_superblock_flat(sl, el, ints, data)
    assert ctx.dim == n
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    schedule = ctx.autotune_superblock(3)   # the autotuner's pick for this superblock, before timing
    tune_table = ctx.autotune_table()
    psi = torch.from_numpy(data[off:off + n].copy()).to(dev)
    out = torch.empty_like(psi)
    torch.cuda.synchronize()
    for _ in range(warmup):
        ctx.hpsi_device(psi.data_ptr(), out.data_ptr())
    torch.cuda.synchronize()
    st = ctx.hpsi_stats()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(dev.index) if clocks else None
    if sampler:
        sampler.__enter__()
    e0.record(stream)
    for _ in range(steps):
        ctx.hpsi_device(psi.data_ptr(), out.data_ptr())
    e1.record(stream)
    e1.synchronize()
    if sampler:
        sampler.__exit__()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if dist is not None:
        ms = max_over_ranks(ms, dist, dev)
        dist.barrier()
    kms = []
    for _ in range(min(20, max(3, steps))):
        ctx.hpsi_device(psi.data_ptr(), out.data_ptr())
        kms.append(ctx.hpsi_stats()["device_ms"])
    res = {"ms_total": ms, "ms_per_step": ms / steps, "ref_flops": st["ref_flops"], "exec_flops": st["exec_flops"],
           "launches_per_step": st["launches"],
           "kernel_ms": float(np.mean(kms)), "schedule": schedule, "tune_table": tune_table,
           "clocks": sampler.summary() if sampler else None, "psi_amplitudes": n, "operator_elements": int(off)}
    return ctx, psi, out, res


def run_gpu(args):
    import torch
    from tsc_tri_t1t2j1j2_b200 import _lib
    dist, rank, ws, local = dist_setup()
    if dist is not None:
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    fixture, model, workload = HEADLINES[args.config]
    sb = make_superblock(scale=args.scale, fixture=fixture)
    sl, el, ints, data, off, n = sb
    ctx, psi, out, r = fp64_hpsi(torch, dev, sb, model, args.steps, args.warmup, dist, clocks=True)
    ms, ref_flops, exec_flops, kernel_ms = r["ms_total"], r["ref_flops"], r["exec_flops"], r["kernel_ms"]
    value = ws * args.steps * ref_flops / (ms * 1e-3) / 1e12
    # end to end through the C-ABI: pinned host psi -> device -> H.psi -> host
    xh = torch.from_numpy(data[off:off + n].copy()).pin_memory()
    yh = torch.empty_like(xh).pin_memory()
    L = _lib.load()
    import ctypes
    P = ctypes.POINTER(ctypes.c_double)
    xp, yp = ctypes.cast(xh.data_ptr(), P), ctypes.cast(yh.data_ptr(), P)
    for _ in range(3):
        assert L.tsc_hpsi(ctx.h, xp, yp) == 0
    ke2e = max(3, args.steps // 4)
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(ke2e):
        L.tsc_hpsi(ctx.h, xp, yp)
    e2e_s = time.perf_counter() - t0
    if dist is not None:
        e2e_s = max_over_ranks(e2e_s, dist, dev)
    e2e = ws * ke2e * ref_flops / e2e_s / 1e12
    gpu_out = out.cpu().numpy()
    ctx.close()
    del psi, out
    line = None
    if rank == 0:
        peak = fp64_peak_tflops(torch, dev)
        achieved = ref_flops / (kernel_ms * 1e-3) / 1e12
        line = {
            "metric": METRIC, "target_metric": TARGET_METRIC, "value": value, "unit": "TFLOP/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "data": f"synthetic: engine-recorded sector structure ({os.path.relpath(fixture, ROOT)}), "
                    "seeded N(0,1) complex values",
            "config": {"workload": workload if args.scale == 1 else
                       workload + f"; every dimension scaled x{args.scale}",
                       "psi_amplitudes": n, "operator_elements": int(off),
                       "ref_gflop_per_step": ref_flops / 1e9, "exec_gflop_per_step": exec_flops / 1e9,
                       "parallelism": f"replicas x{ws}", "cache": f"inputs > L2 (operators {16 * off / 1e6:.0f} MB)"},
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": None,
                         "executed_frac": exec_flops / (kernel_ms * 1e-3) / 1e12 / peak,
                         "note": "achieved counts the reference's GEMM association order; the kernel shares "
                                 "left products and executes exec_gflop_per_step, hence frac slightly above 1 "
                                 "where executed_frac is below it",
                         "algorithmic_bytes": traffic_model(sb),
                         "algorithmic_bytes_note": "every operator sub-block and psi element read once, every "
                                                   "output element written once, per H.psi",
                         "peak_source": "cuBLAS ZGEMM 4096^3 complex128 measured in this run (FP64 DMMA)",
                         "kernel": "grouped_zgemm (2 launches per H.psi, + reduce_partials where a group's terms were split)",
                         "schedule": {"tile": r["schedule"][0], "waves": r["schedule"][1],
                                      "candidates_ms_per_gflop": {str(k): v for k, v in r["tune_table"].items()}}},
            "e2e": {"value": e2e, "unit": "TFLOP/s", "h2d_bytes_per_step": 16 * n, "d2h_bytes_per_step": 16 * n},
            # the grouped GEMM of each phase plus the fixed-order reductions of split groups
            "gpu_launches": r["launches_per_step"] * args.steps,
            "clocks": r["clocks"],
        }
        # side legs only at N = 1: under torchrun the other ranks wait at the closing
        # barrier, whose process-group timeout the legs' minutes would exceed
        side = ws == 1
        if side:
            line["split"] = split_leg(torch, dev, sb, max(10, args.steps // 4), gpu_out, model, r["kernel_ms"])
        if side and args.config != 2:
            line["config2_hpsi"] = config2_leg(torch, dev, args.warmup)
        if side and not args.no_synthetic:
            line["config5"] = config5_leg(torch, dev, peak)
        if side and not args.no_sweep:
            line["sweep"] = sweep_leg(dev)
            line["sweep_config1"] = config1_leg(dev, ws == 1 and not args.no_cpu)
            line["parameter_points"] = points_leg(dev)
        if ws == 1 and not args.no_cpu:
            cpu_out, sec, flops, wall = cpu_hpsi(sb, 1, model)
            err = float(np.max(np.abs(gpu_out - cpu_out)) / np.max(np.abs(cpu_out)))
            line["cpu_baseline"] = {"value": flops / sec / 1e12, "unit": "TFLOP/s", "cores": os.cpu_count(),
                                    "kind": "port", "sample": "1 H.psi of the same superblock (oracle, OpenBLAS "
                                                              f"threads={os.cpu_count()}), {sec:.2f} s"}
            line["parity"] = {"max_rel_err_vs_oracle": err, "tolerance": 1e-13}
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)
    return 0


def config2_leg(torch, dev, warmup):
    """The config-2 superblock (YC4x12 m=1000) in both forms: FP64 TFLOP/s, split
    TFLOP/s, the split/FP64 time ratio and the split form's error."""
    sb = make_superblock()
    ctx, psi, out, r = fp64_hpsi(torch, dev, sb, MODEL, 20, warmup)
    fp64_out = out.cpu().numpy()
    ctx.close()
    res = {"workload": WORKLOAD, "fp64": {"ms_per_hpsi": r["ms_per_step"], "kernel_ms": r["kernel_ms"],
                                          "hpsi_tflops": r["ref_flops"] / (r["ms_per_step"] * 1e-3) / 1e12}}
    res["split"] = split_leg(torch, dev, sb, 20, fp64_out, MODEL, r["kernel_ms"])
    return res


def traffic_model(sb):
    """Bytes one H.psi must move at least: the superblock's operator sub-blocks and
    psi read once (16 B per complex element) and the output written once."""
    _sl, _el, _ints, _data, off, n = sb
    return 16 * (int(off) + 2 * int(n))


def dmrg_steps(args):
    """Config 3 whole DMRG steps in both forms: YC4x24, warm-up to m=4000 (FP64 in
    both forms, the reference's warm-up tolerance 1e-3), then the first
    `--dmrg-steps` steps of the following half sweep at lanzero 1e-10, once with
    the plain FP64 form and once with the split form.  Prints one JSON line with
    the seconds of every step (and of its Lanczos solve), iteration counts,
    energies and the split form's per-step |dE/E| against FP64.  Not a bench
    line: about 30 GPU-minutes."""
    from tsc_tri_t1t2j1j2_b200 import Context
    N = MODEL3["Nx"] * MODEL3["Ny"]
    nwarm = N // 2 - 1
    res = {"workload": f"YC4x24 warm-up to m=4000 (lanzero 1e-3) + {args.dmrg_steps} steps of the first half sweep "
                       "at m=4000, lanzero 1e-10", "forms": {}}
    forms = [f for f in (("fp64", Context.FP64), ("split", Context.SPLIT_BF16)) if f[0] in args.dmrg_forms.split(",")]
    for name, mode in forms:
        ctx = Context(device=0, **MODEL3)
        ctx.set_precision(mode, 1e-11)
        t0 = time.perf_counter()
        st = ctx.get_ground_state(4000, 4000, [4000], lanzero=1e-10, seed=1, max_solves=nwarm + args.dmrg_steps,
                                  lanzero_warmup=1e-3)
        wall = time.perf_counter() - t0
        spill = ctx.spill_stats()
        ctx.close()
        keys = ("phase", "sys_len", "e0", "lanczos_iters", "split_iters", "num_state", "trun_err", "step_seconds",
                "lanczos_seconds", "hpsi_seconds", "set_seconds", "truncate_seconds", "grow_seconds", "wave_seconds")
        res["forms"][name] = {"wall_seconds": wall, "warmup_seconds": sum(x["step_seconds"] for x in st[:nwarm]),
                              "spill": spill, "steps": [{k: x[k] for k in keys} for x in st[nwarm:]]}
        print(name, wall, flush=True, file=sys.stderr)
    res["step_seconds"] = {k: sum(x["step_seconds"] for x in v["steps"]) for k, v in res["forms"].items()}
    if len(res["forms"]) == 2:
        a, b = res["forms"]["fp64"]["steps"], res["forms"]["split"]["steps"]
        res["dE_over_E_split_vs_fp64"] = [abs(x["e0"] - y["e0"]) / abs(x["e0"]) for x, y in zip(a, b)]
        res["steps_speedup_split_over_fp64"] = res["step_seconds"]["fp64"] / res["step_seconds"]["split"]
    print(json.dumps(res), flush=True)
    return 0


def sweep_study(args):
    """The YC4x12 whole run of the sweep leg five ways: FP64 at lanzero 1e-13 (the
    converged reference energy), the split form with the reference's stop for its
    FP64 finish, the split form with the residual stop 0.1 sqrt(lanzero), the
    split form with its U^H O U renormalisation split too, and FP64 at lanzero
    1e-10.  Prints one JSON line: seconds, iterations and each final energy's
    distance from the FP64 and the converged runs."""
    from tsc_tri_t1t2j1j2_b200 import Context
    runs = (("fp64_lanzero_1e-13", Context.FP64, 1e-13, None, False),
            ("split_reference_stop", Context.SPLIT_BF16, 1e-10, 0.0, False),
            ("split_residual_0.1", Context.SPLIT_BF16, 1e-10, 0.1, False),
            ("split_renormalization_split", Context.SPLIT_BF16, 1e-10, 0.0, True),
            ("fp64", Context.FP64, 1e-10, None, False))
    out = {"workload": SWEEP_WORKLOAD}
    for name, mode, lz, refine, renorm in runs:
        ctx = Context(device=0, **MODEL)
        ctx.set_precision(mode, 1e-11)
        if refine is not None:
            ctx.set_split_refinement(refine)
        ctx.set_split_renormalization(renorm)
        t0 = time.perf_counter()
        st = ctx.get_ground_state(**dict(SWEEP_CONFIG, lanzero=lz))
        wall = time.perf_counter() - t0
        ctx.close()
        sw = [x for x in st if x["phase"] != 0]
        out[name] = {"wall_seconds": wall, "sweep_seconds": sum(x["step_seconds"] for x in sw),
                     "lanczos_seconds": sum(x["lanczos_seconds"] for x in sw),
                     "lanczos_iters": int(sum(x["lanczos_iters"] for x in sw)),
                     "split_iters": int(sum(x["split_iters"] for x in sw)), "final_e0": st[-1]["e0"],
                     "grow_seconds": sum(x["grow_seconds"] for x in sw)}
    t, f = out["fp64_lanzero_1e-13"]["final_e0"], out["fp64"]["final_e0"]
    for name, *_ in runs:
        e = out[name]["final_e0"]
        out[name]["dE_over_E_vs_fp64"] = abs(e - f) / abs(f)
        out[name]["dE_over_E_vs_converged"] = abs(e - t) / abs(t)
    print(json.dumps(out), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-sweep", action="store_true", help="skip the whole-run (sweep seconds) leg")
    ap.add_argument("--no-synthetic", action="store_true", help="skip the synthetic block-sparse leg")
    ap.add_argument("--config", type=int, default=3 if os.path.exists(FIXTURE3) else 2, choices=[2, 3],
                    help="headline superblock: 3 = YC4x24 m=4000 (default), 2 = YC4x12 m=1000")
    ap.add_argument("--scale", type=int, default=1,
                    help="multiply every dimension of the superblock by this (4: m ~ 4000 size class)")
    ap.add_argument("--sweep-study", action="store_true",
                    help="instead of the bench line: the YC4x12 whole run in four solver settings")
    ap.add_argument("--dmrg-steps", type=int, default=0,
                    help="instead of the bench line: config-3 warm-up + this many m=4000 DMRG steps in both forms")
    ap.add_argument("--dmrg-forms", default="fp64,split", help="forms run by --dmrg-steps (comma-separated)")
    ap.add_argument("--config5", default="",
                    help="instead of the bench line: the synthetic block-sparse H.psi for these K (comma-separated)")
    args = ap.parse_args()
    if args.dmrg_steps > 0:
        return dmrg_steps(args)
    if args.config5:
        import torch
        dev = torch.device("cuda", 0)
        ks = tuple(int(k) for k in args.config5.split(","))
        print(json.dumps(config5_leg(torch, dev, fp64_peak_tflops(torch, dev), ks, batch=False)), flush=True)
        return 0
    if args.sweep_study:
        return sweep_study(args)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
