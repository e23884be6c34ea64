"""Parity on the benchmark list's own configurations, through the C-ABI.

Config 1 (YC4x6, 24 sites, 22 electrons, t1=1, J1=0.4, t2=J2=0; warm-up
m=100, sweeps m=100/200/300/400, lanzero 1e-10), the reference's CPU-runnable
case, whole on the device in the plain FP64 form against the oracle at every
one of its 211 DMRG steps: identical kept multiplet counts and Lanczos
iteration counts; truncation weights within 1e-12 absolute; the final energy
within |dE/E| <= 1e-12 (observed 1.5e-15).  Each step's energy is a Lanczos
result stopped when successive Ritz values agree to lanzero = 1e-10 absolute,
so rounding differences between two correct implementations move it within
that tolerance: per step |dE/E| <= 1e-11 (observed <= 1.5e-12, 3.4e-12 with
the four-multiplication complex product), entanglement entropies within 1e-9
(sums over the whole spectrum, observed <= 1.3e-10).  At one step of the last
sweep (m=400, mid-lattice) the sorted density-matrix spectrum itself is
compared to 1e-12.

Config 2 (YC4x12, 48 sites, 44 electrons, t2=0.3, J2=0.036): one H.psi of the
m=1000 superblock (the engine-recorded sector structure with seeded values,
tests/golden/superblock_yc4x12_m1000.npz) against the oracle's model_wave to
1e-13 relative; and real superblocks of its first sweeps (m=200, captured
from an FP64 run) solved by Lanczos (lanzero 1e-10) in the split-precision
form and in FP64 from the same start vector: |dE/E| <= 1e-10.

Config 3 (YC4x24, 96 sites, 88 electrons): one H.psi of the m=4000 middle
superblock (the structure of the engine's own warm-up to m=4000,
tests/golden/superblock_yc4x24_m4000.npz, seeded values) against the oracle's
model_wave to 1e-13 relative.
"""
import numpy as np
import pytest

import orc
from _capture import parse_oracle_capture
from tsc_tri_t1t2j1j2_b200 import Context

CONFIG1 = dict(Nx=6, Ny=4, t1=1.0, t2=0.0, J1=0.4, J2=0.0)
CONFIG1_RUN = dict(kept_min=100, kept_warm=100, sweeps=[100, 200, 300, 400], lanzero=1e-10)
CAPTURE = 200   # a right_to_left step of the m=400 sweep, mid-lattice
TRUN_ERR = 1.0000000036274937e-15


@pytest.fixture(scope="module")
def config1():
    cfg = orc.RunConfig(kept_min=100, kept_warm=100, sweeps=[100, 200, 300, 400], lanzero=1e-10,
                        seed=1, **CONFIG1)
    o = orc.Oracle(cfg, capture_step=CAPTURE)
    ref = o.run()
    cap = parse_oracle_capture(*o.capture())
    ctx = Context(device=0, **CONFIG1)
    got = ctx.get_ground_state(seed=1, **CONFIG1_RUN)
    yield ref, cap, got, ctx
    ctx.close()


@pytest.mark.gpu
def test_config1_every_step_matches_oracle(config1):
    ref, _cap, got, _ctx = config1
    assert len(got) == len(ref) == 211
    for k, (g, r) in enumerate(zip(got, ref)):
        assert (g["phase"], g["sys_len"], g["env_len"]) == (int(r["phase"]), int(r["sys_len"]), int(r["env_len"])), k
        assert abs(g["e0"] - r["e0"]) <= 1e-11 * abs(r["e0"]), (k, g["e0"], r["e0"])
        assert g["num_state"] == int(r["num_state"]), k
        assert g["lanczos_iters"] == int(r["iters"]), (k, g["lanczos_iters"], r["iters"])
        assert abs(g["trun_err"] - r["trun_err"]) <= 1e-12, (k, g["trun_err"], r["trun_err"])
        assert abs(g["entropy"] - r["entropy"]) <= 1e-9, (k, g["entropy"], r["entropy"])
        assert abs(g["entropy_mult"] - r["entropy_mult"]) <= 1e-9, (k, g["entropy_mult"], r["entropy_mult"])
    assert abs(got[-1]["e0"] - ref[-1]["e0"]) <= 1e-12 * abs(ref[-1]["e0"])


@pytest.mark.gpu
def test_config1_density_matrix_spectrum_matches_oracle(config1):
    _ref, cap, _got, ctx = config1
    assert len(cap["spectrum"]) > 0 and cap["num_state"] == 400
    ctx.set_superblock(cap["sys"], cap["env"], cap["sys_bs"], cap["env_bs"], cap["psi0"])
    side = 0 if cap["sys_side"] else 1
    r = ctx.get_truncation_operator(side, cap["gs"].vec, 100, 400, TRUN_ERR)
    n = len(cap["spectrum"])
    assert np.max(np.abs(r["spectrum"][:n] - cap["spectrum"])) <= 1e-12
    assert r["num_state"] == cap["num_state"]
    assert abs(r["err"] - cap["err"]) <= 1e-12


@pytest.mark.gpu
def test_config2_superblock_hpsi_matches_oracle():
    import bench
    sl, el, ints, data, off, n = bench.make_superblock()
    o = orc.Oracle(orc.RunConfig(**bench.MODEL))
    ref, _sec, _flops = o.hpsi_flat(sl, el, ints, data, n)
    ctx = Context(device=0, **bench.MODEL)
    try:
        ctx.set_superblock_flat(sl, el, ints, data)
        out = ctx.model_wave(data[off:off + n])
    finally:
        ctx.close()
    assert float(np.max(np.abs(out - ref)) / np.max(np.abs(ref))) <= 1e-13


@pytest.mark.parametrize("step", [30, 60, 90])
@pytest.mark.gpu
def test_config2_split_solve_matches_fp64(step):
    """A real config-2 superblock (captured at `step` of an FP64 run: warm-up and
    the two half sweeps at m=200) solved in both forms from its start vector."""
    model = dict(Nx=12, Ny=4, t1=1.0, t2=0.3, J1=0.4, J2=0.036)
    ctx = Context(device=0, **model)
    try:
        ctx.get_ground_state(200, 200, [], lanzero=1e-10, seed=1, capture_step=step)
        ints, data, sl, el = ctx.capture()
    finally:
        ctx.close()
    e = {}
    for mode in (Context.FP64, Context.SPLIT_BF16):
        c = Context(device=0, **model)
        try:
            c.set_precision(mode, 1e-11)
            c.set_superblock_flat(sl, el, ints, data)
            n = c.dim
            _vec, e[mode], _iters = c.lanczos_memo_new(np.ascontiguousarray(data[len(data) - n:]), 1e-10)
        finally:
            c.close()
    assert abs(e[Context.SPLIT_BF16] - e[Context.FP64]) <= 1e-10 * abs(e[Context.FP64])


@pytest.mark.gpu
def test_config3_superblock_hpsi_matches_oracle():
    import bench
    sl, el, ints, data, off, n = bench.make_superblock(fixture=bench.FIXTURE3)
    o = orc.Oracle(orc.RunConfig(**bench.MODEL3))
    ref, _sec, _flops = o.hpsi_flat(sl, el, ints, data, n)
    del o
    ctx = Context(device=0, **bench.MODEL3)
    try:
        ctx.set_superblock_flat(sl, el, ints, data)
        out = ctx.model_wave(data[off:off + n])
    finally:
        ctx.close()
    assert float(np.max(np.abs(out - ref)) / np.max(np.abs(ref))) <= 1e-13
