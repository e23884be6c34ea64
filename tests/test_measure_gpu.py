"""Site densities <n_i> measured on the device after a whole run
(tsc_measure_density) against the oracle's measure_operator_dia.

FP64 form at lanzero 1e-10, where the run follows the oracle's step by step:
<= 1e-11 per site.  Split form at lanzero 1e-13 against the oracle at the same
lanzero: <= 1e-7 per site (a density is first order in the difference of the
two ground-state vectors, ~1e-8 measured).  Both sum to N_e to 1e-10."""
import numpy as np
import pytest

import orc
from tsc_tri_t1t2j1j2_b200 import Context

RUN = dict(kept_min=60, kept_warm=60, sweeps=[60, 80])


def oracle_density(lanzero):
    cfg = orc.RunConfig(Nx=4, Ny=4, t1=1.0, t2=0.3, J1=0.4, J2=0.036, lanzero=lanzero, **RUN)
    o = orc.Oracle(cfg)
    o.run()
    return o.measure_density()


@pytest.mark.gpu
@pytest.mark.parametrize("mode,lanzero,tol", [(Context.FP64, 1e-10, 1e-11), (Context.SPLIT_BF16, 1e-13, 1e-7)])
def test_density_matches_oracle(mode, lanzero, tol):
    ref = oracle_density(lanzero)
    ctx = Context(4, 4, 1.0, 0.3, 0.4, 0.036)
    try:
        ctx.set_precision(mode, 1e-11)
        ctx.get_ground_state(lanzero=lanzero, **RUN)
        dens = ctx.measure_density()
    finally:
        ctx.close()
    assert np.max(np.abs(dens - ref)) <= tol
    assert abs(dens.sum() - round(ref.sum())) <= 1e-10


def oracle_density_cor(lanzero, sites):
    cfg = orc.RunConfig(Nx=4, Ny=4, t1=1.0, t2=0.3, J1=0.4, J2=0.036, lanzero=lanzero, final_half_sweep=True, **RUN)
    o = orc.Oracle(cfg)
    o.run()
    return {s: o.density_cor(s).real for s in sites}


@pytest.mark.gpu
@pytest.mark.parametrize("mode,lanzero,tol", [(Context.FP64, 1e-10, 1e-11), (Context.SPLIT_BF16, 1e-13, 1e-7)])
def test_density_cor_matches_oracle(mode, lanzero, tol):
    """tsc_measure_density_cor after the final half sweep (YC4x4: the wave ends at
    sys_len 13) for sites 1-4, whose partners cover the four kinds of
    Get_density_cor, against the oracle's restatement; tolerances as for <n_i>."""
    sites = (1, 2, 3, 4)
    ref = oracle_density_cor(lanzero, sites)
    ctx = Context(4, 4, 1.0, 0.3, 0.4, 0.036)
    try:
        ctx.set_precision(mode, 1e-11)
        ctx.get_ground_state(lanzero=lanzero, final_half_sweep=True, **RUN)
        got = {s: ctx.measure_density_cor(s) for s in sites}
    finally:
        ctx.close()
    for s in sites:
        assert np.count_nonzero(ref[s]) >= 3
        assert np.max(np.abs(got[s] - ref[s])) <= tol, s
        assert np.array_equal(got[s] == 0, ref[s] == 0)


def oracle_correlations(lanzero, sites):
    cfg = orc.RunConfig(Nx=4, Ny=4, t1=1.0, t2=0.3, J1=0.4, J2=0.036, lanzero=lanzero, final_half_sweep=True, **RUN)
    o = orc.Oracle(cfg)
    o.run()
    out = {}
    for kind, get in (("density", o.density_cor), ("spin", o.spin_cor), ("electron", o.elec_cor)):
        out[kind] = {s: get(s) for s in sites}
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("mode,lanzero,tol", [(Context.FP64, 1e-10, 1e-11), (Context.SPLIT_BF16, 1e-13, 3e-7)])
def test_spin_and_electron_cor_match_oracle(mode, lanzero, tol):
    """tsc_measure_correlation for the spin (st_sd x st_sd, rank 1, 'B') and
    electron (st_elec_up x st_elec_down, rank 1/2, 'F') correlations after the
    final half sweep, sites 1-4 (partners inside the system block, on its added
    site, on the environment's added site and inside the environment block),
    complex, against the oracle's oper_cor: FP64 <= 1e-11; split <= 3e-7 (first
    order in the ground-state difference like <n_i>; the spin operator's
    reduced elements are sqrt(3) larger, 1.1e-7 measured); the density kind
    equals tsc_measure_density_cor."""
    sites = (1, 2, 3, 4)
    ref = oracle_correlations(lanzero, sites)
    ctx = Context(4, 4, 1.0, 0.3, 0.4, 0.036)
    try:
        ctx.set_precision(mode, 1e-11)
        ctx.get_ground_state(lanzero=lanzero, final_half_sweep=True, **RUN)
        got = {k: {s: ctx.measure_correlation(k, s) for s in sites} for k in ("density", "spin", "electron")}
        dens = {s: ctx.measure_density_cor(s) for s in sites}
    finally:
        ctx.close()
    for s in sites:
        assert np.array_equal(got["density"][s].real, dens[s]) and not got["density"][s].imag.any()
        for kind in ("spin", "electron"):
            r, g = ref[kind][s], got[kind][s]
            assert np.count_nonzero(r) >= 3, (kind, s)
            assert np.max(np.abs(g - r)) <= tol, (kind, s, np.max(np.abs(g - r)))
            assert np.array_equal(g == 0, r == 0), (kind, s)


@pytest.mark.gpu
@pytest.mark.parametrize("stop", [0, 7])
def test_pair_cor_matches_oracle(stop):
    """tsc_measure_pair_correlation (Get_mSCOP_Operator_Cor0, Flags 'S0') in the
    FP64 form against the oracle's pair_cor on YC4x4, first bonds (xc1,
    neib(xc1, 1|3|5)) for xc1 = 1..4.  stop 0 ends the final half sweep where
    the reference measures (second bonds in the system block, Get_sys_two1);
    stop 7 = Num_site/2 - 1 leaves some second bonds in the environment block
    (Get_SCOP_Operator_Env and the block-block correlator).  Same records in the
    same order, values within 1e-11."""
    n = 16
    cfg = orc.RunConfig(Nx=4, Ny=4, t1=1.0, t2=0.3, J1=0.4, J2=0.036, lanzero=1e-10, final_half_sweep=True,
                        final_stop=stop, **RUN)
    o = orc.Oracle(cfg)
    o.run()
    ctx = Context(4, 4, 1.0, 0.3, 0.4, 0.036)
    try:
        ctx.get_ground_state(lanzero=1e-10, final_half_sweep=True, final_stop=stop, **RUN)
        nrec = 0
        env_partner = False
        for xc1 in (1, 2, 3, 4):
            for ij1 in (1, 3, 5):
                try:
                    ref = o.pair_cor(xc1, n, 0, ij1)
                except RuntimeError:   # first bond outside the system block of this wave
                    with pytest.raises(Exception):
                        ctx.measure_pair_correlation(xc1, n, 0, ij1)
                    continue
                got = ctx.measure_pair_correlation(xc1, n, 0, ij1)
                assert [g[:4] for g in got] == [tuple(int(x) for x in r[:4]) for r in ref], (xc1, ij1)
                for g, r in zip(got, ref):
                    assert abs(g[4] - r[4]) <= 1e-11, (xc1, ij1, g, r)
                    env_partner |= max(g[2], g[3]) > n // 2 + 1
                nrec += len(got)
    finally:
        ctx.close()
    assert nrec > 0
    if stop:
        assert env_partner
