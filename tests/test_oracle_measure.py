"""Site densities and two-point correlations of the oracle (measure_operator_dia
and Get_density_cor restated) against exact
diagonalisation: <n_i> of the S=0 ground state of YC4x2 and YC4x3 with and
without t2/J2 (tests/golden/ed_and_6j.json, make_ed_fixtures.py), DMRG keeping
every multiplet.  Tolerance 1e-8 per site (Lanczos stops at lanzero 1e-12);
the densities sum to the electron number to 1e-10."""
import json
import os

import numpy as np
import pytest

import orc

FIX = os.path.join(os.path.dirname(__file__), "golden", "ed_and_6j.json")
CASES = json.load(open(FIX))["ed"]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"YC4x{c['Nx']}_t2{c['t2']}")
def test_density_matches_ed(case):
    cfg = orc.RunConfig(Nx=case["Nx"], Ny=4, t1=1.0, t2=case["t2"], J1=0.4, J2=case["J2"], kept_min=400,
                        kept_warm=400, sweeps=[400, 400], lanzero=1e-12)
    o = orc.Oracle(cfg)
    o.run()
    dens = o.measure_density()
    assert np.max(np.abs(dens - np.array(case["density"]))) <= 1e-8
    assert abs(dens.sum() - case["n_electrons"]) <= 1e-10


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"YC4x{c['Nx']}_t2{c['t2']}")
def test_correlations_match_ed(case):
    """<n_i n_j>, <S_i . S_j> and sum_s <c+_is c_js> of Get_density_cor restated
    (num_elec, main.f90:299; st_sd, main.f90:275: rank 1, scaled by -sqrt(3) as
    measure.f90:2586-2587 and 2662-2663 do; st_elec_up and st_elec_down with
    Flags 'F', main.f90:288: rank 1/2, scaled by sqrt(2), fermion parity signs),
    after the final half sweep to 5 Num_site / 6 (main.f90:205-206),
    against the ED correlation matrices.  Sites 1-4 reach all four partner kinds
    (inside the system block through the product at the partner's length, the
    system site, the environment site, the environment block).  Tolerance 1e-8 on
    the real part and on the imaginary part (rounding noise of the complex wave)."""
    cfg = orc.RunConfig(Nx=case["Nx"], Ny=4, t1=1.0, t2=case["t2"], J1=0.4, J2=case["J2"], kept_min=400,
                        kept_warm=400, sweeps=[400, 400], lanzero=1e-12, final_half_sweep=True)
    o = orc.Oracle(cfg)
    o.run()
    n = case["n_sites"]
    for name, get in (("density_cor", o.density_cor), ("spin_cor", o.spin_cor), ("elec_cor", o.elec_cor)):
        ed = np.array(case[name])
        for site in (1, 2, 3, 4):
            row = get(site)
            partners = [j for j in range(site + 4, n + 1, 4)]
            assert partners, "no partner on the leg"
            for j in range(1, n + 1):
                if j in partners:
                    assert abs(row[j - 1].real - ed[site - 1, j - 1]) <= 1e-8, (name, site, j)
                    assert abs(row[j - 1].imag) <= 1e-8
                else:
                    assert row[j - 1] == 0


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"YC4x{c['Nx']}_t2{c['t2']}")
def test_pair_cor_matches_ed(case):
    """Singlet pair correlations <O+_ab O_cd>, O+_ab = (c+_{a up} c+_{b dn} -
    c+_{a dn} c+_{b up}) / sqrt(2), of Get_mSCOP_Operator_Cor0 restated (Flags 'S0',
    main.f90:259-262) against ED over nearest-neighbour bonds, for first bonds
    (xc1, neib(xc1, 1|3|5)), xc1 = 1..4.  At the reference's measuring position
    (after the final half sweep to 5 Num_site / 6) the second bonds lie in the
    system block (Get_sys_two1); with the half sweep stopped at Num_site / 2 some
    lie in the environment block (Get_SCOP_Operator_Env and the block-block
    correlator).  Tolerance 1e-8."""
    n = case["n_sites"]
    bonds = {tuple(b): i for i, b in enumerate(case["pair_bonds"])}
    ed = np.array(case["pair_cor"])
    stops = [0] if case["Nx"] == 2 else [0, n // 2 - 1]
    for stop in stops:
        cfg = orc.RunConfig(Nx=case["Nx"], Ny=4, t1=1.0, t2=case["t2"], J1=0.4, J2=case["J2"], kept_min=400,
                            kept_warm=400, sweeps=[400, 400], lanzero=1e-12, final_half_sweep=True, final_stop=stop)
        o = orc.Oracle(cfg)
        o.run()
        recs = []
        for xc1 in (1, 2, 3, 4):
            for ij1 in (1, 3, 5):
                try:
                    recs += o.pair_cor(xc1, n, 0, ij1)
                except RuntimeError:   # first bond outside the system block of this wave
                    pass
        assert recs
        if stop:
            assert any(max(c, d) > n // 2 + 1 for _, _, c, d, _ in recs), "no environment-block partner"
        for a, b, c, d, v in recs:
            ref = ed[bonds[(min(a, b), max(a, b))], bonds[(min(c, d), max(c, d))]]
            assert abs(v.real - ref) <= 1e-8 and abs(v.imag) <= 1e-8, (stop, a, b, c, d)
