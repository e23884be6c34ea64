"""Site densities of the oracle (measure_operator_dia restated) against exact
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
def test_density_cor_matches_ed(case):
    """<n_i n_j> of Get_density_cor restated, after the final half sweep to
    5 Num_site / 6 (main.f90:205-206), against the ED correlation matrix.  Sites
    1-4 reach all four partner kinds (inside the system block through the
    product at the partner's length, the system site, the environment site, the
    environment block).  Tolerance 1e-8 as for <n_i>."""
    cfg = orc.RunConfig(Nx=case["Nx"], Ny=4, t1=1.0, t2=case["t2"], J1=0.4, J2=case["J2"], kept_min=400,
                        kept_warm=400, sweeps=[400, 400], lanzero=1e-12, final_half_sweep=True)
    o = orc.Oracle(cfg)
    o.run()
    ed = np.array(case["density_cor"])
    n = case["n_sites"]
    for site in (1, 2, 3, 4):
        row = o.density_cor(site)
        partners = [j for j in range(site + 4, n + 1, 4)]
        assert partners, "no partner on the leg"
        for j in range(1, n + 1):
            if j in partners:
                assert abs(row[j - 1].real - ed[site - 1, j - 1]) <= 1e-8, (site, j)
                assert abs(row[j - 1].imag) <= 1e-12
            else:
                assert row[j - 1] == 0
