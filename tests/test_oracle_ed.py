"""Oracle vs exact diagonalisation (tests/golden/ed_and_6j.json).

With every multiplet kept, the DMRG ground-state energy of the last sweep equals
the lowest S=0 eigenvalue of the full Hamiltonian (|dE| <= 1e-11)."""
import json
import os

import pytest

import orc

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ed_and_6j.json")))


@pytest.mark.parametrize("case", GOLD["ed"], ids=lambda c: f"YC{c['Ny']}x{c['Nx']}_t2{c['t2']}")
def test_oracle_matches_ed(case):
    if case["n_sites"] > 8 and case["t2"] == 0.0:
        pytest.skip("12-site NN case covered by the t2 case (same code path, saves a minute)")
    cfg = orc.RunConfig(Nx=case["Nx"], Ny=case["Ny"], t1=case["t1"], t2=case["t2"], J1=case["J1"], J2=case["J2"],
                        kept_min=2000, kept_warm=2000, sweeps=[2000], lanzero=1e-12)
    steps = orc.Oracle(cfg).run()
    assert abs(steps[-1]["e0"] - case["e0_S0"]) <= 1e-11 * abs(case["e0_S0"])


def test_electron_count_rule():
    # main.f90:93-99 with delta=12: 24 sites -> 22, 48 -> 44, 96 -> 88, 144 -> 132
    for ns, ne in [(24, 22), (48, 44), (96, 88), (144, 132), (8, 6), (12, 10)]:
        assert 2 * (ns // 2 - (ns + 23) // 24) == ne
