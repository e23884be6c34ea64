"""SU(2) coefficients of the oracle (W6JS / W3JS, block.f90:3702-3795) against sympy."""
import json
import os

import numpy as np
import pytest

import orc

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ed_and_6j.json")))


def test_w6js_matches_sympy_fixture():
    for w in GOLD["w6j"]:
        assert abs(orc.w6js(*w["args2"]) - w["value"]) <= 1e-13


def test_w3js_matches_sympy():
    from sympy import Rational
    from sympy.physics.wigner import wigner_3j
    rng = np.random.default_rng(3)
    n = 0
    while n < 40:
        j1, j2 = (int(x) for x in rng.integers(0, 7, 2))
        j3 = int(rng.integers(abs(j1 - j2), j1 + j2 + 1))
        if (j1 + j2 + j3) % 2:
            continue
        m1 = int(rng.choice(range(-j1, j1 + 1, 2)))
        m2 = int(rng.choice(range(-j2, j2 + 1, 2)))
        m3 = -m1 - m2
        if abs(m3) > j3:
            continue
        ref = float(wigner_3j(*[Rational(x, 2) for x in (j1, j2, j3, m1, m2, m3)]))
        assert abs(orc.w3js(j1, j2, j3, m1, m2, m3) - ref) <= 1e-13
        n += 1


@pytest.mark.parametrize("args", [(1, 1, 2, 1, 1, 0), (2, 2, 2, 1, 1, 1), (3, 1, 2, 1, 3, 2)])
def test_w6js_symmetry(args):
    a, b, c, d, e, f = args
    v = orc.w6js(a, b, c, d, e, f)
    assert abs(v - orc.w6js(b, a, c, e, d, f)) <= 1e-14   # column permutation
    assert abs(v - orc.w6js(d, e, c, a, b, f)) <= 1e-14   # swap upper/lower in two columns
