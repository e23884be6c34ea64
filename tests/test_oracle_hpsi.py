"""Self-consistency of the oracle's H.psi on captured superblocks: H is Hermitian
in the superblock basis and the Lanczos energy is the Rayleigh quotient of the
returned ground state (eigen.f90:137-156)."""
import numpy as np
import pytest

import orc
from _capture import parse_oracle_capture
from tsc_tri_t1t2j1j2_b200.layout import pack


@pytest.fixture(scope="module")
def cap():
    cfg = orc.RunConfig(Nx=4, Ny=4, t2=0.3, J2=0.036, kept_min=40, kept_warm=40, sweeps=[40], lanzero=1e-11)
    o = orc.Oracle(cfg, capture_step=9)
    o.run()
    return o, parse_oracle_capture(*o.capture())


def hpsi(o, c, vec):
    ints, data = [], []
    c["sys"].write(ints, data)
    c["env"].write(ints, data)
    c["sys_bs"].write(ints, data)
    c["env_bs"].write(ints, data)
    w = c["psi0"]
    w.vec = vec
    w.write(ints, data)
    i, d = pack(ints, data)
    out, _, flops = o.hpsi_flat(c["sys"].len, c["env"].len, i, d, len(vec))
    return out, flops


def test_hpsi_reproduces_capture(cap):
    o, c = cap
    out, flops = hpsi(o, c, c["psi0"].vec.copy())
    assert np.max(np.abs(out - c["hpsi"].vec)) <= 1e-14 * np.max(np.abs(out))
    assert flops > 0


def test_hamiltonian_is_hermitian(cap):
    o, c = cap
    rng = np.random.default_rng(5)
    n = len(c["psi0"].vec)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    y = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    hx, _ = hpsi(o, c, x)
    hy, _ = hpsi(o, c, y)
    lhs, rhs = np.vdot(x, hy), np.vdot(hx, y)
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_lanczos_energy_is_rayleigh_quotient(cap):
    o, c = cap
    g = c["gs"].vec
    hg, _ = hpsi(o, c, g.copy())
    rq = np.vdot(g, hg).real / np.vdot(g, g).real
    assert abs(rq - c["e0"]) <= 1e-9 * abs(c["e0"])
