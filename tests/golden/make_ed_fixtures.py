"""Exact-diagonalisation known answers for the t1-t2-J1-J2 model on small
triangular cylinders, plus sympy Wigner-6j values.

These pin the oracle's physics where the reference itself cannot run (no Fortran
compiler): a DMRG that keeps every multiplet must reproduce the lowest S=0
energy of the full many-body Hamiltonian

    H = sum_<ij> [ -t_ij sum_s (c+_is c_js + h.c.) + J_ij (S_i.S_j - n_i n_j / 4) ]

on the same lattice, and its ground-state measurements the reference computes
(main.f90:259-299): site densities <n_a>, the correlation matrices <n_a n_b>,
<S_a . S_b> and sum_s <c+_as c_bs>, and singlet pair correlations <O+_ab O_cd>
over nearest-neighbour bonds.  Lattice (restating dmrg_sub.f90:453-583): sites
i = (x-1)*Ny + y, periodic in y, open in x; nearest neighbours along (0,1),
(1,0), (1,-1) carry (t1, J1); next-nearest along (1,1), (2,-1), (1,-2) carry
(t2, J2).  Electron count from main.f90:93-99.  Run:  python make_ed_fixtures.py
"""
from __future__ import annotations

import itertools
import json
import os

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as sla


def bonds(Nx, Ny):
    def idx(x, y):
        return (x - 1) * Ny + ((y - 1) % Ny) + 1
    nn, nnn = set(), set()
    for x in range(1, Nx + 1):
        for y in range(1, Ny + 1):
            i = idx(x, y)
            for dx, dy, kind in [(0, 1, 1), (1, 0, 1), (1, -1, 1), (1, 1, 2), (2, -1, 2), (1, -2, 2)]:
                if x + dx > Nx:
                    continue
                j = idx(x + dx, y + dy)
                if j == i:
                    continue
                b = (min(i, j), max(i, j))
                (nn if kind == 1 else nnn).add(b)
    nnn -= nn
    return sorted(nn), sorted(nnn)


def n_electrons(ns, delta=12):
    return 2 * (ns // 2 - (ns + 2 * delta - 1) // (2 * delta))


def tj_ground_state(Nx, Ny, t1, t2, J1, J2, sign_t=-1.0, penalty=10.0):
    ns = Nx * Ny
    ne = n_electrons(ns)
    nup = ne // 2
    # basis: (up mask, down mask), no double occupancy, Sz = 0
    states = []
    for occ in itertools.combinations(range(ns), ne):
        for ups in itertools.combinations(occ, nup):
            um = sum(1 << q for q in ups)
            dm = sum(1 << q for q in occ) ^ um
            states.append((um, dm))
    index = {s: k for k, s in enumerate(states)}
    nn, nnn = bonds(Nx, Ny)
    blist = [(i - 1, j - 1, t1, J1) for i, j in nn] + [(i - 1, j - 1, t2, J2) for i, j in nnn]

    # fermion ordering: modes (site, spin) -> 2*site + spin
    def occ_modes(um, dm):
        m = 0
        for q in range(ns):
            if (um >> q) & 1:
                m |= 1 << (2 * q)
            if (dm >> q) & 1:
                m |= 1 << (2 * q + 1)
        return m

    def hop_sign(mode_mask, a, b):
        lo, hi = min(a, b), max(a, b)
        between = mode_mask & (((1 << hi) - 1) ^ ((1 << (lo + 1)) - 1))
        return -1.0 if bin(between).count("1") % 2 else 1.0

    rows, cols, vals = [], [], []
    srows, scols, svals = [], [], []
    for k, (um, dm) in enumerate(states):
        mm = occ_modes(um, dm)
        diag = 0.0
        for i, j, t, J in blist:
            ni = ((um >> i) | (dm >> i)) & 1
            nj = ((um >> j) | (dm >> j)) & 1
            szi = 0.5 * (((um >> i) & 1) - ((dm >> i) & 1))
            szj = 0.5 * (((um >> j) & 1) - ((dm >> j) & 1))
            diag += J * (szi * szj - 0.25 * ni * nj)
            # spin flip S+_i S-_j + S-_i S+_j (no fermion sign for a swap of adjacent spins of one pair)
            if ni and nj and (((um >> i) & 1) != ((um >> j) & 1)) and J != 0.0:
                num, ndm = um ^ (1 << i) ^ (1 << j), dm ^ (1 << i) ^ (1 << j)
                # express as c+_{i s'} c_{i s} c+_{j s} c_{j s'} with explicit Jordan-Wigner signs
                s_i = 0 if (um >> i) & 1 else 1
                s_j = 1 - s_i
                m1 = mm
                sg = 1.0
                for (ann, cre) in [(2 * j + s_j, 2 * j + s_i), (2 * i + s_i, 2 * i + s_j)]:
                    sg *= hop_sign(m1, ann, cre)
                    m1 = (m1 ^ (1 << ann)) | (1 << cre)
                rows.append(index[(num, ndm)]); cols.append(k); vals.append(0.5 * J * sg)
            # hopping
            if t != 0.0:
                for s, msk in ((0, um), (1, dm)):
                    for a, b in ((i, j), (j, i)):
                        if ((msk >> b) & 1) and not (((um >> a) | (dm >> a)) & 1):
                            ma, mb = 2 * a + s, 2 * b + s
                            sg = hop_sign(mm, mb, ma)
                            if s == 0:
                                nstate = (um ^ (1 << a) ^ (1 << b), dm)
                            else:
                                nstate = (um, dm ^ (1 << a) ^ (1 << b))
                            rows.append(index[nstate]); cols.append(k); vals.append(sign_t * t * sg)
        rows.append(k); cols.append(k); vals.append(diag)
        # total S^2 = (Sz)^2 + (S+S- + S-S+)/2 ; Sz = 0 here -> S^2 = sum_ij (Sz_i Sz_j + (S+_i S-_j + h.c.)/2)
        sz = [0.5 * (((um >> q) & 1) - ((dm >> q) & 1)) for q in range(ns)]
        s2d = sum(sz[a] * sz[b] for a in range(ns) for b in range(ns))
        s2d += sum(0.5 for q in range(ns) if ((um | dm) >> q) & 1)   # S+_i S-_i + S-_i S+_i halves on site
        srows.append(k); scols.append(k); svals.append(s2d)
        for a in range(ns):
            for b in range(ns):
                if a == b:
                    continue
                if ((um >> b) & 1) and ((dm >> a) & 1):   # S+_a S-_b : a down->up, b up->down
                    num, ndm = um ^ (1 << a) ^ (1 << b), dm ^ (1 << a) ^ (1 << b)
                    m1, sg = mm, 1.0
                    for (ann, cre) in [(2 * b, 2 * b + 1), (2 * a + 1, 2 * a)]:
                        sg *= hop_sign(m1, ann, cre)
                        m1 = (m1 ^ (1 << ann)) | (1 << cre)
                    srows.append(index[(num, ndm)]); scols.append(k); svals.append(sg)
    n = len(states)
    H = sp.csr_matrix((vals, (rows, cols)), shape=(n, n))
    S2 = sp.csr_matrix((svals, (srows, scols)), shape=(n, n))
    Hp = H + penalty * S2
    w, v = sla.eigsh(Hp, k=1, which="SA", tol=1e-13, maxiter=100000)
    e = float(w[0])
    s2 = float(np.real(v[:, 0].conj() @ (S2 @ v[:, 0])))
    # site densities <n_q> of the ground state (site q+1 in the lattice numbering)
    p = np.abs(v[:, 0]) ** 2
    dens = [float(sum(p[k] for k, (um, dm) in enumerate(states) if ((um | dm) >> q) & 1)) for q in range(ns)]
    # density-density correlations <n_a n_b> (row a, column b; sites a+1, b+1)
    occ = np.array([[((um | dm) >> q) & 1 for q in range(ns)] for (um, dm) in states], dtype=np.float64)
    ncor = (occ.T * p) @ occ
    # spin-spin correlations <S_a . S_b> = <Sz_a Sz_b> + (<S+_a S-_b> + <S+_b S-_a>) / 2,
    # diagonal 3/4 <n_a>; their sum is <S^2> = 0 for the S=0 ground state
    vg = v[:, 0]
    szm = np.array([[0.5 * (((um >> q) & 1) - ((dm >> q) & 1)) for q in range(ns)] for (um, dm) in states])
    flip = np.zeros((ns, ns))
    for k, (um, dm) in enumerate(states):
        mm = occ_modes(um, dm)
        for a in range(ns):
            if not (dm >> a) & 1:
                continue
            for b in range(ns):
                if a == b or not (um >> b) & 1:
                    continue
                # S+_a S-_b: b up -> down, then a down -> up
                num, ndm = um ^ (1 << a) ^ (1 << b), dm ^ (1 << a) ^ (1 << b)
                m1, sg = mm, 1.0
                for (ann, cre) in [(2 * b, 2 * b + 1), (2 * a + 1, 2 * a)]:
                    sg *= hop_sign(m1, ann, cre)
                    m1 = (m1 ^ (1 << ann)) | (1 << cre)
                flip[a, b] += float(np.real(np.conj(vg[index[(num, ndm)]]) * sg * vg[k]))
    scor = (szm.T * p) @ szm + 0.5 * (flip + flip.T)
    np.fill_diagonal(scor, 0.75 * np.array(dens))
    # one-particle correlations G_ab = sum_s <c+_{a s} c_{b s}> (diagonal <n_a>)
    ecor = np.zeros((ns, ns))
    for k, (um, dm) in enumerate(states):
        mm = occ_modes(um, dm)
        for s, msk in ((0, um), (1, dm)):
            for b in range(ns):
                if not (msk >> b) & 1:
                    continue
                for a in range(ns):
                    if a == b or (((um >> a) | (dm >> a)) & 1):
                        continue
                    sg = hop_sign(mm, 2 * b + s, 2 * a + s)
                    nstate = (um ^ (1 << a) ^ (1 << b), dm) if s == 0 else (um, dm ^ (1 << a) ^ (1 << b))
                    ecor[a, b] += float(np.real(np.conj(vg[index[nstate]]) * sg * vg[k]))
    np.fill_diagonal(ecor, np.array(dens))
    # singlet pair correlations <O+_ab O_cd> over the nearest-neighbour bonds,
    # O+_ab = (c+_{a up} c+_{b dn} - c+_{a dn} c+_{b up}) / sqrt(2); O_cd |psi> is
    # kept as a sparse vector of (N-2)-electron mode masks
    def annihilate(m, mode):
        if not (m >> mode) & 1:
            return None, 0.0
        return m ^ (1 << mode), (-1.0 if bin(m & ((1 << mode) - 1)).count("1") % 2 else 1.0)

    bonds_nn = sorted({(min(i, j) - 1, max(i, j) - 1) for i, j in nn})
    opsi = []
    for (a, b) in bonds_nn:
        w = {}
        for k, (um, dm) in enumerate(states):
            m = occ_modes(um, dm)
            # O_ab = (c_{b dn} c_{a up} - c_{b up} c_{a dn}) / sqrt(2)
            for (m1, m2, c) in ((2 * a, 2 * b + 1, 1.0), (2 * a + 1, 2 * b, -1.0)):
                x, s1 = annihilate(m, m1)
                if x is None:
                    continue
                y, s2 = annihilate(x, m2)
                if y is None:
                    continue
                w[y] = w.get(y, 0.0) + c * s1 * s2 * float(np.real(vg[k])) / np.sqrt(2.0)
        opsi.append(w)
    pcor = [[sum(wx.get(key, 0.0) * val for key, val in wy.items()) for wy in opsi] for wx in opsi]
    return {"Nx": Nx, "Ny": Ny, "t1": t1, "t2": t2, "J1": J1, "J2": J2, "n_sites": ns,
            "n_electrons": ne, "dim": n, "e0_S0": e - penalty * s2, "S2": s2, "sign_t": sign_t,
            "density": dens, "density_cor": ncor.tolist(), "spin_cor": scor.tolist(),
            "elec_cor": ecor.tolist(), "pair_bonds": [[a + 1, b + 1] for a, b in bonds_nn],
            "pair_cor": pcor}


def main():
    out = {"ed": [], "w6j": []}
    cases = [(2, 4, 1.0, 0.0, 0.4, 0.0), (2, 4, 1.0, 0.3, 0.4, 0.036), (3, 4, 1.0, 0.0, 0.4, 0.0),
             (3, 4, 1.0, 0.3, 0.4, 0.036)]
    for c in cases:
        r = tj_ground_state(*c)
        print(r)
        out["ed"].append(r)
    from sympy.physics.wigner import wigner_6j
    from sympy import Rational
    rng = np.random.default_rng(7)
    count = 0
    while count < 60:
        j = [int(x) for x in rng.integers(0, 9, size=6)]
        try:
            val = wigner_6j(*[Rational(x, 2) for x in j])
        except ValueError:   # sympy rejects non-triangular arguments; the symbol is zero
            val = 0
        if val == 0 and rng.random() < 0.8:
            continue
        out["w6j"].append({"args2": j, "value": float(val)})
        count += 1
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ed_and_6j.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    main()
