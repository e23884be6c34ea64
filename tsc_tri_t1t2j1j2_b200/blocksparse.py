"""Block-sparse H.psi problems for tsc_blocksparse_set (layout in include/tsc_gpu.h)
and the seeded synthetic workload of the benchmark list.

A problem has K sectors (psi sector i: d_i x e_i), left operator sets (shift s,
blocks L[i] of d_{i+s} x d_i), right sets (shift s, blocks R[i] of e_{i+s} x e_i)
and terms (alpha, a, b) adding alpha * L_a[i] X_i R_b[i]^H to Y_{i+s}.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Problem:
    d: list[int]
    e: list[int]
    left: list[tuple[int, list]] = field(default_factory=list)    # (shift, [block or None per sector])
    right: list[tuple[int, list]] = field(default_factory=list)
    terms: list[tuple[complex, int, int]] = field(default_factory=list)

    @property
    def K(self):
        return len(self.d)

    def psi_len(self):
        return int(sum(int(a) * int(b) for a, b in zip(self.d, self.e)))


def pack(problems):
    """-> (nproblems, int32 descriptors, complex128 data)."""
    ints, chunks = [], []
    for P in problems:
        ints += [P.K, len(P.left), len(P.right), len(P.terms)]
        for a, b in zip(P.d, P.e):
            ints += [int(a), int(b)]
        ints += [s for s, _ in P.left] + [s for s, _ in P.right]
        for _, a, b in P.terms:
            ints += [a, b]
        for sets, dims in ((P.left, P.d), (P.right, P.e)):
            for s, blocks in sets:
                for i in range(P.K):
                    j = i + s
                    if 0 <= j < P.K:
                        blk = np.asarray(blocks[i], np.complex128)
                        assert blk.shape == (dims[j], dims[i])
                        chunks.append(blk.ravel(order="F"))
        chunks.append(np.array([t[0] for t in P.terms], np.complex128))
    data = np.concatenate(chunks) if chunks else np.zeros(0, np.complex128)
    return len(problems), np.asarray(ints, np.int32), data


def synthetic(rng, K, dmin, dmax, n_left=8, n_right=8, n_terms=200, shifts=(-2, -1, 0, 1, 2)):
    """The benchmark list's synthetic H.psi: sector dimensions log-uniform in
    [dmin, dmax], entries re/im i.i.d. N(0,1), square blocks of shift 0
    Hermitised, n_terms terms with alpha ~ U[-1, 1] drawn from pools of
    n_left / n_right operator sets whose shifts come from `shifts` (a term
    pairs a left and a right set of equal shift)."""
    d = np.exp(rng.uniform(np.log(dmin), np.log(dmax), K)).astype(int).tolist()
    e = np.exp(rng.uniform(np.log(dmin), np.log(dmax), K)).astype(int).tolist()
    P = Problem(d=d, e=e)
    ls = [int(rng.choice(shifts)) for _ in range(n_left)]
    # every left shift has at least one right set of the same shift
    rs = [ls[k % n_left] for k in range(n_right)]

    def blocks(s, dims):
        out = []
        for i in range(K):
            j = i + s
            if not 0 <= j < K:
                out.append(None)
                continue
            b = rng.standard_normal((dims[j], dims[i])) + 1j * rng.standard_normal((dims[j], dims[i]))
            if s == 0:
                b = 0.5 * (b + b.conj().T)
            out.append(b)
        return out

    P.left = [(s, blocks(s, d)) for s in ls]
    P.right = [(s, blocks(s, e)) for s in rs]
    by_shift = {}
    for b, s in enumerate(rs):
        by_shift.setdefault(s, []).append(b)
    for _ in range(n_terms):
        a = int(rng.integers(n_left))
        b = int(rng.choice(by_shift[ls[a]]))
        P.terms.append((complex(rng.uniform(-1.0, 1.0)), a, b))
    return P


def synthetic_packed(rng, K, dmin, dmax, n_left=8, n_right=8, n_terms=200, shifts=(-2, -1, 0, 1, 2)):
    """synthetic() for one problem written straight into pack()'s layout: the same
    random draws in the same order, so (1, ints, data) equals
    pack([synthetic(rng, ...)]) for the same generator state, without holding
    the blocks twice (K = 400 operator sets take ~45 GB).  Returns (Problem with
    dims, shifts and terms but no blocks, ints, data)."""
    d = np.exp(rng.uniform(np.log(dmin), np.log(dmax), K)).astype(int).tolist()
    e = np.exp(rng.uniform(np.log(dmin), np.log(dmax), K)).astype(int).tolist()
    P = Problem(d=d, e=e)
    ls = [int(rng.choice(shifts)) for _ in range(n_left)]
    rs = [ls[k % n_left] for k in range(n_right)]
    sizes = [dims[i + s_] * dims[i] for s_, dims in [(s_, d) for s_ in ls] + [(s_, e) for s_ in rs]
             for i in range(K) if 0 <= i + s_ < K]
    data = np.empty(int(sum(sizes)) + n_terms, np.complex128)
    pos = 0
    for s_, dims in [(s_, d) for s_ in ls] + [(s_, e) for s_ in rs]:
        for i in range(K):
            j = i + s_
            if not 0 <= j < K:
                continue
            b = rng.standard_normal((dims[j], dims[i])) + 1j * rng.standard_normal((dims[j], dims[i]))
            if s_ == 0:
                b = 0.5 * (b + b.conj().T)
            data[pos:pos + b.size] = b.ravel(order="F")
            pos += b.size
    P.left = [(s_, None) for s_ in ls]
    P.right = [(s_, None) for s_ in rs]
    by_shift = {}
    for bi, s_ in enumerate(rs):
        by_shift.setdefault(s_, []).append(bi)
    for _ in range(n_terms):
        a = int(rng.integers(n_left))
        bb = int(rng.choice(by_shift[ls[a]]))
        P.terms.append((complex(rng.uniform(-1.0, 1.0)), a, bb))
    data[pos:] = [t[0] for t in P.terms]
    ints = [K, n_left, n_right, n_terms]
    for x, y in zip(d, e):
        ints += [int(x), int(y)]
    ints += ls + rs
    for _, a, bb in P.terms:
        ints += [a, bb]
    return P, np.asarray(ints, np.int32), data


def random_psi(rng, problems):
    n = sum(P.psi_len() for P in problems)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    return (x / np.linalg.norm(x)).astype(np.complex128)
