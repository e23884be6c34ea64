"""Block-sparse batch (tsc_blocksparse_set / tsc_blocksparse_apply): several
independent problems in one pair of launches, against a numpy evaluation of
sum_t alpha_t L_a[i] X_i R_b[i]^H.  Tolerances: FP64 max|dx|/max|x| <= 1e-13,
split form <= 2e-5."""
import numpy as np
import pytest

from tsc_tri_t1t2j1j2_b200 import Context
from tsc_tri_t1t2j1j2_b200.blocksparse import Problem, pack, random_psi, synthetic
from tsc_tri_t1t2j1j2_b200._lib import TscError


def apply_numpy(problems, x):
    y = np.zeros_like(x)
    base = 0
    for P in problems:
        offs = np.concatenate([[0], np.cumsum([a * b for a, b in zip(P.d, P.e)])]).astype(int) + base
        X = [x[offs[i]:offs[i + 1]].reshape(P.d[i], P.e[i], order="F") for i in range(P.K)]
        Y = [np.zeros((P.d[i], P.e[i]), complex) for i in range(P.K)]
        for alpha, a, b in P.terms:
            s = P.left[a][0]
            for i in range(P.K):
                j = i + s
                if 0 <= j < P.K:
                    Y[j] += alpha * P.left[a][1][i] @ X[i] @ P.right[b][1][i].conj().T
        for i in range(P.K):
            y[offs[i]:offs[i + 1]] = Y[i].ravel(order="F")
        base = offs[-1]
    return y


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def batch():
    rng = np.random.default_rng(11)
    probs = [synthetic(rng, K, 3, 70, n_left=4, n_right=5, n_terms=9) for K in (5, 3, 7, 1)]
    x = random_psi(rng, probs)
    return probs, x, apply_numpy(probs, x)


@pytest.mark.gpu
@pytest.mark.parametrize("mode,tol", [(Context.FP64, 1e-13), (Context.SPLIT_BF16, 2e-5)])
def test_blocksparse_batch(batch, mode, tol):
    import torch
    probs, x, ref = batch
    ctx = Context(3, 4)
    try:
        n, flops, xflops = ctx.blocksparse_set(probs)
        assert n == len(x) and 0 < xflops <= flops
        xd = torch.from_numpy(x).cuda()
        yd = torch.full_like(xd, complex(np.nan, np.nan))
        torch.cuda.synchronize()
        for _ in range(2):   # twice: the second call must not depend on the first
            ctx.blocksparse_apply(xd.data_ptr(), yd.data_ptr(), mode)
        torch.cuda.synchronize()
        assert rel(yd.cpu().numpy(), ref) <= tol
    finally:
        ctx.close()


@pytest.mark.gpu
def test_blocksparse_split_long_terms():
    """Split form with inner dimensions up to 700 (terms of up to 44 K steps,
    several accumulator segments each): the kernel breaks segments at every term
    and applies the term's coefficient in the epilogue (views shared by all terms
    of an operator); against numpy <= 2e-6 of the largest element, and the
    sliced operator views are no larger than one copy per operator block."""
    import torch
    rng = np.random.default_rng(5)
    probs = [synthetic(rng, 4, 200, 700, n_left=3, n_right=3, n_terms=12)]
    x = random_psi(rng, probs)
    ref = apply_numpy(probs, x)
    ctx = Context(3, 4)
    try:
        ctx.blocksparse_set(probs)
        xd = torch.from_numpy(x).cuda()
        yd = torch.empty_like(xd)
        ctx.blocksparse_apply(xd.data_ptr(), yd.data_ptr(), Context.SPLIT_BF16)
        torch.cuda.synchronize()
        assert rel(yd.cpu().numpy(), ref) <= 2e-6
        P = probs[0]
        elems = sum(b.size for _, blks in P.left + P.right for b in blks if b is not None)
        # 12 bytes per complex element in the six BF16 planes, tiles padded to 128 x 16 / 16 x 64
        assert ctx.split_views()["operators"][0] <= 12 * elems * 2.5
    finally:
        ctx.close()


@pytest.mark.gpu
def test_blocksparse_rejects_mismatched_shifts():
    rng = np.random.default_rng(3)
    P = synthetic(rng, 4, 3, 9, n_left=2, n_right=2, n_terms=2, shifts=(0,))
    P.right[1] = (1, [rng.standard_normal((P.e[i + 1], P.e[i])) if i + 1 < 4 else None for i in range(4)])
    P.terms.append((0.5 + 0j, 0, 1))
    ctx = Context(3, 4)
    try:
        with pytest.raises(TscError) as ei:
            ctx.blocksparse_set([P])
        assert ei.value.code == -2
    finally:
        ctx.close()
