"""Packing of block-sparse problems (tsc_blocksparse_set layout) and the
synthetic generator, on the CPU."""
import numpy as np

from tsc_tri_t1t2j1j2_b200.blocksparse import pack, random_psi, synthetic


def test_pack_lengths_and_layout():
    rng = np.random.default_rng(5)
    probs = [synthetic(rng, K, 2, 30, n_left=3, n_right=3, n_terms=7) for K in (4, 2)]
    nprob, ints, data = pack(probs)
    assert nprob == 2
    n_ints = sum(4 + 2 * P.K + len(P.left) + len(P.right) + 2 * len(P.terms) for P in probs)
    assert len(ints) == n_ints
    n_data = 0
    for P in probs:
        for sets, dims in ((P.left, P.d), (P.right, P.e)):
            for s, _ in sets:
                n_data += sum(dims[i + s] * dims[i] for i in range(P.K) if 0 <= i + s < P.K)
        n_data += len(P.terms)
    assert len(data) == n_data
    # header of the first problem, then its dimensions
    P = probs[0]
    assert list(ints[:4]) == [P.K, 3, 3, 7]
    assert list(ints[4:4 + 2 * P.K:2]) == list(P.d)
    # the alphas close each problem's data
    assert np.allclose(data[n_data - len(probs[1].terms):], [t[0] for t in probs[1].terms])


def test_synthetic_rules():
    rng = np.random.default_rng(9)
    P = synthetic(rng, 6, 16, 2048, n_terms=50)
    assert all(16 <= d <= 2048 for d in P.d + P.e)
    shifts_l = [s for s, _ in P.left]
    shifts_r = [s for s, _ in P.right]
    for _, a, b in P.terms:
        assert shifts_l[a] == shifts_r[b]
        assert -1.0 <= _.real <= 1.0
    for s, blocks in P.left:
        if s == 0:
            for b in blocks:
                assert np.allclose(b, b.conj().T)
    x = random_psi(rng, [P])
    assert len(x) == P.psi_len() and abs(np.linalg.norm(x) - 1) < 1e-12


def test_synthetic_packed_equals_pack_of_synthetic():
    """The packed generator (used for the K = 128..400 synthetic problems) draws
    the same numbers in the same order as synthetic() + pack()."""
    import numpy as np
    from tsc_tri_t1t2j1j2_b200.blocksparse import pack, synthetic, synthetic_packed
    for K in (1, 4, 11):
        n, ints, data = pack([synthetic(np.random.default_rng(K), K, 3, 50)])
        P, ints2, data2 = synthetic_packed(np.random.default_rng(K), K, 3, 50)
        assert n == 1 and np.array_equal(ints, ints2) and np.array_equal(data, data2)
        assert P.K == K and len(P.terms) == 200
