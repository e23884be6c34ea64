"""Split-precision form (BF16 slices on tcgen05, FP32 accumulation, Lanczos
finished in FP64) against the FP64 engine and the oracle, through the C-ABI.

Tolerances: split H.psi max|dx|/max|x| <= 2e-5 against the FP64 H.psi (three
BF16 slices, FP32 accumulators restarted every 128 of K and summed in FP64:
3.8e-7 on the random-valued YC4x12 m=1000 superblock); ground-state energy after the FP64
refinement |dE/E| <= 1e-10 against the oracle, for single solves and for the
last quarter of the steps of a full small run at lanzero = 1e-13.
"""
import numpy as np
import pytest

import orc
from _capture import parse_oracle_capture
from tsc_tri_t1t2j1j2_b200 import Context

SPLIT = Context.SPLIT_BF16


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module", params=[(4, 0.3, 0.036, 60, 6), (4, 0.3, 0.036, 120, 9), (4, 0.0, 0.0, 80, 22)],
                ids=lambda c: f"Nx{c[0]}_t2{c[1]}_m{c[3]}_s{c[4]}")
def captured(request):
    Nx, t2, J2, kept, step = request.param
    cfg = orc.RunConfig(Nx=Nx, Ny=4, t1=1.0, t2=t2, J1=0.4, J2=J2, kept_min=kept, kept_warm=kept,
                        sweeps=[kept], lanzero=1e-10)
    o = orc.Oracle(cfg, capture_step=step)
    o.run()
    cap = parse_oracle_capture(*o.capture())
    ctx = Context(Nx, 4, 1.0, t2, 0.4, J2)
    ctx.set_precision(SPLIT)
    ctx.set_superblock(cap["sys"], cap["env"], cap["sys_bs"], cap["env_bs"], cap["psi0"])
    yield cap, ctx
    ctx.close()


@pytest.mark.gpu
def test_split_hpsi_close_to_fp64(captured):
    cap, ctx = captured
    out = ctx.model_wave(cap["psi0"].vec)
    assert rel(out, cap["hpsi"].vec) <= 2e-5


@pytest.mark.gpu
def test_split_lanczos_energy(captured):
    cap, ctx = captured
    vec, e0, iters = ctx.lanczos_memo_new(cap["psi0"].vec, 1e-10)
    assert abs(e0 - cap["e0"]) <= 1e-10 * abs(cap["e0"])
    assert abs(abs(np.vdot(vec, cap["gs"].vec)) - 1.0) <= 1e-8


@pytest.mark.gpu
def test_split_hpsi_bench_superblock():
    """YC4x12 m=1000 superblock: the split H.psi with shared operator views
    (coefficients applied per term in the epilogue) and with one
    coefficient-folded view per term both within 1e-6 of FP64 (3.8e-7 measured);
    the shared views take less than a third of the folded ones' memory."""
    import bench
    sl, el, ints, data, off, n = bench.make_superblock()
    outs, views = [], []
    for mode, shared in ((Context.FP64, True), (SPLIT, True), (SPLIT, False)):
        ctx = Context(**bench.MODEL)
        try:
            ctx.set_precision(mode)
            ctx.set_split_view_sharing(shared)
            ctx.set_superblock_flat(sl, el, ints, data)
            outs.append(ctx.model_wave(data[off:off + n]))
            views.append(ctx.split_views()["operators"][0])
        finally:
            ctx.close()
    assert rel(outs[1], outs[0]) <= 1e-6
    assert rel(outs[2], outs[0]) <= 1e-6
    assert 0 < 3 * views[1] < views[2]


@pytest.mark.gpu
def test_split_full_run_energies():
    """A whole run in the split form against the oracle's.  The reference stops
    Lanczos when successive Ritz values agree to lanzero, which leaves its
    vectors about sqrt(lanzero/gap) from the eigenvector; a different (correct)
    solver then truncates a slightly different basis and the two runs drift
    apart by ~1e-9 at lanzero = 1e-10.  With lanzero = 1e-13 and the split
    solves finished to a Ritz residual of 0.1*sqrt(lanzero) the last quarter of
    the steps agree to better than 1e-10 relative (about 4e-11 measured); with
    the reference's stop for the FP64 finish (the default) the split vector
    keeps more of its BF16 error and the tail differs by ~2e-10."""
    cfg = orc.RunConfig(Nx=3, Ny=4, t1=1.0, t2=0.3, J1=0.4, J2=0.036, kept_min=40, kept_warm=40, sweeps=[40],
                        lanzero=1e-13)
    ref_steps = orc.Oracle(cfg).run()
    ctx = Context(3, 4, 1.0, 0.3, 0.4, 0.036)
    try:
        ctx.set_precision(SPLIT, 1e-11)
        ctx.set_split_refinement(0.1)
        steps = ctx.get_ground_state(kept_min=40, kept_warm=40, sweeps=[40], lanzero=1e-13)
    finally:
        ctx.close()
    assert len(steps) == len(ref_steps)
    assert sum(s["split_iters"] for s in steps) > 0
    tail = len(steps) // 4
    e = np.array([s["e0"] for s in steps])[-tail:]
    er = np.array([s["e0"] for s in ref_steps])[-tail:]
    assert np.max(np.abs(e - er) / np.abs(er)) <= 1e-10


@pytest.mark.gpu
def test_split_error_against_inner_dimension():
    """Error of one split product Y = X R^H (one sector, one term, the left
    operator the identity) against the inner dimension K, entries N(0,1).  A
    single FP32 accumulator in tensor memory loses a biased part of its last
    place on each MMA, so one long chain grows like K (5.5e-5 at K=4096 when
    all slice pairs shared one accumulator for the whole K).  With the (0,0)
    pair in its own accumulator and both restarted every few K steps, drained
    into FP64, the error stays flat: measured 5e-8 at K=16, 1.2e-7 at K=64 and
    2.3e-7 from K=256 to K=4096, as the same product rounded to nearest in
    FP32 (numpy complex64, 2.1e-7 to 2.7e-7).  Bounds: <= 5e-7 at K=16 and
    <= 1e-6 at K=4096."""
    import torch
    from tsc_tri_t1t2j1j2_b200.blocksparse import Problem
    rng = np.random.default_rng(5)
    errs = {}
    for K in (16, 4096):
        d = 32
        X = rng.normal(size=(d, K)) + 1j * rng.normal(size=(d, K))
        R = rng.normal(size=(K, K)) + 1j * rng.normal(size=(K, K))
        P = Problem(d=[d], e=[K], left=[(0, [np.eye(d, dtype=complex)])], right=[(0, [R])], terms=[(1.0 + 0j, 0, 0)])
        ref = X @ R.conj().T
        ctx = Context(3, 4)
        try:
            ctx.blocksparse_set([P])
            xd = torch.from_numpy(X.ravel(order="F").copy()).cuda()
            yd = torch.zeros_like(xd)
            ctx.blocksparse_apply(xd.data_ptr(), yd.data_ptr(), SPLIT)
            torch.cuda.synchronize()
            y = yd.cpu().numpy().reshape((d, K), order="F")
        finally:
            ctx.close()
        errs[K] = float(np.linalg.norm(y - ref) / np.linalg.norm(ref))
    assert errs[16] <= 5e-7
    assert errs[4096] <= 1e-6


@pytest.mark.gpu
def test_split_wait_timeout_is_reported_and_context_recovers(captured):
    """A bounded wait of the split kernel that runs out (poll limit 0: every wait
    gives up at once) comes back as TSC_E_CUDA from tsc_hpsi_device through the
    context's own status word; with the default limit restored the next call on
    the same context succeeds and matches the FP64 H.psi."""
    import torch
    from tsc_tri_t1t2j1j2_b200._lib import TscError
    cap, ctx = captured
    x = torch.from_numpy(cap["psi0"].vec.astype(np.complex128)).cuda()
    y = torch.zeros_like(x)
    torch.cuda.synchronize()
    ctx.set_split_wait_limit(0)
    try:
        with pytest.raises(TscError) as ei:
            ctx.hpsi_device(x.data_ptr(), y.data_ptr())
        assert ei.value.code == -3
        assert "bounded wait" in str(ei.value)
    finally:
        ctx.set_split_wait_limit(1 << 20)
    ctx.hpsi_device(x.data_ptr(), y.data_ptr())
    torch.cuda.synchronize()
    assert rel(y.cpu().numpy(), cap["hpsi"].vec) <= 2e-5


@pytest.mark.gpu
def test_split_renormalization_error(captured):
    """tsc_set_split_renormalization: Get_Hamiltonian_Sys/Env with U^H O U on the
    split kernel, against the same growth in FP64 (the oracle's renormalised
    model to 1e-12).  Every renormalised block within 2e-6 of the largest
    element of H, and not bit-equal (the split path ran); this error would stay
    in every later Hamiltonian, hence the FP64 default."""
    cap, ctx = captured
    side = 0 if cap["sys_side"] else 1
    pre = cap["sys"] if side == 0 else cap["env"]
    sys_len, env_len = cap["sys"].len, cap["env"].len
    mshift = 0 if side == 0 else (sys_len + 1)
    ctx.set_split_renormalization(True)
    try:
        grown = ctx.get_hamiltonian(side, pre, cap["grow_basis"], cap["trun"], sys_len, env_len, mshift)
    finally:
        ctx.set_split_renormalization(False)
    ref = cap["grown"]
    scale = max(np.max(np.abs(m)) for m in ref.ham.mats)
    err = max(np.max(np.abs(a - b), initial=0.0) for a, b in zip(grown.ham.mats, ref.ham.mats))
    for oa, ob in zip(grown.ops, ref.ops):
        for ba, bb in zip(oa, ob):
            for a, b in zip(ba.mats, bb.mats):
                err = max(err, float(np.max(np.abs(a - b), initial=0.0)))
    assert 0.0 < err <= 2e-6 * scale
