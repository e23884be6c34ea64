"""tsc_hpsi_noalloc (H.psi with its scratch in a fixed device array) against
tsc_hpsi_device and the oracle, through the C-ABI, in both precisions.

Two calls in a row on different inputs, then the first input again: each must
agree with tsc_hpsi_device on the same input to max|dx|/max|x| <= 1e-13 (the
same task lists run in the same order, so in practice bit for bit), and the
repeat must reproduce the first call exactly although the shared array still
holds the second call's contents.  Against the oracle's H.psi the FP64 form
agrees to 1e-13 and the split-precision form to 2e-5 (its documented
accuracy).  The device's free memory is the same before and after the
noalloc calls: the array was placed when the context was created.  A
superblock whose scratch exceeds the fixed maximum is rejected with
TSC_E_LIMIT.
"""
import numpy as np
import pytest

import orc
from _capture import parse_oracle_capture
from tsc_tri_t1t2j1j2_b200 import Context
from tsc_tri_t1t2j1j2_b200._lib import TscError

TSC_E_LIMIT = -6


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module", params=[(4, 0.3, 0.036, 60, 6, 0), (4, 0.3, 0.036, 120, 9, 0),
                                        (4, 0.3, 0.036, 120, 9, 1)],
                ids=lambda c: f"Nx{c[0]}_m{c[3]}_s{c[4]}_{'split' if c[5] else 'fp64'}")
def captured(request):
    Nx, t2, J2, kept, step, mode = request.param
    cfg = orc.RunConfig(Nx=Nx, Ny=4, t1=1.0, t2=t2, J1=0.4, J2=J2, kept_min=kept, kept_warm=kept,
                        sweeps=[kept], lanzero=1e-10)
    o = orc.Oracle(cfg, capture_step=step)
    o.run()
    cap = parse_oracle_capture(*o.capture())
    ctx = Context(Nx, 4, 1.0, t2, 0.4, J2)
    ctx.set_precision(mode)
    ctx.set_superblock(cap["sys"], cap["env"], cap["sys_bs"], cap["env_bs"], cap["psi0"])
    yield cap, ctx, mode
    ctx.close()


@pytest.mark.gpu
def test_noalloc_matches_device_entry(captured):
    import torch
    cap, ctx, mode = captured
    n = ctx.dim
    rng = np.random.default_rng(7)
    x1 = torch.from_numpy(cap["psi0"].vec.astype(np.complex128)).cuda()
    x2 = torch.from_numpy(rng.standard_normal(n) + 1j * rng.standard_normal(n)).cuda()
    ref1, ref2 = torch.empty_like(x1), torch.empty_like(x1)
    y1, y2, y3 = torch.empty_like(x1), torch.empty_like(x1), torch.empty_like(x1)
    torch.cuda.synchronize()
    ctx.hpsi_device(x1.data_ptr(), ref1.data_ptr())
    ctx.hpsi_device(x2.data_ptr(), ref2.data_ptr())
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    ctx.hpsi_noalloc(x1.data_ptr(), y1.data_ptr())
    ctx.hpsi_noalloc(x2.data_ptr(), y2.data_ptr())
    ctx.hpsi_noalloc(x1.data_ptr(), y3.data_ptr())
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    r1, r2, o1, o2, o3 = (t.cpu().numpy() for t in (ref1, ref2, y1, y2, y3))
    assert rel(o1, r1) <= 1e-13
    assert rel(o2, r2) <= 1e-13
    assert np.array_equal(o1, o3)
    assert rel(o1, cap["hpsi"].vec) <= (2e-5 if mode else 1e-13)


@pytest.mark.gpu
def test_noalloc_rejects_oversized_superblock():
    import torch
    import bench
    sl, el, ints, data, _off, n = bench.make_superblock()
    ctx = Context(12, 4, 1.0, 0.3, 0.4, 0.036)
    try:
        ctx.set_superblock_flat(sl, el, ints, data)
        x = torch.zeros(ctx.dim, dtype=torch.complex128, device="cuda")
        y = torch.empty_like(x)
        torch.cuda.synchronize()
        with pytest.raises(TscError) as ei:
            ctx.hpsi_noalloc(x.data_ptr(), y.data_ptr())
        assert ei.value.code == TSC_E_LIMIT
        assert "fixed maximum" in str(ei.value)
    finally:
        ctx.close()
