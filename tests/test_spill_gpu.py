"""Host spill of stored block models (tsc_set_resident_limit), through the C-ABI.

The reference writes every block model to disk after each step and reads it
back when the sweep returns (block.f90:1715-1900, dmrg_sub.f90:1119-1139).  The
engine keeps them in HBM under a byte limit and moves the least recently used
to host memory beyond it.  A whole ground-state search with limit 0 (every
stored model lives in host memory between its uses) must give bit-identical
energies, kept counts and truncation weights to the run that keeps everything
on the device, and must have moved models both ways.
"""
import pytest

from tsc_tri_t1t2j1j2_b200 import Context

MODEL = dict(Nx=4, Ny=4, t1=1.0, t2=0.3, J1=0.4, J2=0.036)
RUN = dict(kept_min=60, kept_warm=60, sweeps=[60, 80], lanzero=1e-10, seed=1)


def run(limit):
    ctx = Context(device=0, **MODEL)
    try:
        ctx.set_autotune(False)
        ctx.set_resident_limit(limit)
        steps = ctx.get_ground_state(**RUN)
        return steps, ctx.spill_stats()
    finally:
        ctx.close()


@pytest.mark.gpu
def test_spilled_run_is_bit_identical():
    ref, st0 = run(-1)
    got, st = run(0)
    assert st0["spills"] == 0 and st0["restores"] == 0
    assert st["spills"] > 0 and st["restores"] > 0 and st["bytes"] > 0
    assert st["limit_bytes"] == 0
    assert len(got) == len(ref)
    for g, r in zip(got, ref):
        assert g["e0"] == r["e0"]
        assert g["num_state"] == r["num_state"]
        assert g["trun_err"] == r["trun_err"]
        assert g["lanczos_iters"] == r["lanczos_iters"]


@pytest.mark.gpu
def test_disk_tier_run_is_bit_identical(tmp_path):
    """Resident limit 0 and host limit 0 with a spill directory: every stored
    model goes to a file between its uses (the reference's own disk round trip)
    and the run stays bit-identical to the resident one; the files are gone when
    the context closes."""
    ref, _ = run(-1)
    ctx = Context(device=0, **MODEL)
    try:
        ctx.set_autotune(False)
        ctx.set_resident_limit(0)
        ctx.set_spill_directory(str(tmp_path), 0)
        got = ctx.get_ground_state(**RUN)
        disk = ctx.disk_spill_stats()
    finally:
        ctx.close()
    assert disk["writes"] > 0 and disk["reads"] > 0 and disk["bytes"] > 0
    assert list(tmp_path.iterdir()) == []
    assert len(got) == len(ref)
    for g, r in zip(got, ref):
        assert g["e0"] == r["e0"]
        assert g["num_state"] == r["num_state"]
        assert g["trun_err"] == r["trun_err"]
