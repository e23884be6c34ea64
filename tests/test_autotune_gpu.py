"""The FP64 H.psi schedule autotuner: a run whose superblocks reach >= 8 GFLOP
per H.psi times the candidate schedules and keeps the per-class fastest; its
per-step energies equal those of the same run with the schedule fixed
(autotune off) to 1e-10 relative (only the summation order of split term lists
differs), and a fixed-schedule run repeats bit for bit."""
import numpy as np
import pytest

from tsc_tri_t1t2j1j2_b200 import Context

RUN = dict(kept_min=300, kept_warm=300, sweeps=[300, 600], lanzero=1e-10)


def run(autotune):
    ctx = Context(8, 4, 1.0, 0.3, 0.4, 0.036)
    try:
        ctx.set_autotune(autotune)
        steps = ctx.get_ground_state(**RUN)
        return np.array([s["e0"] for s in steps]), ctx.autotune_table()
    finally:
        ctx.close()


@pytest.mark.gpu
def test_autotune_times_candidates_and_keeps_energies():
    e_on, table = run(True)
    e_off, table_off = run(False)
    e_off2, _ = run(False)
    assert table and not table_off
    assert any(all(v is not None for v in ms) for ms in table.values())
    assert np.max(np.abs(e_on - e_off) / np.abs(e_off)) <= 1e-10
    assert np.array_equal(e_off, e_off2)
