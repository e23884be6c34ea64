"""Several independent ground-state searches on one GPU at once
(run_parameter_points: one context per point, host threads): each point's
per-step energies equal those of the same point run alone (<= 1e-12 relative;
same arithmetic on separate streams)."""
import numpy as np
import pytest

from tsc_tri_t1t2j1j2_b200 import Context, run_parameter_points

SWEEP = dict(kept_min=40, kept_warm=40, sweeps=[40, 60], lanzero=1e-10)
POINTS = [dict(Nx=3, Ny=4, t1=1.0, t2=t2, J1=0.4, J2=0.4 * t2 * t2) for t2 in (0.0, 0.2, 0.3)]


@pytest.mark.gpu
def test_concurrent_points_equal_solo_runs():
    together = run_parameter_points(POINTS, SWEEP)
    for p, steps in zip(POINTS, together):
        ctx = Context(**p)
        try:
            solo = ctx.get_ground_state(**SWEEP)
        finally:
            ctx.close()
        assert len(steps) == len(solo)
        e = np.array([s["e0"] for s in steps])
        es = np.array([s["e0"] for s in solo])
        assert np.max(np.abs(e - es) / np.abs(es)) <= 1e-12
