"""Lanczos iterations replayed as a CUDA graph (tsc_set_lanczos_graph, the
default) against the same runs launched step by step from the host: the graph
holds the same kernels on the same data, so whole runs are bit-identical --
every step's energy, iteration count, truncation weight and kept count -- in
both forms."""
import pytest

from tsc_tri_t1t2j1j2_b200 import Context

RUN = dict(kept_min=40, kept_warm=40, sweeps=[40, 60], lanzero=1e-10)


def run(mode, graph):
    ctx = Context(4, 4, 1.0, 0.3, 0.4, 0.036)
    try:
        ctx.set_precision(mode, 1e-11)
        ctx.set_lanczos_graph(graph)
        steps = ctx.get_ground_state(**RUN)
        stats = ctx.lanczos_graph_stats()
    finally:
        ctx.close()
    if graph:   # the graphed run really replayed its iterations
        assert stats["fallbacks"] == 0, stats["reason"]
        assert stats["replays"] > len(steps)
    else:
        assert stats["replays"] == 0
    return steps


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [Context.FP64, Context.SPLIT_BF16], ids=["fp64", "split"])
def test_graph_run_is_bit_identical(mode):
    a, b = run(mode, True), run(mode, False)
    assert len(a) == len(b) > 50
    for x, y in zip(a, b):
        for k in ("e0", "lanczos_iters", "split_iters", "num_state", "trun_err", "entropy"):
            assert x[k] == y[k], (k, x["phase"], x["sys_len"], x[k], y[k])
