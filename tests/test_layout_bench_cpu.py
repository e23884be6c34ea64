"""Host logic: flat layout round trips, the bench workload generator and the
max-over-ranks timing reduction used for N>1 (gloo, world_size 2)."""
import os
import socket
import subprocess
import sys

import numpy as np

import bench
import orc
from _capture import parse_oracle_capture
from tsc_tri_t1t2j1j2_b200.layout import Cursor, Model, pack


def test_layout_round_trip():
    cfg = orc.RunConfig(Nx=3, Ny=4, kept_min=30, kept_warm=30, sweeps=[30], lanzero=1e-10)
    o = orc.Oracle(cfg, capture_step=5)
    o.run()
    ints, data = o.capture()
    c = parse_oracle_capture(ints, data)
    ii, dd = [], []
    c["sys"].write(ii, dd)
    i2, d2 = pack(ii, dd)
    back = Model.read(Cursor(i2, d2))
    assert back.len == c["sys"].len and len(back.ops) == len(c["sys"].ops)
    for a, b in zip(back.ham.mats, c["sys"].ham.mats):
        assert np.array_equal(a, b)


def test_bench_superblock_generator():
    sl, el, ints, data, off, n = bench.make_superblock()
    assert (sl, el) == (23, 23)
    assert len(data) == off + n
    assert abs(np.linalg.norm(data[off:]) - 1.0) < 1e-12
    sl2, el2, ints2, data2, off2, n2 = bench.make_superblock()
    assert np.array_equal(data, data2)   # seeded: every arm sees the same input


WORKER = r"""
import os, sys
sys.path.insert(0, sys.argv[1])
import torch.distributed as dist
import bench
dist.init_process_group("gloo", init_method="tcp://127.0.0.1:" + sys.argv[2], rank=int(sys.argv[3]), world_size=2)
v = bench.max_over_ranks(1.5 + int(sys.argv[3]), dist, "cpu")
print("MAX", v)
dist.destroy_process_group()
"""


def test_max_over_ranks_gloo_two_ranks(tmp_path):
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = str(s.getsockname()[1])
    s.close()
    script = tmp_path / "w.py"
    script.write_text(WORKER)
    procs = [subprocess.Popen([sys.executable, str(script), root, port, str(r)], stdout=subprocess.PIPE, text=True)
             for r in range(2)]
    outs = [p.communicate(timeout=120)[0] for p in procs]
    assert all(p.returncode == 0 for p in procs)
    assert all("MAX 2.5" in o for o in outs)
