"""Checkpoint files in the reference's format (tsc_checkpoint_write/_read) and
resuming a run from them, through the C-ABI.

The files are decoded here independently of the engine, by the rules the
Fortran runtime writes them with: unformatted sequential records framed by
4-byte length markers (block.f90:1547-1576 wave_to_disk, :1713-1737
block_to_disk, :1802-1845 model_to_disk), the basis as fixed-width text
(formats 101-104 of basis_to_disk, :1983-2026).  Checks: every file parses to
the end; the wave is normalised and its sector sizes add up to its dimension;
every truncation sub-block has orthonormal columns; basis pieces tile their
sectors.  Then a run stopped after one sweep, written, read into a fresh
context and resumed for a second sweep reproduces, bit for bit, the last sweep
of the uninterrupted two-sweep run (energies, kept counts, truncation weights).
"""
import os
import struct

import numpy as np
import pytest

from tsc_tri_t1t2j1j2_b200 import Context

MODEL = dict(Nx=4, Ny=4, t1=1.0, t2=0.3, J1=0.4, J2=0.036)


def records(path):
    """Fortran unformatted sequential records (subrecords joined)."""
    out, cur = [], b""
    with open(path, "rb") as f:
        data = f.read()
    i = 0
    while i < len(data):
        head = struct.unpack_from("<i", data, i)[0]
        n = abs(head)
        cur += data[i + 4:i + 4 + n]
        tail = struct.unpack_from("<i", data, i + 4 + n)[0]
        assert abs(tail) == n
        i += 8 + n
        if head >= 0:
            out.append(cur)
            cur = b""
    assert i == len(data) and cur == b""
    return out


def ints(rec, n):
    assert len(rec) == 4 * n
    return struct.unpack(f"<{n}i", rec)


def blocks(recs, k=0):
    """Decodes consecutive Total_Block record groups from recs[k:]."""
    out = []
    while k < len(recs):
        ln, num, dim, upd, dnd = (ints(recs[k + j], 1)[0] for j in range(5))
        k += 5
        subs = []
        for _ in range(num):
            assert recs[k] == b""
            nu, nd, dd = ints(recs[k + 1], 3)
            r, c = ints(recs[k + 2], 2)
            m = np.frombuffer(recs[k + 3], dtype=np.complex128).reshape((r, c), order="F")
            subs.append(((nu, nd, dd), m))
            k += 4
        out.append((ln, num, dim, upd, dnd, subs))
    return out


@pytest.mark.gpu
def test_checkpoint_files_and_resume(tmp_path):
    ctx = Context(device=0, **MODEL)
    try:
        ctx.set_autotune(False)
        full = ctx.get_ground_state(60, 60, [60, 80], lanzero=1e-10, seed=1)
    finally:
        ctx.close()
    ctx = Context(device=0, **MODEL)
    try:
        ctx.set_autotune(False)
        first = ctx.get_ground_state(60, 60, [60], lanzero=1e-10, seed=1)
        nfiles = ctx.checkpoint_write(str(tmp_path))
    finally:
        ctx.close()
    assert [s["e0"] for s in first] == [s["e0"] for s in full[:len(first)]]
    names = sorted(os.listdir(tmp_path))
    assert len(names) == nfiles and "eigvec1" in names

    # the wave: sys_len, env_len, num, dim, then per sector an empty record, QNs, dims, vec
    w = records(tmp_path / "eigvec1")
    sl, el, num, dim = (ints(w[j], 1)[0] for j in range(4))
    assert len(w) == 4 + 5 * num
    tot, norm = 0, 0.0
    for s in range(num):
        base = 4 + 5 * s
        assert w[base] == b""
        sd, ed = ints(w[base + 3], 2)
        v = np.frombuffer(w[base + 4], dtype=np.complex128)
        assert len(v) == sd * ed
        tot += sd * ed
        norm += float(np.vdot(v, v).real)
    assert tot == dim and abs(norm - 1.0) <= 1e-12

    # models: len, then whole Total_Blocks (ham and 4 operators per boundary site)
    for nm in (n for n in names if n.startswith(("sysblocks", "envblocks"))):
        r = records(tmp_path / nm)
        ln = ints(r[0], 1)[0]
        assert nm.endswith(str(ln))
        bl = blocks(r, 1)
        assert (len(bl) - 1) % 4 == 0
    # truncations: orthonormal columns in every sub-block
    for nm in (n for n in names if n.startswith(("systruns", "envtruns"))):
        (b,) = blocks(records(tmp_path / nm))
        for _qn, m in b[5]:
            if m.size:
                assert np.max(np.abs(m.conj().T @ m - np.eye(m.shape[1]))) <= 1e-10
    # bases: fixed-width text, pieces tile each sector
    for nm in (n for n in names if n.startswith(("sysbs", "envbs"))):
        lines = (tmp_path / nm).read_text().split("\n")
        assert lines[0].startswith("len=") and lines[1].startswith("num=") and lines[2].startswith("dim=")
        nsec, bdim = int(lines[1][4:10]), int(lines[2][4:10])
        i, tot = 3, 0
        for _ in range(nsec):
            assert lines[i].strip() == ""
            npc, sdim = int(lines[i + 2][4:10]), int(lines[i + 3][4:10])
            assert lines[i + 4].startswith("new_num_up=") and lines[i + 5].startswith("new_num_down=")
            i += 6
            pos = 0
            for _ in range(npc):
                assert int(lines[i][4:10]) == pos
                pos += int(lines[i + 1][4:10])
                assert lines[i + 2][:10] == "bl_num_up=" and lines[i + 2][16:28] == "bl_num_down="
                i += 4
            assert pos == sdim
            tot += sdim
        assert tot == bdim

    ctx = Context(device=0, **MODEL)
    try:
        ctx.set_autotune(False)
        ctx.checkpoint_read(str(tmp_path))
        resumed = ctx.get_ground_state(60, 60, [80], lanzero=1e-10, seed=1, resume=True)
    finally:
        ctx.close()
    tail = full[len(full) - len(resumed):]
    assert len(resumed) == len(full) - len(first)
    for g, r in zip(resumed, tail):
        assert (g["phase"], g["sys_len"], g["env_len"]) == (r["phase"], r["sys_len"], r["env_len"])
        assert g["e0"] == r["e0"]
        assert g["num_state"] == r["num_state"]
        assert g["trun_err"] == r["trun_err"]
