"""Flat layout of the reference's derived types (DMRG_code/common.f90:84-156).

One object = a run of int32 descriptors plus a run of complex128 data, in the
order documented in include/tsc_gpu.h.  Matrices are column-major (Fortran
order), so a Fortran host passes its ``mat`` / ``vec`` arrays without
reordering.  These helpers parse and emit that layout for tests and the Python
mirror of the reference interface.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


class Cursor:
    """Sequential reader over (ints, data)."""

    def __init__(self, ints, data, i0=0, d0=0):
        self.ints = np.asarray(ints, dtype=np.int32)
        self.data = np.asarray(data, dtype=np.complex128)
        self.i = i0
        self.d = d0

    def take(self, n=1):
        v = self.ints[self.i:self.i + n]
        if len(v) != n:
            raise ValueError("descriptor array too short")
        self.i += n
        return v

    def one(self):
        return int(self.take(1)[0])

    def cdata(self, n):
        v = self.data[self.d:self.d + n]
        if len(v) != n:
            raise ValueError("data array too short")
        self.d += n
        return v


@dataclass
class Block:
    """Total_Block / Sub_Block (common.f90:134-142)."""
    len: int
    up_dif: int
    down_dif: int
    subs: np.ndarray            # (num, 5): num_up, num_down, down_dif, row_dim, sdim
    mats: list = field(default_factory=list)   # complex (row_dim, sdim) Fortran-ordered arrays
    dim: int = 0

    @property
    def num(self):
        return len(self.subs)

    @staticmethod
    def read(c: Cursor) -> "Block":
        ln, num, dim, up, dn = (int(x) for x in c.take(5))
        subs = c.take(5 * num).reshape(num, 5).copy() if num else np.zeros((0, 5), np.int32)
        mats = []
        for s in subs:
            r, q = int(s[3]), int(s[4])
            mats.append(c.cdata(r * q).reshape((r, q), order="F").copy())
        return Block(ln, up, dn, subs, mats, dim)

    def write(self, ints: list, data: list):
        ints += [self.len, self.num, self.dim, self.up_dif, self.down_dif]
        for s, m in zip(self.subs, self.mats):
            ints += [int(x) for x in s]
            data.append(np.asarray(m, dtype=np.complex128).ravel(order="F"))


@dataclass
class Basis:
    """Total_Basis / Basis_Map / Sub_Basis_Map (common.f90:84-101)."""
    len: int
    dim: int
    sectors: np.ndarray   # (num, 4): new_num_up, new_num_down, dim, npieces
    pieces: np.ndarray    # (P, 6): bl_num_up, bl_num_down, st_num_up, st_num_down, spos, sdim

    @staticmethod
    def read(c: Cursor) -> "Basis":
        ln, num, dim = (int(x) for x in c.take(3))
        sec = c.take(4 * num).reshape(num, 4).copy() if num else np.zeros((0, 4), np.int32)
        npc = int(sec[:, 3].sum()) if num else 0
        pcs = c.take(6 * npc).reshape(npc, 6).copy() if npc else np.zeros((0, 6), np.int32)
        return Basis(ln, dim, sec, pcs)

    def write(self, ints: list, data: list):
        ints += [self.len, len(self.sectors), self.dim]
        for s in self.sectors:
            ints += [int(x) for x in s]
        for p in self.pieces:
            ints += [int(x) for x in p]


@dataclass
class Wave:
    """Wavefunction / Sub_Wave (common.f90:119-129); vec is the flat column-major data."""
    sys_len: int
    env_len: int
    secs: np.ndarray     # (num, 6): sys_num_up, sys_num_down, env_num_up, env_num_down, sys_dim, env_dim
    vec: np.ndarray

    @property
    def dim(self):
        return int((self.secs[:, 4].astype(np.int64) * self.secs[:, 5]).sum()) if len(self.secs) else 0

    @staticmethod
    def read(c: Cursor, with_data=True) -> "Wave":
        sl, el, num, _dim = (int(x) for x in c.take(4))
        secs = c.take(6 * num).reshape(num, 6).copy() if num else np.zeros((0, 6), np.int32)
        n = int((secs[:, 4].astype(np.int64) * secs[:, 5]).sum()) if num else 0
        vec = c.cdata(n).copy() if with_data else np.zeros(n, np.complex128)
        return Wave(sl, el, secs, vec)

    def write(self, ints: list, data: list, with_data=True):
        ints += [self.sys_len, self.env_len, len(self.secs), min(self.dim, 2**31 - 1)]
        for s in self.secs:
            ints += [int(x) for x in s]
        if with_data:
            data.append(np.asarray(self.vec, dtype=np.complex128))

    def sector(self, k):
        off = int((self.secs[:k, 4].astype(np.int64) * self.secs[:k, 5]).sum())
        r, q = int(self.secs[k, 4]), int(self.secs[k, 5])
        return self.vec[off:off + r * q].reshape((r, q), order="F")


@dataclass
class Model:
    """Total_Model (common.f90:167-174): ham + boundary-site operator sets."""
    len: int
    ham: Block
    ops: list   # ops[i] = [elec_up, elec_down, spin_sd, num_sn] for boundary op i+1

    @staticmethod
    def read(c: Cursor) -> "Model":
        ln = c.one()
        nops = c.one()
        ham = Block.read(c)
        ops = [[Block.read(c) for _ in range(4)] for _ in range(nops)]
        return Model(ln, ham, ops)

    def write(self, ints: list, data: list):
        ints += [self.len, len(self.ops)]
        self.ham.write(ints, data)
        for o in self.ops:
            for b in o:
                b.write(ints, data)


def pack(ints: list, data: list):
    """Finalise (ints, data) lists into contiguous arrays for the C-ABI."""
    iarr = np.asarray(ints, dtype=np.int32)
    darr = np.concatenate(data) if data else np.zeros(0, np.complex128)
    return iarr, np.ascontiguousarray(darr, dtype=np.complex128)
