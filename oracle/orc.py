"""ctypes wrapper of the oracle (oracle/_build/liborc.so).

TEST INFRASTRUCTURE ONLY: the oracle is the CPU restatement of the reference
DMRG hot path (hyx15903/TSC_Tri_t1t2J1J2, DMRG_code/*.f90).  Only tests/,
``__graft_entry__.smoke`` and bench.py's cpu_baseline leg may import it, and
only as the checker / CPU baseline, never as the thing measured or shipped.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liborc.so")

_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++ + scipy's OpenBLAS)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.orc_new.restype = vp
        L.orc_new.argtypes = [i, i, d, d, d, d, i, i, i, ctypes.POINTER(i), i, d, ctypes.c_ulonglong, i, i]
        L.orc_free.argtypes = [vp]
        L.orc_error.restype = ctypes.c_char_p
        L.orc_error.argtypes = [vp]
        L.orc_run.argtypes = [vp]
        L.orc_run.restype = i
        L.orc_tot_num_up.argtypes = [vp]
        L.orc_steps.argtypes = [vp, ctypes.POINTER(d)]
        L.orc_capture_serialize.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]
        L.orc_serialized_copy.argtypes = [vp, ctypes.POINTER(i), ctypes.POINTER(d)]
        L.orc_w6js.restype = d
        L.orc_w6js.argtypes = [i] * 6
        L.orc_w3js.restype = d
        L.orc_w3js.argtypes = [i] * 6
        L.orc_hpsi_flat.argtypes = [vp, i, i, ctypes.POINTER(i), ctypes.POINTER(d), ctypes.POINTER(d), i,
                                    ctypes.POINTER(d), ctypes.POINTER(d)]
        L.orc_hpsi_flat.restype = i
        L.orc_measure_density.argtypes = [vp, ctypes.POINTER(d)]
        L.orc_measure_density.restype = i
        L.orc_density_cor.argtypes = [vp, i, ctypes.POINTER(d)]
        L.orc_density_cor.restype = i
        L.orc_oper_cor.argtypes = [vp, i, i, ctypes.POINTER(d)]
        L.orc_oper_cor.restype = i
        L.orc_set_final_stop.argtypes = [vp, i]
        L.orc_pair_cor.argtypes = [vp, i, i, i, i, ctypes.POINTER(d), i]
        L.orc_pair_cor.restype = i
        _lib = L
    return _lib


@dataclass
class RunConfig:
    """Model and schedule (restates main.f90:54-99 as data)."""
    Nx: int = 6
    Ny: int = 4
    t1: float = 1.0
    t2: float = 0.0
    J1: float = 0.4
    J2: float = 0.0
    delta: int = 12
    kept_min: int = 100
    kept_warm: int = 100
    sweeps: list = field(default_factory=lambda: [100])
    lanzero: float = -1.0      # >0 overrides the reference's Lanczos tolerance schedule
    seed: int = 1
    final_half_sweep: bool = False   # main.f90:205-206: end at 5 Num_site / 6 (the measuring position)
    final_stop: int = 0              # test knob: last label of that half sweep (0: the reference's)


STEP_FIELDS = ["phase", "sys_len", "env_len", "e0", "iters", "num_state", "trun_err",
               "entropy", "entropy_mult", "hpsi_calls", "hpsi_seconds", "hpsi_flops"]


class Oracle:
    def __init__(self, cfg: RunConfig, capture_step: int = -1):
        L = lib()
        sk = (ctypes.c_int * max(1, len(cfg.sweeps)))(*cfg.sweeps)
        self.h = L.orc_new(cfg.Nx, cfg.Ny, cfg.t1, cfg.t2, cfg.J1, cfg.J2, cfg.delta, cfg.kept_min,
                           cfg.kept_warm, sk, len(cfg.sweeps), cfg.lanzero, cfg.seed, capture_step,
                           1 if cfg.final_half_sweep else 0)
        err = L.orc_error(self.h)
        if err:
            raise RuntimeError(err.decode())
        if cfg.final_stop:
            L.orc_set_final_stop(self.h, int(cfg.final_stop))
        self.cfg = cfg

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_free(self.h)
            self.h = None

    def run(self) -> list[dict]:
        L = lib()
        n = L.orc_run(self.h)
        if n < 0:
            raise RuntimeError(L.orc_error(self.h).decode())
        buf = np.zeros(12 * max(n, 1), dtype=np.float64)
        L.orc_steps(self.h, buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return [dict(zip(STEP_FIELDS, buf[12 * k:12 * k + 12].tolist())) for k in range(n)]

    def measure_density(self):
        """<n_i> of every site in the last ground state (measure_operator_dia)."""
        L = lib()
        out = np.zeros(self.cfg.Nx * self.cfg.Ny, dtype=np.float64)
        n = L.orc_measure_density(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        if n < 0:
            raise RuntimeError(L.orc_error(self.h).decode())
        return out

    def density_cor(self, site):
        """<n_site n_j>, j = 1..Num_site, of the last ground state (Get_density_cor,
        measure.f90:2525-2681); zero where the reference computes nothing."""
        L = lib()
        out = np.zeros(2 * self.cfg.Nx * self.cfg.Ny, dtype=np.float64)
        n = L.orc_density_cor(self.h, int(site), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        if n < 0:
            raise RuntimeError(L.orc_error(self.h).decode())
        return out[0::2] + 1j * out[1::2]

    def spin_cor(self, site):
        """<S_site . S_j>, j = 1..Num_site, of the last ground state (Get_density_cor
        with st_sd, main.f90:275); zero where the reference computes nothing."""
        L = lib()
        out = np.zeros(2 * self.cfg.Nx * self.cfg.Ny, dtype=np.float64)
        n = L.orc_oper_cor(self.h, 1, int(site), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        if n < 0:
            raise RuntimeError(L.orc_error(self.h).decode())
        return out[0::2] + 1j * out[1::2]

    def elec_cor(self, site):
        """Electron correlation of the last ground state (Get_density_cor with
        st_elec_up, st_elec_down, Flags 'F', main.f90:288), j = 1..Num_site; zero
        where the reference computes nothing."""
        L = lib()
        out = np.zeros(2 * self.cfg.Nx * self.cfg.Ny, dtype=np.float64)
        n = L.orc_oper_cor(self.h, 2, int(site), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        if n < 0:
            raise RuntimeError(L.orc_error(self.h).decode())
        return out[0::2] + 1j * out[1::2]

    def pair_cor(self, xc1, xc2, ij=0, ij1=1):
        """Singlet pair correlations of the last ground state (Get_mSCOP_Operator_Cor0,
        Flags 'S0', measure.f90:2683-2834): [(s1, s2, s3, s4, value)] for the bond
        (xc1, neib(xc1, ij1)) against the bonds (s3, neib(s3, 1|3|5)) the
        reference visits."""
        L = lib()
        out = np.zeros(6 * 4096, dtype=np.float64)
        n = L.orc_pair_cor(self.h, int(xc1), int(xc2), int(ij), int(ij1),
                           out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 4096)
        if n < 0:
            raise RuntimeError(L.orc_error(self.h).decode())
        r = out[:6 * min(n, 4096)].reshape(-1, 6)
        return [(int(a), int(b), int(c), int(e), complex(x, y)) for a, b, c, e, x, y in r]

    def capture(self):
        """Flat (ints, complex) serialisation of the captured superblock."""
        L = lib()
        ni, nc = ctypes.c_longlong(), ctypes.c_longlong()
        if L.orc_capture_serialize(self.h, ctypes.byref(ni), ctypes.byref(nc)) != 0:
            raise RuntimeError("no capture")
        ints = np.zeros(ni.value, dtype=np.int32)
        data = np.zeros(nc.value, dtype=np.complex128)
        L.orc_serialized_copy(self.h, ints.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                              data.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return ints, data

    def hpsi_flat(self, sys_len, env_len, ints, data, npsi, nreps=1):
        """model_wave on a flat superblock (sys model, env model, bases, psi)."""
        L = lib()
        ints = np.ascontiguousarray(ints, dtype=np.int32)
        data = np.ascontiguousarray(data, dtype=np.complex128)
        out = np.zeros(npsi, dtype=np.complex128)
        sec, flops = ctypes.c_double(), ctypes.c_double()
        rc = L.orc_hpsi_flat(self.h, sys_len, env_len, ints.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                             data.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                             out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), nreps,
                             ctypes.byref(sec), ctypes.byref(flops))
        if rc != 0:
            raise RuntimeError(L.orc_error(self.h).decode())
        return out, sec.value, flops.value


def w6js(*a) -> float:
    return lib().orc_w6js(*[int(x) for x in a])


def w3js(*a) -> float:
    return lib().orc_w3js(*[int(x) for x in a])
