"""Loader and ctypes signatures of the in-tree CUDA library libtscgpu.so.

There is no CPU fallback: if the library is missing or no CUDA device is
visible, every entry point raises instead of computing something else.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libtscgpu.so")

c_int, c_double, c_ll, c_void = ctypes.c_int, ctypes.c_double, ctypes.c_longlong, ctypes.c_void_p
P = ctypes.POINTER

# every symbol include/tsc_gpu.h declares
EXPORTED = [
    "tsc_create", "tsc_destroy", "tsc_last_error", "tsc_tot_num_up", "tsc_superblock_set",
    "tsc_superblock_dim", "tsc_hpsi", "tsc_hpsi_device", "tsc_lanczos", "tsc_truncate",
    "tsc_density_matrix", "tsc_truncation_operator",
    "tsc_renormalize", "tsc_wave_transform", "tsc_dmrg_run", "tsc_set_capture", "tsc_get_capture",
    "tsc_hpsi_stats", "tsc_stream", "tsc_hpsi_noalloc", "tsc_set_precision", "tsc_set_split_wait_limit",
    "tsc_set_resident_limit", "tsc_spill_stats", "tsc_set_spill_directory", "tsc_disk_spill_stats", "tsc_split_views",
    "tsc_checkpoint_write", "tsc_checkpoint_read", "tsc_set_split_refinement",
    "tsc_set_split_renormalization", "tsc_set_lanczos_graph", "tsc_lanczos_graph_stats",
    "tsc_set_split_view_sharing", "tsc_set_split_finish_tolerance",
    "tsc_blocksparse_set", "tsc_blocksparse_apply", "tsc_measure_density", "tsc_measure_density_cor", "tsc_measure_correlation", "tsc_measure_pair_correlation",
    "tsc_set_autotune",
    "tsc_autotune_table", "tsc_autotune_superblock",
]


class ModelConfig(ctypes.Structure):
    _fields_ = [("Nx", c_int), ("Ny", c_int), ("t1", c_double), ("t2", c_double), ("J1", c_double),
                ("J2", c_double), ("delta", c_int), ("device", c_int)]


class SweepConfig(ctypes.Structure):
    _fields_ = [("kept_min", c_int), ("kept_max_warmup", c_int), ("nsweeps", c_int),
                ("sweep_kept_max", P(c_int)), ("lanzero", c_double), ("seed", ctypes.c_ulonglong),
                ("warmup_only", c_int), ("final_half_sweep", c_int), ("resume", c_int), ("max_solves", c_int),
                ("lanzero_warmup", c_double), ("final_stop", c_int)]


class StepLog(ctypes.Structure):
    _fields_ = [("phase", c_int), ("sys_len", c_int), ("env_len", c_int), ("e0", c_double),
                ("lanczos_iters", c_int), ("num_state", c_int), ("trun_err", c_double), ("entropy", c_double),
                ("entropy_mult", c_double), ("hpsi_calls", c_int), ("hpsi_seconds", c_double),
                ("hpsi_flops", c_double), ("step_seconds", c_double), ("set_seconds", c_double),
                ("lanczos_seconds", c_double), ("truncate_seconds", c_double), ("grow_seconds", c_double),
                ("wave_seconds", c_double), ("split_iters", c_int), ("split_e0", c_double)]


class TscError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"tsc error {code}: {msg}")
        self.code = code


_lib = None


def load():
    """Load libtscgpu.so (fails loudly when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} not built: run __graft_entry__.build() (nvcc, sm_100a)")
    L = ctypes.CDLL(LIB_PATH)
    pi, pd = P(c_int), P(c_double)
    L.tsc_create.argtypes = [P(c_void), P(ModelConfig)]
    L.tsc_destroy.argtypes = [c_void]
    L.tsc_last_error.argtypes = [c_void]
    L.tsc_last_error.restype = ctypes.c_char_p
    L.tsc_tot_num_up.argtypes = [c_void]
    L.tsc_superblock_set.argtypes = [c_void, c_int, c_int, pi, c_ll, pd, c_ll]
    L.tsc_superblock_dim.argtypes = [c_void]
    L.tsc_superblock_dim.restype = c_ll
    L.tsc_hpsi.argtypes = [c_void, pd, pd]
    L.tsc_hpsi_device.argtypes = [c_void, c_void, c_void]
    L.tsc_lanczos.argtypes = [c_void, pd, c_double, pi, pd]
    L.tsc_truncate.argtypes = [c_void, c_int, pd, c_int, c_int, c_double, pi, pd, pd, pd, P(pi), P(c_ll), P(pd),
                               P(c_ll), pd, c_ll]
    L.tsc_density_matrix.argtypes = [c_void, c_int, pd, c_int, P(pi), P(c_ll), P(pd), P(c_ll)]
    L.tsc_truncation_operator.argtypes = [c_void, pi, c_ll, pd, c_ll, c_int, c_int, c_double, pi, pd, pd, pd, P(pi),
                                          P(c_ll), P(pd), P(c_ll), pd, c_ll]
    L.tsc_renormalize.argtypes = [c_void, c_int, c_int, c_int, c_int, pi, c_ll, pd, c_ll, P(pi), P(c_ll), P(pd),
                                  P(c_ll)]
    L.tsc_wave_transform.argtypes = [c_void, c_int, pi, c_ll, pd, c_ll, pd]
    L.tsc_dmrg_run.argtypes = [c_void, P(SweepConfig), P(StepLog), c_int]
    L.tsc_set_capture.argtypes = [c_void, c_int]
    L.tsc_get_capture.argtypes = [c_void, P(pi), P(c_ll), P(pd), P(c_ll), pi, pi]
    L.tsc_hpsi_stats.argtypes = [c_void, pd, pd, pd, pi]
    L.tsc_stream.argtypes = [c_void]
    L.tsc_stream.restype = c_void
    L.tsc_hpsi_noalloc.argtypes = [c_void, c_void, c_void]
    L.tsc_set_precision.argtypes = [c_void, c_int, c_double]
    L.tsc_set_split_wait_limit.argtypes = [c_void, c_ll]
    L.tsc_set_resident_limit.argtypes = [c_void, c_ll]
    L.tsc_split_views.argtypes = [c_void, P(c_ll), P(c_int)]
    L.tsc_checkpoint_write.argtypes = [c_void, ctypes.c_char_p]
    L.tsc_set_split_refinement.argtypes = [c_void, c_double]
    L.tsc_set_split_renormalization.argtypes = [c_void, c_int]
    L.tsc_set_lanczos_graph.argtypes = [c_void, c_int]
    L.tsc_set_split_view_sharing.argtypes = [c_void, c_int]
    L.tsc_set_split_finish_tolerance.argtypes = [c_void, c_double]
    L.tsc_lanczos_graph_stats.argtypes = [c_void, P(c_ll), P(c_ll), ctypes.c_char_p, c_int]
    L.tsc_checkpoint_read.argtypes = [c_void, ctypes.c_char_p]
    L.tsc_spill_stats.argtypes = [c_void, P(c_ll), P(c_ll), P(c_double), P(c_double), P(c_ll), P(c_ll)]
    L.tsc_set_spill_directory.argtypes = [c_void, ctypes.c_char_p, c_ll]
    L.tsc_disk_spill_stats.argtypes = [c_void, P(c_ll), P(c_ll), P(c_double), P(c_double), P(c_ll)]
    L.tsc_blocksparse_set.argtypes = [c_void, c_int, ctypes.POINTER(c_int), c_ll, ctypes.POINTER(c_double), c_ll,
                                      ctypes.POINTER(c_ll), ctypes.POINTER(c_double), ctypes.POINTER(c_double)]
    L.tsc_blocksparse_apply.argtypes = [c_void, c_void, c_void, c_int]
    L.tsc_measure_density.argtypes = [c_void, ctypes.POINTER(c_double), c_int]
    L.tsc_measure_density_cor.argtypes = [c_void, c_int, ctypes.POINTER(c_double), c_int]
    L.tsc_measure_correlation.argtypes = [c_void, c_int, c_int, ctypes.POINTER(c_double), c_int]
    L.tsc_measure_pair_correlation.argtypes = [c_void, c_int, c_int, c_int, c_int, ctypes.POINTER(c_int),
                                               ctypes.POINTER(c_double), c_int]
    L.tsc_set_autotune.argtypes = [c_void, c_int]
    L.tsc_autotune_table.argtypes = [c_void, ctypes.POINTER(c_int), ctypes.POINTER(c_double), c_int]
    L.tsc_autotune_superblock.argtypes = [c_void, c_int]
    _lib = L
    return L


def exported_symbols():
    """Names of include/tsc_gpu.h that the loaded library exports."""
    L = ctypes.CDLL(LIB_PATH)
    return [n for n in EXPORTED if hasattr(L, n)]
