"""Python mirror of the reference's hot-path interface over the C-ABI.

Method names follow the Fortran subroutines they replace:

=========================  ==============================================
method                     reference
=========================  ==============================================
``model_wave``             get_sys.f90:6915 (H.psi, after hmerge :7398)
``lanczos_memo_new``       eigen.f90:4
``get_truncation_operator`` den_mat.f90:106/146 + :184
``get_hamiltonian``        get_sys.f90:4 (sys) / :305 (env)
``wave_trans``             dmrg_sub.f90:1471 (LR) / :1637 (RL)
``get_ground_state``       main.f90:114 (warm-up + sweeps)
=========================  ==============================================

Arguments are the flat descriptor objects of ``layout``; every call runs on
the GPU (there is no CPU path) and raises ``TscError`` with the library's
status code and message on failure.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _lib
from .layout import Basis, Block, Cursor, Model, Wave, pack

P = ctypes.POINTER


def _dptr(a):
    return a.ctypes.data_as(P(ctypes.c_double))


def _iptr(a):
    return a.ctypes.data_as(P(ctypes.c_int))


class Context:
    """One device-resident model (lattice + couplings) and its current superblock."""

    def __init__(self, Nx, Ny, t1=1.0, t2=0.0, J1=0.4, J2=0.0, delta=12, device=0):
        self.L = _lib.load()
        cfg = _lib.ModelConfig(Nx, Ny, t1, t2, J1, J2, delta, device)
        h = ctypes.c_void_p()
        rc = self.L.tsc_create(ctypes.byref(h), ctypes.byref(cfg))
        self.h = h
        if rc != 0:
            msg = self.L.tsc_last_error(h).decode() if h else "tsc_create failed"
            if h:
                self.L.tsc_destroy(h)
            self.h = None
            raise _lib.TscError(rc, msg)
        self.Nx, self.Ny = Nx, Ny
        self.sys_len = self.env_len = 0

    def close(self):
        if getattr(self, "h", None):
            self.L.tsc_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _check(self, rc):
        if rc < 0:
            raise _lib.TscError(rc, self.L.tsc_last_error(self.h).decode())
        return rc

    @property
    def tot_num_up(self):
        return self.L.tsc_tot_num_up(self.h)

    # ---------------------------------------------------------------- superblock
    def set_superblock(self, sys: Model, env: Model, sys_bs: Basis, env_bs: Basis, layout: Wave):
        ints, data = [], []
        sys.write(ints, data)
        env.write(ints, data)
        sys_bs.write(ints, data)
        env_bs.write(ints, data)
        layout.write(ints, data, with_data=False)
        self.set_superblock_flat(sys.len, env.len, *pack(ints, data))
        self.layout = layout

    def set_superblock_flat(self, sys_len, env_len, ints, data):
        ints = np.ascontiguousarray(ints, np.int32)
        data = np.ascontiguousarray(data, np.complex128)
        self._check(self.L.tsc_superblock_set(self.h, sys_len, env_len, _iptr(ints), len(ints), _dptr(data), len(data)))
        self.sys_len, self.env_len = sys_len, env_len
        self.dim = self.L.tsc_superblock_dim(self.h)

    def model_wave(self, vec):
        """out = H vec (host buffers, copies included)."""
        x = np.ascontiguousarray(vec, np.complex128)
        if len(x) != self.dim:
            raise ValueError("vector length does not match the superblock")
        out = np.empty_like(x)
        self._check(self.L.tsc_hpsi(self.h, _dptr(x), _dptr(out)))
        return out

    def hpsi_device(self, d_in: int, d_out: int):
        """H.psi on device pointers (e.g. torch tensors' data_ptr()), enqueued on the context stream."""
        self._check(self.L.tsc_hpsi_device(self.h, ctypes.c_void_p(d_in), ctypes.c_void_p(d_out)))

    FP64, SPLIT_BF16 = 0, 1

    def set_precision(self, mode: int, split_tol: float = 0.0):
        """H.psi arithmetic: Context.FP64 (default) or Context.SPLIT_BF16 (BF16 slices
        on the tensor cores, Lanczos finished in FP64).  Applies from the next
        superblock set."""
        self._check(self.L.tsc_set_precision(self.h, int(mode), float(split_tol)))

    def set_split_refinement(self, residual_factor: float):
        """FP64 finish of split solves: stop at residual <= factor * sqrt(lanzero);
        0 (the default) = the reference's stop (successive Ritz values within
        lanzero, eigen.f90:101)."""
        self._check(self.L.tsc_set_split_refinement(self.h, float(residual_factor)))

    def set_lanczos_graph(self, on: bool):
        """Lanczos iterations as CUDA-graph replays (default on; off launches every
        step from the host; results bit-identical)."""
        self._check(self.L.tsc_set_lanczos_graph(self.h, 1 if on else 0))

    def set_split_finish_tolerance(self, multiplier: float):
        """Split form: the FP64 finish stops when successive Ritz values agree to
        multiplier * lanzero (1: the reference's tolerance)."""
        self._check(self.L.tsc_set_split_finish_tolerance(self.h, float(multiplier)))

    def set_split_view_sharing(self, shared):
        """Split form: one sliced copy per operator block with the coefficients applied
        per term by the kernel (True, the default), one copy per term with the
        coefficient folded in (False: 1-2 % faster H.psi, ~4.5x the slice memory),
        or None to choose by the superblock's operator memory."""
        self._check(self.L.tsc_set_split_view_sharing(self.h, -1 if shared is None else (1 if shared else 0)))

    def lanczos_graph_stats(self):
        """{"replays": iterations replayed as graphs, "fallbacks": failed captures,
        "reason": the last failure's message}."""
        r, f = ctypes.c_longlong(), ctypes.c_longlong()
        buf = ctypes.create_string_buffer(512)
        self._check(self.L.tsc_lanczos_graph_stats(self.h, ctypes.byref(r), ctypes.byref(f), buf, 512))
        return {"replays": r.value, "fallbacks": f.value, "reason": buf.value.decode()}

    def set_split_renormalization(self, on: bool):
        """Split form only: U^H O U of block growth on the split kernel too (off by
        default; its error stays in every later Hamiltonian)."""
        self._check(self.L.tsc_set_split_renormalization(self.h, 1 if on else 0))

    def set_split_wait_limit(self, polls: int):
        """Poll limit of the split kernel's bounded waits (default 1<<20; 0 makes
        every wait give up at once, so the next split call fails with TSC_E_CUDA)."""
        self._check(self.L.tsc_set_split_wait_limit(self.h, int(polls)))

    def split_views(self):
        """Bytes and counts of the split form's pre-sliced operand views of the current
        superblock: {"operators": (bytes, views), "input": ..., "intermediates": ...}."""
        b, v = (ctypes.c_longlong * 3)(), (ctypes.c_int * 3)()
        self._check(self.L.tsc_split_views(self.h, b, v))
        return {k: (b[i], v[i]) for i, k in enumerate(("operators", "input", "intermediates"))}

    def checkpoint_write(self, directory) -> int:
        """Writes the last run's stored models, truncations, bases and wave as the
        reference's checkpoint files (sysblocks<i>, systruns<i>, sysbs<i>, env...,
        eigvec1) into `directory`; returns the number of files."""
        return self._check(self.L.tsc_checkpoint_write(self.h, os.fsencode(directory)))

    def checkpoint_read(self, directory):
        """Loads such a file set; get_ground_state(..., resume=True) continues from it."""
        self._check(self.L.tsc_checkpoint_read(self.h, os.fsencode(directory)))

    def set_resident_limit(self, nbytes: int):
        """Device bytes the stored block models may hold before the least recently
        used move to host memory (< 0: 45 % of the device, the default; 0: all)."""
        self._check(self.L.tsc_set_resident_limit(self.h, int(nbytes)))

    def spill_stats(self):
        """{spills, restores, bytes, seconds, resident_bytes, limit_bytes} of the stored models."""
        sp, rs, rb, lb = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        by, sec = ctypes.c_double(), ctypes.c_double()
        self._check(self.L.tsc_spill_stats(self.h, ctypes.byref(sp), ctypes.byref(rs), ctypes.byref(by),
                                           ctypes.byref(sec), ctypes.byref(rb), ctypes.byref(lb)))
        return {"spills": sp.value, "restores": rs.value, "bytes": by.value, "seconds": sec.value,
                "resident_bytes": rb.value, "limit_bytes": lb.value}

    def set_spill_directory(self, directory, host_bytes):
        """Disk tier under the host spill: spilled models past host_bytes of host
        memory go to files in `directory` (None: no disk tier)."""
        d = os.fsencode(directory) if directory else None
        self._check(self.L.tsc_set_spill_directory(self.h, d, int(host_bytes)))

    def disk_spill_stats(self):
        """{writes, reads, bytes, seconds, host_bytes} of the disk tier."""
        w, r, hb = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        by, sec = ctypes.c_double(), ctypes.c_double()
        self._check(self.L.tsc_disk_spill_stats(self.h, ctypes.byref(w), ctypes.byref(r), ctypes.byref(by),
                                                ctypes.byref(sec), ctypes.byref(hb)))
        return {"writes": w.value, "reads": r.value, "bytes": by.value, "seconds": sec.value, "host_bytes": hb.value}

    def blocksparse_set(self, problems):
        """Block-sparse batch (tsc_blocksparse_set): `problems` is a list of
        blocksparse.Problem; returns (psi length, algorithmic flops of one
        application, flops executed)."""
        from .blocksparse import pack
        return self.blocksparse_set_packed(*pack(problems))

    def blocksparse_set_packed(self, nprob, ints, data):
        """blocksparse_set on problems already in pack()'s layout."""
        ints = np.ascontiguousarray(ints, np.int32)
        data = np.ascontiguousarray(data, np.complex128)
        dim, flops, xflops = ctypes.c_longlong(), ctypes.c_double(), ctypes.c_double()
        self._check(self.L.tsc_blocksparse_set(self.h, nprob, _iptr(ints), len(ints), _dptr(data), len(data),
                                               ctypes.byref(dim), ctypes.byref(flops), ctypes.byref(xflops)))
        return dim.value, flops.value, xflops.value

    def blocksparse_apply(self, d_in: int, d_out: int, mode: int = 0):
        """Applies the batch on device pointers (context stream)."""
        self._check(self.L.tsc_blocksparse_apply(self.h, ctypes.c_void_p(d_in), ctypes.c_void_p(d_out), int(mode)))

    def set_autotune(self, on: bool):
        """FP64 H.psi schedule autotuner (on by default; off = fixed schedule)."""
        self._check(self.L.tsc_set_autotune(self.h, 1 if on else 0))

    def autotune_table(self):
        """{size class (floor log2 GFLOP): ms per GFLOP of TUNE_CANDIDATES,
        None where not timed}."""
        cls = (ctypes.c_int * 64)()
        ms = (ctypes.c_double * 256)()
        n = self._check(self.L.tsc_autotune_table(self.h, cls, ms, 64))
        return {cls[i]: [ms[4 * i + c] if ms[4 * i + c] >= 0 else None for c in range(4)] for i in range(min(n, 64))}

    TUNE_CANDIDATES = (("32x32", 4), ("32x32", 8), ("64x32", 8), ("32x64", 8))   # (CTA tile, waves)

    def autotune_superblock(self, reps: int = 3):
        """Times every candidate H.psi schedule on the current superblock and keeps
        the fastest; returns its (CTA tile, waves)."""
        return self.TUNE_CANDIDATES[self._check(self.L.tsc_autotune_superblock(self.h, int(reps)))]

    def hpsi_noalloc(self, d_in: int, d_out: int):
        """H.psi on device pointers that allocates nothing (scratch: a fixed 64 MiB
        device array shared by all calls; see include/tsc_gpu.h)."""
        self._check(self.L.tsc_hpsi_noalloc(self.h, ctypes.c_void_p(d_in), ctypes.c_void_p(d_out)))

    @property
    def stream(self) -> int:
        """cudaStream_t of this context (device-pointer calls are enqueued on it)."""
        return self.L.tsc_stream(self.h) or 0

    def hpsi_stats(self):
        ms, rf, ef, nl = ctypes.c_double(), ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        self._check(self.L.tsc_hpsi_stats(self.h, ctypes.byref(ms), ctypes.byref(rf), ctypes.byref(ef), ctypes.byref(nl)))
        return {"device_ms": ms.value, "ref_flops": rf.value, "exec_flops": ef.value, "launches": nl.value}

    def lanczos_memo_new(self, vec, lanzero):
        x = np.ascontiguousarray(vec, np.complex128).copy()
        it, e0 = ctypes.c_int(), ctypes.c_double()
        self._check(self.L.tsc_lanczos(self.h, _dptr(x), lanzero, ctypes.byref(it), ctypes.byref(e0)))
        return x, e0.value, it.value

    def get_truncation_operator(self, side, vec, kept_min, kept_max, trun_err):
        """side 0: sys density matrix (den_mat.f90:106), 1: env (den_mat.f90:146)."""
        x = np.ascontiguousarray(vec, np.complex128)
        ns = ctypes.c_int()
        err, ent, entm = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        ti, tn, td, tc = P(ctypes.c_int)(), ctypes.c_longlong(), P(ctypes.c_double)(), ctypes.c_longlong()
        spec = np.zeros(max(1, int(self.dim)), np.float64)
        self._check(self.L.tsc_truncate(self.h, side, _dptr(x), kept_min, kept_max, trun_err, ctypes.byref(ns),
                                        ctypes.byref(err), ctypes.byref(ent), ctypes.byref(entm), ctypes.byref(ti),
                                        ctypes.byref(tn), ctypes.byref(td), ctypes.byref(tc), _dptr(spec), len(spec)))
        ints = np.ctypeslib.as_array(ti, shape=(tn.value,)).copy()
        data = (np.ctypeslib.as_array(td, shape=(2 * tc.value,)).copy().view(np.complex128)
                if tc.value else np.zeros(0, np.complex128))
        trun = Block.read(Cursor(ints, data))
        return {"trun": trun, "num_state": ns.value, "err": err.value, "entropy": ent.value,
                "entropy_mult": entm.value, "spectrum": spec}

    def get_density_matrix(self, side, waves, levels=None):
        """Get_density_matrix_sys_new (side 0, den_mat.f90:103-138) / _env_new (side 1,
        den_mat.f90:143-177) on the current superblock: `waves` is one vector or a
        list of vectors (levels of them; the reference averages the first two when
        levels >= 2).  Returns the density matrix as a Block."""
        ws = [waves] if np.ndim(waves) == 1 else list(waves)
        levels = len(ws) if levels is None else int(levels)
        x = np.ascontiguousarray(np.concatenate([np.asarray(w, np.complex128) for w in ws[:2]]))
        ti, tn, td, tc = P(ctypes.c_int)(), ctypes.c_longlong(), P(ctypes.c_double)(), ctypes.c_longlong()
        self._check(self.L.tsc_density_matrix(self.h, side, _dptr(x), levels, ctypes.byref(ti), ctypes.byref(tn),
                                              ctypes.byref(td), ctypes.byref(tc)))
        ints = np.ctypeslib.as_array(ti, shape=(tn.value,)).copy()
        data = (np.ctypeslib.as_array(td, shape=(2 * tc.value,)).copy().view(np.complex128)
                if tc.value else np.zeros(0, np.complex128))
        return Block.read(Cursor(ints, data))

    def truncation_from_density(self, den: Block, kept_min, kept_max, trun_err):
        """Get_truncation_operator (den_mat.f90:190-418) on a given density matrix."""
        ints, data = [], []
        den.write(ints, data)
        ints, data = pack(ints, data)
        ns = ctypes.c_int()
        err, ent, entm = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        ti, tn, td, tc = P(ctypes.c_int)(), ctypes.c_longlong(), P(ctypes.c_double)(), ctypes.c_longlong()
        spec = np.zeros(max(1, int(den.dim)), np.float64)
        self._check(self.L.tsc_truncation_operator(self.h, _iptr(ints), len(ints), _dptr(data), len(data), kept_min,
                                                   kept_max, trun_err, ctypes.byref(ns), ctypes.byref(err),
                                                   ctypes.byref(ent), ctypes.byref(entm), ctypes.byref(ti),
                                                   ctypes.byref(tn), ctypes.byref(td), ctypes.byref(tc), _dptr(spec),
                                                   len(spec)))
        ints = np.ctypeslib.as_array(ti, shape=(tn.value,)).copy()
        data = (np.ctypeslib.as_array(td, shape=(2 * tc.value,)).copy().view(np.complex128)
                if tc.value else np.zeros(0, np.complex128))
        return {"trun": Block.read(Cursor(ints, data)), "num_state": ns.value, "err": err.value,
                "entropy": ent.value, "entropy_mult": entm.value, "spectrum": spec}

    def get_hamiltonian(self, side, model: Model, basis: Basis, trun: Block, sys_len, env_len, mshift=0):
        """Get_Hamiltonian_Sys (side 0) / Get_Hamiltonian_Env (side 1): enlarge + renormalise."""
        ints, data = [], []
        model.write(ints, data)
        basis.write(ints, data)
        trun.write(ints, data)
        ints, data = pack(ints, data)
        oi, on, od, oc = P(ctypes.c_int)(), ctypes.c_longlong(), P(ctypes.c_double)(), ctypes.c_longlong()
        self._check(self.L.tsc_renormalize(self.h, side, sys_len, env_len, mshift, _iptr(ints), len(ints), _dptr(data),
                                           len(data), ctypes.byref(oi), ctypes.byref(on), ctypes.byref(od),
                                           ctypes.byref(oc)))
        gi = np.ctypeslib.as_array(oi, shape=(on.value,)).copy()
        gd = (np.ctypeslib.as_array(od, shape=(2 * oc.value,)).copy().view(np.complex128)
              if oc.value else np.zeros(0, np.complex128))
        return Model.read(Cursor(gi, gd))

    def wave_trans(self, direction, sys_bs: Basis, env_bs: Basis, sys_trun: Block, env_trun: Block, old: Wave,
                   new_layout: Wave) -> Wave:
        """direction 0: wave_trans_LR, 1: wave_trans_RL."""
        ints, data = [], []
        sys_bs.write(ints, data)
        env_bs.write(ints, data)
        sys_trun.write(ints, data)
        env_trun.write(ints, data)
        old.write(ints, data)
        new_layout.write(ints, data, with_data=False)
        ints, data = pack(ints, data)
        out = np.zeros(new_layout.dim, np.complex128)
        self._check(self.L.tsc_wave_transform(self.h, direction, _iptr(ints), len(ints), _dptr(data), len(data),
                                              _dptr(out)))
        return Wave(new_layout.sys_len, new_layout.env_len, new_layout.secs, out)

    # ------------------------------------------------------------------ full run
    def get_ground_state(self, kept_min, kept_warm, sweeps, lanzero=-1.0, seed=1, capture_step=-1, max_steps=100000,
                         warmup_only=False, final_half_sweep=False, resume=False, max_solves=0,
                         lanzero_warmup=-1.0, final_stop=0):
        """Get_Ground_State (main.f90:114-209); resume=True continues with the sweeps
        from the state checkpoint_read loaded (no warm-up, no first half sweeps);
        max_solves > 0 stops the run after that many DMRG steps; lanzero_warmup > 0
        sets the warm-up's tolerance alone; final_stop > 0 ends the final half
        sweep at that label instead of 5 Num_site / 6 - 1."""
        self._check(self.L.tsc_set_capture(self.h, capture_step))
        sk = (ctypes.c_int * max(1, len(sweeps)))(*sweeps)
        cfg = _lib.SweepConfig(kept_min, kept_warm, len(sweeps), sk, lanzero, seed, 1 if warmup_only else 0,
                               1 if final_half_sweep else 0, 1 if resume else 0, int(max_solves),
                               float(lanzero_warmup), int(final_stop))
        logs = (_lib.StepLog * max_steps)()
        n = self._check(self.L.tsc_dmrg_run(self.h, ctypes.byref(cfg), logs, max_steps))
        out = []
        for k in range(min(n, max_steps)):
            s = logs[k]
            out.append({f: getattr(s, f) for f, _ in _lib.StepLog._fields_})
        return out

    def measure_density(self):
        """<n_i> of every site in the last ground state of get_ground_state
        (measure_operator_dia, measure.f90:3-62)."""
        out = np.zeros(self.Nx * self.Ny, dtype=np.float64)
        self._check(self.L.tsc_measure_density(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(out)))
        return out

    def measure_density_cor(self, site=None):
        """<n_site n_j> (j = 1..Nx*Ny; zero where the reference computes nothing)
        of the last ground state (Get_density_cor, measure.f90:2525-2681).  The
        default site is the reference's xi1 = (Nx/4)*Ny + 2 - Ny (main.f90:255),
        which needs the wave left by get_ground_state(..., final_half_sweep=True)."""
        if site is None:
            site = (self.Nx // 4) * self.Ny + 2 - self.Ny
        out = np.zeros(self.Nx * self.Ny, dtype=np.float64)
        self._check(self.L.tsc_measure_density_cor(self.h, int(site),
                                                   out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(out)))
        return out

    # kinds of measure_correlation (TSC_COR_* in include/tsc_gpu.h)
    COR_KINDS = {"density": 0, "spin": 1, "electron": 2}

    def measure_correlation(self, kind, site=None):
        """Row `site` of one of the three correlation matrices main.f90 writes
        (Get_density_cor, measure.f90:2525-2681): "density" <n_site n_j>
        (main.f90:299), "spin" <S_site . S_j> (st_sd x st_sd, Flags 'B',
        main.f90:275) or "electron" sum_s <c+_site,s c_j,s> (st_elec_up x
        st_elec_down, Flags 'F', main.f90:288), complex as the reference writes
        them (main.f90:282, 294; the density kind's imaginary part is 0).  Same
        site default, partners and layout as measure_density_cor."""
        if site is None:
            site = (self.Nx // 4) * self.Ny + 2 - self.Ny
        n = self.Nx * self.Ny
        out = np.zeros(2 * n, dtype=np.float64)
        self._check(self.L.tsc_measure_correlation(self.h, self.COR_KINDS[kind], int(site),
                                                   out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n))
        return out[0::2] + 1j * out[1::2]

    def measure_pair_correlation(self, xc1, xc2=None, ij=0, ij1=1):
        """Singlet pair correlations (Get_mSCOP_Operator_Cor0, Flags 'S0',
        measure.f90:2683-2834; main.f90:259-262 calls it with xc1 = xi1, xc2 =
        xj1, ij = 0, ij1 = 1 | 3 | 5): [(s1, s2, s3, s4, value)] for the bond
        (xc1, neib(xc1, ij1)) against the bonds (s3, neib(s3, 1|3|5)) the
        reference visits; xc2 defaults to the reference's xj1 = 3 Nx / 4 Ny + 2,
        capped at the lattice."""
        if xc2 is None:
            xc2 = min(self.Nx * 3 // 4 * self.Ny + 2, self.Nx * self.Ny)
        cap = 256
        while True:
            bonds = np.zeros(4 * cap, dtype=np.int32)
            vals = np.zeros(2 * cap, dtype=np.float64)
            n = self._check(self.L.tsc_measure_pair_correlation(
                self.h, int(xc1), int(xc2), int(ij), int(ij1), bonds.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                vals.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), cap))
            if n <= cap:
                break
            cap = n
        return [(int(bonds[4 * k]), int(bonds[4 * k + 1]), int(bonds[4 * k + 2]), int(bonds[4 * k + 3]),
                 complex(vals[2 * k], vals[2 * k + 1])) for k in range(n)]

    def capture(self):
        ti, tn, td, tc = P(ctypes.c_int)(), ctypes.c_longlong(), P(ctypes.c_double)(), ctypes.c_longlong()
        sl, el = ctypes.c_int(), ctypes.c_int()
        self._check(self.L.tsc_get_capture(self.h, ctypes.byref(ti), ctypes.byref(tn), ctypes.byref(td),
                                           ctypes.byref(tc), ctypes.byref(sl), ctypes.byref(el)))
        ints = np.ctypeslib.as_array(ti, shape=(tn.value,)).copy()
        data = np.ctypeslib.as_array(td, shape=(2 * tc.value,)).copy().view(np.complex128)
        return ints, data, sl.value, el.value


def run_parameter_points(points, sweep, precision=0, device=0, workers=None, measure=False):
    """Independent ground-state searches, one per model-parameter dict of
    `points` (keyword arguments of Context), on one GPU at the same time.  Small
    systems leave most of the GPU idle; each point gets its own context (stream,
    device-memory arena, eigensolver lanes) driven from its own host thread, so
    their kernels interleave on the device.  `sweep` holds the keyword arguments
    of get_ground_state.  Returns, per point, the step records (and the site
    densities when `measure` is set)."""
    from concurrent.futures import ThreadPoolExecutor

    def one(p):
        ctx = Context(device=device, **p)
        try:
            ctx.set_precision(precision)
            steps = ctx.get_ground_state(**sweep)
            return (steps, ctx.measure_density()) if measure else steps
        finally:
            ctx.close()

    with ThreadPoolExecutor(max_workers=workers or len(points)) as ex:
        return list(ex.map(one, points))
