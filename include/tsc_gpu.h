/*
 * tsc_gpu.h -- C-ABI of the B200 superblock engine for the SU(2) two-site DMRG of
 * the t1-t2-J1-J2 model on triangular cylinders (drop-in for the hot path of
 * hyx15903/TSC_Tri_t1t2J1J2, DMRG_code/*.f90).
 *
 * Layout contract (the reference's derived types flattened, DMRG_code/common.f90:84-156):
 *   Block  (Total_Block):  ints  [len, num, dim, up_dif, down_dif]
 *                          then num x [num_up, num_down, down_dif, row_dim, sdim]
 *                          data  concatenated column-major complex128 sub-block matrices
 *   Basis  (Total_Basis):  ints  [len, num, dim], num x [new_num_up, new_num_down, dim, npieces],
 *                          then all pieces x [bl_num_up, bl_num_down, st_num_up, st_num_down, spos, sdim]
 *   Wave   (Wavefunction): ints  [sys_len, env_len, num, dim]
 *                          then num x [sys_num_up, sys_num_down, env_num_up, env_num_down, sys_dim, env_dim]
 *                          data  concatenated column-major complex128 sectors
 *   Model  (Total_Model):  ints  [len, nops], Block ham, then for op = 1..nops the four
 *                          Blocks elec_up, elec_down, spin_sd, num_sn of boundary site op
 * Complex data is interleaved (re, im) double pairs, in the element order of the
 * Fortran mat/vec arrays.  The caller owns every host buffer; the library owns
 * device-resident copies per context and never frees caller memory.
 *
 * Every entry point returns 0 on success or a negative TSC_E* status; it never
 * aborts the host process.  tsc_last_error() gives a one-line reason.
 * One host thread per context; distinct contexts are independent.
 */
#ifndef TSC_GPU_H
#define TSC_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define TSC_OK 0
#define TSC_E_ARG -1        /* bad argument / descriptor */
#define TSC_E_QN -2         /* quantum-number mismatch (reference stops, get_sys.f90:3166-3168) */
#define TSC_E_CUDA -3       /* CUDA runtime / library failure */
#define TSC_E_STATE -4      /* call out of order (no superblock set, ...) */
#define TSC_E_NOMEM -5      /* device allocation failed */
#define TSC_E_LIMIT -6      /* size above a documented limit */

/* Model: lattice and couplings (main.f90:59-99, dmrg_setup dmrg_sub.f90:334-644). */
typedef struct tsc_model_config {
  int Nx, Ny;              /* YC cylinder: Ny legs periodic in y, Nx columns open in x */
  double t1, t2, J1, J2;   /* jt=-t*sqrt(2), jz=J, jd=-sqrt(3)*J, jn=-J/4 on bonds 1-6 / 7-12 */
  int delta;               /* inverse hole doping; electrons from main.f90:93-99 */
  int device;              /* CUDA device ordinal */
} tsc_model_config;

/* Sweep schedule (main.f90:114-209, dmrg_sub.f90:974-1465). */
typedef struct tsc_sweep_config {
  int kept_min;            /* den_mat.f90:299-318 */
  int kept_max_warmup;     /* kept_max of warm-up and the first two half sweeps */
  int nsweeps;
  const int* sweep_kept_max;   /* nsweeps entries */
  double lanzero;          /* >0: Lanczos tolerance in every phase; <=0: reference schedule */
  unsigned long long seed; /* random initial states (block.f90:1154-1180 stand-in) */
  int warmup_only;         /* 1: stop after warm_up_point (dmrg_sub.f90:974-1147) */
  int final_half_sweep;    /* 1: end with left_to_right up to 5*Num_site/6 (main.f90:205-206),
                            * the position where the reference measures */
  int resume;              /* 1: skip the warm-up and the two half sweeps and run the sweeps
                            * from the state tsc_checkpoint_read loaded (the reference's
                            * restart1 = 1 from restart.dat, main.f90:36-38, 147-174) */
  int max_solves;          /* > 0: stop the run after this many Lanczos solves (DMRG steps);
                            * 0: run the whole schedule */
  double lanzero_warmup;   /* > 0: Lanczos tolerance of the warm-up steps alone (else as lanzero) */
  int final_stop;          /* > 0: last label of the final half sweep (0: the reference's
                            * 5*Num_site/6 - 1, main.f90:205-206) */
} tsc_sweep_config;

/* One record per Lanczos solve (eigen.f90:169-173, den_mat.f90:342-350). */
typedef struct tsc_step_log {
  int phase;               /* 0 warm-up, 1 left_to_right, 2 right_to_left */
  int sys_len, env_len;
  double e0;
  int lanczos_iters;
  int num_state;
  double trun_err, entropy, entropy_mult;
  int hpsi_calls;
  double hpsi_seconds;     /* device time of the H.psi launches of this solve */
  double hpsi_flops;       /* algorithmic flops (reference association order) */
  double step_seconds;     /* wall time of the whole DMRG step on the device */
  /* wall time of the step's parts: superblock set-up (hmerge + task lists),
   * Lanczos (H.psi included), density matrix + truncation, block growth +
   * renormalisation, wave transformation */
  double set_seconds, lanczos_seconds, truncate_seconds, grow_seconds, wave_seconds;
  /* split-precision form only (else 0): iterations on the BF16-sliced H.psi
   * and their last Ritz value, before the FP64 iterations that finish the solve */
  int split_iters;
  double split_e0;
} tsc_step_log;

typedef struct tsc_ctx tsc_ctx;

/* Replaces the global set-up of main.f90:29-99 (Get_Lattice, site operators,
 * couplings, dmrg_setup0). */
int tsc_create(tsc_ctx** ctx, const tsc_model_config* cfg);
int tsc_destroy(tsc_ctx* ctx);
const char* tsc_last_error(tsc_ctx* ctx);
int tsc_tot_num_up(tsc_ctx* ctx);

/* Uploads one superblock: what model_wave(sys,env,sys_bs,env_bs,...) receives
 * (get_sys.f90:6915) -- the sys and env Total_Model (ham + boundary operators)
 * and the enlarged bases -- followed by the Wave layout of psi that fixes the
 * sector list (Super_Basis, block.f90:2194-2247; its data part is ignored).
 * Builds hmerge's merged operators (get_sys.f90:7398-7626) and the H.psi task
 * list on the device. */
int tsc_superblock_set(tsc_ctx* ctx, int sys_len, int env_len, const int* ints, long long nints,
                       const double* data, long long ncplx);
long long tsc_superblock_dim(tsc_ctx* ctx);

/* model_wave (get_sys.f90:6915-7393): out = H in, host complex128 buffers of
 * tsc_superblock_dim() elements (host->device and device->host copies included). */
int tsc_hpsi(tsc_ctx* ctx, const double* in, double* out);
/* Same on device pointers, enqueued on the context stream (no host copies).
 * In the TSC_SPLIT_BF16 form the call also waits for its launches and reads the
 * context's device status word: a bounded wait of the split kernel that ran out
 * (see tsc_set_split_wait_limit) is returned as TSC_E_CUDA, the output then
 * being incomplete. */
int tsc_hpsi_device(tsc_ctx* ctx, const void* d_in, void* d_out);

/* lanczos_memo_new (eigen.f90:4-199, levels=1): psi_inout is the start vector
 * on entry and the normalised ground state on exit (host buffer). */
int tsc_lanczos(tsc_ctx* ctx, double* psi_inout, double lanzero, int* iters, double* e0);

/* Get_density_matrix_{sys,env}_new + Get_truncation_operator (den_mat.f90:4-418)
 * on the ground state psi (host buffer).  side 0 = sys, 1 = env.  Writes the
 * kept count, discarded weight, entropies; the truncation operator U in the Block
 * layout is returned through *trun_ints / *trun_data (library-owned, valid until
 * the next call on ctx). spectrum (may be NULL) receives the sorted normalised
 * density-matrix spectrum (up to spectrum_cap entries). */
int tsc_truncate(tsc_ctx* ctx, int side, const double* psi, int kept_min, int kept_max,
                 double trun_err, int* num_state, double* err, double* entropy,
                 double* entropy_mult, const int** trun_ints, long long* ntrun_ints,
                 const double** trun_data, long long* ntrun_cplx, double* spectrum,
                 long long spectrum_cap);

/* The two halves of tsc_truncate as the reference calls them.
 * tsc_density_matrix: Get_density_matrix_sys_new (side 0, den_mat.f90:103-138) /
 * Get_density_matrix_env_new (side 1, den_mat.f90:143-177) on the current
 * superblock.  psi holds min(levels, 2) waves one after the other (host buffer,
 * tsc_superblock_dim() elements each): levels = 1 takes the normalised wave;
 * levels >= 2 averages the density matrices of the first two waves,
 * unnormalised, as the reference does.  The density matrix (one square
 * sub-block per wave sector, the reference's sys_den / env_den) is returned in
 * the Block layout through *den_ints / *den_data (library-owned, valid until the
 * next call on ctx).
 * tsc_truncation_operator: Get_truncation_operator (den_mat.f90:190-418) on a
 * density matrix given in the Block layout (square sub-blocks, down_dif 0);
 * outputs as tsc_truncate. */
int tsc_density_matrix(tsc_ctx* ctx, int side, const double* psi, int levels, const int** den_ints,
                       long long* nden_ints, const double** den_data, long long* nden_cplx);
int tsc_truncation_operator(tsc_ctx* ctx, const int* den_ints, long long nden_ints, const double* den_data,
                            long long nden_cplx, int kept_min, int kept_max, double trun_err, int* num_state,
                            double* err, double* entropy, double* entropy_mult, const int** trun_ints,
                            long long* ntrun_ints, const double** trun_data, long long* ntrun_cplx, double* spectrum,
                            long long spectrum_cap);

/* Get_Hamiltonian_Sys / Get_Hamiltonian_Env (get_sys.f90:4-592): enlarges the
 * block of the given side with one site (update_block_*, update_site_*,
 * Get_hamiltonian_*) and renormalises every operator with U (update_trun_dia /
 * update_trun_ndia, block.f90:3465-3683).  Inputs: the Model, the enlarged Basis
 * and the truncation Block.  mshift is the reference's mshift for the env side.
 * The grown Model is returned through *out_ints / *out_data (library-owned). */
int tsc_renormalize(tsc_ctx* ctx, int side, int sys_len, int env_len, int mshift,
                    const int* ints, long long nints, const double* data, long long ncplx,
                    const int** out_ints, long long* nout_ints, const double** out_data,
                    long long* nout_cplx);

/* wave_trans_LR / wave_trans_RL (dmrg_sub.f90:1471-1789): dir 0 = LR, 1 = RL.
 * ints/data: sys Basis, env Basis, sys truncation Block, env truncation Block,
 * old Wave, new Wave layout (data ignored).  new_out receives the new wave. */
int tsc_wave_transform(tsc_ctx* ctx, int dir, const int* ints, long long nints, const double* data,
                       long long ncplx, double* new_out);

/* Whole ground-state search on the device (Get_Ground_State, main.f90:114-209):
 * warm-up, two half sweeps and nsweeps full sweeps, blocks resident in HBM.
 * Writes up to max_steps records; returns the number of Lanczos solves. */
int tsc_dmrg_run(tsc_ctx* ctx, const tsc_sweep_config* sweep, tsc_step_log* log, int max_steps);

/* Device memory the stored block models of tsc_dmrg_run may hold.  The
 * reference writes every model to disk after each step and reads it back when
 * the sweep returns (model_to_disk / block_to_disk, block.f90:1715-1900,
 * dmrg_sub.f90:1119-1139); here models stay in HBM while the resident ones fit
 * under this many bytes, and past it the least recently used ones move to host
 * memory and return to the device when the sweep reads them (results are
 * unchanged: the data round-trips exactly).  bytes < 0 (the default): 45 % of
 * the device's memory in the FP64 form, 30 % in the split form (whose
 * pre-sliced operand views need room beside the superblock); 0: every stored
 * model lives in host memory between its uses. */
int tsc_set_resident_limit(tsc_ctx* ctx, long long bytes);
/* Spill counters of the stored models since the context was created: models
 * moved to host memory, models brought back, bytes moved both ways and the wall
 * seconds spent, the bytes now resident and the limit in force. */
int tsc_spill_stats(tsc_ctx* ctx, long long* spills, long long* restores, double* bytes, double* seconds,
                    long long* resident_bytes, long long* limit_bytes);
/* Disk tier under the host spill, the reference's own out-of-core storage
 * (model_to_disk / block_to_disk, block.f90:1715-1900): once the spilled
 * models' host copies pass host_bytes, the least recently used go to one file
 * each in directory dir (created by the caller) and come back, through host
 * memory, when the sweep reads them; each file is removed when its model comes
 * back or the context is destroyed.  host_bytes < 0 or dir NULL/empty: no disk
 * tier (the default).  Results are unchanged (the data round-trips exactly). */
int tsc_set_spill_directory(tsc_ctx* ctx, const char* dir, long long host_bytes);
/* Models written to and read from the disk tier, bytes moved both ways, wall
 * seconds, and the host bytes the spilled models hold now. */
int tsc_disk_spill_stats(tsc_ctx* ctx, long long* writes, long long* reads, double* bytes, double* seconds,
                         long long* host_bytes);

/* <n_i> of every site in the last ground state of tsc_dmrg_run, sites 1..Nx*Ny
 * in the lattice order (measure_operator_dia with num_elec, measure.f90:3-62,
 * main.f90:268): the site operator is carried into the system / environment
 * block through the run's stored bases and truncations (Get_sys_oper_dia,
 * get_sys.f90:1147-1277) and measured on the last wavefunction.  Writes nsites
 * >= Nx*Ny values; returns the number written. */
int tsc_measure_density(tsc_ctx* ctx, double* out, int nsites);

/* Density-density correlations <n_site n_j> of the last ground state
 * (Get_density_cor with oper1 = oper2 = num_elec, Flags 'B', xi = xj = site,
 * measure.f90:2525-2681, main.f90:299).  `site` must lie in the system block of
 * the last wavefunction (1 <= site <= sys_len - 1; the reference calls it with
 * xi1 = (Nx/4)*Ny + 2 - Ny after the final half sweep that tsc_sweep_config's
 * final_half_sweep runs).  The partners are the reference's: j = site + Ny,
 * site + 2 Ny, ... up to min(Nx*Ny, Nx*Ny - Nx*Ny/6 + Ny).  Writes nsites >=
 * Nx*Ny values, out[j-1] = Re <n_site n_j> for those j and 0 elsewhere (as the
 * reference's zero-initialised correlation matrix row); returns Nx*Ny. */
int tsc_measure_density_cor(tsc_ctx* ctx, int site, double* out, int nsites);

/* The three two-site correlations main.f90 measures with Get_density_cor
 * (measure.f90:2525-2681), selected by kind:
 *   TSC_COR_DENSITY   <n_site n_j>            (num_elec, Flags 'B'; main.f90:299)
 *   TSC_COR_SPIN      <S_site . S_j>          (st_sd x st_sd, Flags 'B', rank 1; main.f90:275)
 *   TSC_COR_ELECTRON  sum_s <c+_site,s c_j,s> (st_elec_up x st_elec_down, Flags 'F',
 *                                              rank 1/2; main.f90:288)
 * Operators of nonzero rank travel into the blocks by the reference's ndia
 * transport (Get_sys_oper_ndia / Change_sys_oper_ndia, get_sys.f90:1536-1723),
 * results carry the reference's scale sqrt(1+K)*(K==2 ? -1 : 1)
 * (measure.f90:2586-2587).  Same site range and partners as
 * tsc_measure_density_cor; out holds 2*nsites doubles, the complex value of
 * partner j as out[2(j-1)] (real) and out[2(j-1)+1] (imaginary), as main.f90
 * writes both parts (main.f90:282, 294); the density kind's imaginary part is
 * written as 0.  Returns Nx*Ny. */
#define TSC_COR_DENSITY 0
#define TSC_COR_SPIN 1
#define TSC_COR_ELECTRON 2
int tsc_measure_correlation(tsc_ctx* ctx, int kind, int site, double* out, int nsites);

/* Singlet pair correlations <O+_(s1 s2) O_(s3 s4)> of the last ground state,
 * O+_ab = (c+_a,up c+_b,dn - c+_a,dn c+_b,up)/sqrt(2) (Get_mSCOP_Operator_Cor0 with
 * Flags 'S0' from the label main.f90:259-262 reaches, measure.f90:2683-2834):
 * first bond (xc1, neib(xc1, ij1)), which must lie in the system block of the
 * wave; second bonds (s3, neib(s3, 1|3|5)) for s3 = xc1 + Ny + ij, ... up to
 * xc2 <= Nx*Ny, in the system block (Get_sys_two / Get_sys_two1) and then in the
 * environment block (Get_SCOP_Operator_Env and the block-block correlator,
 * value conjugated as the reference writes it).  Record k: bonds[4k..4k+3] =
 * s1 s2 s3 s4, values[2k], values[2k+1] = real, imaginary part; at most cap
 * records are written.  Returns the number of records (which may exceed cap). */
int tsc_measure_pair_correlation(tsc_ctx* ctx, int xc1, int xc2, int ij, int ij1, int* bonds, double* values,
                                 int cap);

/* Checkpoint in the reference's file format (names dmrg_sub.f90:657-709):
 * writes into directory dir, for every model, truncation and basis the last
 * tsc_dmrg_run stored, the files sysblocks<i> / envblocks<i> (model_to_disk,
 * block.f90:1802-1845), systruns<i> / envtruns<i> (truns_to_disk, :1936-1956),
 * sysbs<i> / envbs<i> (basis_to_disk, :1983-2026, formatted) and eigvec1, the
 * last wavefunction (wave_to_disk, :1547-1576).  Unformatted files are Fortran
 * sequential records with 4-byte length markers, 4-byte integers and 16-byte
 * complex values, as gfortran and ifort write them.  Returns the number of
 * files written.  A run that ended with a full sweep leaves the wave at the
 * left end, where a resumed run starts. */
int tsc_checkpoint_write(tsc_ctx* ctx, const char* dir);
/* Reads such a file set (all lengths 1..Nx*Ny present in dir) into the
 * context; tsc_dmrg_run with resume = 1 then continues from it. */
int tsc_checkpoint_read(tsc_ctx* ctx, const char* dir);

/* Serialises the superblock of the most recent step of tsc_dmrg_run whose
 * global solve index equals capture_step (set before the run with
 * tsc_set_capture); layout = tsc_superblock_set input with psi data. */
int tsc_set_capture(tsc_ctx* ctx, int capture_step);
int tsc_get_capture(tsc_ctx* ctx, const int** ints, long long* nints, const double** data,
                    long long* ncplx, int* sys_len, int* env_len);

/* Timing of the last tsc_hpsi / tsc_hpsi_device: device milliseconds of its
 * grouped-GEMM launches (CUDA events on the context stream), the algorithmic
 * flops of one model_wave in the reference's GEMM association order, the flops
 * the kernels execute (fewer: shared left products), and the launch count. */
int tsc_hpsi_stats(tsc_ctx* ctx, double* device_ms, double* ref_flops, double* exec_flops, int* launches);

/* The context's CUDA stream (cudaStream_t as void*): device-pointer calls are
 * enqueued on it, so callers can order their own work and time it with events. */
void* tsc_stream(tsc_ctx* ctx);

/* Arithmetic of the H.psi sector GEMMs (the reference computes everything in
 * complex FP64 and has no such switch).  TSC_FP64: complex FP64 throughout.
 * TSC_SPLIT_BF16: every FP64 operand split into three BF16 slices multiplied
 * on the tensor cores with FP32 accumulators restarted every 128 of the inner
 * dimension and summed in FP64 (a few 1e-7 relative error per H.psi; the
 * operator slices are built when the superblock is set, see
 * tsc_set_split_view_sharing); Lanczos iterates on that H.psi until successive
 * Ritz values agree to split_tol relative (<= 0 keeps the current value, 1e-11
 * at creation: on YC4x12 whole runs 1e-10, 1e-9 and 1e-8 left more work to the
 * FP64 iterations and ended farther from FP64), then runs the reference's FP64
 * iterations from that vector, with
 * the reference's stop unless tsc_set_split_refinement asks for a residual
 * bound, so the energy and vector it returns are FP64 results.  Orthogonalisation, tridiagonal solve,
 * density-matrix eigensolver, renormalisation and wave transforms stay FP64,
 * and so do the warm-up steps of tsc_dmrg_run.  Takes effect from the next
 * superblock set. */
#define TSC_FP64 0
#define TSC_SPLIT_BF16 1
int tsc_set_precision(tsc_ctx* ctx, int mode, double split_tol);

/* How the FP64 iterations that finish a TSC_SPLIT_BF16 solve stop (no
 * counterpart in the reference): 0 (at creation) uses the reference's own
 * stop, successive Ritz values within lanzero (eigen.f90:101), from the split
 * solve's vector; residual_factor > 0 stops instead when the FP64 Ritz
 * residual ||H psi - E psi|| is <= residual_factor * sqrt(lanzero) (tighter
 * and costlier: 0.1 takes ~4x the FP64 iterations on a YC4x12 sweep). */
int tsc_set_split_refinement(tsc_ctx* ctx, double residual_factor);

/* Pre-sliced operand views of the split-precision task lists of the superblock
 * or block-sparse batch set last (no counterpart in the reference): bytes[0..2]
 * and views[0..2] for the operator views (sliced once per superblock; with the
 * terms' coefficients folded in for a superblock, one view per operator block
 * for a batch, whose coefficients the kernel applies per term), the
 * input-vector views (sliced on every H.psi) and the phase-1 intermediates.
 * All zero in the FP64 form. */
int tsc_split_views(tsc_ctx* ctx, long long* bytes, int* views);

/* Split form only: on = 1 runs the U^H O U renormalisation of block growth
 * (update_trun_dia / update_trun_ndia, block.f90:3465-3683, inside
 * tsc_renormalize and tsc_dmrg_run after the warm-up) on the split kernel too,
 * as eff = (U_l^H O) U_r; 0 (the default) keeps it FP64.  Its ~1e-7 relative
 * error stays in every later Hamiltonian, where no FP64 Lanczos refinement can
 * remove it. */
int tsc_set_split_renormalization(tsc_ctx* ctx, int on);

/* Split form: the FP64 iterations that finish a split solve stop, with the
 * reference's test, when successive Ritz values agree to multiplier * lanzero
 * (1 at creation: the reference's own tolerance; 10 cut a YC4x12 run's FP64
 * iterations from 1,672 to 1,216 but left its final energy 2.3e-10 from the
 * FP64 form's, against 3.2e-11 at 1). */
int tsc_set_split_finish_tolerance(tsc_ctx* ctx, double multiplier);

/* on = 1 (the default): every Lanczos iteration after the first of a solve
 * (eigen.f90:65-98: three-term update, Gram_Schmidt_process, normalisation,
 * H.psi, alpha, the tridiagonal Ritz value and its read-back) is one CUDA graph
 * launch, the graph built once per solve (updated in place when only its
 * parameters change) and replayed with the iteration index; the results are
 * bit-identical to on = 0, which launches every step from the host. */
int tsc_set_lanczos_graph(tsc_ctx* ctx, int on);

/* Split form: shared = 1 (the default) slices every operator sub-block once and
 * lets the kernel's epilogue apply each term's coefficient; shared = 0 slices
 * one copy per term with its coefficient folded in (1-2 % faster H.psi, ~4.5x
 * the memory of the operator slices: 14.3 GB against 3.2 GB on the YC4x24
 * m=4000 superblock, and more slicing when a superblock is set); shared = -1
 * picks shared once the folded copies would pass 4 GiB.  Applies from the next
 * superblock set on. */
int tsc_set_split_view_sharing(tsc_ctx* ctx, int shared);
/* Iterations replayed as graphs since the context was created, and captures that
 * failed (the iteration then ran eagerly and graphs stayed off for the context);
 * reason (may be NULL) receives the last failure's message, NUL-terminated. */
int tsc_lanczos_graph_stats(tsc_ctx* ctx, long long* replays, long long* fallbacks, char* reason, int reason_cap);

/* Poll limit of every bounded mbarrier wait in the split-precision kernel (no
 * counterpart in the reference; default 1<<20, far above any wait of a healthy
 * launch).  A wait that runs out sets the context's status word and the kernel
 * returns; the next split call then reports TSC_E_CUDA and clears the word, and
 * the context stays usable.  0 makes every wait give up at once, which tests of
 * that error path use. */
int tsc_set_split_wait_limit(tsc_ctx* ctx, long long polls);

/* The FP64 H.psi schedule autotuner (on at creation; no counterpart in the
 * reference).  For superblocks of >= 8 GFLOP per H.psi it times candidate
 * schedules (CTA tile of output rows x columns, long term lists split into
 * chunks for 4 or 8 waves of CTAs), one candidate on the first H.psi of each superblock of a
 * size class (log2 GFLOP), and keeps each class's fastest.  Results are the
 * same H.psi up to the summation order of split term lists; off (0) fixes the
 * schedule, so repeated runs are bit-identical. */
int tsc_set_autotune(tsc_ctx* ctx, int on);
/* The autotuner's measurements: for up to max_classes size classes, class[i]
 * (floor log2 of the H.psi GFLOP) and ms_per_gflop[4*i + c] for candidate c =
 * (tile 32x32, 4 waves), (32x32, 8), (64x32, 8), (32x64, 8); negative = not
 * timed yet.
 * Returns the number of classes. */
int tsc_autotune_table(tsc_ctx* ctx, int* cls, double* ms_per_gflop, int max_classes);
/* Times every candidate schedule on the current superblock now (best of reps
 * FP64 H.psi each, on a scratch vector), records them for its size class and
 * keeps the fastest for this superblock; returns that candidate's index. */
int tsc_autotune_superblock(tsc_ctx* ctx, int reps);

/* Block-sparse H.psi on a batch of independent problems, all of them in the
 * same two grouped launches (no counterpart in the reference, which applies
 * model_wave to one superblock at a time; this is the synthetic H.psi of the
 * benchmark list).  Problem p has K sectors; its psi is the sector blocks X_i
 * (d_i x e_i, column-major) one after another, problems one after another, and
 * the output has the same layout.  Left operator sets L_a hold blocks L_a[i]
 * (d_{i+s_a} x d_i), right sets R_b blocks R_b[i] (e_{i+s_b} x e_i), for every i
 * with 0 <= i+s < K.  A term (alpha, a, b), s_a == s_b, adds
 * alpha * L_a[i] X_i R_b[i]^H to Y_{i+s}; sectors no term reaches are zero.
 *   ints, per problem: K, nL, nR, nterms; d_0, e_0, ..., d_{K-1}, e_{K-1};
 *        the shifts s of the left then right sets; per term a, b.
 *   data (complex), per problem: the left sets' blocks (set by set, i
 *        ascending, column-major), the right sets' blocks, the terms' alphas.
 * Returns the psi length, the algorithmic flops of one application (8 m n k
 * per complex GEMM, both GEMMs of every (term, sector)) and the flops executed
 * (each left product L_a[i] X_i is formed once and shared by its terms). */
int tsc_blocksparse_set(tsc_ctx* ctx, int nproblems, const int* ints, long long nints, const double* data,
                        long long ncplx, long long* dim, double* flops, double* exec_flops);
/* Applies the batch on device pointers on the context stream, in TSC_FP64 or
 * TSC_SPLIT_BF16 arithmetic (both sets of job lists are built by _set);
 * tsc_hpsi_stats then reports its device time. */
int tsc_blocksparse_apply(tsc_ctx* ctx, const void* d_in, void* d_out, int mode);

/* H.psi on device pointers that allocates nothing (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc or any allocating
 * library routine when they need H.psi (a host that owns the whole device
 * memory budget through its own pool, an iteration that must not change the
 * allocation state).  Same result as tsc_hpsi_device in the context's precision
 * (TSC_FP64 enqueued on the context stream; TSC_SPLIT_BF16, like
 * tsc_hpsi_device, also waits and reports a timed-out wait as TSC_E_CUDA); its
 * scratch is one fixed array of TSC_NOALLOC_SCRATCH_ELEMS complex128 elements
 * (64 MiB) in device global memory, held by every GPU that loads the library
 * until exit.  Superblocks needing more scratch are rejected with TSC_E_LIMIT.
 * tsc_create places the array on its device and resolves its address, so this
 * entry changes no allocation state.  All calls share the array: calls that
 * overlap on the GPU race. */
#define TSC_NOALLOC_SCRATCH_ELEMS 4194304LL
int tsc_hpsi_noalloc(tsc_ctx* ctx, const void* d_in, void* d_out);

#ifdef __cplusplus
}
#endif
#endif /* TSC_GPU_H */
