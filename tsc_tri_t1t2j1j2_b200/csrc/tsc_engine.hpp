// Host side of the B200 superblock engine: device-resident block operators,
// SU(2) bases, task-list builders for the grouped-GEMM kernel, the Lanczos /
// truncation / renormalisation / wave-transformation steps and the sweep driver.
// Sector conventions follow the reference data model (DMRG_code/common.f90:84-156):
// a sector is (num_up, num_down) = (electrons, 2S); operator sub-blocks are keyed
// by their column sector and carry their own down_dif; matrices hold reduced
// (Wigner-Eckart) elements.
#pragma once
#include <cuda_runtime.h>

#include <array>
#include <complex>
#include <map>
#include <memory>
#include <shared_mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "tsc_kernels.cuh"

namespace tsc {

using cplx = std::complex<double>;

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void cuda_check(cudaError_t e, const char* what);

// Engines of one process share this lock: a stream capture (the Lanczos graph)
// holds it shared, engine construction and destruction hold it exclusively,
// because their device-synchronising calls (pinned host memory, pool trims)
// would invalidate a capture running in another thread.
std::shared_mutex& capture_mutex();

// ---- device memory -----------------------------------------------------------
// Device buffer of complex elements, stream-ordered on `st`.  Buffers are carved
// from per-stream arenas (chunks of the device pool, best fit, coalesced on
// free), so a DMRG step makes no driver calls once its arena has grown;
// blocks of 4 GiB and more come from the pool directly, which reuses them
// across sizes; release_stream_cache() hands a stream's chunks back to the pool.
struct DevBuf {
  double2* p = nullptr;
  size_t n = 0;   // complex elements
  size_t cls = 0; // bytes of the arena block behind p
  bool direct = false;   // allocated from the pool itself (large blocks)
  cudaStream_t st = nullptr;
  DevBuf() = default;
  DevBuf(size_t count, cudaStream_t s, bool zero);
  ~DevBuf();
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
};
using DevBufP = std::shared_ptr<DevBuf>;
cudaMemPool_t device_pool();   // the current device's buffer pool
void release_stream_cache(cudaStream_t s);   // free the cached blocks of stream s

// ---- data model ----------------------------------------------------------------
struct SubDesc {
  int num_up = 0, num_down = 0, down_dif = 0, row_dim = 0, sdim = 0;
  long long off = 0;   // complex elements from the block's buffer start
};
struct DBlock {
  int len = 0, num = 0, dim = 0, up_dif = 0, down_dif = 0;
  std::vector<SubDesc> sub;
  DevBufP buf;
  double2* ptr(int i) const { return buf->p + sub[i].off; }
  long long total() const {
    long long t = 0;
    for (auto& s : sub) t += (long long)s.row_dim * s.sdim;
    return t;
  }
};
enum OpIdx { OP_UP = 0, OP_DOWN = 1, OP_SD = 2, OP_SN = 3 };
struct OpSet {
  DBlock op[4];
};
struct DModel {
  int len = 0;
  DBlock ham;
  std::vector<OpSet> sub;   // 1-based boundary-site operators
};
struct Piece {
  int spos = 0, sdim = 0, bl_num_up = 0, bl_num_down = 0, st_num_up = 0, st_num_down = 0;
};
struct Sector {
  int num_up = 0, num_down = 0, dim = 0;
  std::vector<Piece> pcs;
};
struct Basis {
  int len = 0, num = 0, dim = 0;
  std::vector<Sector> sec;
  int find(int up, int down) const {
    for (int x = 0; x < num; ++x)
      if (sec[x].num_up == up && sec[x].num_down == down) return x;
    return -1;
  }
};
struct WSec {
  int sys_num_up = 0, sys_num_down = 0, env_num_up = 0, env_num_down = 0, sys_dim = 0, env_dim = 0;
  long long off = 0;
};
struct WLayout {
  int sys_len = 0, env_len = 0, num = 0;
  long long dim = 0;
  std::vector<WSec> sec;
  int find(int su, int sd, int eu, int ed) const {
    for (int k = 0; k < num; ++k) {
      const WSec& s = sec[k];
      if (s.sys_num_up == su && s.sys_num_down == sd && s.env_num_up == eu && s.env_num_down == ed) return k;
    }
    return -1;
  }
};

// site operators (dmrg_sub.f90:733-908) held on the host: one 1x1 element per sub-block
struct SiteSub {
  int num_up, num_down, down_dif;
  double val;
};
struct SiteOp {
  int up_dif = 0, down_dif = 0;
  std::vector<SiteSub> sub;
};

// ---- lattice and couplings (dmrg_sub.f90:304-644, main.f90:59-99) ----------------
struct Lattice {
  int Nx = 0, Ny = 0, nleg = 0, num_site = 0, openy = 0;
  static constexpr int neibt = 18;
  std::vector<int> neib, neiba, nposi, nposi_dm, nposi_lat, inb1, nleg11, inb;
  std::vector<double> jt, jz, jd, jn;
  int nxc = 0;
  int coup_bs[2][2] = {{0, 0}, {0, 0}}, coup_bb[2] = {0, 0};
  void init(int Nx, int Ny, double t1, double t2, double J1, double J2, int openy);
  void setup(int ns, int ns21);   // dmrg_setup
  void setup0();                  // dmrg_setup0
  int& NEIB(int i, int k) { return neib[(size_t)i * (neibt + 1) + k]; }
  int& NEIBA(int i, int j) { return neiba[(size_t)i * (num_site + 1) + j]; }
  int& INB1(int i, int ns) { return inb1[(size_t)i * (num_site + 1) + ns]; }
  int& INB(int i) { return inb[(size_t)(i + 4)]; }
  double JT(int k, int s) const { return jt[(size_t)s * (neibt + 1) + k]; }
  double JZ(int k, int s) const { return jz[(size_t)s * (neibt + 1) + k]; }
  double JD(int k, int s) const { return jd[(size_t)s * (neibt + 1) + k]; }
  double JN(int k, int s) const { return jn[(size_t)s * (neibt + 1) + k]; }
  int npos(int latt) const { return nposi[nposi_dm[latt]]; }
};

double w6j(int j1, int j2, int j3, int l1, int l2, int l3);   // doubled arguments
double w3j(int j1, int j2, int j3, int m1, int m2, int m3);   // doubled arguments

// ---- task lists -------------------------------------------------------------------
struct TaskList {
  std::vector<GGroup> groups;
  std::vector<std::vector<GTerm>> gterms;   // per-group terms while building
  // device copies
  DevBufP dev;   // jobs + groups + terms packed (as raw bytes in a double2 buffer)
  GJob* d_jobs = nullptr;
  GGroup* d_groups = nullptr;
  GTerm* d_terms = nullptr;
  GReduce* d_reds = nullptr;
  int njobs = 0, nreds = 0;
  int tile = 64;           // CTA tile code used for this list (TILE_* in tsc_kernels.cuh)
  bool split = false;      // jobs are 128 x 64 tiles for the split-precision kernel
  long long max_red_elems = 0;
  DevBufP part;            // partial tiles of split groups
  long long part_elems = 0;
  double exec_flops = 0;   // flops the kernel executes
  long long nterms = 0;
  SplitArenas arenas{};    // split lists: the arenas of their pre-sliced operand views
  bool term_alpha = false; // split lists: coefficients applied per term by the kernel (not folded)
  int add_group(double2* abs_c, uint8_t base, long long c_off, int ld, int M, int N, int beta);
  // Packs the lists for the device.  Groups whose term list is much longer than
  // total_cost / (slots * waves) are split into contiguous term chunks, each
  // computing a partial tile; a fixed-order reduction then writes the group.
  void upload(cudaStream_t st, int slots = 296, int waves = 4, int tile_override = 0);
  // The same lists for the split-precision kernel (the host lists are kept).
  void upload_split(cudaStream_t st);
};

// Stored block models of both sides by length (the reference writes every
// model to disk and reads it back when the sweep returns, block.f90:1715-1900,
// dmrg_sub.f90:1119-1139).  Here models stay in HBM while the resident models
// fit under a byte limit; past it, the least recently used ones move to host
// memory and come back to the device when read.  A spilled model keeps its
// descriptors; only its device buffers are released.
class ModelStore {
 public:
  void put(int side, int len, const DModel& m);   // store; may spill older models
  DModel get(int side, int len);                  // resident copy (restored if spilled)
  bool has(int side, int len) const { return map_.count(key(side, len)) > 0; }
  std::vector<std::pair<int, int>> keys() const {   // (side, length) of every stored model
    std::vector<std::pair<int, int>> k;
    for (const auto& kv : map_) k.push_back({(int)(kv.first >> 32), (int)(kv.first & 0xffffffff)});
    return k;
  }
  void clear();   // drops every model (and the files of those on disk)
  ~ModelStore() { clear(); }
  void bind(cudaStream_t st) { st_ = st; }
  // bytes of device memory the stored models may hold; < 0: default_frac of the device
  void set_limit(long long bytes) { limit_ = bytes; }
  // the default's share of device memory (the split form's operand views need room)
  void set_default_frac(double f) { default_frac_ = f; }
  long long limit() const;
  long long resident_bytes() const { return resident_; }
  long long spills = 0, restores = 0;
  double moved_bytes = 0, moved_seconds = 0;
  // Disk tier: spilled models beyond host_bytes of host memory go to files in
  // dir (the reference's own out-of-core storage); host_bytes < 0 or an empty
  // dir: no disk tier (the default).
  void set_disk(long long host_bytes, const std::string& dir) {
    host_limit_ = host_bytes;
    disk_dir_ = dir;
  }
  long long host_bytes() const { return host_bytes_; }
  long long disk_writes = 0, disk_reads = 0;
  double disk_bytes = 0, disk_seconds = 0;

 private:
  struct Entry {
    DModel m;
    std::vector<std::vector<double2>> host;   // per block (ham, then ops), when spilled
    bool spilled = false;
    bool on_disk = false;                     // spilled, and its host copy moved to `file`
    std::string file;
    long long bytes = 0;
    unsigned long long tick = 0;
  };
  static long long key(int side, int len) { return (long long)side << 32 | (unsigned)len; }
  void spill(Entry& e);
  void restore(Entry& e);
  void enforce(long long keep);
  void to_disk(long long key, Entry& e);
  void from_disk(Entry& e);
  void enforce_host(long long keep);
  std::map<long long, Entry> map_;
  cudaStream_t st_ = nullptr;
  long long limit_ = -1;
  double default_frac_ = 0.45;
  long long resident_ = 0;
  unsigned long long clock_ = 0;
  long long host_limit_ = -1;
  std::string disk_dir_;
  long long host_bytes_ = 0;   // bytes of the spilled models' host copies
};

// Pre-sliced operand views of a pair of split-precision lists (phase 1, phase 2).
struct SplitData {
  DevBufP fixed, in, t;      // arenas of SPLIT_UNIT-byte tiles: operators, input vector, intermediates
  DevBufP in_lists;          // the input vector's views and tiles (sliced again on every call)
  const SView* d_in_views = nullptr;
  const STile* d_in_tiles = nullptr;
  int n_in_tiles = 0;
  SplitArenas arenas{};
  long long units[3] = {0, 0, 0};
  int nviews[3] = {0, 0, 0};
};
// Rewrites the GEMM terms of the split lists p1 (phase 1) and p2 (phase 2),
// copies of the FP64 lists, to reference pre-sliced views: each operator
// operand (with the term's coefficient folded in), each rectangle of the input
// vector, each phase-1 intermediate read by phase 2.  Allocates the arenas,
// slices the operator views, and keeps the input vector's tile list.
// term_alpha: keep the terms' coefficients in the lists (applied per term by the
// kernel's epilogue) instead of folding them into per-term operator views
void build_split_views(TaskList& p1, TaskList& p2, SplitData& sd, cudaStream_t st, bool term_alpha = false);
// Slices the input vector's views of sd (before phase 1 of every call).
void slice_input(const SplitData& sd, const double2* d_in, cudaStream_t st);

struct Stats {
  double hpsi_ms = 0, hpsi_flops = 0, hpsi_bytes = 0;
  int launches = 0;
};

class Engine {
 public:
  Engine(int Nx, int Ny, double t1, double t2, double J1, double J2, int delta, int device);
  ~Engine();

  cudaStream_t st = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<cudaEvent_t> hpsi_events;   // per-call H.psi brackets of a Lanczos solve
  int device_ = 0;
  struct EigLanes;                          // concurrent per-sector eigensolvers (tsc_dmrg.cu)
  std::shared_ptr<EigLanes> eig;
  Lattice L;
  int tot_num_up = 0, tot_num_down = 0;
  SiteOp st_elec_up, st_elec_down, num_elec, st_sd, st_sz;
  std::string last_error;

  // ---- superblock (one Lanczos problem) ----
  struct Superblock {
    DModel sys, env;
    Basis sys_bs, env_bs;
    WLayout wl;
    DBlock snc_sys[2][4], snc_env[2][4];
    std::vector<OpSet> sub_s_sys, sub_s_env;   // merged block-block operators
    TaskList merge;            // hmerge axpy tasks
    TaskList p1, p2;           // H.psi phase 1 (intermediates) and phase 2 (outputs)
    TaskList p1s, p2s;         // the same, tiled for the split-precision kernel
    SplitData sv;              // their pre-sliced operand views
    TaskList q1, q2;           // a candidate schedule being timed by the autotuner
    int tune_class = -1;       // size class of this superblock (-1: not tuned)
    int tune_cand = -1;        // candidate in q1/q2, used by the next H.psi
    bool tune_pending = false; // that H.psi ran and its time is still to be read
    long long scratch_elems = 0;
    DevBufP scratch;
    double ref_flops = 0;      // algorithmic flops of one model_wave (reference order)
    bool valid = false;
  } sb;

  void superblock_set(DModel&& sys, DModel&& env, Basis&& sys_bs, Basis&& env_bs, WLayout&& wl);
  void hpsi(const double2* d_in, double2* d_out);   // enqueue on st, in the context's precision
  void hpsi_form(const double2* d_in, double2* d_out, bool split);

  // block-sparse batch (tsc_blocksparse_set/_apply, csrc/tsc_blocksparse.cu)
  struct BlockSparse {
    DevBufP ops, scratch;
    TaskList p1, p2, p1s, p2s;
    SplitData sv;
    long long dim = 0;
    double ref_flops = 0;
    int nprob = 0;
    bool valid = false;
  } bs;
  void blocksparse_set(int nprob, const int* ints, long long nints, const cplx* data, long long ncplx);
  bool views_of_batch_ = false;   // the last set was a block-sparse batch (tsc_split_views reports its views)
  void blocksparse_apply(const double2* d_in, double2* d_out, bool split);

  // measurement of the last ground state (csrc/tsc_measure.cu, measure.f90)
  std::vector<double> measure_density();
  DBlock oper_dia_in_block(const SiteOp& so, int old_idx, int new_idx, bool sys, bool trunc = true);
  // <n_site n_j> for the partners j of Get_density_cor (tsc_measure.cu)
  std::vector<double> measure_density_cor(int site);
  DBlock carry_dia(const DBlock& op, int from, int to, bool sys);
  DBlock product_dia(const DBlock& a, const DBlock& b, const Basis& basis);
  double corr_block_site(const DBlock& bl, const SiteOp& so, const Basis& bs);
  double corr_block_env(const DBlock& bl, const DBlock* ebl, const SiteOp* eso, const Basis& sbs, const Basis& ebs);
  DBlock site_as_block(const SiteOp& so);
  DBlock site_dia(const SiteOp& so, const Basis& basis);
  DBlock block_dia(const DBlock& blk, const Basis& basis);
  DBlock trun_dia(const DBlock& ori, const DBlock& trun);
  double expect_dia(const DBlock* bl, const SiteOp* so, const Basis& bs, bool sys, double* imag = nullptr);
  // <op1_site op2_j> for operators of any rank (Get_density_cor, tsc_correlate.cu)
  std::vector<cplx> measure_oper_cor(const SiteOp& op1, const SiteOp& op2, char flag, int site);
  DBlock ndia_layout(const Basis& basis, int up_dif, int K, TaskList& tl, std::vector<int>& g);
  DBlock site_ndia(const SiteOp& so, const Basis& basis, bool env, char flag);
  DBlock block_ndia(const DBlock& blk, const Basis& basis, bool env, char flag);
  DBlock trun_ndia(const DBlock& ori, const DBlock& trun);
  DBlock oper_ndia_in_block(const SiteOp& so, int old_idx, int new_idx, bool sys, bool trunc, char flag);
  DBlock carry_ndia(const DBlock& op, int from, int to, bool sys, char flag, bool trunc_end = true);
  DBlock product_ndia(const DBlock& o1, const DBlock& o2, int K, const Basis& basis);
  DBlock transfer_trans(const DBlock& in);
  struct PairSum;
  cplx pair_sum(PairSum& ps);
  cplx corr_site_ndia(const DBlock& bl, const SiteOp& st_op, const Basis& bs, char flag);
  cplx corr_env_site_ndia(const DBlock& bl, const SiteOp& est, const Basis& sbs, const Basis& ebs, char flag);
  cplx corr_env_block_ndia(const DBlock& bl, const DBlock& ebl, const Basis& sbs, const Basis& ebs, char flag);
  // singlet pair correlations (Get_mSCOP_Operator_Cor0, tsc_correlate.cu)
  struct PairCor {
    int s1, s2, s3, s4;
    cplx value;
  };
  std::vector<PairCor> measure_pair_cor(int xc1, int xc2, int ij, int ij1);
  DBlock sys_pair(int idx1, int idx2);
  DBlock sys_pair_four(int idx2, int idx3, int idx4, const DBlock& pair);
  DBlock env_pair(int idx1, int idx2, int new_idx, bool trunc_end);
  // 0: complex FP64 throughout; 1: H.psi sector GEMMs as BF16 slices on the
  // tensor cores, Lanczos finished by FP64 iterations.  Applies from the next
  // superblock set on.
  int precision_ = 0;
  double split_tol_ = 1e-11;  // relative Ritz-value change that ends the split iterations
  // FP64 iterations that finish a split solve stop when the Ritz residual is
  // <= refine_res_ * sqrt(lanzero); 0 (the default): the reference's own stop
  // (successive Ritz values within lanzero, eigen.f90:101)
  double refine_res_ = 0.0;
  // the reference's stop of that FP64 finish compares successive Ritz values
  // with finish_mult_ * lanzero
  double finish_mult_ = 1.0;
  bool split_now_ = false;    // the current superblock's solve uses the split form
  // split form only: the U^H O U renormalisation of block growth on the split
  // kernel too (off by default: its ~1e-7 relative error stays in every later H)
  bool split_renorm_ = false;
  // split form: operator views shared by all terms (1, the default: coefficients
  // in the epilogue), one view per term with its coefficient folded in (0), or
  // chosen by the superblock's operator memory (-1)
  int split_shared_views_ = 1;
  // Lanczos iterations replayed as one CUDA graph per solve (on by default)
  bool lanczos_graph_ = true;
  cudaGraphExec_t graph_exec_ = nullptr;   // reused across solves through cudaGraphExecUpdate
  cudaEvent_t graph_ev_[2] = {nullptr, nullptr};
  long long graph_replays_ = 0, graph_fallbacks_ = 0;   // iterations replayed; failed captures
  std::string graph_fallback_reason_;
  bool in_warmup_ = false;    // set while the warm-up (infinite-lattice) steps run

  // Autotuner of the FP64 H.psi schedule: for each size class (log2 of the
  // H.psi GFLOP, superblocks of >= 8 GFLOP) the candidate (CTA tile, waves)
  // schedules are timed, one per superblock on its first H.psi, in device
  // milliseconds per algorithmic GFLOP; once all are timed the class keeps the
  // fastest.  tsc_set_autotune switches it off (schedule fixed, results
  // bit-reproducible run to run).
  struct TuneCand {
    int tile, waves;
  };
  static constexpr int kTuneCands = 4;
  const TuneCand tune_cands_[kTuneCands] = {{TILE_32x32, 4}, {TILE_32x32, 8}, {TILE_64x32, 8}, {TILE_32x64, 8}};
  std::map<int, std::array<double, kTuneCands>> tune_ms_;   // class -> ms/GFLOP (<0: not timed)
  bool autotune_ = true;
  cudaEvent_t tune_ev_[2] = {nullptr, nullptr};   // bracket the candidate's H.psi
  void tune_setup();          // called by build_hpsi_tasks once p1/p2 are built
  void tune_observe();        // after a synchronisation: records a pending timing
  int tune_superblock(int reps);   // times every candidate on the current superblock
  Stats last_stats;

  // Lanczos (eigen.f90:4-199) on the current superblock; psi device buffer in/out
  void lanczos(double2* d_psi, double lanzero, int* iters, double* e0, double* hpsi_ms, int* hpsi_calls);
  void lanczos_run(double2* d_psi, double lanzero, double rel_tol, bool split, int* iters, double* e0,
                   double* hpsi_ms, int* hpsi_calls, double res_tol = 0.0);
  int last_split_iters = 0;     // split-precision iterations of the last solve
  double last_split_e0 = 0.0;   // their final Ritz value

  // density matrix + truncation (den_mat.f90)
  struct TruncResult {
    DBlock trun;
    int num_state = 0;
    double err = 0, ent = 0, ent_mult = 0;
    std::vector<double> spectrum;
  };
  void truncate(int side, const double2* d_psi, const WLayout& wl, int kept_min, int kept_max,
                double trun_err, TruncResult& out);
  DBlock density_matrix(int side, const double2* d_psi, const WLayout& wl, int levels);
  void truncation_operator(DBlock& den, int kept_min, int kept_max, double trun_err, TruncResult& out);
  // Kept zero-weight columns of one sector of U: W is the sector's d x (m + sig)
  // block (ld d), m completion columns followed by the sig significant kept
  // eigenvectors; the first m columns are overwritten by the canonical
  // complement basis (tsc_nullspace.cu).
  struct NullJob {
    double2* W;
    int d, sig, m;
  };
  void null_complete(const std::vector<NullJob>& jobs);

  // block growth + renormalisation (get_sys.f90:4-592)
  void grow(int side, DModel& pre, const Basis& basis, const DBlock& trun, int mshift);

  // wave transformations (dmrg_sub.f90:1471-1789); new_w zeroed and written
  void wave_trans(int dir, const Basis& sys_bs, const Basis& env_bs, const DBlock& sys_trun,
                  const DBlock& env_trun, const WLayout& old_l, const double2* d_old, const WLayout& new_l,
                  double2* d_new);

  // bases (block.f90:2087-2247)
  Basis get_basis(const DBlock& block) const;
  WLayout get_super(const Basis& sys_bs, const Basis& env_bs, int tot_up, int tot_down) const;
  DModel site_model() const;

  // sweep driver (dmrg_sub.f90:974-1465, main.f90:114-209)
  struct StepRec {
    int phase, sys_len, env_len;
    double e0;
    int iters, num_state;
    double err, ent, ent_mult;
    int hpsi_calls;
    double hpsi_seconds, hpsi_flops, step_seconds;
    // wall time of the step's parts (stream synchronised at each boundary)
    double set_seconds, lanczos_seconds, truncate_seconds, grow_seconds, wave_seconds;
    int split_iters;
    double split_e0;
  };
  // resume: skip the warm-up and the two half sweeps and continue with the
  // sweeps from the state checkpoint_read loaded (restart1 = 1, main.f90:36-38)
  void run(int kept_min, int kept_warm, const std::vector<int>& sweeps, double lanzero_override,
           unsigned long long seed, std::vector<StepRec>* log, bool warmup_only = false, bool final_half = false,
           bool resume = false, int max_solves = 0);
  // a run stops once it has made max_solves_ Lanczos solves (0: no cap)
  int max_solves_ = 0;
  double lanzero_warmup_ = 0.0;   // > 0: the warm-up's Lanczos tolerance (else the run's)
  int final_stop_ = 0;            // > 0: last label of the final half sweep (else 5 N / 6 - 1)
  bool solve_cap_reached() const { return max_solves_ > 0 && nsolve_ >= max_solves_; }
  // the reference's checkpoint files (tsc_checkpoint.cu): every stored model,
  // truncation and basis of the last run and its last wavefunction
  int checkpoint_write(const std::string& dir);
  void checkpoint_read(const std::string& dir);
  int capture_step = -1;
  struct Capture {
    bool valid = false;
    std::vector<int> ints;
    std::vector<cplx> data;
    int sys_len = 0, env_len = 0;
  } cap;

  ModelStore& model_store() { return models_; }

  // helpers
  void normalize(double2* d, long long n);
  double wave_norm2(const double2* d, long long n);
  DBlock upload_block(const int*& ip, const cplx*& dp);
  void download_block(const DBlock& b, std::vector<int>& ints, std::vector<cplx>& data) const;
  DBlock copy_block(const DBlock& b);

  // scratch for reductions
  DevBufP red_buf;
  double* d_red = nullptr;   // partials
  double* d_scal = nullptr;  // scalars: [0..255] alpha, [256..511] beta, [512..767] uv, [768..1023] uu, misc
  double* h_scal = nullptr;  // pinned mirror
  // This context's device status word (a slot of d_scal): the split kernel sets
  // it when one of its bounded waits runs out.  One word per context, so
  // contexts running side by side never see each other's faults.
  static constexpr int S_FAULT = 2040;
  int* d_fault = nullptr;
  long long split_wait_limit_ = SPLIT_WAIT_LIMIT;   // polls per bounded wait of the split kernel
  // Waits for the stream, reads the status word and clears it; a set word
  // becomes Error(TSC_E_CUDA).
  void check_split_fault();

 private:
  uint64_t rng = 1;
  double rand01();
  void wave_initialize(const WLayout& wl, double2* d);
  ModelStore models_;   // side 0: system models by length, side 1: environment models
  std::map<int, DBlock> sys_truns, env_truns;
  std::map<int, Basis> sys_bsm, env_bsm;
  WLayout disk_layout;
  DevBufP disk_wave;
  int restart1 = 0;
  bool resume_ready_ = false;   // checkpoint_read has loaded a state to continue from
  int kept_min_ = 0, kept_max_ = 0;
  double lanzero_ = 0;
  int nsolve_ = 0;
  void lanczos_step(int phase, DModel& sys, DModel& env, const Basis& sys_bs, const Basis& env_bs,
                    const WLayout& wl, DevBufP& psi, StepRec& rec);
  void build_hpsi_tasks();
  void build_merge();
  void run_tasks(TaskList& tl, double2* in, double2* out, double2* scr);
  void capture_superblock(const DevBufP& psi);
  void record_step(const StepRec& rec, std::vector<StepRec>* log);
  void warm_up(int end_id, double trun_err, std::vector<StepRec>* log);
  void left_to_right(int bg_id, int end_id, double trun_err, std::vector<StepRec>* log);
  void right_to_left(int bg_id, int end_id, double trun_err, std::vector<StepRec>* log);
};

}  // namespace tsc
