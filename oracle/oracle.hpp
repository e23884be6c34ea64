// Oracle: CPU restatement of the reference SU(2) DMRG (hyx15903/TSC_Tri_t1t2J1J2,
// DMRG_code/*.f90) for the superblock hot path and the sweep that drives it.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the product package may include, link or
// call this code; it is the checker that the CUDA path is compared against and
// the timed CPU baseline.  Every routine cites the reference file:line it
// restates.  Arithmetic is complex FP64 throughout (realcode=.false.,
// main.f90:17); dense linear algebra goes through the reference's own BLAS /
// LAPACK call sites (ZGEMM, ZHEEV, DSTEV), bound here to the OpenBLAS that ships
// with scipy (the reference links MKL, makefile.txt:3; no pinned version).
//
// Parity status against the reference binary: UNPINNED (no Fortran compiler in
// this image).  The restatement is pinned by exact-diagonalisation known
// answers and by sympy Wigner-6j tables (tests/golden/).
#pragma once
#include <complex>
#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace orc {

using cplx = std::complex<double>;

// ---- data model: common.f90:84-156 ------------------------------------------
struct SubBlock {            // common.f90:134-137 (Sub_Block)
  int num_up = 0, num_down = 0, down_dif = 0, row_dim = 0, sdim = 0;
  std::vector<cplx> mat;     // column-major row_dim x sdim
  cplx& at(int r, int c) { return mat[(size_t)c * row_dim + r]; }
  const cplx& at(int r, int c) const { return mat[(size_t)c * row_dim + r]; }
};
struct Block {               // common.f90:139-142 (Total_Block)
  int len = 0, num = 0, dim = 0, up_dif = 0, down_dif = 0;
  std::vector<SubBlock> sub;
};
struct SubBasisMap {         // common.f90:84-88
  int spos = 0, sdim = 0, bl_num_up = 0, bl_num_down = 0, st_num_up = 0, st_num_down = 0;
};
struct BasisMap {            // common.f90:91-95
  int idx = 0, num = 0, dim = 0, new_num_up = 0, new_num_down = 0;
  std::vector<SubBasisMap> sub;
};
struct Basis {               // common.f90:98-101
  int len = 0, num = 0, dim = 0;
  std::vector<BasisMap> sub;
};
struct SubSuper {            // common.f90:107-111
  int sys_num_up = 0, sys_num_down = 0, env_num_up = 0, env_num_down = 0, sys_dim = 0, env_dim = 0;
};
struct Super {               // common.f90:113-116
  int sys_len = 0, env_len = 0, num = 0, dim = 0, idx = 0;
  std::vector<SubSuper> sub;
};
struct SubWave {             // common.f90:119-124
  int sys_num_up = 0, sys_num_down = 0, env_num_up = 0, env_num_down = 0, sys_dim = 0, env_dim = 0;
  std::vector<cplx> vec;     // column-major sys_dim x env_dim
};
struct Wave {                // common.f90:126-129
  int sys_len = 0, env_len = 0, num = 0, dim = 0;
  std::vector<SubWave> sub;
};
struct BlockSet {            // common.f90:160-162 (only the t-J members)
  Block elec_up, elec_down, spin_sd, num_sn;
};
struct Model {               // common.f90:167-174 (Total_Model)
  int len = 0;
  Block ham;
  std::vector<BlockSet> sub;     // sub(1..nxx)   boundary-site operators
  BlockSet snc[2];               // merged block-site couplings (hmerge)
  std::vector<BlockSet> sub_s;   // merged block-block couplings (hmerge)
};

// ---- run configuration (main.f90:4-209, restated as data) --------------------
struct Config {
  int Nx = 6, Ny = 4;            // common.f90:11 (Nx, Ny); nleg = Ny (nc=1, nly=1)
  int openy = 0;                 // main.f90:50  (periodic y)
  double t1 = 1.0, t2 = 0.0, J1 = 0.4, J2 = 0.0;  // main.f90:59-70
  int delta = 12;                // main.f90:78  (inverse hole doping)
  // kept-state schedule (main.f90:54-57,178-182)
  int kept_min = 110;
  int kept_max_warmup = 300;     // kept_max during warm-up and the first half sweeps
  std::vector<int> sweep_kept_max;   // kept_max for sweep 1..n (size = number of sweeps)
  double trun_err = 1.0000000036274937e-15;  // main.f90:8  (single-precision literal)
  double lanerr = 1.0e-6;        // main.f90:124 (single-precision literal rounded, see scale)
  bool lanerr_single = true;     // lanerr=1.0e-6 is a default-real literal
  double lanzero_override = -1;  // >0: use this Lanczos tolerance in every phase
  uint64_t seed = 1;             // seeds the random_number stand-in
  bool final_half_sweep = false; // main.f90:205-206
  int final_stop = 0;            // last label of that half sweep; 0: the reference's 5 Num_site / 6 - 1
};

// Per-Lanczos-step record (eigen.f90:169-173, den_mat.f90:342-350).
struct StepLog {
  int phase;          // 0 warm-up, 1 left_to_right, 2 right_to_left
  int sys_len, env_len;
  double e0;
  int lanczos_iters;
  int num_state;      // kept multiplets of the truncation done after this step (sys or env)
  double trun_err;    // discarded weight
  double entropy;     // Entropys
  double entropy_mult;// entropy1 (2S+1 multiplicity weighted)
  int hpsi_calls;
  double hpsi_seconds;
  double hpsi_flops;  // algorithmic flops of all H.psi calls in this step
};

// ---- global state of the reference (module pubdata, common.f90:5-79) --------
struct Lattice {
  int Nx, Ny, nleg, num_site, neibt = 18, neibt1 = 6;
  int openy, open_x = 1;
  // neighbour tables, 1-based (dmrg_sub.f90:334-644)
  std::vector<int> neib;      // (0:num_site, 1:neibt)
  std::vector<int> neiba;     // (0:num_site, 0:num_site)
  std::vector<int> nposi, nposi_dm, nposi_lat;   // (0:num_site+4)
  std::vector<int> inb1;      // (0:num_site, 0:num_site)
  std::vector<int> nleg11;    // (0:num_site)
  std::vector<int> inb;       // (-4:num_site) stored with offset 4
  int coup_bs[2][2] = {{0, 0}, {0, 0}}, coup_bb[2] = {0, 0};
  int nxc = 0;
  // couplings (k, site) with 1-based k and site (main.f90:59-70)
  std::vector<cplx> jt, jz, jd, jn;
  int& NEIB(int i, int k) { return neib[(size_t)i * (neibt + 1) + k]; }
  int& NEIBA(int i, int j) { return neiba[(size_t)i * (num_site + 1) + j]; }
  int& INB1(int i, int ns) { return inb1[(size_t)i * (num_site + 1) + ns]; }
  int& INB(int i) { return inb[(size_t)(i + 4)]; }
  cplx JT(int k, int s) const { return jt[(size_t)s * (neibt + 1) + k]; }
  cplx JZ(int k, int s) const { return jz[(size_t)s * (neibt + 1) + k]; }
  cplx JD(int k, int s) const { return jd[(size_t)s * (neibt + 1) + k]; }
  cplx JN(int k, int s) const { return jn[(size_t)s * (neibt + 1) + k]; }
};

// Flat interchange of one superblock (the C-ABI layout of the product).
struct FlatSuperblock;

class Oracle {
 public:
  explicit Oracle(const Config& cfg);
  // Get_Ground_State (main.f90:114-209) with the configured schedule.
  void run(std::vector<StepLog>* log);
  // measure_operator_dia with num_elec (measure.f90:3-62, called at main.f90:268):
  // <n_i> of every site in the last ground state of run(), site order 1..Num_site.
  std::vector<double> measure_density();
  // Get_sys_oper_dia / Get_env_oper_dia (get_sys.f90:1147-1277), trun_idx = 1
  // (main.f90:89), Truns = .true.: site operator `st` of site old_idx carried
  // into the (truncated) block of length new_idx.
  Block oper_dia_in_block(const Block& st, int old_idx, int new_idx, bool sys);
  // Get_density_cor (measure.f90:2525-2681) with oper1 = oper2 = num_elec, Flags
  // 'B' and xi = xj = site (main.f90:299): <n_site n_j> of the last ground state
  // for the partners j on the leg of `site` the reference visits (j = site + Ny,
  // site + 2 Ny, ... up to Num_site - Num_site/6 + Ny), indexed 1..Num_site,
  // zero where the reference computes nothing.
  std::vector<cplx> density_cor(int site);
  // The same with oper1 = oper2 = st_sd (main.f90:275): <S_site . S_j>.
  std::vector<cplx> spin_cor(int site);
  // The same with oper1 = st_elec_up, oper2 = st_elec_down, Flags 'F' (main.f90:288).
  std::vector<cplx> elec_cor(int site);
  // Get_density_cor for any pair of site operators and Flags (scaled by
  // sqrt(1 + rank of oper1), negated for rank 1, measure.f90:2586-2587, 2662-2663).
  std::vector<cplx> oper_cor(const Block& op1, const Block& op2, char flags, int site);
  // Get_sys_oper_ndia / Get_env_oper_ndia (get_sys.f90:1536-1668), Types = flags.
  Block oper_ndia(const Block& st, int old_idx, int new_idx, bool sys, bool trunc, char flags = 'B');
  // Change_sys/env_oper_ndia (get_sys.f90:1672-1778) or _dia (get_sys.f90:1281-1331);
  // trunc_end is their Truns argument.
  Block change_oper(const Block& op, int old_idx, int new_idx, bool sys, bool ndia, char flags = 'B',
                    bool trunc_end = true);
  // Singlet pair correlations (Get_mSCOP_Operator_Cor0 with Flags 'S0',
  // measure.f90:2683-2834, as main.f90:259-262 calls it): one record per pair
  // of bonds (s1, s2) and (s3, s4) the reference visits, with its value.
  struct PairRec {
    int s1, s2, s3, s4;
    cplx value;
  };
  std::vector<PairRec> pair_cor(int xc1, int xc2, int ij, int ij1);
  Block sys_two(int idx1, int idx2);                                      // Get_sys_two
  Block sys_two1(int idx2, int idx3, int idx4, const Block& pair);        // Get_sys_two1
  Block env_scop(int idx1, int idx2, int new_idx, bool truns);            // Get_SCOP_Operator_Env

  // hot-path entry points restated (used directly by parity tests)
  void model_wave(Model& sys, Model& env, const Basis& sys_bs, const Basis& env_bs,
                  const Wave& in, Wave& out);
  void hmerge(Model& sys, Model& env, const Basis& sys_bs, const Basis& env_bs);
  void lanczos_memo_new(Model& sys, Model& env, const Basis& sys_bs, const Basis& env_bs,
                        const Super& super, Wave& eigvec, int* iters, double* e0);
  void density_matrix_sys(const Wave& w, Block& den);
  void density_matrix_env(const Wave& w, Block& den);
  void truncation_operator(const Block& den, Block& trun, double trun_err, int* num_state,
                           double* err, double* ent, double* ent_mult, bool system_block,
                           std::vector<double>* spectrum);
  void wave_trans_LR(const Basis& sys_bs, const Basis& env_bs, const Block& sys_trun,
                     const Block& env_trun, const Wave& old_w, Wave& new_w);
  void wave_trans_RL(const Basis& sys_bs, const Basis& env_bs, const Block& sys_trun,
                     const Block& env_trun, const Wave& old_w, Wave& new_w);
  void hamiltonian_sys(Model& pre, const Basis& basis, const Block& trun);
  void hamiltonian_env(Model& pre, const Basis& basis, const Block& trun);

  // set-up pieces
  void dmrg_setup(int ns, int ns21);
  void get_basis(const Block& block, const Block& site, Basis& basis);
  void get_super_basis(const Basis& sys_bs, const Basis& env_bs, Super& super, int tot_up, int tot_down);
  void hamiltonian_site(Model& m);
  void allocate_wave(const Super& s, Wave& w);
  void wave_initialize(Wave& w);

  // superblock capture: when set, the step with this global Lanczos-call index
  // (0-based) is copied out before its Lanczos solve.
  int capture_step = -1;
  struct Capture {
    bool valid = false;
    Model sys, env;
    Basis sys_bs, env_bs;
    Super super;
    Wave psi0;         // Lanczos start vector
    Wave hpsi;         // model_wave(psi0) (after hmerge)
    Wave gs;           // converged ground state
    double e0 = 0;
    int iters = 0;
    Block den;         // density matrix of the side truncated after this step
    Block trun;        // truncation operator
    int num_state = 0;
    double err = 0, ent = 0, ent_mult = 0;
    std::vector<double> spectrum;   // sorted, normalised density-matrix spectrum
    bool sys_side = true;
    int nxc = 0;
    // block growth after the truncation: the enlarged-and-renormalised block
    Model grown;
    Basis grow_basis;
    // wave transformation into the next superblock (input and output)
    bool has_wt = false;
    bool wt_lr = true;
    Basis wt_sys_bs, wt_env_bs;
    Block wt_sys_trun, wt_env_trun;
    Wave wt_old, wt_new;
    Super wt_super;
  } cap;

  Config cfg;
  Lattice L;
  // site operators (dmrg_sub.f90:733-908)
  Block st_elec_up, st_elec_down, num_elec, st_sd, st_sz, st_si;
  // H.psi accounting
  long long hpsi_calls = 0;
  double hpsi_seconds = 0, hpsi_flops = 0;
  int lanczos_calls = 0;
  int tot_num_up = 0, tot_num_down = 0;
  int kept_min = 0, kept_max = 0;
  double lanzero = 0;
  int restart1 = 0, restart2 = 0;
  int mshift = 0;

 private:
  uint64_t rng_state;
  double rand01();
  void setup0();
  void site_operators();
  // disk stand-ins (block.f90:1547-2077): blocks, truncations and bases by length
  std::map<int, Model> sys_models, env_models;
  std::map<int, Block> sys_truns, env_truns;
  std::map<int, Basis> sys_bsm, env_bsm;
  Wave disk_wave;
  void warm_up_point(int bg_id, int end_id, double trun_err, std::vector<StepLog>* log);
  void left_to_right(int bg_id, int end_id, double trun_err, std::vector<StepLog>* log);
  void right_to_left(int bg_id, int end_id, double trun_err, std::vector<StepLog>* log);
  void step_capture_pre(Model& sys, Model& env, const Basis& sys_bs, const Basis& env_bs,
                        const Super& super, const Wave& psi0);
};

// helpers shared by the oracle translation units
double w6js(int j1, int j2, int j3, int l1, int l2, int l3);   // block.f90:3744-3795
double w3js(int j1, int j2, int j3, int m1, int m2, int m3);   // block.f90:3702-3741
void zgemm(char ta, char tb, int m, int n, int k, cplx alpha, const cplx* a, int lda,
           const cplx* b, int ldb, cplx beta, cplx* c, int ldc);
extern double g_gemm_flops;   // running count of 8*m*n*k over all zgemm calls
void block_transfer_trans(const Block& in, Block& out);        // block.f90:33-64
void block_pass_info(const Block& old_b, Block& new_b);        // block.f90:132-159
void block_add_block_two(const Block& b1, cplx coef1, Block& nb);  // block.f90:177-215
double wave_product(const Wave& l, const Wave& r);             // block.f90:1092-1108
double wave_norm(const Wave& w);                                // block.f90:1112-1131
void wave_normalize(Wave& w);                                   // block.f90:1135-1150

}  // namespace orc
