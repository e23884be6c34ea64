// Device task formats shared by the host task builders and the kernels.
#pragma once
#include <atomic>
#include <cuda_runtime.h>
#include <cstdint>

namespace tsc {

// Operand pointer = base[id] + off (complex128 elements).  Base 0 is the null
// pointer (off is then an absolute address / 16); bases 1..3 are rebound per
// launch (input vector, output vector, scratch) so one task list serves every
// Lanczos iteration.
enum BaseId : uint8_t { BASE_ABS = 0, BASE_IN = 1, BASE_OUT = 2, BASE_SCR = 3 };
enum TermKind : uint8_t { TK_GEMM = 0, TK_AXPY = 1, TK_DIAG = 2 };
enum Op : uint8_t { OP_N = 0, OP_C = 1 };

// One contribution to an output group:
//   GEMM:  C += alpha * op(L)[M x K] * op(R)[K x N]          (whole group)
//   AXPY:  C[r0:r0+rm, c0:c0+rn] += alpha * op(R)[rm x rn]
//   DIAG:  C[r0+i, c0+i] += alpha   for i < rm
struct GTerm {
  long long l_off, r_off;
  int l_ld, r_ld;
  int K;
  int r0, c0, rm, rn;
  double ar, ai;
  uint8_t l_base, r_base, l_op, r_op, kind, pad0, pad1, pad2;
};

// Output rectangle C (M x N, column-major, leading dimension c_ld).  After the
// launch C = sum(terms) + beta * C_old; every element of C is written.
struct GGroup {
  long long c_off;
  int c_ld, M, N;
  int t0, t1;
  uint8_t c_base, beta, pad0, pad1;
  // split-precision lists only: >= 0 when the next launch reads this group's
  // output as an A operand; the output is then also written, sliced, into the
  // A tiles of that view (ARENA_T, first tile at s_off units)
  long long s_off = -1;
};

// One CTA's work: tile (tm, tn) of a group over terms [t0, t1).  part < 0 writes
// the group's output; otherwise the tile is a partial sum written to the partial
// buffer at part_off (ld = group M) and reduced by launch_reduce_partials.
struct GJob {
  int group, tm, tn, t0, t1, part;
  long long part_off;
};

// Partial sums of one split group: C = sum_{p<nparts} P[p] + beta*C_old.
struct GReduce {
  int group, nparts;
  long long part_off;   // first partial; partial p at part_off + p*M*N
};

struct Bases {
  double2* p[4];
  double2* part;
};

constexpr int GEMM_TK = 16, GEMM_THREADS = 128;

// tile = CTA output tile edge (64: 64x64, 2 CTAs/SM; 32: 32x32, 6 CTAs/SM)
cudaError_t launch_grouped_zgemm(const GJob* jobs, int njobs, const GGroup* groups, const GTerm* terms,
                                 Bases bases, cudaStream_t st, int tile);
// ---- split-precision form: operands pre-sliced into stage tiles ----------------------
// A tile of an operand view holds six BF16 planes (3 slices x re/im) of op(X) in
// the kernel's shared-memory stage layout: A role 128 rows x 16 k (24 KB, two
// units), B role 16 k x 64 columns (12 KB, one unit).  Views of fixed operators
// carry the term's coefficient and are sliced once per superblock; views of the
// input vector are sliced once per call; phase-1 intermediates are written
// sliced by the launch that computes them.
constexpr int SPLIT_UNIT = 12288;
enum SplitArena : uint8_t { ARENA_FIXED = 0, ARENA_IN = 1, ARENA_T = 2 };
struct SView {
  long long src;       // operator: absolute address / 16; input vector: element offset
  long long dst;       // first tile, in SPLIT_UNIT from its arena's base
  double ar, ai;       // coefficient folded into the slices
  int ld, rows, cols;  // source leading dimension; op(X) is rows x cols (A: M x K, B: K x N)
  int nks;             // tiles along K
  uint8_t from_in, op, role, pad;   // role 0: A operand, 1: B operand
};
struct STile {
  int view, t, ks, pad;   // tile (t, ks) of a view: t = row tile (A) or column tile (B)
};
struct SplitArenas {
  unsigned char* a[3];
  long long units[3];   // size of each arena in SPLIT_UNIT (tile accesses are checked against it)
};
// Slices the listed tiles (one CTA each) of `views` into `arena`; `in` is the
// input vector for views with from_in set.
cudaError_t launch_slice_tiles(const SView* views, const STile* tiles, int ntiles, const double2* in,
                               unsigned char* arena, long long arena_units, cudaStream_t st);
// Split-precision form of launch_grouped_zgemm (BF16 slices on tcgen05, FP32
// accumulation in tensor memory); jobs are 128 x 64 tiles of the same groups.
// GEMM terms of its lists reference pre-sliced views: l_base / r_base = arena,
// l_off / r_off = the view's first tile (units), l_ld / r_ld = its tiles along K.
// Every mbarrier wait of the kernel gives up after wait_limit polls; it then
// sets *fault (the caller's device status word) to 1 and the CTA returns with
// its tiles partly written.  term_alpha = 0: the GEMM terms' coefficients are
// folded into their operand views (ar = 1, ai = 0 in the list) and accumulator
// segments run across terms; 1: segments break at every term and the epilogue
// multiplies each by its term's coefficient (views shared by all terms of an
// operator).
cudaError_t launch_grouped_zgemm_split(const GJob* jobs, int njobs, const GGroup* groups, const GTerm* terms,
                                       Bases bases, SplitArenas arenas, int* fault, long long wait_limit,
                                       int term_alpha, cudaStream_t st);
// default poll limit of the split kernel's waits (far above any wait of a healthy launch)
constexpr long long SPLIT_WAIT_LIMIT = 1ll << 20;
constexpr int SPLIT_TILE_M = 128, SPLIT_TILE_N = 64;
// CTA tile codes of launch_grouped_zgemm (rows x columns of the output tile)
constexpr int TILE_32x32 = 32, TILE_64x64 = 64, TILE_64x32 = 6432, TILE_32x64 = 3264;
inline void tile_dims(int code, int& tm, int& tn) {
  tm = code == TILE_64x32 || code == TILE_64x64 ? 64 : 32;
  tn = code == TILE_32x64 || code == TILE_64x64 ? 64 : 32;
}

// Sets a kernel's dynamic shared-memory limit once per device (the attribute
// belongs to the current device's context; concurrent first calls set the same
// value).  `done` is the kernel's own bitmask of devices already set.
template <class K>
cudaError_t ensure_smem_attr(K kernel, int bytes, std::atomic<unsigned long long>& done) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = 1ull << (dev & 63);
  if (done.load(std::memory_order_acquire) & bit) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) done.fetch_or(bit, std::memory_order_acq_rel);
  return e;
}
cudaError_t launch_reduce_partials(const GReduce* reds, int nred, const GGroup* groups, Bases bases,
                                   long long max_elems, cudaStream_t st);

// ---- vector kernels (Lanczos, eigen.f90 / block.f90:1092-1354) -------------------
// partial sums of Re<x_j, y> for j < nvec (x_j = X + j*ld), deterministic two-pass
cudaError_t launch_multi_dot(const double2* X, long long ld, int nvec, const double2* y, long long n,
                             double* partial, double* out, cudaStream_t st);
// <x, y> = sum conj(x) y into out[0] (real), out[1] (imaginary); partial holds
// 2 * ceil(n / 8192) doubles; deterministic two-pass
cudaError_t launch_zdot(const double2* x, const double2* y, long long n, double* partial, double* out,
                        cudaStream_t st);
cudaError_t launch_lanczos_update(double2* w, const double2* v, const double2* vprev, const double* alpha,
                                  const double* beta_prev, long long n, cudaStream_t st);
cudaError_t launch_scale(double2* w, const double* norm2, long long n, int invert_sqrt, cudaStream_t st);
cudaError_t launch_gs_subtract(double2* w, const double2* X, long long ld, int nvec, const double* uv,
                               const double* uu, long long n, cudaStream_t st);
cudaError_t launch_combine(double2* out, const double2* X, long long ld, int nvec, const double* z,
                           long long n, cudaStream_t st);

// Canonical phase of each column of U (rows x cols, column-major): u *= conj(z)/|z|
// with z = sum_r u_r / (1 + r/10).  Eigensolvers return arbitrary phases; fixing
// them makes renormalised operators independent of the eigensolver.
cudaError_t launch_phase_fix(double2* U, int rows, int cols, cudaStream_t st);

// tridiagonal lowest eigenpair (dstev stand-in): d[0..n), e[0..n-1); writes
// res[0]=E0 and, if want_vec, z[0..n) the normalised eigenvector.
cudaError_t launch_tridiag_lowest(const double* d, const double* e, int n, int want_vec, double* res,
                                  double* z, cudaStream_t st);
// beta[k-1] = sqrt(*n2); res[0] = lowest eigenvalue of T_k (alpha[1..k], beta[1..k-1],
// 1-based slots); packet = {res[0], *n2, alpha[k], |z[k-1]|} where z (written to
// zbuf when it is not null, else 0) is that eigenvalue's unit eigenvector.  k <= 127.
cudaError_t launch_lanczos_tail(const double* n2, double* alpha, double* beta, int k, double* res, double* packet,
                                double* zbuf, cudaStream_t st);

// ---- the Lanczos iteration's vector steps with the index read on the device --------
// (replayable as one CUDA graph: *it = last, the 1-based Lanczos index of
// eigen.f90).  An ItRef {base, ld, add} is base + (*it + add) * ld, or base when ld = 0.
struct ItRef {
  double2* base;
  long long ld;
  int add;
};
// w = v(last+1) -= alpha_last v(last) + beta_(last-1) v(last-1), V = v(1), vectors ld apart
cudaError_t launch_it_update(double2* V, long long ld, const double* alpha, const double* beta, long long n,
                             const int* it, cudaStream_t st);
// out[(out_it ? last : 0) + out_add + j] = Re<x + j*xs, y> for j < (nvec_it ? last : 0) + nvec_add
// (at most nvec_max); partial holds nvec_max * ceil(n / 8192) doubles
cudaError_t launch_it_dot(ItRef x, long long xs, int nvec_it, int nvec_add, int nvec_max, ItRef y, long long n,
                          double* partial, double* out, int out_it, int out_add, const int* it, cudaStream_t st);
cudaError_t launch_it_scale(ItRef w, const double* norm2, long long n, const int* it, cudaStream_t st);
// v(last+1) -= sum_{j<last} (uv_j / uu_j) v(j+1)   (Gram_Schmidt_process)
cudaError_t launch_it_gs(double2* V, long long ld, const double* uv, const double* uu, long long n, const int* it,
                         cudaStream_t st);
cudaError_t launch_it_copy(ItRef dst, ItRef src, long long n, const int* it, cudaStream_t st);
// launch_lanczos_tail with k = last + 1
cudaError_t launch_it_tail(const double* n2, double* alpha, double* beta, double* res, double* packet, double* zbuf,
                           const int* it, cudaStream_t st);

}  // namespace tsc
