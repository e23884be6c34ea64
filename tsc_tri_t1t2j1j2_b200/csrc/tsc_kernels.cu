// B200 (sm_100a) kernels of the superblock engine.
//
// grouped_zgemm: output-stationary grouped complex-FP64 GEMM.  Every job is a
// tile (32x32 .. 64x64) of one output group; the CTA sums all terms of the group
// in registers (DMMA m8n8k4.f64 warp tiles, 3 real MMAs per complex product by
// the Gauss three-multiplication form, alpha folded into the B fragments) and
// writes the tile once: no atomics, the result
// does not depend on launch order.  Operand tiles are staged in shared memory by
// 16-byte cp.async (double buffered, zero fill at the ragged edges); the conj of
// op(.)=C is applied when fragments are read.  Shared-memory rows are padded by
// two complex elements so fragment reads are bank-conflict free.
//
// Vector kernels: the Lanczos recurrences of eigen.f90:64-94 and the classical
// Gram-Schmidt of block.f90:1251-1289 as deterministic two-pass reductions, and
// a tridiagonal lowest-eigenpair solver standing in for LAPACK dstev
// (eigen.f90:99,117,141): Sturm-sequence bisection for the eigenvalue, inverse
// iteration with a pivoted tridiagonal LU for the eigenvector.
#include "tsc_kernels.cuh"

#include <cfloat>
#include <cmath>

namespace tsc {

namespace {

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool pred) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int sz = pred ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}
__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

constexpr int TK = GEMM_TK;

template <int TM, int TN>
struct SmemTiles {
  static constexpr int LDS_A = TM + 2, LDS_B = TN + 2;   // complex per shared row (+2: no bank conflicts)
  double2 a[2][TK * LDS_A];
  double2 b[2][TK * LDS_B];
};

// Stage op(L)[m0.., k0..] (TM x TK) and op(R)[k0.., n0..] (TK x TN) into shared memory
// with 128 threads; every 16-byte copy is a single complex element.
template <int TM, int TN>
__device__ __forceinline__ void load_tiles(SmemTiles<TM, TN>& s, int stage, const GTerm& t, const double2* L,
                                           const double2* R, int M, int N, int m0, int n0, int k0) {
  constexpr int LDA = SmemTiles<TM, TN>::LDS_A, LDB = SmemTiles<TM, TN>::LDS_B;
  const int tid = threadIdx.x;
  const int K = t.K;
  double2* As = s.a[stage];
  double2* Bs = s.b[stage];
  if (t.l_op == OP_N) {
    // L[(m0+i) + (k0+kk)*ld] : contiguous in i
    const int i = tid % TM;
#pragma unroll
    for (int r = 0; r < TM * TK / GEMM_THREADS; ++r) {
      int kk = tid / TM + (GEMM_THREADS / TM) * r;
      bool ok = (m0 + i < M) && (k0 + kk < K);
      const double2* src = ok ? L + (long long)(m0 + i) + (long long)(k0 + kk) * t.l_ld : L;
      cp_async16(&As[kk * LDA + i], src, ok);
    }
  } else {
    // op(L)[m][k] = conj(L[k + m*ld]) : contiguous in k
    const int kk = tid & 15;
#pragma unroll
    for (int r = 0; r < TM * TK / GEMM_THREADS; ++r) {
      int i = (tid >> 4) + 8 * r;
      bool ok = (m0 + i < M) && (k0 + kk < K);
      const double2* src = ok ? L + (long long)(k0 + kk) + (long long)(m0 + i) * t.l_ld : L;
      cp_async16(&As[kk * LDA + i], src, ok);
    }
  }
  if (t.r_op == OP_N) {
    // R[(k0+kk) + (n0+j)*ld] : contiguous in k
    const int kk = tid & 15;
#pragma unroll
    for (int r = 0; r < TN * TK / GEMM_THREADS; ++r) {
      int j = (tid >> 4) + 8 * r;
      bool ok = (n0 + j < N) && (k0 + kk < K);
      const double2* src = ok ? R + (long long)(k0 + kk) + (long long)(n0 + j) * t.r_ld : R;
      cp_async16(&Bs[kk * LDB + j], src, ok);
    }
  } else {
    // op(R)[k][n] = conj(R[n + k*ld]) : contiguous in n
    const int j = tid % TN;
#pragma unroll
    for (int r = 0; r < TN * TK / GEMM_THREADS; ++r) {
      int kk = tid / TN + (GEMM_THREADS / TN) * r;
      bool ok = (n0 + j < N) && (k0 + kk < K);
      const double2* src = ok ? R + (long long)(n0 + j) + (long long)(k0 + kk) * t.r_ld : R;
      cp_async16(&Bs[kk * LDB + j], src, ok);
    }
  }
}

template <int TM, int TN, int MINB>
__global__ void __launch_bounds__(GEMM_THREADS, MINB)
grouped_zgemm_kernel(const GJob* __restrict__ jobs, const GGroup* __restrict__ groups,
                     const GTerm* __restrict__ terms, Bases bases) {
  constexpr int MI = TM / 16, NI = TN / 16;   // 8x8 MMA sub-tiles per warp (2x2 warps)
  constexpr int LDS_A = SmemTiles<TM, TN>::LDS_A, LDS_B = SmemTiles<TM, TN>::LDS_B;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SmemTiles<TM, TN>& s = *reinterpret_cast<SmemTiles<TM, TN>*>(smem_raw);
  const GJob job = jobs[blockIdx.x];
  const GGroup g = groups[job.group];
  const int m0 = job.tm * TM, n0 = job.tn * TN;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = warp & 1, wn = warp >> 1;
  const int lg = lane >> 2, lt = lane & 3;
  // The tile's valid 8x8 MMA sub-tiles are split evenly between the 2x2 warps
  // (warp-uniform counts), so partly filled tiles keep all four SMSPs busy.
  const int mtot = min(2 * MI, (g.M - m0 + 7) / 8), ntot = min(2 * NI, (g.N - n0 + 7) / 8);
  const int mh = (mtot + 1) / 2, nh = (ntot + 1) / 2;
  const int wrow = wm ? mh * 8 : 0, wcol = wn ? nh * 8 : 0;
  const int mt = wm ? mtot - mh : mh, nt = wn ? ntot - nh : nh;

  // Complex products by the three-multiplication (Gauss) form: with
  // T1 = Ar Br, T2 = Ai Bi, T3 = (Ar + Ai)(Br + Bi), the product is
  // (T1 - T2) + i (T3 - T1 - T2); three DMMAs per complex multiply-add instead
  // of four.  The sums are formed once per term (the result is assembled at the end).
  double t1[MI][NI][2], t2[MI][NI][2], t3[MI][NI][2];
#pragma unroll
  for (int a = 0; a < MI; ++a)
#pragma unroll
    for (int b = 0; b < NI; ++b)
#pragma unroll
      for (int e = 0; e < 2; ++e) t1[a][b][e] = t2[a][b][e] = t3[a][b][e] = 0.0;

  for (int ti = job.t0; ti < job.t1; ++ti) {
    const GTerm t = terms[ti];
    if (t.kind == TK_GEMM) {
      const double2* L = bases.p[t.l_base] + t.l_off;
      const double2* R = bases.p[t.r_base] + t.r_off;
      const int nk = (t.K + TK - 1) / TK;
      __syncthreads();   // previous term done with the shared tiles
      load_tiles(s, 0, t, L, R, g.M, g.N, m0, n0, 0);
      cp_async_commit();
      const bool lc = t.l_op == OP_C, rc = t.r_op == OP_C;
      for (int kt = 0; kt < nk; ++kt) {
        if (kt + 1 < nk) {
          load_tiles(s, (kt + 1) & 1, t, L, R, g.M, g.N, m0, n0, (kt + 1) * TK);
          cp_async_commit();
          cp_async_wait<1>();
        } else {
          cp_async_wait<0>();
        }
        __syncthreads();
        const double2* As = s.a[kt & 1];
        const double2* Bs = s.b[kt & 1];
        const int krem = t.K - kt * TK;   // k-steps of 4 past K are all zero padding
#pragma unroll
        for (int kb = 0; kb < TK / 4; ++kb) {
          if (kb * 4 >= krem) break;
          const int krow = kb * 4 + lt;
          double ar[MI], ai[MI], as[MI], br[NI], bi[NI], bs[NI];
#pragma unroll
          for (int mi = 0; mi < MI; ++mi) {
            double2 v = As[krow * LDS_A + wrow + mi * 8 + lg];
            ar[mi] = v.x;
            ai[mi] = lc ? -v.y : v.y;
            as[mi] = ar[mi] + ai[mi];
          }
#pragma unroll
          for (int ni = 0; ni < NI; ++ni) {
            double2 v = Bs[krow * LDS_B + wcol + ni * 8 + lg];
            double vr = v.x, vi = rc ? -v.y : v.y;
            br[ni] = t.ar * vr - t.ai * vi;
            bi[ni] = t.ar * vi + t.ai * vr;
            bs[ni] = br[ni] + bi[ni];
          }
          // three passes so successive updates of each accumulator are MI*NI MMAs apart
#pragma unroll
          for (int mi = 0; mi < MI; ++mi)
#pragma unroll
            for (int ni = 0; ni < NI; ++ni)
              if (mi < mt && ni < nt) dmma(t1[mi][ni][0], t1[mi][ni][1], ar[mi], br[ni]);
#pragma unroll
          for (int mi = 0; mi < MI; ++mi)
#pragma unroll
            for (int ni = 0; ni < NI; ++ni)
              if (mi < mt && ni < nt) dmma(t2[mi][ni][0], t2[mi][ni][1], ai[mi], bi[ni]);
#pragma unroll
          for (int mi = 0; mi < MI; ++mi)
#pragma unroll
            for (int ni = 0; ni < NI; ++ni)
              if (mi < mt && ni < nt) dmma(t3[mi][ni][0], t3[mi][ni][1], as[mi], bs[ni]);
        }
        __syncthreads();
      }
    } else {
      // element-wise terms on the accumulator layout
      const double2* R = bases.p[t.r_base] + t.r_off;
#pragma unroll
      for (int mi = 0; mi < MI; ++mi)
#pragma unroll
        for (int ni = 0; ni < NI; ++ni)
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            int row = m0 + wrow + mi * 8 + lg;
            int col = n0 + wcol + ni * 8 + 2 * lt + e;
            int rr = row - t.r0, cc = col - t.c0;
            if (mi >= mt || ni >= nt) continue;
            if (row >= g.M || col >= g.N || rr < 0 || cc < 0 || rr >= t.rm || cc >= t.rn) continue;
            double vr, vi;
            if (t.kind == TK_AXPY) {
              double2 v = (t.r_op == OP_N) ? R[(long long)rr + (long long)cc * t.r_ld]
                                           : R[(long long)cc + (long long)rr * t.r_ld];
              vr = v.x;
              vi = (t.r_op == OP_C) ? -v.y : v.y;
            } else {
              if (rr != cc) continue;
              vr = 1.0;
              vi = 0.0;
            }
            // adds (dr, di) to the result: dr to T1 (real part T1 - T2), di + dr to T3 (imaginary T3 - T1 - T2)
            const double dr = t.ar * vr - t.ai * vi, di = t.ar * vi + t.ai * vr;
            t1[mi][ni][e] += dr;
            t3[mi][ni][e] += di + dr;
          }
    }
  }

  const bool partial = job.part >= 0;
  double2* C = partial ? bases.part + job.part_off : bases.p[g.c_base] + g.c_off;
  const long long ldc = partial ? g.M : g.c_ld;
  const bool acc_old = !partial && g.beta;
#pragma unroll
  for (int mi = 0; mi < MI; ++mi)
#pragma unroll
    for (int ni = 0; ni < NI; ++ni)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        int row = m0 + wrow + mi * 8 + lg;
        int col = n0 + wcol + ni * 8 + 2 * lt + e;
        if (mi < mt && ni < nt && row < g.M && col < g.N) {
          double2* p = C + (long long)row + (long long)col * ldc;
          const double x1 = t1[mi][ni][e], x2 = t2[mi][ni][e];
          double2 v = make_double2(x1 - x2, t3[mi][ni][e] - x1 - x2);
          if (acc_old) {
            double2 o = *p;
            v.x += o.x;
            v.y += o.y;
          }
          *p = v;
        }
      }
}

// C = sum of the partial tiles of a split group in fixed order (+ beta*C_old)
__global__ void reduce_partials_kernel(const GReduce* __restrict__ reds, const GGroup* __restrict__ groups,
                                       Bases bases) {
  const GReduce r = reds[blockIdx.y];
  const GGroup g = groups[r.group];
  const long long mn = (long long)g.M * g.N;
  double2* C = bases.p[g.c_base] + g.c_off;
  const double2* P = bases.part + r.part_off;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < mn; e += (long long)gridDim.x * blockDim.x) {
    double sr = 0.0, si = 0.0;
    for (int p = 0; p < r.nparts; ++p) {
      double2 v = P[(long long)p * mn + e];
      sr += v.x;
      si += v.y;
    }
    const long long row = e % g.M, col = e / g.M;
    double2* c = C + row + col * g.c_ld;
    if (g.beta) {
      double2 o = *c;
      sr += o.x;
      si += o.y;
    }
    *c = make_double2(sr, si);
  }
}

// ---------------------------------------------------------------- vector kernels
constexpr int VB = 256;          // threads per block
constexpr int VCHUNK = 8192;     // elements per block in reductions

__global__ void multi_dot_partial(const double2* __restrict__ X, long long ld, int nvec,
                                  const double2* __restrict__ y, long long n, double* __restrict__ partial,
                                  int nblk) {
  __shared__ double red[VB / 32];
  long long beg = (long long)blockIdx.x * VCHUNK;
  long long end = beg + VCHUNK < n ? beg + VCHUNK : n;
  for (int j = 0; j < nvec; ++j) {
    const double2* x = X + (long long)j * ld;
    double acc = 0.0;
    for (long long e = beg + threadIdx.x; e < end; e += VB) {
      double2 a = x[e], b = y[e];
      acc = fma(a.x, b.x, acc);
      acc = fma(a.y, b.y, acc);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < VB / 32; ++w) s += red[w];
      partial[(long long)j * nblk + blockIdx.x] = s;
    }
    __syncthreads();
  }
}

// partial sums of <x, y> = sum conj(x) y: real parts at partial[b], imaginary at partial[nblk + b]
__global__ void zdot_partial(const double2* __restrict__ x, const double2* __restrict__ y, long long n,
                             double* __restrict__ partial, int nblk) {
  __shared__ double red[2][VB / 32];
  const long long beg = (long long)blockIdx.x * VCHUNK;
  const long long end = beg + VCHUNK < n ? beg + VCHUNK : n;
  double ar = 0.0, ai = 0.0;
  for (long long e = beg + threadIdx.x; e < end; e += VB) {
    const double2 a = x[e], b = y[e];
    ar = fma(a.x, b.x, ar);
    ar = fma(a.y, b.y, ar);
    ai = fma(a.x, b.y, ai);
    ai = fma(-a.y, b.x, ai);
  }
  for (int o = 16; o > 0; o >>= 1) {
    ar += __shfl_xor_sync(0xffffffffu, ar, o);
    ai += __shfl_xor_sync(0xffffffffu, ai, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = ar;
    red[1][threadIdx.x >> 5] = ai;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sr = 0.0, si = 0.0;
    for (int w = 0; w < VB / 32; ++w) {
      sr += red[0][w];
      si += red[1][w];
    }
    partial[blockIdx.x] = sr;
    partial[nblk + blockIdx.x] = si;
  }
}

__global__ void multi_dot_final(const double* __restrict__ partial, int nblk, int nvec, double* __restrict__ out) {
  int j = blockIdx.x;
  if (j >= nvec) return;
  __shared__ double red[32];
  double acc = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) acc += partial[(long long)j * nblk + b];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    out[j] = s;
  }
}

// w = w - alpha*v - beta_prev*vprev   (eigen.f90:65-75)
__global__ void lanczos_update_kernel(double2* __restrict__ w, const double2* __restrict__ v,
                                      const double2* __restrict__ vprev, const double* __restrict__ alpha,
                                      const double* __restrict__ beta_prev, long long n) {
  const double a = *alpha;
  const double b = vprev ? *beta_prev : 0.0;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    double2 x = w[e], p = v[e];
    x.x = x.x - a * p.x;
    x.y = x.y - a * p.y;
    if (vprev) {
      double2 q = vprev[e];
      x.x = x.x - b * q.x;
      x.y = x.y - b * q.y;
    }
    w[e] = x;
  }
}

// w = w / sqrt(norm2)   (wave_normalize, block.f90:1135-1150)
__global__ void scale_kernel(double2* __restrict__ w, const double* __restrict__ norm2, long long n, int invert_sqrt) {
  const double s = invert_sqrt ? sqrt(*norm2) : *norm2;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    double2 x = w[e];
    x.x = x.x / s;
    x.y = x.y / s;
    w[e] = x;
  }
}

// w = w - sum_j (uv_j/uu_j) x_j   (Gram_Schmidt_process, block.f90:1265-1285)
__global__ void gs_subtract_kernel(double2* __restrict__ w, const double2* __restrict__ X, long long ld, int nvec,
                                   const double* __restrict__ uv, const double* __restrict__ uu, long long n) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    double tr = 0.0, tim = 0.0;
    for (int j = 0; j < nvec; ++j) {
      const double c = uv[j] / uu[j];
      double2 x = X[(long long)j * ld + e];
      tr = tr + c * x.x;
      tim = tim + c * x.y;
    }
    double2 x = w[e];
    x.x = x.x - tr;
    x.y = x.y - tim;
    w[e] = x;
  }
}

// out = sum_i z_i x_i   (eigen.f90:146-153)
__global__ void combine_kernel(double2* __restrict__ out, const double2* __restrict__ X, long long ld, int nvec,
                               const double* __restrict__ z, long long n) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    double r = 0.0, im = 0.0;
    for (int j = 0; j < nvec; ++j) {
      double2 x = X[(long long)j * ld + e];
      r = r + z[j] * x.x;
      im = im + z[j] * x.y;
    }
    out[e] = make_double2(r, im);
  }
}

// number of eigenvalues of T below x (Sturm sequence)
__device__ int sturm_count(const double* d, const double* e, int n, double x, double pivmin) {
  int c = 0;
  double q = d[0] - x;
  if (fabs(q) < pivmin) q = -pivmin;
  if (q < 0) c++;
  for (int i = 1; i < n; ++i) {
    q = d[i] - x - e[i - 1] * e[i - 1] / q;
    if (fabs(q) < pivmin) q = -pivmin;
    if (q < 0) c++;
  }
  return c;
}

// Lowest eigenpair of the symmetric tridiagonal T (diag d[0..n), off-diagonal
// e[0..n-1)), the part of dstev the Lanczos loop uses (eigen.f90:99-141).  One
// warp: the eigenvalue by Sturm-count multisection (32 interior points per
// round, each lane counting at one point, so a round shrinks the bracket 33x),
// the eigenvector by inverse iteration in lane 0.  n <= 127.
__device__ void tridiag_lowest_warp(const double* __restrict__ d, const double* __restrict__ e, int n,
                                    int want_vec, double* __restrict__ res, double* __restrict__ z) {
  const int lane = threadIdx.x & 31;
  if (n == 1) {
    if (lane == 0) {
      res[0] = d[0];
      if (want_vec) z[0] = 1.0;
    }
    return;
  }
  double lo = d[0], hi = d[0], emax = 0.0;
  for (int i = 0; i < n; ++i) {
    double r = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i < n - 1 ? fabs(e[i]) : 0.0);
    lo = fmin(lo, d[i] - r);
    hi = fmax(hi, d[i] + r);
    if (i < n - 1) emax = fmax(emax, e[i] * e[i]);
  }
  const double tnorm = fmax(fabs(lo), fabs(hi));
  const double pivmin = DBL_MIN * fmax(1.0, emax);
  lo -= 2.0 * DBL_EPSILON * tnorm + pivmin;
  hi += 2.0 * DBL_EPSILON * tnorm + pivmin;
  // invariant: count(lo) == 0, count(hi) >= 1 (Gershgorin bounds)
  for (int round = 0; round < 64; ++round) {
    if (hi - lo <= 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi)) + pivmin) break;
    const double x = lo + (hi - lo) * (double)(lane + 1) * (1.0 / 33.0);
    const bool above = (x < hi) && (x > lo) && sturm_count(d, e, n, x, pivmin) >= 1;
    const unsigned ball = __ballot_sync(0xffffffffu, above);
    const unsigned below = __ballot_sync(0xffffffffu, (x > lo) && (x < hi) && !above);
    // new bracket: the lowest point with count >= 1, and the highest point
    // under it with count 0 (points outside (lo, hi) by rounding are skipped)
    const int j = ball ? __ffs(ball) - 1 : 32;
    const unsigned under = below & (j >= 32 ? 0xffffffffu : ((1u << j) - 1u));
    const int i = under ? 31 - __clz(under) : -1;
    const double xj = __shfl_sync(0xffffffffu, x, j & 31);
    const double xi = __shfl_sync(0xffffffffu, x, i < 0 ? 0 : i);
    const double nhi = (j < 32) ? xj : hi;
    const double nlo = (i >= 0) ? xi : lo;
    if (nhi >= hi && nlo <= lo) break;   // no representable progress
    lo = nlo;
    hi = nhi;
  }
  const double lam = 0.5 * (lo + hi);
  if (lane != 0) return;
  res[0] = lam;
  if (!want_vec) return;
  // inverse iteration on (T - lam I) with a partially pivoted tridiagonal LU
  // (rows kept as diag/super1/super2 of U plus multipliers); n <= 127.
  double u0[128], u1[128], u2[128], lm[128], y[128];
  int piv[128];
  const double shift = lam;
  const double tiny = DBL_EPSILON * tnorm + pivmin;
  {
    double a = d[0] - shift, b = (n > 1) ? e[0] : 0.0, c = 0.0;
    for (int i = 0; i < n - 1; ++i) {
      double sub = e[i], na = d[i + 1] - shift, nb = (i + 1 < n - 1) ? e[i + 1] : 0.0;
      if (fabs(a) >= fabs(sub)) {
        piv[i] = 0;
        if (fabs(a) < tiny) a = (a < 0 ? -tiny : tiny);
        double l = sub / a;
        lm[i] = l;
        u0[i] = a; u1[i] = b; u2[i] = c;
        a = na - l * b;
        b = nb - l * c;
        c = 0.0;
      } else {
        piv[i] = 1;
        double l = a / sub;
        lm[i] = l;
        u0[i] = sub; u1[i] = na; u2[i] = nb;
        double a2 = b - l * na, b2 = c - l * nb;
        a = a2;
        b = b2;
        c = 0.0;
      }
    }
    if (fabs(a) < tiny) a = (a < 0 ? -tiny : tiny);
    u0[n - 1] = a; u1[n - 1] = 0.0; u2[n - 1] = 0.0;
  }
  for (int i = 0; i < n; ++i) y[i] = 1.0;
  for (int pass = 0; pass < 3; ++pass) {
    // forward: apply row swaps and multipliers to y
    for (int i = 0; i < n - 1; ++i) {
      if (piv[i]) {
        double t = y[i];
        y[i] = y[i + 1];
        y[i + 1] = t;
      }
      y[i + 1] -= lm[i] * y[i];
    }
    // back substitution with U (diag u0, super u1, u2)
    for (int i = n - 1; i >= 0; --i) {
      double s = y[i];
      if (i + 1 < n) s -= u1[i] * y[i + 1];
      if (i + 2 < n) s -= u2[i] * y[i + 2];
      y[i] = s / u0[i];
    }
    double nrm = 0.0;
    for (int i = 0; i < n; ++i) nrm += y[i] * y[i];
    nrm = sqrt(nrm);
    for (int i = 0; i < n; ++i) y[i] /= nrm;
  }
  int imax = 0;
  for (int i = 1; i < n; ++i)
    if (fabs(y[i]) > fabs(y[imax])) imax = i;
  const double sg = y[imax] < 0 ? -1.0 : 1.0;
  for (int i = 0; i < n; ++i) z[i] = sg * y[i];
}


__global__ void tridiag_lowest_kernel(const double* __restrict__ d, const double* __restrict__ e, int n,
                                      int want_vec, double* __restrict__ res, double* __restrict__ z) {
  tridiag_lowest_warp(d, e, n, want_vec, res, z);
}

// End of one Lanczos iteration, on the device: beta[k-1] = sqrt(n2), the
// lowest Ritz value of T_k (alpha[1..k], beta[1..k-1]), and a packet
// {ritz, n2, alpha[k]} for a single read-back by the host.
__global__ void lanczos_tail_kernel(const double* __restrict__ n2, double* __restrict__ alpha,
                                    double* __restrict__ beta, int k, double* __restrict__ res,
                                    double* __restrict__ packet, double* __restrict__ zbuf) {
  __shared__ double sd[128], se[128];
  const int lane = threadIdx.x & 31;
  const double b = sqrt(n2[0]);
  for (int i = lane; i < k; i += 32) {
    sd[i] = alpha[i + 1];
    se[i] = (i + 1 < k - 1) ? beta[i + 1] : (i + 1 == k - 1 ? b : 0.0);
  }
  __syncwarp();
  if (lane == 0) beta[k - 1] = b;
  tridiag_lowest_warp(sd, se, k, zbuf ? 1 : 0, res, zbuf);
  __syncwarp();
  if (lane == 0) {
    packet[0] = res[0];
    packet[1] = n2[0];
    packet[2] = alpha[k];
    packet[3] = zbuf ? fabs(zbuf[k - 1]) : 0.0;   // last component of the Ritz vector of T_k
  }
}

__global__ void phase_fix_kernel(double2* __restrict__ U, int rows) {
  double2* u = U + (long long)blockIdx.x * rows;
  __shared__ double sr[32], si[32];
  double zr = 0.0, zi = 0.0;
  for (int r = threadIdx.x; r < rows; r += blockDim.x) {
    double w = 1.0 / (1.0 + 0.1 * r);
    zr += u[r].x * w;
    zi += u[r].y * w;
  }
  for (int o = 16; o > 0; o >>= 1) {
    zr += __shfl_xor_sync(0xffffffffu, zr, o);
    zi += __shfl_xor_sync(0xffffffffu, zi, o);
  }
  if ((threadIdx.x & 31) == 0) {
    sr[threadIdx.x >> 5] = zr;
    si[threadIdx.x >> 5] = zi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      a += sr[w];
      b += si[w];
    }
    sr[0] = a;
    si[0] = b;
  }
  __syncthreads();
  const double a = hypot(sr[0], si[0]);
  if (a < 1e-10) return;
  const double fr = sr[0] / a, fi = -si[0] / a;
  for (int r = threadIdx.x; r < rows; r += blockDim.x) {
    double2 x = u[r];
    u[r] = make_double2(x.x * fr - x.y * fi, x.x * fi + x.y * fr);
  }
}

// ---- the same vector steps with the Lanczos index read on the device ---------------
// For a CUDA graph of one Lanczos iteration, replayed with a different index
// each time: *it is `last` (1-based, as eigen.f90), and a vector reference
// {base, ld, add} means base + (*it + add) * ld (ld = 0: base itself).
__device__ __forceinline__ double2* vref(double2* base, long long ld, int add, const int* it) {
  return ld ? base + (long long)(*it + add) * ld : base;
}

__global__ void it_update_kernel(double2* __restrict__ V, long long ld, const double* __restrict__ alpha,
                                 const double* __restrict__ beta, long long n, const int* __restrict__ it) {
  const int last = *it;
  double2* w = V + (long long)last * ld;
  const double2* v = V + (long long)(last - 1) * ld;
  const double2* vprev = last >= 2 ? V + (long long)(last - 2) * ld : nullptr;
  const double a = alpha[last];
  const double b = last >= 2 ? beta[last - 1] : 0.0;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    double2 x = w[e], p = v[e];
    x.x = x.x - a * p.x;
    x.y = x.y - a * p.y;
    if (vprev) {
      double2 q = vprev[e];
      x.x = x.x - b * q.x;
      x.y = x.y - b * q.y;
    }
    w[e] = x;
  }
}

// partial sums of Re<x_j, y>, j < nvec = (nvec_it ? *it : 0) + nvec_add, x_j = X + j * xs
__global__ void it_dot_partial(double2* X, long long xld, int xadd, long long xs, int nvec_it, int nvec_add,
                               double2* Y, long long yld, int yadd, long long n, double* __restrict__ partial,
                               int nblk, const int* __restrict__ it) {
  __shared__ double red[VB / 32];
  const double2* x0 = vref(X, xld, xadd, it);
  const double2* y = vref(Y, yld, yadd, it);
  const int nvec = (nvec_it ? *it : 0) + nvec_add;
  const long long beg = (long long)blockIdx.x * VCHUNK;
  const long long end = beg + VCHUNK < n ? beg + VCHUNK : n;
  for (int j = 0; j < nvec; ++j) {
    const double2* x = x0 + (long long)j * xs;
    double acc = 0.0;
    for (long long e = beg + threadIdx.x; e < end; e += VB) {
      double2 a = x[e], b = y[e];
      acc = fma(a.x, b.x, acc);
      acc = fma(a.y, b.y, acc);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double sacc = 0.0;
      for (int w = 0; w < VB / 32; ++w) sacc += red[w];
      partial[(long long)j * nblk + blockIdx.x] = sacc;
    }
    __syncthreads();
  }
}

// out[(out_it ? *it : 0) + out_add + j] = sum of the partials of j, for j < nvec (one block per j)
__global__ void it_dot_final(const double* __restrict__ partial, int nblk, int nvec_it, int nvec_add,
                             double* __restrict__ out, int out_it, int out_add, const int* __restrict__ it) {
  const int j = blockIdx.x;
  if (j >= (nvec_it ? *it : 0) + nvec_add) return;
  __shared__ double red[32];
  double acc = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) acc += partial[(long long)j * nblk + b];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double sacc = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) sacc += red[w];
    out[(out_it ? *it : 0) + out_add + j] = sacc;
  }
}

__global__ void it_scale_kernel(double2* W, long long wld, int wadd, const double* __restrict__ norm2, long long n,
                                const int* __restrict__ it) {
  double2* w = vref(W, wld, wadd, it);
  const double s = sqrt(*norm2);
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    double2 x = w[e];
    x.x = x.x / s;
    x.y = x.y / s;
    w[e] = x;
  }
}

// w = v(last+1) - sum_{j<last} (uv_j/uu_j) v(j+1)
__global__ void it_gs_kernel(double2* __restrict__ V, long long ld, const double* __restrict__ uv,
                             const double* __restrict__ uu, long long n, const int* __restrict__ it) {
  const int nvec = *it;
  double2* w = V + (long long)nvec * ld;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    double tr = 0.0, tim = 0.0;
    for (int j = 0; j < nvec; ++j) {
      const double c = uv[j] / uu[j];
      double2 x = V[(long long)j * ld + e];
      tr = tr + c * x.x;
      tim = tim + c * x.y;
    }
    double2 x = w[e];
    x.x = x.x - tr;
    x.y = x.y - tim;
    w[e] = x;
  }
}

__global__ void it_copy_kernel(double2* D, long long dld, int dadd, double2* S, long long sld, int sadd, long long n,
                               const int* __restrict__ it) {
  double2* d = vref(D, dld, dadd, it);
  const double2* src = vref(S, sld, sadd, it);
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
    d[e] = src[e];
}

__global__ void it_tail_kernel(const double* __restrict__ n2, double* __restrict__ alpha, double* __restrict__ beta,
                               double* __restrict__ res, double* __restrict__ packet, double* __restrict__ zbuf,
                               const int* __restrict__ it) {
  __shared__ double sd[128], se[128];
  const int k = *it + 1;
  if (k < 1 || k > 127) return;
  const int lane = threadIdx.x & 31;
  const double b = sqrt(n2[0]);
  for (int i = lane; i < k; i += 32) {
    sd[i] = alpha[i + 1];
    se[i] = (i + 1 < k - 1) ? beta[i + 1] : (i + 1 == k - 1 ? b : 0.0);
  }
  __syncwarp();
  if (lane == 0) beta[k - 1] = b;
  tridiag_lowest_warp(sd, se, k, zbuf ? 1 : 0, res, zbuf);
  __syncwarp();
  if (lane == 0) {
    packet[0] = res[0];
    packet[1] = n2[0];
    packet[2] = alpha[k];
    packet[3] = zbuf ? fabs(zbuf[k - 1]) : 0.0;
  }
}

inline int grid_for(long long n) {
  long long b = (n + VB - 1) / VB;
  if (b > 148 * 16) b = 148 * 16;
  if (b < 1) b = 1;
  return (int)b;
}

}  // namespace

template <int TM, int TN, int MINB>
cudaError_t launch_tile(const GJob* jobs, int njobs, const GGroup* groups, const GTerm* terms, Bases bases,
                        cudaStream_t st) {
  const size_t smem = sizeof(SmemTiles<TM, TN>);
  static std::atomic<unsigned long long> attr{0};
  cudaError_t e = ensure_smem_attr(grouped_zgemm_kernel<TM, TN, MINB>, (int)smem, attr);
  if (e != cudaSuccess) return e;
  grouped_zgemm_kernel<TM, TN, MINB><<<njobs, GEMM_THREADS, smem, st>>>(jobs, groups, terms, bases);
  return cudaGetLastError();
}

cudaError_t launch_grouped_zgemm(const GJob* jobs, int njobs, const GGroup* groups, const GTerm* terms,
                                 Bases bases, cudaStream_t st, int tile) {
  if (njobs <= 0) return cudaSuccess;
  switch (tile) {
    case TILE_32x32: return launch_tile<32, 32, 6>(jobs, njobs, groups, terms, bases, st);
    case TILE_64x32: return launch_tile<64, 32, 4>(jobs, njobs, groups, terms, bases, st);
    case TILE_32x64: return launch_tile<32, 64, 4>(jobs, njobs, groups, terms, bases, st);
    default: return launch_tile<64, 64, 2>(jobs, njobs, groups, terms, bases, st);
  }
}

cudaError_t launch_reduce_partials(const GReduce* reds, int nred, const GGroup* groups, Bases bases,
                                   long long max_elems, cudaStream_t st) {
  if (nred <= 0) return cudaSuccess;
  long long bx = (max_elems + 255) / 256;
  if (bx > 64) bx = 64;
  if (bx < 1) bx = 1;
  dim3 grid((unsigned)bx, (unsigned)nred);
  reduce_partials_kernel<<<grid, 256, 0, st>>>(reds, groups, bases);
  return cudaGetLastError();
}

cudaError_t launch_multi_dot(const double2* X, long long ld, int nvec, const double2* y, long long n,
                             double* partial, double* out, cudaStream_t st) {
  if (nvec <= 0) return cudaSuccess;
  int nblk = (int)((n + VCHUNK - 1) / VCHUNK);
  if (nblk < 1) nblk = 1;
  multi_dot_partial<<<nblk, VB, 0, st>>>(X, ld, nvec, y, n, partial, nblk);
  multi_dot_final<<<nvec, 256, 0, st>>>(partial, nblk, nvec, out);
  return cudaGetLastError();
}

cudaError_t launch_zdot(const double2* x, const double2* y, long long n, double* partial, double* out,
                        cudaStream_t st) {
  int nblk = (int)((n + VCHUNK - 1) / VCHUNK);
  if (nblk < 1) nblk = 1;
  zdot_partial<<<nblk, VB, 0, st>>>(x, y, n, partial, nblk);
  multi_dot_final<<<2, 256, 0, st>>>(partial, nblk, 2, out);
  return cudaGetLastError();
}

cudaError_t launch_lanczos_update(double2* w, const double2* v, const double2* vprev, const double* alpha,
                                  const double* beta_prev, long long n, cudaStream_t st) {
  lanczos_update_kernel<<<grid_for(n), VB, 0, st>>>(w, v, vprev, alpha, beta_prev, n);
  return cudaGetLastError();
}

cudaError_t launch_scale(double2* w, const double* norm2, long long n, int invert_sqrt, cudaStream_t st) {
  scale_kernel<<<grid_for(n), VB, 0, st>>>(w, norm2, n, invert_sqrt);
  return cudaGetLastError();
}

cudaError_t launch_gs_subtract(double2* w, const double2* X, long long ld, int nvec, const double* uv,
                               const double* uu, long long n, cudaStream_t st) {
  gs_subtract_kernel<<<grid_for(n), VB, 0, st>>>(w, X, ld, nvec, uv, uu, n);
  return cudaGetLastError();
}

cudaError_t launch_combine(double2* out, const double2* X, long long ld, int nvec, const double* z, long long n,
                           cudaStream_t st) {
  combine_kernel<<<grid_for(n), VB, 0, st>>>(out, X, ld, nvec, z, n);
  return cudaGetLastError();
}

cudaError_t launch_phase_fix(double2* U, int rows, int cols, cudaStream_t st) {
  if (rows <= 0 || cols <= 0) return cudaSuccess;
  phase_fix_kernel<<<cols, 128, 0, st>>>(U, rows);
  return cudaGetLastError();
}

cudaError_t launch_tridiag_lowest(const double* d, const double* e, int n, int want_vec, double* res, double* z,
                                  cudaStream_t st) {
  if (n < 1 || n > 127) return cudaErrorInvalidValue;
  tridiag_lowest_kernel<<<1, 32, 0, st>>>(d, e, n, want_vec, res, z);
  return cudaGetLastError();
}

cudaError_t launch_it_update(double2* V, long long ld, const double* alpha, const double* beta, long long n,
                             const int* it, cudaStream_t st) {
  it_update_kernel<<<grid_for(n), VB, 0, st>>>(V, ld, alpha, beta, n, it);
  return cudaGetLastError();
}

cudaError_t launch_it_dot(ItRef x, long long xs, int nvec_it, int nvec_add, int nvec_max, ItRef y, long long n,
                          double* partial, double* out, int out_it, int out_add, const int* it, cudaStream_t st) {
  int nblk = (int)((n + VCHUNK - 1) / VCHUNK);
  if (nblk < 1) nblk = 1;
  if (nvec_max <= 0) return cudaSuccess;
  it_dot_partial<<<nblk, VB, 0, st>>>(x.base, x.ld, x.add, xs, nvec_it, nvec_add, y.base, y.ld, y.add, n, partial,
                                      nblk, it);
  it_dot_final<<<nvec_max, 256, 0, st>>>(partial, nblk, nvec_it, nvec_add, out, out_it, out_add, it);
  return cudaGetLastError();
}

cudaError_t launch_it_scale(ItRef w, const double* norm2, long long n, const int* it, cudaStream_t st) {
  it_scale_kernel<<<grid_for(n), VB, 0, st>>>(w.base, w.ld, w.add, norm2, n, it);
  return cudaGetLastError();
}

cudaError_t launch_it_gs(double2* V, long long ld, const double* uv, const double* uu, long long n, const int* it,
                         cudaStream_t st) {
  it_gs_kernel<<<grid_for(n), VB, 0, st>>>(V, ld, uv, uu, n, it);
  return cudaGetLastError();
}

cudaError_t launch_it_copy(ItRef dst, ItRef src, long long n, const int* it, cudaStream_t st) {
  it_copy_kernel<<<grid_for(n), VB, 0, st>>>(dst.base, dst.ld, dst.add, src.base, src.ld, src.add, n, it);
  return cudaGetLastError();
}

cudaError_t launch_it_tail(const double* n2, double* alpha, double* beta, double* res, double* packet, double* zbuf,
                           const int* it, cudaStream_t st) {
  it_tail_kernel<<<1, 32, 0, st>>>(n2, alpha, beta, res, packet, zbuf, it);
  return cudaGetLastError();
}

cudaError_t launch_lanczos_tail(const double* n2, double* alpha, double* beta, int k, double* res, double* packet,
                                double* zbuf, cudaStream_t st) {
  if (k < 1 || k > 127) return cudaErrorInvalidValue;
  lanczos_tail_kernel<<<1, 32, 0, st>>>(n2, alpha, beta, k, res, packet, zbuf);
  return cudaGetLastError();
}

}  // namespace tsc
