// Canonical complement basis for kept zero-weight multiplets, on the GPU.
//
// When a sector keeps more multiplets than its density matrix has weight, the
// kept zero-weight columns of U are replaced by a canonical orthonormal basis:
// Gram-Schmidt of the unit vectors e_0, e_1, ... against the kept significant
// eigenvectors Q and the vectors accepted so far, a candidate being accepted
// when its residual norm exceeds 0.5, then (second sweep over j) 0.1, then 1e-3.
// The reference keeps whatever null-space eigenvectors its LAPACK returns
// (den_mat.f90:395-396); the canonical choice makes the kept space independent
// of the eigensolver.
//
// Candidates are processed in blocks of kNullB unit vectors, every sector of the
// step in the same launches:
//   C  = E_J - W W[J,:]^H               first projection (W = [Q | accepted])
//   C -= W (W^H C)                       second projection
//   select: within the block, each candidate in order is projected against the
//           block's newly accepted vectors (twice), tested against the
//           threshold and, if accepted, normalised into the next free column.
// The three products run on the grouped FP64 tensor-core GEMM; the selection is
// one CTA per sector.  In exact arithmetic this is the sequential procedure.
#include <algorithm>

#include "tsc_engine.hpp"

namespace tsc {
namespace {

constexpr int kNullB = 32;         // candidate unit vectors per block
constexpr int kNullThreads = 256;
constexpr int kNullChunk = 8;      // accepted vectors per dot-product chunk

struct NullSel {
  double2* C;     // d x bw candidate block (ld d), already projected against W
  double2* N;     // accepted vectors go to columns got, got+1, ... (ld d)
  int d, bw, j0, got, cap;
  double thr;
};

__global__ void null_unit_kernel(const NullSel* jobs) {
  const NullSel J = jobs[blockIdx.x];
  const long long n = (long long)J.d * J.bw;
  for (long long i = threadIdx.x; i < n; i += blockDim.x) {
    const int c = (int)(i / J.d), r = (int)(i - (long long)c * J.d);
    J.C[i] = make_double2(r == J.j0 + c ? 1.0 : 0.0, 0.0);
  }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__global__ void __launch_bounds__(kNullThreads) null_select_kernel(const NullSel* jobs, int* counts) {
  const NullSel J = jobs[blockIdx.x];
  __shared__ double red[kNullThreads / 32][2 * kNullChunk];
  __shared__ double coef[2 * kNullChunk];
  __shared__ double nrm_s;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int na = 0;
  for (int c = 0; c < J.bw && na < J.cap; ++c) {
    double2* v = J.C + (long long)c * J.d;
    for (int pass = 0; pass < 2; ++pass) {
      for (int a0 = 0; a0 < na; a0 += kNullChunk) {
        const int nc = min(kNullChunk, na - a0);
        const double2* Nb = J.N + (long long)(J.got + a0) * J.d;
        double acc[2 * kNullChunk];
#pragma unroll
        for (int i = 0; i < 2 * kNullChunk; ++i) acc[i] = 0.0;
        for (int r = tid; r < J.d; r += kNullThreads) {
          const double2 x = v[r];
#pragma unroll
          for (int a = 0; a < kNullChunk; ++a)
            if (a < nc) {
              const double2 q = Nb[(long long)a * J.d + r];
              acc[2 * a] += q.x * x.x + q.y * x.y;       // conj(q) x
              acc[2 * a + 1] += q.x * x.y - q.y * x.x;
            }
        }
#pragma unroll
        for (int i = 0; i < 2 * kNullChunk; ++i) {
          const double s = warp_sum(acc[i]);
          if (lane == 0) red[warp][i] = s;
        }
        __syncthreads();
        if (tid < 2 * kNullChunk) {
          double s = 0.0;
          for (int w = 0; w < kNullThreads / 32; ++w) s += red[w][tid];
          coef[tid] = s;
        }
        __syncthreads();
        for (int r = tid; r < J.d; r += kNullThreads) {
          double2 x = v[r];
#pragma unroll
          for (int a = 0; a < kNullChunk; ++a)
            if (a < nc) {
              const double2 q = Nb[(long long)a * J.d + r];
              const double cr = coef[2 * a], ci = coef[2 * a + 1];
              x.x -= cr * q.x - ci * q.y;
              x.y -= cr * q.y + ci * q.x;
            }
          v[r] = x;
        }
        __syncthreads();
      }
    }
    double s = 0.0;
    for (int r = tid; r < J.d; r += kNullThreads) {
      const double2 x = v[r];
      s += x.x * x.x + x.y * x.y;
    }
    s = warp_sum(s);
    if (lane == 0) red[warp][0] = s;
    __syncthreads();
    if (tid == 0) {
      double t = 0.0;
      for (int w = 0; w < kNullThreads / 32; ++w) t += red[w][0];
      nrm_s = sqrt(t);
    }
    __syncthreads();
    const double nrm = nrm_s;
    if (nrm > J.thr) {
      double2* out = J.N + (long long)(J.got + na) * J.d;
      for (int r = tid; r < J.d; r += kNullThreads) {
        const double2 x = v[r];
        out[r] = make_double2(x.x / nrm, x.y / nrm);
      }
      ++na;
    }
    __syncthreads();
  }
  if (tid == 0) counts[blockIdx.x] = na;
}

inline long long abs_index(const double2* p) { return (long long)((uintptr_t)p / sizeof(double2)); }

GTerm gemm_term(const double2* l, int l_ld, uint8_t l_op, const double2* r, int r_ld, uint8_t r_op, int K, double ar) {
  GTerm t{};
  t.kind = TK_GEMM;
  t.ar = ar;
  t.l_base = t.r_base = BASE_ABS;
  t.l_off = abs_index(l);
  t.l_ld = l_ld;
  t.l_op = l_op;
  t.r_off = abs_index(r);
  t.r_ld = r_ld;
  t.r_op = r_op;
  t.K = K;
  return t;
}

}  // namespace

void Engine::null_complete(const std::vector<NullJob>& jobs) {
  if (jobs.empty()) return;
  const double thrs[3] = {0.5, 0.1, 1e-3};
  const int nj = (int)jobs.size();
  struct State {
    int thr = 0, j0 = 0, got = 0;
    bool done = false;
  };
  std::vector<State> S(nj);
  // scratch per job: C (d x B) and H ((sig + m) x B)
  std::vector<long long> coff(nj), hoff(nj);
  long long tot = 0;
  for (int i = 0; i < nj; ++i) {
    const NullJob& J = jobs[i];
    if (J.d < 1 || J.sig < 0 || J.m < 1 || J.sig + J.m > J.d) throw Error(-1, "null completion: bad sector shape");
    coff[i] = tot;
    tot += (long long)J.d * kNullB;
    hoff[i] = tot;
    tot += (long long)(J.sig + J.m) * kNullB;
  }
  DevBuf scr((size_t)tot, st, false);
  DevBuf dsel((size_t)(nj * sizeof(NullSel) + sizeof(double2) - 1) / sizeof(double2) + 1, st, false);
  DevBuf dcnt((size_t)(nj + 3) / 4 + 1, st, false);
  NullSel* d_sel = reinterpret_cast<NullSel*>(dsel.p);
  int* d_cnt = reinterpret_cast<int*>(dcnt.p);
  std::vector<NullSel> sel;
  std::vector<int> act, cnt(nj);
  while (true) {
    act.clear();
    sel.clear();
    for (int i = 0; i < nj; ++i) {
      if (S[i].done) continue;
      const NullJob& J = jobs[i];
      NullSel s;
      s.C = scr.p + coff[i];
      s.N = J.W;
      s.d = J.d;
      s.j0 = S[i].j0;
      s.bw = std::min(kNullB, J.d - S[i].j0);
      s.got = S[i].got;
      s.cap = J.m - S[i].got;
      s.thr = thrs[S[i].thr];
      act.push_back(i);
      sel.push_back(s);
    }
    if (act.empty()) break;
    const int na = (int)act.size();
    cuda_check(cudaMemcpyAsync(d_sel, sel.data(), na * sizeof(NullSel), cudaMemcpyHostToDevice, st), "h2d");
    null_unit_kernel<<<na, 256, 0, st>>>(d_sel);
    cuda_check(cudaGetLastError(), "null_unit");
    TaskList t1, t2, t3;
    for (int a = 0; a < na; ++a) {
      const int i = act[a];
      const NullJob& J = jobs[i];
      const NullSel& s = sel[a];
      const int g = s.got;
      if (J.sig + g == 0) continue;
      const double2* Q = J.W + (long long)J.m * J.d;   // significant vectors, after the m completion columns
      const double2* Nv = J.W;
      double2* H = scr.p + hoff[i];
      const int hld = J.sig + J.m;
      // C -= Q Q[J,:]^H + N N[J,:]^H
      int gi = t1.add_group(s.C, BASE_ABS, 0, J.d, J.d, s.bw, 1);
      if (J.sig) t1.gterms[gi].push_back(gemm_term(Q, J.d, OP_N, Q + s.j0, J.d, OP_C, J.sig, -1.0));
      if (g) t1.gterms[gi].push_back(gemm_term(Nv, J.d, OP_N, Nv + s.j0, J.d, OP_C, g, -1.0));
      // H = [Q N]^H C
      if (J.sig) {
        gi = t2.add_group(H, BASE_ABS, 0, hld, J.sig, s.bw, 0);
        t2.gterms[gi].push_back(gemm_term(Q, J.d, OP_C, s.C, J.d, OP_N, J.d, 1.0));
      }
      if (g) {
        gi = t2.add_group(H + J.sig, BASE_ABS, 0, hld, g, s.bw, 0);
        t2.gterms[gi].push_back(gemm_term(Nv, J.d, OP_C, s.C, J.d, OP_N, J.d, 1.0));
      }
      // C -= Q H_Q + N H_N
      gi = t3.add_group(s.C, BASE_ABS, 0, J.d, J.d, s.bw, 1);
      if (J.sig) t3.gterms[gi].push_back(gemm_term(Q, J.d, OP_N, H, hld, OP_N, J.sig, -1.0));
      if (g) t3.gterms[gi].push_back(gemm_term(Nv, J.d, OP_N, H + J.sig, hld, OP_N, g, -1.0));
    }
    if (!t1.groups.empty()) {
      t1.upload(st);
      run_tasks(t1, nullptr, nullptr, nullptr);
      t2.upload(st);
      run_tasks(t2, nullptr, nullptr, nullptr);
      t3.upload(st);
      run_tasks(t3, nullptr, nullptr, nullptr);
    }
    null_select_kernel<<<na, kNullThreads, 0, st>>>(d_sel, d_cnt);
    cuda_check(cudaGetLastError(), "null_select");
    cuda_check(cudaMemcpyAsync(cnt.data(), d_cnt, na * sizeof(int), cudaMemcpyDeviceToHost, st), "d2h");
    cuda_check(cudaStreamSynchronize(st), "null completion sync");
    for (int a = 0; a < na; ++a) {
      State& s = S[act[a]];
      const NullJob& J = jobs[act[a]];
      s.got += cnt[a];
      if (s.got >= J.m) {
        s.done = true;
        continue;
      }
      s.j0 += kNullB;
      if (s.j0 >= J.d) {
        s.j0 = 0;
        if (++s.thr == 3) throw Error(-1, "null completion: complement too small");
      }
    }
  }
}

}  // namespace tsc
