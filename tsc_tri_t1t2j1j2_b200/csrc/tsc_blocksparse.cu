// Block-sparse H.psi on a batch of independent problems, every problem of the
// batch in the same two grouped launches (the benchmark list's synthetic H.psi
// and its "uneven batches of independent superblocks"; no counterpart in the
// reference, whose model_wave handles one superblock at a time).
//
// Problem p: K sectors, psi sector i a d_i x e_i block.  Left operator sets L_a
// hold blocks L_a[i] (d_{i+s_a} x d_i), right sets R_b blocks R_b[i]
// (e_{i+s_b} x e_i), for every i with 0 <= i+s < K.  A term (alpha, a, b) with
// s_a == s_b adds alpha * L_a[i] * X_i * R_b[i]^H to Y_{i+s}.  As in model_wave's
// block-block terms (get_sys.f90:3131-3569) the left product T = L_a[i] X_i is
// formed once per (a, i) in phase 1 and shared by every term that uses it;
// phase 2 sums, per output sector, alpha * T * R_b[i]^H over its terms.
#include <algorithm>
#include <map>
#include <tuple>

#include "../../include/tsc_gpu.h"
#include "tsc_ctx.hpp"
#include "tsc_engine.hpp"

using namespace tsc;

namespace tsc {

void Engine::blocksparse_set(int nprob, const int* ints, long long nints, const cplx* data, long long ncplx) {
  bs = BlockSparse();
  std::vector<cplx> ops;          // host copy of every operator block, then uploaded once
  struct OpRefB {
    long long off;                // element offset in ops
    int rows, cols;
  };
  struct Prob {
    int K;
    std::vector<int> d, e;
    std::vector<long long> xoff;  // psi sector offsets (global)
    std::vector<int> ls, rs;      // shifts of the left / right sets
    std::vector<std::vector<OpRefB>> L, R;   // [set][i]
    std::vector<std::pair<int, int>> terms;
    std::vector<cplx> alpha;
  };
  std::vector<Prob> probs(nprob);
  const int* ip = ints;
  const int* iend = ints + nints;
  const cplx* dp = data;
  const cplx* dend = data + ncplx;
  auto take = [&](int n) {
    if (ip + n > iend) throw Error(TSC_E_ARG, "blocksparse: descriptor ints run short");
    const int* r = ip;
    ip += n;
    return r;
  };
  long long dim = 0;
  double flops = 0.0;
  for (auto& P : probs) {
    const int* h = take(4);
    P.K = h[0];
    const int nL = h[1], nR = h[2], nT = h[3];
    if (P.K < 1 || nL < 0 || nR < 0 || nT < 0 || P.K > 1000000) throw Error(TSC_E_ARG, "blocksparse: bad problem header");
    const int* de = take(2 * P.K);
    for (int i = 0; i < P.K; ++i) {
      P.d.push_back(de[2 * i]);
      P.e.push_back(de[2 * i + 1]);
      if (de[2 * i] < 1 || de[2 * i + 1] < 1) throw Error(TSC_E_ARG, "blocksparse: sector dimensions must be positive");
      P.xoff.push_back(dim);
      dim += (long long)de[2 * i] * de[2 * i + 1];
    }
    const int* sh = take(nL + nR);
    P.ls.assign(sh, sh + nL);
    P.rs.assign(sh + nL, sh + nL + nR);
    const int* tt = take(2 * nT);
    for (int t = 0; t < nT; ++t) {
      const int a = tt[2 * t], b = tt[2 * t + 1];
      if (a < 0 || a >= nL || b < 0 || b >= nR) throw Error(TSC_E_ARG, "blocksparse: term names no such operator set");
      if (P.ls[a] != P.rs[b]) throw Error(TSC_E_QN, "blocksparse: a term's left and right sets shift sectors differently");
      P.terms.push_back({a, b});
    }
    auto read_sets = [&](const std::vector<int>& shifts, const std::vector<int>& rdim, std::vector<std::vector<OpRefB>>& S) {
      S.resize(shifts.size());
      for (size_t a = 0; a < shifts.size(); ++a) {
        S[a].assign(P.K, OpRefB{-1, 0, 0});
        for (int i = 0; i < P.K; ++i) {
          const int j = i + shifts[a];
          if (j < 0 || j >= P.K) continue;
          const long long n = (long long)rdim[j] * rdim[i];
          if (dp + n > dend) throw Error(TSC_E_ARG, "blocksparse: operator data run short");
          S[a][i] = OpRefB{(long long)ops.size(), rdim[j], rdim[i]};
          ops.insert(ops.end(), dp, dp + n);
          dp += n;
        }
      }
    };
    read_sets(P.ls, P.d, P.L);
    read_sets(P.rs, P.e, P.R);
    if (dp + nT > dend) throw Error(TSC_E_ARG, "blocksparse: term coefficients run short");
    P.alpha.assign(dp, dp + nT);
    dp += nT;
  }
  if (ip != iend || dp != dend) throw Error(TSC_E_ARG, "blocksparse: descriptor and data lengths do not match the problems");

  bs.ops = std::make_shared<DevBuf>((size_t)std::max<size_t>(ops.size(), 1), st, false);
  if (!ops.empty())
    cuda_check(cudaMemcpyAsync(bs.ops->p, ops.data(), ops.size() * sizeof(double2), cudaMemcpyHostToDevice, st), "h2d");
  const double2* obase = bs.ops->p;
  auto op_abs = [&](const OpRefB& r) { return (long long)((uintptr_t)(obase + r.off) / sizeof(double2)); };

  long long scr = 0;
  for (auto& P : probs) {
    // phase 1: T(a, i) = L_a[i] X_i, once per (a, i) that some term uses
    std::map<std::pair<int, int>, long long> tmid;
    // phase 2 groups: every output sector, written once (zero when no term reaches it)
    std::vector<int> g2(P.K);
    for (int j = 0; j < P.K; ++j) g2[j] = bs.p2.add_group(nullptr, BASE_OUT, P.xoff[j], P.d[j], P.d[j], P.e[j], 0);
    for (size_t t = 0; t < P.terms.size(); ++t) {
      const int a = P.terms[t].first, b = P.terms[t].second, s = P.ls[a];
      for (int i = 0; i < P.K; ++i) {
        const int j = i + s;
        if (j < 0 || j >= P.K) continue;
        auto key = std::make_pair(a, i);
        auto it = tmid.find(key);
        if (it == tmid.end()) {
          const long long off = scr;
          scr += (long long)P.d[j] * P.e[i];
          const int g = bs.p1.add_group(nullptr, BASE_SCR, off, P.d[j], P.d[j], P.e[i], 0);
          GTerm m{};
          m.kind = TK_GEMM;
          m.ar = 1.0;
          m.l_base = BASE_ABS;
          m.l_off = op_abs(P.L[a][i]);
          m.l_ld = P.d[j];
          m.l_op = OP_N;
          m.r_base = BASE_IN;
          m.r_off = P.xoff[i];
          m.r_ld = P.d[i];
          m.r_op = OP_N;
          m.K = P.d[i];
          bs.p1.gterms[g].push_back(m);
          it = tmid.emplace(key, off).first;
        }
        GTerm o{};
        o.kind = TK_GEMM;
        o.ar = P.alpha[t].real();
        o.ai = P.alpha[t].imag();
        o.l_base = BASE_SCR;
        o.l_off = it->second;
        o.l_ld = P.d[j];
        o.l_op = OP_N;
        o.r_base = BASE_ABS;
        o.r_off = op_abs(P.R[b][i]);
        o.r_ld = P.e[j];
        o.r_op = OP_C;
        o.K = P.e[i];
        bs.p2.gterms[g2[j]].push_back(o);
        // algorithmic flops: both GEMMs of the term, as model_wave's block-block kernels count them
        flops += 8.0 * P.d[j] * P.d[i] * P.e[i] + 8.0 * P.d[j] * P.e[i] * P.e[j];
      }
    }
  }
  bs.scratch = std::make_shared<DevBuf>((size_t)std::max<long long>(scr, 1), st, false);
  bs.p1s.groups = bs.p1.groups;
  bs.p1s.gterms = bs.p1.gterms;
  bs.p2s.groups = bs.p2.groups;
  bs.p2s.gterms = bs.p2.gterms;
  bs.p1.upload(st);
  bs.p2.upload(st);
  // 200 terms share 16 operator sets: one view per operator block, coefficients in the epilogue
  build_split_views(bs.p1s, bs.p2s, bs.sv, st, true);
  bs.p1s.upload_split(st);
  bs.p2s.upload_split(st);
  bs.p1.gterms.clear();
  bs.p2.gterms.clear();
  bs.p1s.gterms.clear();
  bs.p2s.gterms.clear();
  bs.dim = dim;
  bs.ref_flops = flops;
  bs.nprob = nprob;
  cuda_check(cudaStreamSynchronize(st), "blocksparse sync");
  bs.valid = true;
  views_of_batch_ = true;
}

void Engine::blocksparse_apply(const double2* d_in, double2* d_out, bool split) {
  if (!bs.valid) throw Error(TSC_E_STATE, "no block-sparse batch set");
  TaskList& a = split ? bs.p1s : bs.p1;
  TaskList& b = split ? bs.p2s : bs.p2;
  cuda_check(cudaEventRecord(ev0, st), "event");
  if (split) slice_input(bs.sv, d_in, st);
  run_tasks(a, const_cast<double2*>(d_in), d_out, bs.scratch->p);
  run_tasks(b, const_cast<double2*>(d_in), d_out, bs.scratch->p);
  cuda_check(cudaEventRecord(ev1, st), "event");
  last_stats.hpsi_flops = bs.ref_flops;
  last_stats.launches = (a.njobs > 0) + (b.njobs > 0) + (a.nreds > 0) + (b.nreds > 0) + (split ? 1 : 0);
}

}  // namespace tsc

extern "C" int tsc_blocksparse_set(tsc_ctx* ctx, int nproblems, const int* ints, long long nints, const double* data,
                                   long long ncplx, long long* dim, double* flops, double* exec_flops) {
  return guard(ctx, [&] {
    if (!ctx->eng) throw Error(TSC_E_STATE, "no engine");
    if (nproblems < 1 || !ints || nints < 4 || (ncplx > 0 && !data) || ncplx < 0)
      throw Error(TSC_E_ARG, "blocksparse: bad arguments");
    ctx->eng->blocksparse_set(nproblems, ints, nints, reinterpret_cast<const cplx*>(data), ncplx);
    if (dim) *dim = ctx->eng->bs.dim;
    if (flops) *flops = ctx->eng->bs.ref_flops;
    if (exec_flops) *exec_flops = ctx->eng->bs.p1.exec_flops + ctx->eng->bs.p2.exec_flops;
  });
}

extern "C" int tsc_blocksparse_apply(tsc_ctx* ctx, const void* d_in, void* d_out, int mode) {
  return guard(ctx, [&] {
    if (!ctx->eng) throw Error(TSC_E_STATE, "no engine");
    if (!d_in || !d_out) throw Error(TSC_E_ARG, "null buffers");
    if (mode != TSC_FP64 && mode != TSC_SPLIT_BF16) throw Error(TSC_E_ARG, "unknown precision mode");
    ctx->eng->blocksparse_apply(static_cast<const double2*>(d_in), static_cast<double2*>(d_out), mode == TSC_SPLIT_BF16);
    // the split form waits for its launches and reports a wait that ran out
    if (mode == TSC_SPLIT_BF16) ctx->eng->check_split_fault();
  });
}
