// H.psi on the device: hmerge (get_sys.f90:7398-7626) and the model_wave term
// list (get_sys.f90:6915-7068) turned into grouped-GEMM tasks.
//
// Output groups are the (psi sector, sys piece, env piece) rectangles of H.psi;
// each group sums every term that lands in it, so phase 2 writes the whole
// output exactly once (no zeroing pass, no atomics).  Products with an operator
// on both sides (block_vec_block_*) keep the reference's association
// (O_sys.psi).O_env: the left products O_sys.psi_(i,m,n) are computed once in
// phase 1 and shared by every (env op sub-block, new total spin) that uses them
// -- the reuse the reference forgoes when it recomputes GEMM1 per task
// (get_sys.f90:3384-3389).  Coefficients, signs and sector searches follow the
// reference kernels (get_sys.f90:1783-5204) term by term.
#include <algorithm>
#include <cmath>
#include <map>
#include <tuple>

#include "tsc_engine.hpp"

namespace tsc {

namespace {

inline uint8_t flip(uint8_t op) { return op == OP_N ? OP_C : OP_N; }
inline double sgn(int n) { return (n % 2 == 0) ? 1.0 : -1.0; }
inline double pm1(int e) { return ((e % 2) + 2) % 2 == 0 ? 1.0 : -1.0; }

// A block operator or its conjugate transpose (block_transfer_trans, block.f90:33-64)
struct OpRef {
  const DBlock* b = nullptr;
  bool ct = false;
  int up_dif() const { return ct ? -b->up_dif : b->up_dif; }
  int K() const { return b->down_dif; }
  int num() const { return b->num; }
  SubDesc s(int k) const {
    const SubDesc& x = b->sub[k];
    if (!ct) return x;
    SubDesc y;
    y.num_up = x.num_up + b->up_dif;
    y.num_down = x.num_down + x.down_dif;
    y.down_dif = -x.down_dif;
    y.row_dim = x.sdim;
    y.sdim = x.row_dim;
    y.off = x.off;
    return y;
  }
  int find2(int up, int down) const {
    for (int k = 0; k < num(); ++k) {
      SubDesc x = s(k);
      if (x.num_up == up && x.num_down == down) return k;
    }
    return -1;
  }
  int find3(int up, int down, int dd) const {
    for (int k = 0; k < num(); ++k) {
      SubDesc x = s(k);
      if (x.num_up == up && x.num_down == down && x.down_dif == dd) return k;
    }
    return -1;
  }
};

// Site operator (1x1 sub-blocks) and its conjugate transpose
struct SiteRef {
  int up_dif, down_dif;
  std::vector<SiteSub> sub;
  int find2(int up, int down) const {
    for (size_t k = 0; k < sub.size(); ++k)
      if (sub[k].num_up == up && sub[k].num_down == down) return (int)k;
    return -1;
  }
  int find3(int up, int down, int dd) const {
    for (size_t k = 0; k < sub.size(); ++k)
      if (sub[k].num_up == up && sub[k].num_down == down && sub[k].down_dif == dd) return (int)k;
    return -1;
  }
};
SiteRef site(const SiteOp& o) { return SiteRef{o.up_dif, o.down_dif, o.sub}; }
SiteRef site_ct(const SiteOp& o) {
  SiteRef r{-o.up_dif, o.down_dif, {}};
  for (auto& s : o.sub) r.sub.push_back({s.num_up + o.up_dif, s.num_down + s.down_dif, -s.down_dif, s.val});
  return r;
}

struct Builder {
  Engine& E;
  Engine::Superblock& S;
  const Basis& sbs;
  const Basis& ebs;
  const WLayout& wl;
  std::vector<int> xs, ye;                      // psi sector -> sys_bs / env_bs sector
  std::vector<std::vector<std::vector<int>>> grp;   // [k][a][b] -> phase-2 group
  std::map<std::tuple<long long, int, int, int, int, int, int>, long long> inter;
  double ref_flops = 0;
  long long scr = 0;

  Builder(Engine& e) : E(e), S(e.sb), sbs(e.sb.sys_bs), ebs(e.sb.env_bs), wl(e.sb.wl) {
    S.p1 = TaskList();
    S.p2 = TaskList();
    for (int k = 0; k < wl.num; ++k) {
      const WSec& w = wl.sec[k];
      int x = sbs.find(w.sys_num_up, w.sys_num_down), y = ebs.find(w.env_num_up, w.env_num_down);
      if (x < 0 || y < 0) throw Error(-2, "psi sector without basis sector");
      if (sbs.sec[x].dim != w.sys_dim || ebs.sec[y].dim != w.env_dim) throw Error(-1, "psi sector dims mismatch");
      xs.push_back(x);
      ye.push_back(y);
      std::vector<std::vector<int>> ga;
      for (const auto& pa : sbs.sec[x].pcs) {
        std::vector<int> gb;
        for (const auto& pb : ebs.sec[y].pcs)
          gb.push_back(S.p2.add_group(nullptr, BASE_OUT, w.off + pa.spos + (long long)pb.spos * w.sys_dim, w.sys_dim,
                                      pa.sdim, pb.sdim, 0));
        ga.push_back(gb);
      }
      grp.push_back(ga);
    }
  }

  long long in_off(int i, int r, int c) const { return wl.sec[i].off + r + (long long)c * wl.sec[i].sys_dim; }
  int pidx_sys(int k, int spos) const {
    const auto& p = sbs.sec[xs[k]].pcs;
    for (size_t a = 0; a < p.size(); ++a)
      if (p[a].spos == spos) return (int)a;
    throw Error(-1, "piece not found");
  }
  int pidx_env(int k, int spos) const {
    const auto& p = ebs.sec[ye[k]].pcs;
    for (size_t a = 0; a < p.size(); ++a)
      if (p[a].spos == spos) return (int)a;
    throw Error(-1, "piece not found");
  }
  GTerm base_term(cplx a) {
    GTerm t{};
    t.ar = a.real();
    t.ai = a.imag();
    return t;
  }
  void opnd(const OpRef& A, int k, uint8_t op, long long& off, int& ld, uint8_t& eop) {
    off = (long long)((uintptr_t)A.b->ptr(k) / sizeof(double2));
    ld = A.b->sub[k].row_dim;
    eop = A.ct ? flip(op) : op;
  }
  // C(group) += a * op(A_k) * in_i[r.., c..]
  void tLX(int g, cplx a, const OpRef& A, int k, uint8_t op, int K, int i, int r, int c) {
    GTerm t = base_term(a);
    t.kind = TK_GEMM;
    t.l_base = BASE_ABS;
    opnd(A, k, op, t.l_off, t.l_ld, t.l_op);
    t.r_base = BASE_IN;
    t.r_off = in_off(i, r, c);
    t.r_ld = wl.sec[i].sys_dim;
    t.r_op = OP_N;
    t.K = K;
    S.p2.gterms[g].push_back(t);
  }
  // C(group) += a * in_i[r.., c..] * op(B_k)
  void tXR(int g, cplx a, int i, int r, int c, int K, const OpRef& B, int k, uint8_t op) {
    GTerm t = base_term(a);
    t.kind = TK_GEMM;
    t.l_base = BASE_IN;
    t.l_off = in_off(i, r, c);
    t.l_ld = wl.sec[i].sys_dim;
    t.l_op = OP_N;
    t.r_base = BASE_ABS;
    opnd(B, k, op, t.r_off, t.r_ld, t.r_op);
    t.K = K;
    S.p2.gterms[g].push_back(t);
  }
  // C(group) += a * T(scratch) * op(B_k)
  void tTR(int g, cplx a, long long toff, int tld, int K, const OpRef& B, int k, uint8_t op) {
    GTerm t = base_term(a);
    t.kind = TK_GEMM;
    t.l_base = BASE_SCR;
    t.l_off = toff;
    t.l_ld = tld;
    t.l_op = OP_N;
    t.r_base = BASE_ABS;
    opnd(B, k, op, t.r_off, t.r_ld, t.r_op);
    t.K = K;
    S.p2.gterms[g].push_back(t);
  }
  // C(group) += a * in_i[r.., c..]  (rect = whole group)
  void tAX(int g, cplx a, int i, int r, int c) {
    GTerm t = base_term(a);
    t.kind = TK_AXPY;
    t.r_base = BASE_IN;
    t.r_off = in_off(i, r, c);
    t.r_ld = wl.sec[i].sys_dim;
    t.r_op = OP_N;
    t.r0 = 0;
    t.c0 = 0;
    t.rm = S.p2.groups[g].M;
    t.rn = S.p2.groups[g].N;
    S.p2.gterms[g].push_back(t);
  }
  // phase-1 intermediate T = op(A_k) [M x K] * in_i[r.., c..] [K x N]; returns scratch offset
  long long tmid(const OpRef& A, int k, uint8_t op, int M, int K, int i, int r, int c, int N) {
    long long aoff;
    int ald;
    uint8_t aop;
    opnd(A, k, op, aoff, ald, aop);
    auto key = std::make_tuple(aoff, (int)aop, i, r, c, M, N);
    auto it = inter.find(key);
    if (it != inter.end()) return it->second;
    long long off = scr;
    scr += (long long)M * N;
    int gi = S.p1.add_group(nullptr, BASE_SCR, off, M, M, N, 0);
    GTerm t{};
    t.ar = 1.0;
    t.kind = TK_GEMM;
    t.l_base = BASE_ABS;
    t.l_off = aoff;
    t.l_ld = ald;
    t.l_op = aop;
    t.r_base = BASE_IN;
    t.r_off = in_off(i, r, c);
    t.r_ld = wl.sec[i].sys_dim;
    t.r_op = OP_N;
    t.K = K;
    S.p1.gterms[gi].push_back(t);
    inter[key] = off;
    return off;
  }

  // ----------------------------------------------------------------------- diagonal kernels
  // block_vec_dia, get_sys.f90:1783-1832
  void block_vec_dia(const OpRef& H, cplx coef) {
    for (int i = 0; i < wl.num; ++i) {
      const auto& pcs = sbs.sec[xs[i]].pcs;
      for (size_t a = 0; a < pcs.size(); ++a) {
        const Piece& p = pcs[a];
        cplx c1 = coef / std::sqrt(1.0 + p.bl_num_down);
        int k = H.find2(p.bl_num_up, p.bl_num_down);
        if (k < 0) continue;
        const auto& epcs = ebs.sec[ye[i]].pcs;
        for (size_t b = 0; b < epcs.size(); ++b) tLX(grp[i][a][b], c1, H, k, OP_N, p.sdim, i, p.spos, epcs[b].spos);
        ref_flops += 8.0 * p.sdim * wl.sec[i].env_dim * p.sdim;
      }
    }
  }
  // vec_block_dia, get_sys.f90:1836-1885
  void vec_block_dia(const OpRef& H, cplx coef) {
    for (int i = 0; i < wl.num; ++i) {
      const auto& pcs = ebs.sec[ye[i]].pcs;
      for (size_t b = 0; b < pcs.size(); ++b) {
        const Piece& p = pcs[b];
        cplx c1 = coef / std::sqrt(1.0 + p.bl_num_down);
        int k = H.find2(p.bl_num_up, p.bl_num_down);
        if (k < 0) continue;
        const auto& spcs = sbs.sec[xs[i]].pcs;
        for (size_t a = 0; a < spcs.size(); ++a) tXR(grp[i][a][b], c1, i, spcs[a].spos, p.spos, p.sdim, H, k, OP_C);
        ref_flops += 8.0 * wl.sec[i].sys_dim * p.sdim * p.sdim;
      }
    }
  }
  // block_site_vec_dia, get_sys.f90:2006-2077
  void block_site_vec_dia(const OpRef& B, const SiteRef& st, cplx coef) {
    for (int i = 0; i < wl.num; ++i) {
      const auto& pcs = sbs.sec[xs[i]].pcs;
      for (size_t a = 0; a < pcs.size(); ++a) {
        const Piece& p = pcs[a];
        int bl = B.find2(p.bl_num_up, p.bl_num_down), s = st.find2(p.st_num_up, p.st_num_down);
        if (bl < 0 || s < 0) continue;
        cplx c = coef * st.sub[s].val;
        c = c / std::sqrt((1.0 + p.bl_num_down) * (1.0 + p.st_num_down));
        const auto& epcs = ebs.sec[ye[i]].pcs;
        for (size_t b = 0; b < epcs.size(); ++b) tLX(grp[i][a][b], c, B, bl, OP_N, p.sdim, i, p.spos, epcs[b].spos);
        ref_flops += 8.0 * p.sdim * wl.sec[i].env_dim * p.sdim;
      }
    }
  }
  // vec_block_site_dia, get_sys.f90:2081-2154
  void vec_block_site_dia(const OpRef& B, const SiteRef& st, cplx coef) {
    for (int i = 0; i < wl.num; ++i) {
      const auto& pcs = ebs.sec[ye[i]].pcs;
      for (size_t b = 0; b < pcs.size(); ++b) {
        const Piece& p = pcs[b];
        int bl = B.find2(p.bl_num_up, p.bl_num_down), s = st.find2(p.st_num_up, p.st_num_down);
        if (bl < 0 || s < 0) continue;
        cplx c = coef * st.sub[s].val;
        c = c / std::sqrt((1.0 + p.bl_num_down) * (1.0 + p.st_num_down));
        const auto& spcs = sbs.sec[xs[i]].pcs;
        for (size_t a = 0; a < spcs.size(); ++a) tXR(grp[i][a][b], c, i, spcs[a].spos, p.spos, p.sdim, B, bl, OP_C);
        ref_flops += 8.0 * wl.sec[i].sys_dim * p.sdim * p.sdim;
      }
    }
  }
  // site_vec_site_dia, get_sys.f90:2158-2254
  void site_vec_site_dia(const SiteRef& ss, const SiteRef& es, cplx coef) {
    for (int i = 0; i < wl.num; ++i) {
      const auto& sp = sbs.sec[xs[i]].pcs;
      const auto& ep = ebs.sec[ye[i]].pcs;
      for (size_t a = 0; a < sp.size(); ++a) {
        int s1 = ss.find2(sp[a].st_num_up, sp[a].st_num_down);
        for (size_t b = 0; b < ep.size(); ++b) {
          int s2 = es.find2(ep[b].st_num_up, ep[b].st_num_down);
          if (s1 < 0 || s2 < 0) continue;
          cplx c = coef * ss.sub[s1].val * es.sub[s2].val;
          c = c / std::sqrt((1.0 + sp[a].st_num_down) * (1.0 + ep[b].st_num_down));
          tAX(grp[i][a][b], c, i, sp[a].spos, ep[b].spos);
          ref_flops += 8.0 * sp[a].sdim * ep[b].sdim;
        }
      }
    }
  }
  // block_vec_site_dia, get_sys.f90:2258-2357
  void block_vec_site_dia(const OpRef& B, const SiteRef& es, cplx coef) {
    for (int i = 0; i < wl.num; ++i) {
      const auto& sp = sbs.sec[xs[i]].pcs;
      const auto& ep = ebs.sec[ye[i]].pcs;
      for (size_t a = 0; a < sp.size(); ++a) {
        int bl = B.find2(sp[a].bl_num_up, sp[a].bl_num_down);
        for (size_t b = 0; b < ep.size(); ++b) {
          int s2 = es.find2(ep[b].st_num_up, ep[b].st_num_down);
          if (bl < 0 || s2 < 0) continue;
          cplx c = coef * es.sub[s2].val;
          c = c / std::sqrt((1.0 + ep[b].st_num_down) * (1.0 + sp[a].bl_num_down));
          tLX(grp[i][a][b], c, B, bl, OP_N, sp[a].sdim, i, sp[a].spos, ep[b].spos);
          ref_flops += 8.0 * sp[a].sdim * ep[b].sdim * sp[a].sdim;
        }
      }
    }
  }
  // site_vec_block_dia, get_sys.f90:2361-2460
  void site_vec_block_dia(const SiteRef& ss, const OpRef& B, cplx coef) {
    for (int i = 0; i < wl.num; ++i) {
      const auto& sp = sbs.sec[xs[i]].pcs;
      const auto& ep = ebs.sec[ye[i]].pcs;
      for (size_t a = 0; a < sp.size(); ++a) {
        int s1 = ss.find2(sp[a].st_num_up, sp[a].st_num_down);
        for (size_t b = 0; b < ep.size(); ++b) {
          int eb = B.find2(ep[b].bl_num_up, ep[b].bl_num_down);
          if (s1 < 0 || eb < 0) continue;
          cplx c = coef * ss.sub[s1].val;
          c = c / std::sqrt((1.0 + ep[b].bl_num_down) * (1.0 + sp[a].st_num_down));
          tXR(grp[i][a][b], c, i, sp[a].spos, ep[b].spos, ep[b].sdim, B, eb, OP_C);
          ref_flops += 8.0 * sp[a].sdim * ep[b].sdim * ep[b].sdim;
        }
      }
    }
  }
  // block_vec_block_dia, get_sys.f90:2464-2569
  void block_vec_block_dia(const OpRef& SB, const OpRef& EB, cplx coef) {
    for (int i = 0; i < wl.num; ++i) {
      const auto& sp = sbs.sec[xs[i]].pcs;
      const auto& ep = ebs.sec[ye[i]].pcs;
      for (size_t a = 0; a < sp.size(); ++a) {
        int sb = SB.find2(sp[a].bl_num_up, sp[a].bl_num_down);
        for (size_t b = 0; b < ep.size(); ++b) {
          int eb = EB.find2(ep[b].bl_num_up, ep[b].bl_num_down);
          if (sb < 0 || eb < 0) continue;
          if (sp[a].sdim * ep[b].sdim == 0) throw Error(-1, "dimen wrong");
          cplx c1 = coef / std::sqrt((1.0 + ep[b].bl_num_down) * (1.0 + sp[a].bl_num_down));
          long long T = tmid(SB, sb, OP_N, sp[a].sdim, sp[a].sdim, i, sp[a].spos, ep[b].spos, ep[b].sdim);
          tTR(grp[i][a][b], c1, T, sp[a].sdim, ep[b].sdim, EB, eb, OP_C);
          ref_flops += 8.0 * sp[a].sdim * ep[b].sdim * sp[a].sdim + 8.0 * sp[a].sdim * ep[b].sdim * ep[b].sdim;
        }
      }
    }
  }

  // -------------------------------------------------------------------- non-diagonal kernels
  // block_site_vec_ndia, get_sys.f90:2578-2742
  void block_site_vec_ndia(const OpRef& B, const SiteRef& st, char FlagST, cplx coef) {
    int up_dif = B.up_dif(), K = B.K();
    if (up_dif != st.up_dif || K != st.down_dif) throw Error(-2, "Quantum number error in block_site_vec");
    for (int i = 0; i < wl.num; ++i) {
      int S = wl.sec[i].sys_num_down;
      const auto& pcs = sbs.sec[xs[i]].pcs;
      const auto& epcs = ebs.sec[ye[i]].pcs;
      for (size_t a = 0; a < pcs.size(); ++a) {
        const Piece& p = pcs[a];
        for (int dd = -K; dd <= K; dd += 2)
          for (int sdd = -K; sdd <= K; sdd += 2) {
            int bl = B.find3(p.bl_num_up, p.bl_num_down, dd);
            int nsu = p.st_num_up - up_dif, nsd = p.st_num_down - sdd;
            int s = st.find3(nsu, nsd, sdd);
            int nbu = p.bl_num_up + up_dif, nbd = p.bl_num_down + dd;
            if (bl < 0 || s < 0) continue;
            int an = -1;
            for (size_t q = 0; q < pcs.size(); ++q)
              if (pcs[q].bl_num_up == nbu && pcs[q].bl_num_down == nbd && pcs[q].st_num_up == nsu &&
                  pcs[q].st_num_down == nsd) {
                an = (int)q;
                break;
              }
            if (an < 0) continue;
            double sgnst = FlagST == 'F' ? sgn(p.bl_num_up) : 1.0;
            int j1 = nbd, j2 = p.bl_num_down, j3 = K, j4 = p.st_num_down, j5 = nsd, j6 = S;
            double c1 = w6j(j1, j2, j3, j4, j5, j6);
            if (c1 == 0.0) continue;
            c1 = c1 * pm1((j2 + j5 + j3 + j6) / 2) / std::sqrt(1.0 + K);
            cplx ct = (sgnst * c1) * coef * st.sub[s].val;
            int nd = pcs[an].sdim, od = p.sdim;
            for (size_t b = 0; b < epcs.size(); ++b) tLX(grp[i][an][b], ct, B, bl, OP_N, od, i, p.spos, epcs[b].spos);
            ref_flops += 8.0 * nd * wl.sec[i].env_dim * od;
            if (up_dif != 0) {
              cplx cc = std::conj(ct);
              for (size_t b = 0; b < epcs.size(); ++b)
                tLX(grp[i][a][b], cc, B, bl, OP_C, nd, i, pcs[an].spos, epcs[b].spos);
              ref_flops += 8.0 * od * wl.sec[i].env_dim * nd;
            }
          }
      }
    }
  }
  // vec_block_site_ndia, get_sys.f90:2842-3023
  void vec_block_site_ndia(const OpRef& B, char FlagBL, const SiteRef& st, char FlagST, cplx coef) {
    int up_dif = B.up_dif(), K = B.K();
    if (up_dif != st.up_dif || K != st.down_dif) throw Error(-2, "Quantum number error in vec_block_site");
    for (int i = 0; i < wl.num; ++i) {
      int Nsys = wl.sec[i].sys_num_up, Se = wl.sec[i].env_num_down;
      const auto& pcs = ebs.sec[ye[i]].pcs;
      const auto& spcs = sbs.sec[xs[i]].pcs;
      for (size_t b = 0; b < pcs.size(); ++b) {
        const Piece& p = pcs[b];
        for (int bdd = -K; bdd <= K; bdd += 2) {
          int bl = B.find3(p.bl_num_up, p.bl_num_down, bdd);
          for (int sdd = -K; sdd <= K; sdd += 2) {
            int nsu = p.st_num_up - up_dif, nsd = p.st_num_down - sdd;
            int s = st.find3(nsu, nsd, sdd);
            int nbu = p.bl_num_up + up_dif, nbd = p.bl_num_down + bdd;
            if (s < 0 || bl < 0) continue;
            int bn = -1;
            for (size_t q = 0; q < pcs.size(); ++q)
              if (pcs[q].bl_num_up == nbu && pcs[q].bl_num_down == nbd && pcs[q].st_num_up == nsu &&
                  pcs[q].st_num_down == nsd) {
                bn = (int)q;
                break;
              }
            if (bn < 0) continue;
            double s_bl = FlagBL == 'F' ? sgn(Nsys + nsu) : 1.0;
            double s_st = FlagST == 'F' ? sgn(Nsys) : 1.0;
            int j1 = nbd, j2 = p.bl_num_down, j3 = K, j4 = p.st_num_down, j5 = nsd, j6 = Se;
            double c1 = w6j(j1, j2, j3, j4, j5, j6);
            if (c1 == 0.0) continue;
            c1 = c1 * pm1((j2 + j5 + j3 + j6) / 2) / std::sqrt(1.0 + K);
            cplx ct = (s_bl * s_st * c1) * coef * st.sub[s].val;
            int nd = pcs[bn].sdim, od = p.sdim;
            for (size_t a = 0; a < spcs.size(); ++a) tXR(grp[i][a][bn], ct, i, spcs[a].spos, p.spos, od, B, bl, OP_C);
            ref_flops += 8.0 * wl.sec[i].sys_dim * nd * od;
            if (up_dif != 0) {
              cplx cc = std::conj(ct);
              for (size_t a = 0; a < spcs.size(); ++a)
                tXR(grp[i][a][b], cc, i, spcs[a].spos, pcs[bn].spos, nd, B, bl, OP_N);
              ref_flops += 8.0 * wl.sec[i].sys_dim * od * nd;
            }
          }
        }
      }
    }
  }
  // block_vec_block_ndia, get_sys.f90:3131-3420
  void block_vec_block_ndia(const OpRef& SB, const OpRef& EB, char FlagEL, cplx coef) {
    int up_dif = SB.up_dif(), K = SB.K();
    if (up_dif != EB.up_dif() || K != EB.K()) throw Error(-2, "Quantum number error in block_vec_block");
    for (int i = 0; i < wl.num; ++i) {
      const WSec& wi = wl.sec[i];
      const auto& sp = sbs.sec[xs[i]].pcs;
      const auto& ep = ebs.sec[ye[i]].pcs;
      for (size_t a = 0; a < sp.size(); ++a)
        for (size_t b = 0; b < ep.size(); ++b) {
          const Piece &ps = sp[a], &pe = ep[b];
          for (int dd = -K; dd <= K; dd += 2) {
            int sb = SB.find3(ps.bl_num_up, ps.bl_num_down, dd);
            int nsbu = ps.bl_num_up + up_dif, nsbd = ps.bl_num_down + dd;
            for (int edd = -K; edd <= K; edd += 2) {
              int nebu = pe.bl_num_up - up_dif, nebd = pe.bl_num_down - edd;
              int eb = EB.find3(nebu, nebd, edd);
              if (sb < 0 || eb < 0) continue;
              for (int nS = std::abs(wi.sys_num_down - K); nS <= wi.sys_num_down + K; nS += 2) {
                int nsu = wi.sys_num_up + up_dif, neu = wi.env_num_up - up_dif;
                int ks = sbs.find(nsu, nS), ke = ebs.find(neu, nS);
                int qa = -1, qb = -1;
                if (ks >= 0)
                  for (size_t q = 0; q < sbs.sec[ks].pcs.size(); ++q) {
                    const Piece& x = sbs.sec[ks].pcs[q];
                    if (x.bl_num_up == nsbu && x.bl_num_down == nsbd && x.st_num_down == ps.st_num_down &&
                        x.st_num_up == ps.st_num_up) {
                      qa = (int)q;
                      break;
                    }
                  }
                if (ke >= 0)
                  for (size_t q = 0; q < ebs.sec[ke].pcs.size(); ++q) {
                    const Piece& x = ebs.sec[ke].pcs[q];
                    if (x.bl_num_up == nebu && x.bl_num_down == nebd && x.st_num_down == pe.st_num_down &&
                        x.st_num_up == pe.st_num_up) {
                      qb = (int)q;
                      break;
                    }
                  }
                if (qa < 0 || qb < 0) continue;
                int kk = wl.find(nsu, nS, neu, nS);
                if (kk < 0) continue;
                double sEL = FlagEL == 'F' ? sgn(wi.sys_num_up + pe.st_num_up) : 1.0;
                double c1 = w6j(nS, K, wi.sys_num_down, ps.bl_num_down, ps.st_num_down, nsbd);
                if (c1 == 0.0) continue;
                double c11 = w6j(nS, K, wi.env_num_down, pe.bl_num_down, pe.st_num_down, nebd);
                if (c11 == 0.0) continue;
                c1 = c1 * c11;
                c1 = c1 * std::sqrt((1.0 + nS) * (1.0 + wi.env_num_down) / (1.0 + K));
                if ((((nsbd + ps.st_num_down + wi.sys_num_down + K) / 2 +
                      (nebd + pe.st_num_down + wi.env_num_down + K) / 2) % 2) == 1)
                  c1 = -c1;
                cplx ct = sEL * coef * c1;
                const Piece& ns_ = sbs.sec[ks].pcs[qa];
                const Piece& ne_ = ebs.sec[ke].pcs[qb];
                int nsd = ns_.sdim, osd = ps.sdim, oed = pe.sdim, ned = ne_.sdim;
                long long T = tmid(SB, sb, OP_N, nsd, osd, i, ps.spos, pe.spos, oed);
                tTR(grp[kk][qa][qb], ct, T, nsd, oed, EB, eb, OP_N);
                ref_flops += 8.0 * nsd * oed * osd + 8.0 * nsd * ned * oed;
                if (up_dif != 0) {
                  cplx cc = std::conj(ct);
                  long long T2 = tmid(SB, sb, OP_C, osd, nsd, kk, ns_.spos, ne_.spos, ned);
                  tTR(grp[i][a][b], cc, T2, osd, ned, EB, eb, OP_C);
                  ref_flops += 8.0 * osd * ned * nsd + 8.0 * osd * oed * ned;
                }
              }
            }
          }
        }
    }
  }
  // block_vec_site_ndia, get_sys.f90:3970-4206
  void block_vec_site_ndia(const OpRef& SB, const SiteRef& es, char FlagET, cplx coef) {
    int up_dif = SB.up_dif(), K = SB.K();
    if (up_dif != es.up_dif || K != es.down_dif) throw Error(-2, "Quantum number error in block_vec_site");
    for (int i = 0; i < wl.num; ++i) {
      const WSec& wi = wl.sec[i];
      const auto& sp = sbs.sec[xs[i]].pcs;
      const auto& ep = ebs.sec[ye[i]].pcs;
      for (size_t a = 0; a < sp.size(); ++a)
        for (size_t b = 0; b < ep.size(); ++b) {
          const Piece &ps = sp[a], &pe = ep[b];
          for (int bdd = -K; bdd <= K; bdd += 2) {
            int nsbu = ps.bl_num_up + up_dif, nsbd = ps.bl_num_down + bdd;
            int sb = SB.find3(ps.bl_num_up, ps.bl_num_down, bdd);
            for (int sdd = -es.down_dif; sdd <= es.down_dif; sdd += 2) {
              int nesu = pe.st_num_up - up_dif, nesd = pe.st_num_down - sdd;
              int s = es.find3(nesu, nesd, sdd);
              int nsu = wi.sys_num_up + up_dif, neu = wi.env_num_up - up_dif;
              if (sb < 0 || s < 0) continue;
              for (int nS = std::abs(wi.sys_num_down - K); nS <= wi.sys_num_down + K; nS += 2) {
                int ks = sbs.find(nsu, nS), ke = ebs.find(neu, nS);
                int qa = -1, qb = -1;
                if (ks >= 0)
                  for (size_t q = 0; q < sbs.sec[ks].pcs.size(); ++q) {
                    const Piece& x = sbs.sec[ks].pcs[q];
                    if (x.bl_num_up == nsbu && x.bl_num_down == nsbd && x.st_num_down == ps.st_num_down) {
                      qa = (int)q;
                      break;
                    }
                  }
                if (ke >= 0)
                  for (size_t q = 0; q < ebs.sec[ke].pcs.size(); ++q) {
                    const Piece& x = ebs.sec[ke].pcs[q];
                    if (x.st_num_up == nesu && x.st_num_down == nesd && x.bl_num_down == pe.bl_num_down) {
                      qb = (int)q;
                      break;
                    }
                  }
                if (qa < 0 || qb < 0) continue;
                int kk = wl.find(nsu, nS, neu, nS);
                if (kk < 0) continue;
                double sET = FlagET == 'F' ? sgn(wi.sys_num_up) : 1.0;
                double c1 = w6j(nS, K, wi.sys_num_down, ps.bl_num_down, ps.st_num_down, nsbd);
                if (c1 == 0.0) continue;
                double c11 = w6j(nS, K, wi.env_num_down, pe.st_num_down, pe.bl_num_down, nesd);
                if (c11 == 0.0) continue;
                c1 = c1 * c11;
                c1 = c1 * std::sqrt((1.0 + nS) * (1.0 + wi.env_num_down) / (1.0 + K));
                if ((((nsbd + ps.st_num_down + wi.sys_num_down + K) / 2 + (pe.bl_num_down + pe.st_num_down + nS + K) / 2) %
                     2) != 0)
                  c1 = -c1;
                cplx ct = (sET * c1) * coef * es.sub[s].val;
                const Piece& ns_ = sbs.sec[ks].pcs[qa];
                const Piece& ne_ = ebs.sec[ke].pcs[qb];
                tLX(grp[kk][qa][qb], ct, SB, sb, OP_N, ps.sdim, i, ps.spos, pe.spos);
                ref_flops += 8.0 * ns_.sdim * pe.sdim * ps.sdim;
                if (up_dif != 0) {
                  cplx cc = std::conj(ct);
                  tLX(grp[i][a][b], cc, SB, sb, OP_C, ns_.sdim, kk, ns_.spos, ne_.spos);
                  ref_flops += 8.0 * ps.sdim * pe.sdim * ns_.sdim;
                }
              }
            }
          }
        }
    }
  }
  // site_vec_block_ndia, get_sys.f90:4349-4637
  void site_vec_block_ndia(const SiteRef& ss, char FlagST, const OpRef& EB, char FlagEL, cplx coef) {
    int up_dif = ss.up_dif, K = ss.down_dif;
    if (up_dif != EB.up_dif() || K != EB.K()) throw Error(-2, "Quantum number error in site_vec_block");
    for (int i = 0; i < wl.num; ++i) {
      const WSec& wi = wl.sec[i];
      const auto& sp = sbs.sec[xs[i]].pcs;
      const auto& ep = ebs.sec[ye[i]].pcs;
      for (size_t a = 0; a < sp.size(); ++a)
        for (size_t b = 0; b < ep.size(); ++b) {
          const Piece &ps = sp[a], &pe = ep[b];
          for (int sdd = -ss.down_dif; sdd <= ss.down_dif; sdd += 2) {
            int nssu = ps.st_num_up + up_dif, nssd = ps.st_num_down + sdd;
            int s = ss.find3(ps.st_num_up, ps.st_num_down, sdd);
            for (int bdd = -EB.K(); bdd <= EB.K(); bdd += 2) {
              int nebu = pe.bl_num_up - up_dif, nebd = pe.bl_num_down - bdd;
              int eb = EB.find3(nebu, nebd, bdd);
              int nsu = wi.sys_num_up + up_dif, neu = wi.env_num_up - up_dif;
              if (s < 0 || eb < 0) continue;
              for (int nS = std::abs(wi.sys_num_down - ss.down_dif); nS <= wi.sys_num_down + ss.down_dif; nS += 2) {
                int ks = sbs.find(nsu, nS), ke = ebs.find(neu, nS);
                int qa = -1, qb = -1;
                if (ks >= 0)
                  for (size_t q = 0; q < sbs.sec[ks].pcs.size(); ++q) {
                    const Piece& x = sbs.sec[ks].pcs[q];
                    if (x.st_num_up == nssu && x.st_num_down == nssd && x.bl_num_down == ps.bl_num_down &&
                        x.bl_num_up == ps.bl_num_up) {
                      qa = (int)q;
                      break;
                    }
                  }
                if (ke >= 0)
                  for (size_t q = 0; q < ebs.sec[ke].pcs.size(); ++q) {
                    const Piece& x = ebs.sec[ke].pcs[q];
                    if (x.bl_num_up == nebu && x.bl_num_down == nebd && x.st_num_up == pe.st_num_up &&
                        x.st_num_down == pe.st_num_down) {
                      qb = (int)q;
                      break;
                    }
                  }
                if (qa < 0 || qb < 0) continue;
                int kk = wl.find(nsu, nS, neu, nS);
                if (kk < 0) continue;
                double c1 = w6j(nS, K, wi.sys_num_down, ps.st_num_down, ps.bl_num_down, nssd);
                if (c1 == 0.0) continue;
                double c11 = w6j(nS, K, wi.env_num_down, pe.bl_num_down, pe.st_num_down, nebd);
                if (c11 == 0.0) continue;
                c1 = c1 * c11;
                c1 = c1 * std::sqrt((1.0 + nS) * (wi.env_num_down + 1.0) / (1.0 + K));
                if ((((nebd + pe.st_num_down + wi.env_num_down + K) / 2 + (ps.bl_num_down + ps.st_num_down + nS + K) / 2) %
                     2) != 0)
                  c1 = -c1;
                double sST = FlagST == 'F' ? sgn(ps.bl_num_up) : 1.0;
                double sEL = FlagEL == 'F' ? sgn(wi.sys_num_up + pe.st_num_up) : 1.0;
                cplx ct = (sST * sEL * c1) * coef * ss.sub[s].val;
                const Piece& ns_ = sbs.sec[ks].pcs[qa];
                const Piece& ne_ = ebs.sec[ke].pcs[qb];
                tXR(grp[kk][qa][qb], ct, i, ps.spos, pe.spos, pe.sdim, EB, eb, OP_N);
                ref_flops += 8.0 * ps.sdim * ne_.sdim * pe.sdim;
                if (up_dif != 0) {
                  cplx cc = std::conj(ct);
                  tXR(grp[i][a][b], cc, kk, ns_.spos, ne_.spos, ne_.sdim, EB, eb, OP_C);
                  ref_flops += 8.0 * ps.sdim * pe.sdim * ne_.sdim;
                }
              }
            }
          }
        }
    }
  }
  // site_vec_site_ndia, get_sys.f90:4816-5073
  void site_vec_site_ndia(const SiteRef& ss, char FlagST, const SiteRef& es, char FlagET, cplx coef) {
    int up_dif = ss.up_dif, K = ss.down_dif;
    if (up_dif != es.up_dif || K != es.down_dif) throw Error(-2, "Quantum number error in site_vec_site");
    for (int i = 0; i < wl.num; ++i) {
      const WSec& wi = wl.sec[i];
      const auto& sp = sbs.sec[xs[i]].pcs;
      const auto& ep = ebs.sec[ye[i]].pcs;
      for (size_t a = 0; a < sp.size(); ++a)
        for (size_t b = 0; b < ep.size(); ++b) {
          const Piece &ps = sp[a], &pe = ep[b];
          for (int d1 = -ss.down_dif; d1 <= ss.down_dif; d1 += 2) {
            int s1 = ss.find3(ps.st_num_up, ps.st_num_down, d1);
            int nssu = ps.st_num_up + up_dif, nssd = ps.st_num_down + d1;
            for (int d2 = -es.down_dif; d2 <= es.down_dif; d2 += 2) {
              int nesu = pe.st_num_up - up_dif, nesd = pe.st_num_down - d2;
              int s2 = es.find3(nesu, nesd, d2);
              int nsu = wi.sys_num_up + up_dif, neu = wi.env_num_up - up_dif;
              if (s1 < 0 || s2 < 0) continue;
              for (int nS = std::abs(wi.sys_num_down - ss.down_dif); nS <= wi.sys_num_down + ss.down_dif; nS += 2) {
                int ks = sbs.find(nsu, nS), ke = ebs.find(neu, nS);
                int qa = -1, qb = -1;
                if (ks >= 0)
                  for (size_t q = 0; q < sbs.sec[ks].pcs.size(); ++q) {
                    const Piece& x = sbs.sec[ks].pcs[q];
                    if (x.st_num_up == nssu && x.st_num_down == nssd && x.bl_num_down == ps.bl_num_down) {
                      qa = (int)q;
                      break;
                    }
                  }
                if (ke >= 0)
                  for (size_t q = 0; q < ebs.sec[ke].pcs.size(); ++q) {
                    const Piece& x = ebs.sec[ke].pcs[q];
                    if (x.st_num_up == nesu && x.st_num_down == nesd && x.bl_num_down == pe.bl_num_down) {
                      qb = (int)q;
                      break;
                    }
                  }
                if (qa < 0 || qb < 0) continue;
                int kk = wl.find(nsu, nS, neu, nS);
                if (kk < 0) continue;
                double sST = FlagST == 'F' ? sgn(ps.bl_num_up) : 1.0;
                double sET = FlagET == 'F' ? sgn(wi.sys_num_up) : 1.0;
                cplx ct = (sST * sET) * coef;
                double c1 = w6j(nS, K, wi.sys_num_down, ps.st_num_down, ps.bl_num_down, nssd);
                if (c1 == 0.0) continue;
                double c11 = w6j(nS, K, wi.env_num_down, pe.st_num_down, pe.bl_num_down, nesd);
                if (c11 == 0.0) continue;
                c1 = c1 * c11;
                c1 = c1 * std::sqrt((1.0 + nS) * (1.0 + wi.env_num_down) / (1.0 + K));
                if ((((pe.bl_num_down + pe.st_num_down + nS + K) / 2 + (ps.bl_num_down + ps.st_num_down + nS + K) / 2) %
                     2) != 0)
                  c1 = -c1;
                cplx cc = ct * c1 * ss.sub[s1].val * es.sub[s2].val;
                const Piece& ns_ = sbs.sec[ks].pcs[qa];
                const Piece& ne_ = ebs.sec[ke].pcs[qb];
                tAX(grp[kk][qa][qb], cc, i, ps.spos, pe.spos);
                ref_flops += 8.0 * ps.sdim * pe.sdim;
                if (up_dif != 0) {
                  tAX(grp[i][a][b], std::conj(cc), kk, ns_.spos, ne_.spos);
                  ref_flops += 8.0 * ps.sdim * pe.sdim;
                }
              }
            }
          }
        }
    }
  }
};

OpRef R(const DBlock& b) { return OpRef{&b, false}; }
OpRef RT(const DBlock& b) { return OpRef{&b, true}; }

}  // namespace

// hmerge (get_sys.f90:7398-7626): merged operators as device axpy tasks
void Engine::build_merge() {
  Superblock& S = sb;
  DModel& sys = S.sys;
  DModel& env = S.env;
  TaskList& tl = S.merge;
  tl = TaskList();
  int dmsite = sys.len + env.len + 2, syssite = sys.len + 1;
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b) L.coup_bs[a][b] = 0;
  for (int k = 1; k <= Lattice::neibt; ++k) {
    int j = L.NEIB(syssite, k);
    if (L.npos(j) == 3) L.coup_bs[1][0] = 1;
    if (L.npos(j) == 1) L.coup_bs[0][0] = 1;
    j = L.NEIB(L.nposi_lat[dmsite], k);
    if (L.npos(j) == 3) L.coup_bs[1][1] = 1;
    if (L.npos(j) == 1) L.coup_bs[0][1] = 1;
  }
  // a zeroed operator with the structure of src (block_pass_info, block.f90:132-159)
  auto zero_like = [&](const DBlock& src) {
    DBlock b = src;
    long long off = 0;
    for (auto& s : b.sub) {
      s.off = off;
      off += (long long)s.row_dim * s.sdim;
    }
    b.buf = std::make_shared<DevBuf>((size_t)off, st, true);
    return b;
  };
  // per merged operator: one group per sub-block, filled by axpy terms
  struct Acc {
    DBlock* dst;
    std::vector<int> gids;
  };
  std::vector<Acc> accs;
  auto open = [&](DBlock& dst, const DBlock& like) {
    dst = zero_like(like);
    Acc a{&dst, {}};
    for (int i = 0; i < dst.num; ++i)
      a.gids.push_back(tl.add_group(dst.ptr(i), BASE_ABS, 0, dst.sub[i].row_dim, dst.sub[i].row_dim, dst.sub[i].sdim, 0));
    accs.push_back(a);
    return (int)accs.size() - 1;
  };
  // block_add_block_two (block.f90:177-215)
  auto add = [&](int acc, const DBlock& src, double coef) {
    DBlock& nb = *accs[acc].dst;
    int x1 = 0;
    for (int i = 0; i < nb.num; ++i) {
      int idx = -1;
      for (int x = x1; x < src.num; ++x)
        if (src.sub[x].num_up == nb.sub[i].num_up && src.sub[x].num_down == nb.sub[i].num_down &&
            src.sub[x].down_dif == nb.sub[i].down_dif) {
          idx = x;
          x1 = x + 1;
          break;
        }
      if (idx < 0) continue;
      if (src.sub[idx].row_dim != nb.sub[i].row_dim || src.sub[idx].sdim != nb.sub[i].sdim)
        throw Error(-1, "hmerge: operator structure mismatch");
      GTerm t{};
      t.kind = TK_AXPY;
      t.ar = coef;
      t.r_base = BASE_ABS;
      t.r_off = (long long)((uintptr_t)src.ptr(idx) / sizeof(double2));
      t.r_ld = src.sub[idx].row_dim;
      t.r_op = OP_N;
      t.rm = nb.sub[i].row_dim;
      t.rn = nb.sub[i].sdim;
      tl.gterms[accs[acc].gids[i]].push_back(t);
    }
  };
  auto chk = [&](const DModel& m, int idx) {
    if (idx < 1 || idx >= (int)m.sub.size() || !m.sub[idx].op[0].buf) throw Error(-1, "hmerge: missing boundary operator");
  };
  int accS[2][4], accE[2][4];
  for (int ia = 0; ia < 2; ++ia)
    for (int o = 0; o < 4; ++o) accS[ia][o] = accE[ia][o] = -1;
  accs.reserve(4096);
  for (int ia = 0; ia < 2; ++ia) {
    if (L.coup_bs[0][ia] == 1) {
      chk(sys, 1);
      for (int o : {OP_UP, OP_SD, OP_SN}) accS[ia][o] = open(S.snc_sys[ia][o], sys.sub[1].op[o]);
    }
    if (L.coup_bs[1][ia] == 1) {
      chk(env, 1);
      for (int o : {OP_UP, OP_DOWN, OP_SD, OP_SN}) accE[ia][o] = open(S.snc_env[ia][o], env.sub[1].op[o]);
    }
  }
  for (int ia = 1; ia <= 2; ++ia) {
    int j = sys.len + 1 + (env.len + 1) * (ia - 1);
    int latt = L.nposi_lat[j];
    for (int k1 = 1; k1 <= Lattice::neibt; ++k1) {
      int ib = L.NEIB(latt, k1);
      double jd1 = L.JD(k1, latt), jt1 = L.JT(k1, latt), jn1 = L.JN(k1, latt);
      if (L.npos(ib) == 3 && L.coup_bs[1][ia - 1] != 0) {
        int ib1 = L.INB1(L.nposi_dm[ib] - sys.len - 1, env.len);
        chk(env, ib1);
        if (jt1 != 0.0) {
          add(accE[ia - 1][OP_UP], env.sub[ib1].op[OP_UP], jt1);
          add(accE[ia - 1][OP_DOWN], env.sub[ib1].op[OP_DOWN], jt1);
        }
        if (jd1 != 0.0) add(accE[ia - 1][OP_SD], env.sub[ib1].op[OP_SD], jd1);
        if (jn1 != 0.0) add(accE[ia - 1][OP_SN], env.sub[ib1].op[OP_SN], jn1);
      }
      if (L.npos(ib) == 1 && L.coup_bs[0][ia - 1] == 1) {
        int ib1 = L.INB1(L.nposi_dm[ib], sys.len);
        chk(sys, ib1);
        if (jt1 != 0.0) add(accS[ia - 1][OP_UP], sys.sub[ib1].op[OP_UP], jt1);
        if (jd1 != 0.0) add(accS[ia - 1][OP_SD], sys.sub[ib1].op[OP_SD], jd1);
        if (jn1 != 0.0) add(accS[ia - 1][OP_SN], sys.sub[ib1].op[OP_SN], jn1);
      }
    }
  }
  // block-block pivots (get_sys.f90:7498-7533)
  int k11 = 0;
  for (int I = 1; I <= sys.len; ++I) {
    int k1 = 0;
    for (int k = 1; k <= Lattice::neibt; ++k)
      if (L.npos(L.NEIB(I, k)) == 3) k1++;
    L.INB(I) = k1;
    if (L.nleg11[env.len] < L.nleg11[sys.len]) L.INB(I) = 0;
    if (L.INB(I) != 0) k11++;
  }
  L.coup_bb[0] = k11;
  L.INB(sys.len + 1) = 0;
  L.INB(sys.len + env.len + 2) = 0;
  for (int I = 1; I <= env.len; ++I) {
    int k1 = 0;
    L.INB(I + sys.len + 1) = 0;
    for (int k = 1; k <= Lattice::neibt; ++k) {
      int J = L.NEIB(L.nposi_lat[I + sys.len + 1], k);
      if (L.npos(J) == 1 && L.INB(J) == 0) k1++;
    }
    L.INB(I + sys.len + 1) = k1;
    if (k1 != 0) k11++;
  }
  L.coup_bb[1] = k11 - L.coup_bb[0];
  S.sub_s_env.assign(L.coup_bb[0] + 1, OpSet());
  S.sub_s_sys.assign(L.coup_bb[1] + 1, OpSet());
  std::vector<std::array<int, 4>> accSE(L.coup_bb[0] + 1), accSS(L.coup_bb[1] + 1);
  for (int i = 1; i <= L.coup_bb[0]; ++i) {
    chk(env, 1);
    for (int o = 0; o < 4; ++o) accSE[i][o] = open(S.sub_s_env[i].op[o], env.sub[1].op[o]);
  }
  for (int i = 1; i <= L.coup_bb[1]; ++i) {
    chk(sys, 1);
    accSS[i][OP_DOWN] = -1;
    for (int o : {OP_UP, OP_SD, OP_SN}) accSS[i][o] = open(S.sub_s_sys[i].op[o], sys.sub[1].op[o]);
  }
  int jc = 0;
  for (int I = 1; I <= sys.len + env.len + 1; ++I) {
    if (L.INB(I) == 0) continue;
    int Ia = L.nposi_lat[I];
    jc++;
    for (int k1 = 1; k1 <= Lattice::neibt; ++k1) {
      int Ib = L.NEIB(Ia, k1);
      double jt1 = L.JT(k1, Ia), jd1 = L.JD(k1, Ia), jn1 = L.JN(k1, Ia);
      if (L.npos(Ib) == 3 && I <= sys.len) {
        int Ib1 = L.INB1(L.nposi_dm[Ib] - sys.len - 1, env.len);
        chk(env, Ib1);
        if (jt1 != 0.0) {
          add(accSE[jc][OP_UP], env.sub[Ib1].op[OP_UP], jt1);
          add(accSE[jc][OP_DOWN], env.sub[Ib1].op[OP_DOWN], jt1);
        }
        if (jd1 != 0.0) add(accSE[jc][OP_SD], env.sub[Ib1].op[OP_SD], jd1);
        if (jn1 != 0.0) add(accSE[jc][OP_SN], env.sub[Ib1].op[OP_SN], jn1);
      }
      if (L.npos(Ib) == 1 && I > sys.len + 1 && L.INB(L.nposi_dm[Ib]) == 0) {
        int Ib1 = L.INB1(Ib, sys.len);
        int jc1 = jc - L.coup_bb[0];
        chk(sys, Ib1);
        if (jt1 != 0.0) add(accSS[jc1][OP_UP], sys.sub[Ib1].op[OP_UP], jt1);
        if (jd1 != 0.0) add(accSS[jc1][OP_SD], sys.sub[Ib1].op[OP_SD], jd1);
        if (jn1 != 0.0) add(accSS[jc1][OP_SN], sys.sub[Ib1].op[OP_SN], jn1);
      }
    }
  }
  tl.upload(st);
  run_tasks(tl, nullptr, nullptr, nullptr);
}

// model_wave term list (get_sys.f90:6915-7059, add_op=1, t-J, lring=0)
void Engine::build_hpsi_tasks() {
  Superblock& S = sb;
  Builder B(*this);
  const cplx cone(1.0, 0.0);
  DModel& sys = S.sys;
  DModel& env = S.env;
  B.block_vec_dia(R(sys.ham), cone);
  B.vec_block_dia(R(env.ham), cone);
  int is = L.nposi_lat[sys.len + 1], js = L.nposi_lat[sys.len + env.len + 2];
  int ii = L.NEIBA(is, js);
  if (ii != 0) {
    double jd1 = L.JD(ii, is), cx = L.JT(ii, is), jn1 = L.JN(ii, is);
    if (cx != 0.0) B.site_vec_site_ndia(site(st_elec_up), 'F', site_ct(st_elec_down), 'F', cx);
    if (jd1 != 0.0) B.site_vec_site_ndia(site(st_sd), 'B', site(st_sd), 'B', jd1);
    if (jn1 != 0.0) B.site_vec_site_dia(site(num_elec), site(num_elec), jn1);
  }
  if (L.coup_bs[0][0] == 1) {
    B.block_site_vec_ndia(R(S.snc_sys[0][OP_UP]), site_ct(st_elec_down), 'F', cone);
    B.block_site_vec_ndia(R(S.snc_sys[0][OP_SD]), site(st_sd), 'B', cone);
    B.block_site_vec_dia(R(S.snc_sys[0][OP_SN]), site(num_elec), cone);
  }
  if (L.coup_bs[0][1] == 1) {
    B.block_vec_site_ndia(R(S.snc_sys[1][OP_UP]), site_ct(st_elec_down), 'F', cone);
    B.block_vec_site_ndia(R(S.snc_sys[1][OP_SD]), site(st_sd), 'B', cone);
    B.block_vec_site_dia(R(S.snc_sys[1][OP_SN]), site(num_elec), cone);
  }
  if (L.coup_bs[1][0] == 1) {
    B.site_vec_block_ndia(site(st_elec_up), 'F', RT(S.snc_env[0][OP_DOWN]), 'F', cone);
    B.site_vec_block_ndia(site(st_sd), 'B', RT(S.snc_env[0][OP_SD]), 'B', cone);
    B.site_vec_block_dia(site(num_elec), R(S.snc_env[0][OP_SN]), cone);
  }
  if (L.coup_bs[1][1] == 1) {
    B.vec_block_site_ndia(R(S.snc_env[1][OP_UP]), 'F', site_ct(st_elec_down), 'F', cone);
    B.vec_block_site_ndia(R(S.snc_env[1][OP_SD]), 'B', site(st_sd), 'B', cone);
    B.vec_block_site_dia(R(S.snc_env[1][OP_SN]), site(num_elec), cone);
  }
  int jc = 0;
  for (int i = 1; i <= sys.len + 1 + env.len; ++i) {
    if (L.INB(i) == 0) continue;
    jc++;
    if (i <= sys.len) {
      int i1 = L.INB1(i, sys.len);
      if (i1 < 1 || i1 >= (int)sys.sub.size()) throw Error(-1, "missing sys boundary operator");
      B.block_vec_block_ndia(R(sys.sub[i1].op[OP_UP]), RT(S.sub_s_env[jc].op[OP_DOWN]), 'F', cone);
      B.block_vec_block_ndia(R(sys.sub[i1].op[OP_SD]), RT(S.sub_s_env[jc].op[OP_SD]), 'B', cone);
      B.block_vec_block_dia(R(sys.sub[i1].op[OP_SN]), R(S.sub_s_env[jc].op[OP_SN]), cone);
    } else {
      int i1 = L.INB1(i - sys.len - 1, env.len);
      int jc1 = jc - L.coup_bb[0];
      if (i1 < 1 || i1 >= (int)env.sub.size()) throw Error(-1, "missing env boundary operator");
      B.block_vec_block_ndia(R(S.sub_s_sys[jc1].op[OP_UP]), RT(env.sub[i1].op[OP_DOWN]), 'F', cone);
      B.block_vec_block_ndia(R(S.sub_s_sys[jc1].op[OP_SD]), RT(env.sub[i1].op[OP_SD]), 'B', cone);
      B.block_vec_block_dia(R(S.sub_s_sys[jc1].op[OP_SN]), R(env.sub[i1].op[OP_SN]), cone);
    }
  }
  S.ref_flops = B.ref_flops;
  S.scratch_elems = B.scr;
  if (split_now_) {
    S.p1s.groups = S.p1.groups;
    S.p1s.gterms = S.p1.gterms;
    S.p2s.groups = S.p2.groups;
    S.p2s.gterms = S.p2.gterms;
    // shared views (the default): one sliced copy per operator block, the terms'
    // coefficients applied by the kernel's epilogue; ~4.5x less memory than views
    // with the coefficients folded in (YC4x24 m=4000: 3.2 GB against 14.3 GB) and
    // as much less slicing when the superblock is set, for ~1-2 % more H.psi time
    // (segments break at every term).  Automatic choice (-1): shared once the
    // folded copies (~3.5x the operators' FP64 bytes) would pass 4 GiB.
    bool shared = split_shared_views_ > 0;
    if (split_shared_views_ < 0) {
      double op_bytes = 0.0;
      for (const DModel* m : {&S.sys, &S.env}) {
        op_bytes += 16.0 * (double)m->ham.total();
        for (const OpSet& o : m->sub)
          for (const DBlock& b : o.op)
            if (b.buf) op_bytes += 16.0 * (double)b.total();
      }
      shared = 3.5 * op_bytes > 4.0 * 1073741824.0;
    }
    build_split_views(S.p1s, S.p2s, S.sv, st, shared);
    S.p1s.upload_split(st);
    S.p2s.upload_split(st);
    S.p1s.gterms.clear();
    S.p2s.gterms.clear();
  }
  tune_setup();
  S.q1.gterms.clear();
  S.q2.gterms.clear();
  S.scratch = std::make_shared<DevBuf>((size_t)std::max<long long>(B.scr, 1), st, false);
}

void Engine::tune_setup() {
  Superblock& S = sb;
  const double gflop = S.ref_flops / 1e9;
  S.tune_class = (autotune_ && gflop >= 8.0) ? (int)std::floor(std::log2(gflop)) : -1;
  S.tune_cand = -1;
  S.tune_pending = false;
  if (S.tune_class < 0) {
    S.p1.upload(st);
    S.p2.upload(st);
    return;
  }
  auto it = tune_ms_.find(S.tune_class);
  if (it == tune_ms_.end()) {
    std::array<double, kTuneCands> none;
    none.fill(-1.0);
    it = tune_ms_.emplace(S.tune_class, none).first;
  }
  const auto& ms = it->second;
  int best = 0, next = -1;
  for (int c = 0; c < kTuneCands; ++c) {
    if (ms[c] < 0 && next < 0) next = c;
    if (ms[c] >= 0 && (ms[best] < 0 || ms[c] < ms[best])) best = c;
  }
  if (next < 0) {   // class tuned: its fastest schedule only
    S.p1.upload(st, 296, tune_cands_[best].waves, tune_cands_[best].tile);
    S.p2.upload(st, 296, tune_cands_[best].waves, tune_cands_[best].tile);
    return;
  }
  // the class's best so far (or the default) for the solve, the next untimed
  // candidate for its first H.psi
  const TuneCand base = ms[best] >= 0 ? tune_cands_[best] : tune_cands_[0];
  S.q1.groups = S.p1.groups;
  S.q1.gterms = S.p1.gterms;
  S.q2.groups = S.p2.groups;
  S.q2.gterms = S.p2.gterms;
  S.p1.upload(st, 296, base.waves, base.tile);
  S.p2.upload(st, 296, base.waves, base.tile);
  S.q1.upload(st, 296, tune_cands_[next].waves, tune_cands_[next].tile);
  S.q2.upload(st, 296, tune_cands_[next].waves, tune_cands_[next].tile);
  S.tune_cand = next;
}

// Times every candidate schedule on the current superblock (FP64 H.psi of a
// scratch vector, best of `reps` device timings each), records them for its size
// class and keeps the fastest for the superblock.  Returns that candidate.
int Engine::tune_superblock(int reps) {
  Superblock& S = sb;
  if (!S.valid) throw Error(-4, "no superblock");
  const long long n = S.wl.dim;
  DevBuf x((size_t)std::max<long long>(n, 1), st, true), y((size_t)std::max<long long>(n, 1), st, false);
  const int cls = (int)std::floor(std::log2(std::max(S.ref_flops / 1e9, 1e-9)));
  std::array<double, kTuneCands> ms;
  for (int c = 0; c < kTuneCands; ++c) {
    TaskList a, b;
    a.groups = S.p1.groups;
    a.gterms = S.p1.gterms;
    b.groups = S.p2.groups;
    b.gterms = S.p2.gterms;
    a.upload(st, 296, tune_cands_[c].waves, tune_cands_[c].tile);
    b.upload(st, 296, tune_cands_[c].waves, tune_cands_[c].tile);
    double best = 1e30;
    for (int r = 0; r < std::max(reps, 1) + 1; ++r) {   // the first run warms up
      cuda_check(cudaEventRecord(ev0, st), "event");
      run_tasks(a, x.p, y.p, S.scratch->p);
      run_tasks(b, x.p, y.p, S.scratch->p);
      cuda_check(cudaEventRecord(ev1, st), "event");
      cuda_check(cudaEventSynchronize(ev1), "sync");
      float t = 0.f;
      cuda_check(cudaEventElapsedTime(&t, ev0, ev1), "elapsed");
      if (r > 0) best = std::min(best, (double)t);
    }
    ms[c] = best / (S.ref_flops / 1e9);
  }
  tune_ms_[cls] = ms;
  const int win = (int)(std::min_element(ms.begin(), ms.end()) - ms.begin());
  S.p1.upload(st, 296, tune_cands_[win].waves, tune_cands_[win].tile);
  S.p2.upload(st, 296, tune_cands_[win].waves, tune_cands_[win].tile);
  S.tune_cand = -1;
  S.tune_pending = false;
  S.q1 = TaskList();
  S.q2 = TaskList();
  cuda_check(cudaStreamSynchronize(st), "sync");
  return win;
}

void Engine::tune_observe() {
  Superblock& S = sb;
  if (!S.tune_pending || cudaEventQuery(tune_ev_[1]) != cudaSuccess) return;
  S.tune_pending = false;
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, tune_ev_[0], tune_ev_[1]) != cudaSuccess) return;
  tune_ms_[S.tune_class][S.tune_cand] = ms / (S.ref_flops / 1e9);
  S.tune_cand = -1;
  S.q1 = TaskList();
  S.q2 = TaskList();
}

void Engine::superblock_set(DModel&& sys, DModel&& env, Basis&& sys_bs, Basis&& env_bs, WLayout&& wl) {
  if (sb.valid && sb.tune_pending) {   // a candidate timed on the previous superblock is read first
    cudaEventSynchronize(tune_ev_[1]);
    tune_observe();
  }
  sb = Superblock();
  sb.sys = std::move(sys);
  sb.env = std::move(env);
  sb.sys_bs = std::move(sys_bs);
  sb.env_bs = std::move(env_bs);
  sb.wl = std::move(wl);
  L.setup(sb.sys.len, sb.env.len);
  // warm-up steps stop Lanczos at a loose tolerance, where the reference's
  // iteration path decides the result: they stay FP64 in either precision
  split_now_ = precision_ == 1 && !in_warmup_;
  build_merge();
  build_hpsi_tasks();
  cuda_check(cudaStreamSynchronize(st), "superblock sync");
  sb.valid = true;
  views_of_batch_ = false;
}

void Engine::hpsi(const double2* d_in, double2* d_out) { hpsi_form(d_in, d_out, sb.p1s.split); }

void Engine::hpsi_form(const double2* d_in, double2* d_out, bool split) {
  if (!sb.valid) throw Error(-4, "no superblock");
  // the autotuner's candidate runs the first FP64 H.psi after the superblock is set
  const bool probe = !split && sb.tune_cand >= 0 && !sb.tune_pending;
  TaskList& a = split ? sb.p1s : (probe ? sb.q1 : sb.p1);
  TaskList& b = split ? sb.p2s : (probe ? sb.q2 : sb.p2);
  if (split && !a.split) throw Error(-4, "split-precision lists were not built for this superblock");
  if (probe) {
    sb.tune_pending = true;
    for (auto& e : tune_ev_)
      if (!e) cuda_check(cudaEventCreate(&e), "cudaEventCreate");
    cuda_check(cudaEventRecord(tune_ev_[0], st), "event");
  }
  cuda_check(cudaEventRecord(ev0, st), "event");
  if (split) slice_input(sb.sv, d_in, st);
  run_tasks(a, const_cast<double2*>(d_in), d_out, sb.scratch->p);
  run_tasks(b, const_cast<double2*>(d_in), d_out, sb.scratch->p);
  cuda_check(cudaEventRecord(ev1, st), "event");
  if (probe) cuda_check(cudaEventRecord(tune_ev_[1], st), "event");
  last_stats.launches = (a.njobs > 0) + (b.njobs > 0) + (a.nreds > 0) + (b.nreds > 0) + (split ? 1 : 0);
  last_stats.hpsi_flops = sb.ref_flops;
}

}  // namespace tsc
