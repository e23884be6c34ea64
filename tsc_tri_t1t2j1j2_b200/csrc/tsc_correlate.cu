// Two-site correlations <op1_xi op2_j> (complex) of the last ground state for site
// operators of any tensor rank: Get_density_cor (measure.f90:2525-2681) as main.f90
// calls it for the spin-spin correlation (st_sd, st_sd, Flags 'B', rank 1,
// main.f90:275) and the electron correlation (st_elec_up, st_elec_down, Flags
// 'F', rank 1/2, main.f90:288).  The density-density case (rank 0) has its own,
// cheaper path in tsc_measure.cu.
//
// Operators travel into the system / environment block through the run's stored
// bases and truncations as the reference's ndia transport does
// (Get_sys_oper_ndia / Change_sys_oper_ndia, get_sys.f90:1536-1723: update_site_ndia,
// update_block_ndia, update_trun_ndia, block.f90:2624-3683).  Each step is one
// grouped launch (AXPY / DIAG scatters for the enlargement, two GEMM launches for
// U^H O U).  A correlation value is a sum over terms of <P_t, Q_t> for matrices
// P_t, Q_t the reference forms one by one (sys_block_site_cor_ndia,
// sys_block_env_site_cor_ndia, sys_block_env_block_cor_ndia, measure.f90:4064-4903);
// here every term's P_t and Q_t is a rectangle of two scratch buffers, written by
// one grouped launch each, and one dot sums them all.
#include <algorithm>
#include <cmath>
#include <map>
#include <tuple>

#include "../../include/tsc_gpu.h"
#include "tsc_ctx.hpp"
#include "tsc_engine.hpp"

namespace tsc {

namespace {
inline long long absoff(const double2* p) { return (long long)((uintptr_t)p / sizeof(double2)); }
inline double pm1(int e) { return ((e % 2) + 2) % 2 == 0 ? 1.0 : -1.0; }
constexpr int S_COR = 1970;   // scalar slot of the dot product (free range of d_scal)

int find_sub3(const DBlock& b, int up, int down, int dd) {
  for (int z = 0; z < b.num; ++z)
    if (b.sub[z].num_up == up && b.sub[z].num_down == down && b.sub[z].down_dif == dd) return z;
  return -1;
}
const SiteSub* site_sub3(const SiteOp& so, int up, int down, int dd) {
  for (const auto& s : so.sub)
    if (s.num_up == up && s.num_down == down && s.down_dif == dd) return &s;
  return nullptr;
}
const Piece* find_piece(const Sector& S, int bu, int bd, int su, int sd) {
  for (const auto& p : S.pcs)
    if (p.bl_num_up == bu && p.bl_num_down == bd && p.st_num_up == su && p.st_num_down == sd) return &p;
  return nullptr;
}
// the sign of the correlators' electron-number parity term: 'B' +1, 'F' (-1)^n
// (measure.f90:4167-4178, 4569-4580, 4830-4841)
inline double flag_sign(char flag, int n) { return flag == 'F' && (n % 2) ? -1.0 : 1.0; }

// Conjugate transpose of a site operator (block_transfer_trans, block.f90:33-64, on 1x1 elements)
SiteOp site_trans(const SiteOp& o) {
  SiteOp r;
  r.up_dif = -o.up_dif;
  r.down_dif = o.down_dif;
  for (const auto& s : o.sub) r.sub.push_back({s.num_up + o.up_dif, s.num_down + s.down_dif, -s.down_dif, s.val});
  return r;
}
}  // namespace

// sub-block layout of an operator of (up_dif, rank K) on `basis` (block.f90:2655-2712), zeroed
DBlock Engine::ndia_layout(const Basis& basis, int up_dif, int K, TaskList& tl, std::vector<int>& g) {
  DBlock b;
  b.len = basis.len;
  b.up_dif = up_dif;
  b.down_dif = K;
  long long off = 0;
  for (int x = 0; x < basis.num; ++x)
    for (int dd = -K; dd <= K; dd += 2) {
      const int y = basis.find(basis.sec[x].num_up + up_dif, basis.sec[x].num_down + dd);
      if (y < 0) continue;
      SubDesc s;
      s.num_up = basis.sec[x].num_up;
      s.num_down = basis.sec[x].num_down;
      s.down_dif = dd;
      s.row_dim = basis.sec[y].dim;
      s.sdim = basis.sec[x].dim;
      s.off = off;
      off += (long long)s.row_dim * s.sdim;
      b.dim += s.sdim;
      b.sub.push_back(s);
    }
  b.num = (int)b.sub.size();
  b.buf = std::make_shared<DevBuf>((size_t)std::max<long long>(off, 1), st, false);
  for (int i = 0; i < b.num; ++i)
    g.push_back(tl.add_group(b.ptr(i), BASE_ABS, 0, b.sub[i].row_dim, b.sub[i].row_dim, b.sub[i].sdim, 0));
  return b;
}

// update_site_ndia_sys / _env (block.f90:3047-3459): the added site's operator on the enlarged basis
DBlock Engine::site_ndia(const SiteOp& so, const Basis& basis, bool env, char flag) {
  TaskList tl;
  std::vector<int> g;
  DBlock b = ndia_layout(basis, so.up_dif, so.down_dif, tl, g);
  const int up_dif = so.up_dif, K = so.down_dif;
  for (int i = 0; i < b.num; ++i) {
    const SubDesc& o = b.sub[i];
    const int rid = basis.find(o.num_up, o.num_down), lid = basis.find(o.num_up + up_dif, o.num_down + o.down_dif);
    if (rid < 0 || lid < 0) continue;
    const int lnd = o.num_down + o.down_dif, rnd = o.num_down;
    for (const auto& p : basis.sec[rid].pcs)
      for (int sdd = -K; sdd <= K; sdd += 2) {
        const SiteSub* ss = site_sub3(so, p.st_num_up, p.st_num_down, sdd);
        if (!ss) continue;
        const int lsu = p.st_num_up + up_dif, lsd = p.st_num_down + sdd;
        const Piece* q = nullptr;
        for (const auto& qq : basis.sec[lid].pcs)
          if (qq.st_num_up == lsu && qq.st_num_down == lsd && qq.bl_num_down == p.bl_num_down) {
            q = &qq;
            break;
          }
        if (!q) continue;
        const double sg = (!env && flag == 'F') ? pm1(p.bl_num_up) : 1.0;
        double c = w6j(lnd, K, rnd, p.st_num_down, p.bl_num_down, lsd);
        c *= pm1((p.bl_num_down + p.st_num_down + lnd + K) / 2) * std::sqrt((1.0 + lnd) * (1.0 + rnd));
        if (c == 0.0) continue;
        GTerm t{};
        t.kind = TK_DIAG;
        t.ar = c * sg * ss->val;
        t.r0 = q->spos;
        t.c0 = p.spos;
        t.rm = t.rn = p.sdim;
        tl.gterms[g[i]].push_back(t);
      }
  }
  tl.upload(st);
  run_tasks(tl, nullptr, nullptr, nullptr);
  return b;
}

// update_block_ndia_sys / _env (block.f90:2624-3036): a block operator on the enlarged basis
DBlock Engine::block_ndia(const DBlock& blk, const Basis& basis, bool env, char flag) {
  TaskList tl;
  std::vector<int> g;
  DBlock b = ndia_layout(basis, blk.up_dif, blk.down_dif, tl, g);
  const int up_dif = blk.up_dif, K = blk.down_dif;
  for (int i = 0; i < b.num; ++i) {
    const SubDesc& o = b.sub[i];
    const int rid = basis.find(o.num_up, o.num_down), lid = basis.find(o.num_up + up_dif, o.num_down + o.down_dif);
    if (rid < 0 || lid < 0) continue;
    const int lnd = o.num_down + o.down_dif, rnd = o.num_down;
    for (const auto& p : basis.sec[rid].pcs)
      for (int sdd = -K; sdd <= K; sdd += 2) {
        const int bid = find_sub3(blk, p.bl_num_up, p.bl_num_down, sdd);
        if (bid < 0) continue;
        const int lsu = p.bl_num_up + up_dif, lsd = p.bl_num_down + sdd;
        const Piece* q = nullptr;
        for (const auto& qq : basis.sec[lid].pcs)
          if (qq.bl_num_up == lsu && qq.bl_num_down == lsd && qq.st_num_down == p.st_num_down) {
            q = &qq;
            break;
          }
        if (!q) continue;
        const double sg = (env && flag == 'F') ? pm1(p.st_num_up) : 1.0;
        double c = w6j(lnd, K, rnd, p.bl_num_down, p.st_num_down, lsd);
        c *= std::sqrt((1.0 + lnd) * (1.0 + rnd)) * pm1((lsd + p.st_num_down + rnd + K) / 2);
        if (c == 0.0) continue;
        GTerm t{};
        t.kind = TK_AXPY;
        t.ar = c * sg;
        t.r_base = BASE_ABS;
        t.r_off = absoff(blk.ptr(bid));
        t.r_ld = blk.sub[bid].row_dim;
        t.r_op = OP_N;
        t.r0 = q->spos;
        t.c0 = p.spos;
        t.rm = q->sdim;
        t.rn = p.sdim;
        tl.gterms[g[i]].push_back(t);
      }
  }
  tl.upload(st);
  run_tasks(tl, nullptr, nullptr, nullptr);
  return b;
}

// update_trun_ndia (block.f90:3535-3683): eff = U_lhs^H ori U_rhs per (lhs, rhs) sector pair
DBlock Engine::trun_ndia(const DBlock& ori, const DBlock& trun) {
  const int up_dif = ori.up_dif, K = ori.down_dif;
  auto find_t = [&](int up, int down) {
    for (int z = 0; z < trun.num; ++z)
      if (trun.sub[z].num_up == up && trun.sub[z].num_down == down) return z;
    return -1;
  };
  DBlock e;
  e.len = ori.len;
  e.up_dif = up_dif;
  e.down_dif = K;
  long long off = 0;
  for (int x = 0; x < trun.num; ++x)
    for (int dd = -K; dd <= K; dd += 2) {
      const int y = find_t(trun.sub[x].num_up + up_dif, trun.sub[x].num_down + dd);
      if (y < 0) continue;
      SubDesc s;
      s.num_up = trun.sub[x].num_up;
      s.num_down = trun.sub[x].num_down;
      s.down_dif = dd;
      s.row_dim = trun.sub[y].sdim;
      s.sdim = trun.sub[x].sdim;
      s.off = off;
      off += (long long)s.row_dim * s.sdim;
      e.dim += s.sdim;
      e.sub.push_back(s);
    }
  e.num = (int)e.sub.size();
  e.buf = std::make_shared<DevBuf>((size_t)std::max<long long>(off, 1), st, true);
  TaskList t1, t2;
  long long mid_elems = 0;
  for (int i = 0; i < e.num; ++i) {
    const SubDesc& s = e.sub[i];
    const int rid = find_t(s.num_up, s.num_down), lid = find_t(s.num_up + up_dif, s.num_down + s.down_dif);
    const int oid = find_sub3(ori, s.num_up, s.num_down, s.down_dif);
    if (rid < 0 || lid < 0 || oid < 0) continue;
    const int orow = ori.sub[oid].row_dim, ocol = ori.sub[oid].sdim, rd = trun.sub[rid].sdim;
    const long long moff = mid_elems;
    mid_elems += (long long)orow * rd;
    const int g1 = t1.add_group(nullptr, BASE_SCR, moff, orow, orow, rd, 0);
    GTerm a{};
    a.kind = TK_GEMM;
    a.ar = 1.0;
    a.l_base = a.r_base = BASE_ABS;
    a.l_off = absoff(ori.ptr(oid));
    a.l_ld = orow;
    a.r_off = absoff(trun.ptr(rid));
    a.r_ld = trun.sub[rid].row_dim;
    a.l_op = a.r_op = OP_N;
    a.K = ocol;
    t1.gterms[g1].push_back(a);
    const int g2 = t2.add_group(e.ptr(i), BASE_ABS, 0, s.row_dim, s.row_dim, rd, 0);
    GTerm b{};
    b.kind = TK_GEMM;
    b.ar = 1.0;
    b.l_base = BASE_ABS;
    b.l_off = absoff(trun.ptr(lid));
    b.l_ld = trun.sub[lid].row_dim;
    b.l_op = OP_C;
    b.r_base = BASE_SCR;
    b.r_off = moff;
    b.r_ld = orow;
    b.r_op = OP_N;
    b.K = orow;
    t2.gterms[g2].push_back(b);
  }
  DevBuf mid((size_t)std::max<long long>(mid_elems, 1), st, false);
  t1.upload(st);
  t2.upload(st);
  run_tasks(t1, nullptr, nullptr, mid.p);
  run_tasks(t2, nullptr, nullptr, mid.p);
  cuda_check(cudaStreamSynchronize(st), "trun_ndia sync");
  return e;
}

// Get_sys_oper_ndia / Get_env_oper_ndia (get_sys.f90:1536-1668), trun_idx = 1:
// the site operator of site old_idx carried into the block of length new_idx
DBlock Engine::oper_ndia_in_block(const SiteOp& so, int old_idx, int new_idx, bool sys, bool trunc, char flag) {
  const auto& bsm = sys ? sys_bsm : env_bsm;
  const auto& truns = sys ? sys_truns : env_truns;
  const int trun_idx = 1;
  const int one = std::min(old_idx, new_idx), two = std::max(old_idx, new_idx);
  DBlock cur, out;
  if (one <= two - 1) {
    if (one <= 1) cur = site_as_block(so);
    else if (one <= trun_idx) cur = site_ndia(so, bsm.at(one), !sys, flag);
    else cur = trun_ndia(site_ndia(so, bsm.at(one), !sys, flag), truns.at(one));
    int idx = one;
    while (idx + 1 <= two - 1) {
      DBlock mid = block_ndia(cur, bsm.at(idx + 1), !sys, flag);
      idx++;
      cur = (idx <= trun_idx) ? mid : trun_ndia(mid, truns.at(idx));
    }
    out = block_ndia(cur, bsm.at(idx + 1), !sys, flag);
  } else {
    out = (one <= 1) ? site_as_block(so) : site_ndia(so, bsm.at(two), !sys, flag);
  }
  auto it = truns.find(two);
  if (!trunc || it == truns.end()) return out;
  return trun_ndia(out, it->second);
}

// Change_sys_oper_ndia / Change_env_oper_ndia (get_sys.f90:1672-1723); Truns = trunc_end
DBlock Engine::carry_ndia(const DBlock& op, int from, int to, bool sys, char flag, bool trunc_end) {
  const auto& bsm = sys ? sys_bsm : env_bsm;
  const auto& truns = sys ? sys_truns : env_truns;
  const int trun_idx = 1;
  if (from == to) return op;
  DBlock cur = op;
  int idx = from;
  while (idx + 1 <= to - 1) {
    DBlock mid = block_ndia(cur, bsm.at(idx + 1), !sys, flag);
    idx++;
    cur = (idx <= trun_idx) ? mid : trun_ndia(mid, truns.at(idx));
  }
  DBlock out = block_ndia(cur, bsm.at(idx + 1), !sys, flag);
  auto it = truns.find(to);
  if (!trunc_end || it == truns.end()) return out;
  return trun_ndia(out, it->second);
}

// block_mul_block_ndia (block.f90:376-635) with Flag1 = Flag2 = 'N', coefficient 1:
// (o1 o2) coupled to rank K on the sectors of `basis`; sub-block (sector, new
// spin) exists for new spin in |S-K| .. S+K present in the basis, and
// product[k] = sum_mid c(k, mid) o1[.., mid] o2[mid, k] with the 3j sums of
// block.f90:584-613 as written
DBlock Engine::product_ndia(const DBlock& o1, const DBlock& o2, int K, const Basis& basis) {
  const int up_dif = o1.up_dif + o2.up_dif, up_dif2 = o2.up_dif, K1 = o1.down_dif, K2 = o2.down_dif;
  DBlock p;
  p.len = basis.len;
  p.up_dif = up_dif;
  p.down_dif = K;
  long long off = 0;
  for (int x = 0; x < basis.num; ++x) {
    const int nd = basis.sec[x].num_down;
    for (int nnd = std::abs(nd - K); nnd <= nd + K; nnd += 2) {
      const int y = basis.find(basis.sec[x].num_up + up_dif, nnd);
      if (y < 0) continue;
      SubDesc d;
      d.num_up = basis.sec[x].num_up;
      d.num_down = nd;
      d.down_dif = nnd - nd;
      d.row_dim = basis.sec[y].dim;
      d.sdim = basis.sec[x].dim;
      d.off = off;
      off += (long long)d.row_dim * d.sdim;
      p.dim += d.sdim;
      p.sub.push_back(d);
    }
  }
  p.num = (int)p.sub.size();
  p.buf = std::make_shared<DevBuf>((size_t)std::max<long long>(off, 1), st, false);
  TaskList tl;
  for (int i = 0; i < p.num; ++i) {
    const SubDesc& s = p.sub[i];
    const int g = tl.add_group(p.ptr(i), BASE_ABS, 0, s.row_dim, s.row_dim, s.sdim, 0);
    const int num_up = s.num_up, num_down = s.num_down, new_num_down = num_down + s.down_dif;
    for (int mid = std::abs(num_down - K2); mid <= num_down + K2; mid += 2) {
      const int i2 = find_sub3(o2, num_up, num_down, mid - num_down);
      const int i1 = find_sub3(o1, num_up + up_dif2, mid, new_num_down - mid);
      if (i1 < 0 || i2 < 0) continue;
      const int kq = new_num_down - num_down;
      const double c11 = w3j(new_num_down, K, num_down, -new_num_down, kq, num_down);
      if (c11 == 0.0) throw Error(TSC_E_QN, "correlation: vanishing 3j normalisation");
      double c1 = 0.0;
      for (int m6 = -mid; m6 <= mid; m6 += 2) {
        const int m5 = new_num_down - m6;
        double c12 = w3j(new_num_down, K1, mid, -new_num_down, m5, m6);
        const int m44 = -m6, m55 = -m44 - num_down;
        c12 *= w3j(mid, K2, num_down, m44, m55, num_down) * pm1((mid + m44) / 2);
        c12 *= w3j(K1, K2, K, m5, m55, -kq) * pm1((-K1 + K2 + kq) / 2) * std::sqrt(K + 1.0);
        c1 += c12;
      }
      if (c1 == 0.0) continue;
      GTerm t{};
      t.kind = TK_GEMM;
      t.ar = c1 / c11;
      t.l_base = t.r_base = BASE_ABS;
      t.l_off = absoff(o1.ptr(i1));
      t.l_ld = o1.sub[i1].row_dim;
      t.r_off = absoff(o2.ptr(i2));
      t.r_ld = o2.sub[i2].row_dim;
      t.l_op = t.r_op = OP_N;
      t.K = o1.sub[i1].sdim;
      tl.gterms[g].push_back(t);
    }
  }
  tl.upload(st);
  run_tasks(tl, nullptr, nullptr, nullptr);
  return p;
}

// block_transfer_trans (block.f90:33-64): every sub-block conjugate-transposed,
// keyed by its row quantum numbers
DBlock Engine::transfer_trans(const DBlock& in) {
  DBlock out;
  out.len = in.len;
  out.num = in.num;
  out.dim = in.dim;
  out.up_dif = -in.up_dif;
  out.down_dif = in.down_dif;
  long long off = 0;
  for (const auto& x : in.sub) {
    SubDesc s;
    s.num_up = x.num_up + in.up_dif;
    s.num_down = x.num_down + x.down_dif;
    s.down_dif = -x.down_dif;
    s.row_dim = x.sdim;
    s.sdim = x.row_dim;
    s.off = off;
    off += (long long)s.row_dim * s.sdim;
    out.sub.push_back(s);
  }
  out.buf = std::make_shared<DevBuf>((size_t)std::max<long long>(off, 1), st, false);
  TaskList tl;
  for (int i = 0; i < out.num; ++i) {
    const int g = tl.add_group(out.ptr(i), BASE_ABS, 0, out.sub[i].row_dim, out.sub[i].row_dim, out.sub[i].sdim, 0);
    GTerm t{};
    t.kind = TK_AXPY;
    t.ar = 1.0;
    t.r_base = BASE_ABS;
    t.r_off = absoff(in.ptr(i));
    t.r_ld = in.sub[i].row_dim;
    t.r_op = OP_C;
    t.rm = out.sub[i].row_dim;
    t.rn = out.sub[i].sdim;
    tl.gterms[g].push_back(t);
  }
  tl.upload(st);
  run_tasks(tl, nullptr, nullptr, nullptr);
  return out;
}

// ---- correlators: sum over terms of Re <P_t, Q_t> ----------------------------------
// A PairSum collects terms: P_t = an AXPY copy of (or GEMM into) a rectangle, Q_t a
// GEMM product, each written to its own rectangle of scratch buffers S1 / S2.
struct Engine::PairSum {
  TaskList t1, t2;
  long long elems = 0;
  // adds a term's rectangle (rows x cols, ld rows) to both lists; returns the groups
  std::pair<int, int> add(int rows, int cols) {
    const long long off = elems;
    elems += (long long)rows * cols;
    return {t1.add_group(nullptr, BASE_OUT, off, rows, rows, cols, 0),
            t2.add_group(nullptr, BASE_SCR, off, rows, rows, cols, 0)};
  }
};

cplx Engine::pair_sum(PairSum& ps) {
  if (ps.elems == 0) return 0.0;
  DevBuf S1((size_t)ps.elems, st, false), S2((size_t)ps.elems, st, false);
  ps.t1.upload(st);
  ps.t2.upload(st);
  run_tasks(ps.t1, disk_wave->p, S1.p, nullptr);
  run_tasks(ps.t2, disk_wave->p, nullptr, S2.p);
  DevBuf part((size_t)((ps.elems + 8191) / 8192 + 1), st, false);
  cuda_check(launch_zdot(S1.p, S2.p, ps.elems, reinterpret_cast<double*>(part.p), d_scal + S_COR, st), "dot");
  cuda_check(cudaMemcpyAsync(h_scal + S_COR, d_scal + S_COR, 2 * sizeof(double), cudaMemcpyDeviceToHost, st), "d2h");
  cuda_check(cudaStreamSynchronize(st), "sync");
  return cplx(h_scal[S_COR], h_scal[S_COR + 1]);
}

namespace {
// P_t: alpha * psi[rect] copied (AXPY) into group g of a PairSum list
GTerm copy_rect(long long off, int ld, int rows, int cols, double a) {
  GTerm t{};
  t.kind = TK_AXPY;
  t.ar = a;
  t.r_base = BASE_IN;
  t.r_off = off;
  t.r_ld = ld;
  t.r_op = OP_N;
  t.rm = rows;
  t.rn = cols;
  return t;
}
// Q_t: alpha * L * psi[rect] (L of `lrows` rows, K = psi rect rows)
GTerm left_prod(const double2* L, int lrows, long long off, int ld, int K, double a) {
  GTerm t{};
  t.kind = TK_GEMM;
  t.ar = a;
  t.l_base = BASE_ABS;
  t.l_off = absoff(L);
  t.l_ld = lrows;
  t.r_base = BASE_IN;
  t.r_off = off;
  t.r_ld = ld;
  t.l_op = t.r_op = OP_N;
  t.K = K;
  return t;
}
}  // namespace

// sys_block_site_cor_ndia (measure.f90:4064-4218): <psi | (O_block x O_site) | psi>
cplx Engine::corr_site_ndia(const DBlock& bl, const SiteOp& st_op, const Basis& bs, char flag) {
  const WLayout& w = disk_layout;
  const int K = bl.down_dif, up_dif = bl.up_dif;
  PairSum ps;
  for (const WSec& ws : w.sec) {
    const int j = bs.find(ws.sys_num_up, ws.sys_num_down);
    if (j < 0) continue;
    for (const auto& p : bs.sec[j].pcs)
      for (int dd = -K; dd <= K; dd += 2)
        for (int sdd = -K; sdd <= K; sdd += 2) {
          const int nbu = p.bl_num_up + up_dif, nbd = p.bl_num_down + dd;
          const int nsu = p.st_num_up - up_dif, nsd = p.st_num_down - sdd;
          const int bid = find_sub3(bl, p.bl_num_up, p.bl_num_down, dd);
          const SiteSub* sv = site_sub3(st_op, nsu, nsd, sdd);
          const Piece* q = find_piece(bs.sec[j], nbu, nbd, nsu, nsd);
          if (bid < 0 || !sv || !q) continue;
          double c = w6j(nbd, p.bl_num_down, K, p.st_num_down, nsd, ws.sys_num_down) / std::sqrt(1.0 + K);
          if (c == 0.0) continue;
          c *= pm1((p.bl_num_down + nsd + K + ws.sys_num_down) / 2) * flag_sign(flag, p.bl_num_up) * sv->val;
          auto g = ps.add(q->sdim, ws.env_dim);
          ps.t1.gterms[g.first].push_back(copy_rect(ws.off + q->spos, ws.sys_dim, q->sdim, ws.env_dim, 1.0));
          ps.t2.gterms[g.second].push_back(left_prod(bl.ptr(bid), q->sdim, ws.off + p.spos, ws.sys_dim, p.sdim, c));
        }
  }
  return pair_sum(ps);
}

// sys_block_env_site_cor_ndia (measure.f90:4666-4903): block operator in the system
// block, site operator on the environment's added site
cplx Engine::corr_env_site_ndia(const DBlock& bl, const SiteOp& est, const Basis& sbs, const Basis& ebs, char flag) {
  const WLayout& w = disk_layout;
  const int K = bl.down_dif, Ke = est.down_dif, up_dif = bl.up_dif;
  PairSum ps;
  for (const WSec& ws : w.sec) {
    const int j = sbs.find(ws.sys_num_up, ws.sys_num_down), k = ebs.find(ws.env_num_up, ws.env_num_down);
    if (j < 0 || k < 0) continue;
    for (const auto& x : sbs.sec[j].pcs)
      for (const auto& y : ebs.sec[k].pcs)
        for (int bdd = -K; bdd <= K; bdd += 2) {
          const int nsbu = x.bl_num_up + up_dif, nsbd = x.bl_num_down + bdd;
          const int sys_id = find_sub3(bl, x.bl_num_up, x.bl_num_down, bdd);
          for (int sdd = -Ke; sdd <= Ke; sdd += 2) {
            const int neu = y.st_num_up - up_dif, ned = y.st_num_down - sdd;
            const SiteSub* ev = site_sub3(est, neu, ned, sdd);
            if (sys_id < 0 || !ev) continue;
            for (int nsd = std::abs(ws.sys_num_down - K); nsd <= ws.sys_num_down + K; nsd += 2) {
              const int nsu = ws.sys_num_up + up_dif, nenu = ws.env_num_up - up_dif, nend = nsd;
              const int m1 = sbs.find(nsu, nsd), m2 = ebs.find(nenu, nend);
              const Piece* qs = m1 < 0 ? nullptr : find_piece(sbs.sec[m1], nsbu, nsbd, x.st_num_up, x.st_num_down);
              const Piece* qe = nullptr;
              if (m2 >= 0)
                for (const auto& p : ebs.sec[m2].pcs)
                  if (p.st_num_up == neu && p.st_num_down == ned && p.bl_num_down == y.bl_num_down) {
                    qe = &p;
                    break;
                  }
              const int wid = w.find(nsu, nsd, nenu, nend);
              if (!qs || !qe || wid < 0) continue;
              double c = w6j(nsd, K, ws.sys_num_down, x.bl_num_down, x.st_num_down, nsbd);
              if (c == 0.0) continue;
              c *= w6j(nend, K, ws.env_num_down, y.st_num_down, y.bl_num_down, ned);
              if (c == 0.0) continue;
              c *= std::sqrt((1.0 + nend) * (1.0 + ws.env_num_down) / (1.0 + K));
              if ((((nsbd + x.st_num_down + ws.sys_num_down + K) / 2 + (y.bl_num_down + y.st_num_down + nend + K) / 2) %
                   2) != 0)
                c = -c;
              c *= flag_sign(flag, ws.sys_num_up) * ev->val;
              const WSec& nw = w.sec[wid];
              auto g = ps.add(qs->sdim, y.sdim);
              ps.t1.gterms[g.first].push_back(
                  copy_rect(nw.off + qs->spos + (long long)qe->spos * nw.sys_dim, nw.sys_dim, qs->sdim, y.sdim, 1.0));
              ps.t2.gterms[g.second].push_back(left_prod(bl.ptr(sys_id), qs->sdim,
                                                         ws.off + x.spos + (long long)y.spos * ws.sys_dim, ws.sys_dim,
                                                         x.sdim, c));
            }
          }
        }
  }
  return pair_sum(ps);
}

// sys_block_env_block_cor_ndia (measure.f90:4398-4661): block operators in both blocks;
// P_t = O_sys psi_xy, Q_t = c psi_(qs,qe) O_env^H
cplx Engine::corr_env_block_ndia(const DBlock& bl, const DBlock& ebl, const Basis& sbs, const Basis& ebs,
                                   char flag) {
  const WLayout& w = disk_layout;
  const int K = bl.down_dif, up_dif = bl.up_dif;
  PairSum ps;
  for (const WSec& ws : w.sec) {
    const int j = sbs.find(ws.sys_num_up, ws.sys_num_down), k = ebs.find(ws.env_num_up, ws.env_num_down);
    if (j < 0 || k < 0) continue;
    for (const auto& x : sbs.sec[j].pcs)
      for (const auto& y : ebs.sec[k].pcs)
        for (int dd = -K; dd <= K; dd += 2) {
          const int nsbu = x.bl_num_up + up_dif, nsbd = x.bl_num_down + dd;
          const int sys_id = find_sub3(bl, x.bl_num_up, x.bl_num_down, dd);
          for (int edd = -K; edd <= K; edd += 2) {
            const int nebu = y.bl_num_up - up_dif, nebd = y.bl_num_down - edd;
            const int env_id = find_sub3(ebl, nebu, nebd, edd);
            if (sys_id < 0 || env_id < 0) continue;
            for (int nsd = std::abs(ws.sys_num_down - K); nsd <= ws.sys_num_down + K; nsd += 2) {
              const int nsu = ws.sys_num_up + up_dif, nenu = ws.env_num_up - up_dif, nend = nsd;
              const int m1 = sbs.find(nsu, nsd), m2 = ebs.find(nenu, nend);
              const Piece* qs = m1 < 0 ? nullptr : find_piece(sbs.sec[m1], nsbu, nsbd, x.st_num_up, x.st_num_down);
              const Piece* qe = m2 < 0 ? nullptr : find_piece(ebs.sec[m2], nebu, nebd, y.st_num_up, y.st_num_down);
              const int wid = w.find(nsu, nsd, nenu, nend);
              if (!qs || !qe || wid < 0) continue;
              double c = w6j(nsd, K, ws.sys_num_down, x.bl_num_down, x.st_num_down, nsbd);
              if (c == 0.0) continue;
              c *= w6j(nend, K, ws.env_num_down, y.bl_num_down, y.st_num_down, nebd);
              if (c == 0.0) continue;
              c *= std::sqrt((1.0 + nend) * (1.0 + ws.env_num_down) / (1.0 + K));
              if ((((nsbd + x.st_num_down + ws.sys_num_down + K) / 2 + (nebd + y.st_num_down + ws.env_num_down + K) / 2) %
                   2) == 1)
                c = -c;
              c *= flag_sign(flag, ws.sys_num_up + y.st_num_up);
              const WSec& nw = w.sec[wid];
              auto g = ps.add(qs->sdim, y.sdim);
              ps.t1.gterms[g.first].push_back(left_prod(bl.ptr(sys_id), qs->sdim,
                                                        ws.off + x.spos + (long long)y.spos * ws.sys_dim, ws.sys_dim,
                                                        x.sdim, 1.0));
              GTerm b{};   // c psi_wid[qs rows, qe cols] * O_env^H  (O_env sub-block: y.sdim x qe.sdim)
              b.kind = TK_GEMM;
              b.ar = c;
              b.l_base = BASE_IN;
              b.l_off = nw.off + qs->spos + (long long)qe->spos * nw.sys_dim;
              b.l_ld = nw.sys_dim;
              b.l_op = OP_N;
              b.r_base = BASE_ABS;
              b.r_off = absoff(ebl.ptr(env_id));
              b.r_ld = ebl.sub[env_id].row_dim;
              b.r_op = OP_C;
              b.K = qe->sdim;
              ps.t2.gterms[g.second].push_back(b);
            }
          }
        }
  }
  return pair_sum(ps);
}

// Get_density_cor (measure.f90:2525-2681), xi = xj: the row <op1_xi op2_j> over the
// partners the reference visits, scaled as it scales the result (measure.f90:2586-2587)
std::vector<cplx> Engine::measure_oper_cor(const SiteOp& op1, const SiteOp& op2, char flag, int xi) {
  if (!disk_wave || disk_layout.num == 0) throw Error(TSC_E_STATE, "no ground state: run tsc_dmrg_run first");
  const int N = L.num_site, ny = L.Ny, sl = disk_layout.sys_len, el = disk_layout.env_len;
  if (xi < 1 || xi > sl - 1) throw Error(TSC_E_ARG, "correlation: the site must lie in the system block of the wave");
  const double scale = std::sqrt(1.0 + op1.down_dif) * (op1.down_dif == 2 ? -1.0 : 1.0);
  std::vector<cplx> out(N, 0.0);
  // partners inside the system block: Get_sys2b (measure.f90:2486-2523) + measure_sys_block
  for (int j = xi + ny; j <= sl - 1; j += ny) {
    DBlock a = oper_ndia_in_block(op1, xi, j, true, false, flag);
    DBlock b = oper_ndia_in_block(op2, j, j, true, false, flag);
    DBlock p = product_ndia(a, b, 0, sys_bsm.at(j));
    auto it = sys_truns.find(j);
    DBlock q = (j <= 1 || it == sys_truns.end()) ? p : trun_dia(p, it->second);
    DBlock s = carry_dia(q, j, sl - 1, true);
    double im = 0.0;
    const double re = expect_dia(&s, nullptr, sys_bsm.at(sl), true, &im);
    out[j - 1] = scale * cplx(re, im);
  }
  const int last = N - N / 6 + ny;
  if (sl > last) return out;
  DBlock s1 = oper_ndia_in_block(op1, xi, xi, true, false, flag);
  if (xi > 1) {
    auto it = sys_truns.find(xi);
    if (it != sys_truns.end()) s1 = trun_ndia(s1, it->second);
  }
  const DBlock sys_oper = carry_ndia(s1, xi, sl - 1, true, flag);
  const SiteOp site_op = op2.down_dif == 1 ? site_trans(op2) : op2;
  for (int j = sl; j <= std::min(last, N); ++j) {
    if ((j - xi) % ny != 0) continue;
    cplx v = 0.0;
    if (j == sl) {
      v = corr_site_ndia(sys_oper, site_op, sys_bsm.at(sl), flag);
    } else if (j == sl + 1) {
      v = corr_env_site_ndia(sys_oper, site_op, sys_bsm.at(sl), env_bsm.at(el), flag);
    } else {
      const int e = N - j + 1;
      DBlock e1 = oper_ndia_in_block(op2, e, e, false, false, flag);
      if (e > 1) {
        auto it = env_truns.find(e);
        if (it != env_truns.end()) e1 = trun_ndia(e1, it->second);
      }
      DBlock env_oper = carry_ndia(e1, e, el - 1, false, flag);
      if (op2.down_dif != 0) env_oper = transfer_trans(env_oper);
      v = corr_env_block_ndia(sys_oper, env_oper, sys_bsm.at(sl), env_bsm.at(el), flag);
    }
    out[j - 1] = scale * v;
  }
  return out;
}

// ---- singlet pair correlations (Get_mSCOP_Operator_Cor0, measure.f90:2683-2834) ----
//
// O+_ab = (c+_{a up} c+_{b dn} - c+_{a dn} c+_{b up}) / sqrt(2) (measure.f90:5441-5442)
// is the rank-0 coupling of two st_elec_up, formed at the longer length.

// Get_sys_two (measure.f90:2837-2874): O+_{idx1 idx2} on the system block of
// length idx2, truncated there
DBlock Engine::sys_pair(int idx1, int idx2) {
  DBlock a = oper_ndia_in_block(st_elec_up, idx1, idx2, true, false, 'F');
  DBlock b = oper_ndia_in_block(st_elec_up, idx2, idx2, true, false, 'F');
  DBlock p = product_ndia(a, b, 0, sys_bsm.at(idx2));
  auto it = sys_truns.find(idx2);
  if (idx2 <= 1 || it == sys_truns.end()) return p;
  return trun_ndia(p, it->second);
}

// Get_sys_two1 (measure.f90:2877-2932): the pair of length idx2 times st_elec_down
// at idx3 (coupled to rank 1/2), times st_elec_down at idx4 (coupled to rank 0),
// carried into the system block of the wave
DBlock Engine::sys_pair_four(int idx2, int idx3, int idx4, const DBlock& pair) {
  const int sl = disk_layout.sys_len;
  DBlock m = carry_ndia(pair, idx2, idx3, true, 'B', false);
  DBlock c3 = oper_ndia_in_block(st_elec_down, idx3, idx3, true, false, 'F');
  DBlock t3 = product_ndia(m, c3, 1, sys_bsm.at(idx3));
  auto it3 = sys_truns.find(idx3);
  if (idx3 > 1 && it3 != sys_truns.end()) t3 = trun_ndia(t3, it3->second);
  DBlock m4 = carry_ndia(t3, idx3, idx4, true, 'F', false);
  DBlock c4 = oper_ndia_in_block(st_elec_down, idx4, idx4, true, false, 'F');
  DBlock t4 = product_ndia(m4, c4, 0, sys_bsm.at(idx4));
  auto it4 = sys_truns.find(idx4);
  if (idx4 > 1 && it4 != sys_truns.end()) t4 = trun_dia(t4, it4->second);
  return carry_dia(t4, idx4, sl - 1, true);
}

// Get_SCOP_Operator_Env, Flags 'S0' (measure.f90:5450-5505): O+_{idx1 idx2} on the
// environment block of length idx2, carried to new_idx (truncated there when trunc_end)
DBlock Engine::env_pair(int idx1, int idx2, int new_idx, bool trunc_end) {
  DBlock a = oper_ndia_in_block(st_elec_up, idx1, idx2, false, false, 'F');
  DBlock b = oper_ndia_in_block(st_elec_up, idx2, idx2, false, false, 'F');
  DBlock e = product_ndia(a, b, 0, env_bsm.at(idx2));
  auto it = env_truns.find(idx2);
  if (idx2 > 1 && it != env_truns.end()) e = trun_ndia(e, it->second);
  return carry_ndia(e, idx2, new_idx, false, 'B', trunc_end);
}

// Get_mSCOP_Operator_Cor0 from label 11 (the part main.f90:259-262 reaches), Flags
// 'S0': the pair on the bond (xc1, neib(xc1, ij1)) against the bonds (s3, neib(s3,
// 1|3|5)) for s3 on the leg of xc1 up to xc2, first in the system block, then in
// the environment block (values conjugated there, as the reference writes them)
std::vector<Engine::PairCor> Engine::measure_pair_cor(int xc1, int xc2, int ij, int ij1) {
  if (!disk_wave || disk_layout.num == 0) throw Error(TSC_E_STATE, "no ground state: run tsc_dmrg_run first");
  const int N = L.num_site, ny = L.Ny, sl = disk_layout.sys_len, el = disk_layout.env_len;
  if (xc1 < 1 || xc1 > N || ij1 < 1 || ij1 > Lattice::neibt) throw Error(TSC_E_ARG, "pair_cor: bad first bond");
  if (xc2 > N) throw Error(TSC_E_ARG, "pair_cor: the last site lies past the lattice");
  std::vector<PairCor> out;
  const int sid1 = xc1, sid2 = L.NEIB(sid1, ij1);
  if (sid2 < 1) throw Error(TSC_E_ARG, "pair_cor: the first bond leaves the lattice");
  const int lo = std::min(sid1, sid2), hi = std::max(sid1, sid2);
  if (hi > sl - 1) throw Error(TSC_E_ARG, "pair_cor: the first bond must lie in the system block of the wave");
  const DBlock pair = sys_pair(lo, hi);
  for (int sid3 = sid1 + ny + ij; sid3 <= sl - 1; sid3 += ny) {
    if (sid3 <= hi || sid3 > xc2) continue;
    for (int i = 1; i <= 5; i += 2) {
      const int sid4 = L.NEIB(sid3, i);
      if (std::min(sid4, sid3) <= hi) continue;
      if (std::max(sid3, sid4) > sl - 1) continue;
      DBlock four = sys_pair_four(hi, std::min(sid3, sid4), std::max(sid3, sid4), pair);
      double im = 0.0;
      const double re = expect_dia(&four, nullptr, sys_bsm.at(sl), true, &im);
      out.push_back(PairCor{sid1, sid2, sid3, sid4, cplx(re, im)});
    }
  }
  const DBlock sys_oper = carry_ndia(pair, hi, sl - 1, true, 'B', true);
  const int m0 = (sl + 2) % ny, m1 = (sid1 - 1) % ny;
  for (int sid3 = sl + 2 - m0 + m1 + 1 + ij; sid3 <= xc2; sid3 += ny) {
    const int eid1 = N - sid3 + 1;
    if (eid1 > el - 1) continue;
    for (int i = 1; i <= 5; i += 2) {
      const int sid4 = L.NEIB(sid3, i);
      if (sid4 < 1) continue;
      const int eid2 = N - sid4 + 1;
      if (std::max(eid1, eid2) > el - 1) continue;
      DBlock env_oper = env_pair(std::min(eid1, eid2), std::max(eid1, eid2), el - 1, true);
      const cplx v = corr_env_block_ndia(sys_oper, env_oper, sys_bsm.at(sl), env_bsm.at(el), 'B');
      out.push_back(PairCor{sid1, sid2, sid3, sid4, std::conj(v)});
    }
  }
  return out;
}

}  // namespace tsc

using namespace tsc;

extern "C" int tsc_measure_correlation(tsc_ctx* ctx, int kind, int site, double* out, int nsites) {
  int n = 0;
  const int rc = guard(ctx, [&] {
    if (!ctx->eng) throw Error(TSC_E_STATE, "no engine");
    Engine& E = *ctx->eng;
    std::vector<cplx> d;
    if (kind == TSC_COR_DENSITY) {
      for (double v : E.measure_density_cor(site)) d.push_back(v);
    } else if (kind == TSC_COR_SPIN) {
      d = E.measure_oper_cor(E.st_sd, E.st_sd, 'B', site);
    } else if (kind == TSC_COR_ELECTRON) {
      d = E.measure_oper_cor(E.st_elec_up, E.st_elec_down, 'F', site);
    } else {
      throw Error(TSC_E_ARG, "unknown correlation kind");
    }
    if (!out || nsites < (int)d.size()) throw Error(TSC_E_ARG, "output holds fewer values than the lattice has sites");
    for (size_t j = 0; j < d.size(); ++j) {
      out[2 * j] = d[j].real();
      out[2 * j + 1] = d[j].imag();
    }
    n = (int)d.size();
  });
  return rc == TSC_OK ? n : rc;
}

extern "C" int tsc_measure_pair_correlation(tsc_ctx* ctx, int xc1, int xc2, int ij, int ij1, int* bonds,
                                            double* values, int cap) {
  int n = 0;
  const int rc = guard(ctx, [&] {
    if (!ctx->eng) throw Error(TSC_E_STATE, "no engine");
    if (cap > 0 && (!bonds || !values)) throw Error(TSC_E_ARG, "null output");
    const auto r = ctx->eng->measure_pair_cor(xc1, xc2, ij, ij1);
    for (int k = 0; k < (int)r.size() && k < cap; ++k) {
      bonds[4 * k] = r[k].s1;
      bonds[4 * k + 1] = r[k].s2;
      bonds[4 * k + 2] = r[k].s3;
      bonds[4 * k + 3] = r[k].s4;
      values[2 * k] = r[k].value.real();
      values[2 * k + 1] = r[k].value.imag();
    }
    n = (int)r.size();
  });
  return rc == TSC_OK ? n : rc;
}
