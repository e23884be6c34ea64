// Site densities <n_i> of the last ground state of a run (measure_operator_dia,
// measure.f90:3-62, called at main.f90:268 with num_elec).  The site operator
// of site i is carried into the current system (or environment) block through
// the stored bases and truncations exactly as Get_sys_oper_dia /
// Get_env_oper_dia do (get_sys.f90:1147-1277, trun_idx = 1 as main.f90:89 sets
// it): update_site_dia once, then update_block_dia + update_trun_dia per
// length.  Each expectation value (measure_sys/env_block, measure_sys/env_site,
// measure.f90:778-1030) is one grouped launch that writes M = (O x 1) psi, or
// psi (1 x O), piece by piece into a psi-shaped buffer, and one Re<psi, M>.
#include <algorithm>
#include <cmath>

#include "../../include/tsc_gpu.h"
#include "tsc_ctx.hpp"
#include "tsc_engine.hpp"

namespace tsc {

namespace {
inline long long absoff(const double2* p) { return (long long)((uintptr_t)p / sizeof(double2)); }
constexpr int S_MEAS = 1960;   // scalar slot of the dot product (free range of d_scal)
}  // namespace

DBlock Engine::site_as_block(const SiteOp& so) {
  DBlock b;
  b.len = 1;
  b.num = (int)so.sub.size();
  b.dim = b.num;
  b.up_dif = so.up_dif;
  b.down_dif = so.down_dif;
  b.buf = std::make_shared<DevBuf>((size_t)std::max(b.num, 1), st, false);
  std::vector<double2> h(std::max(b.num, 1));
  for (int i = 0; i < b.num; ++i) {
    SubDesc s;
    s.num_up = so.sub[i].num_up;
    s.num_down = so.sub[i].num_down;
    s.down_dif = so.sub[i].down_dif;
    s.row_dim = s.sdim = 1;
    s.off = i;
    b.sub.push_back(s);
    h[i] = make_double2(so.sub[i].val, 0.0);
  }
  cuda_check(cudaMemcpyAsync(b.buf->p, h.data(), b.num * sizeof(double2), cudaMemcpyHostToDevice, st), "upload");
  cuda_check(cudaStreamSynchronize(st), "sync");
  return b;
}

// a block shaped like the (square, diagonal) sectors of `basis`, one group per sector
static DBlock dia_like(const Basis& basis, TaskList& tl, std::vector<int>& g, cudaStream_t s) {
  DBlock b;
  b.len = basis.len;
  b.num = basis.num;
  b.dim = basis.dim;
  long long off = 0;
  for (const auto& S : basis.sec) {
    SubDesc d;
    d.num_up = S.num_up;
    d.num_down = S.num_down;
    d.row_dim = d.sdim = S.dim;
    d.off = off;
    off += (long long)S.dim * S.dim;
    b.sub.push_back(d);
  }
  b.buf = std::make_shared<DevBuf>((size_t)std::max<long long>(off, 1), s, false);
  for (int i = 0; i < b.num; ++i)
    g.push_back(tl.add_group(b.ptr(i), BASE_ABS, 0, b.sub[i].row_dim, b.sub[i].row_dim, b.sub[i].sdim, 0));
  return b;
}

// update_site_dia (block.f90:2554-2615)
DBlock Engine::site_dia(const SiteOp& so, const Basis& basis) {
  TaskList tl;
  std::vector<int> g;
  DBlock b = dia_like(basis, tl, g, st);
  for (int k = 0; k < b.num; ++k)
    for (const auto& p : basis.sec[k].pcs)
      for (const auto& s : so.sub)
        if (s.num_up == p.st_num_up && s.num_down == p.st_num_down) {
          GTerm t{};
          t.kind = TK_DIAG;
          t.ar = s.val * std::sqrt((1.0 + b.sub[k].num_down) / (1.0 + s.num_down));
          t.r0 = t.c0 = p.spos;
          t.rm = t.rn = p.sdim;
          tl.gterms[g[k]].push_back(t);
          break;
        }
  tl.upload(st);
  run_tasks(tl, nullptr, nullptr, nullptr);
  return b;
}

// update_block_dia (block.f90:2495-2548)
DBlock Engine::block_dia(const DBlock& blk, const Basis& basis) {
  TaskList tl;
  std::vector<int> g;
  DBlock b = dia_like(basis, tl, g, st);
  for (int k = 0; k < b.num; ++k)
    for (const auto& p : basis.sec[k].pcs)
      for (int i = 0; i < blk.num; ++i)
        if (blk.sub[i].num_up == p.bl_num_up && blk.sub[i].num_down == p.bl_num_down) {
          GTerm t{};
          t.kind = TK_AXPY;
          t.ar = std::sqrt((1.0 + b.sub[k].num_down) / (1.0 + blk.sub[i].num_down));
          t.r_base = BASE_ABS;
          t.r_off = absoff(blk.ptr(i));
          t.r_ld = blk.sub[i].row_dim;
          t.r_op = OP_N;
          t.r0 = t.c0 = p.spos;
          t.rm = t.rn = p.sdim;
          tl.gterms[g[k]].push_back(t);
          break;
        }
  tl.upload(st);
  run_tasks(tl, nullptr, nullptr, nullptr);
  return b;
}

// update_trun_dia (block.f90:3465-3527): eff_i = U_i^H ori_x U_i
DBlock Engine::trun_dia(const DBlock& ori, const DBlock& trun) {
  DBlock e;
  e.len = ori.len;
  e.num = trun.num;
  e.dim = trun.dim;
  long long off = 0;
  for (const auto& u : trun.sub) {
    SubDesc d;
    d.num_up = u.num_up;
    d.num_down = u.num_down;
    d.row_dim = d.sdim = u.sdim;
    d.off = off;
    off += (long long)u.sdim * u.sdim;
    e.sub.push_back(d);
  }
  e.buf = std::make_shared<DevBuf>((size_t)std::max<long long>(off, 1), st, false);
  TaskList t1, t2;
  long long mid = 0;
  for (int i = 0; i < e.num; ++i) {
    const int g2 = t2.add_group(e.ptr(i), BASE_ABS, 0, e.sub[i].row_dim, e.sub[i].row_dim, e.sub[i].sdim, 0);
    int x = -1;
    for (int z = 0; z < ori.num; ++z)
      if (ori.sub[z].num_up == e.sub[i].num_up && ori.sub[z].num_down == e.sub[i].num_down) {
        x = z;
        break;
      }
    if (x < 0) continue;
    const int od = ori.sub[x].row_dim, ed = e.sub[i].sdim;
    const int g1 = t1.add_group(nullptr, BASE_SCR, mid, od, od, ed, 0);
    GTerm a{};
    a.kind = TK_GEMM;
    a.ar = 1.0;
    a.l_base = a.r_base = BASE_ABS;
    a.l_off = absoff(ori.ptr(x));
    a.l_ld = od;
    a.l_op = OP_N;
    a.r_off = absoff(trun.ptr(i));
    a.r_ld = trun.sub[i].row_dim;
    a.r_op = OP_N;
    a.K = od;
    t1.gterms[g1].push_back(a);
    GTerm b{};
    b.kind = TK_GEMM;
    b.ar = 1.0;
    b.l_base = BASE_ABS;
    b.l_off = absoff(trun.ptr(i));
    b.l_ld = trun.sub[i].row_dim;
    b.l_op = OP_C;
    b.r_base = BASE_SCR;
    b.r_off = mid;
    b.r_ld = od;
    b.r_op = OP_N;
    b.K = od;
    t2.gterms[g2].push_back(b);
    mid += (long long)od * ed;
  }
  DevBuf scr((size_t)std::max<long long>(mid, 1), st, false);
  t1.upload(st);
  t2.upload(st);
  run_tasks(t1, nullptr, nullptr, scr.p);
  run_tasks(t2, nullptr, nullptr, scr.p);
  cuda_check(cudaStreamSynchronize(st), "sync");
  return e;
}

DBlock Engine::oper_dia_in_block(const SiteOp& so, int old_idx, int new_idx, bool sys, bool trunc) {
  const auto& bsm = sys ? sys_bsm : env_bsm;
  const auto& truns = sys ? sys_truns : env_truns;
  const int trun_idx = 1;
  const int one = std::min(old_idx, new_idx), two = std::max(old_idx, new_idx);
  DBlock cur, out;
  if (one <= two - 1) {
    if (one <= 1) cur = site_as_block(so);
    else if (one <= trun_idx) cur = site_dia(so, bsm.at(one));
    else cur = trun_dia(site_dia(so, bsm.at(one)), truns.at(one));
    int idx = one;
    while (idx + 1 <= two - 1) {
      DBlock mid = block_dia(cur, bsm.at(idx + 1));
      idx++;
      cur = (idx <= trun_idx) ? mid : trun_dia(mid, truns.at(idx));
    }
    out = block_dia(cur, bsm.at(idx + 1));
  } else {
    out = (one <= 1) ? site_as_block(so) : site_dia(so, bsm.at(two));
  }
  auto it = truns.find(two);
  if (!trunc || it == truns.end()) return out;
  return trun_dia(out, it->second);
}

// Re <psi | (O x 1) | psi> (sys) or Re <psi | (1 x O) | psi> (env) for a block
// operator `bl`, or for the site operator `so` on the block's added site; the
// imaginary part into *imag when given.
double Engine::expect_dia(const DBlock* bl, const SiteOp* so, const Basis& bs, bool sys, double* imag) {
  const WLayout& w = disk_layout;
  const long long n = w.dim;
  DevBuf M((size_t)std::max<long long>(n, 1), st, false);
  TaskList tl;
  for (const WSec& ws : w.sec) {
    const int qup = sys ? ws.sys_num_up : ws.env_num_up, qdn = sys ? ws.sys_num_down : ws.env_num_down;
    const int k = bs.find(qup, qdn);
    if (k < 0) throw Error(TSC_E_QN, "measure: wave sector missing from the block basis");
    for (const Piece& p : bs.sec[k].pcs) {
      const long long goff = sys ? ws.off + p.spos : ws.off + (long long)p.spos * ws.sys_dim;
      const int gm = sys ? p.sdim : ws.sys_dim, gn = sys ? ws.env_dim : p.sdim;
      const int g = tl.add_group(nullptr, BASE_OUT, goff, ws.sys_dim, gm, gn, 0);
      if (bl) {
        int y = -1;
        for (int z = 0; z < bl->num; ++z)
          if (bl->sub[z].num_up == p.bl_num_up && bl->sub[z].num_down == p.bl_num_down) {
            y = z;
            break;
          }
        if (y < 0) continue;
        GTerm t{};
        t.kind = TK_GEMM;
        t.ar = 1.0 / std::sqrt(1.0 + p.bl_num_down);
        if (sys) {   // coef * O_y * psi[spos.., :]
          t.l_base = BASE_ABS;
          t.l_off = absoff(bl->ptr(y));
          t.l_ld = p.sdim;
          t.r_base = BASE_IN;
          t.r_off = goff;
          t.r_ld = ws.sys_dim;
        } else {     // coef * psi[:, spos..] * O_y
          t.l_base = BASE_IN;
          t.l_off = goff;
          t.l_ld = ws.sys_dim;
          t.r_base = BASE_ABS;
          t.r_off = absoff(bl->ptr(y));
          t.r_ld = p.sdim;
        }
        t.l_op = t.r_op = OP_N;
        t.K = p.sdim;
        tl.gterms[g].push_back(t);
      } else {
        for (const auto& s : so->sub)
          if (s.num_up == p.st_num_up && s.num_down == p.st_num_down) {
            GTerm t{};
            t.kind = TK_AXPY;
            t.ar = s.val / std::sqrt(1.0 + p.st_num_down);
            t.r_base = BASE_IN;
            t.r_off = goff;
            t.r_ld = ws.sys_dim;
            t.r_op = OP_N;
            t.r0 = t.c0 = 0;
            t.rm = gm;
            t.rn = gn;
            tl.gterms[g].push_back(t);
            break;
          }
      }
    }
  }
  tl.upload(st);
  run_tasks(tl, disk_wave->p, M.p, nullptr);
  DevBuf part((size_t)((n + 8191) / 8192 + 1), st, false);
  cuda_check(launch_zdot(disk_wave->p, M.p, n, reinterpret_cast<double*>(part.p), d_scal + S_MEAS, st), "dot");
  cuda_check(cudaMemcpyAsync(h_scal + S_MEAS, d_scal + S_MEAS, 2 * sizeof(double), cudaMemcpyDeviceToHost, st), "d2h");
  cuda_check(cudaStreamSynchronize(st), "sync");
  if (imag) *imag = h_scal[S_MEAS + 1];
  return h_scal[S_MEAS];
}

std::vector<double> Engine::measure_density() {
  if (!disk_wave || disk_layout.num == 0) throw Error(TSC_E_STATE, "no ground state: run tsc_dmrg_run first");
  const int N = L.num_site, sl = disk_layout.sys_len, el = disk_layout.env_len;
  std::vector<double> ave(N, 0.0);
  for (int i = 1; i <= sl - 1; ++i) {
    DBlock op = oper_dia_in_block(num_elec, i, sl - 1, true);
    ave[i - 1] = expect_dia(&op, nullptr, sys_bsm.at(sl), true);
  }
  ave[sl - 1] = expect_dia(nullptr, &num_elec, sys_bsm.at(sl), true);
  for (int i = 1; i <= el - 1; ++i) {
    DBlock op = oper_dia_in_block(num_elec, i, el - 1, false);
    ave[N - i] = expect_dia(&op, nullptr, env_bsm.at(el), false);
  }
  ave[N - el] = expect_dia(nullptr, &num_elec, env_bsm.at(el), false);
  return ave;
}

// ---- density-density correlation (Get_density_cor, measure.f90:2525-2681) -------
//
// For oper1 = oper2 = num_elec (charge- and spin-conserving, tensor rank 0) the
// reference's ndia transport (Get_sys/env_oper_ndia, get_sys.f90:1536-1668)
// reduces to the dia one: update_block_ndia_sys with rank 0 scales by
// sqrt((1+J)/(1+j)), the factor update_block_dia applies.

// Change_sys_oper_dia / Change_env_oper_dia (get_sys.f90:1281-1331), Truns = .true.:
// a block operator of length `from` carried into the block of length `to`.
DBlock Engine::carry_dia(const DBlock& op, int from, int to, bool sys) {
  const auto& bsm = sys ? sys_bsm : env_bsm;
  const auto& truns = sys ? sys_truns : env_truns;
  const int trun_idx = 1;
  if (from == to) return op;
  DBlock cur = op;
  int idx = from;
  while (idx + 1 <= to - 1) {
    DBlock mid = block_dia(cur, bsm.at(idx + 1));
    idx++;
    cur = (idx <= trun_idx) ? mid : trun_dia(mid, truns.at(idx));
  }
  DBlock out = block_dia(cur, bsm.at(idx + 1));
  auto it = truns.find(to);
  if (it == truns.end()) return out;
  return trun_dia(out, it->second);
}

// block_mul_block_ndia (block.f90:376-635) for two rank-0 operators on the
// sectors of `basis`: the 3j sums there reduce to 1/sqrt(2J+1) per sector.
DBlock Engine::product_dia(const DBlock& a, const DBlock& b, const Basis& basis) {
  TaskList tl;
  std::vector<int> g;
  DBlock p = dia_like(basis, tl, g, st);
  if (a.num != p.num || b.num != p.num) throw Error(TSC_E_QN, "density_cor: operators not on the product basis");
  for (int k = 0; k < p.num; ++k) {
    const int d = p.sub[k].row_dim;
    GTerm t{};
    t.kind = TK_GEMM;
    t.ar = 1.0 / std::sqrt(1.0 + p.sub[k].num_down);
    t.l_base = t.r_base = BASE_ABS;
    t.l_off = absoff(a.ptr(k));
    t.r_off = absoff(b.ptr(k));
    t.l_ld = t.r_ld = d;
    t.l_op = t.r_op = OP_N;
    t.K = d;
    tl.gterms[g[k]].push_back(t);
  }
  tl.upload(st);
  run_tasks(tl, nullptr, nullptr, nullptr);
  return p;
}

namespace {
const SiteSub* site_entry(const SiteOp& so, int up, int down) {
  for (const auto& s : so.sub)
    if (s.num_up == up && s.num_down == down) return &s;
  return nullptr;
}
int block_entry(const DBlock& b, int up, int down) {
  for (int z = 0; z < b.num; ++z)
    if (b.sub[z].num_up == up && b.sub[z].num_down == down) return z;
  return -1;
}
}  // namespace

// sys_block_site_cor_ndia (measure.f90:4064-4218), FlagSign 'B', rank 0:
// Re <psi | (O_block x n_site) | psi> within the system block.
double Engine::corr_block_site(const DBlock& bl, const SiteOp& so, const Basis& bs) {
  const WLayout& w = disk_layout;
  const long long n = w.dim;
  DevBuf M((size_t)std::max<long long>(n, 1), st, false);
  TaskList tl;
  for (const WSec& ws : w.sec) {
    const int k = bs.find(ws.sys_num_up, ws.sys_num_down);
    if (k < 0) throw Error(TSC_E_QN, "measure: wave sector missing from the block basis");
    for (const Piece& p : bs.sec[k].pcs) {
      const long long goff = ws.off + p.spos;
      const int g = tl.add_group(nullptr, BASE_OUT, goff, ws.sys_dim, p.sdim, ws.env_dim, 0);
      const int y = block_entry(bl, p.bl_num_up, p.bl_num_down);
      const SiteSub* e = site_entry(so, p.st_num_up, p.st_num_down);
      if (y < 0 || !e) continue;
      double c = w6j(p.bl_num_down, p.bl_num_down, 0, p.st_num_down, p.st_num_down, ws.sys_num_down);
      if (c == 0.0) continue;
      if (((p.bl_num_down + p.st_num_down + ws.sys_num_down) / 2) % 2) c = -c;
      GTerm t{};
      t.kind = TK_GEMM;
      t.ar = e->val * c;
      t.l_base = BASE_ABS;
      t.l_off = absoff(bl.ptr(y));
      t.l_ld = p.sdim;
      t.r_base = BASE_IN;
      t.r_off = goff;
      t.r_ld = ws.sys_dim;
      t.l_op = t.r_op = OP_N;
      t.K = p.sdim;
      tl.gterms[g].push_back(t);
    }
  }
  tl.upload(st);
  run_tasks(tl, disk_wave->p, M.p, nullptr);
  DevBuf part((size_t)((n + 8191) / 8192 + 2) / 2 + 1, st, false);
  cuda_check(launch_multi_dot(disk_wave->p, 0, 1, M.p, n, reinterpret_cast<double*>(part.p), d_scal + S_MEAS, st),
             "dot");
  cuda_check(cudaMemcpyAsync(h_scal + S_MEAS, d_scal + S_MEAS, sizeof(double), cudaMemcpyDeviceToHost, st), "d2h");
  cuda_check(cudaStreamSynchronize(st), "sync");
  return h_scal[S_MEAS];
}

// sys_block_env_site_cor_ndia (measure.f90:4666-4903; eso) and
// sys_block_env_block_cor_ndia (measure.f90:4398-4661; ebl), FlagSign 'B', rank 0.
// Per (system piece x, environment piece y) of every wave sector:
//   site:  coef * st_y * <psi_xy, O_x psi_xy>
//   block: coef * <O_x psi_xy, psi_xy O_y^H>
// with coef the two 6j factors of the reference; one grouped launch per side
// writes the psi-shaped products, one dot sums them.
double Engine::corr_block_env(const DBlock& bl, const DBlock* ebl, const SiteOp* eso, const Basis& sbs,
                              const Basis& ebs) {
  const WLayout& w = disk_layout;
  const long long n = w.dim;
  DevBuf M1((size_t)std::max<long long>(n, 1), st, false);
  DevBuf M2((size_t)std::max<long long>(n, 1), st, false);
  TaskList t1, t2;
  for (const WSec& ws : w.sec) {
    const int ks = sbs.find(ws.sys_num_up, ws.sys_num_down), ke = ebs.find(ws.env_num_up, ws.env_num_down);
    if (ks < 0 || ke < 0) throw Error(TSC_E_QN, "measure: wave sector missing from the block basis");
    const int Js = ws.sys_num_down, Je = ws.env_num_down;
    for (const Piece& x : sbs.sec[ks].pcs)
      for (const Piece& y : ebs.sec[ke].pcs) {
        const long long goff = ws.off + (long long)y.spos * ws.sys_dim + x.spos;
        const int g1 = t1.add_group(nullptr, BASE_OUT, goff, ws.sys_dim, x.sdim, y.sdim, 0);
        const int g2 = ebl ? t2.add_group(nullptr, BASE_SCR, goff, ws.sys_dim, x.sdim, y.sdim, 0) : -1;
        const int sid = block_entry(bl, x.bl_num_up, x.bl_num_down);
        if (sid < 0) continue;
        double c = w6j(Js, 0, Js, x.bl_num_down, x.st_num_down, x.bl_num_down);
        if (c == 0.0) continue;
        double ev = 1.0;
        int eid = -1;
        if (eso) {
          const SiteSub* e = site_entry(*eso, y.st_num_up, y.st_num_down);
          if (!e) continue;
          ev = e->val;
          c *= w6j(Js, 0, Je, y.st_num_down, y.bl_num_down, y.st_num_down);
          if (((x.bl_num_down + x.st_num_down + Js) / 2 + (y.bl_num_down + y.st_num_down + Js) / 2) % 2) c = -c;
        } else {
          eid = block_entry(*ebl, y.bl_num_up, y.bl_num_down);
          if (eid < 0) continue;
          c *= w6j(Js, 0, Je, y.bl_num_down, y.st_num_down, y.bl_num_down);
          if (((x.bl_num_down + x.st_num_down + Js) / 2 + (y.bl_num_down + y.st_num_down + Je) / 2) % 2) c = -c;
        }
        if (c == 0.0) continue;
        c *= std::sqrt((1.0 + Js) * (1.0 + Je));
        GTerm a{};   // coef * ev * O_x psi_xy
        a.kind = TK_GEMM;
        a.ar = c * ev;
        a.l_base = BASE_ABS;
        a.l_off = absoff(bl.ptr(sid));
        a.l_ld = x.sdim;
        a.r_base = BASE_IN;
        a.r_off = goff;
        a.r_ld = ws.sys_dim;
        a.l_op = a.r_op = OP_N;
        a.K = x.sdim;
        t1.gterms[g1].push_back(a);
        if (ebl) {   // psi_xy O_y^H
          GTerm b{};
          b.kind = TK_GEMM;
          b.ar = 1.0;
          b.l_base = BASE_IN;
          b.l_off = goff;
          b.l_ld = ws.sys_dim;
          b.l_op = OP_N;
          b.r_base = BASE_ABS;
          b.r_off = absoff(ebl->ptr(eid));
          b.r_ld = y.sdim;
          b.r_op = OP_C;
          b.K = y.sdim;
          t2.gterms[g2].push_back(b);
        }
      }
  }
  t1.upload(st);
  run_tasks(t1, disk_wave->p, M1.p, nullptr);
  if (ebl) {
    t2.upload(st);
    run_tasks(t2, disk_wave->p, nullptr, M2.p);
  }
  DevBuf part((size_t)((n + 8191) / 8192 + 2) / 2 + 1, st, false);
  cuda_check(launch_multi_dot(M1.p, 0, 1, ebl ? M2.p : disk_wave->p, n, reinterpret_cast<double*>(part.p),
                              d_scal + S_MEAS, st),
             "dot");
  cuda_check(cudaMemcpyAsync(h_scal + S_MEAS, d_scal + S_MEAS, sizeof(double), cudaMemcpyDeviceToHost, st), "d2h");
  cuda_check(cudaStreamSynchronize(st), "sync");
  return h_scal[S_MEAS];
}

std::vector<double> Engine::measure_density_cor(int xi) {
  if (!disk_wave || disk_layout.num == 0) throw Error(TSC_E_STATE, "no ground state: run tsc_dmrg_run first");
  const int N = L.num_site, ny = L.Ny, sl = disk_layout.sys_len, el = disk_layout.env_len;
  if (xi < 1 || xi > sl - 1) throw Error(TSC_E_ARG, "density_cor: the site must lie in the system block of the wave");
  std::vector<double> out(N, 0.0);
  // partners inside the system block: Get_sys2b (measure.f90:2486-2523) + measure_sys_block
  for (int j = xi + ny; j <= sl - 1; j += ny) {
    DBlock a = oper_dia_in_block(num_elec, xi, j, true, false);
    DBlock b = site_dia(num_elec, sys_bsm.at(j));
    DBlock p = product_dia(a, b, sys_bsm.at(j));
    auto it = sys_truns.find(j);
    DBlock q = (j <= 1 || it == sys_truns.end()) ? p : trun_dia(p, it->second);
    DBlock s = carry_dia(q, j, sl - 1, true);
    out[j - 1] = expect_dia(&s, nullptr, sys_bsm.at(sl), true);
  }
  const int last = N - N / 6 + ny;
  if (sl > last) return out;
  DBlock sys_oper = oper_dia_in_block(num_elec, xi, sl - 1, true);
  for (int j = sl; j <= std::min(last, N); ++j) {
    if ((j - xi) % ny != 0) continue;
    if (j == sl) {
      out[j - 1] = corr_block_site(sys_oper, num_elec, sys_bsm.at(sl));
    } else if (j == sl + 1) {
      out[j - 1] = corr_block_env(sys_oper, nullptr, &num_elec, sys_bsm.at(sl), env_bsm.at(el));
    } else {
      DBlock env_oper = oper_dia_in_block(num_elec, N - j + 1, el - 1, false);
      out[j - 1] = corr_block_env(sys_oper, &env_oper, nullptr, sys_bsm.at(sl), env_bsm.at(el));
    }
  }
  return out;
}

}  // namespace tsc

using namespace tsc;

extern "C" int tsc_measure_density(tsc_ctx* ctx, double* out, int nsites) {
  if (!ctx) return TSC_E_ARG;
  try {
    if (!ctx->eng) throw Error(TSC_E_STATE, "no engine");
    std::vector<double> d = ctx->eng->measure_density();
    if (!out || nsites < (int)d.size()) throw Error(TSC_E_ARG, "output holds fewer values than the lattice has sites");
    std::copy(d.begin(), d.end(), out);
    ctx->err.clear();
    return (int)d.size();
  } catch (Error& e) {
    ctx->err = e.what();
    return e.code;
  } catch (std::exception& e) {
    ctx->err = e.what();
    return TSC_E_ARG;
  }
}

extern "C" int tsc_measure_density_cor(tsc_ctx* ctx, int site, double* out, int nsites) {
  if (!ctx) return TSC_E_ARG;
  try {
    if (!ctx->eng) throw Error(TSC_E_STATE, "no engine");
    std::vector<double> d = ctx->eng->measure_density_cor(site);
    if (!out || nsites < (int)d.size()) throw Error(TSC_E_ARG, "output holds fewer values than the lattice has sites");
    std::copy(d.begin(), d.end(), out);
    ctx->err.clear();
    return (int)d.size();
  } catch (Error& e) {
    ctx->err = e.what();
    return e.code;
  } catch (std::exception& e) {
    ctx->err = e.what();
    return TSC_E_ARG;
  }
}
