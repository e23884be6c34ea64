// Oracle H.psi: model_wave (get_sys.f90:6915-7393), hmerge (get_sys.f90:7398-7626)
// and the live block-sparse kernels it calls (get_sys.f90:1783-5204).  Loop nests,
// sector searches, coefficients, signs and ZGEMM operand modes follow the
// reference line by line; dead code behind `go to 110` / `go to 1051` is omitted.
// TEST INFRASTRUCTURE ONLY (see oracle.hpp).
#include <chrono>
#include <cmath>
#include <cstdio>
#include <stdexcept>

#include "oracle.hpp"

namespace orc {

namespace {

inline int find_bs(const Basis& b, int up, int down) {
  for (int x = 0; x < b.num; ++x)
    if (b.sub[x].new_num_up == up && b.sub[x].new_num_down == down) return x;
  return -1;
}
inline int find_blk(const Block& b, int up, int down) {
  for (int k = 0; k < b.num; ++k)
    if (b.sub[k].num_up == up && b.sub[k].num_down == down) return k;
  return -1;
}
inline int find_blk3(const Block& b, int up, int down, int dd) {
  for (int k = 0; k < b.num; ++k)
    if (b.sub[k].num_up == up && b.sub[k].num_down == down && b.sub[k].down_dif == dd) return k;
  return -1;
}
inline int find_wave(const Wave& w, int su, int sd, int eu, int ed) {
  for (int k = 0; k < w.num; ++k) {
    const SubWave& s = w.sub[k];
    if (s.sys_num_up == su && s.sys_num_down == sd && s.env_num_up == eu && s.env_num_down == ed)
      return k;
  }
  return -1;
}
inline double sgn_parity(int n) { return (n % 2 == 0) ? 1.0 : -1.0; }
inline double pm1(int e) { return ((e % 2) + 2) % 2 == 0 ? 1.0 : -1.0; }   // (-1)**e
const cplx cone(1.0, 0.0), czero(0.0, 0.0);

inline cplx* at(SubWave& s, int r, int c) { return &s.vec[(size_t)c * s.sys_dim + r]; }
inline const cplx* at(const SubWave& s, int r, int c) { return &s.vec[(size_t)c * s.sys_dim + r]; }

// out(r0:r0+m, c0:c0+n) += a * in(r1:r1+m, c1:c1+n)
void axpy_rect(SubWave& out, int r0, int c0, const SubWave& in, int r1, int c1, int m, int n, cplx a) {
  for (int c = 0; c < n; ++c)
    for (int r = 0; r < m; ++r) *at(out, r0 + r, c0 + c) += a * *at(in, r1 + r, c1 + c);
  g_gemm_flops += 8.0 * m * n;
}

// ---------------------------------------------------------------- diagonal kernels
// block_vec_dia, get_sys.f90:1783-1832
void block_vec_dia(const Block& sys_bl, const Basis& sys_bs, const Wave& in, Wave& out, cplx coef) {
  for (int i = 0; i < in.num; ++i) {
    const SubWave& wi = in.sub[i];
    int x = find_bs(sys_bs, wi.sys_num_up, wi.sys_num_down);
    if (x < 0) continue;
    for (const auto& p : sys_bs.sub[x].sub) {
      cplx coef1 = coef / std::sqrt(1.0 + p.bl_num_down);
      int k = find_blk(sys_bl, p.bl_num_up, p.bl_num_down);
      if (k < 0) continue;
      zgemm('N', 'N', p.sdim, wi.env_dim, p.sdim, coef1, sys_bl.sub[k].mat.data(), p.sdim,
            at(wi, p.spos, 0), wi.sys_dim, cone, at(out.sub[i], p.spos, 0), wi.sys_dim);
    }
  }
}

// vec_block_dia, get_sys.f90:1836-1885
void vec_block_dia(const Block& env_bl, const Basis& env_bs, const Wave& in, Wave& out, cplx coef) {
  for (int i = 0; i < in.num; ++i) {
    const SubWave& wi = in.sub[i];
    int x = find_bs(env_bs, wi.env_num_up, wi.env_num_down);
    if (x < 0) continue;
    for (const auto& p : env_bs.sub[x].sub) {
      cplx coef1 = coef / std::sqrt(1.0 + p.bl_num_down);
      int k = find_blk(env_bl, p.bl_num_up, p.bl_num_down);
      if (k < 0) continue;
      zgemm('N', 'C', wi.sys_dim, p.sdim, p.sdim, coef1, at(wi, 0, p.spos), wi.sys_dim,
            env_bl.sub[k].mat.data(), p.sdim, cone, at(out.sub[i], 0, p.spos), wi.sys_dim);
    }
  }
}

// block_site_vec_dia, get_sys.f90:2006-2077
void block_site_vec_dia(const Block& sys_bl, const Block& sys_st, const Basis& sys_bs,
                        const Wave& in, Wave& out, cplx coef) {
  for (int i = 0; i < in.num; ++i) {
    const SubWave& wi = in.sub[i];
    int x = find_bs(sys_bs, wi.sys_num_up, wi.sys_num_down);
    if (x < 0) continue;
    for (const auto& p : sys_bs.sub[x].sub) {
      int bl = find_blk(sys_bl, p.bl_num_up, p.bl_num_down);
      int st = find_blk(sys_st, p.st_num_up, p.st_num_down);
      if (bl < 0 || st < 0) continue;
      cplx c = coef * sys_st.sub[st].mat[0];
      c = c / std::sqrt((1.0 + p.bl_num_down) * (1.0 + p.st_num_down));
      zgemm('N', 'N', p.sdim, wi.env_dim, p.sdim, c, sys_bl.sub[bl].mat.data(), p.sdim,
            at(wi, p.spos, 0), wi.sys_dim, cone, at(out.sub[i], p.spos, 0), wi.sys_dim);
    }
  }
}

// vec_block_site_dia, get_sys.f90:2081-2154
void vec_block_site_dia(const Block& env_bl, const Block& env_st, const Basis& env_bs,
                        const Wave& in, Wave& out, cplx coef) {
  for (int i = 0; i < in.num; ++i) {
    const SubWave& wi = in.sub[i];
    int x = find_bs(env_bs, wi.env_num_up, wi.env_num_down);
    if (x < 0) continue;
    for (const auto& p : env_bs.sub[x].sub) {
      int bl = find_blk(env_bl, p.bl_num_up, p.bl_num_down);
      int st = find_blk(env_st, p.st_num_up, p.st_num_down);
      if (bl < 0 || st < 0) continue;
      cplx c = coef * env_st.sub[st].mat[0];
      c = c / std::sqrt((1.0 + p.bl_num_down) * (1.0 + p.st_num_down));
      zgemm('N', 'C', wi.sys_dim, p.sdim, p.sdim, c, at(wi, 0, p.spos), wi.sys_dim,
            env_bl.sub[bl].mat.data(), p.sdim, cone, at(out.sub[i], 0, p.spos), wi.sys_dim);
    }
  }
}

// site_vec_site_dia, get_sys.f90:2158-2254
void site_vec_site_dia(const Block& sys_st, const Block& env_st, const Basis& sys_bs,
                       const Basis& env_bs, const Wave& in, Wave& out, cplx coef) {
  for (int i = 0; i < in.num; ++i) {
    const SubWave& wi = in.sub[i];
    int xs = find_bs(sys_bs, wi.sys_num_up, wi.sys_num_down);
    int ye = find_bs(env_bs, wi.env_num_up, wi.env_num_down);
    if (xs < 0 || ye < 0) continue;
    for (const auto& ps : sys_bs.sub[xs].sub) {
      int ss = find_blk(sys_st, ps.st_num_up, ps.st_num_down);
      for (const auto& pe : env_bs.sub[ye].sub) {
        int es = find_blk(env_st, pe.st_num_up, pe.st_num_down);
        if (ss < 0 || es < 0) continue;
        cplx c = coef * sys_st.sub[ss].mat[0] * env_st.sub[es].mat[0];
        c = c / std::sqrt((1.0 + ps.st_num_down) * (1.0 + pe.st_num_down));
        axpy_rect(out.sub[i], ps.spos, pe.spos, wi, ps.spos, pe.spos, ps.sdim, pe.sdim, c);
      }
    }
  }
}

// block_vec_site_dia, get_sys.f90:2258-2357
void block_vec_site_dia(const Block& sys_bl, const Block& env_st, const Basis& sys_bs,
                        const Basis& env_bs, const Wave& in, Wave& out, cplx coef) {
  for (int i = 0; i < in.num; ++i) {
    const SubWave& wi = in.sub[i];
    int xs = find_bs(sys_bs, wi.sys_num_up, wi.sys_num_down);
    int ye = find_bs(env_bs, wi.env_num_up, wi.env_num_down);
    if (xs < 0 || ye < 0) continue;
    for (const auto& ps : sys_bs.sub[xs].sub) {
      int sb = find_blk(sys_bl, ps.bl_num_up, ps.bl_num_down);
      for (const auto& pe : env_bs.sub[ye].sub) {
        int es = find_blk(env_st, pe.st_num_up, pe.st_num_down);
        if (sb < 0 || es < 0) continue;
        cplx c = coef * env_st.sub[es].mat[0];
        c = c / std::sqrt((1.0 + pe.st_num_down) * (1.0 + ps.bl_num_down));
        zgemm('N', 'N', ps.sdim, pe.sdim, ps.sdim, c, sys_bl.sub[sb].mat.data(), ps.sdim,
              at(wi, ps.spos, pe.spos), wi.sys_dim, cone, at(out.sub[i], ps.spos, pe.spos), wi.sys_dim);
      }
    }
  }
}

// site_vec_block_dia, get_sys.f90:2361-2460
void site_vec_block_dia(const Block& sys_st, const Block& env_bl, const Basis& sys_bs,
                        const Basis& env_bs, const Wave& in, Wave& out, cplx coef) {
  for (int i = 0; i < in.num; ++i) {
    const SubWave& wi = in.sub[i];
    int xs = find_bs(sys_bs, wi.sys_num_up, wi.sys_num_down);
    int ye = find_bs(env_bs, wi.env_num_up, wi.env_num_down);
    if (xs < 0 || ye < 0) continue;
    for (const auto& ps : sys_bs.sub[xs].sub) {
      int ss = find_blk(sys_st, ps.st_num_up, ps.st_num_down);
      for (const auto& pe : env_bs.sub[ye].sub) {
        int eb = find_blk(env_bl, pe.bl_num_up, pe.bl_num_down);
        if (ss < 0 || eb < 0) continue;
        cplx c = coef * sys_st.sub[ss].mat[0];
        c = c / std::sqrt((1.0 + pe.bl_num_down) * (1.0 + ps.st_num_down));
        zgemm('N', 'C', ps.sdim, pe.sdim, pe.sdim, c, at(wi, ps.spos, pe.spos), wi.sys_dim,
              env_bl.sub[eb].mat.data(), pe.sdim, cone, at(out.sub[i], ps.spos, pe.spos), wi.sys_dim);
      }
    }
  }
}

// block_vec_block_dia, get_sys.f90:2464-2569
void block_vec_block_dia(const Block& sys_bl, const Block& env_bl, const Basis& sys_bs,
                         const Basis& env_bs, const Wave& in, Wave& out, cplx coef) {
  std::vector<cplx> mat;
  for (int i = 0; i < in.num; ++i) {
    const SubWave& wi = in.sub[i];
    int xs = find_bs(sys_bs, wi.sys_num_up, wi.sys_num_down);
    int ye = find_bs(env_bs, wi.env_num_up, wi.env_num_down);
    if (xs < 0 || ye < 0) continue;
    for (const auto& ps : sys_bs.sub[xs].sub) {
      int sb = find_blk(sys_bl, ps.bl_num_up, ps.bl_num_down);
      for (const auto& pe : env_bs.sub[ye].sub) {
        int eb = find_blk(env_bl, pe.bl_num_up, pe.bl_num_down);
        if (sb < 0 || eb < 0) continue;
        if (ps.sdim * pe.sdim == 0) throw std::runtime_error("dimen wrong");   // :2550-2551
        mat.assign((size_t)ps.sdim * pe.sdim, 0.0);
        cplx c1 = coef / std::sqrt((1.0 + pe.bl_num_down) * (1.0 + ps.bl_num_down));
        zgemm('N', 'N', ps.sdim, pe.sdim, ps.sdim, cone, sys_bl.sub[sb].mat.data(), ps.sdim,
              at(wi, ps.spos, pe.spos), wi.sys_dim, czero, mat.data(), ps.sdim);
        zgemm('N', 'C', ps.sdim, pe.sdim, pe.sdim, c1, mat.data(), ps.sdim,
              env_bl.sub[eb].mat.data(), pe.sdim, cone, at(out.sub[i], ps.spos, pe.spos), wi.sys_dim);
      }
    }
  }
}

// ------------------------------------------------------------ non-diagonal kernels
// block_site_vec_ndia, get_sys.f90:2578-2838 (live branch, before `go to 110`)
void block_site_vec_ndia(const Block& sys_bl, char FlagBL, const Block& sys_st, char FlagST,
                         const Basis& sys_bs, const Wave& in, Wave& out, cplx coef) {
  (void)FlagBL;
  int up_dif = sys_bl.up_dif, K = sys_bl.down_dif;
  if (up_dif != sys_st.up_dif || K != sys_st.down_dif)
    throw std::runtime_error("Quantum number error in block_site_vec!");
  for (int i = 0; i < in.num; ++i) {
    const SubWave& wi = in.sub[i];
    int sys_num_down = wi.sys_num_down, env_dim = wi.env_dim;
    int k = find_bs(sys_bs, wi.sys_num_up, wi.sys_num_down);
    if (k < 0) continue;
    const BasisMap& bm = sys_bs.sub[k];
    for (const auto& p : bm.sub) {
      for (int dd = -K; dd <= K; dd += 2) {
        for (int sdd = -K; sdd <= K; sdd += 2) {
          int bl_id = find_blk3(sys_bl, p.bl_num_up, p.bl_num_down, dd);
          int nst_up = p.st_num_up - up_dif, nst_down = p.st_num_down - sdd;
          int st_id = find_blk3(sys_st, nst_up, nst_down, sdd);
          int nbl_up = p.bl_num_up + up_dif, nbl_down = p.bl_num_down + dd;
          if (bl_id < 0 || st_id < 0) continue;
          int new_pos = -1, new_dim = 0;
          for (const auto& q : bm.sub)
            if (q.bl_num_up == nbl_up && q.bl_num_down == nbl_down && q.st_num_up == nst_up &&
                q.st_num_down == nst_down) {
              new_pos = q.spos;
              new_dim = q.sdim;
              break;
            }
          if (new_pos < 0) continue;
          double SignST = 1.0;
          if (FlagST == 'F') SignST = sgn_parity(p.bl_num_up);
          int j1 = nbl_down, j2 = p.bl_num_down, j3 = K, j4 = p.st_num_down, j5 = nst_down,
              j6 = sys_num_down;
          double c1 = w6js(j1, j2, j3, j4, j5, j6);
          if (c1 == 0.0) continue;
          c1 = c1 * pm1((j2 + j5 + j3 + j6) / 2) / std::sqrt(1.0 + K);
          double Signs = SignST * c1;
          cplx ct = Signs * coef * sys_st.sub[st_id].mat[0];
          int old_pos = p.spos, old_dim = p.sdim;
          zgemm('N', 'N', new_dim, env_dim, old_dim, ct, sys_bl.sub[bl_id].mat.data(), new_dim,
                at(wi, old_pos, 0), wi.sys_dim, cone, at(out.sub[i], new_pos, 0), wi.sys_dim);
          if (up_dif != 0) {
            ct = std::conj(ct);
            zgemm('C', 'N', old_dim, env_dim, new_dim, ct, sys_bl.sub[bl_id].mat.data(), new_dim,
                  at(wi, new_pos, 0), wi.sys_dim, cone, at(out.sub[i], old_pos, 0), wi.sys_dim);
          }
        }
      }
    }
  }
}

// vec_block_site_ndia, get_sys.f90:2842-3128 (live branch)
void vec_block_site_ndia(const Block& env_bl, char FlagBL, const Block& env_st, char FlagST,
                         const Basis& env_bs, const Wave& in, Wave& out, cplx coef) {
  int up_dif = env_bl.up_dif, K = env_bl.down_dif;
  if (up_dif != env_st.up_dif || K != env_st.down_dif)
    throw std::runtime_error("Quantum number error in vec_block_site!");
  for (int i = 0; i < in.num; ++i) {
    const SubWave& wi = in.sub[i];
    int sys_num_up = wi.sys_num_up, env_num_down = wi.env_num_down, sys_dim = wi.sys_dim;
    int k = find_bs(env_bs, wi.env_num_up, wi.env_num_down);
    if (k < 0) continue;
    const BasisMap& bm = env_bs.sub[k];
    for (const auto& p : bm.sub) {
      for (int bdd = -K; bdd <= K; bdd += 2) {
        int bl_id = find_blk3(env_bl, p.bl_num_up, p.bl_num_down, bdd);
        for (int sdd = -K; sdd <= K; sdd += 2) {
          int nst_up = p.st_num_up - up_dif, nst_down = p.st_num_down - sdd;
          int st_id = find_blk3(env_st, nst_up, nst_down, sdd);
          int nbl_up = p.bl_num_up + up_dif, nbl_down = p.bl_num_down + bdd;
          if (st_id < 0 || bl_id < 0) continue;
          int new_pos = -1, new_dim = 0;
          for (const auto& q : bm.sub)
            if (q.bl_num_up == nbl_up && q.bl_num_down == nbl_down && q.st_num_up == nst_up &&
                q.st_num_down == nst_down) {
              new_pos = q.spos;
              new_dim = q.sdim;
              break;
            }
          if (new_pos < 0) continue;
          double SignBL = 1.0, SignST = 1.0;
          if (FlagBL == 'F') SignBL = sgn_parity(sys_num_up + nst_up);
          if (FlagST == 'F') SignST = sgn_parity(sys_num_up);
          int j1 = nbl_down, j2 = p.bl_num_down, j3 = K, j4 = p.st_num_down, j5 = nst_down,
              j6 = env_num_down;
          double c1 = w6js(j1, j2, j3, j4, j5, j6);
          if (c1 == 0.0) continue;
          c1 = c1 * pm1((j2 + j5 + j3 + j6) / 2) / std::sqrt(1.0 + K);
          double Signs = SignBL * SignST * c1;
          cplx ct = Signs * coef * env_st.sub[st_id].mat[0];
          int old_pos = p.spos, old_dim = p.sdim;
          zgemm('N', 'C', sys_dim, new_dim, old_dim, ct, at(wi, 0, old_pos), sys_dim,
                env_bl.sub[bl_id].mat.data(), new_dim, cone, at(out.sub[i], 0, new_pos), sys_dim);
          if (up_dif != 0) {
            ct = std::conj(ct);
            zgemm('N', 'N', sys_dim, old_dim, new_dim, ct, at(wi, 0, new_pos), sys_dim,
                  env_bl.sub[bl_id].mat.data(), new_dim, cone, at(out.sub[i], 0, old_pos), sys_dim);
          }
        }
      }
    }
  }
}

// block_vec_block_ndia, get_sys.f90:3131-3569 (live branch)
void block_vec_block_ndia(const Block& sys_bl, char FlagSL, const Block& env_bl, char FlagEL,
                          const Basis& sys_bs, const Basis& env_bs, const Wave& in, Wave& out,
                          cplx coef) {
  (void)FlagSL;
  int up_dif = sys_bl.up_dif, K = sys_bl.down_dif;
  if (up_dif != env_bl.up_dif || K != env_bl.down_dif)
    throw std::runtime_error("Quantum number error in block_vec_block!");
  std::vector<cplx> mat;
  for (int i = 0; i < in.num; ++i) {
    const SubWave& wi = in.sub[i];
    int sys_num_up = wi.sys_num_up, sys_num_down = wi.sys_num_down;
    int env_num_up = wi.env_num_up, env_num_down = wi.env_num_down;
    int x = find_bs(sys_bs, sys_num_up, sys_num_down);
    int y = find_bs(env_bs, env_num_up, env_num_down);
    if (x < 0 || y < 0) continue;
    for (const auto& ps : sys_bs.sub[x].sub) {
      for (const auto& pe : env_bs.sub[y].sub) {
        for (int dd = -K; dd <= K; dd += 2) {
          int sb_id = find_blk3(sys_bl, ps.bl_num_up, ps.bl_num_down, dd);
          int nsb_up = ps.bl_num_up + up_dif, nsb_down = ps.bl_num_down + dd;
          for (int edd = -K; edd <= K; edd += 2) {
            int neb_up = pe.bl_num_up - up_dif, neb_down = pe.bl_num_down - edd;
            int eb_id = find_blk3(env_bl, neb_up, neb_down, edd);
            if (sb_id < 0 || eb_id < 0) continue;
            for (int nS = std::abs(sys_num_down - K); nS <= sys_num_down + K; nS += 2) {
              int nsys_up = sys_num_up + up_dif, nenv_up = env_num_up - up_dif, nenv_down = nS;
              int nsp = -1, nsd = 0, nep = -1, ned = 0;
              int ks = find_bs(sys_bs, nsys_up, nS);
              if (ks >= 0)
                for (const auto& q : sys_bs.sub[ks].sub)
                  if (q.bl_num_up == nsb_up && q.bl_num_down == nsb_down &&
                      q.st_num_down == ps.st_num_down && q.st_num_up == ps.st_num_up) {
                    nsp = q.spos; nsd = q.sdim; break;
                  }
              int ke = find_bs(env_bs, nenv_up, nenv_down);
              if (ke >= 0)
                for (const auto& q : env_bs.sub[ke].sub)
                  if (q.bl_num_up == neb_up && q.bl_num_down == neb_down &&
                      q.st_num_down == pe.st_num_down && q.st_num_up == pe.st_num_up) {
                    nep = q.spos; ned = q.sdim; break;
                  }
              if (nsp < 0 || nep < 0) continue;
              int kk = find_wave(out, nsys_up, nS, nenv_up, nenv_down);
              if (kk < 0) continue;
              double SignEL = 1.0;
              if (FlagEL == 'F') SignEL = sgn_parity(sys_num_up + pe.st_num_up);
              double c1 = w6js(nS, K, sys_num_down, ps.bl_num_down, ps.st_num_down, nsb_down);
              if (c1 == 0.0) continue;
              double c11 = w6js(nS, K, env_num_down, pe.bl_num_down, pe.st_num_down, neb_down);
              if (c11 == 0.0) continue;
              c1 = c1 * c11;
              c1 = c1 * std::sqrt((1.0 + nS) * (1.0 + env_num_down) / (1.0 + K));
              if ((((nsb_down + ps.st_num_down + sys_num_down + K) / 2 +
                    (neb_down + pe.st_num_down + env_num_down + K) / 2) % 2) == 1)
                c1 = -c1;
              cplx ct = SignEL * coef * c1;
              int osp = ps.spos, osd = ps.sdim, oep = pe.spos, oed = pe.sdim;
              mat.assign((size_t)nsd * oed, 0.0);
              zgemm('N', 'N', nsd, oed, osd, cone, sys_bl.sub[sb_id].mat.data(), nsd,
                    at(wi, osp, oep), wi.sys_dim, czero, mat.data(), nsd);
              zgemm('N', 'N', nsd, ned, oed, ct, mat.data(), nsd, env_bl.sub[eb_id].mat.data(),
                    oed, cone, at(out.sub[kk], nsp, nep), out.sub[kk].sys_dim);
              if (up_dif != 0) {
                ct = std::conj(ct);
                const SubWave& wk = in.sub[kk];
                mat.assign((size_t)osd * ned, 0.0);
                zgemm('C', 'N', osd, ned, nsd, cone, sys_bl.sub[sb_id].mat.data(), nsd,
                      at(wk, nsp, nep), wk.sys_dim, czero, mat.data(), osd);
                zgemm('N', 'C', osd, oed, ned, ct, mat.data(), osd, env_bl.sub[eb_id].mat.data(),
                      oed, cone, at(out.sub[i], osp, oep), out.sub[i].sys_dim);
              }
            }
          }
        }
      }
    }
  }
}

// block_vec_site_ndia, get_sys.f90:3970-4345 (live branch)
void block_vec_site_ndia(const Block& sys_bl, char FlagSL, const Block& env_st, char FlagET,
                         const Basis& sys_bs, const Basis& env_bs, const Wave& in, Wave& out,
                         cplx coef) {
  (void)FlagSL;
  int up_dif = sys_bl.up_dif, K = sys_bl.down_dif;
  if (up_dif != env_st.up_dif || K != env_st.down_dif)
    throw std::runtime_error("Quantum number error in block_vec_site!");
  for (int i = 0; i < in.num; ++i) {
    const SubWave& wi = in.sub[i];
    int sys_num_up = wi.sys_num_up, sys_num_down = wi.sys_num_down;
    int env_num_up = wi.env_num_up, env_num_down = wi.env_num_down;
    int x = find_bs(sys_bs, sys_num_up, sys_num_down);
    int y = find_bs(env_bs, env_num_up, env_num_down);
    if (x < 0 || y < 0) continue;
    for (const auto& ps : sys_bs.sub[x].sub) {
      for (const auto& pe : env_bs.sub[y].sub) {
        for (int bdd = -sys_bl.down_dif; bdd <= sys_bl.down_dif; bdd += 2) {
          int nsb_up = ps.bl_num_up + up_dif, nsb_down = ps.bl_num_down + bdd;
          int sb_id = find_blk3(sys_bl, ps.bl_num_up, ps.bl_num_down, bdd);
          for (int sdd = -env_st.down_dif; sdd <= env_st.down_dif; sdd += 2) {
            int nes_up = pe.st_num_up - up_dif, nes_down = pe.st_num_down - sdd;
            int es_id = find_blk3(env_st, nes_up, nes_down, sdd);
            int nsys_up = sys_num_up + up_dif, nenv_up = env_num_up - up_dif;
            if (sb_id < 0 || es_id < 0) continue;
            for (int nS = std::abs(sys_num_down - K); nS <= sys_num_down + K; nS += 2) {
              int nenv_down = nS;
              int nsp = -1, nsd = 0, nep = -1;
              int ks = find_bs(sys_bs, nsys_up, nS);
              if (ks >= 0)
                for (const auto& q : sys_bs.sub[ks].sub)
                  if (q.bl_num_up == nsb_up && q.bl_num_down == nsb_down &&
                      q.st_num_down == ps.st_num_down) {
                    nsp = q.spos; nsd = q.sdim; break;
                  }
              int ke = find_bs(env_bs, nenv_up, nenv_down);
              if (ke >= 0)
                for (const auto& q : env_bs.sub[ke].sub)
                  if (q.st_num_up == nes_up && q.st_num_down == nes_down &&
                      q.bl_num_down == pe.bl_num_down) {
                    nep = q.spos; break;
                  }
              if (nsp < 0 || nep < 0) continue;
              int kk = find_wave(out, nsys_up, nS, nenv_up, nenv_down);
              if (kk < 0) continue;
              double SignET = 1.0;
              if (FlagET == 'F') SignET = sgn_parity(sys_num_up);
              double c1 = w6js(nS, K, sys_num_down, ps.bl_num_down, ps.st_num_down, nsb_down);
              if (c1 == 0.0) continue;
              double c11 = w6js(nS, K, env_num_down, pe.st_num_down, pe.bl_num_down, nes_down);
              if (c11 == 0.0) continue;
              c1 = c1 * c11;
              c1 = c1 * std::sqrt((1.0 + nS) * (1.0 + env_num_down) / (1.0 + K));
              if ((((nsb_down + ps.st_num_down + sys_num_down + K) / 2 +
                    (pe.bl_num_down + pe.st_num_down + nS + K) / 2) % 2) != 0)
                c1 = -c1;
              double Signs = SignET * c1;
              cplx ct = Signs * coef * env_st.sub[es_id].mat[0];
              int osp = ps.spos, osd = ps.sdim, oep = pe.spos, ed = pe.sdim;
              zgemm('N', 'N', nsd, ed, osd, ct, sys_bl.sub[sb_id].mat.data(), nsd,
                    at(wi, osp, oep), wi.sys_dim, cone, at(out.sub[kk], nsp, nep), out.sub[kk].sys_dim);
              if (up_dif != 0) {
                ct = std::conj(ct);
                const SubWave& wk = in.sub[kk];
                zgemm('C', 'N', osd, ed, nsd, ct, sys_bl.sub[sb_id].mat.data(), nsd,
                      at(wk, nsp, nep), wk.sys_dim, cone, at(out.sub[i], osp, oep), out.sub[i].sys_dim);
              }
            }
          }
        }
      }
    }
  }
}

// site_vec_block_ndia, get_sys.f90:4349-4812 (live branch)
void site_vec_block_ndia(const Block& sys_st, char FlagST, const Block& env_bl, char FlagEL,
                         const Basis& sys_bs, const Basis& env_bs, const Wave& in, Wave& out,
                         cplx coef) {
  int up_dif = sys_st.up_dif, K = sys_st.down_dif;
  if (up_dif != env_bl.up_dif || K != env_bl.down_dif)
    throw std::runtime_error("Quantum number error in site_vec_block!");
  for (int i = 0; i < in.num; ++i) {
    const SubWave& wi = in.sub[i];
    int sys_num_up = wi.sys_num_up, sys_num_down = wi.sys_num_down;
    int env_num_up = wi.env_num_up, env_num_down = wi.env_num_down;
    int x = find_bs(sys_bs, sys_num_up, sys_num_down);
    int y = find_bs(env_bs, env_num_up, env_num_down);
    if (x < 0 || y < 0) continue;
    for (const auto& ps : sys_bs.sub[x].sub) {
      for (const auto& pe : env_bs.sub[y].sub) {
        for (int sdd = -sys_st.down_dif; sdd <= sys_st.down_dif; sdd += 2) {
          int nss_up = ps.st_num_up + up_dif, nss_down = ps.st_num_down + sdd;
          int ss_id = find_blk3(sys_st, ps.st_num_up, ps.st_num_down, sdd);
          for (int bdd = -env_bl.down_dif; bdd <= env_bl.down_dif; bdd += 2) {
            int neb_up = pe.bl_num_up - up_dif, neb_down = pe.bl_num_down - bdd;
            int eb_id = find_blk3(env_bl, neb_up, neb_down, bdd);
            int nsys_up = sys_num_up + up_dif, nenv_up = env_num_up - up_dif;
            if (ss_id < 0 || eb_id < 0) continue;
            for (int nS = std::abs(sys_num_down - sys_st.down_dif); nS <= sys_num_down + sys_st.down_dif;
                 nS += 2) {
              int nenv_down = nS;
              int nsp = -1, nep = -1, ned = 0;
              int ks = find_bs(sys_bs, nsys_up, nS);
              if (ks >= 0)
                for (const auto& q : sys_bs.sub[ks].sub)
                  if (q.st_num_up == nss_up && q.st_num_down == nss_down &&
                      q.bl_num_down == ps.bl_num_down && q.bl_num_up == ps.bl_num_up) {
                    nsp = q.spos; break;
                  }
              int ke = find_bs(env_bs, nenv_up, nenv_down);
              if (ke >= 0)
                for (const auto& q : env_bs.sub[ke].sub)
                  if (q.bl_num_up == neb_up && q.bl_num_down == neb_down &&
                      q.st_num_up == pe.st_num_up && q.st_num_down == pe.st_num_down) {
                    nep = q.spos; ned = q.sdim; break;
                  }
              if (nsp < 0 || nep < 0) continue;
              int kk = find_wave(out, nsys_up, nS, nenv_up, nenv_down);
              if (kk < 0) continue;
              double c1 = w6js(nS, K, sys_num_down, ps.st_num_down, ps.bl_num_down, nss_down);
              if (c1 == 0.0) continue;
              double c11 = w6js(nS, K, env_num_down, pe.bl_num_down, pe.st_num_down, neb_down);
              if (c11 == 0.0) continue;
              c1 = c1 * c11;
              c1 = c1 * std::sqrt((1.0 + nS) * (env_num_down + 1.0) / (1.0 + K));
              if ((((neb_down + pe.st_num_down + env_num_down + K) / 2 +
                    (ps.bl_num_down + ps.st_num_down + nS + K) / 2) % 2) != 0)
                c1 = -c1;
              double SignST = 1.0, SignEL = 1.0;
              if (FlagST == 'F') SignST = sgn_parity(ps.bl_num_up);
              if (FlagEL == 'F') SignEL = sgn_parity(sys_num_up + pe.st_num_up);
              double Signs = SignST * SignEL * c1;
              cplx ct = Signs * coef * sys_st.sub[ss_id].mat[0];
              int osp = ps.spos, sd = ps.sdim, oep = pe.spos, oed = pe.sdim;
              zgemm('N', 'N', sd, ned, oed, ct, at(wi, osp, oep), wi.sys_dim,
                    env_bl.sub[eb_id].mat.data(), oed, cone, at(out.sub[kk], nsp, nep), out.sub[kk].sys_dim);
              if (up_dif != 0) {
                ct = std::conj(ct);
                const SubWave& wk = in.sub[kk];
                zgemm('N', 'C', sd, oed, ned, ct, at(wk, nsp, nep), wk.sys_dim,
                      env_bl.sub[eb_id].mat.data(), oed, cone, at(out.sub[i], osp, oep), out.sub[i].sys_dim);
              }
            }
          }
        }
      }
    }
  }
}

// site_vec_site_ndia, get_sys.f90:4816-5204 (live branch)
void site_vec_site_ndia(const Block& sys_st, char FlagST, const Block& env_st, char FlagET,
                        const Basis& sys_bs, const Basis& env_bs, const Wave& in, Wave& out,
                        cplx coef) {
  int up_dif = sys_st.up_dif, K = sys_st.down_dif;
  if (up_dif != env_st.up_dif || K != env_st.down_dif)
    throw std::runtime_error("Quantum number error in site_vec_site!");
  for (int i = 0; i < in.num; ++i) {
    const SubWave& wi = in.sub[i];
    int sys_num_up = wi.sys_num_up, sys_num_down = wi.sys_num_down;
    int env_num_up = wi.env_num_up, env_num_down = wi.env_num_down;
    int x = find_bs(sys_bs, sys_num_up, sys_num_down);
    int y = find_bs(env_bs, env_num_up, env_num_down);
    if (x < 0 || y < 0) continue;
    for (const auto& ps : sys_bs.sub[x].sub) {
      for (const auto& pe : env_bs.sub[y].sub) {
        for (int sd1 = -sys_st.down_dif; sd1 <= sys_st.down_dif; sd1 += 2) {
          int ss_id = find_blk3(sys_st, ps.st_num_up, ps.st_num_down, sd1);
          int nss_up = ps.st_num_up + up_dif, nss_down = ps.st_num_down + sd1;
          for (int sd2 = -env_st.down_dif; sd2 <= env_st.down_dif; sd2 += 2) {
            int nes_up = pe.st_num_up - up_dif, nes_down = pe.st_num_down - sd2;
            int es_id = find_blk3(env_st, nes_up, nes_down, sd2);
            int nsys_up = sys_num_up + up_dif, nenv_up = env_num_up - up_dif;
            if (ss_id < 0 || es_id < 0) continue;
            for (int nS = std::abs(sys_num_down - sys_st.down_dif); nS <= sys_num_down + sys_st.down_dif;
                 nS += 2) {
              int nenv_down = nS;
              int nsp = -1, nep = -1;
              int ks = find_bs(sys_bs, nsys_up, nS);
              if (ks >= 0)
                for (const auto& q : sys_bs.sub[ks].sub)
                  if (q.st_num_up == nss_up && q.st_num_down == nss_down &&
                      q.bl_num_down == ps.bl_num_down) {
                    nsp = q.spos; break;
                  }
              int ke = find_bs(env_bs, nenv_up, nenv_down);
              if (ke >= 0)
                for (const auto& q : env_bs.sub[ke].sub)
                  if (q.st_num_up == nes_up && q.st_num_down == nes_down &&
                      q.bl_num_down == pe.bl_num_down) {
                    nep = q.spos; break;
                  }
              if (nsp < 0 || nep < 0) continue;
              int kk = find_wave(out, nsys_up, nS, nenv_up, nenv_down);
              if (kk < 0) continue;
              double SignST = 1.0, SignET = 1.0;
              if (FlagST == 'F') SignST = sgn_parity(ps.bl_num_up);
              if (FlagET == 'F') SignET = sgn_parity(sys_num_up);
              cplx ct = SignST * SignET * coef;
              double c1 = w6js(nS, K, sys_num_down, ps.st_num_down, ps.bl_num_down, nss_down);
              if (c1 == 0.0) continue;
              double c11 = w6js(nS, K, env_num_down, pe.st_num_down, pe.bl_num_down, nes_down);
              if (c11 == 0.0) continue;
              c1 = c1 * c11;
              c1 = c1 * std::sqrt((1.0 + nS) * (1.0 + env_num_down) / (1.0 + K));
              if ((((pe.bl_num_down + pe.st_num_down + nS + K) / 2 +
                    (ps.bl_num_down + ps.st_num_down + nS + K) / 2) % 2) != 0)
                c1 = -c1;
              cplx cc = ct * c1 * sys_st.sub[ss_id].mat[0] * env_st.sub[es_id].mat[0];
              axpy_rect(out.sub[kk], nsp, nep, wi, ps.spos, pe.spos, ps.sdim, pe.sdim, cc);
              if (up_dif != 0) {
                cc = std::conj(cc);
                axpy_rect(out.sub[i], ps.spos, pe.spos, in.sub[kk], nsp, nep, ps.sdim, pe.sdim, cc);
              }
            }
          }
        }
      }
    }
  }
}

}  // namespace

// hmerge, get_sys.f90:7398-7626
void Oracle::hmerge(Model& sys, Model& env, const Basis&, const Basis&) {
  int dmsite = sys.len + env.len + 2;
  int syssite = sys.len + 1;
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b) L.coup_bs[a][b] = 0;
  auto npos = [&](int latt) { return L.nposi[L.nposi_dm[latt]]; };
  for (int k = 1; k <= L.neibt; ++k) {
    int j = L.NEIB(syssite, k);
    if (npos(j) == 3) L.coup_bs[1][0] = 1;
    if (npos(j) == 1) L.coup_bs[0][0] = 1;
    j = L.NEIB(L.nposi_lat[dmsite], k);
    if (npos(j) == 3) L.coup_bs[1][1] = 1;
    if (npos(j) == 1) L.coup_bs[0][1] = 1;
  }
  for (int ia = 0; ia < 2; ++ia) {
    if (L.coup_bs[0][ia] == 1) {
      block_pass_info(sys.sub[1].elec_up, sys.snc[ia].elec_up);
      block_pass_info(sys.sub[1].spin_sd, sys.snc[ia].spin_sd);
      block_pass_info(sys.sub[1].num_sn, sys.snc[ia].num_sn);
    }
    if (L.coup_bs[1][ia] == 1) {
      block_pass_info(env.sub[1].elec_up, env.snc[ia].elec_up);
      block_pass_info(env.sub[1].elec_down, env.snc[ia].elec_down);
      block_pass_info(env.sub[1].spin_sd, env.snc[ia].spin_sd);
      block_pass_info(env.sub[1].num_sn, env.snc[ia].num_sn);
    }
  }
  for (int ia = 1; ia <= 2; ++ia) {
    int j = sys.len + 1 + (env.len + 1) * (ia - 1);
    int latt = L.nposi_lat[j];
    for (int k1 = 1; k1 <= L.neibt; ++k1) {
      int ib = L.NEIB(latt, k1);
      if (npos(ib) == 3) {
        int ib1 = L.nposi_dm[ib] - sys.len - 1;
        ib1 = L.INB1(ib1, env.len);
        if (L.coup_bs[1][ia - 1] != 0) {
          cplx jd1 = L.JD(k1, latt), jt1 = L.JT(k1, latt), jn1 = L.JN(k1, latt);
          if (jt1 != 0.0) {
            block_add_block_two(env.sub[ib1].elec_up, jt1, env.snc[ia - 1].elec_up);
            block_add_block_two(env.sub[ib1].elec_down, jt1, env.snc[ia - 1].elec_down);
          }
          if (jd1 != 0.0) block_add_block_two(env.sub[ib1].spin_sd, jd1, env.snc[ia - 1].spin_sd);
          if (jn1 != 0.0) block_add_block_two(env.sub[ib1].num_sn, jn1, env.snc[ia - 1].num_sn);
        }
      }
      if (npos(ib) == 1) {
        int ib1 = L.nposi_dm[ib];
        ib1 = L.INB1(ib1, sys.len);
        if (L.coup_bs[0][ia - 1] == 1) {
          cplx jd1 = L.JD(k1, latt), jt1 = L.JT(k1, latt), jn1 = L.JN(k1, latt);
          if (jt1 != 0.0) block_add_block_two(sys.sub[ib1].elec_up, jt1, sys.snc[ia - 1].elec_up);
          if (jd1 != 0.0) block_add_block_two(sys.sub[ib1].spin_sd, jd1, sys.snc[ia - 1].spin_sd);
          if (jn1 != 0.0) block_add_block_two(sys.sub[ib1].num_sn, jn1, sys.snc[ia - 1].num_sn);
        }
      }
    }
  }
  // block-block pivots (get_sys.f90:7498-7533)
  L.coup_bb[0] = L.coup_bb[1] = 0;
  int k11 = 0;
  for (int I = 1; I <= sys.len; ++I) {
    int k1 = 0;
    L.INB(I) = 0;
    for (int k = 1; k <= L.neibt; ++k) {
      int J = L.NEIB(I, k);
      if (npos(J) == 3) k1++;
    }
    L.INB(I) = k1;
    if (L.nleg11[env.len] < L.nleg11[sys.len]) L.INB(I) = 0;
    if (L.INB(I) != 0) k11++;
  }
  L.coup_bb[0] = k11;
  L.INB(sys.len + 1) = 0;
  L.INB(sys.len + 1 + env.len + 1) = 0;
  for (int I = 1; I <= env.len; ++I) {
    int k1 = 0;
    L.INB(I + sys.len + 1) = 0;
    for (int k = 1; k <= L.neibt; ++k) {
      int J = L.NEIB(L.nposi_lat[I + sys.len + 1], k);
      if (npos(J) == 1)
        if (L.INB(J) == 0) k1++;
    }
    L.INB(I + sys.len + 1) = k1;
    if (L.INB(I + sys.len + 1) != 0) k11++;
  }
  L.coup_bb[1] = k11 - L.coup_bb[0];
  if ((int)env.sub_s.size() < L.num_site + 1) env.sub_s.resize(L.num_site + 1);
  if ((int)sys.sub_s.size() < L.num_site + 1) sys.sub_s.resize(L.num_site + 1);
  for (int i = 1; i <= L.coup_bb[0]; ++i) {
    block_pass_info(env.sub[1].elec_up, env.sub_s[i].elec_up);
    block_pass_info(env.sub[1].elec_down, env.sub_s[i].elec_down);
    block_pass_info(env.sub[1].spin_sd, env.sub_s[i].spin_sd);
    block_pass_info(env.sub[1].num_sn, env.sub_s[i].num_sn);
  }
  for (int i = 1; i <= L.coup_bb[1]; ++i) {
    block_pass_info(sys.sub[1].elec_up, sys.sub_s[i].elec_up);
    block_pass_info(sys.sub[1].spin_sd, sys.sub_s[i].spin_sd);
    block_pass_info(sys.sub[1].num_sn, sys.sub_s[i].num_sn);
  }
  int jc = 0;
  for (int I = 1; I <= sys.len + env.len + 1; ++I) {
    if (L.INB(I) == 0) continue;
    int Ia = L.nposi_lat[I];
    jc++;
    for (int k1 = 1; k1 <= L.neibt; ++k1) {
      int Ib = L.NEIB(Ia, k1);
      if (npos(Ib) == 3 && I <= sys.len) {
        int Ib1 = L.INB1(L.nposi_dm[Ib] - sys.len - 1, env.len);
        cplx jt1 = L.JT(k1, Ia), jd1 = L.JD(k1, Ia), jn1 = L.JN(k1, Ia);
        if (jt1 != 0.0) {
          block_add_block_two(env.sub[Ib1].elec_up, jt1, env.sub_s[jc].elec_up);
          block_add_block_two(env.sub[Ib1].elec_down, jt1, env.sub_s[jc].elec_down);
        }
        if (jd1 != 0.0) block_add_block_two(env.sub[Ib1].spin_sd, jd1, env.sub_s[jc].spin_sd);
        if (jn1 != 0.0) block_add_block_two(env.sub[Ib1].num_sn, jn1, env.sub_s[jc].num_sn);
      }
      if (npos(Ib) == 1 && I > sys.len + 1) {
        if (L.INB(L.nposi_dm[Ib]) == 0) {
          int Ib1 = L.INB1(Ib, sys.len);
          int jc1 = jc - L.coup_bb[0];
          cplx jt1 = L.JT(k1, Ia), jd1 = L.JD(k1, Ia), jn1 = L.JN(k1, Ia);
          if (jt1 != 0.0) block_add_block_two(sys.sub[Ib1].elec_up, jt1, sys.sub_s[jc1].elec_up);
          if (jd1 != 0.0) block_add_block_two(sys.sub[Ib1].spin_sd, jd1, sys.sub_s[jc1].spin_sd);
          if (jn1 != 0.0) block_add_block_two(sys.sub[Ib1].num_sn, jn1, sys.sub_s[jc1].num_sn);
        }
      }
    }
  }
}

// model_wave, get_sys.f90:6915-7068 (add_op=1, t-J branch, lring=0)
void Oracle::model_wave(Model& sys, Model& env, const Basis& sys_bs, const Basis& env_bs,
                        const Wave& in, Wave& out) {
  auto t0 = std::chrono::steady_clock::now();
  double f0 = g_gemm_flops;
  for (auto& s : out.sub) std::fill(s.vec.begin(), s.vec.end(), czero);
  block_vec_dia(sys.ham, sys_bs, in, out, cone);
  vec_block_dia(env.ham, env_bs, in, out, cone);
  int is = L.nposi_lat[sys.len + 1];
  int js = L.nposi_lat[sys.len + env.len + 2];
  int ii = L.NEIBA(is, js);
  Block tmp_bl, tmp_bl1;
  if (ii != 0) {
    cplx jd1 = L.JD(ii, is), coefx = L.JT(ii, is), jn1 = L.JN(ii, is);
    if (coefx != 0.0) {
      block_transfer_trans(st_elec_down, tmp_bl);
      site_vec_site_ndia(st_elec_up, 'F', tmp_bl, 'F', sys_bs, env_bs, in, out, coefx);
    }
    if (jd1 != 0.0) site_vec_site_ndia(st_sd, 'B', st_sd, 'B', sys_bs, env_bs, in, out, jd1);
    if (jn1 != 0.0) site_vec_site_dia(num_elec, num_elec, sys_bs, env_bs, in, out, jn1);
  }
  if (L.coup_bs[0][0] == 1) {
    block_transfer_trans(st_elec_down, tmp_bl);
    block_site_vec_ndia(sys.snc[0].elec_up, 'F', tmp_bl, 'F', sys_bs, in, out, cone);
    block_site_vec_ndia(sys.snc[0].spin_sd, 'B', st_sd, 'B', sys_bs, in, out, cone);
    block_site_vec_dia(sys.snc[0].num_sn, num_elec, sys_bs, in, out, cone);
  }
  if (L.coup_bs[0][1] == 1) {
    block_transfer_trans(st_elec_down, tmp_bl);
    block_vec_site_ndia(sys.snc[1].elec_up, 'F', tmp_bl, 'F', sys_bs, env_bs, in, out, cone);
    block_vec_site_ndia(sys.snc[1].spin_sd, 'B', st_sd, 'B', sys_bs, env_bs, in, out, cone);
    block_vec_site_dia(sys.snc[1].num_sn, num_elec, sys_bs, env_bs, in, out, cone);
  }
  if (L.coup_bs[1][0] == 1) {
    block_transfer_trans(env.snc[0].elec_down, tmp_bl1);
    site_vec_block_ndia(st_elec_up, 'F', tmp_bl1, 'F', sys_bs, env_bs, in, out, cone);
    block_transfer_trans(env.snc[0].spin_sd, tmp_bl);
    site_vec_block_ndia(st_sd, 'B', tmp_bl, 'B', sys_bs, env_bs, in, out, cone);
    site_vec_block_dia(num_elec, env.snc[0].num_sn, sys_bs, env_bs, in, out, cone);
  }
  if (L.coup_bs[1][1] == 1) {
    block_transfer_trans(st_elec_down, tmp_bl);
    vec_block_site_ndia(env.snc[1].elec_up, 'F', tmp_bl, 'F', env_bs, in, out, cone);
    vec_block_site_ndia(env.snc[1].spin_sd, 'B', st_sd, 'B', env_bs, in, out, cone);
    vec_block_site_dia(env.snc[1].num_sn, num_elec, env_bs, in, out, cone);
  }
  int jc = 0;
  for (int i = 1; i <= sys.len + 1 + env.len; ++i) {
    if (L.INB(i) == 0) continue;
    jc++;
    if (i <= sys.len) {
      int i1 = L.INB1(i, sys.len);
      block_transfer_trans(env.sub_s[jc].elec_down, tmp_bl1);
      block_vec_block_ndia(sys.sub[i1].elec_up, 'F', tmp_bl1, 'F', sys_bs, env_bs, in, out, cone);
      block_transfer_trans(env.sub_s[jc].spin_sd, tmp_bl);
      block_vec_block_ndia(sys.sub[i1].spin_sd, 'B', tmp_bl, 'B', sys_bs, env_bs, in, out, cone);
      block_vec_block_dia(sys.sub[i1].num_sn, env.sub_s[jc].num_sn, sys_bs, env_bs, in, out, cone);
    } else {
      int i1 = L.INB1(i - sys.len - 1, env.len);
      int jc1 = jc - L.coup_bb[0];
      block_transfer_trans(env.sub[i1].elec_down, tmp_bl1);
      block_vec_block_ndia(sys.sub_s[jc1].elec_up, 'F', tmp_bl1, 'F', sys_bs, env_bs, in, out, cone);
      block_transfer_trans(env.sub[i1].spin_sd, tmp_bl);
      block_vec_block_ndia(sys.sub_s[jc1].spin_sd, 'B', tmp_bl, 'B', sys_bs, env_bs, in, out, cone);
      block_vec_block_dia(sys.sub_s[jc1].num_sn, env.sub[i1].num_sn, sys_bs, env_bs, in, out, cone);
    }
  }
  hpsi_calls++;
  hpsi_flops += g_gemm_flops - f0;
  hpsi_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace orc
