// Oracle DMRG: Lanczos (eigen.f90), density matrix + truncation (den_mat.f90),
// operator enlargement and U^dagger O U (block.f90:2495-3683, get_sys.f90:4-1055),
// wave transformations and sweep drivers (dmrg_sub.f90:974-1789, main.f90:114-209).
// TEST INFRASTRUCTURE ONLY (see oracle.hpp).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <stdexcept>

#include "oracle.hpp"

extern "C" {
void scipy_zheev_(const char*, const char*, const int*, void*, const int*, double*, void*,
                  const int*, double*, int*);
void scipy_dstev_(const char*, const int*, double*, double*, double*, const int*, double*, int*);
}

namespace orc {

namespace {
const cplx cone(1.0, 0.0), czero(0.0, 0.0);
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
inline double pm1(int e) { return ((e % 2) + 2) % 2 == 0 ? 1.0 : -1.0; }

// dstev wrapper; d/e overwritten; z (n x n) when jobz=='V'
void dstev(char jobz, int n, std::vector<double>& d, std::vector<double>& e, std::vector<double>* z) {
  if (n <= 0) return;
  std::vector<double> work(std::max(1, 2 * n - 2));
  std::vector<double> zz;
  int ldz = n, info = 0;
  if (jobz == 'V') zz.assign((size_t)n * n, 0.0);
  else zz.assign(1, 0.0);
  scipy_dstev_(&jobz, &n, d.data(), e.data(), zz.data(), &ldz, work.data(), &info);
  if (z) *z = zz;
}

// update_block_dia, block.f90:2495-2548
void update_block_dia(const Block& block, const Basis& basis, Block& nb) {
  nb = Block();
  nb.len = basis.len;
  nb.num = basis.num;
  nb.dim = basis.dim;
  nb.sub.assign(nb.num, SubBlock());
  for (int i = 0; i < nb.num; ++i) {
    SubBlock& s = nb.sub[i];
    s.num_up = basis.sub[i].new_num_up;
    s.num_down = basis.sub[i].new_num_down;
    s.down_dif = 0;
    s.row_dim = s.sdim = basis.sub[i].dim;
    s.mat.assign((size_t)s.sdim * s.sdim, 0.0);
  }
  for (int k = 0; k < nb.num; ++k)
    for (const auto& p : basis.sub[k].sub) {
      for (int i = 0; i < block.num; ++i) {
        const SubBlock& b = block.sub[i];
        if (b.num_up == p.bl_num_up && b.num_down == p.bl_num_down) {
          double c1 = std::sqrt((1.0 + nb.sub[k].num_down) / (1.0 + b.num_down));
          for (int c = 0; c < p.sdim; ++c)
            for (int r = 0; r < p.sdim; ++r) nb.sub[k].at(p.spos + r, p.spos + c) += b.at(r, c) * c1;
          break;
        }
      }
    }
}

// update_site_dia, block.f90:2554-2615
void update_site_dia(const Block& site, const Basis& basis, Block& ns) {
  ns = Block();
  ns.len = basis.len;
  ns.num = basis.num;
  ns.dim = basis.dim;
  ns.sub.assign(ns.num, SubBlock());
  for (int i = 0; i < ns.num; ++i) {
    SubBlock& s = ns.sub[i];
    s.num_up = basis.sub[i].new_num_up;
    s.num_down = basis.sub[i].new_num_down;
    s.down_dif = 0;
    s.row_dim = s.sdim = basis.sub[i].dim;
    s.mat.assign((size_t)s.sdim * s.sdim, 0.0);
  }
  for (int k = 0; k < ns.num; ++k)
    for (const auto& p : basis.sub[k].sub) {
      for (int i = 0; i < site.num; ++i) {
        const SubBlock& st = site.sub[i];
        if (st.num_up == p.st_num_up && st.num_down == p.st_num_down) {
          double c1 = std::sqrt((1.0 + ns.sub[k].num_down) / (1.0 + st.num_down));
          for (int y = 0; y < p.sdim; ++y) ns.sub[k].at(p.spos + y, p.spos + y) += st.mat[0] * c1;
          break;
        }
      }
    }
}

// sub-block structure shared by update_*_ndia_* (block.f90:2655-2712)
void ndia_structure(const Basis& basis, int up_dif, int K, Block& nb) {
  nb.sub.clear();
  nb.dim = 0;
  for (int x = 0; x < basis.num; ++x)
    for (int dd = -K; dd <= K; dd += 2) {
      int lu = basis.sub[x].new_num_up + up_dif, ld = basis.sub[x].new_num_down + dd;
      int y = find_bs(basis, lu, ld);
      if (y < 0) continue;
      SubBlock s;
      s.num_up = basis.sub[x].new_num_up;
      s.num_down = basis.sub[x].new_num_down;
      s.down_dif = dd;
      s.row_dim = basis.sub[y].dim;
      s.sdim = basis.sub[x].dim;
      s.mat.assign((size_t)s.row_dim * s.sdim, 0.0);
      nb.dim += s.sdim;
      nb.sub.push_back(std::move(s));
    }
  nb.num = (int)nb.sub.size();
}

// update_block_ndia_sys (block.f90:2624-2820) and _env (block.f90:2828-3036)
void update_block_ndia(const Block& block, const Basis& basis, Block& nb, char FlagSign, bool env) {
  nb = Block();
  nb.len = basis.len;
  nb.up_dif = block.up_dif;
  nb.down_dif = block.down_dif;
  int up_dif = block.up_dif, K = block.down_dif;
  ndia_structure(basis, up_dif, K, nb);
  for (int i = 0; i < nb.num; ++i) {
    SubBlock& o = nb.sub[i];
    int rhs_id = find_bs(basis, o.num_up, o.num_down);
    int lhs_id = find_bs(basis, o.num_up + up_dif, o.num_down + o.down_dif);
    if (rhs_id < 0 || lhs_id < 0) continue;
    int lhs_num_down = o.num_down + o.down_dif, rhs_num_down = o.num_down;
    for (const auto& p : basis.sub[rhs_id].sub) {
      for (int sdd = -K; sdd <= K; sdd += 2) {
        int bid = find_blk3(block, p.bl_num_up, p.bl_num_down, sdd);
        if (bid < 0) continue;
        int lsu = p.bl_num_up + up_dif, lsd = p.bl_num_down + sdd;
        const SubBasisMap* q = nullptr;
        for (const auto& qq : basis.sub[lhs_id].sub)
          if (qq.bl_num_up == lsu && qq.bl_num_down == lsd && qq.st_num_down == p.st_num_down) {
            q = &qq;
            break;
          }
        if (!q) continue;
        double Signs = 1.0;
        if (env && FlagSign == 'F') Signs = (p.st_num_up % 2 == 0) ? 1.0 : -1.0;
        int j1 = lhs_num_down, j2 = K, j3 = rhs_num_down, j4 = p.bl_num_down, j5 = p.st_num_down, j6 = lsd;
        double coef = w6js(j1, j2, j3, j4, j5, j6);
        if (!env) {
          coef = coef * std::sqrt((1.0 + j1) * (1.0 + j3));
          coef = coef * pm1((j6 + j5 + j3 + j2) / 2);
        } else {
          coef = coef * pm1((j6 + j5 + j3 + j2) / 2) * std::sqrt((1.0 + j1) * (1.0 + j3));
        }
        if (coef == 0.0) continue;
        coef = coef * Signs;
        const SubBlock& b = block.sub[bid];
        for (int c = 0; c < p.sdim; ++c)
          for (int r = 0; r < q->sdim; ++r) o.at(q->spos + r, p.spos + c) += coef * b.at(r, c);
      }
    }
  }
}

// update_site_ndia_sys (block.f90:3047-3260) and _env (block.f90:3269-3459)
void update_site_ndia(const Block& site, const Basis& basis, Block& ns, char FlagSign, bool env) {
  ns = Block();
  ns.len = basis.len;
  ns.up_dif = site.up_dif;
  ns.down_dif = site.down_dif;
  int up_dif = site.up_dif, K = site.down_dif;
  ndia_structure(basis, up_dif, K, ns);
  for (int i = 0; i < ns.num; ++i) {
    SubBlock& o = ns.sub[i];
    int rhs_id = find_bs(basis, o.num_up, o.num_down);
    int lhs_id = find_bs(basis, o.num_up + up_dif, o.num_down + o.down_dif);
    if (rhs_id < 0 || lhs_id < 0) continue;
    int lhs_num_down = o.num_down + o.down_dif, rhs_num_down = o.num_down;
    for (const auto& p : basis.sub[rhs_id].sub) {
      for (int sdd = -K; sdd <= K; sdd += 2) {
        int sid = find_blk3(site, p.st_num_up, p.st_num_down, sdd);
        if (sid < 0) continue;
        int lsu = p.st_num_up + up_dif, lsd = p.st_num_down + sdd;
        const SubBasisMap* q = nullptr;
        for (const auto& qq : basis.sub[lhs_id].sub)
          if (qq.st_num_up == lsu && qq.st_num_down == lsd && qq.bl_num_down == p.bl_num_down) {
            q = &qq;
            break;
          }
        if (!q) continue;
        double Signs = 1.0;
        if (!env && FlagSign == 'F') Signs = (p.bl_num_up % 2 == 0) ? 1.0 : -1.0;
        int j1 = lhs_num_down, j2 = K, j3 = rhs_num_down, j4 = p.st_num_down, j5 = p.bl_num_down, j6 = lsd;
        double coef = w6js(j1, j2, j3, j4, j5, j6);
        if (!env) coef = coef * pm1((j5 + j4 + j1 + j2) / 2) * std::sqrt((1.0 + j1) * (1.0 + j3));
        else coef = coef * std::sqrt((1.0 + j1) * (1.0 + j3)) * pm1((j5 + j4 + j1 + j2) / 2);
        if (coef == 0.0) continue;
        coef = coef * Signs;
        cplx v = site.sub[sid].mat[0];
        for (int y = 0; y < p.sdim; ++y) o.at(q->spos + y, p.spos + y) += coef * v;
      }
    }
  }
}

// Get_hamiltonian_dia, get_sys.f90:776-854 (Flag1=Flag2='N', FlagConjg=.false.)
void hamiltonian_dia(const Block& o1, const Block& o2, cplx coef, Block& ham) {
  std::vector<cplx> mat;
  for (int i = 0; i < ham.num; ++i) {
    SubBlock& h = ham.sub[i];
    int a = find_blk(o1, h.num_up, h.num_down);
    int b = find_blk(o2, h.num_up, h.num_down);
    if (a < 0 || b < 0) continue;
    int sdim = h.sdim;
    mat.assign((size_t)sdim * sdim, 0.0);
    cplx c1 = coef / std::sqrt(1.0 + h.num_down);
    zgemm('N', 'N', sdim, sdim, sdim, c1, o1.sub[a].mat.data(), sdim, o2.sub[b].mat.data(), sdim,
          czero, mat.data(), sdim);
    for (size_t e = 0; e < mat.size(); ++e) h.mat[e] += mat[e];
  }
}

// Get_hamiltonian_ndia, get_sys.f90:865-1055
void hamiltonian_ndia(const Block& block, const Block& site, const Basis& basis, cplx coef,
                      Block& ham, char FlagSign, char Flags) {
  int up_dif = block.up_dif, K = block.down_dif;
  for (int i = 0; i < ham.num; ++i) {
    SubBlock& h = ham.sub[i];
    int rhs_id = find_bs(basis, h.num_up, h.num_down);
    int lhs_id = find_bs(basis, h.num_up, h.num_down + h.down_dif);
    if (rhs_id < 0 || lhs_id < 0) continue;
    int rhs_num_down = h.num_down;
    for (const auto& p : basis.sub[rhs_id].sub) {
      for (int sdd = -K; sdd <= K; sdd += 2) {
        int bid = find_blk3(block, p.bl_num_up, p.bl_num_down, sdd);
        if (bid < 0) continue;
        int lsu = p.bl_num_up + up_dif, lsd = p.bl_num_down + sdd;
        for (int nsd = std::abs(p.st_num_down - site.down_dif); nsd <= p.st_num_down + site.down_dif;
             nsd += 2) {
          int st_down_dif = p.st_num_down - nsd;
          int nsu = p.st_num_up - site.up_dif;
          int sid = find_blk3(site, nsu, nsd, st_down_dif);
          const SubBasisMap* q = nullptr;
          for (const auto& qq : basis.sub[lhs_id].sub)
            if (qq.bl_num_up == lsu && qq.bl_num_down == lsd && qq.st_num_down == nsd) {
              q = &qq;
              break;
            }
          if (!q || sid < 0) continue;
          int j1 = lsd, j2 = p.bl_num_down, j3 = K, j4 = p.st_num_down, j5 = nsd, j6 = rhs_num_down;
          double c11 = w6js(j1, j2, j3, j4, j5, j6);
          c11 = c11 * std::sqrt((1.0 + j6) / (1.0 + j3)) * pm1((j2 + j5 + j3 + j6) / 2) *
                site.sub[sid].mat[0].real();
          cplx smat = site.sub[sid].mat[0];
          double Sign = 1.0;
          if (Flags == 'S') {
            if (FlagSign == 'F' && (p.bl_num_up % 2) == 1) Sign = -1.0;
          } else {
            if (FlagSign == 'F' && (p.st_num_up % 2) == 0) Sign = -1.0;
          }
          (void)smat;
          if (c11 == 0.0) continue;
          cplx c1 = c11 * coef * Sign;
          const SubBlock& b = block.sub[bid];
          int ld = q->sdim, rd = p.sdim;
          for (int c = 0; c < rd; ++c)
            for (int r = 0; r < ld; ++r) h.at(q->spos + r, p.spos + c) += c1 * b.at(r, c);
          if (site.up_dif != 0) {
            cplx cc = std::conj(c1);
            for (int c = 0; c < ld; ++c)
              for (int r = 0; r < rd; ++r) h.at(p.spos + r, q->spos + c) += cc * std::conj(b.at(c, r));
          }
        }
      }
    }
  }
}

// update_trun_dia, block.f90:3465-3527
void update_trun_dia(const Block& ori, Block& eff, const Block& trun) {
  eff = Block();
  eff.len = ori.len;
  eff.num = trun.num;
  eff.dim = trun.dim;
  eff.up_dif = ori.up_dif;
  eff.down_dif = ori.down_dif;
  eff.sub.assign(eff.num, SubBlock());
  std::vector<cplx> mid;
  for (int i = 0; i < eff.num; ++i) {
    SubBlock& e = eff.sub[i];
    e.num_up = trun.sub[i].num_up;
    e.num_down = trun.sub[i].num_down;
    e.down_dif = 0;
    e.row_dim = e.sdim = trun.sub[i].sdim;
    e.mat.assign((size_t)e.sdim * e.sdim, 0.0);
  }
  for (int i = 0; i < eff.num; ++i) {
    SubBlock& e = eff.sub[i];
    int x = find_blk(ori, e.num_up, e.num_down);
    if (x < 0) continue;
    int od = ori.sub[x].row_dim, ed = e.sdim;
    mid.assign((size_t)od * ed, 0.0);
    zgemm('N', 'N', od, ed, od, cone, ori.sub[x].mat.data(), od, trun.sub[i].mat.data(), od, czero,
          mid.data(), od);
    zgemm('C', 'N', ed, ed, od, cone, trun.sub[i].mat.data(), od, mid.data(), od, czero,
          e.mat.data(), ed);
  }
}

// update_trun_ndia, block.f90:3535-3683
void update_trun_ndia(const Block& ori, Block& eff, const Block& trun) {
  eff = Block();
  eff.len = ori.len;
  eff.up_dif = ori.up_dif;
  eff.down_dif = ori.down_dif;
  int up_dif = ori.up_dif, K = ori.down_dif;
  for (int x = 0; x < trun.num; ++x)
    for (int dd = -K; dd <= K; dd += 2) {
      int y = find_blk(trun, trun.sub[x].num_up + up_dif, trun.sub[x].num_down + dd);
      if (y < 0) continue;
      SubBlock s;
      s.num_up = trun.sub[x].num_up;
      s.num_down = trun.sub[x].num_down;
      s.down_dif = dd;
      s.row_dim = trun.sub[y].sdim;
      s.sdim = trun.sub[x].sdim;
      s.mat.assign((size_t)s.row_dim * s.sdim, 0.0);
      eff.dim += s.sdim;
      eff.sub.push_back(std::move(s));
    }
  eff.num = (int)eff.sub.size();
  std::vector<cplx> mid;
  for (int i = 0; i < eff.num; ++i) {
    SubBlock& e = eff.sub[i];
    int rhs_id = find_blk(trun, e.num_up, e.num_down);
    int lhs_id = find_blk(trun, e.num_up + up_dif, e.num_down + e.down_dif);
    int ori_id = find_blk3(ori, e.num_up, e.num_down, e.down_dif);
    if (rhs_id < 0 || lhs_id < 0 || ori_id < 0) continue;
    int orow = ori.sub[ori_id].row_dim, ocol = ori.sub[ori_id].sdim;
    int rd = trun.sub[rhs_id].sdim, ld = trun.sub[lhs_id].sdim;
    mid.assign((size_t)orow * rd, 0.0);
    zgemm('N', 'N', orow, rd, ocol, cone, ori.sub[ori_id].mat.data(), orow,
          trun.sub[rhs_id].mat.data(), ocol, czero, mid.data(), orow);
    zgemm('C', 'N', ld, rd, orow, cone, trun.sub[lhs_id].mat.data(), orow, mid.data(), orow, czero,
          e.mat.data(), ld);
  }
}

// Density-matrix eigenvalues below this are rounding noise (rho has unit trace).
const double kZeroWeight = 1e-13;

// Canonical orthonormal basis of the complement of span(Q) (d x s): Gram-Schmidt
// of the unit vectors e_0, e_1, ... in order, keeping candidates whose projected
// norm exceeds a threshold.  Depends on Q only through its projector, so every
// eigensolver yields the same kept zero-weight states.  Not in the reference
// (den_mat.f90:395-396 keeps whatever null vectors its LAPACK returns).
void null_completion(int d, int s, const cplx* Q, int m, cplx* N) {
  int got = 0;
  std::vector<cplx> v(d);
  for (double thr : {0.5, 0.1, 1e-3}) {
    for (int j = 0; j < d && got < m; ++j) {
      std::fill(v.begin(), v.end(), cplx(0.0));
      v[j] = 1.0;
      for (int pass = 0; pass < 2; ++pass) {
        for (int q = 0; q < s; ++q) {
          cplx dot = 0.0;
          for (int r = 0; r < d; ++r) dot += std::conj(Q[(size_t)q * d + r]) * v[r];
          for (int r = 0; r < d; ++r) v[r] -= dot * Q[(size_t)q * d + r];
        }
        for (int q = 0; q < got; ++q) {
          cplx dot = 0.0;
          for (int r = 0; r < d; ++r) dot += std::conj(N[(size_t)q * d + r]) * v[r];
          for (int r = 0; r < d; ++r) v[r] -= dot * N[(size_t)q * d + r];
        }
      }
      double nrm = 0.0;
      for (int r = 0; r < d; ++r) nrm += std::norm(v[r]);
      nrm = std::sqrt(nrm);
      if (nrm <= thr) continue;
      for (int r = 0; r < d; ++r) N[(size_t)got * d + r] = v[r] / nrm;
      got++;
    }
    if (got >= m) return;
  }
  throw std::runtime_error("null_completion: complement too small");
}

// Canonical phase of every eigenvector column: multiply by conj(z)/|z| with
// z = sum_r w_r u_r, w_r = 1/(1 + r/10).  Eigensolvers return eigenvectors with
// arbitrary phases (the reference inherits MKL's); fixing them makes the
// renormalised operators, and therefore a random start vector's meaning,
// independent of the eigensolver.  Not in the reference.
void phase_fix(int rows, int cols, cplx* U) {
  for (int c = 0; c < cols; ++c) {
    cplx* u = U + (size_t)c * rows;
    cplx z = 0.0;
    for (int r = 0; r < rows; ++r) z += u[r] * (1.0 / (1.0 + 0.1 * r));
    double a = std::abs(z);
    if (a < 1e-10) continue;
    cplx f = std::conj(z) / a;
    for (int r = 0; r < rows; ++r) u[r] *= f;
  }
}

// QuickSort_Double, block.f90:2398-2444 (descending, carries an index array)
void quicksort_double(std::vector<double>& arr, std::vector<int>& idx, int lower, int upper) {
  int i = lower, j = upper;
  int index = (int)((lower + upper) / 2.0);
  double mn = arr[index];
  while (i <= j) {
    while (arr[i] > mn) i++;
    while (arr[j] < mn) j--;
    if (i <= j) {
      std::swap(arr[i], arr[j]);
      std::swap(idx[i], idx[j]);
      i++;
      j--;
    }
  }
  if (lower < j) quicksort_double(arr, idx, lower, j);
  if (i < upper) quicksort_double(arr, idx, i, upper);
}

}  // namespace

// ---- Lanczos (eigen.f90:4-199), levels=1 ------------------------------------------
void Oracle::lanczos_memo_new(Model& sys, Model& env, const Basis& sys_bs, const Basis& env_bs,
                              const Super& super, Wave& eigvec, int* iters, double* e0) {
  const int loop_out = 4, loop_in = 100;
  int iter_out = 0, last = 1;
  double lastmin = 1024.0, ritzmin = 0.0;
  std::vector<double> alpha1(loop_in + 1), beta1(loop_in + 1);
  std::vector<Wave> t(loop_in + 2);
  bool done = false;
  while (iter_out <= loop_out && !done) {
    iter_out++;
    last = 1;
    std::fill(alpha1.begin(), alpha1.end(), 0.0);
    std::fill(beta1.begin(), beta1.end(), 0.0);
    ritzmin = lastmin;
    t[last] = eigvec;
    wave_normalize(t[last]);
    allocate_wave(super, t[last + 1]);
    hmerge(sys, env, sys_bs, env_bs);
    model_wave(sys, env, sys_bs, env_bs, t[last], t[last + 1]);
    alpha1[last] = wave_product(t[last], t[last + 1]);
    ritzmin = alpha1[last];
    bool converged = false;
    while (last < loop_in) {
      Wave& w = t[last + 1];
      for (int i = 0; i < w.num; ++i) {
        auto& v = w.sub[i].vec;
        const auto& a = t[last].sub[i].vec;
        if (last < 2) {
          for (size_t e = 0; e < v.size(); ++e) v[e] = v[e] - alpha1[last] * a[e];
        } else {
          const auto& b = t[last - 1].sub[i].vec;
          for (size_t e = 0; e < v.size(); ++e) v[e] = v[e] - alpha1[last] * a[e] - beta1[last - 1] * b[e];
        }
      }
      beta1[last] = wave_norm(w);
      if (std::fabs(beta1[last]) <= lanzero) {
        converged = true;
        break;
      }
      wave_normalize(w);
      // Gram_Schmidt_process (block.f90:1251-1289) against t[1..last]
      {
        std::vector<double> uv(last + 1), uu(last + 1);
        for (int j = 1; j <= last; ++j) {
          uv[j] = wave_product(t[j], w);
          uu[j] = wave_product(t[j], t[j]);
        }
        Wave tmp = w;
        for (auto& s : tmp.sub) std::fill(s.vec.begin(), s.vec.end(), czero);
        for (int j = 1; j <= last; ++j)
          for (int i = 0; i < tmp.num; ++i) {
            auto& tv = tmp.sub[i].vec;
            const auto& pv = t[j].sub[i].vec;
            double c = uv[j] / uu[j];
            for (size_t e = 0; e < tv.size(); ++e) tv[e] = tv[e] + c * pv[e];
          }
        for (int i = 0; i < w.num; ++i)
          for (size_t e = 0; e < w.sub[i].vec.size(); ++e) w.sub[i].vec[e] = w.sub[i].vec[e] - tmp.sub[i].vec[e];
        wave_normalize(w);
      }
      last++;
      allocate_wave(super, t[last + 1]);
      model_wave(sys, env, sys_bs, env_bs, t[last], t[last + 1]);
      alpha1[last] = wave_product(t[last], t[last + 1]);
      std::vector<double> d(alpha1.begin() + 1, alpha1.begin() + 1 + last);
      std::vector<double> e(beta1.begin() + 1, beta1.begin() + 1 + last);
      dstev('N', last, d, e, nullptr);
      if (std::fabs(d[0] - ritzmin) <= lanzero || (last == loop_in && iter_out == loop_out)) {
        ritzmin = d[0];
        lastmin = ritzmin;
        converged = true;
        break;
      }
      ritzmin = d[0];
      lastmin = ritzmin;
    }
    if (converged) {
      done = true;
      break;
    }
    // restart: eigen.f90:114-134
    std::vector<double> d(alpha1.begin() + 1, alpha1.begin() + 1 + last);
    std::vector<double> e(beta1.begin() + 1, beta1.begin() + 1 + last);
    std::vector<double> z;
    dstev('V', last, d, e, &z);
    ritzmin = d[0];
    lastmin = ritzmin;
    for (auto& s : eigvec.sub) std::fill(s.vec.begin(), s.vec.end(), czero);
    for (int i = 1; i <= last; ++i)
      for (int x = 0; x < eigvec.num; ++x) {
        auto& ev = eigvec.sub[x].vec;
        const auto& tv = t[i].sub[x].vec;
        for (size_t q = 0; q < ev.size(); ++q) ev[q] = ev[q] + z[(size_t)0 * last + (i - 1)] * tv[q];
      }
    wave_normalize(eigvec);
  }
  // label 411: eigen.f90:137-160
  std::vector<double> d(alpha1.begin() + 1, alpha1.begin() + 1 + last);
  std::vector<double> e(beta1.begin() + 1, beta1.begin() + 1 + last);
  std::vector<double> z;
  dstev('V', last, d, e, &z);
  ritzmin = d[0];
  for (auto& s : eigvec.sub) std::fill(s.vec.begin(), s.vec.end(), czero);
  for (int i = 1; i <= last; ++i)
    for (int x = 0; x < eigvec.num; ++x) {
      auto& ev = eigvec.sub[x].vec;
      const auto& tv = t[i].sub[x].vec;
      double zi = z[(size_t)(i - 1)];
      for (size_t q = 0; q < ev.size(); ++q) ev[q] = ev[q] + zi * tv[q];
    }
  wave_normalize(eigvec);
  *iters = (iter_out - 1) * loop_in + last;
  *e0 = ritzmin;
}

// ---- density matrix (den_mat.f90:4-183), levels=1 ---------------------------------
void Oracle::density_matrix_sys(const Wave& wave, Block& den) {
  Wave w = wave;
  wave_normalize(w);   // Get_density_matrix_sys_new, den_mat.f90:118-124
  den = Block();
  den.len = w.sys_len;
  den.num = w.num;
  den.sub.assign(den.num, SubBlock());
  for (int i = 0; i < w.num; ++i) {
    SubBlock& s = den.sub[i];
    s.num_up = w.sub[i].sys_num_up;
    s.num_down = w.sub[i].sys_num_down;
    s.down_dif = 0;
    s.row_dim = s.sdim = w.sub[i].sys_dim;
    den.dim += s.sdim;
    int sd = w.sub[i].sys_dim, ed = w.sub[i].env_dim;
    s.mat.assign((size_t)sd * sd, 0.0);
    zgemm('N', 'C', sd, sd, ed, cone, w.sub[i].vec.data(), sd, w.sub[i].vec.data(), sd, czero,
          s.mat.data(), sd);
  }
}

void Oracle::density_matrix_env(const Wave& wave, Block& den) {
  Wave w = wave;
  wave_normalize(w);   // Get_density_matrix_env_new, den_mat.f90:158-164
  den = Block();
  den.len = w.env_len;
  den.num = w.num;
  den.sub.assign(den.num, SubBlock());
  for (int i = 0; i < w.num; ++i) {
    SubBlock& s = den.sub[i];
    s.num_up = w.sub[i].env_num_up;
    s.num_down = w.sub[i].env_num_down;
    s.down_dif = 0;
    s.row_dim = s.sdim = w.sub[i].env_dim;
    den.dim += s.sdim;
    int sd = w.sub[i].sys_dim, ed = w.sub[i].env_dim;
    s.mat.assign((size_t)ed * ed, 0.0);
    zgemm('C', 'N', ed, ed, sd, cone, w.sub[i].vec.data(), sd, w.sub[i].vec.data(), sd, czero,
          s.mat.data(), ed);
  }
}

// ---- truncation (den_mat.f90:184-418) ---------------------------------------------
void Oracle::truncation_operator(const Block& den, Block& trun, double trun_err, int* num_state_out,
                                 double* err_out, double* ent_out, double* ent_mult_out,
                                 bool system_block, std::vector<double>* spectrum) {
  (void)system_block;
  const double thr = 1.0000000036274937e-15;   // 1.0E-15 (default real), den_mat.f90:278,330
  int num = den.num;
  std::vector<std::vector<cplx>> evec(num);
  std::vector<std::vector<double>> eval(num);
  std::vector<std::vector<int>> sidx(num);
  int dim = 0;
  for (int k = 0; k < num; ++k) {
    int n = den.sub[k].sdim;
    evec[k] = den.sub[k].mat;
    eval[k].assign(n, 0.0);
    sidx[k].assign(n, 0);
    if (n > 0) {
      int lda = n, lwork = 3 * n, info = 0;
      std::vector<cplx> work(lwork);
      std::vector<double> rwork(lwork);
      char jobz = 'V', uplo = 'U';
      scipy_zheev_(&jobz, &uplo, &n, evec[k].data(), &lda, eval[k].data(), work.data(), &lwork,
                   rwork.data(), &info);
    }
    phase_fix(n, n, evec[k].data());
    // eigenvalues at rounding-noise level count as exact zeros (see null_completion)
    for (int i = 0; i < n; ++i)
      if (eval[k][i] < kZeroWeight) eval[k][i] = 0.0;
    for (int i = 0; i < n; ++i) sidx[k][i] = dim + i + 1;
    dim += n;
  }
  std::vector<int> idx(dim + 1), eigs(dim + 1);
  std::vector<double> ev(dim + 1);
  int p = 0;
  for (int k = 0; k < num; ++k)
    for (int i = 0; i < den.sub[k].sdim; ++i) {
      ++p;
      idx[p] = sidx[k][i];
      ev[p] = eval[k][i];
      eigs[p] = den.sub[k].num_down + 1;
    }
  double entropy1 = 0.0;
  for (int i = 1; i <= dim; ++i)
    if (ev[i] >= thr) {
      double v1 = ev[i] / eigs[i];
      entropy1 = entropy1 - v1 * std::log(v1) * eigs[i];
    }
  if (dim >= 1) quicksort_double(ev, idx, 1, dim);
  double tot = 0.0;
  for (int i = 1; i <= dim; ++i) tot += ev[i];
  for (int i = 1; i <= dim; ++i) ev[i] = ev[i] / tot;
  double tmp_err = 0.0;
  int num_state;
  if (dim <= kept_min) {
    num_state = dim;
    tmp_err = 0.0;
  } else {
    for (int i = kept_min + 1; i <= dim; ++i) tmp_err += ev[i];
    num_state = kept_min;
    while (tmp_err > trun_err) {
      num_state++;
      tmp_err = tmp_err - ev[num_state];
      if (tmp_err <= trun_err || num_state >= kept_max) break;
    }
  }
  double entropys = 0.0;
  for (int i = 1; i <= dim; ++i)
    if (ev[i] >= thr) entropys = entropys - ev[i] * std::log(ev[i]);
  std::vector<int> tmpidx(num, 0);
  for (int k = 1; k <= num_state; ++k) {
    bool f = false;
    for (int i = 0; i < num && !f; ++i)
      for (int x = 0; x < den.sub[i].sdim; ++x)
        if (sidx[i][x] == idx[k]) {
          tmpidx[i]++;
          f = true;
          break;
        }
  }
  trun = Block();
  for (int i = 0; i < num; ++i) {
    if (tmpidx[i] <= 0) continue;
    SubBlock s;
    s.num_up = den.sub[i].num_up;
    s.num_down = den.sub[i].num_down;
    s.down_dif = 0;
    s.row_dim = den.sub[i].sdim;
    s.sdim = tmpidx[i];
    s.mat.assign((size_t)s.row_dim * s.sdim, 0.0);
    int row = s.row_dim, col = s.sdim;
    for (int c = 0; c < col; ++c)
      for (int r = 0; r < row; ++r) s.at(r, c) = evec[i][(size_t)(row - col + c) * row + r];
    // kept columns of zero weight: canonical null-space basis instead of the
    // eigensolver's arbitrary vectors (columns stay in ascending-weight order)
    int sig = 0;
    for (int c = 0; c < col; ++c)
      if (eval[i][row - col + c] > 0.0) sig++;
    if (sig < col) {
      std::vector<cplx> nul((size_t)row * (col - sig));
      null_completion(row, sig, &s.mat[(size_t)(col - sig) * row], col - sig, nul.data());
      std::copy(nul.begin(), nul.end(), s.mat.begin());
    }
    trun.sub.push_back(std::move(s));
  }
  trun.num = (int)trun.sub.size();
  trun.len = den.len;
  trun.up_dif = den.up_dif;
  trun.down_dif = den.down_dif;
  trun.dim = 0;
  for (auto& s : trun.sub) trun.dim += s.sdim;
  *num_state_out = num_state;
  *err_out = tmp_err;
  *ent_out = entropys;
  *ent_mult_out = entropy1;
  if (spectrum) spectrum->assign(ev.begin() + 1, ev.end());
}

// ---- wave transformations (dmrg_sub.f90:1471-1789) --------------------------------
void Oracle::wave_trans_LR(const Basis& sys_bs, const Basis& env_bs, const Block& sys_trun,
                           const Block& env_trun, const Wave& old_w, Wave& new_w) {
  std::vector<cplx> sub;
  for (int i = 0; i < old_w.num; ++i) {
    const SubWave& o = old_w.sub[i];
    int st_id = find_blk(sys_trun, o.sys_num_up, o.sys_num_down);
    if (st_id < 0) continue;
    for (int k = 0; k < env_bs.num; ++k) {
      if (env_bs.sub[k].new_num_up != o.env_num_up || env_bs.sub[k].new_num_down != o.env_num_down) continue;
      for (const auto& p : env_bs.sub[k].sub) {
        int et_id = find_blk(env_trun, p.bl_num_up, p.bl_num_down);
        int neu = p.bl_num_up, ned = p.bl_num_down;
        for (int nsd = std::abs(o.sys_num_down - p.st_num_down); nsd <= o.sys_num_down + p.st_num_down;
             nsd += 2) {
          int nsu = o.sys_num_up + p.st_num_up;
          int y = find_bs(sys_bs, nsu, nsd);
          const SubBasisMap* q = nullptr;
          if (y >= 0)
            for (const auto& qq : sys_bs.sub[y].sub)
              if (qq.bl_num_up == o.sys_num_up && qq.bl_num_down == o.sys_num_down &&
                  qq.st_num_up == p.st_num_up && qq.st_num_down == p.st_num_down) {
                q = &qq;
                break;
              }
          int nw = -1;
          for (int yy = 0; yy < new_w.num; ++yy) {
            const SubWave& s = new_w.sub[yy];
            if (s.sys_num_up == nsu && s.sys_num_down == nsd && s.env_num_up == neu && s.env_num_down == ned) {
              nw = yy;
              break;
            }
          }
          if (et_id < 0 || !q || nw < 0) continue;
          SubWave& n = new_w.sub[nw];
          int new_env_dim = n.env_dim, new_pos = q->spos, nsub = q->sdim;
          int j12 = o.sys_num_down, j3 = p.st_num_down, j4 = ned, j123 = nsd, j34 = o.env_num_down;
          double c11 = pm1((j12 + j3 + j123) / 2) / std::sqrt((1.0 + j12) * (1.0 + j123));
          if (c11 == 0.0) continue;
          c11 = c11 * std::sqrt((1.0 + j123) * (j34 + 1.0));
          if (((j12 + j3 + j4) / 2) % 2 != 0) c11 = -c11;
          if (((j3 + j4 - j34) / 2) % 2 != 0) c11 = -c11;
          cplx coef1 = c11;
          int osd = o.sys_dim, opos = p.spos, osub = p.sdim;
          sub.assign((size_t)nsub * osub, 0.0);
          zgemm('C', 'N', nsub, osub, osd, coef1, sys_trun.sub[st_id].mat.data(), osd,
                &o.vec[(size_t)opos * osd], osd, czero, sub.data(), nsub);
          zgemm('N', 'C', nsub, new_env_dim, osub, cone, sub.data(), nsub,
                env_trun.sub[et_id].mat.data(), new_env_dim, cone, &n.vec[new_pos], n.sys_dim);
        }
      }
    }
  }
  wave_normalize(new_w);
}

void Oracle::wave_trans_RL(const Basis& sys_bs, const Basis& env_bs, const Block& sys_trun,
                           const Block& env_trun, const Wave& old_w, Wave& new_w) {
  std::vector<cplx> sub;
  for (int i = 0; i < old_w.num; ++i) {
    const SubWave& o = old_w.sub[i];
    int et_id = find_blk(env_trun, o.env_num_up, o.env_num_down);
    if (et_id < 0) continue;
    for (int k = 0; k < sys_bs.num; ++k) {
      if (sys_bs.sub[k].new_num_up != o.sys_num_up || sys_bs.sub[k].new_num_down != o.sys_num_down) continue;
      for (const auto& p : sys_bs.sub[k].sub) {
        int nsu = p.bl_num_up, nsd = p.bl_num_down;
        for (int ned = std::abs(o.env_num_down - p.st_num_down); ned <= o.env_num_down + p.st_num_down;
             ned += 2) {
          int neu = o.env_num_up + p.st_num_up;
          int st_id = find_blk(sys_trun, nsu, nsd);
          int y = find_bs(env_bs, neu, ned);
          const SubBasisMap* q = nullptr;
          if (y >= 0)
            for (const auto& qq : env_bs.sub[y].sub)
              if (qq.bl_num_up == o.env_num_up && qq.bl_num_down == o.env_num_down &&
                  qq.st_num_up == p.st_num_up && qq.st_num_down == p.st_num_down) {
                q = &qq;
                break;
              }
          int nw = -1;
          for (int yy = 0; yy < new_w.num; ++yy) {
            const SubWave& s = new_w.sub[yy];
            if (s.sys_num_up == nsu && s.sys_num_down == nsd && s.env_num_up == neu && s.env_num_down == ned) {
              nw = yy;
              break;
            }
          }
          if (st_id < 0 || !q || nw < 0) continue;
          SubWave& n = new_w.sub[nw];
          int new_sys_dim = n.sys_dim, new_pos = q->spos, nsub = q->sdim;
          int j12 = o.env_num_down, j3 = p.st_num_down, j4 = nsd, j123 = ned, j34 = o.sys_num_down;
          double c11 = pm1((j34 + j4 + j3) / 2) / std::sqrt((1.0 + j12) * (1.0 + j4));
          if (c11 == 0.0) continue;
          c11 = c11 * std::sqrt((1.0 + j123) * (j34 + 1.0));
          if (((j4 + j3 + j12) / 2) % 2 != 0) c11 = -c11;
          if (((j12 + j3 - j123) / 2) % 2 != 0) c11 = -c11;
          cplx coef1 = c11;
          int oed = o.env_dim, opos = p.spos, osub = p.sdim;
          sub.assign((size_t)new_sys_dim * oed, 0.0);
          zgemm('N', 'N', new_sys_dim, oed, osub, coef1, sys_trun.sub[st_id].mat.data(), new_sys_dim,
                &o.vec[opos], o.sys_dim, czero, sub.data(), new_sys_dim);
          zgemm('N', 'N', new_sys_dim, nsub, oed, cone, sub.data(), new_sys_dim,
                env_trun.sub[et_id].mat.data(), oed, cone, &n.vec[(size_t)new_pos * n.sys_dim], n.sys_dim);
        }
      }
    }
  }
  wave_normalize(new_w);
}

// ---- block growth (get_sys.f90:4-592) ---------------------------------------------
void Oracle::hamiltonian_sys(Model& pre, const Basis& basis, const Block& trun) {
  Model next;
  next.len = pre.len + 1;
  next.sub.assign(L.num_site + 1, BlockSet());
  update_block_dia(pre.ham, basis, next.ham);
  Block tmp, tmp1, tt;
  const int ijs[3] = {1, 3, 5};
  for (int ij : ijs) {
    int j = pre.len + 1;
    for (int k = 1; k <= L.neibt; ++k) {
      int I = L.NEIB(j, k);
      if (I <= pre.len && I > 0) {
        int i1 = L.INB1(I, pre.len);
        if (i1 > 0 && i1 <= L.nleg11[pre.len]) {
          cplx cx = L.JT(k, j), csd = L.JD(k, j);
          if (ij == 1 && cx != 0.0) {
            block_transfer_trans(st_elec_down, tt);
            hamiltonian_ndia(pre.sub[i1].elec_up, tt, basis, cx, next.ham, 'F', 'S');
          }
          if (ij == 3 && csd != 0.0) hamiltonian_ndia(pre.sub[i1].spin_sd, st_sd, basis, csd, next.ham, 'B', 'S');
        }
      }
    }
    for (int y = 1; y <= pre.len; ++y) {
      int i1 = L.INB1(y, pre.len);
      if (i1 <= L.nleg11[pre.len]) {
        if (ij == 1) {
          update_block_ndia(pre.sub[i1].elec_up, basis, next.sub[i1].elec_up, 'F', false);
          update_block_ndia(pre.sub[i1].elec_down, basis, next.sub[i1].elec_down, 'F', false);
          pre.sub[i1].elec_up = Block();
          pre.sub[i1].elec_down = Block();
        }
        if (ij == 3) {
          update_block_ndia(pre.sub[i1].spin_sd, basis, next.sub[i1].spin_sd, 'B', false);
          pre.sub[i1].spin_sd = Block();
        }
        if (ij == 5) {
          update_block_dia(pre.sub[i1].num_sn, basis, next.sub[i1].num_sn);
          pre.sub[i1].num_sn = Block();
        }
      }
    }
    if (ij == 1) {
      update_site_ndia(st_elec_up, basis, tmp, 'F', false);
      update_site_ndia(st_elec_down, basis, tmp1, 'F', false);
    }
    if (ij == 3) update_site_ndia(st_sd, basis, tmp, 'B', false);
    if (ij == 5) update_site_dia(num_elec, basis, tmp);
    for (int k = 1; k <= L.neibt; ++k) {
      int I = L.NEIB(j, k);
      if (I <= pre.len && I > 0) {
        int i1 = L.INB1(I, pre.len);
        if (i1 > 0 && i1 <= L.nleg11[pre.len]) {
          cplx csn = L.JN(k, j);
          if (ij == 5 && csn != 0.0) hamiltonian_dia(next.sub[i1].num_sn, tmp, csn, next.ham);
        }
      }
    }
    int nleg1 = L.nleg11[pre.len + 1];
    for (int I = 1; I <= pre.len; ++I) {
      int i1 = L.INB1(I, pre.len), J = L.INB1(I, pre.len + 1);
      if (J <= nleg1 && J != i1) {
        if (ij == 1) {
          next.sub[J].elec_up = next.sub[i1].elec_up;
          next.sub[J].elec_down = next.sub[i1].elec_down;
        }
        if (ij == 3) next.sub[J].spin_sd = next.sub[i1].spin_sd;
        if (ij == 5) next.sub[J].num_sn = next.sub[i1].num_sn;
      }
    }
    int jn = L.INB1(pre.len + 1, pre.len + 1);
    if (ij == 1) {
      next.sub[jn].elec_up = tmp;
      next.sub[jn].elec_down = tmp1;
    }
    if (ij == 3) next.sub[jn].spin_sd = tmp;
    if (ij == 5) next.sub[jn].num_sn = tmp;
    for (int jj = nleg1 + 1; jj <= L.nleg11[pre.len]; ++jj) {
      if (ij == 1) next.sub[jj].elec_up = next.sub[jj].elec_down = Block();
      if (ij == 3) next.sub[jj].spin_sd = Block();
      if (ij == 5) next.sub[jj].num_sn = Block();
    }
    for (int ii = 1; ii <= L.nleg11[next.len]; ++ii) {
      if (ij == 1) {
        update_trun_ndia(next.sub[ii].elec_up, pre.sub[ii].elec_up, trun);
        update_trun_ndia(next.sub[ii].elec_down, pre.sub[ii].elec_down, trun);
        next.sub[ii].elec_up = next.sub[ii].elec_down = Block();
      }
      if (ij == 3) {
        update_trun_ndia(next.sub[ii].spin_sd, pre.sub[ii].spin_sd, trun);
        next.sub[ii].spin_sd = Block();
      }
      if (ij == 5) {
        update_trun_dia(next.sub[ii].num_sn, pre.sub[ii].num_sn, trun);
        next.sub[ii].num_sn = Block();
      }
    }
  }
  Block h;
  update_trun_dia(next.ham, h, trun);
  pre.ham = h;
  pre.len = next.len;
}

void Oracle::hamiltonian_env(Model& pre, const Basis& basis, const Block& trun) {
  Model next;
  next.len = pre.len + 1;
  next.sub.assign(L.num_site + 1, BlockSet());
  update_block_dia(pre.ham, basis, next.ham);
  Block tmp, tmp1, tt;
  const int ijs[3] = {1, 3, 5};
  int j = pre.len + 1 + mshift;
  int lat = L.nposi_lat[j];
  for (int ij : ijs) {
    for (int k = 1; k <= L.neibt; ++k) {
      int I = L.NEIB(lat, k);
      int II = L.nposi_dm[I] - mshift;
      if (II <= pre.len && II > 0) {
        int i1 = L.INB1(II, pre.len);
        if (i1 > 0 && i1 <= L.nleg11[pre.len]) {
          cplx cx = L.JT(k, lat), csd = L.JD(k, lat);
          if (ij == 1 && cx != 0.0) {
            block_transfer_trans(st_elec_up, tt);
            hamiltonian_ndia(pre.sub[i1].elec_down, tt, basis, cx, next.ham, 'F', 'E');
          }
          if (ij == 3 && csd != 0.0) hamiltonian_ndia(pre.sub[i1].spin_sd, st_sd, basis, csd, next.ham, 'B', 'E');
        }
      }
    }
    for (int y = 1; y <= pre.len; ++y) {
      int i1 = L.INB1(y, pre.len);
      if (i1 <= L.nleg11[pre.len]) {
        if (ij == 1) {
          update_block_ndia(pre.sub[i1].elec_up, basis, next.sub[i1].elec_up, 'F', true);
          update_block_ndia(pre.sub[i1].elec_down, basis, next.sub[i1].elec_down, 'F', true);
          pre.sub[i1].elec_up = Block();
          pre.sub[i1].elec_down = Block();
        }
        if (ij == 3) {
          update_block_ndia(pre.sub[i1].spin_sd, basis, next.sub[i1].spin_sd, 'B', true);
          pre.sub[i1].spin_sd = Block();
        }
        if (ij == 5) {
          update_block_dia(pre.sub[i1].num_sn, basis, next.sub[i1].num_sn);
          pre.sub[i1].num_sn = Block();
        }
      }
    }
    if (ij == 1) {
      update_site_ndia(st_elec_up, basis, tmp, 'F', true);
      update_site_ndia(st_elec_down, basis, tmp1, 'F', true);
    }
    if (ij == 3) update_site_ndia(st_sd, basis, tmp, 'B', true);
    if (ij == 5) update_site_dia(num_elec, basis, tmp);
    for (int k = 1; k <= L.neibt; ++k) {
      int I = L.NEIB(lat, k);
      int II = L.nposi_dm[I] - mshift;
      if (II <= pre.len && II > 0) {
        int i1 = L.INB1(II, pre.len);
        if (i1 > 0 && i1 <= L.nleg11[pre.len]) {
          cplx csn = L.JN(k, lat);
          if (ij == 5 && csn != 0.0) hamiltonian_dia(next.sub[i1].num_sn, tmp, csn, next.ham);
        }
      }
    }
    int nleg1 = L.nleg11[pre.len + 1];
    for (int I = 1; I <= pre.len; ++I) {
      int i1 = L.INB1(I, pre.len), J = L.INB1(I, pre.len + 1);
      if (J <= nleg1 && J != i1) {
        if (ij == 1) {
          next.sub[J].elec_up = next.sub[i1].elec_up;
          next.sub[J].elec_down = next.sub[i1].elec_down;
        }
        if (ij == 3) next.sub[J].spin_sd = next.sub[i1].spin_sd;
        if (ij == 5) next.sub[J].num_sn = next.sub[i1].num_sn;
      }
    }
    int jn = L.INB1(pre.len + 1, pre.len + 1);
    if (ij == 1) {
      next.sub[jn].elec_up = tmp;
      next.sub[jn].elec_down = tmp1;
    }
    if (ij == 3) next.sub[jn].spin_sd = tmp;
    if (ij == 5) next.sub[jn].num_sn = tmp;
    for (int jj = nleg1 + 1; jj <= L.nleg11[pre.len]; ++jj) {
      if (ij == 1) next.sub[jj].elec_up = next.sub[jj].elec_down = Block();
      if (ij == 3) next.sub[jj].spin_sd = Block();
      if (ij == 5) next.sub[jj].num_sn = Block();
    }
    for (int ii = 1; ii <= L.nleg11[next.len]; ++ii) {
      if (ij == 1) {
        update_trun_ndia(next.sub[ii].elec_up, pre.sub[ii].elec_up, trun);
        update_trun_ndia(next.sub[ii].elec_down, pre.sub[ii].elec_down, trun);
        next.sub[ii].elec_up = next.sub[ii].elec_down = Block();
      }
      if (ij == 3) {
        update_trun_ndia(next.sub[ii].spin_sd, pre.sub[ii].spin_sd, trun);
        next.sub[ii].spin_sd = Block();
      }
      if (ij == 5) {
        update_trun_dia(next.sub[ii].num_sn, pre.sub[ii].num_sn, trun);
        next.sub[ii].num_sn = Block();
      }
    }
  }
  Block h;
  update_trun_dia(next.ham, h, trun);
  pre.ham = h;
  pre.len = next.len;
}

// ---- measurement of <n_i> (measure.f90) ------------------------------------------

Block Oracle::oper_dia_in_block(const Block& st, int old_idx, int new_idx, bool sys) {
  const auto& bsm = sys ? sys_bsm : env_bsm;
  const auto& truns = sys ? sys_truns : env_truns;
  const int trun_idx = 1;
  const int one = std::min(old_idx, new_idx), two = std::max(old_idx, new_idx);
  Block cur, mid, out;
  if (one <= two - 1) {
    if (one <= 1) {
      cur = st;
    } else if (one <= trun_idx) {
      update_site_dia(st, bsm.at(one), cur);
    } else {
      update_site_dia(st, bsm.at(one), mid);
      update_trun_dia(mid, cur, truns.at(one));
    }
    int idx = one;
    while (idx + 1 <= two - 1) {
      update_block_dia(cur, bsm.at(idx + 1), mid);
      idx++;
      if (idx <= trun_idx) cur = mid;
      else update_trun_dia(mid, cur, truns.at(idx));
    }
    update_block_dia(cur, bsm.at(idx + 1), out);
  } else {
    if (one <= 1) out = st;
    else update_site_dia(st, bsm.at(two), out);
  }
  auto it = truns.find(two);
  if (it == truns.end()) return out;   // lengths below trun_idx+1 carry no truncation
  Block t;
  update_trun_dia(out, t, it->second);
  return t;
}

// measure_sys_block / measure_env_block (measure.f90:778-840, 905-970)
static cplx measure_block(const Block& bl, const Basis& bs, const Wave& w, bool sys) {
  cplx value = 0.0;
  std::vector<cplx> mid;
  for (const auto& ws : w.sub) {
    const int qup = sys ? ws.sys_num_up : ws.env_num_up, qdn = sys ? ws.sys_num_down : ws.env_num_down;
    for (const auto& S : bs.sub) {
      if (S.new_num_up != qup || S.new_num_down != qdn) continue;
      for (const auto& p : S.sub) {
        const int y = find_blk(bl, p.bl_num_up, p.bl_num_down);
        if (y < 0) continue;
        const cplx coef = 1.0 / std::sqrt(1.0 + p.bl_num_down);
        if (sys) {
          mid.assign((size_t)p.sdim * ws.env_dim, 0.0);
          zgemm('N', 'N', p.sdim, ws.env_dim, p.sdim, coef, bl.sub[y].mat.data(), p.sdim,
                ws.vec.data() + p.spos, ws.sys_dim, czero, mid.data(), p.sdim);
          for (int z = 0; z < ws.env_dim; ++z)
            for (int r = 0; r < p.sdim; ++r)
              value += std::conj(ws.vec[(size_t)z * ws.sys_dim + p.spos + r]) * mid[(size_t)z * p.sdim + r];
        } else {
          mid.assign((size_t)ws.sys_dim * p.sdim, 0.0);
          zgemm('N', 'N', ws.sys_dim, p.sdim, p.sdim, coef, ws.vec.data() + (size_t)p.spos * ws.sys_dim,
                ws.sys_dim, bl.sub[y].mat.data(), p.sdim, czero, mid.data(), ws.sys_dim);
          for (int z = 0; z < p.sdim; ++z)
            for (int r = 0; r < ws.sys_dim; ++r)
              value += std::conj(mid[(size_t)z * ws.sys_dim + r]) * ws.vec[(size_t)(p.spos + z) * ws.sys_dim + r];
        }
      }
    }
  }
  return value;
}

// measure_sys_site / measure_env_site (measure.f90:842-903, 971-1030)
static cplx measure_site(const Block& st, const Basis& bs, const Wave& w, bool sys) {
  cplx value = 0.0;
  for (const auto& ws : w.sub) {
    const int qup = sys ? ws.sys_num_up : ws.env_num_up, qdn = sys ? ws.sys_num_down : ws.env_num_down;
    for (const auto& S : bs.sub) {
      if (S.new_num_up != qup || S.new_num_down != qdn) continue;
      for (const auto& p : S.sub) {
        const int y = find_blk(st, p.st_num_up, p.st_num_down);
        if (y < 0) continue;
        const cplx coef = 1.0 / std::sqrt(1.0 + p.st_num_down);
        cplx yita = 0.0;
        if (sys) {
          for (int z = 0; z < ws.env_dim; ++z)
            for (int r = 0; r < p.sdim; ++r) yita += std::norm(ws.vec[(size_t)z * ws.sys_dim + p.spos + r]);
        } else {
          for (int z = 0; z < p.sdim; ++z)
            for (int r = 0; r < ws.sys_dim; ++r) yita += std::norm(ws.vec[(size_t)(p.spos + z) * ws.sys_dim + r]);
        }
        value += yita * st.sub[y].mat[0] * coef;
      }
    }
  }
  return value;
}

std::vector<double> Oracle::measure_density() {
  const Wave& w = disk_wave;
  const int N = L.num_site, sl = w.sys_len, el = w.env_len;
  std::vector<double> ave(N, 0.0);
  for (int i = 1; i <= sl - 1; ++i)
    ave[i - 1] = measure_block(oper_dia_in_block(num_elec, i, sl - 1, true), sys_bsm.at(sl), w, true).real();
  ave[sl - 1] = measure_site(num_elec, sys_bsm.at(sl), w, true).real();
  for (int i = 1; i <= el - 1; ++i)
    ave[N - i] = measure_block(oper_dia_in_block(num_elec, i, el - 1, false), env_bsm.at(el), w, false).real();
  ave[N - el] = measure_site(num_elec, env_bsm.at(el), w, false).real();
  return ave;
}

}  // namespace orc

// ---- density-density correlation (Get_density_cor, measure.f90:2525-2681) ---------

namespace orc {
namespace {

// block_mul_block_ndia (block.f90:376-635) with Flag1 = Flag2 = 'N', coef = 1:
// (o1 o2) coupled to rank new_down_dif on the sectors of `basis`, the 3j sums
// of block.f90:584-613 evaluated as written.
Block block_mul_ndia_nn(const Block& o1, const Block& o2, int new_down_dif, const Basis& basis) {
  const int up_dif2 = o2.up_dif, K1 = o1.down_dif, K2 = o2.down_dif;
  Block nb;
  nb.len = basis.len;
  nb.up_dif = o1.up_dif + o2.up_dif;
  nb.down_dif = new_down_dif;
  const int up_dif = nb.up_dif, down_dif = new_down_dif;
  for (int i = 0; i < basis.num; ++i) {
    const int num_up = basis.sub[i].new_num_up, num_down = basis.sub[i].new_num_down;
    const int new_num_up = num_up + up_dif;
    for (int new_num_down = std::abs(num_down - down_dif); new_num_down <= num_down + down_dif; new_num_down += 2) {
      const int bs_idx = find_bs(basis, new_num_up, new_num_down);
      if (bs_idx < 0) continue;
      SubBlock s;
      s.num_up = num_up;
      s.num_down = num_down;
      s.down_dif = new_num_down - num_down;
      s.row_dim = basis.sub[bs_idx].dim;
      s.sdim = basis.sub[i].dim;
      s.mat.assign((size_t)s.row_dim * s.sdim, czero);
      for (int mid_num_down = std::abs(num_down - K2); mid_num_down <= num_down + K2; mid_num_down += 2) {
        const int idx2 = find_blk3(o2, num_up, num_down, mid_num_down - num_down);
        const int idx1 = find_blk3(o1, num_up + up_dif2, mid_num_down, new_num_down - mid_num_down);
        if (idx1 < 0 || idx2 < 0) continue;
        const int kq = new_num_down - num_down;   // j5 = -j4 - j6 of the normalising 3j
        const double c11 = w3js(new_num_down, down_dif, num_down, -new_num_down, kq, num_down);
        if (c11 == 0.0) throw std::runtime_error("block_mul_ndia: vanishing 3j normalisation");
        double c1 = 0.0;
        for (int m6 = -mid_num_down; m6 <= mid_num_down; m6 += 2) {
          const int m5 = new_num_down - m6;
          double c12 = w3js(new_num_down, K1, mid_num_down, -new_num_down, m5, m6);
          const int m44 = -m6, m55 = -m44 - num_down;
          c12 *= w3js(mid_num_down, K2, num_down, m44, m55, num_down) * pm1((mid_num_down + m44) / 2);
          c12 *= w3js(K1, K2, down_dif, m5, m55, -kq) * pm1((-K1 + K2 + kq) / 2) * std::sqrt(down_dif + 1.0);
          c1 += c12;
        }
        if (c1 == 0.0) continue;
        const SubBlock& a = o1.sub[idx1];
        const SubBlock& b = o2.sub[idx2];
        zgemm('N', 'N', s.row_dim, s.sdim, a.sdim, cplx(c1 / c11, 0.0), a.mat.data(), s.row_dim, b.mat.data(),
              a.sdim, cone, s.mat.data(), s.row_dim);
      }
      nb.dim += s.sdim;
      nb.sub.push_back(std::move(s));
    }
  }
  nb.num = (int)nb.sub.size();
  return nb;
}

// block_transfer_trans (block.f90:33-64): conjugate transpose of every sub-block,
// keyed by its row quantum numbers.
Block block_transfer_trans(const Block& in) {
  Block out;
  out.len = in.len;
  out.num = in.num;
  out.up_dif = -in.up_dif;
  out.down_dif = in.down_dif;
  for (const auto& x : in.sub) {
    SubBlock s;
    s.num_up = x.num_up + in.up_dif;
    s.num_down = x.num_down + x.down_dif;
    s.down_dif = -x.down_dif;
    s.row_dim = x.sdim;
    s.sdim = x.row_dim;
    s.mat.assign((size_t)s.row_dim * s.sdim, czero);
    for (int c = 0; c < s.sdim; ++c)
      for (int r = 0; r < s.row_dim; ++r) s.mat[(size_t)c * s.row_dim + r] = std::conj(x.mat[(size_t)r * x.row_dim + c]);
    out.dim += s.sdim;
    out.sub.push_back(std::move(s));
  }
  return out;
}

const SubBasisMap* find_piece(const BasisMap& S, int bu, int bd, int su, int sd) {
  for (const auto& p : S.sub)
    if (p.bl_num_up == bu && p.bl_num_down == bd && p.st_num_up == su && p.st_num_down == sd) return &p;
  return nullptr;
}

int find_wave(const Wave& w, int su, int sd, int eu, int ed) {
  for (int m = 0; m < (int)w.sub.size(); ++m)
    if (w.sub[m].sys_num_up == su && w.sub[m].sys_num_down == sd && w.sub[m].env_num_up == eu &&
        w.sub[m].env_num_down == ed)
      return m;
  return -1;
}

// sign of the electron-number parity term of the correlators: 'B' always +1,
// 'F' (-1)^tot_num (measure.f90:4167-4178, 4830-4841, 4569-4580)
inline double flag_sign(char flag, int tot_num) { return flag == 'F' && (tot_num % 2) ? -1.0 : 1.0; }

// sys_block_site_cor_ndia (measure.f90:4064-4218)
cplx block_site_cor(const Block& bl, const Block& st, const Basis& bs, const Wave& w, char flag) {
  const int K = bl.down_dif, up_dif = bl.up_dif;
  cplx value = 0.0;
  std::vector<cplx> mid;
  for (const auto& ws : w.sub) {
    const int j = find_bs(bs, ws.sys_num_up, ws.sys_num_down);
    if (j < 0) continue;
    for (const auto& p : bs.sub[j].sub)
      for (int dd = -K; dd <= K; dd += 2)
        for (int sdd = -K; sdd <= K; sdd += 2) {
          const int nbu = p.bl_num_up + up_dif, nbd = p.bl_num_down + dd;
          const int nsu = p.st_num_up - up_dif, nsd = p.st_num_down - sdd;
          const int bid = find_blk3(bl, p.bl_num_up, p.bl_num_down, dd);
          const int sid = find_blk3(st, nsu, nsd, sdd);
          const SubBasisMap* q = find_piece(bs.sub[j], nbu, nbd, nsu, nsd);
          if (bid < 0 || sid < 0 || !q) continue;
          double c = 1.0 / std::sqrt(1.0 + K) * w6js(nbd, p.bl_num_down, K, p.st_num_down, nsd, ws.sys_num_down);
          if (c == 0.0) continue;
          c *= pm1((p.bl_num_down + nsd + K + ws.sys_num_down) / 2);
          const cplx coef = flag_sign(flag, p.bl_num_up) * st.sub[sid].mat[0] * c;
          mid.assign((size_t)q->sdim * ws.env_dim, czero);
          zgemm('N', 'N', q->sdim, ws.env_dim, p.sdim, coef, bl.sub[bid].mat.data(), q->sdim, ws.vec.data() + p.spos,
                ws.sys_dim, czero, mid.data(), q->sdim);
          for (int z = 0; z < ws.env_dim; ++z)
            for (int r = 0; r < q->sdim; ++r)
              value += std::conj(ws.vec[(size_t)z * ws.sys_dim + q->spos + r]) * mid[(size_t)z * q->sdim + r];
        }
  }
  return value;
}

// sys_block_env_site_cor_ndia (measure.f90:4666-4903)
cplx block_env_site_cor(const Block& bl, const Block& est, const Basis& sbs, const Basis& ebs, const Wave& w,
                        char flag) {
  const int K = bl.down_dif, Ke = est.down_dif, up_dif = bl.up_dif;
  cplx value = 0.0;
  std::vector<cplx> mat;
  for (const auto& ws : w.sub) {
    const int j = find_bs(sbs, ws.sys_num_up, ws.sys_num_down), k = find_bs(ebs, ws.env_num_up, ws.env_num_down);
    if (j < 0 || k < 0) continue;
    for (const auto& x : sbs.sub[j].sub)
      for (const auto& y : ebs.sub[k].sub)
        for (int bdd = -K; bdd <= K; bdd += 2) {
          const int nsbu = x.bl_num_up + up_dif, nsbd = x.bl_num_down + bdd;
          const int sys_id = find_blk3(bl, x.bl_num_up, x.bl_num_down, bdd);
          for (int sdd = -Ke; sdd <= Ke; sdd += 2) {
            const int neu = y.st_num_up - up_dif, ned = y.st_num_down - sdd;
            const int env_id = find_blk3(est, neu, ned, sdd);
            if (sys_id < 0 || env_id < 0) continue;
            for (int nsd = std::abs(ws.sys_num_down - K); nsd <= ws.sys_num_down + K; nsd += 2) {
              const int nsu = ws.sys_num_up + up_dif, nenu = ws.env_num_up - up_dif, nend = nsd;
              const int m1 = find_bs(sbs, nsu, nsd), m2 = find_bs(ebs, nenu, nend);
              const SubBasisMap* qs = m1 < 0 ? nullptr : find_piece(sbs.sub[m1], nsbu, nsbd, x.st_num_up, x.st_num_down);
              const SubBasisMap* qe = nullptr;
              if (m2 >= 0)
                for (const auto& p : ebs.sub[m2].sub)
                  if (p.st_num_up == neu && p.st_num_down == ned && p.bl_num_down == y.bl_num_down) {
                    qe = &p;
                    break;
                  }
              const int wid = find_wave(w, nsu, nsd, nenu, nend);
              if (!qs || !qe || wid < 0) continue;
              double c = w6js(nsd, K, ws.sys_num_down, x.bl_num_down, x.st_num_down, nsbd);
              if (c == 0.0) continue;
              c *= w6js(nend, K, ws.env_num_down, y.st_num_down, y.bl_num_down, ned);
              if (c == 0.0) continue;
              c *= std::sqrt((1.0 + nend) * (1.0 + ws.env_num_down) / (1.0 + K));
              if ((((nsbd + x.st_num_down + ws.sys_num_down + K) / 2 + (y.bl_num_down + y.st_num_down + nend + K) / 2) %
                   2) != 0)
                c = -c;
              const cplx coef = flag_sign(flag, ws.sys_num_up) * est.sub[env_id].mat[0] * c;
              mat.assign((size_t)qs->sdim * y.sdim, czero);
              zgemm('N', 'N', qs->sdim, y.sdim, x.sdim, coef, bl.sub[sys_id].mat.data(), qs->sdim,
                    ws.vec.data() + (size_t)y.spos * ws.sys_dim + x.spos, ws.sys_dim, czero, mat.data(), qs->sdim);
              const SubWave& nw = w.sub[wid];
              for (int m = 0; m < y.sdim; ++m)
                for (int r = 0; r < qs->sdim; ++r)
                  value += std::conj(nw.vec[(size_t)(qe->spos + m) * nw.sys_dim + qs->spos + r]) * mat[(size_t)m * qs->sdim + r];
            }
          }
        }
  }
  return value;
}

// sys_block_env_block_cor_ndia (measure.f90:4398-4661)
cplx block_env_block_cor(const Block& bl, const Block& ebl, const Basis& sbs, const Basis& ebs, const Wave& w,
                         char flag) {
  const int K = bl.down_dif, up_dif = bl.up_dif;
  cplx value = 0.0;
  std::vector<cplx> mat1, mat2;
  for (const auto& ws : w.sub) {
    const int j = find_bs(sbs, ws.sys_num_up, ws.sys_num_down), k = find_bs(ebs, ws.env_num_up, ws.env_num_down);
    if (j < 0 || k < 0) continue;
    for (const auto& x : sbs.sub[j].sub)
      for (const auto& y : ebs.sub[k].sub)
        for (int dd = -K; dd <= K; dd += 2) {
          const int nsbu = x.bl_num_up + up_dif, nsbd = x.bl_num_down + dd;
          const int sys_id = find_blk3(bl, x.bl_num_up, x.bl_num_down, dd);
          for (int edd = -K; edd <= K; edd += 2) {
            const int nebu = y.bl_num_up - up_dif, nebd = y.bl_num_down - edd;
            const int env_id = find_blk3(ebl, nebu, nebd, edd);
            if (sys_id < 0 || env_id < 0) continue;
            for (int nsd = std::abs(ws.sys_num_down - K); nsd <= ws.sys_num_down + K; nsd += 2) {
              const int nsu = ws.sys_num_up + up_dif, nenu = ws.env_num_up - up_dif, nend = nsd;
              const int m1 = find_bs(sbs, nsu, nsd), m2 = find_bs(ebs, nenu, nend);
              const SubBasisMap* qs = m1 < 0 ? nullptr : find_piece(sbs.sub[m1], nsbu, nsbd, x.st_num_up, x.st_num_down);
              const SubBasisMap* qe = m2 < 0 ? nullptr : find_piece(ebs.sub[m2], nebu, nebd, y.st_num_up, y.st_num_down);
              const int wid = find_wave(w, nsu, nsd, nenu, nend);
              if (!qs || !qe || wid < 0) continue;
              double c = w6js(nsd, K, ws.sys_num_down, x.bl_num_down, x.st_num_down, nsbd);
              if (c == 0.0) continue;
              c *= w6js(nend, K, ws.env_num_down, y.bl_num_down, y.st_num_down, nebd);
              if (c == 0.0) continue;
              c *= std::sqrt((1.0 + nend) * (1.0 + ws.env_num_down) / (1.0 + K));
              if ((((nsbd + x.st_num_down + ws.sys_num_down + K) / 2 + (nebd + y.st_num_down + ws.env_num_down + K) / 2) %
                   2) == 1)
                c = -c;
              c *= flag_sign(flag, ws.sys_num_up + y.st_num_up);
              const SubWave& nw = w.sub[wid];
              mat1.assign((size_t)qs->sdim * y.sdim, czero);
              mat2.assign((size_t)qs->sdim * y.sdim, czero);
              zgemm('N', 'N', qs->sdim, y.sdim, x.sdim, cone, bl.sub[sys_id].mat.data(), qs->sdim,
                    ws.vec.data() + (size_t)y.spos * ws.sys_dim + x.spos, ws.sys_dim, czero, mat1.data(), qs->sdim);
              zgemm('N', 'C', qs->sdim, y.sdim, qe->sdim, cplx(c, 0.0),
                    nw.vec.data() + (size_t)qe->spos * nw.sys_dim + qs->spos, nw.sys_dim, ebl.sub[env_id].mat.data(),
                    y.sdim, czero, mat2.data(), qs->sdim);
              for (size_t e = 0; e < mat1.size(); ++e) value += std::conj(mat1[e]) * mat2[e];
            }
          }
        }
  }
  return value;
}

}  // namespace

// Get_sys_oper_ndia / Get_env_oper_ndia (get_sys.f90:1536-1668), trun_idx = 1,
// Types 'B'; with trunc the result is truncated at the longer length (Truns).
Block Oracle::oper_ndia(const Block& st, int old_idx, int new_idx, bool sys, bool trunc, char flags) {
  const auto& bsm = sys ? sys_bsm : env_bsm;
  const auto& truns = sys ? sys_truns : env_truns;
  const int trun_idx = 1;
  const int one = std::min(old_idx, new_idx), two = std::max(old_idx, new_idx);
  Block cur, mid, out;
  if (one <= two - 1) {
    if (one <= 1) {
      cur = st;
    } else if (one <= trun_idx) {
      update_site_ndia(st, bsm.at(one), cur, flags, !sys);
    } else {
      update_site_ndia(st, bsm.at(one), mid, flags, !sys);
      update_trun_ndia(mid, cur, truns.at(one));
    }
    int idx = one;
    while (idx + 1 <= two - 1) {
      update_block_ndia(cur, bsm.at(idx + 1), mid, flags, !sys);
      idx++;
      if (idx <= trun_idx) cur = mid;
      else update_trun_ndia(mid, cur, truns.at(idx));
    }
    update_block_ndia(cur, bsm.at(idx + 1), out, flags, !sys);
  } else {
    if (one <= 1) out = st;
    else update_site_ndia(st, bsm.at(two), out, flags, !sys);
  }
  auto it = truns.find(two);
  if (!trunc || it == truns.end()) return out;
  Block t;
  update_trun_ndia(out, t, it->second);
  return t;
}

// Change_sys_oper_ndia (get_sys.f90:1672-1723; ndia) or Change_sys_oper_dia
// (get_sys.f90:1281-1331; dia), and their env twins, with Truns = .true.
Block Oracle::change_oper(const Block& op, int old_idx, int new_idx, bool sys, bool ndia, char flags,
                          bool trunc_end) {
  const auto& bsm = sys ? sys_bsm : env_bsm;
  const auto& truns = sys ? sys_truns : env_truns;
  const int trun_idx = 1;
  const int one = std::min(old_idx, new_idx), two = std::max(old_idx, new_idx);
  if (one == two) return op;
  auto grow = [&](const Block& b, const Basis& bs, Block& o) {
    if (ndia) update_block_ndia(b, bs, o, flags, !sys);
    else update_block_dia(b, bs, o);
  };
  auto trun = [&](const Block& b, Block& o, const Block& t) {
    if (ndia) update_trun_ndia(b, o, t);
    else update_trun_dia(b, o, t);
  };
  Block cur = op, mid, out;
  int idx = one;
  while (idx + 1 <= two - 1) {
    grow(cur, bsm.at(idx + 1), mid);
    idx++;
    if (idx <= trun_idx) cur = mid;
    else trun(mid, cur, truns.at(idx));
  }
  grow(cur, bsm.at(idx + 1), out);
  auto it = truns.find(two);
  if (!trunc_end || it == truns.end()) return out;
  Block t;
  trun(out, t, it->second);
  return t;
}

// Get_density_cor (measure.f90:2525-2681), xi = xj: the row <op1_xi op2_j>
// over the partners the reference visits, for its Flags ('B' or 'F').
std::vector<cplx> Oracle::oper_cor(const Block& op1, const Block& op2, char flags, int xi) {
  const Wave& w = disk_wave;
  const int N = L.num_site, ny = L.Ny, sl = w.sys_len, el = w.env_len;
  if (xi < 1 || xi > sl - 1) throw std::runtime_error("oper_cor: the site must lie in the system block");
  const double scale = std::sqrt(1.0 + op1.down_dif) * (op1.down_dif == 2 ? -1.0 : 1.0);
  std::vector<cplx> out(N + 1, czero);
  // partners inside the system block: Get_sys2b + measure_sys_block
  for (int j = xi + ny; j <= sl - 1; j += ny) {
    Block a = oper_ndia(op1, xi, j, true, false, flags);
    Block b = oper_ndia(op2, j, j, true, false, flags);
    Block p = block_mul_ndia_nn(a, b, 0, sys_bsm.at(j));
    Block q;
    auto it = sys_truns.find(j);
    if (j <= 1 || it == sys_truns.end()) q = p;
    else update_trun_dia(p, q, it->second);
    Block s = change_oper(q, j, sl - 1, true, false, flags);
    out[j] = measure_block(s, sys_bsm.at(sl), w, true) * scale;
  }
  const int last = N - N / 6 + ny;
  if (sl > last) return out;
  Block s1 = oper_ndia(op1, xi, xi, true, false, flags);
  if (xi > 1) {
    auto it = sys_truns.find(xi);
    if (it != sys_truns.end()) {
      Block t;
      update_trun_ndia(s1, t, it->second);
      s1 = t;
    }
  }
  Block sys_oper = change_oper(s1, xi, sl - 1, true, true, flags);
  const Block site_op = op2.down_dif == 1 ? block_transfer_trans(op2) : op2;
  for (int j = sl; j <= std::min(last, N); ++j) {
    if ((j - xi) % ny != 0) continue;
    cplx v = 0.0;
    if (j == sl) {
      v = block_site_cor(sys_oper, site_op, sys_bsm.at(sl), w, flags);
    } else if (j == sl + 1) {
      v = block_env_site_cor(sys_oper, site_op, sys_bsm.at(sl), env_bsm.at(el), w, flags);
    } else {
      const int e = N - j + 1;
      Block e1 = oper_ndia(op2, e, e, false, false, flags);
      if (e > 1) {
        auto it = env_truns.find(e);
        if (it != env_truns.end()) {
          Block t;
          update_trun_ndia(e1, t, it->second);
          e1 = t;
        }
      }
      Block env_oper = change_oper(e1, e, el - 1, false, true, flags);
      if (op2.down_dif != 0) env_oper = block_transfer_trans(env_oper);
      v = block_env_block_cor(sys_oper, env_oper, sys_bsm.at(sl), env_bsm.at(el), w, flags);
    }
    out[j] = v * scale;
  }
  return out;
}

// ---- singlet pair correlations (Get_mSCOP_Operator_Cor0, measure.f90:2683-2834) ------
//
// O+_ij = (c+_{i up} c+_{j down} - c+_{i down} c+_{j up}) / sqrt(2) (measure.f90:5441-5442)
// is the rank-0 coupling of two st_elec_up, built at the longer length.

// Get_sys_two (measure.f90:2837-2874): O+_{idx1 idx2} on the system block of
// length idx2, truncated there.
Block Oracle::sys_two(int idx1, int idx2) {
  Block a = oper_ndia(st_elec_up, idx1, idx2, true, false, 'F');
  Block b = oper_ndia(st_elec_up, idx2, idx2, true, false, 'F');
  Block p = block_mul_ndia_nn(a, b, 0, sys_bsm.at(idx2));
  auto it = sys_truns.find(idx2);
  if (idx2 <= 1 || it == sys_truns.end()) return p;
  Block t;
  update_trun_ndia(p, t, it->second);
  return t;
}

// Get_sys_two1 (measure.f90:2877-2932): the pair operator of length idx2 times
// st_elec_down at idx3 (coupled to rank 1/2), times st_elec_down at idx4
// (coupled to rank 0), carried to the system block of the wave.
Block Oracle::sys_two1(int idx2, int idx3, int idx4, const Block& pair) {
  const int sl = disk_wave.sys_len;
  Block m = change_oper(pair, idx2, idx3, true, true, 'B', false);
  Block c3 = oper_ndia(st_elec_down, idx3, idx3, true, false, 'F');
  Block p3 = block_mul_ndia_nn(m, c3, 1, sys_bsm.at(idx3));
  Block t3 = p3;
  auto it3 = sys_truns.find(idx3);
  if (idx3 > 1 && it3 != sys_truns.end()) update_trun_ndia(p3, t3, it3->second);
  Block m4 = change_oper(t3, idx3, idx4, true, true, 'F', false);
  Block c4 = oper_ndia(st_elec_down, idx4, idx4, true, false, 'F');
  Block p4 = block_mul_ndia_nn(m4, c4, 0, sys_bsm.at(idx4));
  Block t4 = p4;
  auto it4 = sys_truns.find(idx4);
  if (idx4 > 1 && it4 != sys_truns.end()) update_trun_dia(p4, t4, it4->second);
  return change_oper(t4, idx4, sl - 1, true, false, 'B', true);
}

// Get_SCOP_Operator_Env with Flags 'S0' (measure.f90:5450-5505): O+_{idx1 idx2}
// on the environment block of length idx2, carried to new_idx (truncated there
// when truns).
Block Oracle::env_scop(int idx1, int idx2, int new_idx, bool truns) {
  Block a = oper_ndia(st_elec_up, idx1, idx2, false, false, 'F');
  Block b = oper_ndia(st_elec_up, idx2, idx2, false, false, 'F');
  Block p = block_mul_ndia_nn(a, b, 0, env_bsm.at(idx2));
  Block e = p;
  auto it = env_truns.find(idx2);
  if (idx2 > 1 && it != env_truns.end()) update_trun_ndia(p, e, it->second);
  return change_oper(e, idx2, new_idx, false, true, 'B', truns);
}

// Get_mSCOP_Operator_Cor0 from label 11 (the part main.f90:259-262 reaches),
// Flags 'S0': the pair O+ on the bond (xc1, neib(xc1, ij1)) against the bonds
// (sid3, neib(sid3, 1|3|5)) for sid3 on the leg of xc1 up to xc2, the system
// block first, then the environment (values conjugated there as the reference
// does).  The reference writes these to a file; here they are returned.
std::vector<Oracle::PairRec> Oracle::pair_cor(int xc1, int xc2, int ij, int ij1) {
  const Wave& w = disk_wave;
  const int N = L.num_site, ny = L.Ny, sl = w.sys_len, el = w.env_len;
  std::vector<PairRec> out;
  const int sid1 = xc1, sid2 = L.NEIB(sid1, ij1);
  if (sid2 < 1) throw std::runtime_error("pair_cor: the first bond leaves the lattice");
  const int lo = std::min(sid1, sid2), hi = std::max(sid1, sid2);
  if (hi > sl - 1) throw std::runtime_error("pair_cor: the first bond must lie in the system block");
  Block pair = sys_two(lo, hi);
  for (int sid3 = sid1 + ny + ij; sid3 <= sl - 1; sid3 += ny) {
    if (sid3 <= hi || sid3 > xc2) continue;
    for (int i = 1; i <= 5; i += 2) {
      const int sid4 = L.NEIB(sid3, i);
      if (std::min(sid4, sid3) <= hi) continue;
      if (std::max(sid3, sid4) > sl - 1) continue;
      Block four = sys_two1(hi, std::min(sid3, sid4), std::max(sid3, sid4), pair);
      out.push_back(PairRec{sid1, sid2, sid3, sid4, measure_block(four, sys_bsm.at(sl), w, true)});
    }
  }
  Block sys_oper = change_oper(pair, hi, sl - 1, true, true, 'B', true);
  const int m0 = (sl + 2) % ny, m1 = (sid1 - 1) % ny;
  for (int sid3 = sl + 2 - m0 + m1 + 1 + ij; sid3 <= xc2; sid3 += ny) {
    const int eid1 = N - sid3 + 1;
    if (eid1 > el - 1) continue;
    for (int i = 1; i <= 5; i += 2) {
      const int sid4 = L.NEIB(sid3, i);
      if (sid4 < 1) continue;
      const int eid2 = N - sid4 + 1;
      if (std::max(eid1, eid2) > el - 1) continue;
      Block env_oper = env_scop(std::min(eid1, eid2), std::max(eid1, eid2), el - 1, true);
      const cplx v = block_env_block_cor(sys_oper, env_oper, sys_bsm.at(sl), env_bsm.at(el), w, 'B');
      out.push_back(PairRec{sid1, sid2, sid3, sid4, std::conj(v)});
    }
  }
  return out;
}

std::vector<cplx> Oracle::density_cor(int xi) { return oper_cor(num_elec, num_elec, 'B', xi); }

// main.f90:275: Get_density_cor(spin_cor, st_sd, st_sd, ..., 'B', ..., xi1, xi1)
std::vector<cplx> Oracle::spin_cor(int xi) { return oper_cor(st_sd, st_sd, 'B', xi); }

// main.f90:288: Get_density_cor(elec_cor, st_elec_up, st_elec_down, ..., 'F', ..., xi1, xi1)
std::vector<cplx> Oracle::elec_cor(int xi) { return oper_cor(st_elec_up, st_elec_down, 'F', xi); }

}  // namespace orc
