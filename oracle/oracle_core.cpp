// Oracle core: lattice set-up, site operators, bases, SU(2) coefficients, BLAS
// bindings, wave and block algebra.  TEST INFRASTRUCTURE ONLY (see oracle.hpp).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>

#include "oracle.hpp"

extern "C" {
void scipy_zgemm_(const char*, const char*, const int*, const int*, const int*, const void*,
                  const void*, const int*, const void*, const int*, const void*, void*, const int*);
void scipy_zheev_(const char*, const char*, const int*, void*, const int*, double*, void*,
                  const int*, double*, int*);
void scipy_dstev_(const char*, const int*, double*, double*, double*, const int*, double*, int*);
}

namespace orc {

double g_gemm_flops = 0.0;

void zgemm(char ta, char tb, int m, int n, int k, cplx alpha, const cplx* a, int lda,
           const cplx* b, int ldb, cplx beta, cplx* c, int ldc) {
  if (m <= 0 || n <= 0) return;
  if (k <= 0) {  // BLAS semantics: C = beta*C
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < m; ++i) c[(size_t)j * ldc + i] *= beta;
    return;
  }
  g_gemm_flops += 8.0 * m * n * k;
  scipy_zgemm_(&ta, &tb, &m, &n, &k, &alpha, a, &lda, b, &ldb, &beta, c, &ldc);
}

// FACTRL (block.f90:3688-3696): factorials as the reference builds them.
static double FACT[302];
static bool fact_ready = false;
static void factrl() {
  if (fact_ready) return;
  FACT[0] = 1.0;
  for (int i = 1; i <= 160; ++i) FACT[i] = FACT[i - 1] * (double)(float)i;
  fact_ready = true;
}

// W6JS (block.f90:3744-3795): Racah formula, doubled angular momenta.
double w6js(int J1, int J2, int J3, int L1, int L2, int L3) {
  factrl();
  int IA = J1 + J2;
  if (IA < J3) return 0.0;
  int IB = J1 - J2;
  if (std::abs(IB) > J3) return 0.0;
  int IC = J1 + L2;
  if (IC < L3) return 0.0;
  int ID = J1 - L2;
  if (std::abs(ID) > L3) return 0.0;
  int IE = L1 + J2;
  if (IE < L3) return 0.0;
  int IF = L1 - J2;
  if (std::abs(IF) > L3) return 0.0;
  int IG = L1 + L2;
  if (IG < J3) return 0.0;
  int IH = L1 - L2;
  if (std::abs(IH) > J3) return 0.0;
  int SUM1 = IA + J3, SUM2 = IC + L3, SUM3 = IE + L3, SUM4 = IG + J3;
  if (SUM1 % 2 || SUM2 % 2 || SUM3 % 2 || SUM4 % 2) return 0.0;
  int WMIN = std::max(std::max(SUM1, SUM2), std::max(SUM3, SUM4));
  int II = IA + IG, IJ = J2 + J3 + L2 + L3, IK = J3 + J1 + L3 + L1;
  int WMAX = std::min(II, std::min(IJ, IK));
  double OMEGA = 0.0;
  for (int W = WMIN; W <= WMAX; W += 2) {
    double DENOM = FACT[(W - SUM1) / 2] * FACT[(W - SUM2) / 2] * FACT[(W - SUM3) / 2] *
                   FACT[(W - SUM4) / 2] * FACT[(II - W) / 2] * FACT[(IJ - W) / 2] *
                   FACT[(IK - W) / 2];
    if (W % 4 != 0) DENOM = -DENOM;
    OMEGA = OMEGA + FACT[W / 2 + 1] / DENOM;
  }
  double T1 = FACT[(IA - J3) / 2] * FACT[(J3 + IB) / 2] * FACT[(J3 - IB) / 2] / FACT[SUM1 / 2 + 1];
  double T2 = FACT[(IC - L3) / 2] * FACT[(L3 + ID) / 2] * FACT[(L3 - ID) / 2] / FACT[SUM2 / 2 + 1];
  double T3 = FACT[(IE - L3) / 2] * FACT[(L3 + IF) / 2] * FACT[(L3 - IF) / 2] / FACT[SUM3 / 2 + 1];
  double T4 = FACT[(IG - J3) / 2] * FACT[(J3 + IH) / 2] * FACT[(J3 - IH) / 2] / FACT[SUM4 / 2 + 1];
  double THETA = T1 * T2 * T3 * T4;
  return OMEGA * std::sqrt(THETA);
}

// W3JS (block.f90:3702-3741), kept for the coefficient tests.
double w3js(int J1, int J2, int J3, int M1, int M2, int M3) {
  factrl();
  if (M1 + M2 + M3 != 0) return 0.0;
  int IA = J1 + J2;
  if (J3 > IA) return 0.0;
  int IB = J1 - J2;
  if (J3 < std::abs(IB)) return 0.0;
  int JSUM = J3 + IA, IC = J1 - M1, ID = J2 - M2;
  if (JSUM % 2 || IC % 2 || ID % 2) return 0.0;
  if (std::abs(M1) > J1 || std::abs(M2) > J2 || std::abs(M3) > J3) return 0.0;
  int IE = J3 - J2 + M1, IF = J3 - J1 - M2;
  int ZMIN = std::max(0, std::max(-IE, -IF));
  int IG = IA - J3, IH = J2 + M2;
  int ZMAX = std::min(IG, std::min(IH, IC));
  double CC = 0.0;
  for (int Z = ZMIN; Z <= ZMAX; Z += 2) {
    double DENOM = FACT[Z / 2] * FACT[(IG - Z) / 2] * FACT[(IC - Z) / 2] * FACT[(IH - Z) / 2] *
                   FACT[(IE + Z) / 2] * FACT[(IF + Z) / 2];
    if (Z % 4 != 0) DENOM = -DENOM;
    CC = CC + 1.0 / DENOM;
  }
  double CC1 = FACT[IG / 2] * FACT[(J3 + IB) / 2] * FACT[(J3 - IB) / 2] / FACT[(JSUM + 2) / 2];
  double CC2 = FACT[(J1 + M1) / 2] * FACT[IC / 2] * FACT[IH / 2] * FACT[ID / 2] *
               FACT[(J3 - M3) / 2] * FACT[(J3 + M3) / 2];
  CC = CC * std::sqrt(CC1 * CC2);
  if (((IB - M3) % 4 + 4) % 4 != 0) CC = -CC;
  return CC;
}

// ---- block algebra (block.f90:2-367) -------------------------------------------
void block_transfer_trans(const Block& in, Block& out) {   // block.f90:33-64
  out.len = in.len;
  out.num = in.num;
  out.dim = 0;
  out.up_dif = -in.up_dif;
  out.down_dif = in.down_dif;
  out.sub.assign(in.num, SubBlock());
  for (int i = 0; i < in.num; ++i) {
    const SubBlock& s = in.sub[i];
    SubBlock& o = out.sub[i];
    o.num_up = s.num_up + in.up_dif;
    o.num_down = s.num_down + s.down_dif;
    o.down_dif = -s.down_dif;
    o.row_dim = s.sdim;
    o.sdim = s.row_dim;
    out.dim += o.sdim;
    o.mat.assign((size_t)o.row_dim * o.sdim, 0.0);
    for (int c = 0; c < o.sdim; ++c)
      for (int r = 0; r < o.row_dim; ++r) o.at(r, c) = std::conj(s.at(c, r));
  }
}

void block_pass_info(const Block& ob, Block& nb) {          // block.f90:132-159
  nb.len = ob.len;
  nb.num = ob.num;
  nb.dim = ob.dim;
  nb.up_dif = ob.up_dif;
  nb.down_dif = ob.down_dif;
  nb.sub.assign(ob.num, SubBlock());
  for (int i = 0; i < ob.num; ++i) {
    SubBlock& o = nb.sub[i];
    const SubBlock& s = ob.sub[i];
    o.num_up = s.num_up;
    o.num_down = s.num_down;
    o.down_dif = s.down_dif;
    o.row_dim = s.row_dim;
    o.sdim = s.sdim;
    o.mat.assign((size_t)o.row_dim * o.sdim, 0.0);
  }
}

void block_add_block_two(const Block& b1, cplx coef1, Block& nb) {  // block.f90:177-215
  int x1 = 0;
  for (int i = 0; i < nb.num; ++i) {
    SubBlock& o = nb.sub[i];
    int idx1 = -1;
    for (int x = x1; x < b1.num; ++x) {
      const SubBlock& s = b1.sub[x];
      if (s.num_up == o.num_up && s.num_down == o.num_down && s.down_dif == o.down_dif) {
        idx1 = x;
        x1 = x + 1;
        break;
      }
    }
    if (idx1 >= 0) {
      const SubBlock& s = b1.sub[idx1];
      for (size_t e = 0; e < o.mat.size(); ++e) o.mat[e] += coef1 * s.mat[e];
    }
  }
}

// ---- wave algebra (block.f90:952-1354) ----------------------------------------
void Oracle::allocate_wave(const Super& s, Wave& w) {       // block.f90:952-979
  w.sys_len = s.sys_len;
  w.env_len = s.env_len;
  w.num = s.num;
  w.dim = s.dim;
  w.sub.assign(s.num, SubWave());
  for (int i = 0; i < s.num; ++i) {
    SubWave& o = w.sub[i];
    const SubSuper& t = s.sub[i];
    o.sys_num_up = t.sys_num_up;
    o.sys_num_down = t.sys_num_down;
    o.env_num_up = t.env_num_up;
    o.env_num_down = t.env_num_down;
    o.sys_dim = t.sys_dim;
    o.env_dim = t.env_dim;
    o.vec.assign((size_t)t.sys_dim * t.env_dim, 0.0);
  }
}

double wave_product(const Wave& l, const Wave& r) {         // block.f90:1092-1108
  double p = 0.0;
  for (int i = 0; i < l.num; ++i) {
    const SubWave& a = l.sub[i];
    const SubWave& b = r.sub[i];
    for (int x = 0; x < a.env_dim; ++x) {
      cplx d = 0.0;
      const cplx* pa = &a.vec[(size_t)x * a.sys_dim];
      const cplx* pb = &b.vec[(size_t)x * b.sys_dim];
      for (int y = 0; y < a.sys_dim; ++y) d += std::conj(pa[y]) * pb[y];
      p = (cplx(p, 0.0) + d).real();
    }
  }
  return p;
}

double wave_norm(const Wave& w) {                           // block.f90:1112-1131
  return std::sqrt(wave_product(w, w));
}

void wave_normalize(Wave& w) {                              // block.f90:1135-1150
  double n = wave_norm(w);
  for (auto& s : w.sub)
    for (auto& v : s.vec) v /= n;
}

// random_number stand-in: splitmix64 -> uniform [0,1) with 53-bit mantissa.
double Oracle::rand01() {
  uint64_t z = (rng_state += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z = z ^ (z >> 31);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

void Oracle::wave_initialize(Wave& w) {                     // block.f90:1154-1180
  for (auto& s : w.sub) {
    size_t n = (size_t)s.sys_dim * s.env_dim;
    std::vector<double> mr(n), mi(n);
    for (size_t e = 0; e < n; ++e) mr[e] = rand01();
    for (size_t e = 0; e < n; ++e) mi[e] = rand01();
    for (size_t e = 0; e < n; ++e) s.vec[e] = cplx(mr[e], mi[e]);
  }
  wave_normalize(w);
}

// ---- lattice (dmrg_sub.f90:304-644) --------------------------------------------
Oracle::Oracle(const Config& c) : cfg(c) {
  rng_state = cfg.seed;
  L.Nx = cfg.Nx;
  L.Ny = cfg.Ny;
  L.nleg = cfg.Ny;
  L.num_site = cfg.Nx * cfg.Ny;
  L.openy = cfg.openy;
  int N = L.num_site;
  L.neib.assign((size_t)(N + 1) * (L.neibt + 1), 0);
  L.neiba.assign((size_t)(N + 1) * (N + 1), 0);
  L.nposi.assign(N + 8, 0);
  L.nposi_dm.assign(N + 8, 0);
  L.nposi_lat.assign(N + 8, 0);
  L.inb1.assign((size_t)(N + 1) * (N + 1), 0);
  L.nleg11.assign(N + 1, 0);
  L.inb.assign(N + 8, 0);
  // couplings, main.f90:59-70 (t1/J1 on bonds 1-6, t2/J2 on bonds 7-12)
  size_t nc = (size_t)(N + 1) * (L.neibt + 1);
  L.jt.assign(nc, 0.0);
  L.jz.assign(nc, 0.0);
  L.jd.assign(nc, 0.0);
  L.jn.assign(nc, 0.0);
  for (int s = 1; s <= N; ++s) {
    for (int k = 1; k <= 6; ++k) {
      L.jz[(size_t)s * (L.neibt + 1) + k] = cfg.J1;
      L.jt[(size_t)s * (L.neibt + 1) + k] = -cfg.t1 * std::sqrt(2.0);
    }
    for (int k = 7; k <= 12; ++k) {
      L.jz[(size_t)s * (L.neibt + 1) + k] = cfg.J2;
      L.jt[(size_t)s * (L.neibt + 1) + k] = -cfg.t2 * std::sqrt(2.0);
    }
    for (int k = 1; k <= 18; ++k) {
      size_t e = (size_t)s * (L.neibt + 1) + k;
      L.jd[e] = L.jz[e] * (-std::sqrt(3.0));
      if (k <= 12) L.jn[e] = -0.25 * L.jz[e];
    }
  }
  site_operators();
  // electron count, main.f90:93-99
  int i = N;
  int q = i / 2 - (i + 2 * cfg.delta - 1) / (2 * cfg.delta);
  tot_num_up = 2 * q;
  tot_num_down = 0;
  dmrg_setup(N / 2 - 1, N / 2 - 1);   // main.f90:81
  setup0();                            // main.f90:82
}

void Oracle::dmrg_setup(int ns, int ns21) {                 // dmrg_sub.f90:334-644
  const int nleg = L.nleg, nly = 1;
  int nn = ns + ns21 + 2;
  int nt = L.num_site;
  L.nxc = (nn - 1) / nleg + 1;
  if (L.nxc == 1) L.nxc = 2;
  std::fill(L.nposi.begin(), L.nposi.end(), 0);
  std::fill(L.nposi_lat.begin(), L.nposi_lat.end(), 0);
  std::fill(L.nposi_dm.begin(), L.nposi_dm.end(), 0);
  std::fill(L.neib.begin(), L.neib.end(), 0);
  std::fill(L.neiba.begin(), L.neiba.end(), 0);
  int totsite = nleg * L.nxc;
  for (int i = 1; i <= ns + 1; ++i) {
    L.nposi[i] = 1;
    L.nposi_lat[i] = i;
    L.nposi_dm[i] = i;
  }
  L.nposi[ns + 1] = 2;
  for (int i = 1; i <= ns21 + 1; ++i) {
    L.nposi[ns + 1 + i] = 3;
    L.nposi_dm[totsite + 1 - i] = i + (ns + 1);
    L.nposi_lat[i + ns + 1] = totsite + 1 - i;
  }
  L.nposi[ns + 1 + ns21 + 1] = 4;
  auto set = [&](int a, int ka, int b, int kb) {
    L.NEIB(a, ka) = b;
    L.NEIB(b, kb) = a;
    L.NEIBA(a, b) = ka;
    L.NEIBA(b, a) = kb;
  };
  // triangle=1 branch (dmrg_sub.f90:453-583)
  for (int ix = 1; ix <= L.nxc; ++ix) {
    for (int iy = 1; iy <= nleg; ++iy) {
      int ii = iy + (ix - 1) * nleg;
      int jy = ii - iy + (iy % nleg) + 1;
      if (L.openy != 0 && iy == nleg) jy = 0;
      if (jy != 0) {
        if (iy != nleg || nleg != 2) set(ii, 1, jy, 2);
      }
      int jx = ii + nleg * nly;
      if (jx > nleg * L.nxc) {
        if (L.open_x == 0 && L.nxc >= 3) jx = jx - nleg * L.nxc;
        else jx = 0;
      }
      if (jx != 0) {
        set(ii, 3, jx, 4);
        jy = jx - 1;
        if (iy == 1) {
          if (L.openy == 0) jy = jy + nleg;
          else jy = 0;
        }
        if (jy != 0) set(ii, 5, jy, 6);
      }
    }
  }
  for (int ix = 1; ix <= L.nxc; ++ix) {
    for (int iy = 1; iy <= nleg; ++iy) {
      int ii = iy + (ix - 1) * nleg;
      int j1 = L.NEIB(ii, 1);
      int j2 = L.NEIB(j1, 3);
      if (j1 * j2 != 0) set(ii, 7, j2, 8);
      if (nleg != 3) {
        j1 = L.NEIB(ii, 3);
        j2 = L.NEIB(j1, 5);
        if (j1 * j2 != 0) set(ii, 9, j2, 10);
      }
      j1 = L.NEIB(ii, 2);
      j2 = L.NEIB(j1, 5);
      if (j1 * j2 != 0) set(ii, 11, j2, 12);
      if (nleg != 3) {
        j1 = L.NEIB(ii, 1);
        j2 = L.NEIB(j1, 1);
        if (j1 * j2 != 0 && L.NEIBA(ii, j2) == 0) set(ii, 13, j2, 14);
      }
      j1 = L.NEIB(ii, 3);
      j2 = L.NEIB(j1, 3);
      if (j1 * j2 != 0 && L.NEIBA(ii, j2) == 0) set(ii, 15, j2, 16);
      j1 = L.NEIB(ii, 5);
      j2 = L.NEIB(j1, 5);
      if (j1 * j2 != 0 && L.NEIBA(ii, j2) == 0) set(ii, 17, j2, 18);
    }
  }
  for (int i = 1; i <= nt; ++i) {
    for (int j = L.neibt1 + 1; j <= L.neibt; ++j) {
      if (std::abs(L.JZ(j, 1)) + std::abs(L.JD(j, 1)) + std::abs(L.JT(j, 1)) +
              std::abs(L.JN(j, 1)) == 0.0) {
        int nb = L.NEIB(i, j);
        L.NEIBA(i, nb) = 0;
        L.NEIBA(nb, i) = 0;
        L.NEIB(i, j) = 0;
      }
    }
  }
}

void Oracle::setup0() {                                     // dmrg_sub.f90:304-331
  std::fill(L.nleg11.begin(), L.nleg11.end(), 0);
  for (int ns = 1; ns <= L.num_site - 2; ++ns) {
    int k0 = 0;
    for (int i1 = 1; i1 <= ns; ++i1) {
      L.INB1(i1, ns) = 10000;
      int k00 = 0;
      for (int j = 1; j <= L.neibt; ++j)
        if (L.NEIB(i1, j) >= ns) k00++;
      if (k00 != 0) {
        k0++;
        L.INB1(i1, ns) = k0;
      }
    }
    L.nleg11[ns] = k0;
  }
}

// ---- site operators (dmrg_sub.f90:733-969) -----------------------------------
static SubBlock sb(int nu, int nd, int dd, double v) {
  SubBlock s;
  s.num_up = nu;
  s.num_down = nd;
  s.down_dif = dd;
  s.row_dim = 1;
  s.sdim = 1;
  s.mat.assign(1, cplx(v, 0.0));
  return s;
}

void Oracle::site_operators() {
  // c^+ : dmrg_sub.f90:743-765
  st_elec_up = Block();
  st_elec_up.len = 1; st_elec_up.num = 1; st_elec_up.dim = 1;
  st_elec_up.up_dif = 1; st_elec_up.down_dif = 1;
  st_elec_up.sub = {sb(0, 0, 1, -std::sqrt(2.0))};
  // c : dmrg_sub.f90:779-784
  st_elec_down = st_elec_up;
  st_elec_down.up_dif = -1;
  st_elec_down.sub[0].num_up = 1;
  st_elec_down.sub[0].num_down = 1;
  st_elec_down.sub[0].down_dif = -1;
  // n : dmrg_sub.f90:795-820 (ss=1)
  num_elec = Block();
  num_elec.len = 1; num_elec.num = 2; num_elec.dim = 2;
  num_elec.sub = {sb(1, 1, 0, std::sqrt(2.0)), sb(0, 0, 0, 0.0)};
  // S : dmrg_sub.f90:845-859
  st_sd = Block();
  st_sd.len = 1; st_sd.num = 1; st_sd.dim = 1; st_sd.up_dif = 0; st_sd.down_dif = 2;
  st_sd.sub = {sb(1, 1, 0, std::sqrt(1.5))};
  // Sz : dmrg_sub.f90:862-886 (used as the site basis template)
  st_sz = Block();
  st_sz.len = 1; st_sz.num = 2; st_sz.dim = 2;
  st_sz.sub = {sb(1, 1, 0, 1.0), sb(0, 0, 0, 0.0)};
  // identity-like : dmrg_sub.f90:902-906
  st_si = num_elec;
  for (auto& s : st_si.sub) s.mat[0] = std::sqrt(1.0 + s.down_dif);
}

void Oracle::hamiltonian_site(Model& m) {                   // dmrg_sub.f90:912-938
  m = Model();
  m.len = 1;
  m.ham = st_sz;
  for (auto& s : m.ham.sub) s.mat[0] = 0.0;
  m.sub.assign(L.num_site + 1, BlockSet());
  m.sub[1].elec_up = st_elec_up;
  m.sub[1].elec_down = st_elec_down;
  m.sub[1].spin_sd = st_sd;
  m.sub[1].num_sn = num_elec;
  m.sub_s.assign(L.num_site + 1, BlockSet());
}

// ---- bases (block.f90:2087-2349) ----------------------------------------------
static void quicksort_integer(std::vector<std::pair<int, int>>& a) {  // block.f90:2316-2349
  int num = (int)a.size();
  for (int i = 0; i < num; ++i)
    for (int x = i + 1; x < num; ++x)
      if (a[i].second < a[x].second) std::swap(a[i], a[x]);
  for (int i = 0; i < num; ++i)
    for (int x = i + 1; x < num; ++x)
      if (a[i].second == a[x].second && a[i].first < a[x].first) std::swap(a[i], a[x]);
}

void Oracle::get_basis(const Block& block, const Block& site, Basis& basis) {  // block.f90:2087-2188
  basis = Basis();
  basis.len = block.len + site.len;
  std::vector<std::pair<int, int>> pre;
  for (int i = 0; i < block.num; ++i)
    for (int j = 0; j < site.num; ++j) {
      int s1 = std::abs(block.sub[i].num_down - site.sub[j].num_down);
      int s2 = block.sub[i].num_down + site.sub[j].num_down;
      for (int ss = s1; ss <= s2; ss += 2)
        pre.push_back({block.sub[i].num_up + site.sub[j].num_up, ss});
    }
  quicksort_integer(pre);
  // Get_Unique_QN (block.f90:2251-2286) on the sorted list
  std::vector<std::pair<int, int>> res;
  for (auto& p : pre)
    if (res.empty() || res.back() != p) res.push_back(p);
  basis.num = (int)res.size();
  basis.sub.assign(basis.num, BasisMap());
  for (int i = 0; i < basis.num; ++i) {
    BasisMap& bm = basis.sub[i];
    bm.new_num_up = res[i].first;
    bm.new_num_down = res[i].second;
    bm.idx = 0;
    bm.dim = 0;
    for (int x = 0; x < block.num; ++x)
      for (int y = 0; y < site.num; ++y) {
        if (block.sub[x].num_up + site.sub[y].num_up != bm.new_num_up) continue;
        int s1 = std::abs(block.sub[x].num_down - site.sub[y].num_down);
        int s2 = block.sub[x].num_down + site.sub[y].num_down;
        if (bm.new_num_down >= s1 && bm.new_num_down <= s2) {
          SubBasisMap p;
          p.bl_num_up = block.sub[x].num_up;
          p.bl_num_down = block.sub[x].num_down;
          p.st_num_up = site.sub[y].num_up;
          p.st_num_down = site.sub[y].num_down;
          p.sdim = block.sub[x].sdim * site.sub[y].sdim;
          p.spos = bm.dim;
          bm.dim += p.sdim;
          bm.sub.push_back(p);
          bm.idx++;
        }
      }
    bm.num = (int)bm.sub.size();
  }
  basis.dim = 0;
  for (auto& b : basis.sub) basis.dim += b.dim;
}

void Oracle::get_super_basis(const Basis& sys_bs, const Basis& env_bs, Super& super,
                             int total_up, int total_down) {   // block.f90:2194-2247
  super = Super();
  super.sys_len = sys_bs.len;
  super.env_len = env_bs.len;
  super.dim = 0;
  for (int x = 0; x < sys_bs.num; ++x)
    for (int y = 0; y < env_bs.num; ++y) {
      if (env_bs.sub[y].new_num_up != total_up - sys_bs.sub[x].new_num_up) continue;
      int s1 = std::abs(env_bs.sub[y].new_num_down - sys_bs.sub[x].new_num_down);
      int s2 = env_bs.sub[y].new_num_down + sys_bs.sub[x].new_num_down;
      if (total_down >= s1 && total_down <= s2) {
        SubSuper s;
        s.sys_num_up = sys_bs.sub[x].new_num_up;
        s.sys_num_down = sys_bs.sub[x].new_num_down;
        s.env_num_up = env_bs.sub[y].new_num_up;
        s.env_num_down = env_bs.sub[y].new_num_down;
        s.sys_dim = sys_bs.sub[x].dim;
        s.env_dim = env_bs.sub[y].dim;
        super.dim += s.sys_dim * s.env_dim;
        super.sub.push_back(s);
      }
    }
  super.num = (int)super.sub.size();
  super.idx = super.num;
}

}  // namespace orc
