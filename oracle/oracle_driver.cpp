// Oracle sweep drivers (dmrg_sub.f90:974-1465, main.f90:114-209), flat
// serialisation of superblocks and the extern "C" surface used by tests/ and
// bench.py's cpu_baseline leg.  TEST INFRASTRUCTURE ONLY (see oracle.hpp).
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>

#include "oracle.hpp"

namespace orc {

namespace {
// block_transfer_basis + identity (dmrg_sub.f90:1080-1086)
void identity_trun(const Basis& bs, Block& t) {
  t = Block();
  t.len = bs.len;
  t.num = bs.num;
  t.dim = bs.dim;
  t.sub.assign(bs.num, SubBlock());
  for (int i = 0; i < bs.num; ++i) {
    SubBlock& s = t.sub[i];
    s.num_up = bs.sub[i].new_num_up;
    s.num_down = bs.sub[i].new_num_down;
    s.row_dim = s.sdim = bs.sub[i].dim;
    s.mat.assign((size_t)s.sdim * s.sdim, 0.0);
    for (int j = 0; j < s.sdim; ++j) s.at(j, j) = 1.0;
  }
}
}  // namespace

void Oracle::step_capture_pre(Model& sys, Model& env, const Basis& sys_bs, const Basis& env_bs,
                              const Super& super, const Wave& psi0) {
  cap.valid = true;
  cap.sys = sys;
  cap.env = env;
  cap.sys_bs = sys_bs;
  cap.env_bs = env_bs;
  cap.super = super;
  cap.psi0 = psi0;
  cap.nxc = L.nxc;
  Model s2 = sys, e2 = env;
  hmerge(s2, e2, sys_bs, env_bs);
  allocate_wave(super, cap.hpsi);
  long long c0 = hpsi_calls;
  double t0 = hpsi_seconds, f0 = hpsi_flops;
  model_wave(s2, e2, sys_bs, env_bs, psi0, cap.hpsi);
  hpsi_calls = c0;   // the capture's own H.psi is not part of the step accounting
  hpsi_seconds = t0;
  hpsi_flops = f0;
}

// warm_up_point, dmrg_sub.f90:974-1147 (levels=1)
void Oracle::warm_up_point(int bg_id, int end_id, double trun_err, std::vector<StepLog>* log) {
  (void)bg_id;
  int label = 1;
  dmrg_setup(1, 1);
  Model sys, env;
  hamiltonian_site(sys);
  hamiltonian_site(env);
  sys_models[1] = sys;
  env_models[1] = env;
  while (label + 1 <= end_id) {
    Basis sys_bs, env_bs;
    get_basis(sys.ham, st_sz, sys_bs);
    get_basis(env.ham, st_sz, env_bs);
    dmrg_setup(sys.ham.len, env.ham.len);
    float v = 1.0f * (float)(sys_bs.len + env_bs.len) / (float)L.num_site * (float)tot_num_up + 0.001f;
    int tot_up = (int)v;
    tot_up = tot_up - tot_up % 2;
    int tot_down = 0;
    if (tot_up > tot_num_up) tot_up = tot_num_up;
    if (tot_down > tot_num_down) tot_down = tot_num_down;
    Super super;
    get_super_basis(sys_bs, env_bs, super, tot_up, tot_down);
    Wave eig;
    allocate_wave(super, eig);
    wave_initialize(eig);
    StepLog sl{};
    sl.phase = 0;
    sl.sys_len = sys.len;
    sl.env_len = env.len;
    bool capnow = (lanczos_calls == capture_step);
    if (capnow) step_capture_pre(sys, env, sys_bs, env_bs, super, eig);
    long long c0 = hpsi_calls;
    double t0 = hpsi_seconds, f0 = hpsi_flops;
    lanczos_memo_new(sys, env, sys_bs, env_bs, super, eig, &sl.lanczos_iters, &sl.e0);
    lanczos_calls++;
    Block sys_den, env_den, sys_trun, env_trun;
    density_matrix_sys(eig, sys_den);
    density_matrix_env(eig, env_den);
    int ns = 0;
    double err = 0, ent = 0, entm = 0;
    std::vector<double> spec;
    if (sys_bs.dim <= kept_max) {
      identity_trun(sys_bs, sys_trun);
      ns = sys_bs.dim;
    } else {
      truncation_operator(sys_den, sys_trun, trun_err, &ns, &err, &ent, &entm, true, &spec);
    }
    sl.num_state = ns;
    sl.trun_err = err;
    sl.entropy = ent;
    sl.entropy_mult = entm;
    if (capnow) {
      cap.gs = eig;
      cap.e0 = sl.e0;
      cap.iters = sl.lanczos_iters;
      cap.den = sys_den;
      cap.trun = sys_trun;
      cap.num_state = ns;
      cap.err = err;
      cap.ent = ent;
      cap.ent_mult = entm;
      cap.spectrum = spec;
      cap.sys_side = true;
      cap.grow_basis = sys_bs;
    }
    mshift = 0;
    hamiltonian_sys(sys, sys_bs, sys_trun);
    if (capnow) cap.grown = sys;
    if (env_bs.dim <= kept_max) {
      identity_trun(env_bs, env_trun);
    } else {
      int ns2;
      double e2, en2, em2;
      truncation_operator(env_den, env_trun, trun_err, &ns2, &e2, &en2, &em2, false, nullptr);
    }
    mshift = sys.len;
    hamiltonian_env(env, env_bs, env_trun);
    sys_models[label + 1] = sys;
    env_models[label + 1] = env;
    sys_truns[label + 1] = sys_trun;
    env_truns[label + 1] = env_trun;
    sys_bsm[label + 1] = sys_bs;
    env_bsm[label + 1] = env_bs;
    disk_wave = eig;
    sl.hpsi_calls = (int)(hpsi_calls - c0);
    sl.hpsi_seconds = hpsi_seconds - t0;
    sl.hpsi_flops = hpsi_flops - f0;
    if (log) log->push_back(sl);
    label++;
  }
}

// left_to_right, dmrg_sub.f90:1151-1302 (levels=1)
void Oracle::left_to_right(int bg_id, int end_id, double trun_err, std::vector<StepLog>* log) {
  const int N = L.num_site;
  int label = bg_id;
  Model sys = sys_models.at(label);
  Model env = env_models.at(N - label - 2);
  dmrg_setup(sys.ham.len, env.ham.len);
  mshift = 0;
  Basis sys_bs, env_bs;
  get_basis(sys.ham, st_sz, sys_bs);
  get_basis(env.ham, st_sz, env_bs);
  Super super;
  get_super_basis(sys_bs, env_bs, super, tot_num_up, tot_num_down);
  Wave eig;
  Block sys_trun, env_trun;
  bool first = true;
  while (true) {
    if (!first) {
      if (!(label + 1 <= end_id)) break;
      get_basis(sys.ham, st_sz, sys_bs);
      env_bs = env_bsm.at(N - label - 1);
      Basis env_basis = env_bsm.at(N - label);
      env = env_models.at(N - label - 2);
      dmrg_setup(sys.ham.len, env.ham.len);
      get_super_basis(sys_bs, env_bs, super, tot_num_up, tot_num_down);
      env_trun = env_truns.at(N - label - 1);
      Wave tmp;
      allocate_wave(super, tmp);
      bool capnow = (lanczos_calls == capture_step);
      if (capnow) {
        cap.has_wt = true;
        cap.wt_lr = true;
        cap.wt_sys_bs = sys_bs;
        cap.wt_env_bs = env_basis;
        cap.wt_sys_trun = sys_trun;
        cap.wt_env_trun = env_trun;
        cap.wt_old = eig;
        cap.wt_super = super;
      }
      wave_trans_LR(sys_bs, env_basis, sys_trun, env_trun, eig, tmp);
      eig = tmp;
      if (capnow) cap.wt_new = eig;
    } else {
      if (restart1 == 0) {
        allocate_wave(super, eig);
        wave_initialize(eig);
      } else {
        eig = disk_wave;
        if (eig.sys_len != super.sys_len) {
          Basis env_basis = env_bsm.at(N - label);
          Block st = sys_truns.at(label), et = env_truns.at(N - label - 1);
          Wave tmp;
          allocate_wave(super, tmp);
          wave_trans_LR(sys_bs, env_basis, st, et, eig, tmp);
          eig = tmp;
        }
      }
    }
    StepLog sl{};
    sl.phase = 1;
    sl.sys_len = sys.len;
    sl.env_len = env.len;
    bool capnow = (lanczos_calls == capture_step);
    if (capnow) step_capture_pre(sys, env, sys_bs, env_bs, super, eig);
    long long c0 = hpsi_calls;
    double t0 = hpsi_seconds, f0 = hpsi_flops;
    lanczos_memo_new(sys, env, sys_bs, env_bs, super, eig, &sl.lanczos_iters, &sl.e0);
    lanczos_calls++;
    Block sys_den;
    density_matrix_sys(eig, sys_den);
    disk_wave = eig;
    std::vector<double> spec;
    truncation_operator(sys_den, sys_trun, trun_err, &sl.num_state, &sl.trun_err, &sl.entropy,
                        &sl.entropy_mult, true, &spec);
    if (capnow) {
      cap.gs = eig;
      cap.e0 = sl.e0;
      cap.iters = sl.lanczos_iters;
      cap.den = sys_den;
      cap.trun = sys_trun;
      cap.num_state = sl.num_state;
      cap.err = sl.trun_err;
      cap.ent = sl.entropy;
      cap.ent_mult = sl.entropy_mult;
      cap.spectrum = spec;
      cap.sys_side = true;
      cap.grow_basis = sys_bs;
    }
    mshift = 0;
    hamiltonian_sys(sys, sys_bs, sys_trun);
    if (capnow) cap.grown = sys;
    sys_models[label + 1] = sys;
    sys_truns[label + 1] = sys_trun;
    sys_bsm[label + 1] = sys_bs;
    sl.hpsi_calls = (int)(hpsi_calls - c0);
    sl.hpsi_seconds = hpsi_seconds - t0;
    sl.hpsi_flops = hpsi_flops - f0;
    if (log) log->push_back(sl);
    label++;
    first = false;
  }
}

// right_to_left, dmrg_sub.f90:1306-1465 (levels=1)
void Oracle::right_to_left(int bg_id, int end_id, double trun_err, std::vector<StepLog>* log) {
  const int N = L.num_site;
  int label = bg_id;
  Model sys = sys_models.at(label - 1);
  Model env = env_models.at(N - label - 1);
  dmrg_setup(sys.ham.len, env.ham.len);
  Basis sys_bs, env_bs;
  get_basis(sys.ham, st_sz, sys_bs);
  get_basis(env.ham, st_sz, env_bs);
  Super super;
  get_super_basis(sys_bs, env_bs, super, tot_num_up, tot_num_down);
  Wave eig;
  Block sys_trun, env_trun;
  bool first = true;
  while (true) {
    if (!first) {
      if (!(label - 1 >= end_id)) break;
      sys_bs = sys_bsm.at(label);
      Basis sys_basis = sys_bsm.at(label + 1);
      get_basis(env.ham, st_sz, env_bs);
      get_super_basis(sys_bs, env_bs, super, tot_num_up, tot_num_down);
      sys = sys_models.at(label - 1);
      dmrg_setup(sys.ham.len, env.ham.len);
      sys_trun = sys_truns.at(label);
      Wave tmp;
      allocate_wave(super, tmp);
      bool capnow = (lanczos_calls == capture_step);
      if (capnow) {
        cap.has_wt = true;
        cap.wt_lr = false;
        cap.wt_sys_bs = sys_basis;
        cap.wt_env_bs = env_bs;
        cap.wt_sys_trun = sys_trun;
        cap.wt_env_trun = env_trun;
        cap.wt_old = eig;
        cap.wt_super = super;
      }
      wave_trans_RL(sys_basis, env_bs, sys_trun, env_trun, eig, tmp);
      eig = tmp;
      if (capnow) cap.wt_new = eig;
    } else {
      if (restart1 == 0) {
        allocate_wave(super, eig);
        wave_initialize(eig);
      } else {
        eig = disk_wave;
        if (eig.sys_len != super.sys_len) {
          Basis sys_basis = sys_bsm.at(label + 1);
          Block st = sys_truns.at(label), et = env_truns.at(N - label - 1);
          Wave tmp;
          allocate_wave(super, tmp);
          wave_trans_RL(sys_basis, env_bs, st, et, eig, tmp);
          eig = tmp;
        }
      }
    }
    StepLog sl{};
    sl.phase = 2;
    sl.sys_len = sys.len;
    sl.env_len = env.len;
    bool capnow = (lanczos_calls == capture_step);
    if (capnow) step_capture_pre(sys, env, sys_bs, env_bs, super, eig);
    long long c0 = hpsi_calls;
    double t0 = hpsi_seconds, f0 = hpsi_flops;
    lanczos_memo_new(sys, env, sys_bs, env_bs, super, eig, &sl.lanczos_iters, &sl.e0);
    lanczos_calls++;
    Block env_den;
    density_matrix_env(eig, env_den);
    disk_wave = eig;
    std::vector<double> spec;
    truncation_operator(env_den, env_trun, trun_err, &sl.num_state, &sl.trun_err, &sl.entropy,
                        &sl.entropy_mult, false, &spec);
    if (capnow) {
      cap.gs = eig;
      cap.e0 = sl.e0;
      cap.iters = sl.lanczos_iters;
      cap.den = env_den;
      cap.trun = env_trun;
      cap.num_state = sl.num_state;
      cap.err = sl.trun_err;
      cap.ent = sl.entropy;
      cap.ent_mult = sl.entropy_mult;
      cap.spectrum = spec;
      cap.sys_side = false;
      cap.grow_basis = env_bs;
    }
    mshift = sys.len + 1;
    hamiltonian_env(env, env_bs, env_trun);
    if (capnow) cap.grown = env;
    env_models[N - label] = env;
    env_truns[N - label] = env_trun;
    env_bsm[N - label] = env_bs;
    sl.hpsi_calls = (int)(hpsi_calls - c0);
    sl.hpsi_seconds = hpsi_seconds - t0;
    sl.hpsi_flops = hpsi_flops - f0;
    if (log) log->push_back(sl);
    label--;
    first = false;
  }
}

// Get_Ground_State, main.f90:114-209 (restart1=restart2=0, levels=1)
void Oracle::run(std::vector<StepLog>* log) {
  const int N = L.num_site;
  const double lanerr = cfg.lanerr_single ? (double)(float)cfg.lanerr : cfg.lanerr;
  const double trun_err = cfg.trun_err;
  auto lz = [&](double v) { return cfg.lanzero_override > 0 ? cfg.lanzero_override : v; };
  kept_min = cfg.kept_min;
  kept_max = cfg.kept_max_warmup;
  restart1 = 0;
  restart2 = 0;
  lanzero = lz(lanerr * 1000);
  double tmp_err = trun_err * 100;
  warm_up_point(1, N / 2, tmp_err, log);
  lanzero = lz(lanerr * 15);
  tmp_err = trun_err * 15;
  int idx1 = 1;
  restart1 = restart2;
  left_to_right(N / 2 - 1, N - idx1 - 1, tmp_err, log);
  restart1 = 1;
  restart2 = 1;
  right_to_left(N - idx1 - 1, idx1, tmp_err, log);
  restart1 = 1;
  int nsweeps = (int)cfg.sweep_kept_max.size();
  for (int iter = 1; iter <= nsweeps; ++iter) {
    kept_max = cfg.sweep_kept_max[iter - 1];
    if (kept_min > kept_max) kept_min = kept_max;
    lanzero = lz(lanerr);
    tmp_err = trun_err;
    if (iter >= 5) lanzero = lz(lanerr * 0.5);
    left_to_right(idx1, N - idx1 - 1, tmp_err, log);
    right_to_left(N - idx1 - 1, idx1, tmp_err, log);
  }
  if (cfg.final_half_sweep) left_to_right(idx1, cfg.final_stop > 0 ? cfg.final_stop : 5 * N / 6 - 1, tmp_err, log);
}

// ---- flat serialisation ---------------------------------------------------------
struct Ser {
  std::vector<int> ints;
  std::vector<cplx> data;
  void block(const Block& b) {
    ints.insert(ints.end(), {b.len, b.num, b.dim, b.up_dif, b.down_dif});
    for (const auto& s : b.sub) {
      ints.insert(ints.end(), {s.num_up, s.num_down, s.down_dif, s.row_dim, s.sdim});
      data.insert(data.end(), s.mat.begin(), s.mat.end());
    }
  }
  void basis(const Basis& b) {
    ints.insert(ints.end(), {b.len, b.num, b.dim});
    for (const auto& s : b.sub) ints.insert(ints.end(), {s.new_num_up, s.new_num_down, s.dim, s.num});
    for (const auto& s : b.sub)
      for (const auto& p : s.sub)
        ints.insert(ints.end(), {p.bl_num_up, p.bl_num_down, p.st_num_up, p.st_num_down, p.spos, p.sdim});
  }
  void wave(const Wave& w) {
    ints.insert(ints.end(), {w.sys_len, w.env_len, w.num, w.dim});
    for (const auto& s : w.sub) {
      ints.insert(ints.end(), {s.sys_num_up, s.sys_num_down, s.env_num_up, s.env_num_down, s.sys_dim, s.env_dim});
      data.insert(data.end(), s.vec.begin(), s.vec.end());
    }
  }
  void model(const Model& m, int nops) {
    ints.insert(ints.end(), {m.len, nops});
    block(m.ham);
    for (int i = 1; i <= nops; ++i) {
      block(m.sub[i].elec_up);
      block(m.sub[i].elec_down);
      block(m.sub[i].spin_sd);
      block(m.sub[i].num_sn);
    }
  }
};

struct Des {
  const int* ip;
  const cplx* dp;
  int i() { return *ip++; }
  Block block() {
    Block b;
    b.len = i(); b.num = i(); b.dim = i(); b.up_dif = i(); b.down_dif = i();
    b.sub.resize(b.num);
    for (auto& s : b.sub) {
      s.num_up = i(); s.num_down = i(); s.down_dif = i(); s.row_dim = i(); s.sdim = i();
      s.mat.assign(dp, dp + (size_t)s.row_dim * s.sdim);
      dp += (size_t)s.row_dim * s.sdim;
    }
    return b;
  }
  Basis basis() {
    Basis b;
    b.len = i(); b.num = i(); b.dim = i();
    b.sub.resize(b.num);
    for (auto& s : b.sub) {
      s.new_num_up = i(); s.new_num_down = i(); s.dim = i(); s.num = i();
      s.idx = s.num;
    }
    for (auto& s : b.sub) {
      s.sub.resize(s.num);
      for (auto& p : s.sub) {
        p.bl_num_up = i(); p.bl_num_down = i(); p.st_num_up = i(); p.st_num_down = i();
        p.spos = i(); p.sdim = i();
      }
    }
    return b;
  }
  Wave wave() {
    Wave w;
    w.sys_len = i(); w.env_len = i(); w.num = i(); w.dim = i();
    w.sub.resize(w.num);
    for (auto& s : w.sub) {
      s.sys_num_up = i(); s.sys_num_down = i(); s.env_num_up = i(); s.env_num_down = i();
      s.sys_dim = i(); s.env_dim = i();
      s.vec.assign(dp, dp + (size_t)s.sys_dim * s.env_dim);
      dp += (size_t)s.sys_dim * s.env_dim;
    }
    return w;
  }
  Model model(int num_site) {
    Model m;
    m.len = i();
    int nops = i();
    m.ham = block();
    m.sub.assign(num_site + 1, BlockSet());
    m.sub_s.assign(num_site + 1, BlockSet());
    for (int k = 1; k <= nops; ++k) {
      m.sub[k].elec_up = block();
      m.sub[k].elec_down = block();
      m.sub[k].spin_sd = block();
      m.sub[k].num_sn = block();
    }
    return m;
  }
};

}  // namespace orc

// ---- extern "C" surface ----------------------------------------------------------
using namespace orc;

struct OrcHandle {
  Config cfg;
  Oracle* o = nullptr;
  std::vector<StepLog> log;
  std::string err;
  Ser ser;
};

extern "C" {

void* orc_new(int Nx, int Ny, double t1, double t2, double J1, double J2, int delta, int kept_min,
              int kept_warm, const int* sweep_kept, int nsweeps, double lanzero_override,
              unsigned long long seed, int capture_step, int final_half_sweep) {
  OrcHandle* h = new OrcHandle();
  Config& c = h->cfg;
  c.Nx = Nx; c.Ny = Ny; c.t1 = t1; c.t2 = t2; c.J1 = J1; c.J2 = J2; c.delta = delta;
  c.kept_min = kept_min; c.kept_max_warmup = kept_warm;
  c.sweep_kept_max.assign(sweep_kept, sweep_kept + nsweeps);
  c.lanzero_override = lanzero_override;
  c.seed = seed;
  c.final_half_sweep = final_half_sweep != 0;
  try {
    h->o = new Oracle(c);
    h->o->capture_step = capture_step;
  } catch (std::exception& e) {
    h->err = e.what();
  }
  return h;
}

// test knob: where the final half sweep stops (0: the reference's 5 Num_site / 6 - 1)
void orc_set_final_stop(void* hp, int label) { ((OrcHandle*)hp)->o->cfg.final_stop = label; }

void orc_free(void* hp) {
  OrcHandle* h = (OrcHandle*)hp;
  delete h->o;
  delete h;
}

const char* orc_error(void* hp) { return ((OrcHandle*)hp)->err.c_str(); }

int orc_run(void* hp) {
  OrcHandle* h = (OrcHandle*)hp;
  if (!h->o) return -1;
  try {
    h->o->run(&h->log);
  } catch (std::exception& e) {
    h->err = e.what();
    return -1;
  }
  return (int)h->log.size();
}

int orc_tot_num_up(void* hp) { return ((OrcHandle*)hp)->o->tot_num_up; }

// <n_i> of the last ground state (measure_operator_dia); writes num_site values
int orc_measure_density(void* hp, double* out) {
  OrcHandle* h = (OrcHandle*)hp;
  if (!h->o) return -1;
  try {
    std::vector<double> d = h->o->measure_density();
    std::copy(d.begin(), d.end(), out);
    return (int)d.size();
  } catch (std::exception& e) {
    h->err = e.what();
    return -1;
  }
}

int orc_oper_cor(void* hp, int kind, int site, double* out);

// singlet pair correlations: up to maxrec records of 6 doubles (s1, s2, s3, s4, re, im);
// returns the number of records
int orc_pair_cor(void* hp, int xc1, int xc2, int ij, int ij1, double* out, int maxrec) {
  OrcHandle* h = (OrcHandle*)hp;
  if (!h->o) return -1;
  try {
    std::vector<orc::Oracle::PairRec> r = h->o->pair_cor(xc1, xc2, ij, ij1);
    for (size_t k = 0; k < r.size() && (int)k < maxrec; ++k) {
      double* o = out + 6 * k;
      o[0] = r[k].s1;
      o[1] = r[k].s2;
      o[2] = r[k].s3;
      o[3] = r[k].s4;
      o[4] = r[k].value.real();
      o[5] = r[k].value.imag();
    }
    return (int)r.size();
  } catch (std::exception& e) {
    h->err = e.what();
    return -1;
  }
}

// <n_site n_j> of the last ground state (Get_density_cor): 2 * num_site doubles
// (re, im) for j = 1..num_site, zero where the reference computes nothing
int orc_density_cor(void* hp, int site, double* out) { return orc_oper_cor(hp, 0, site, out); }

// kind 0: <n_site n_j> (num_elec), 1: <S_site . S_j> (st_sd), 2: electron correlation
// (st_elec_up, st_elec_down, 'F'); 2 * num_site doubles
int orc_oper_cor(void* hp, int kind, int site, double* out) {
  OrcHandle* h = (OrcHandle*)hp;
  if (!h->o) return -1;
  try {
    std::vector<orc::cplx> d =
        kind == 1 ? h->o->spin_cor(site) : kind == 2 ? h->o->elec_cor(site) : h->o->density_cor(site);
    for (size_t j = 1; j < d.size(); ++j) {
      out[2 * (j - 1)] = d[j].real();
      out[2 * (j - 1) + 1] = d[j].imag();
    }
    return (int)d.size() - 1;
  } catch (std::exception& e) {
    h->err = e.what();
    return -1;
  }
}

// 12 doubles per step: phase, sys_len, env_len, e0, iters, num_state, trun_err,
// entropy, entropy_mult, hpsi_calls, hpsi_seconds, hpsi_flops
int orc_steps(void* hp, double* out) {
  OrcHandle* h = (OrcHandle*)hp;
  int n = 0;
  for (const auto& s : h->log) {
    double* r = out + 12 * n++;
    r[0] = s.phase; r[1] = s.sys_len; r[2] = s.env_len; r[3] = s.e0; r[4] = s.lanczos_iters;
    r[5] = s.num_state; r[6] = s.trun_err; r[7] = s.entropy; r[8] = s.entropy_mult;
    r[9] = s.hpsi_calls; r[10] = s.hpsi_seconds; r[11] = s.hpsi_flops;
  }
  return n;
}

// Capture serialisation order:
//   ints: [valid, sys_side, iters, num_state, nxc, has_wt, wt_lr, sys_nops, env_nops, grown_nops]
//   doubles (as complex re parts): e0, err, ent, ent_mult
//   sys model, env model, sys_bs, env_bs, psi0, hpsi, gs, den, trun, grow_basis, grown model,
//   spectrum (as complex with zero imaginary part), then if has_wt:
//   wt_sys_bs, wt_env_bs, wt_sys_trun, wt_env_trun, wt_old, wt_new
int orc_capture_serialize(void* hp, long long* nints, long long* ncplx) {
  OrcHandle* h = (OrcHandle*)hp;
  Oracle& o = *h->o;
  auto& c = o.cap;
  if (!c.valid) return -1;
  Ser& s = h->ser;
  s = Ser();
  int sn = o.L.nleg11[c.sys.len], en = o.L.nleg11[c.env.len], gn = o.L.nleg11[c.grown.len];
  s.ints.insert(s.ints.end(), {1, c.sys_side ? 1 : 0, c.iters, c.num_state, c.nxc, c.has_wt ? 1 : 0,
                               c.wt_lr ? 1 : 0, sn, en, gn});
  s.data.insert(s.data.end(), {cplx(c.e0), cplx(c.err), cplx(c.ent), cplx(c.ent_mult)});
  s.model(c.sys, sn);
  s.model(c.env, en);
  s.basis(c.sys_bs);
  s.basis(c.env_bs);
  s.wave(c.psi0);
  s.wave(c.hpsi);
  s.wave(c.gs);
  s.block(c.den);
  s.block(c.trun);
  s.basis(c.grow_basis);
  s.model(c.grown, gn);
  s.ints.push_back((int)c.spectrum.size());
  for (double v : c.spectrum) s.data.push_back(cplx(v));
  if (c.has_wt) {
    s.basis(c.wt_sys_bs);
    s.basis(c.wt_env_bs);
    s.block(c.wt_sys_trun);
    s.block(c.wt_env_trun);
    s.wave(c.wt_old);
    s.wave(c.wt_new);
  }
  *nints = (long long)s.ints.size();
  *ncplx = (long long)s.data.size();
  return 0;
}

void orc_serialized_copy(void* hp, int* ints, double* cplx_interleaved) {
  OrcHandle* h = (OrcHandle*)hp;
  std::memcpy(ints, h->ser.ints.data(), h->ser.ints.size() * sizeof(int));
  std::memcpy(cplx_interleaved, h->ser.data.data(), h->ser.data.size() * sizeof(cplx));
}

double orc_w6js(int a, int b, int c, int d, int e, int f) { return w6js(a, b, c, d, e, f); }
double orc_w3js(int a, int b, int c, int d, int e, int f) { return w3js(a, b, c, d, e, f); }

// Stand-alone H.psi on a flat superblock: the layout of tsc_superblock_set in
// the product's C-ABI (sys model, env model, sys_bs, env_bs) followed by psi.
// Used for parity on product-generated superblocks and for the timed CPU
// baseline.  nreps H.psi applications; returns seconds of the last rep in *sec.
int orc_hpsi_flat(void* hp, int sys_len, int env_len, const int* ints, const double* data,
                  double* out_interleaved, int nreps, double* sec, double* flops) {
  OrcHandle* h = (OrcHandle*)hp;
  Oracle& o = *h->o;
  try {
    Des d{ints, (const cplx*)data};
    Model sys = d.model(o.L.num_site);
    Model env = d.model(o.L.num_site);
    Basis sys_bs = d.basis();
    Basis env_bs = d.basis();
    Wave in = d.wave();
    if (sys.len != sys_len || env.len != env_len) throw std::runtime_error("length mismatch");
    o.dmrg_setup(sys_len, env_len);
    o.hmerge(sys, env, sys_bs, env_bs);
    Wave out = in;
    double f0 = g_gemm_flops;
    for (int r = 0; r < nreps; ++r) {
      auto t0 = std::chrono::steady_clock::now();
      if (r == nreps - 1) f0 = g_gemm_flops;
      o.model_wave(sys, env, sys_bs, env_bs, in, out);
      *sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    *flops = g_gemm_flops - f0;
    size_t off = 0;
    for (const auto& s : out.sub) {
      std::memcpy(out_interleaved + 2 * off, s.vec.data(), s.vec.size() * sizeof(cplx));
      off += s.vec.size();
    }
  } catch (std::exception& e) {
    h->err = e.what();
    return -1;
  }
  return 0;
}

}  // extern "C"
