// extern "C" boundary (include/tsc_gpu.h).  Every entry point converts engine
// exceptions into a negative status and a one-line message; nothing aborts the
// host process.
#include <cstring>
#include <memory>

#include "../../include/tsc_gpu.h"
#include "tsc_ctx.hpp"
#include "tsc_engine.hpp"

using namespace tsc;

namespace {

struct Reader {
  const int* ip;
  const int* iend;
  const cplx* dp;
  const cplx* dend;
  int i() {
    if (ip >= iend) throw Error(TSC_E_ARG, "descriptor array too short");
    return *ip++;
  }
  void need_data(long long n) {
    if (n < 0 || dp + n > dend) throw Error(TSC_E_ARG, "data array too short");
  }
};

DBlock read_block(Engine& E, Reader& r) {
  const int* ip0 = r.ip;
  int hdr[5];
  for (int& h : hdr) h = r.i();
  if (hdr[1] < 0 || hdr[1] > 1000000) throw Error(TSC_E_ARG, "bad block descriptor");
  long long tot = 0;
  for (int k = 0; k < hdr[1]; ++k) {
    int v[5];
    for (int& x : v) x = r.i();
    if (v[3] < 0 || v[4] < 0) throw Error(TSC_E_ARG, "negative sub-block dimension");
    tot += (long long)v[3] * v[4];
  }
  r.need_data(tot);
  const int* ip = ip0;
  const cplx* dp = r.dp;
  DBlock b = E.upload_block(ip, dp);
  r.dp = dp;
  return b;
}

DModel read_model(Engine& E, Reader& r) {
  DModel m;
  m.len = r.i();
  int nops = r.i();
  if (nops < 0 || nops > E.L.num_site) throw Error(TSC_E_ARG, "bad operator count");
  m.ham = read_block(E, r);
  m.sub.resize(E.L.num_site + 1);
  for (int k = 1; k <= nops; ++k)
    for (int o = 0; o < 4; ++o) m.sub[k].op[o] = read_block(E, r);
  return m;
}

Basis read_basis(Reader& r) {
  Basis b;
  b.len = r.i();
  b.num = r.i();
  b.dim = r.i();
  if (b.num < 0 || b.num > 1000000) throw Error(TSC_E_ARG, "bad basis descriptor");
  b.sec.resize(b.num);
  std::vector<int> np(b.num);
  for (int k = 0; k < b.num; ++k) {
    b.sec[k].num_up = r.i();
    b.sec[k].num_down = r.i();
    b.sec[k].dim = r.i();
    np[k] = r.i();
  }
  for (int k = 0; k < b.num; ++k) {
    int pos = 0;
    for (int q = 0; q < np[k]; ++q) {
      Piece p;
      p.bl_num_up = r.i();
      p.bl_num_down = r.i();
      p.st_num_up = r.i();
      p.st_num_down = r.i();
      p.spos = r.i();
      p.sdim = r.i();
      if (p.spos != pos || p.sdim < 0) throw Error(TSC_E_ARG, "basis pieces not contiguous");
      pos += p.sdim;
      b.sec[k].pcs.push_back(p);
    }
    if (pos != b.sec[k].dim) throw Error(TSC_E_ARG, "basis sector dimension mismatch");
  }
  return b;
}

WLayout read_wave_layout(Reader& r, bool has_data, const cplx** data) {
  WLayout w;
  w.sys_len = r.i();
  w.env_len = r.i();
  w.num = r.i();
  r.i();   // dim (recomputed)
  if (w.num < 0 || w.num > 1000000) throw Error(TSC_E_ARG, "bad wave descriptor");
  for (int k = 0; k < w.num; ++k) {
    WSec s;
    s.sys_num_up = r.i();
    s.sys_num_down = r.i();
    s.env_num_up = r.i();
    s.env_num_down = r.i();
    s.sys_dim = r.i();
    s.env_dim = r.i();
    if (s.sys_dim < 0 || s.env_dim < 0) throw Error(TSC_E_ARG, "negative wave dimension");
    s.off = w.dim;
    w.dim += (long long)s.sys_dim * s.env_dim;
    w.sec.push_back(s);
  }
  if (has_data) {
    r.need_data(w.dim);
    if (data) *data = r.dp;
    r.dp += w.dim;
  }
  return w;
}

void check_layout(const Basis& sb, const Basis& eb, const WLayout& w) {
  for (const auto& s : w.sec) {
    int x = sb.find(s.sys_num_up, s.sys_num_down), y = eb.find(s.env_num_up, s.env_num_down);
    if (x < 0 || y < 0) throw Error(TSC_E_QN, "psi sector has no basis sector");
    if (sb.sec[x].dim != s.sys_dim || eb.sec[y].dim != s.env_dim) throw Error(TSC_E_ARG, "psi sector dims mismatch");
  }
}

}  // namespace

extern "C" {

int tsc_create(tsc_ctx** ctx, const tsc_model_config* cfg) {
  if (!ctx || !cfg) return TSC_E_ARG;
  *ctx = nullptr;
  tsc_ctx* c = new tsc_ctx();
  c->device = cfg->device;
  try {
    c->eng.reset(new Engine(cfg->Nx, cfg->Ny, cfg->t1, cfg->t2, cfg->J1, cfg->J2, cfg->delta, cfg->device));
    // tsc_hpsi_noalloc's array is placed on the device here, when the context
    // is created, so that entry point never makes the driver allocate
    noalloc_scratch_address(cfg->device);
  } catch (Error& e) {
    c->err = e.what();
    *ctx = c;
    return e.code;
  } catch (std::exception& e) {
    c->err = e.what();
    *ctx = c;
    return TSC_E_CUDA;
  }
  *ctx = c;
  return TSC_OK;
}

int tsc_destroy(tsc_ctx* ctx) {
  if (!ctx) return TSC_E_ARG;
  try {
    ctx->eng.reset();
  } catch (...) {
  }
  delete ctx;
  return TSC_OK;
}

const char* tsc_last_error(tsc_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int tsc_tot_num_up(tsc_ctx* ctx) { return (ctx && ctx->eng) ? ctx->eng->tot_num_up : TSC_E_ARG; }

int tsc_superblock_set(tsc_ctx* ctx, int sys_len, int env_len, const int* ints, long long nints, const double* data,
                       long long ncplx) {
  return guard(ctx, [&] {
    if (!ctx->eng) throw Error(TSC_E_STATE, "no engine");
    if (!ints || nints <= 0 || (ncplx > 0 && !data)) throw Error(TSC_E_ARG, "null buffers");
    Engine& E = *ctx->eng;
    Reader r{ints, ints + nints, (const cplx*)data, (const cplx*)data + ncplx};
    DModel sys = read_model(E, r);
    DModel env = read_model(E, r);
    if (sys.len != sys_len || env.len != env_len) throw Error(TSC_E_ARG, "block lengths disagree with descriptors");
    if (sys_len < 1 || env_len < 1 || sys_len + env_len + 2 > E.L.num_site) throw Error(TSC_E_ARG, "lengths out of range");
    Basis sb = read_basis(r);
    Basis eb = read_basis(r);
    WLayout w = read_wave_layout(r, false, nullptr);
    check_layout(sb, eb, w);
    E.superblock_set(std::move(sys), std::move(env), std::move(sb), std::move(eb), std::move(w));
  });
}

long long tsc_superblock_dim(tsc_ctx* ctx) {
  if (!ctx || !ctx->eng || !ctx->eng->sb.valid) return TSC_E_STATE;
  return ctx->eng->sb.wl.dim;
}

int tsc_hpsi(tsc_ctx* ctx, const double* in, double* out) {
  return guard(ctx, [&] {
    if (!ctx->eng || !ctx->eng->sb.valid) throw Error(TSC_E_STATE, "no superblock set");
    if (!in || !out) throw Error(TSC_E_ARG, "null buffers");
    Engine& E = *ctx->eng;
    long long n = E.sb.wl.dim;
    DevBuf a((size_t)std::max<long long>(n, 1), E.st, false), b((size_t)std::max<long long>(n, 1), E.st, false);
    cuda_check(cudaMemcpyAsync(a.p, in, n * sizeof(double2), cudaMemcpyHostToDevice, E.st), "h2d");
    E.hpsi(a.p, b.p);
    cuda_check(cudaMemcpyAsync(out, b.p, n * sizeof(double2), cudaMemcpyDeviceToHost, E.st), "d2h");
    cuda_check(cudaStreamSynchronize(E.st), "sync");
    if (E.sb.p1s.split) E.check_split_fault();
  });
}

int tsc_hpsi_device(tsc_ctx* ctx, const void* d_in, void* d_out) {
  return guard(ctx, [&] {
    if (!ctx->eng || !ctx->eng->sb.valid) throw Error(TSC_E_STATE, "no superblock set");
    if (!d_in || !d_out) throw Error(TSC_E_ARG, "null buffers");
    ctx->eng->hpsi((const double2*)d_in, (double2*)d_out);
    // the split form waits for its launches and reports a wait that ran out
    if (ctx->eng->sb.p1s.split) ctx->eng->check_split_fault();
  });
}

int tsc_hpsi_stats(tsc_ctx* ctx, double* device_ms, double* flops, double* exec_flops, int* launches) {
  return guard(ctx, [&] {
    Engine& E = *ctx->eng;
    float ms = 0.f;
    cuda_check(cudaEventSynchronize(E.ev1), "event");
    cuda_check(cudaEventElapsedTime(&ms, E.ev0, E.ev1), "elapsed");
    if (device_ms) *device_ms = ms;
    if (flops) *flops = E.sb.ref_flops;
    if (exec_flops) *exec_flops = E.sb.p2.exec_flops + E.sb.p1.exec_flops;
    if (launches) *launches = E.last_stats.launches;
  });
}

int tsc_lanczos(tsc_ctx* ctx, double* psi_inout, double lanzero, int* iters, double* e0) {
  return guard(ctx, [&] {
    if (!ctx->eng || !ctx->eng->sb.valid) throw Error(TSC_E_STATE, "no superblock set");
    if (!psi_inout || !iters || !e0) throw Error(TSC_E_ARG, "null buffers");
    Engine& E = *ctx->eng;
    long long n = E.sb.wl.dim;
    DevBuf a((size_t)std::max<long long>(n, 1), E.st, false);
    cuda_check(cudaMemcpyAsync(a.p, psi_inout, n * sizeof(double2), cudaMemcpyHostToDevice, E.st), "h2d");
    E.lanczos(a.p, lanzero, iters, e0, nullptr, nullptr);
    cuda_check(cudaMemcpyAsync(psi_inout, a.p, n * sizeof(double2), cudaMemcpyDeviceToHost, E.st), "d2h");
    cuda_check(cudaStreamSynchronize(E.st), "sync");
  });
}

int tsc_truncate(tsc_ctx* ctx, int side, const double* psi, int kept_min, int kept_max, double trun_err,
                 int* num_state, double* err, double* entropy, double* entropy_mult, const int** trun_ints,
                 long long* ntrun_ints, const double** trun_data, long long* ntrun_cplx, double* spectrum,
                 long long spectrum_cap) {
  return guard(ctx, [&] {
    if (!ctx->eng || !ctx->eng->sb.valid) throw Error(TSC_E_STATE, "no superblock set");
    if (side != 0 && side != 1) throw Error(TSC_E_ARG, "side must be 0 or 1");
    if (!psi || !num_state) throw Error(TSC_E_ARG, "null buffers");
    Engine& E = *ctx->eng;
    const WLayout& wl = E.sb.wl;
    DevBuf a((size_t)std::max<long long>(wl.dim, 1), E.st, false);
    cuda_check(cudaMemcpyAsync(a.p, psi, wl.dim * sizeof(double2), cudaMemcpyHostToDevice, E.st), "h2d");
    Engine::TruncResult tr;
    E.truncate(side, a.p, wl, kept_min, kept_max, trun_err, tr);
    *num_state = tr.num_state;
    if (err) *err = tr.err;
    if (entropy) *entropy = tr.ent;
    if (entropy_mult) *entropy_mult = tr.ent_mult;
    ctx->out_ints.clear();
    ctx->out_data.clear();
    E.download_block(tr.trun, ctx->out_ints, ctx->out_data);
    if (trun_ints) *trun_ints = ctx->out_ints.data();
    if (ntrun_ints) *ntrun_ints = (long long)ctx->out_ints.size();
    if (trun_data) *trun_data = (const double*)ctx->out_data.data();
    if (ntrun_cplx) *ntrun_cplx = (long long)ctx->out_data.size();
    if (spectrum)
      for (long long i = 0; i < spectrum_cap && i < (long long)tr.spectrum.size(); ++i) spectrum[i] = tr.spectrum[i];
  });
}

int tsc_density_matrix(tsc_ctx* ctx, int side, const double* psi, int levels, const int** den_ints,
                       long long* nden_ints, const double** den_data, long long* nden_cplx) {
  return guard(ctx, [&] {
    if (!ctx->eng || !ctx->eng->sb.valid) throw Error(TSC_E_STATE, "no superblock set");
    if (side != 0 && side != 1) throw Error(TSC_E_ARG, "side must be 0 or 1");
    if (!psi || levels < 1) throw Error(TSC_E_ARG, "null wave or levels < 1");
    Engine& E = *ctx->eng;
    const WLayout& wl = E.sb.wl;
    const int nw = std::min(levels, 2);   // the reference reads the first two waves
    DevBuf a((size_t)std::max<long long>(wl.dim * nw, 1), E.st, false);
    cuda_check(cudaMemcpyAsync(a.p, psi, wl.dim * nw * sizeof(double2), cudaMemcpyHostToDevice, E.st), "h2d");
    DBlock den = E.density_matrix(side, a.p, wl, levels);
    ctx->out_ints.clear();
    ctx->out_data.clear();
    E.download_block(den, ctx->out_ints, ctx->out_data);
    if (den_ints) *den_ints = ctx->out_ints.data();
    if (nden_ints) *nden_ints = (long long)ctx->out_ints.size();
    if (den_data) *den_data = (const double*)ctx->out_data.data();
    if (nden_cplx) *nden_cplx = (long long)ctx->out_data.size();
  });
}

int tsc_truncation_operator(tsc_ctx* ctx, const int* den_ints, long long nden_ints, const double* den_data,
                            long long nden_cplx, int kept_min, int kept_max, double trun_err, int* num_state,
                            double* err, double* entropy, double* entropy_mult, const int** trun_ints,
                            long long* ntrun_ints, const double** trun_data, long long* ntrun_cplx, double* spectrum,
                            long long spectrum_cap) {
  return guard(ctx, [&] {
    if (!ctx->eng) throw Error(TSC_E_STATE, "no engine");
    if (!den_ints || !den_data || !num_state) throw Error(TSC_E_ARG, "null buffers");
    Engine& E = *ctx->eng;
    Reader r{den_ints, den_ints + nden_ints, (const cplx*)den_data, (const cplx*)den_data + nden_cplx};
    DBlock den = read_block(E, r);
    Engine::TruncResult tr;
    E.truncation_operator(den, kept_min, kept_max, trun_err, tr);
    *num_state = tr.num_state;
    if (err) *err = tr.err;
    if (entropy) *entropy = tr.ent;
    if (entropy_mult) *entropy_mult = tr.ent_mult;
    ctx->out_ints.clear();
    ctx->out_data.clear();
    E.download_block(tr.trun, ctx->out_ints, ctx->out_data);
    if (trun_ints) *trun_ints = ctx->out_ints.data();
    if (ntrun_ints) *ntrun_ints = (long long)ctx->out_ints.size();
    if (trun_data) *trun_data = (const double*)ctx->out_data.data();
    if (ntrun_cplx) *ntrun_cplx = (long long)ctx->out_data.size();
    if (spectrum)
      for (long long i = 0; i < spectrum_cap && i < (long long)tr.spectrum.size(); ++i) spectrum[i] = tr.spectrum[i];
  });
}

int tsc_renormalize(tsc_ctx* ctx, int side, int sys_len, int env_len, int mshift, const int* ints, long long nints,
                    const double* data, long long ncplx, const int** out_ints, long long* nout_ints,
                    const double** out_data, long long* nout_cplx) {
  return guard(ctx, [&] {
    if (!ctx->eng) throw Error(TSC_E_STATE, "no engine");
    if (side != 0 && side != 1) throw Error(TSC_E_ARG, "side must be 0 or 1");
    Engine& E = *ctx->eng;
    Reader r{ints, ints + nints, (const cplx*)data, (const cplx*)data + ncplx};
    DModel m = read_model(E, r);
    Basis b = read_basis(r);
    DBlock trun = read_block(E, r);
    E.L.setup(sys_len, env_len);
    E.grow(side, m, b, trun, mshift);
    ctx->out_ints.clear();
    ctx->out_data.clear();
    int nops = E.L.nleg11[m.len];
    ctx->out_ints.push_back(m.len);
    ctx->out_ints.push_back(nops);
    E.download_block(m.ham, ctx->out_ints, ctx->out_data);
    for (int i = 1; i <= nops; ++i)
      for (int o = 0; o < 4; ++o) E.download_block(m.sub[i].op[o], ctx->out_ints, ctx->out_data);
    if (out_ints) *out_ints = ctx->out_ints.data();
    if (nout_ints) *nout_ints = (long long)ctx->out_ints.size();
    if (out_data) *out_data = (const double*)ctx->out_data.data();
    if (nout_cplx) *nout_cplx = (long long)ctx->out_data.size();
  });
}

int tsc_wave_transform(tsc_ctx* ctx, int dir, const int* ints, long long nints, const double* data, long long ncplx,
                       double* new_out) {
  return guard(ctx, [&] {
    if (!ctx->eng) throw Error(TSC_E_STATE, "no engine");
    if (dir != 0 && dir != 1) throw Error(TSC_E_ARG, "dir must be 0 (LR) or 1 (RL)");
    if (!new_out) throw Error(TSC_E_ARG, "null output");
    Engine& E = *ctx->eng;
    Reader r{ints, ints + nints, (const cplx*)data, (const cplx*)data + ncplx};
    Basis sb = read_basis(r);
    Basis eb = read_basis(r);
    DBlock st = read_block(E, r);
    DBlock et = read_block(E, r);
    const cplx* od = nullptr;
    WLayout ol = read_wave_layout(r, true, &od);
    WLayout nl = read_wave_layout(r, false, nullptr);
    DevBuf a((size_t)std::max<long long>(ol.dim, 1), E.st, false), b((size_t)std::max<long long>(nl.dim, 1), E.st, false);
    cuda_check(cudaMemcpyAsync(a.p, od, ol.dim * sizeof(double2), cudaMemcpyHostToDevice, E.st), "h2d");
    E.wave_trans(dir, sb, eb, st, et, ol, a.p, nl, b.p);
    cuda_check(cudaMemcpyAsync(new_out, b.p, nl.dim * sizeof(double2), cudaMemcpyDeviceToHost, E.st), "d2h");
    cuda_check(cudaStreamSynchronize(E.st), "sync");
  });
}

int tsc_dmrg_run(tsc_ctx* ctx, const tsc_sweep_config* sw, tsc_step_log* log, int max_steps) {
  int nsteps = 0;
  int rc = guard(ctx, [&] {
    if (!ctx->eng) throw Error(TSC_E_STATE, "no engine");
    if (!sw || (sw->nsweeps > 0 && !sw->sweep_kept_max) || sw->nsweeps < 0) throw Error(TSC_E_ARG, "bad sweep config");
    if (sw->kept_min < 1 || sw->kept_max_warmup < 1) throw Error(TSC_E_ARG, "kept sizes must be positive");
    std::vector<int> sweeps(sw->sweep_kept_max, sw->sweep_kept_max + sw->nsweeps);
    std::vector<Engine::StepRec> recs;
    ctx->eng->lanzero_warmup_ = sw->lanzero_warmup > 0 ? sw->lanzero_warmup : 0.0;
    ctx->eng->final_stop_ = sw->final_stop > 0 ? sw->final_stop : 0;
    ctx->eng->run(sw->kept_min, sw->kept_max_warmup, sweeps, sw->lanzero, sw->seed, &recs, sw->warmup_only != 0,
                  sw->final_half_sweep != 0, sw->resume != 0, sw->max_solves > 0 ? sw->max_solves : 0);
    nsteps = (int)recs.size();
    for (int i = 0; i < nsteps && i < max_steps && log; ++i) {
      const auto& s = recs[i];
      log[i] = tsc_step_log{s.phase, s.sys_len, s.env_len, s.e0, s.iters, s.num_state, s.err, s.ent, s.ent_mult,
                            s.hpsi_calls, s.hpsi_seconds, s.hpsi_flops, s.step_seconds,
                            s.set_seconds, s.lanczos_seconds, s.truncate_seconds, s.grow_seconds,
                            s.wave_seconds, s.split_iters, s.split_e0};
    }
  });
  return rc == TSC_OK ? nsteps : rc;
}

void* tsc_stream(tsc_ctx* ctx) { return (ctx && ctx->eng) ? (void*)ctx->eng->st : nullptr; }

int tsc_set_capture(tsc_ctx* ctx, int capture_step) {
  return guard(ctx, [&] {
    if (!ctx->eng) throw Error(TSC_E_STATE, "no engine");
    ctx->eng->capture_step = capture_step;
  });
}

int tsc_get_capture(tsc_ctx* ctx, const int** ints, long long* nints, const double** data, long long* ncplx,
                    int* sys_len, int* env_len) {
  return guard(ctx, [&] {
    if (!ctx->eng || !ctx->eng->cap.valid) throw Error(TSC_E_STATE, "nothing captured");
    auto& c = ctx->eng->cap;
    if (ints) *ints = c.ints.data();
    if (nints) *nints = (long long)c.ints.size();
    if (data) *data = (const double*)c.data.data();
    if (ncplx) *ncplx = (long long)c.data.size();
    if (sys_len) *sys_len = c.sys_len;
    if (env_len) *env_len = c.env_len;
  });
}

}  // extern "C"

int tsc_set_precision(tsc_ctx* ctx, int mode, double split_tol) {
  return guard(ctx, [&] {
    if (!ctx->eng) throw Error(TSC_E_STATE, "no engine");
    if (mode != TSC_FP64 && mode != TSC_SPLIT_BF16) throw Error(TSC_E_ARG, "unknown precision mode");
    ctx->eng->precision_ = mode;
    if (split_tol > 0) ctx->eng->split_tol_ = split_tol;
    // the split form's pre-sliced operand views take about 1.5x the superblock's
    // FP64 operator and intermediate memory: the stored models get less by default
    ctx->eng->model_store().set_default_frac(mode == TSC_SPLIT_BF16 ? 0.30 : 0.45);
  });
}

int tsc_set_split_view_sharing(tsc_ctx* ctx, int shared) {
  return guard(ctx, [&] {
    if (!ctx->eng) throw Error(TSC_E_STATE, "no engine");
    ctx->eng->split_shared_views_ = shared < 0 ? -1 : (shared != 0 ? 1 : 0);
  });
}

int tsc_set_lanczos_graph(tsc_ctx* ctx, int on) {
  return guard(ctx, [&] {
    if (!ctx->eng) throw Error(TSC_E_STATE, "no engine");
    ctx->eng->lanczos_graph_ = on != 0;
  });
}

int tsc_lanczos_graph_stats(tsc_ctx* ctx, long long* replays, long long* fallbacks, char* reason, int reason_cap) {
  return guard(ctx, [&] {
    if (!ctx->eng) throw Error(TSC_E_STATE, "no engine");
    Engine& E = *ctx->eng;
    if (replays) *replays = E.graph_replays_;
    if (fallbacks) *fallbacks = E.graph_fallbacks_;
    if (reason && reason_cap > 0) {
      const size_t n = std::min<size_t>((size_t)reason_cap - 1, E.graph_fallback_reason_.size());
      std::memcpy(reason, E.graph_fallback_reason_.data(), n);
      reason[n] = 0;
    }
  });
}

int tsc_set_split_finish_tolerance(tsc_ctx* ctx, double multiplier) {
  return guard(ctx, [&] {
    if (!ctx->eng) throw Error(TSC_E_STATE, "no engine");
    if (!(multiplier > 0.0)) throw Error(TSC_E_ARG, "multiplier must be > 0");
    ctx->eng->finish_mult_ = multiplier;
  });
}

int tsc_set_split_renormalization(tsc_ctx* ctx, int on) {
  return guard(ctx, [&] {
    if (!ctx->eng) throw Error(TSC_E_STATE, "no engine");
    ctx->eng->split_renorm_ = on != 0;
  });
}

int tsc_set_split_refinement(tsc_ctx* ctx, double residual_factor) {
  return guard(ctx, [&] {
    if (!ctx->eng) throw Error(TSC_E_STATE, "no engine");
    if (!(residual_factor >= 0.0)) throw Error(TSC_E_ARG, "residual factor must be >= 0");
    ctx->eng->refine_res_ = residual_factor;
  });
}

int tsc_set_split_wait_limit(tsc_ctx* ctx, long long polls) {
  return guard(ctx, [&] {
    if (!ctx->eng) throw Error(TSC_E_STATE, "no engine");
    if (polls < 0) throw Error(TSC_E_ARG, "wait limit must be >= 0");
    ctx->eng->split_wait_limit_ = polls > 0 ? polls : 0;
  });
}

int tsc_split_views(tsc_ctx* ctx, long long* bytes, int* views) {
  return guard(ctx, [&] {
    if (!ctx->eng) throw Error(TSC_E_STATE, "no engine");
    Engine& E = *ctx->eng;
    if (E.views_of_batch_ ? !E.bs.valid : !E.sb.valid) throw Error(TSC_E_STATE, "no superblock set");
    const SplitData& sd = E.views_of_batch_ ? E.bs.sv : E.sb.sv;
    for (int a = 0; a < 3; ++a) {
      if (bytes) bytes[a] = sd.units[a] * (long long)SPLIT_UNIT;
      if (views) views[a] = sd.nviews[a];
    }
  });
}

int tsc_set_resident_limit(tsc_ctx* ctx, long long bytes) {
  return guard(ctx, [&] {
    if (!ctx->eng) throw Error(TSC_E_STATE, "no engine");
    ctx->eng->model_store().set_limit(bytes < 0 ? -1 : bytes);
  });
}

int tsc_set_spill_directory(tsc_ctx* ctx, const char* dir, long long host_bytes) {
  return guard(ctx, [&] {
    if (!ctx->eng) throw Error(TSC_E_STATE, "no engine");
    ctx->eng->model_store().set_disk(dir && *dir ? host_bytes : -1, dir ? std::string(dir) : std::string());
  });
}

int tsc_disk_spill_stats(tsc_ctx* ctx, long long* writes, long long* reads, double* bytes, double* seconds,
                         long long* host_bytes) {
  return guard(ctx, [&] {
    if (!ctx->eng) throw Error(TSC_E_STATE, "no engine");
    ModelStore& m = ctx->eng->model_store();
    if (writes) *writes = m.disk_writes;
    if (reads) *reads = m.disk_reads;
    if (bytes) *bytes = m.disk_bytes;
    if (seconds) *seconds = m.disk_seconds;
    if (host_bytes) *host_bytes = m.host_bytes();
  });
}

int tsc_spill_stats(tsc_ctx* ctx, long long* spills, long long* restores, double* bytes, double* seconds,
                    long long* resident_bytes, long long* limit_bytes) {
  return guard(ctx, [&] {
    if (!ctx->eng) throw Error(TSC_E_STATE, "no engine");
    ModelStore& m = ctx->eng->model_store();
    if (spills) *spills = m.spills;
    if (restores) *restores = m.restores;
    if (bytes) *bytes = m.moved_bytes;
    if (seconds) *seconds = m.moved_seconds;
    if (resident_bytes) *resident_bytes = m.resident_bytes();
    if (limit_bytes) *limit_bytes = m.limit();
  });
}

int tsc_set_autotune(tsc_ctx* ctx, int on) {
  return guard(ctx, [&] {
    if (!ctx->eng) throw Error(TSC_E_STATE, "no engine");
    ctx->eng->autotune_ = on != 0;
  });
}

int tsc_autotune_table(tsc_ctx* ctx, int* cls, double* ms_per_gflop, int max_classes) {
  int n = 0;
  int rc = guard(ctx, [&] {
    if (!ctx->eng) throw Error(TSC_E_STATE, "no engine");
    for (const auto& kv : ctx->eng->tune_ms_) {
      if (n < max_classes && cls && ms_per_gflop) {
        cls[n] = kv.first;
        for (int c = 0; c < Engine::kTuneCands; ++c) ms_per_gflop[4 * n + c] = kv.second[c];
      }
      n++;
    }
  });
  return rc < 0 ? rc : n;
}

int tsc_autotune_superblock(tsc_ctx* ctx, int reps) {
  int win = 0;
  int rc = guard(ctx, [&] {
    if (!ctx->eng || !ctx->eng->sb.valid) throw Error(TSC_E_STATE, "no superblock set");
    win = ctx->eng->tune_superblock(reps);
  });
  return rc < 0 ? rc : win;
}
