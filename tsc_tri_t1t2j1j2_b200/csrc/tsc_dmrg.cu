// DMRG steps on the device: Lanczos (eigen.f90:4-199), reduced density matrix and
// truncation (den_mat.f90:4-418), block growth and U^dagger O U renormalisation
// (get_sys.f90:4-592, block.f90:2495-3683), wave transformations
// (dmrg_sub.f90:1471-1789) and the sweep driver (dmrg_sub.f90:974-1465,
// main.f90:114-209).  All block operators stay resident in HBM; the host only
// builds task lists and runs the scalar control flow of the reference.
#include <cusolverDn.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>

#include "tsc_engine.hpp"

namespace tsc {

// Phase timer of the step records: wall clock after the engine stream drains.
static inline std::chrono::steady_clock::time_point phase_clock(cudaStream_t st) {
  cuda_check(cudaStreamSynchronize(st), "sync");
  return std::chrono::steady_clock::now();
}
static inline double secs(std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
  return std::chrono::duration<double>(b - a).count();
}


// Per-sector zheevd calls are independent and each occupies a small part of the
// GPU, but cuSOLVER's zheevd waits on the host inside the call.  So each lane is
// a host thread with its own stream, cuSOLVER handle and workspace; the engine
// stream forks to the lanes through an event and joins their done events.
struct Engine::EigLanes {
  struct Lane {
    cudaStream_t s = nullptr;
    cusolverDnHandle_t h = nullptr;
    cudaEvent_t done = nullptr;
    DevBufP work;
    int lwork = 0;
    std::thread th;
  };
  std::vector<Lane> lane;
  cudaEvent_t fork = nullptr;
  std::mutex mu;
  std::condition_variable cv_go, cv_done;
  std::function<void(int)> task;
  long long gen = 0;
  int pending = 0;
  bool stop = false;
  std::string err;

  EigLanes(int n, int device) : lane(n) {
    cuda_check(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming), "cudaEventCreate");
    for (auto& l : lane) {
      cuda_check(cudaStreamCreateWithFlags(&l.s, cudaStreamNonBlocking), "cudaStreamCreate");
      cuda_check(cudaEventCreateWithFlags(&l.done, cudaEventDisableTiming), "cudaEventCreate");
      if (cusolverDnCreate(&l.h) != CUSOLVER_STATUS_SUCCESS) throw Error(-3, "cusolverDnCreate failed");
      if (cusolverDnSetStream(l.h, l.s) != CUSOLVER_STATUS_SUCCESS) throw Error(-3, "cusolverDnSetStream failed");
    }
    for (int i = 0; i < n; ++i)
      lane[i].th = std::thread([this, i, device] {
        cudaSetDevice(device);
        long long seen = 0;
        while (true) {
          std::function<void(int)> t;
          {
            std::unique_lock<std::mutex> lk(mu);
            cv_go.wait(lk, [&] { return stop || gen != seen; });
            if (stop) return;
            seen = gen;
            t = task;
          }
          std::string e;
          try {
            t(i);
          } catch (std::exception& x) {
            e = x.what();
          }
          std::lock_guard<std::mutex> lk(mu);
          if (!e.empty() && err.empty()) err = e;
          if (--pending == 0) cv_done.notify_all();
        }
      });
  }
  // runs f(lane) on every lane thread and waits for all of them
  void run(std::function<void(int)> f) {
    std::unique_lock<std::mutex> lk(mu);
    task = std::move(f);
    err.clear();
    pending = (int)lane.size();
    gen++;
    cv_go.notify_all();
    cv_done.wait(lk, [&] { return pending == 0; });
    if (!err.empty()) throw Error(-3, err);
  }
  ~EigLanes() {
    {
      std::lock_guard<std::mutex> lk(mu);
      stop = true;
    }
    cv_go.notify_all();
    for (auto& l : lane)
      if (l.th.joinable()) l.th.join();
    for (auto& l : lane) {
      if (l.s) cudaStreamSynchronize(l.s);
      l.work.reset();
      release_stream_cache(l.s);
      if (l.s) cudaStreamSynchronize(l.s);
      if (l.h) cusolverDnDestroy(l.h);
      if (l.done) cudaEventDestroy(l.done);
      if (l.s) cudaStreamDestroy(l.s);
    }
    if (fork) cudaEventDestroy(fork);
  }
};
constexpr int kEigLanes = 8;

namespace {
inline double pm1(int e) { return ((e % 2) + 2) % 2 == 0 ? 1.0 : -1.0; }
inline long long absoff(const double2* p) { return (long long)((uintptr_t)p / sizeof(double2)); }

// scalar slots in d_scal
constexpr int S_ALPHA = 0, S_BETA = 128, S_UV = 256, S_UU = 384, S_RES = 512, S_Z = 520, S_N2 = 700, S_PKT = 704, S_CHK = 712, S_ZR = 768;
constexpr int S_NRM = 1901;   // norm slot of Engine::normalize
constexpr int S_IT = 1990;    // the graphed iteration's index (an int in a double slot)

// Density-matrix eigenvalues below this are rounding noise (rho has unit trace).
constexpr double kZeroWeight = 1e-13;

// QuickSort_Double, block.f90:2398-2444 (descending with an index array)
void quicksort_double(std::vector<double>& a, std::vector<int>& idx, int lo, int hi) {
  int i = lo, j = hi;
  double mn = a[(int)((lo + hi) / 2.0)];
  while (i <= j) {
    while (a[i] > mn) i++;
    while (a[j] < mn) j--;
    if (i <= j) {
      std::swap(a[i], a[j]);
      std::swap(idx[i], idx[j]);
      i++;
      j--;
    }
  }
  if (lo < j) quicksort_double(a, idx, lo, j);
  if (i < hi) quicksort_double(a, idx, i, hi);
}
}  // namespace

// ---------------------------------------------------------------------------- Lanczos
void Engine::lanczos(double2* d_psi, double lanzero, int* iters, double* e0, double* hpsi_ms, int* hpsi_calls) {
  last_split_iters = 0;
  last_split_e0 = 0.0;
  if (!sb.p1s.split) {
    lanczos_run(d_psi, lanzero, 0.0, false, iters, e0, hpsi_ms, hpsi_calls);
    return;
  }
  // Split-precision form: Lanczos on the BF16-sliced H.psi until the Ritz value
  // settles to split_tol relative (the slices' noise floor), then FP64 Lanczos
  // from that vector, stopped by the reference's own test (successive Ritz
  // values within lanzero) or, with refine_res_ > 0, when the residual of its
  // Ritz pair is below refine_res_ sqrt(lanzero).  On the YC4x12 m=1000 sweep
  // the reference's test needs ~1/4 of the FP64 iterations the residual 0.1
  // sqrt(lanzero) does and lands as close to a tightly converged run as the
  // FP64 form itself (final energies 4.6e-10 and 5.3e-10 from a lanzero 1e-13
  // run, 7.6e-11 apart).
  int it1 = 0, it2 = 0, c1 = 0, c2 = 0;
  double ms1 = 0.0, ms2 = 0.0, e_split = 0.0;
  lanczos_run(d_psi, lanzero, split_tol_, true, &it1, &e_split, &ms1, &c1);
  check_split_fault();
  // FP64 Lanczos from that vector, stopped on the Ritz residual
  // ||H psi - E psi|| <= refine_res_ sqrt(lanzero) (from the tridiagonal, no extra
  // H.psi), or, with refine_res_ = 0, by the reference's own test
  lanczos_run(d_psi, lanzero * finish_mult_, 0.0, false, &it2, e0, &ms2, &c2, refine_res_ * std::sqrt(lanzero));
  last_split_iters = it1;
  last_split_e0 = e_split;
  *iters = it1 + it2;
  if (hpsi_ms) *hpsi_ms = ms1 + ms2;
  if (hpsi_calls) *hpsi_calls = c1 + c2;
}

void Engine::lanczos_run(double2* d_psi, double lanzero, double rel_tol, bool split, int* iters, double* e0,
                         double* hpsi_ms, int* hpsi_calls, double res_tol) {
  if (!sb.valid) throw Error(-4, "no superblock");
  const long long n = sb.wl.dim;
  const int loop_in = 100, loop_out = 4;
  const long long ld = (n + 15) / 16 * 16;
  DevBuf V((size_t)ld * (loop_in + 2), st, false);
  auto v = [&](int j) { return V.p + (long long)(j - 1) * ld; };   // 1-based Krylov vectors
  int nblk = (int)((n + 8191) / 8192);
  DevBuf part((size_t)((long long)nblk * (loop_in + 2) + 1) / 2 + 1, st, false);
  double* d_part = reinterpret_cast<double*>(part.p);
  double* a_d = d_scal + S_ALPHA;   // alpha_j at a_d[j], beta_j at b_d[j] (1-based, as eigen.f90)
  double* b_d = d_scal + S_BETA;
  double* uv_d = d_scal + S_UV;
  double* uu_d = d_scal + S_UU;
  double lastmin = 1024.0, ritzmin = 0.0;
  int iter_out = 0, last = 1;
  int calls = 0, eager_calls = 0;   // H.psi calls in all, and those with their own event pair
  // H.psi launches are bracketed by events that are read once, after the solve
  auto do_hpsi = [&](int j) {
    if ((size_t)(2 * eager_calls + 2) > hpsi_events.size()) {
      for (int q = 0; q < 2; ++q) {
        cudaEvent_t e;
        cuda_check(cudaEventCreate(&e), "cudaEventCreate");
        hpsi_events.push_back(e);
      }
    }
    cuda_check(cudaEventRecord(hpsi_events[2 * eager_calls], st), "event");
    hpsi_form(v(j), v(j + 1), split);
    cuda_check(cudaEventRecord(hpsi_events[2 * eager_calls + 1], st), "event");
    eager_calls++;
    calls++;
  };
  auto read_back = [&](int slot, int count) {
    cuda_check(cudaMemcpyAsync(h_scal + slot, d_scal + slot, count * sizeof(double), cudaMemcpyDeviceToHost, st), "d2h");
    cuda_check(cudaStreamSynchronize(st), "sync");
    tune_observe();
  };
  // lowest eigenpair of T_m (alpha_1..m, beta_1..m-1) from the device slots
  auto tridiag_vec = [&](int m) {
    cuda_check(launch_tridiag_lowest(a_d + 1, b_d + 1, m, 1, d_scal + S_RES, d_scal + S_Z, st), "tridiag");
    read_back(S_RES, 1);
    return h_scal[S_RES];
  };
  // One iteration's device work (vector steps, H.psi, tail, packet read-back)
  // as a CUDA graph, replayed with the index written to pinned memory before
  // each launch (its first node copies it to the device).  The H.psi reads and
  // writes two fixed vectors, copied from and to the Krylov block inside the
  // graph; every step computes what the eager iteration computes, bit for bit.
  // Built at the first iteration whose H.psi is not an autotuner probe.
  const bool graphs = lanczos_graph_;
  std::unique_ptr<DevBuf> gx, gy;
  bool graph_built = false;
  double graph_hms = 0.0;
  int* const d_it = reinterpret_cast<int*>(d_scal + S_IT);
  int* const h_it = reinterpret_cast<int*>(h_scal + S_IT);
  // false: the capture failed (the iteration then runs eagerly and graphs stay
  // off for this engine; the eager iteration computes the same numbers)
  auto build_graph = [&]() -> bool {
    gx.reset(new DevBuf((size_t)std::max<long long>(n, 1), st, false));
    gy.reset(new DevBuf((size_t)std::max<long long>(n, 1), st, false));
    for (auto* e : {&graph_ev_[0], &graph_ev_[1]})
      if (!*e) cuda_check(cudaEventCreate(e), "cudaEventCreate");
    const ItRef W{V.p, ld, 0}, V1{V.p, 0, 0}, X{gx->p, 0, 0}, Y{gy->p, 0, 0}, NEXT{V.p, ld, 1};
    cudaGraph_t g = nullptr;
    std::shared_lock<std::shared_mutex> capturing(capture_mutex());
    cuda_check(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed), "graph begin capture");
    try {
      cuda_check(cudaMemcpyAsync(d_it, h_it, sizeof(int), cudaMemcpyHostToDevice, st), "graph it h2d");
      cuda_check(launch_it_update(V.p, ld, a_d, b_d, n, d_it, st), "graph update");
      cuda_check(launch_it_dot(W, 0, 0, 1, 1, W, n, d_part, d_scal + S_N2, 0, 0, d_it, st), "graph norm");
      cuda_check(launch_it_scale(W, d_scal + S_N2, n, d_it, st), "graph normalize");
      cuda_check(launch_it_dot(V1, ld, 1, 0, loop_in, W, n, d_part, uv_d + 1, 0, 0, d_it, st), "graph uv");
      cuda_check(launch_it_gs(V.p, ld, uv_d + 1, uu_d + 1, n, d_it, st), "graph gs");
      cuda_check(launch_it_dot(W, 0, 0, 1, 1, W, n, d_part, d_scal + S_NRM, 0, 0, d_it, st), "graph norm of w");
      cuda_check(launch_it_scale(W, d_scal + S_NRM, n, d_it, st), "graph scale");
      cuda_check(launch_it_dot(W, 0, 0, 1, 1, W, n, d_part, uu_d + 1, 1, 0, d_it, st), "graph uu");
      cuda_check(launch_it_copy(X, W, n, d_it, st), "graph copy in");
      // external records: event nodes of the graph, readable after each replay
      cuda_check(cudaEventRecordWithFlags(graph_ev_[0], st, cudaEventRecordExternal), "graph event");
      hpsi_form(gx->p, gy->p, split);
      cuda_check(cudaEventRecordWithFlags(graph_ev_[1], st, cudaEventRecordExternal), "graph event");
      cuda_check(launch_it_copy(NEXT, Y, n, d_it, st), "graph copy out");
      cuda_check(launch_it_dot(X, 0, 0, 1, 1, Y, n, d_part, a_d + 1, 1, 0, d_it, st), "graph alpha");
      cuda_check(launch_it_tail(d_scal + S_N2, a_d, b_d, d_scal + S_RES, d_scal + S_PKT,
                                res_tol > 0 ? d_scal + S_ZR : nullptr, d_it, st),
                 "graph tail");
      cuda_check(cudaMemcpyAsync(h_scal + S_PKT, d_scal + S_PKT, 4 * sizeof(double), cudaMemcpyDeviceToHost, st),
                 "graph d2h");
    } catch (std::exception& e) {
      cudaStreamEndCapture(st, &g);
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      graph_fallbacks_++;
      graph_fallback_reason_ = e.what();
      lanczos_graph_ = false;
      return false;
    }
    if (cudaStreamEndCapture(st, &g) != cudaSuccess || !g) {
      cudaGetLastError();
      if (g) cudaGraphDestroy(g);
      graph_fallbacks_++;
      graph_fallback_reason_ = "capture invalidated";
      lanczos_graph_ = false;
      return false;
    }
    // reuse the executable graph of the previous solve when only parameters changed
    bool updated = false;
    if (graph_exec_) {
      cudaGraphExecUpdateResultInfo info;
      updated = cudaGraphExecUpdate(graph_exec_, g, &info) == cudaSuccess;
      if (!updated) {
        cudaGetLastError();
        cudaGraphExecDestroy(graph_exec_);
        graph_exec_ = nullptr;
      }
    }
    if (!updated) cuda_check(cudaGraphInstantiate(&graph_exec_, g, 0), "graph instantiate");
    cudaGraphDestroy(g);
    graph_built = true;
    return true;
  };
  auto graph_ok = [&]() { return graphs && lanczos_graph_ && (split || !(sb.tune_cand >= 0 && !sb.tune_pending)); };
  bool done = false;
  while (iter_out <= loop_out && !done) {
    iter_out++;
    last = 1;
    ritzmin = lastmin;
    cuda_check(cudaMemcpyAsync(v(1), d_psi, n * sizeof(double2), cudaMemcpyDeviceToDevice, st), "copy");
    normalize(v(1), n);
    cuda_check(launch_multi_dot(v(1), ld, 1, v(1), n, d_part, uu_d + 1, st), "uu");
    do_hpsi(1);
    cuda_check(launch_multi_dot(v(1), ld, 1, v(2), n, d_part, a_d + 1, st), "alpha");
    read_back(S_ALPHA + 1, 1);
    ritzmin = h_scal[S_ALPHA + 1];
    double zlast = 1.0;   // T_1 = [alpha_1]: its eigenvector is (1)
    bool conv = false;
    while (last < loop_in) {
      // One iteration runs on the device without a host decision; the host
      // reads {ritz of T_(last+1), |w|^2, alpha_(last+1)} once at its end.  The
      // reference stops before the Gram-Schmidt step when beta_last <= lanzero
      // (eigen.f90:70-74); here that test is applied to the read-back value and
      // the iteration's remaining work (vectors last+1, last+2 and slots last+1)
      // is discarded, which leaves the same state.
      if (graph_ok() && (graph_built || build_graph())) {
        *h_it = last;
        cuda_check(cudaGraphLaunch(graph_exec_, st), "graph launch");
        cuda_check(cudaStreamSynchronize(st), "sync");
        tune_observe();
        float ms = 0.f;
        cuda_check(cudaEventElapsedTime(&ms, graph_ev_[0], graph_ev_[1]), "event time");
        graph_hms += ms;
        graph_replays_++;
        calls++;
      } else {
        double2* w = v(last + 1);
        cuda_check(launch_lanczos_update(w, v(last), last >= 2 ? v(last - 1) : nullptr, a_d + last,
                                         b_d + (last >= 2 ? last - 1 : 0), n, st),
                   "update");
        cuda_check(launch_multi_dot(w, ld, 1, w, n, d_part, d_scal + S_N2, st), "iteration norm");
        cuda_check(launch_scale(w, d_scal + S_N2, n, 1, st), "normalize");
        // Gram_Schmidt_process against v(1..last) (block.f90:1251-1289)
        cuda_check(launch_multi_dot(v(1), ld, last, w, n, d_part, uv_d + 1, st), "uv");
        cuda_check(launch_gs_subtract(w, v(1), ld, last, uv_d + 1, uu_d + 1, n, st), "gs");
        normalize(w, n);
        cuda_check(launch_multi_dot(w, ld, 1, w, n, d_part, uu_d + last + 1, st), "uu");
        do_hpsi(last + 1);
        cuda_check(launch_multi_dot(v(last + 1), ld, 1, v(last + 2), n, d_part, a_d + last + 1, st), "alpha");
        cuda_check(launch_lanczos_tail(d_scal + S_N2, a_d, b_d, last + 1, d_scal + S_RES, d_scal + S_PKT,
                                       res_tol > 0 ? d_scal + S_ZR : nullptr, st),
                   "tail");
        read_back(S_PKT, 4);
      }
      const double beta_last = std::sqrt(h_scal[S_PKT + 1]);
      if (std::fabs(beta_last) <= lanzero) {
        conv = true;
        break;
      }
      // residual stop: ||H y - theta y|| = beta_last |z_last| for the Ritz pair of T_last
      if (res_tol > 0 && beta_last * zlast <= res_tol) {
        conv = true;
        break;
      }
      zlast = h_scal[S_PKT + 3];
      last++;
      const double d0 = h_scal[S_PKT];
      const double tol = std::max(lanzero, rel_tol * std::fabs(d0));
      if ((res_tol <= 0 && std::fabs(d0 - ritzmin) <= tol) || (last == loop_in && iter_out == loop_out)) {
        ritzmin = d0;
        lastmin = ritzmin;
        conv = true;
        break;
      }
      ritzmin = d0;
      lastmin = ritzmin;
    }
    if (conv) {
      done = true;
      break;
    }
    // restart (eigen.f90:114-129)
    ritzmin = tridiag_vec(last);
    lastmin = ritzmin;
    cuda_check(launch_combine(d_psi, v(1), ld, last, d_scal + S_Z, n, st), "combine");
    normalize(d_psi, n);
  }
  // eigen.f90:137-156
  ritzmin = tridiag_vec(last);
  cuda_check(launch_combine(d_psi, v(1), ld, last, d_scal + S_Z, n, st), "combine");
  normalize(d_psi, n);
  cuda_check(cudaStreamSynchronize(st), "sync");
  double hms = graph_hms;
  for (int c = 0; c < eager_calls; ++c) {
    float ms = 0.f;
    cuda_check(cudaEventElapsedTime(&ms, hpsi_events[2 * c], hpsi_events[2 * c + 1]), "event time");
    hms += ms;
  }
  *iters = (iter_out - 1) * loop_in + last;
  *e0 = ritzmin;
  if (hpsi_ms) *hpsi_ms = hms;
  if (hpsi_calls) *hpsi_calls = calls;
}

// --------------------------------------------------------------- density matrix + truncation
// Get_density_matrix_sys_new / _env_new (den_mat.f90:103-183): levels = 1 takes
// the normalised wave, levels >= 2 averages the density matrices of the first two
// waves, unnormalised, as the reference does (den_mat.f90:127-135); d_psi holds
// the waves one after the other.  One sub-block per wave sector:
// sys psi psi^H (den_mat.f90:41-43), env psi^H psi (den_mat.f90:89-91).
DBlock Engine::density_matrix(int side, const double2* d_psi, const WLayout& wl, int levels) {
  if (levels < 1) throw Error(-1, "levels must be at least 1");
  DBlock den;
  den.len = side == 0 ? wl.sys_len : wl.env_len;
  den.num = wl.num;
  long long tot = 0;
  for (int k = 0; k < wl.num; ++k) {
    const WSec& w = wl.sec[k];
    SubDesc d;
    d.num_up = side == 0 ? w.sys_num_up : w.env_num_up;
    d.num_down = side == 0 ? w.sys_num_down : w.env_num_down;
    d.row_dim = d.sdim = side == 0 ? w.sys_dim : w.env_dim;
    d.off = tot;
    tot += (long long)d.sdim * d.sdim;
    den.dim += d.sdim;
    den.sub.push_back(d);
  }
  den.buf = std::make_shared<DevBuf>((size_t)std::max<long long>(tot, 1), st, false);
  DevBuf w(levels == 1 ? (size_t)std::max<long long>(wl.dim, 1) : 1, st, false);
  const double2* src = d_psi;
  if (levels == 1) {
    cuda_check(cudaMemcpyAsync(w.p, d_psi, wl.dim * sizeof(double2), cudaMemcpyDeviceToDevice, st), "copy");
    normalize(w.p, wl.dim);
    src = w.p;
  }
  TaskList tl;
  for (int k = 0; k < wl.num; ++k) {
    const WSec& s = wl.sec[k];
    const int d = den.sub[k].sdim;
    const int g = tl.add_group(den.ptr(k), BASE_ABS, 0, d, d, d, 0);
    for (int l = 0; l < std::min(levels, 2); ++l) {
      GTerm t{};
      t.kind = TK_GEMM;
      t.ar = levels == 1 ? 1.0 : 0.5;
      t.l_base = t.r_base = BASE_IN;
      t.l_off = t.r_off = s.off + (long long)l * wl.dim;
      t.l_ld = t.r_ld = s.sys_dim;
      if (side == 0) {
        t.l_op = OP_N;
        t.r_op = OP_C;
        t.K = s.env_dim;
      } else {
        t.l_op = OP_C;
        t.r_op = OP_N;
        t.K = s.sys_dim;
      }
      tl.gterms[g].push_back(t);
    }
  }
  tl.upload(st);
  run_tasks(tl, const_cast<double2*>(src), nullptr, nullptr);
  cuda_check(cudaStreamSynchronize(st), "density matrix sync");
  return den;
}

void Engine::truncate(int side, const double2* d_psi, const WLayout& wl, int kept_min, int kept_max, double trun_err,
                      TruncResult& out) {
  DBlock den = density_matrix(side, d_psi, wl, 1);
  truncation_operator(den, kept_min, kept_max, trun_err, out);
}

// Get_truncation_operator (den_mat.f90:190-418) on a density matrix of one
// sub-block per sector; den is overwritten by its eigenvectors.
void Engine::truncation_operator(DBlock& den, int kept_min, int kept_max, double trun_err, TruncResult& out) {
  const double thr = 1.0000000036274937e-15;   // 1.0E-15 default real, den_mat.f90:278,330
  const int nsec = den.num;
  for (const auto& s : den.sub)
    if (s.row_dim != s.sdim || s.down_dif != 0) throw Error(-1, "density matrix sub-blocks must be square");
  // zheev per sector (den_mat.f90:243): cuSOLVER zheevd, eigenvalues ascending.
  // Sectors are dealt to the lanes largest first, each to the least loaded lane.
  int dim = 0;
  std::vector<int> eoffs(nsec);
  for (int k = 0; k < nsec; ++k) {
    eoffs[k] = dim;
    dim += den.sub[k].sdim;
  }
  DevBuf ev((size_t)(dim + 2) / 2 + 1, st, false);
  double* d_ev = reinterpret_cast<double*>(ev.p);
  DevBuf info((size_t)(nsec + 1) / 4 + 1, st, true);   // one int per sector
  int* d_info = reinterpret_cast<int*>(info.p);
  if (!eig) {   // handles, streams and workspaces: not while another engine captures a graph
    std::unique_lock<std::shared_mutex> no_capture(capture_mutex());
    eig = std::make_shared<EigLanes>(kEigLanes, device_);
  }
  std::vector<int> order(nsec);
  for (int k = 0; k < nsec; ++k) order[k] = k;
  auto sdim = [&](int k) { return den.sub[k].sdim; };
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return sdim(a) > sdim(b); });
  std::vector<std::vector<int>> mine(kEigLanes);
  std::vector<double> load(kEigLanes, 0.0);
  for (int k : order) {
    if (sdim(k) <= 0) continue;
    int l = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    mine[l].push_back(k);
    double d = sdim(k);
    load[l] += d * d * d + 2.0e5;   // O(d^3) work plus a fixed launch cost
  }
  cuda_check(cudaEventRecord(eig->fork, st), "event");
  EigLanes* E = eig.get();
  eig->run([&](int l) {
    if (mine[l].empty()) return;
    auto& L = E->lane[l];
    cuda_check(cudaStreamWaitEvent(L.s, E->fork, 0), "wait");
    const int maxd = sdim(mine[l].front());
    int lwork = 0;
    if (cusolverDnZheevd_bufferSize(L.h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, maxd,
                                    reinterpret_cast<cuDoubleComplex*>(den.buf->p), maxd, d_ev, &lwork) !=
        CUSOLVER_STATUS_SUCCESS)
      throw Error(-3, "zheevd buffer size");
    if (lwork > L.lwork) {
      L.work = std::make_shared<DevBuf>((size_t)lwork + 1, L.s, false);
      L.lwork = lwork;
    }
    for (int k : mine[l]) {
      const int d = sdim(k);
      if (cusolverDnZheevd(L.h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, d,
                           reinterpret_cast<cuDoubleComplex*>(den.ptr(k)), d, d_ev + eoffs[k],
                           reinterpret_cast<cuDoubleComplex*>(L.work->p), L.lwork, d_info + k) !=
          CUSOLVER_STATUS_SUCCESS)
        throw Error(-3, "zheevd");
    }
    cuda_check(cudaEventRecord(L.done, L.s), "event");
  });
  for (int l = 0; l < kEigLanes; ++l)
    if (!mine[l].empty()) cuda_check(cudaStreamWaitEvent(st, eig->lane[l].done, 0), "wait");
  // canonical eigenvector phases (see launch_phase_fix)
  for (int k = 0; k < nsec; ++k) {
    int d = den.sub[k].sdim;
    if (d > 0) cuda_check(launch_phase_fix(den.ptr(k), d, d, st), "phase_fix");
  }
  std::vector<double> evh(dim + 1);
  if (dim) cuda_check(cudaMemcpyAsync(evh.data() + 1, d_ev, dim * sizeof(double), cudaMemcpyDeviceToHost, st), "d2h");
  std::vector<int> infoh(nsec, 0);
  if (nsec) cuda_check(cudaMemcpyAsync(infoh.data(), d_info, nsec * sizeof(int), cudaMemcpyDeviceToHost, st), "d2h");
  cuda_check(cudaStreamSynchronize(st), "sync");
  for (int k = 0; k < nsec; ++k)
    if (infoh[k] != 0) throw Error(-3, "zheevd did not converge");
  // eigenvalues at rounding-noise level count as exact zeros (see null_complete)
  for (int i = 1; i <= dim; ++i)
    if (evh[i] < kZeroWeight) evh[i] = 0.0;
  // den_mat.f90:249-333 on the host (scalars only)
  std::vector<int> idx(dim + 1), eigs(dim + 1), sidx0(nsec);
  std::vector<double> evs(dim + 1);
  int p = 0;
  for (int k = 0; k < nsec; ++k) {
    int d = den.sub[k].sdim;
    int S2 = den.sub[k].num_down;
    sidx0[k] = p + 1;
    for (int i = 0; i < d; ++i) {
      ++p;
      idx[p] = p;
      evs[p] = evh[p];
      eigs[p] = S2 + 1;
    }
  }
  double ent1 = 0.0;
  for (int i = 1; i <= dim; ++i)
    if (evs[i] >= thr) {
      double v1 = evs[i] / eigs[i];
      ent1 = ent1 - v1 * std::log(v1) * eigs[i];
    }
  if (dim >= 1) quicksort_double(evs, idx, 1, dim);
  double tp = 0.0;
  for (int i = 1; i <= dim; ++i) tp += evs[i];
  for (int i = 1; i <= dim; ++i) evs[i] = evs[i] / tp;
  double err = 0.0;
  int ns;
  if (dim <= kept_min) {
    ns = dim;
  } else {
    for (int i = kept_min + 1; i <= dim; ++i) err += evs[i];
    ns = kept_min;
    while (err > trun_err) {
      ns++;
      err = err - evs[ns];
      if (err <= trun_err || ns >= kept_max) break;
    }
  }
  double ent = 0.0;
  for (int i = 1; i <= dim; ++i)
    if (evs[i] >= thr) ent = ent - evs[i] * std::log(evs[i]);
  std::vector<int> cnt(nsec, 0);
  for (int k = 1; k <= ns; ++k) {
    int id = idx[k];
    int sec = (int)(std::upper_bound(sidx0.begin(), sidx0.end(), id) - sidx0.begin()) - 1;
    cnt[sec]++;
  }
  // U = top eigenvectors of every sector (den_mat.f90:352-402)
  DBlock& U = out.trun;
  U = DBlock();
  long long uo = 0;
  for (int k = 0; k < nsec; ++k) {
    if (cnt[k] <= 0) continue;
    SubDesc s;
    s.num_up = den.sub[k].num_up;
    s.num_down = den.sub[k].num_down;
    s.row_dim = den.sub[k].sdim;
    s.sdim = cnt[k];
    s.off = uo;
    uo += (long long)s.row_dim * s.sdim;
    U.sub.push_back(s);
  }
  U.num = (int)U.sub.size();
  U.len = den.len;
  U.buf = std::make_shared<DevBuf>((size_t)std::max<long long>(uo, 1), st, false);
  // kept columns of every sector; kept zero-weight columns are then replaced by
  // the canonical complement basis on the GPU (null_complete)
  std::vector<NullJob> nulls;
  int ui = 0;
  for (int k = 0; k < nsec; ++k) {
    if (cnt[k] <= 0) continue;
    const SubDesc& s = U.sub[ui++];
    int row = s.row_dim, col = s.sdim;
    int sig = 0;
    for (int c = 0; c < col; ++c)
      if (evh[sidx0[k] + row - col + c] > 0.0) sig++;
    cuda_check(cudaMemcpyAsync(U.buf->p + s.off, den.ptr(k) + (long long)(row - col) * row,
                               (size_t)row * col * sizeof(double2), cudaMemcpyDeviceToDevice, st),
               "U copy");
    if (sig < col) nulls.push_back(NullJob{U.buf->p + s.off, row, sig, col - sig});
    U.dim += col;
  }
  null_complete(nulls);
  out.num_state = ns;
  out.err = err;
  out.ent = ent;
  out.ent_mult = ent1;
  out.spectrum.assign(evs.begin() + 1, evs.end());
  cuda_check(cudaStreamSynchronize(st), "sync");
}

// ------------------------------------------------------------------ block growth + U^H O U
void Engine::grow(int side, DModel& pre, const Basis& basis, const DBlock& trun, int mshift) {
  const bool env = side == 1;
  TaskList ta;   // enlargement (scatter) tasks
  auto find_bs = [&](int up, int down) { return basis.find(up, down); };
  auto alloc_like_basis = [&](DBlock& b) {   // diagonal operator on the enlarged basis
    b = DBlock();
    b.len = basis.len;
    b.num = basis.num;
    b.dim = basis.dim;
    long long off = 0;
    for (const auto& S : basis.sec) {
      SubDesc s;
      s.num_up = S.num_up;
      s.num_down = S.num_down;
      s.row_dim = s.sdim = S.dim;
      s.off = off;
      off += (long long)S.dim * S.dim;
      b.sub.push_back(s);
    }
    b.buf = std::make_shared<DevBuf>((size_t)std::max<long long>(off, 1), st, false);
  };
  auto alloc_ndia = [&](DBlock& b, int up_dif, int K) {   // block.f90:2655-2712
    b = DBlock();
    b.len = basis.len;
    b.up_dif = up_dif;
    b.down_dif = K;
    long long off = 0;
    for (int x = 0; x < basis.num; ++x)
      for (int dd = -K; dd <= K; dd += 2) {
        int y = find_bs(basis.sec[x].num_up + up_dif, basis.sec[x].num_down + dd);
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
  };
  auto groups_of = [&](DBlock& b) {
    std::vector<int> g;
    for (int i = 0; i < b.num; ++i)
      g.push_back(ta.add_group(b.ptr(i), BASE_ABS, 0, b.sub[i].row_dim, b.sub[i].row_dim, b.sub[i].sdim, 0));
    return g;
  };
  auto axpy = [&](int g, double2* src, int ld, uint8_t op, int r0, int c0, int rm, int rn, cplx a) {
    GTerm t{};
    t.kind = TK_AXPY;
    t.ar = a.real();
    t.ai = a.imag();
    t.r_base = BASE_ABS;
    t.r_off = absoff(src);
    t.r_ld = ld;
    t.r_op = op;
    t.r0 = r0;
    t.c0 = c0;
    t.rm = rm;
    t.rn = rn;
    ta.gterms[g].push_back(t);
  };
  auto diag = [&](int g, int r0, int c0, int rm, cplx a) {
    GTerm t{};
    t.kind = TK_DIAG;
    t.ar = a.real();
    t.ai = a.imag();
    t.r0 = r0;
    t.c0 = c0;
    t.rm = rm;
    t.rn = rm;
    ta.gterms[g].push_back(t);
  };
  // update_block_dia (block.f90:2495-2548)
  auto update_block_dia = [&](const DBlock& blk, DBlock& nb, const std::vector<int>& g) {
    for (int k = 0; k < nb.num; ++k)
      for (const auto& p : basis.sec[k].pcs)
        for (int i = 0; i < blk.num; ++i)
          if (blk.sub[i].num_up == p.bl_num_up && blk.sub[i].num_down == p.bl_num_down) {
            double c1 = std::sqrt((1.0 + nb.sub[k].num_down) / (1.0 + blk.sub[i].num_down));
            axpy(g[k], blk.ptr(i), blk.sub[i].row_dim, OP_N, p.spos, p.spos, p.sdim, p.sdim, c1);
            break;
          }
  };
  // update_site_dia (block.f90:2554-2615)
  auto update_site_dia = [&](const SiteOp& so, DBlock& nb, const std::vector<int>& g) {
    for (int k = 0; k < nb.num; ++k)
      for (const auto& p : basis.sec[k].pcs)
        for (const auto& s : so.sub)
          if (s.num_up == p.st_num_up && s.num_down == p.st_num_down) {
            double c1 = std::sqrt((1.0 + nb.sub[k].num_down) / (1.0 + s.num_down));
            diag(g[k], p.spos, p.spos, p.sdim, s.val * c1);
            break;
          }
  };
  // update_block_ndia_sys / _env (block.f90:2624-3036)
  auto update_block_ndia = [&](const DBlock& blk, DBlock& nb, const std::vector<int>& g, char flag) {
    int up_dif = blk.up_dif, K = blk.down_dif;
    for (int i = 0; i < nb.num; ++i) {
      const SubDesc& o = nb.sub[i];
      int rid = find_bs(o.num_up, o.num_down), lid = find_bs(o.num_up + up_dif, o.num_down + o.down_dif);
      if (rid < 0 || lid < 0) continue;
      int lnd = o.num_down + o.down_dif, rnd = o.num_down;
      for (const auto& p : basis.sec[rid].pcs)
        for (int sdd = -K; sdd <= K; sdd += 2) {
          int bid = -1;
          for (int y = 0; y < blk.num; ++y)
            if (blk.sub[y].num_up == p.bl_num_up && blk.sub[y].num_down == p.bl_num_down && blk.sub[y].down_dif == sdd) {
              bid = y;
              break;
            }
          if (bid < 0) continue;
          int lsu = p.bl_num_up + up_dif, lsd = p.bl_num_down + sdd;
          const Piece* q = nullptr;
          for (const auto& qq : basis.sec[lid].pcs)
            if (qq.bl_num_up == lsu && qq.bl_num_down == lsd && qq.st_num_down == p.st_num_down) {
              q = &qq;
              break;
            }
          if (!q) continue;
          double sg = (env && flag == 'F') ? ((p.st_num_up % 2 == 0) ? 1.0 : -1.0) : 1.0;
          int j1 = lnd, j2 = K, j3 = rnd, j4 = p.bl_num_down, j5 = p.st_num_down, j6 = lsd;
          double c = w6j(j1, j2, j3, j4, j5, j6);
          c = c * std::sqrt((1.0 + j1) * (1.0 + j3)) * pm1((j6 + j5 + j3 + j2) / 2);
          if (c == 0.0) continue;
          axpy(g[i], blk.ptr(bid), blk.sub[bid].row_dim, OP_N, q->spos, p.spos, q->sdim, p.sdim, c * sg);
        }
    }
  };
  // update_site_ndia_sys / _env (block.f90:3047-3459)
  auto update_site_ndia = [&](const SiteOp& so, DBlock& nb, const std::vector<int>& g, char flag) {
    int up_dif = so.up_dif, K = so.down_dif;
    for (int i = 0; i < nb.num; ++i) {
      const SubDesc& o = nb.sub[i];
      int rid = find_bs(o.num_up, o.num_down), lid = find_bs(o.num_up + up_dif, o.num_down + o.down_dif);
      if (rid < 0 || lid < 0) continue;
      int lnd = o.num_down + o.down_dif, rnd = o.num_down;
      for (const auto& p : basis.sec[rid].pcs)
        for (int sdd = -K; sdd <= K; sdd += 2) {
          const SiteSub* ss = nullptr;
          for (const auto& s : so.sub)
            if (s.num_up == p.st_num_up && s.num_down == p.st_num_down && s.down_dif == sdd) {
              ss = &s;
              break;
            }
          if (!ss) continue;
          int lsu = p.st_num_up + up_dif, lsd = p.st_num_down + sdd;
          const Piece* q = nullptr;
          for (const auto& qq : basis.sec[lid].pcs)
            if (qq.st_num_up == lsu && qq.st_num_down == lsd && qq.bl_num_down == p.bl_num_down) {
              q = &qq;
              break;
            }
          if (!q) continue;
          double sg = (!env && flag == 'F') ? ((p.bl_num_up % 2 == 0) ? 1.0 : -1.0) : 1.0;
          int j1 = lnd, j2 = K, j3 = rnd, j4 = p.st_num_down, j5 = p.bl_num_down, j6 = lsd;
          double c = w6j(j1, j2, j3, j4, j5, j6);
          c = c * pm1((j5 + j4 + j1 + j2) / 2) * std::sqrt((1.0 + j1) * (1.0 + j3));
          if (c == 0.0) continue;
          diag(g[i], q->spos, p.spos, p.sdim, c * sg * ss->val);
        }
    }
  };
  // Get_hamiltonian_ndia (get_sys.f90:865-1055), site = site operator on the host
  auto ham_ndia = [&](const DBlock& blk, const SiteOp& so, double coef, DBlock& ham, const std::vector<int>& g,
                      char FlagSign) {
    int up_dif = blk.up_dif, K = blk.down_dif;
    for (int i = 0; i < ham.num; ++i) {
      const SubDesc& hs = ham.sub[i];
      int rid = find_bs(hs.num_up, hs.num_down), lid = find_bs(hs.num_up, hs.num_down + hs.down_dif);
      if (rid < 0 || lid < 0) continue;
      int rnd = hs.num_down;
      for (const auto& p : basis.sec[rid].pcs)
        for (int sdd = -K; sdd <= K; sdd += 2) {
          int bid = -1;
          for (int y = 0; y < blk.num; ++y)
            if (blk.sub[y].num_up == p.bl_num_up && blk.sub[y].num_down == p.bl_num_down && blk.sub[y].down_dif == sdd) {
              bid = y;
              break;
            }
          if (bid < 0) continue;
          int lsu = p.bl_num_up + up_dif, lsd = p.bl_num_down + sdd;
          for (int nsd = std::abs(p.st_num_down - so.down_dif); nsd <= p.st_num_down + so.down_dif; nsd += 2) {
            int sdd2 = p.st_num_down - nsd, nsu = p.st_num_up - so.up_dif;
            const SiteSub* ss = nullptr;
            for (const auto& s : so.sub)
              if (s.num_up == nsu && s.num_down == nsd && s.down_dif == sdd2) {
                ss = &s;
                break;
              }
            const Piece* q = nullptr;
            for (const auto& qq : basis.sec[lid].pcs)
              if (qq.bl_num_up == lsu && qq.bl_num_down == lsd && qq.st_num_down == nsd) {
                q = &qq;
                break;
              }
            if (!q || !ss) continue;
            int j1 = lsd, j2 = p.bl_num_down, j3 = K, j4 = p.st_num_down, j5 = nsd, j6 = rnd;
            double c11 = w6j(j1, j2, j3, j4, j5, j6);
            c11 = c11 * std::sqrt((1.0 + j6) / (1.0 + j3)) * pm1((j2 + j5 + j3 + j6) / 2) * ss->val;
            double sgn = 1.0;
            if (!env) {
              if (FlagSign == 'F' && (p.bl_num_up % 2) == 1) sgn = -1.0;
            } else {
              if (FlagSign == 'F' && (p.st_num_up % 2) == 0) sgn = -1.0;
            }
            if (c11 == 0.0) continue;
            cplx c1 = c11 * coef * sgn;
            axpy(g[i], blk.ptr(bid), blk.sub[bid].row_dim, OP_N, q->spos, p.spos, q->sdim, p.sdim, c1);
            if (so.up_dif != 0)
              axpy(g[i], blk.ptr(bid), blk.sub[bid].row_dim, OP_C, p.spos, q->spos, p.sdim, q->sdim, std::conj(c1));
          }
        }
    }
  };
  auto site_ct = [](const SiteOp& o) {
    SiteOp r;
    r.up_dif = -o.up_dif;
    r.down_dif = o.down_dif;
    for (auto& s : o.sub) r.sub.push_back({s.num_up + o.up_dif, s.num_down + s.down_dif, -s.down_dif, s.val});
    return r;
  };

  const int N1 = pre.len + 1;
  DModel next;
  next.len = N1;
  next.sub.resize(L.num_site + 1);
  alloc_like_basis(next.ham);
  std::vector<int> gH = groups_of(next.ham);
  update_block_dia(pre.ham, next.ham, gH);
  // neighbours of the new site inside the block
  int jlat, shift = 0;
  if (!env) {
    jlat = pre.len + 1;
  } else {
    jlat = L.nposi_lat[pre.len + 1 + mshift];
    shift = mshift;
  }
  struct Nb {
    int k, i1;
  };
  std::vector<Nb> nbs;
  for (int k = 1; k <= Lattice::neibt; ++k) {
    int I = L.NEIB(jlat, k);
    int II = env ? L.nposi_dm[I] - shift : I;
    if (II <= pre.len && II > 0) {
      int i1 = L.INB1(II, pre.len);
      if (i1 > 0 && i1 <= L.nleg11[pre.len]) nbs.push_back({k, i1});
    }
  }
  auto need = [&](int i1, int o) {
    if (i1 < 1 || i1 >= (int)pre.sub.size() || !pre.sub[i1].op[o].buf) throw Error(-1, "grow: missing operator");
  };
  // ij = 1 (hopping), 3 (spin), 5 (density): get_sys.f90:42-291 / 336-584
  DBlock site_new[4];   // enlarged site operators: up, down, sd, sn
  std::vector<int> gS[4];
  std::vector<std::vector<int>> gOps(L.num_site + 1);
  for (int ij : {1, 3, 5}) {
    for (const auto& nb : nbs) {
      double cx = L.JT(nb.k, jlat), csd = L.JD(nb.k, jlat);
      if (ij == 1 && cx != 0.0) {
        if (!env) {
          need(nb.i1, OP_UP);
          ham_ndia(pre.sub[nb.i1].op[OP_UP], site_ct(st_elec_down), cx, next.ham, gH, 'F');
        } else {
          need(nb.i1, OP_DOWN);
          ham_ndia(pre.sub[nb.i1].op[OP_DOWN], site_ct(st_elec_up), cx, next.ham, gH, 'F');
        }
      }
      if (ij == 3 && csd != 0.0) {
        need(nb.i1, OP_SD);
        ham_ndia(pre.sub[nb.i1].op[OP_SD], st_sd, csd, next.ham, gH, 'B');
      }
    }
    for (int y = 1; y <= pre.len; ++y) {
      int i1 = L.INB1(y, pre.len);
      if (i1 > L.nleg11[pre.len]) continue;
      if (ij == 1) {
        for (int o : {OP_UP, OP_DOWN}) {
          need(i1, o);
          const DBlock& b = pre.sub[i1].op[o];
          alloc_ndia(next.sub[i1].op[o], b.up_dif, b.down_dif);
          update_block_ndia(b, next.sub[i1].op[o], groups_of(next.sub[i1].op[o]), 'F');
        }
      }
      if (ij == 3) {
        need(i1, OP_SD);
        const DBlock& b = pre.sub[i1].op[OP_SD];
        alloc_ndia(next.sub[i1].op[OP_SD], b.up_dif, b.down_dif);
        update_block_ndia(b, next.sub[i1].op[OP_SD], groups_of(next.sub[i1].op[OP_SD]), 'B');
      }
      if (ij == 5) {
        need(i1, OP_SN);
        alloc_like_basis(next.sub[i1].op[OP_SN]);
        update_block_dia(pre.sub[i1].op[OP_SN], next.sub[i1].op[OP_SN], groups_of(next.sub[i1].op[OP_SN]));
      }
    }
    if (ij == 1) {
      alloc_ndia(site_new[OP_UP], st_elec_up.up_dif, st_elec_up.down_dif);
      update_site_ndia(st_elec_up, site_new[OP_UP], groups_of(site_new[OP_UP]), 'F');
      alloc_ndia(site_new[OP_DOWN], st_elec_down.up_dif, st_elec_down.down_dif);
      update_site_ndia(st_elec_down, site_new[OP_DOWN], groups_of(site_new[OP_DOWN]), 'F');
    }
    if (ij == 3) {
      alloc_ndia(site_new[OP_SD], st_sd.up_dif, st_sd.down_dif);
      update_site_ndia(st_sd, site_new[OP_SD], groups_of(site_new[OP_SD]), 'B');
    }
    if (ij == 5) {
      alloc_like_basis(site_new[OP_SN]);
      site_new[OP_SN].down_dif = 0;
      update_site_dia(num_elec, site_new[OP_SN], groups_of(site_new[OP_SN]));
    }
  }
  ta.upload(st);
  run_tasks(ta, nullptr, nullptr, nullptr);
  // density-density bonds: Get_hamiltonian_dia (get_sys.f90:776-854) into H, beta=1
  {
    TaskList tb;
    std::vector<int> gh;
    for (int i = 0; i < next.ham.num; ++i)
      gh.push_back(tb.add_group(next.ham.ptr(i), BASE_ABS, 0, next.ham.sub[i].row_dim, next.ham.sub[i].row_dim,
                                next.ham.sub[i].sdim, 1));
    bool any = false;
    for (const auto& nb : nbs) {
      double csn = L.JN(nb.k, jlat);
      if (csn == 0.0) continue;
      const DBlock& o1 = next.sub[nb.i1].op[OP_SN];
      const DBlock& o2 = site_new[OP_SN];
      for (int i = 0; i < next.ham.num; ++i) {
        const SubDesc& hs = next.ham.sub[i];
        int a = -1, b = -1;
        for (int x = 0; x < o1.num; ++x)
          if (o1.sub[x].num_up == hs.num_up && o1.sub[x].num_down == hs.num_down) {
            a = x;
            break;
          }
        for (int x = 0; x < o2.num; ++x)
          if (o2.sub[x].num_up == hs.num_up && o2.sub[x].num_down == hs.num_down) {
            b = x;
            break;
          }
        if (a < 0 || b < 0) continue;
        GTerm t{};
        t.kind = TK_GEMM;
        cplx c1 = csn / std::sqrt(1.0 + hs.num_down);
        t.ar = c1.real();
        t.ai = c1.imag();
        t.l_base = t.r_base = BASE_ABS;
        t.l_off = absoff(o1.ptr(a));
        t.l_ld = hs.sdim;
        t.r_off = absoff(o2.ptr(b));
        t.r_ld = hs.sdim;
        t.l_op = t.r_op = OP_N;
        t.K = hs.sdim;
        tb.gterms[gh[i]].push_back(t);
        any = true;
      }
    }
    if (any) {
      tb.upload(st);
      run_tasks(tb, nullptr, nullptr, nullptr);
    }
  }
  // reorder (get_sys.f90:187-252) and place the new site's operators
  int nleg1 = L.nleg11[pre.len + 1];
  for (int I = 1; I <= pre.len; ++I) {
    int i1 = L.INB1(I, pre.len), J = L.INB1(I, pre.len + 1);
    if (J <= nleg1 && J != i1) next.sub[J] = next.sub[i1];
  }
  int jn = L.INB1(pre.len + 1, pre.len + 1);
  if (jn < 1 || jn > L.num_site) throw Error(-1, "grow: new site is not a boundary site");
  for (int o = 0; o < 4; ++o) next.sub[jn].op[o] = site_new[o];
  // renormalise every kept operator and H (update_trun_ndia / update_trun_dia)
  DModel res;
  res.len = N1;
  res.sub.resize(L.num_site + 1);
  TaskList t1, t2;
  long long mid_elems = 0;
  // optional split form of the renormalisation: eff = (U_l^H O) U_r, so that the
  // phase-1 intermediate is the A operand of phase 2 as the split kernel wants
  const bool split_uou = split_renorm_ && precision_ == 1 && !in_warmup_;
  TaskList s1, s2;
  long long mid2_elems = 0;
  struct Job {
    const DBlock* ori;
    DBlock* eff;
  };
  std::vector<Job> jobs;
  auto plan = [&](const DBlock& ori, DBlock& eff) {
    eff = DBlock();
    eff.len = ori.len;
    eff.up_dif = ori.up_dif;
    eff.down_dif = ori.down_dif;
    int up_dif = ori.up_dif, K = ori.down_dif;
    bool isdia = (K == 0 && up_dif == 0);
    long long off = 0;
    if (isdia) {   // update_trun_dia structure
      for (const auto& u : trun.sub) {
        SubDesc s;
        s.num_up = u.num_up;
        s.num_down = u.num_down;
        s.row_dim = s.sdim = u.sdim;
        s.off = off;
        off += (long long)u.sdim * u.sdim;
        eff.sub.push_back(s);
      }
      eff.dim = trun.dim;
    } else {       // update_trun_ndia structure
      for (int x = 0; x < trun.num; ++x)
        for (int dd = -K; dd <= K; dd += 2) {
          int y = -1;
          for (int z = 0; z < trun.num; ++z)
            if (trun.sub[z].num_up == trun.sub[x].num_up + up_dif && trun.sub[z].num_down == trun.sub[x].num_down + dd) {
              y = z;
              break;
            }
          if (y < 0) continue;
          SubDesc s;
          s.num_up = trun.sub[x].num_up;
          s.num_down = trun.sub[x].num_down;
          s.down_dif = dd;
          s.row_dim = trun.sub[y].sdim;
          s.sdim = trun.sub[x].sdim;
          s.off = off;
          off += (long long)s.row_dim * s.sdim;
          eff.dim += s.sdim;
          eff.sub.push_back(s);
        }
    }
    eff.num = (int)eff.sub.size();
    eff.buf = std::make_shared<DevBuf>((size_t)std::max<long long>(off, 1), st, true);
    for (int i = 0; i < eff.num; ++i) {
      const SubDesc& e = eff.sub[i];
      int rid = -1, lid = -1, oid = -1;
      for (int z = 0; z < trun.num; ++z) {
        if (rid < 0 && trun.sub[z].num_up == e.num_up && trun.sub[z].num_down == e.num_down) rid = z;
        if (lid < 0 && trun.sub[z].num_up == e.num_up + up_dif && trun.sub[z].num_down == e.num_down + e.down_dif) lid = z;
      }
      for (int z = 0; z < ori.num; ++z)
        if (ori.sub[z].num_up == e.num_up && ori.sub[z].num_down == e.num_down &&
            (isdia || ori.sub[z].down_dif == e.down_dif)) {
          oid = z;
          break;
        }
      if (rid < 0 || lid < 0 || oid < 0) continue;
      int orow = ori.sub[oid].row_dim, ocol = ori.sub[oid].sdim, rd = trun.sub[rid].sdim, ldim = trun.sub[lid].sdim;
      long long moff = mid_elems;
      mid_elems += (long long)orow * rd;
      int g1 = t1.add_group(nullptr, BASE_SCR, moff, orow, orow, rd, 0);
      GTerm a{};
      a.kind = TK_GEMM;
      a.ar = 1.0;
      a.l_base = a.r_base = BASE_ABS;
      a.l_off = absoff(ori.ptr(oid));
      a.l_ld = orow;
      a.l_op = OP_N;
      a.r_off = absoff(trun.ptr(rid));
      a.r_ld = trun.sub[rid].row_dim;
      a.r_op = OP_N;
      a.K = ocol;
      t1.gterms[g1].push_back(a);
      int g2 = t2.add_group(eff.ptr(i), BASE_ABS, 0, ldim, ldim, rd, 0);
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
      if (split_uou) {
        const long long m2 = mid2_elems;
        mid2_elems += (long long)ldim * ocol;
        const int h1 = s1.add_group(nullptr, BASE_SCR, m2, ldim, ldim, ocol, 0);
        GTerm c{};   // U_l^H O
        c.kind = TK_GEMM;
        c.ar = 1.0;
        c.l_base = c.r_base = BASE_ABS;
        c.l_off = absoff(trun.ptr(lid));
        c.l_ld = trun.sub[lid].row_dim;
        c.l_op = OP_C;
        c.r_off = absoff(ori.ptr(oid));
        c.r_ld = orow;
        c.r_op = OP_N;
        c.K = orow;
        s1.gterms[h1].push_back(c);
        const int h2 = s2.add_group(eff.ptr(i), BASE_ABS, 0, ldim, ldim, rd, 0);
        GTerm d{};   // (U_l^H O) U_r
        d.kind = TK_GEMM;
        d.ar = 1.0;
        d.l_base = BASE_SCR;
        d.l_off = m2;
        d.l_ld = ldim;
        d.l_op = OP_N;
        d.r_base = BASE_ABS;
        d.r_off = absoff(trun.ptr(rid));
        d.r_ld = trun.sub[rid].row_dim;
        d.r_op = OP_N;
        d.K = ocol;
        s2.gterms[h2].push_back(d);
      }
    }
  };
  for (int ii = 1; ii <= L.nleg11[N1]; ++ii)
    for (int o = 0; o < 4; ++o) {
      if (!next.sub[ii].op[o].buf) throw Error(-1, "grow: missing enlarged operator");
      plan(next.sub[ii].op[o], res.sub[ii].op[o]);
    }
  plan(next.ham, res.ham);
  if (split_uou) {
    SplitData sv;
    build_split_views(s1, s2, sv, st);
    s1.upload_split(st);
    s2.upload_split(st);
    DevBuf mid2((size_t)std::max<long long>(mid2_elems, 1), st, false);
    run_tasks(s1, nullptr, nullptr, mid2.p);
    run_tasks(s2, nullptr, nullptr, mid2.p);
    cuda_check(cudaStreamSynchronize(st), "grow sync");
    check_split_fault();
  } else {
    DevBuf mid((size_t)std::max<long long>(mid_elems, 1), st, false);
    t1.upload(st);
    t2.upload(st);
    run_tasks(t1, nullptr, nullptr, mid.p);
    run_tasks(t2, nullptr, nullptr, mid.p);
    cuda_check(cudaStreamSynchronize(st), "grow sync");
  }
  pre = std::move(res);
}

// --------------------------------------------------------------------- wave transformations
void Engine::wave_trans(int dir, const Basis& sys_bs, const Basis& env_bs, const DBlock& sys_trun,
                        const DBlock& env_trun, const WLayout& ol, const double2* d_old, const WLayout& nl,
                        double2* d_new) {
  cuda_check(cudaMemsetAsync(d_new, 0, std::max<long long>(nl.dim, 1) * sizeof(double2), st), "memset");
  TaskList t1, t2;
  long long scr = 0;
  std::map<std::pair<int, int>, int> gmap;   // (new sector, piece) -> group
  auto findb = [](const DBlock& b, int up, int down) {
    for (int k = 0; k < b.num; ++k)
      if (b.sub[k].num_up == up && b.sub[k].num_down == down) return k;
    return -1;
  };
  struct P2 {
    int nw, piece;
    long long toff;
    int tld, K;
    const double2* B;
    int bld;
    uint8_t bop;
  };
  std::vector<P2> p2s;
  for (int i = 0; i < ol.num; ++i) {
    const WSec& o = ol.sec[i];
    if (dir == 0) {   // wave_trans_LR, dmrg_sub.f90:1495-1631
      int st_id = findb(sys_trun, o.sys_num_up, o.sys_num_down);
      if (st_id < 0) continue;
      for (const auto& E : env_bs.sec) {
        if (E.num_up != o.env_num_up || E.num_down != o.env_num_down) continue;
        for (const auto& p : E.pcs) {
          int et = findb(env_trun, p.bl_num_up, p.bl_num_down);
          int neu = p.bl_num_up, ned = p.bl_num_down;
          for (int nsd = std::abs(o.sys_num_down - p.st_num_down); nsd <= o.sys_num_down + p.st_num_down; nsd += 2) {
            int nsu = o.sys_num_up + p.st_num_up;
            int y = sys_bs.find(nsu, nsd);
            int qi = -1;
            if (y >= 0)
              for (size_t q = 0; q < sys_bs.sec[y].pcs.size(); ++q) {
                const Piece& x = sys_bs.sec[y].pcs[q];
                if (x.bl_num_up == o.sys_num_up && x.bl_num_down == o.sys_num_down && x.st_num_up == p.st_num_up &&
                    x.st_num_down == p.st_num_down) {
                  qi = (int)q;
                  break;
                }
              }
            int nw = nl.find(nsu, nsd, neu, ned);
            if (et < 0 || qi < 0 || nw < 0) continue;
            const Piece& q = sys_bs.sec[y].pcs[qi];
            int j12 = o.sys_num_down, j3 = p.st_num_down, j4 = ned, j123 = nsd, j34 = o.env_num_down;
            double c = pm1((j12 + j3 + j123) / 2) / std::sqrt((1.0 + j12) * (1.0 + j123));
            if (c == 0.0) continue;
            c = c * std::sqrt((1.0 + j123) * (j34 + 1.0));
            if (((j12 + j3 + j4) / 2) % 2 != 0) c = -c;
            if (((j3 + j4 - j34) / 2) % 2 != 0) c = -c;
            int nsub = q.sdim, osub = p.sdim, osd = o.sys_dim;
            long long toff = scr;
            scr += (long long)nsub * osub;
            int g = t1.add_group(nullptr, BASE_SCR, toff, nsub, nsub, osub, 0);
            GTerm a{};
            a.kind = TK_GEMM;
            a.ar = c;
            a.l_base = BASE_ABS;
            a.l_off = absoff(sys_trun.ptr(st_id));
            a.l_ld = sys_trun.sub[st_id].row_dim;
            a.l_op = OP_C;
            a.r_base = BASE_IN;
            a.r_off = o.off + (long long)p.spos * osd;
            a.r_ld = osd;
            a.r_op = OP_N;
            a.K = osd;
            t1.gterms[g].push_back(a);
            p2s.push_back({nw, qi, toff, nsub, osub, env_trun.ptr(et), env_trun.sub[et].row_dim, OP_C});
          }
        }
      }
    } else {          // wave_trans_RL, dmrg_sub.f90:1660-1785
      int et_id = findb(env_trun, o.env_num_up, o.env_num_down);
      if (et_id < 0) continue;
      for (const auto& Sx : sys_bs.sec) {
        if (Sx.num_up != o.sys_num_up || Sx.num_down != o.sys_num_down) continue;
        for (const auto& p : Sx.pcs) {
          int nsu = p.bl_num_up, nsd = p.bl_num_down;
          for (int ned = std::abs(o.env_num_down - p.st_num_down); ned <= o.env_num_down + p.st_num_down; ned += 2) {
            int neu = o.env_num_up + p.st_num_up;
            int st_id = findb(sys_trun, nsu, nsd);
            int y = env_bs.find(neu, ned);
            int qi = -1;
            if (y >= 0)
              for (size_t q = 0; q < env_bs.sec[y].pcs.size(); ++q) {
                const Piece& x = env_bs.sec[y].pcs[q];
                if (x.bl_num_up == o.env_num_up && x.bl_num_down == o.env_num_down && x.st_num_up == p.st_num_up &&
                    x.st_num_down == p.st_num_down) {
                  qi = (int)q;
                  break;
                }
              }
            int nw = nl.find(nsu, nsd, neu, ned);
            if (st_id < 0 || qi < 0 || nw < 0) continue;
            const Piece& q = env_bs.sec[y].pcs[qi];
            int j12 = o.env_num_down, j3 = p.st_num_down, j4 = nsd, j123 = ned, j34 = o.sys_num_down;
            double c = pm1((j34 + j4 + j3) / 2) / std::sqrt((1.0 + j12) * (1.0 + j4));
            if (c == 0.0) continue;
            c = c * std::sqrt((1.0 + j123) * (j34 + 1.0));
            if (((j4 + j3 + j12) / 2) % 2 != 0) c = -c;
            if (((j12 + j3 - j123) / 2) % 2 != 0) c = -c;
            int nsys = nl.sec[nw].sys_dim, oed = o.env_dim, osub = p.sdim;
            long long toff = scr;
            scr += (long long)nsys * oed;
            int g = t1.add_group(nullptr, BASE_SCR, toff, nsys, nsys, oed, 0);
            GTerm a{};
            a.kind = TK_GEMM;
            a.ar = c;
            a.l_base = BASE_ABS;
            a.l_off = absoff(sys_trun.ptr(st_id));
            a.l_ld = sys_trun.sub[st_id].row_dim;
            a.l_op = OP_N;
            a.r_base = BASE_IN;
            a.r_off = o.off + p.spos;
            a.r_ld = o.sys_dim;
            a.r_op = OP_N;
            a.K = osub;
            t1.gterms[g].push_back(a);
            p2s.push_back({nw, qi, toff, nsys, oed, env_trun.ptr(et_id), env_trun.sub[et_id].row_dim, OP_N});
            (void)q;
          }
        }
      }
    }
  }
  for (const auto& x : p2s) {
    auto key = std::make_pair(x.nw, x.piece);
    auto it = gmap.find(key);
    int g;
    if (it == gmap.end()) {
      const WSec& ns = nl.sec[x.nw];
      if (dir == 0) {
        const Piece& q = sys_bs.sec[sys_bs.find(ns.sys_num_up, ns.sys_num_down)].pcs[x.piece];
        g = t2.add_group(nullptr, BASE_OUT, ns.off + q.spos, ns.sys_dim, q.sdim, ns.env_dim, 0);
      } else {
        const Piece& q = env_bs.sec[env_bs.find(ns.env_num_up, ns.env_num_down)].pcs[x.piece];
        g = t2.add_group(nullptr, BASE_OUT, ns.off + (long long)q.spos * ns.sys_dim, ns.sys_dim, ns.sys_dim, q.sdim, 0);
      }
      gmap[key] = g;
    } else {
      g = it->second;
    }
    GTerm b{};
    b.kind = TK_GEMM;
    b.ar = 1.0;
    b.l_base = BASE_SCR;
    b.l_off = x.toff;
    b.l_ld = x.tld;
    b.l_op = OP_N;
    b.r_base = BASE_ABS;
    b.r_off = absoff(x.B);
    b.r_ld = x.bld;
    b.r_op = x.bop;
    b.K = x.K;
    t2.gterms[g].push_back(b);
  }
  DevBuf sc((size_t)std::max<long long>(scr, 1), st, false);
  t1.upload(st);
  t2.upload(st);
  run_tasks(t1, const_cast<double2*>(d_old), d_new, sc.p);
  run_tasks(t2, const_cast<double2*>(d_old), d_new, sc.p);
  normalize(d_new, nl.dim);
  cuda_check(cudaStreamSynchronize(st), "wave_trans sync");
}

// ------------------------------------------------------------------------------ sweep driver
void Engine::capture_superblock(const DevBufP& psi) {
  cap = Capture();
  auto put_model = [&](const DModel& m) {
    int nops = L.nleg11[m.len];
    cap.ints.push_back(m.len);
    cap.ints.push_back(nops);
    download_block(m.ham, cap.ints, cap.data);
    for (int i = 1; i <= nops; ++i)
      for (int o = 0; o < 4; ++o) download_block(m.sub[i].op[o], cap.ints, cap.data);
  };
  auto put_basis = [&](const Basis& b) {
    cap.ints.insert(cap.ints.end(), {b.len, b.num, b.dim});
    for (const auto& s : b.sec) cap.ints.insert(cap.ints.end(), {s.num_up, s.num_down, s.dim, (int)s.pcs.size()});
    for (const auto& s : b.sec)
      for (const auto& p : s.pcs)
        cap.ints.insert(cap.ints.end(), {p.bl_num_up, p.bl_num_down, p.st_num_up, p.st_num_down, p.spos, p.sdim});
  };
  put_model(sb.sys);
  put_model(sb.env);
  put_basis(sb.sys_bs);
  put_basis(sb.env_bs);
  const WLayout& w = sb.wl;
  cap.ints.insert(cap.ints.end(), {w.sys_len, w.env_len, w.num, (int)w.dim});
  for (const auto& s : w.sec)
    cap.ints.insert(cap.ints.end(), {s.sys_num_up, s.sys_num_down, s.env_num_up, s.env_num_down, s.sys_dim, s.env_dim});
  size_t d0 = cap.data.size();
  cap.data.resize(d0 + w.dim);
  cuda_check(cudaMemcpyAsync(&cap.data[d0], psi->p, w.dim * sizeof(double2), cudaMemcpyDeviceToHost, st), "d2h");
  cuda_check(cudaStreamSynchronize(st), "sync");
  cap.sys_len = sb.sys.len;
  cap.env_len = sb.env.len;
  cap.valid = true;
}

void Engine::lanczos_step(int phase, DModel& sys, DModel& env, const Basis& sys_bs, const Basis& env_bs,
                          const WLayout& wl, DevBufP& psi, StepRec& rec) {
  rec.phase = phase;
  rec.sys_len = sys.len;
  rec.env_len = env.len;
  auto t0 = phase_clock(st);
  superblock_set(DModel(sys), DModel(env), Basis(sys_bs), Basis(env_bs), WLayout(wl));
  auto t1 = phase_clock(st);
  rec.set_seconds = secs(t0, t1);
  if (nsolve_ == capture_step) capture_superblock(psi);
  double hms = 0;
  int calls = 0;
  t1 = phase_clock(st);
  lanczos(psi->p, lanzero_, &rec.iters, &rec.e0, &hms, &calls);
  rec.lanczos_seconds = secs(t1, phase_clock(st));
  rec.split_iters = last_split_iters;
  rec.split_e0 = last_split_e0;
  rec.hpsi_calls = calls;
  rec.hpsi_seconds = hms * 1e-3;
  rec.hpsi_flops = sb.ref_flops * calls;
  nsolve_++;
}

// Appends a step record; with TSC_PROGRESS set in the environment, also prints
// it to stderr (long runs show their progress as they go).
void Engine::record_step(const StepRec& rec, std::vector<StepRec>* log) {
  if (log) log->push_back(rec);
  static const bool progress = std::getenv("TSC_PROGRESS") != nullptr;
  if (progress)
    std::fprintf(stderr, "step phase %d sys %d env %d e0 %.12f iters %d (split %d) kept %d  %.2f s (lanczos %.2f, truncate %.2f, grow %.2f)\n",
                 rec.phase, rec.sys_len, rec.env_len, rec.e0, rec.iters, rec.split_iters, rec.num_state,
                 rec.step_seconds, rec.lanczos_seconds, rec.truncate_seconds, rec.grow_seconds);
}

void Engine::warm_up(int end_id, double trun_err, std::vector<StepRec>* log) {
  struct Flag {
    bool& f;
    explicit Flag(bool& x) : f(x) { f = true; }
    ~Flag() { f = false; }
  } in_warmup(in_warmup_);
  int label = 1;
  L.setup(1, 1);
  DModel sys = site_model(), env = site_model();
  models_.put(0, 1, sys);
  models_.put(1, 1, env);
  while (label + 1 <= end_id && !solve_cap_reached()) {
    auto t0 = std::chrono::steady_clock::now();
    Basis sys_bs = get_basis(sys.ham), env_bs = get_basis(env.ham);
    L.setup(sys.ham.len, env.ham.len);
    float v = 1.0f * (float)(sys_bs.len + env_bs.len) / (float)L.num_site * (float)tot_num_up + 0.001f;
    int tot_up = (int)v;
    tot_up -= tot_up % 2;
    if (tot_up > tot_num_up) tot_up = tot_num_up;
    WLayout wl = get_super(sys_bs, env_bs, tot_up, 0);
    DevBufP psi = std::make_shared<DevBuf>((size_t)std::max<long long>(wl.dim, 1), st, false);
    wave_initialize(wl, psi->p);
    StepRec rec{};
    lanczos_step(0, sys, env, sys_bs, env_bs, wl, psi, rec);
    auto ident = [&](const Basis& bs) {
      DBlock t;
      t.len = bs.len;
      t.num = bs.num;
      t.dim = bs.dim;
      long long off = 0;
      for (const auto& S : bs.sec) {
        SubDesc s;
        s.num_up = S.num_up;
        s.num_down = S.num_down;
        s.row_dim = s.sdim = S.dim;
        s.off = off;
        off += (long long)S.dim * S.dim;
        t.sub.push_back(s);
      }
      t.buf = std::make_shared<DevBuf>((size_t)std::max<long long>(off, 1), st, true);
      std::vector<double2> h((size_t)off, make_double2(0.0, 0.0));
      for (const auto& s : t.sub)
        for (int j = 0; j < s.sdim; ++j) h[s.off + (long long)j * s.row_dim + j] = make_double2(1.0, 0.0);
      cuda_check(cudaMemcpyAsync(t.buf->p, h.data(), off * sizeof(double2), cudaMemcpyHostToDevice, st), "h2d");
      cuda_check(cudaStreamSynchronize(st), "sync");
      return t;
    };
    TruncResult sr, er;
    auto tp = phase_clock(st);
    if (sys_bs.dim <= kept_max_) {
      sr.trun = ident(sys_bs);
      sr.num_state = sys_bs.dim;
    } else {
      truncate(0, psi->p, wl, kept_min_, kept_max_, trun_err, sr);
    }
    rec.num_state = sr.num_state;
    rec.err = sr.err;
    rec.ent = sr.ent;
    rec.ent_mult = sr.ent_mult;
    auto tq = phase_clock(st);
    rec.truncate_seconds += secs(tp, tq);
    grow(0, sys, sys_bs, sr.trun, 0);
    tp = phase_clock(st);
    rec.grow_seconds += secs(tq, tp);
    if (env_bs.dim <= kept_max_) er.trun = ident(env_bs);
    else truncate(1, psi->p, wl, kept_min_, kept_max_, trun_err, er);
    tq = phase_clock(st);
    rec.truncate_seconds += secs(tp, tq);
    grow(1, env, env_bs, er.trun, sys.len);
    rec.grow_seconds += secs(tq, phase_clock(st));
    models_.put(0, label + 1, sys);
    models_.put(1, label + 1, env);
    sys_truns[label + 1] = sr.trun;
    env_truns[label + 1] = er.trun;
    sys_bsm[label + 1] = sys_bs;
    env_bsm[label + 1] = env_bs;
    disk_layout = wl;
    disk_wave = psi;
    rec.step_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    record_step(rec, log);
    label++;
  }
}

void Engine::left_to_right(int bg_id, int end_id, double trun_err, std::vector<StepRec>* log) {
  if (solve_cap_reached()) return;   // a capped run stores no models past its last step
  const int N = L.num_site;
  int label = bg_id;
  DModel sys = models_.get(0, label), env = models_.get(1, N - label - 2);
  L.setup(sys.ham.len, env.ham.len);
  Basis sys_bs = get_basis(sys.ham), env_bs = get_basis(env.ham);
  WLayout wl = get_super(sys_bs, env_bs, tot_num_up, tot_num_down);
  DevBufP psi;
  DBlock sys_trun, env_trun;
  bool first = true;
  while (!solve_cap_reached()) {
    auto t0 = std::chrono::steady_clock::now();
    double wave_s = 0.0;
    if (!first) {
      if (!(label + 1 <= end_id)) break;
      sys_bs = get_basis(sys.ham);
      env_bs = env_bsm.at(N - label - 1);
      Basis env_basis = env_bsm.at(N - label);
      env = models_.get(1, N - label - 2);
      L.setup(sys.ham.len, env.ham.len);
      WLayout nl = get_super(sys_bs, env_bs, tot_num_up, tot_num_down);
      env_trun = env_truns.at(N - label - 1);
      DevBufP np = std::make_shared<DevBuf>((size_t)std::max<long long>(nl.dim, 1), st, false);
      auto tw = phase_clock(st);
      wave_trans(0, sys_bs, env_basis, sys_trun, env_trun, wl, psi->p, nl, np->p);
      wave_s = secs(tw, phase_clock(st));
      wl = nl;
      psi = np;
    } else {
      psi = std::make_shared<DevBuf>((size_t)std::max<long long>(wl.dim, 1), st, false);
      if (restart1 == 0) {
        wave_initialize(wl, psi->p);
      } else if (disk_layout.sys_len != wl.sys_len) {
        wave_trans(0, sys_bs, env_bsm.at(N - label), sys_truns.at(label), env_truns.at(N - label - 1), disk_layout,
                   disk_wave->p, wl, psi->p);
      } else {
        cuda_check(cudaMemcpyAsync(psi->p, disk_wave->p, wl.dim * sizeof(double2), cudaMemcpyDeviceToDevice, st), "copy");
      }
    }
    StepRec rec{};
    rec.wave_seconds = wave_s;
    lanczos_step(1, sys, env, sys_bs, env_bs, wl, psi, rec);
    disk_layout = wl;
    disk_wave = psi;
    TruncResult tr;
    auto tp = phase_clock(st);
    truncate(0, psi->p, wl, kept_min_, kept_max_, trun_err, tr);
    sys_trun = tr.trun;
    rec.num_state = tr.num_state;
    rec.err = tr.err;
    rec.ent = tr.ent;
    rec.ent_mult = tr.ent_mult;
    auto tq = phase_clock(st);
    rec.truncate_seconds = secs(tp, tq);
    grow(0, sys, sys_bs, sys_trun, 0);
    rec.grow_seconds = secs(tq, phase_clock(st));
    models_.put(0, label + 1, sys);
    sys_truns[label + 1] = sys_trun;
    sys_bsm[label + 1] = sys_bs;
    rec.step_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    record_step(rec, log);
    label++;
    first = false;
  }
}

void Engine::right_to_left(int bg_id, int end_id, double trun_err, std::vector<StepRec>* log) {
  if (solve_cap_reached()) return;
  const int N = L.num_site;
  int label = bg_id;
  DModel sys = models_.get(0, label - 1), env = models_.get(1, N - label - 1);
  L.setup(sys.ham.len, env.ham.len);
  Basis sys_bs = get_basis(sys.ham), env_bs = get_basis(env.ham);
  WLayout wl = get_super(sys_bs, env_bs, tot_num_up, tot_num_down);
  DevBufP psi;
  DBlock sys_trun, env_trun;
  bool first = true;
  while (!solve_cap_reached()) {
    auto t0 = std::chrono::steady_clock::now();
    double wave_s = 0.0;
    if (!first) {
      if (!(label - 1 >= end_id)) break;
      sys_bs = sys_bsm.at(label);
      Basis sys_basis = sys_bsm.at(label + 1);
      env_bs = get_basis(env.ham);
      WLayout nl = get_super(sys_bs, env_bs, tot_num_up, tot_num_down);
      sys = models_.get(0, label - 1);
      L.setup(sys.ham.len, env.ham.len);
      sys_trun = sys_truns.at(label);
      DevBufP np = std::make_shared<DevBuf>((size_t)std::max<long long>(nl.dim, 1), st, false);
      auto tw = phase_clock(st);
      wave_trans(1, sys_basis, env_bs, sys_trun, env_trun, wl, psi->p, nl, np->p);
      wave_s = secs(tw, phase_clock(st));
      wl = nl;
      psi = np;
    } else {
      psi = std::make_shared<DevBuf>((size_t)std::max<long long>(wl.dim, 1), st, false);
      if (restart1 == 0) {
        wave_initialize(wl, psi->p);
      } else if (disk_layout.sys_len != wl.sys_len) {
        wave_trans(1, sys_bsm.at(label + 1), env_bs, sys_truns.at(label), env_truns.at(N - label - 1), disk_layout,
                   disk_wave->p, wl, psi->p);
      } else {
        cuda_check(cudaMemcpyAsync(psi->p, disk_wave->p, wl.dim * sizeof(double2), cudaMemcpyDeviceToDevice, st), "copy");
      }
    }
    StepRec rec{};
    rec.wave_seconds = wave_s;
    lanczos_step(2, sys, env, sys_bs, env_bs, wl, psi, rec);
    disk_layout = wl;
    disk_wave = psi;
    TruncResult tr;
    auto tp = phase_clock(st);
    truncate(1, psi->p, wl, kept_min_, kept_max_, trun_err, tr);
    env_trun = tr.trun;
    rec.num_state = tr.num_state;
    rec.err = tr.err;
    rec.ent = tr.ent;
    rec.ent_mult = tr.ent_mult;
    auto tq = phase_clock(st);
    rec.truncate_seconds = secs(tp, tq);
    grow(1, env, env_bs, env_trun, sys.len + 1);
    rec.grow_seconds = secs(tq, phase_clock(st));
    models_.put(1, N - label, env);
    env_truns[N - label] = env_trun;
    env_bsm[N - label] = env_bs;
    rec.step_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    record_step(rec, log);
    label--;
    first = false;
  }
}

void Engine::run(int kept_min, int kept_warm, const std::vector<int>& sweeps, double lanzero_override,
                 unsigned long long seed, std::vector<StepRec>* log, bool warmup_only, bool final_half, bool resume,
                 int max_solves) {
  max_solves_ = max_solves;
  const int N = L.num_site;
  rng = seed;
  nsolve_ = 0;
  models_.bind(st);
  const double lanerr = (double)1.0e-6f, trun_err = 1.0000000036274937e-15;
  auto lz = [&](double v) { return lanzero_override > 0 ? lanzero_override : v; };
  kept_min_ = kept_min;
  kept_max_ = kept_warm;
  double tmp_err = trun_err * 15;
  if (resume) {
    // the stores hold the checkpoint's models, truncations, bases and wave
    if (!resume_ready_) throw Error(-4, "resume: no checkpoint has been read");
    restart1 = 1;
  } else {
    models_.clear();
    sys_truns.clear();
    env_truns.clear();
    sys_bsm.clear();
    env_bsm.clear();
    restart1 = 0;
    lanzero_ = lanzero_warmup_ > 0 ? lanzero_warmup_ : lz(lanerr * 1000);
    warm_up(N / 2, trun_err * 100, log);
    if (warmup_only) return;
    lanzero_ = lz(lanerr * 15);
    left_to_right(N / 2 - 1, N - 2, tmp_err, log);
    restart1 = 1;
    right_to_left(N - 2, 1, tmp_err, log);
  }
  resume_ready_ = false;
  for (size_t it = 1; it <= sweeps.size(); ++it) {
    kept_max_ = sweeps[it - 1];
    if (kept_min_ > kept_max_) kept_min_ = kept_max_;
    lanzero_ = lz(it >= 5 ? lanerr * 0.5 : lanerr);
    left_to_right(1, N - 2, trun_err, log);
    right_to_left(N - 2, 1, trun_err, log);
  }
  // main.f90:205-206: a last half sweep stops at 5 Num_site / 6, where Measurement reads the wave
  if (final_half)
    left_to_right(1, final_stop_ > 0 ? final_stop_ : 5 * N / 6 - 1, sweeps.empty() ? tmp_err : trun_err, log);
}

}  // namespace tsc
