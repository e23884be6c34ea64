// Host set-up of the engine: device memory, lattice tables, SU(2) 6j symbols,
// site operators, bases and task-list packing.
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "tsc_engine.hpp"

namespace tsc {

std::shared_mutex& capture_mutex() {
  static std::shared_mutex m;
  return m;
}

void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw Error(e == cudaErrorMemoryAllocation ? -5 : -3,
                                    std::string(what) + ": " + cudaGetErrorString(e));
}

// One stream-ordered pool per device that keeps freed memory for reuse (the
// default pool hands it back to the driver at every synchronisation, so each
// DMRG step would map its Krylov space and task buffers afresh).  Engines trim
// it when they are destroyed.
static std::mutex g_pool_mu;
static cudaMemPool_t g_pools[256] = {};

cudaMemPool_t device_pool() {
  int dev = 0;
  cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= 256) throw Error(-1, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_pool_mu);
  if (!g_pools[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    cuda_check(cudaMemPoolCreate(&pool, &props), "cudaMemPoolCreate");
    uint64_t keep = UINT64_MAX;
    cuda_check(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "cudaMemPoolSetAttribute");
    g_pools[dev] = pool;
  }
  return g_pools[dev];
}

namespace {
// Per-stream arena: chunks from the device pool, carved best fit, freed blocks
// coalesced with their neighbours inside a chunk.  All blocks of one arena are
// used in the order of its stream, so a block freed by the host can be handed
// out again at once.
struct Arena {
  struct Chunk {
    char* base;
    size_t bytes;
  };
  std::vector<Chunk> chunks;
  std::map<char*, size_t> free_at;             // block start -> bytes
  std::multimap<size_t, char*> free_size;      // bytes -> block start
  std::map<char*, char*> chunk_end;            // chunk base -> one past its end
  size_t reserved = 0;

  void insert_free(char* p, size_t n) {
    free_at[p] = n;
    free_size.emplace(n, p);
  }
  void erase_free(std::map<char*, size_t>::iterator it) {
    auto r = free_size.equal_range(it->second);
    for (auto q = r.first; q != r.second; ++q)
      if (q->second == it->first) {
        free_size.erase(q);
        break;
      }
    free_at.erase(it);
  }
  char* chunk_limit(char* p) const {   // end of the chunk holding p
    auto it = chunk_end.upper_bound(p);
    --it;
    return it->second;
  }
  char* take(size_t n) {
    auto it = free_size.lower_bound(n);
    if (it == free_size.end()) return nullptr;
    char* p = it->second;
    size_t have = it->first;
    free_size.erase(it);
    free_at.erase(p);
    if (have > n) insert_free(p + n, have - n);
    return p;
  }
  void give(char* p, size_t n) {
    char* lim = chunk_limit(p);
    auto nx = free_at.find(p + n);   // merge with the following free block
    if (nx != free_at.end() && p + n < lim) {
      n += nx->second;
      erase_free(nx);
    }
    auto pv = free_at.lower_bound(p);   // and with the preceding one
    if (pv != free_at.begin()) {
      --pv;
      if (pv->first + pv->second == p && chunk_limit(pv->first) == lim) {
        p = pv->first;
        n += pv->second;
        erase_free(pv);
      }
    }
    insert_free(p, n);
  }
};
std::mutex g_arena_mu;
std::unordered_map<cudaStream_t, Arena> g_arena;

constexpr size_t kAlign = 256;
constexpr size_t kMinChunk = 64ull << 20;
constexpr size_t kMaxChunk = 4ull << 30;
constexpr size_t kDirect = 4ull << 30;   // blocks at least this large bypass the arenas
}  // namespace

void release_stream_cache(cudaStream_t s) {
  std::lock_guard<std::mutex> lock(g_arena_mu);
  auto it = g_arena.find(s);
  if (it == g_arena.end()) return;
  for (auto& c : it->second.chunks) cudaFreeAsync(c.base, s);
  g_arena.erase(it);
}

DevBuf::DevBuf(size_t count, cudaStream_t s, bool zero) : n(count), st(s) {
  if (count == 0) return;
  cls = (count * sizeof(double2) + kAlign - 1) / kAlign * kAlign;
  if (cls >= kDirect) {   // large blocks come straight from the pool, which reuses them across sizes
    cuda_check(cudaMallocFromPoolAsync((void**)&p, cls, device_pool(), s), "cudaMallocFromPoolAsync");
    direct = true;
  } else {
    std::lock_guard<std::mutex> lock(g_arena_mu);
    Arena& A = g_arena[s];
    char* q = A.take(cls);
    if (!q) {   // new chunk: geometric growth between 64 MiB and 4 GiB, at least the request
      size_t want = std::max(cls, std::min(kMaxChunk, std::max(kMinChunk, A.reserved / 2)));
      void* base = nullptr;
      cudaError_t e = cudaMallocFromPoolAsync(&base, want, device_pool(), s);
      if (e == cudaErrorMemoryAllocation && want > cls) {   // fall back to the exact request
        cudaGetLastError();
        want = cls;
        e = cudaMallocFromPoolAsync(&base, want, device_pool(), s);
      }
      cuda_check(e, "cudaMallocFromPoolAsync");
      A.chunks.push_back({static_cast<char*>(base), want});
      A.chunk_end[static_cast<char*>(base)] = static_cast<char*>(base) + want;
      A.reserved += want;
      A.insert_free(static_cast<char*>(base), want);
      q = A.take(cls);
    }
    p = reinterpret_cast<double2*>(q);
  }
  if (zero) cuda_check(cudaMemsetAsync(p, 0, count * sizeof(double2), s), "cudaMemsetAsync");
}
DevBuf::~DevBuf() {
  if (!p) return;
  if (direct) {
    cudaFreeAsync(p, st);
    return;
  }
  std::lock_guard<std::mutex> lock(g_arena_mu);
  auto it = g_arena.find(st);
  if (it != g_arena.end()) it->second.give(reinterpret_cast<char*>(p), cls);
}

// ---- SU(2) coefficients --------------------------------------------------------
// Racah's closed form for the 6j symbol with doubled arguments (the reference's
// W6JS, block.f90:3744-3795, evaluates the same sum with a table of factorials).
// factorials as FACTRL builds them (block.f90:3688-3696); initialised once,
// thread-safely, by the first caller of any engine
static const double* factorials() {
  static const std::array<double, 171> f = [] {
    std::array<double, 171> a{};
    a[0] = 1.0;
    for (int i = 1; i <= 170; ++i) a[i] = a[i - 1] * (double)(float)i;
    return a;
  }();
  return f.data();
}

double w6j(int j1, int j2, int j3, int l1, int l2, int l3) {
  const double* g_fact = factorials();
  // triangle (j1 j2 j3), (j1 l2 l3), (l1 j2 l3), (l1 l2 j3) with integer sums
  auto tri = [](int a, int b, int c) { return c <= a + b && c >= std::abs(a - b) && ((a + b + c) & 1) == 0; };
  if (!tri(j1, j2, j3) || !tri(j1, l2, l3) || !tri(l1, j2, l3) || !tri(l1, l2, j3)) return 0.0;
  const int s1 = j1 + j2 + j3, s2 = j1 + l2 + l3, s3 = l1 + j2 + l3, s4 = l1 + l2 + j3;
  const int p1 = j1 + j2 + l1 + l2, p2 = j2 + j3 + l2 + l3, p3 = j3 + j1 + l3 + l1;
  const int wlo = std::max(std::max(s1, s2), std::max(s3, s4));
  const int whi = std::min(p1, std::min(p2, p3));
  double omega = 0.0;
  for (int w = wlo; w <= whi; w += 2) {
    double den = g_fact[(w - s1) / 2] * g_fact[(w - s2) / 2] * g_fact[(w - s3) / 2] * g_fact[(w - s4) / 2] *
                 g_fact[(p1 - w) / 2] * g_fact[(p2 - w) / 2] * g_fact[(p3 - w) / 2];
    if (w % 4 != 0) den = -den;
    omega = omega + g_fact[w / 2 + 1] / den;
  }
  auto delta = [g_fact](int a, int b, int c) {
    return g_fact[(a + b - c) / 2] * g_fact[(a - b + c) / 2] * g_fact[(-a + b + c) / 2] / g_fact[(a + b + c) / 2 + 1];
  };
  double th = delta(j1, j2, j3) * delta(j1, l2, l3) * delta(l1, j2, l3) * delta(l1, l2, j3);
  return omega * std::sqrt(th);
}

// Wigner 3j symbol with doubled arguments by Racah's single-sum formula
// (the reference's W3JS, block.f90:3702-3741, evaluates the same sum):
// (-1)^(j1-j2-m3) sqrt(D(j1 j2 j3) prod (j+-m)!) sum_k (-1)^k / [k! (j3-j2+m1+k)!
// (j3-j1-m2+k)! (j1+j2-j3-k)! (j1-m1-k)! (j2+m2-k)!]
double w3j(int j1, int j2, int j3, int m1, int m2, int m3) {
  const double* f = factorials();
  if (m1 + m2 + m3 != 0) return 0.0;
  if (j3 > j1 + j2 || j3 < std::abs(j1 - j2)) return 0.0;
  if (((j1 + j2 + j3) & 1) || ((j1 - m1) & 1) || ((j2 - m2) & 1)) return 0.0;
  if (std::abs(m1) > j1 || std::abs(m2) > j2 || std::abs(m3) > j3) return 0.0;
  // k in doubled units
  const int klo = std::max(0, std::max(j2 - j3 - m1, j1 - j3 + m2));
  const int khi = std::min(j1 + j2 - j3, std::min(j1 - m1, j2 + m2));
  double sum = 0.0;
  for (int k = klo; k <= khi; k += 2) {
    double den = f[k / 2] * f[(j3 - j2 + m1 + k) / 2] * f[(j3 - j1 - m2 + k) / 2] * f[(j1 + j2 - j3 - k) / 2] *
                 f[(j1 - m1 - k) / 2] * f[(j2 + m2 - k) / 2];
    sum += (k % 4 == 0) ? 1.0 / den : -1.0 / den;
  }
  const double tri = f[(j1 + j2 - j3) / 2] * f[(j1 - j2 + j3) / 2] * f[(-j1 + j2 + j3) / 2] / f[(j1 + j2 + j3) / 2 + 1];
  const double mf = f[(j1 + m1) / 2] * f[(j1 - m1) / 2] * f[(j2 + m2) / 2] * f[(j2 - m2) / 2] * f[(j3 + m3) / 2] *
                    f[(j3 - m3) / 2];
  const double v = sum * std::sqrt(tri * mf);
  return (((j1 - j2 - m3) / 2) % 2 != 0) ? -v : v;
}

// ---- lattice (dmrg_sub.f90:304-644) -------------------------------------------------
void Lattice::init(int nx, int ny, double t1, double t2, double J1, double J2, int oy) {
  Nx = nx;
  Ny = ny;
  nleg = ny;
  num_site = nx * ny;
  openy = oy;
  int N = num_site;
  neib.assign((size_t)(N + 1) * (neibt + 1), 0);
  neiba.assign((size_t)(N + 1) * (N + 1), 0);
  nposi.assign(N + 8, 0);
  nposi_dm.assign(N + 8, 0);
  nposi_lat.assign(N + 8, 0);
  inb1.assign((size_t)(N + 1) * (N + 1), 0);
  nleg11.assign(N + 1, 0);
  inb.assign(N + 8, 0);
  size_t nc = (size_t)(N + 1) * (neibt + 1);
  jt.assign(nc, 0.0);
  jz.assign(nc, 0.0);
  jd.assign(nc, 0.0);
  jn.assign(nc, 0.0);
  for (int s = 1; s <= N; ++s) {
    for (int k = 1; k <= 12; ++k) {
      size_t e = (size_t)s * (neibt + 1) + k;
      jz[e] = k <= 6 ? J1 : J2;
      jt[e] = -(k <= 6 ? t1 : t2) * std::sqrt(2.0);
      jn[e] = -0.25 * jz[e];
    }
    for (int k = 1; k <= 18; ++k) {
      size_t e = (size_t)s * (neibt + 1) + k;
      jd[e] = jz[e] * (-std::sqrt(3.0));
    }
  }
}

void Lattice::setup(int ns, int ns21) {
  int nn = ns + ns21 + 2;
  nxc = (nn - 1) / nleg + 1;
  if (nxc == 1) nxc = 2;
  std::fill(nposi.begin(), nposi.end(), 0);
  std::fill(nposi_dm.begin(), nposi_dm.end(), 0);
  std::fill(nposi_lat.begin(), nposi_lat.end(), 0);
  std::fill(neib.begin(), neib.end(), 0);
  std::fill(neiba.begin(), neiba.end(), 0);
  int totsite = nleg * nxc;
  for (int i = 1; i <= ns + 1; ++i) {
    nposi[i] = 1;
    nposi_lat[i] = i;
    nposi_dm[i] = i;
  }
  nposi[ns + 1] = 2;
  for (int i = 1; i <= ns21 + 1; ++i) {
    nposi[ns + 1 + i] = 3;
    nposi_dm[totsite + 1 - i] = i + ns + 1;
    nposi_lat[i + ns + 1] = totsite + 1 - i;
  }
  nposi[ns + ns21 + 2] = 4;
  auto link = [&](int a, int ka, int b, int kb) {
    NEIB(a, ka) = b;
    NEIB(b, kb) = a;
    NEIBA(a, b) = ka;
    NEIBA(b, a) = kb;
  };
  for (int ix = 1; ix <= nxc; ++ix)
    for (int iy = 1; iy <= nleg; ++iy) {
      int ii = iy + (ix - 1) * nleg;
      int jy = ii - iy + (iy % nleg) + 1;
      if (openy != 0 && iy == nleg) jy = 0;
      if (jy != 0 && (iy != nleg || nleg != 2)) link(ii, 1, jy, 2);
      int jx = ii + nleg;
      if (jx > nleg * nxc) jx = 0;   // open in x
      if (jx != 0) {
        link(ii, 3, jx, 4);
        jy = jx - 1;
        if (iy == 1) jy = openy == 0 ? jy + nleg : 0;
        if (jy != 0) link(ii, 5, jy, 6);
      }
    }
  for (int ix = 1; ix <= nxc; ++ix)
    for (int iy = 1; iy <= nleg; ++iy) {
      int ii = iy + (ix - 1) * nleg;
      int a = NEIB(ii, 1), b = NEIB(a, 3);
      if (a * b != 0) link(ii, 7, b, 8);
      if (nleg != 3) {
        a = NEIB(ii, 3);
        b = NEIB(a, 5);
        if (a * b != 0) link(ii, 9, b, 10);
      }
      a = NEIB(ii, 2);
      b = NEIB(a, 5);
      if (a * b != 0) link(ii, 11, b, 12);
      if (nleg != 3) {
        a = NEIB(ii, 1);
        b = NEIB(a, 1);
        if (a * b != 0 && NEIBA(ii, b) == 0) link(ii, 13, b, 14);
      }
      a = NEIB(ii, 3);
      b = NEIB(a, 3);
      if (a * b != 0 && NEIBA(ii, b) == 0) link(ii, 15, b, 16);
      a = NEIB(ii, 5);
      b = NEIB(a, 5);
      if (a * b != 0 && NEIBA(ii, b) == 0) link(ii, 17, b, 18);
    }
  for (int i = 1; i <= num_site; ++i)
    for (int j = 7; j <= neibt; ++j)
      if (std::fabs(JZ(j, 1)) + std::fabs(JD(j, 1)) + std::fabs(JT(j, 1)) + std::fabs(JN(j, 1)) == 0.0) {
        int nb = NEIB(i, j);
        NEIBA(i, nb) = 0;
        NEIBA(nb, i) = 0;
        NEIB(i, j) = 0;
      }
}

void Lattice::setup0() {
  std::fill(nleg11.begin(), nleg11.end(), 0);
  for (int ns = 1; ns <= num_site - 2; ++ns) {
    int k0 = 0;
    for (int i1 = 1; i1 <= ns; ++i1) {
      int cnt = 0;
      for (int j = 1; j <= neibt; ++j)
        if (NEIB(i1, j) >= ns) cnt++;
      INB1(i1, ns) = cnt ? ++k0 : 10000;
    }
    nleg11[ns] = k0;
  }
}

// ---- engine -------------------------------------------------------------------------
Engine::Engine(int Nx, int Ny, double t1, double t2, double J1, double J2, int delta, int device) {
  std::unique_lock<std::shared_mutex> no_capture(capture_mutex());
  if (Nx < 2 || Ny < 2 || Nx * Ny > 1024) throw Error(-1, "lattice size out of range");
  if (delta < 1) throw Error(-1, "delta must be >= 1");
  int ndev = 0;
  cuda_check(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
  if (device < 0 || device >= ndev) throw Error(-1, "no such CUDA device");
  cuda_check(cudaSetDevice(device), "cudaSetDevice");
  device_ = device;
  cuda_check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
  cuda_check(cudaEventCreate(&ev0), "cudaEventCreate");
  cuda_check(cudaEventCreate(&ev1), "cudaEventCreate");
  models_.bind(st);
  L.init(Nx, Ny, t1, t2, J1, J2, 0);
  // site operators (dmrg_sub.f90:743-906)
  st_elec_up.up_dif = 1;
  st_elec_up.down_dif = 1;
  st_elec_up.sub = {{0, 0, 1, -std::sqrt(2.0)}};
  st_elec_down.up_dif = -1;
  st_elec_down.down_dif = 1;
  st_elec_down.sub = {{1, 1, -1, -std::sqrt(2.0)}};
  num_elec.sub = {{1, 1, 0, std::sqrt(2.0)}, {0, 0, 0, 0.0}};
  st_sd.down_dif = 2;
  st_sd.sub = {{1, 1, 0, std::sqrt(1.5)}};
  st_sz.sub = {{1, 1, 0, 1.0}, {0, 0, 0, 0.0}};
  int N = L.num_site;
  tot_num_up = 2 * (N / 2 - (N + 2 * delta - 1) / (2 * delta));
  tot_num_down = 0;
  L.setup(N / 2 - 1, N / 2 - 1);
  L.setup0();
  red_buf = std::make_shared<DevBuf>((size_t)(1 << 16) + 1024, st, true);
  d_red = reinterpret_cast<double*>(red_buf->p);
  d_scal = d_red + (1 << 16);
  d_fault = reinterpret_cast<int*>(d_scal + S_FAULT);   // zero: red_buf is zero-filled
  cuda_check(cudaMallocHost((void**)&h_scal, 2048 * sizeof(double)), "cudaMallocHost");
}

void Engine::check_split_fault() {
  cuda_check(cudaMemcpyAsync(h_scal + S_FAULT, d_fault, sizeof(int), cudaMemcpyDeviceToHost, st), "d2h");
  cuda_check(cudaStreamSynchronize(st), "sync");
  int f = 0;
  std::memcpy(&f, h_scal + S_FAULT, sizeof(int));
  if (!f) return;
  cuda_check(cudaMemsetAsync(d_fault, 0, sizeof(int), st), "memset");
  cuda_check(cudaStreamSynchronize(st), "sync");
  throw Error(-3, "split-precision kernel: a bounded wait ran out (output incomplete)");
}

Engine::~Engine() {
  std::unique_lock<std::shared_mutex> no_capture(capture_mutex());
  sb = Superblock();
  bs = BlockSparse();
  models_.clear();
  sys_truns.clear();
  env_truns.clear();
  disk_wave.reset();
  red_buf.reset();
  eig.reset();
  release_stream_cache(st);
  if (st) cudaStreamSynchronize(st);
  try {
    cudaMemPoolTrimTo(device_pool(), 0);
  } catch (...) {
  }
  if (h_scal) cudaFreeHost(h_scal);
  if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
  for (cudaEvent_t e : graph_ev_)
    if (e) cudaEventDestroy(e);
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  for (cudaEvent_t e : hpsi_events) cudaEventDestroy(e);
  for (cudaEvent_t e : tune_ev_)
    if (e) cudaEventDestroy(e);
  if (st) cudaStreamDestroy(st);
}

DModel Engine::site_model() const {   // Get_hamiltonian_site, dmrg_sub.f90:912-938
  DModel m;
  m.len = 1;
  auto mk = [&](const SiteOp& so, int nsub_override_zero) {
    DBlock b;
    b.len = 1;
    b.num = (int)so.sub.size();
    b.dim = b.num;
    b.up_dif = so.up_dif;
    b.down_dif = so.down_dif;
    b.buf = std::make_shared<DevBuf>((size_t)b.num, st, false);
    std::vector<double2> h(b.num);
    for (int i = 0; i < b.num; ++i) {
      SubDesc s;
      s.num_up = so.sub[i].num_up;
      s.num_down = so.sub[i].num_down;
      s.down_dif = so.sub[i].down_dif;
      s.row_dim = s.sdim = 1;
      s.off = i;
      b.sub.push_back(s);
      h[i] = make_double2(nsub_override_zero ? 0.0 : so.sub[i].val, 0.0);
    }
    cuda_check(cudaMemcpyAsync(b.buf->p, h.data(), b.num * sizeof(double2), cudaMemcpyHostToDevice, st), "upload");
    cuda_check(cudaStreamSynchronize(st), "sync");
    return b;
  };
  m.ham = mk(st_sz, 1);
  m.sub.resize(L.num_site + 1);
  m.sub[1].op[OP_UP] = mk(st_elec_up, 0);
  m.sub[1].op[OP_DOWN] = mk(st_elec_down, 0);
  m.sub[1].op[OP_SD] = mk(st_sd, 0);
  m.sub[1].op[OP_SN] = mk(num_elec, 0);
  return m;
}

// Get_basis, block.f90:2087-2188 (site = st_sz: (1,1) then (0,0), sdim 1)
Basis Engine::get_basis(const DBlock& block) const {
  Basis b;
  b.len = block.len + 1;
  std::vector<std::pair<int, int>> q;   // (N, 2S)
  for (const auto& s : block.sub)
    for (const auto& t : st_sz.sub)
      for (int ss = std::abs(s.num_down - t.num_down); ss <= s.num_down + t.num_down; ss += 2)
        q.push_back({s.num_up + t.num_up, ss});
  // descending 2S, then descending N (QuickSort_Integer, block.f90:2316-2349), unique
  std::sort(q.begin(), q.end(), [](const std::pair<int, int>& a, const std::pair<int, int>& c) {
    if (a.second != c.second) return a.second > c.second;
    return a.first > c.first;
  });
  q.erase(std::unique(q.begin(), q.end()), q.end());
  b.num = (int)q.size();
  b.sec.resize(b.num);
  for (int i = 0; i < b.num; ++i) {
    Sector& S = b.sec[i];
    S.num_up = q[i].first;
    S.num_down = q[i].second;
    for (const auto& s : block.sub)
      for (const auto& t : st_sz.sub) {
        if (s.num_up + t.num_up != S.num_up) continue;
        if (S.num_down < std::abs(s.num_down - t.num_down) || S.num_down > s.num_down + t.num_down) continue;
        Piece p;
        p.bl_num_up = s.num_up;
        p.bl_num_down = s.num_down;
        p.st_num_up = t.num_up;
        p.st_num_down = t.num_down;
        p.sdim = s.sdim;
        p.spos = S.dim;
        S.dim += p.sdim;
        S.pcs.push_back(p);
      }
    b.dim += S.dim;
  }
  return b;
}

// Get_super_basis, block.f90:2194-2247
WLayout Engine::get_super(const Basis& sys_bs, const Basis& env_bs, int tot_up, int tot_down) const {
  WLayout w;
  w.sys_len = sys_bs.len;
  w.env_len = env_bs.len;
  for (const auto& s : sys_bs.sec)
    for (const auto& e : env_bs.sec) {
      if (e.num_up != tot_up - s.num_up) continue;
      if (tot_down < std::abs(e.num_down - s.num_down) || tot_down > e.num_down + s.num_down) continue;
      WSec x;
      x.sys_num_up = s.num_up;
      x.sys_num_down = s.num_down;
      x.env_num_up = e.num_up;
      x.env_num_down = e.num_down;
      x.sys_dim = s.dim;
      x.env_dim = e.dim;
      x.off = w.dim;
      w.dim += (long long)s.dim * e.dim;
      w.sec.push_back(x);
    }
  w.num = (int)w.sec.size();
  return w;
}

// ---- task lists ------------------------------------------------------------------------
int TaskList::add_group(double2* abs_c, uint8_t base, long long c_off, int ld, int M, int N, int beta) {
  GGroup g{};
  g.c_base = base;
  g.c_off = base == BASE_ABS ? (long long)((uintptr_t)abs_c / sizeof(double2)) + c_off : c_off;
  g.c_ld = ld;
  g.M = M;
  g.N = N;
  g.beta = (uint8_t)beta;
  groups.push_back(g);
  gterms.emplace_back();
  return (int)groups.size() - 1;
}

// CTA tile of the grouped GEMM when no schedule is chosen: 32x32 (6 CTAs/SM);
// the autotuner (Engine::tune_*) picks among 32x32, 64x32 and 32x64 per size class.
int default_tile() { return TILE_32x32; }

// ---- split-precision form: pre-sliced operand views ----------------------------------
namespace {
struct ViewKey {
  uint8_t base, op, role;
  long long off;
  int ld, rows, cols;
  double ar, ai;
  bool operator<(const ViewKey& o) const {
    return std::tie(base, op, role, off, ld, rows, cols, ar, ai) <
           std::tie(o.base, o.op, o.role, o.off, o.ld, o.rows, o.cols, o.ar, o.ai);
  }
};
int view_tiles_along(const SView& v) {   // row tiles (A) or column tiles (B)
  return v.role == 0 ? (v.rows + SPLIT_TILE_M - 1) / SPLIT_TILE_M : (v.cols + SPLIT_TILE_N - 1) / SPLIT_TILE_N;
}
long long view_units(const SView& v) { return (long long)view_tiles_along(v) * v.nks * (v.role == 0 ? 2 : 1); }
}  // namespace

void build_split_views(TaskList& p1, TaskList& p2, SplitData& sd, cudaStream_t st, bool term_alpha) {
  sd = SplitData();
  std::vector<SView> views[3];
  std::map<ViewKey, int> index[3];
  // phase-1 groups by their scratch offset: the intermediates phase 2 reads
  std::map<long long, int> scr_group;
  for (size_t g = 0; g < p1.groups.size(); ++g)
    if (p1.groups[g].c_base == BASE_SCR) scr_group[p1.groups[g].c_off] = (int)g;
  std::map<int, int> tview_of_group;
  auto add_view = [&](int arena, const ViewKey& k) -> int {
    auto it = index[arena].find(k);
    if (it != index[arena].end()) return it->second;
    SView v{};
    v.src = k.off;
    v.ar = k.ar;
    v.ai = k.ai;
    v.ld = k.ld;
    v.rows = k.rows;
    v.cols = k.cols;
    v.role = k.role;
    v.op = k.op;
    v.from_in = arena == ARENA_IN;
    v.nks = ((k.role == 0 ? k.cols : k.rows) + 15) / 16;
    v.dst = sd.units[arena];
    sd.units[arena] += view_units(v);
    views[arena].push_back(v);
    return index[arena][k] = (int)views[arena].size() - 1;
  };
  // the view of one operand of a term; returns (arena, view)
  auto operand = [&](uint8_t base, long long off, int ld, uint8_t op, int role, int rows, int cols, double ar,
                     double ai) -> std::pair<int, int> {
    if (base == BASE_ABS) return {ARENA_FIXED, add_view(ARENA_FIXED, ViewKey{base, op, (uint8_t)role, off, ld, rows, cols, ar, ai})};
    if (ar != 1.0 || ai != 0.0) throw Error(-1, "split views: coefficient on a live operand");
    if (base == BASE_IN) return {ARENA_IN, add_view(ARENA_IN, ViewKey{base, op, (uint8_t)role, off, ld, rows, cols, 1.0, 0.0})};
    if (base == BASE_SCR) {
      auto it = scr_group.find(off);
      if (it == scr_group.end() || role != 0 || op != OP_N) throw Error(-1, "split views: unexpected scratch operand");
      GGroup& g = p1.groups[it->second];
      if (g.M != rows || g.c_ld != ld || g.N != cols || p1.gterms[it->second].size() != 1)
        throw Error(-1, "split views: scratch operand is not a whole phase-1 output");
      auto tv = tview_of_group.find(it->second);
      if (tv != tview_of_group.end()) return {ARENA_T, tv->second};
      const int v = add_view(ARENA_T, ViewKey{base, op, 0, off, ld, rows, cols, 1.0, 0.0});
      g.s_off = views[ARENA_T][v].dst;
      tview_of_group[it->second] = v;
      return {ARENA_T, v};
    }
    throw Error(-1, "split views: operand base");
  };
  for (TaskList* tl : {&p1, &p2})
    for (size_t gi = 0; gi < tl->groups.size(); ++gi) {
      const GGroup& g = tl->groups[gi];
      for (GTerm& t : tl->gterms[gi]) {
        if (t.kind != TK_GEMM || t.K <= 0) continue;
        // the coefficient rides on the operator operand (on A when both are
        // operators), or stays with the term (term_alpha)
        const bool fold_a = t.l_base == BASE_ABS;
        const double cr = term_alpha ? 1.0 : t.ar, ci = term_alpha ? 0.0 : t.ai;
        const double aar = fold_a ? cr : 1.0, aai = fold_a ? ci : 0.0;
        const double bar = fold_a ? 1.0 : cr, bai = fold_a ? 0.0 : ci;
        auto A = operand(t.l_base, t.l_off, t.l_ld, t.l_op, 0, g.M, t.K, aar, aai);
        auto B = operand(t.r_base, t.r_off, t.r_ld, t.r_op, 1, t.K, g.N, bar, bai);
        const SView& va = views[A.first][A.second];
        const SView& vb = views[B.first][B.second];
        t.l_base = (uint8_t)A.first;
        t.l_off = va.dst;
        t.l_ld = va.nks;
        t.r_base = (uint8_t)B.first;
        t.r_off = vb.dst;
        t.r_ld = vb.nks;
        t.l_op = t.r_op = OP_N;
        if (!term_alpha) {
          t.ar = 1.0;
          t.ai = 0.0;
        }
        t.pad0 = 1;   // references pre-sliced views
      }
    }
  // arenas; intermediates' tiles start zeroed (their padding is never written)
  DevBufP* arena[3] = {&sd.fixed, &sd.in, &sd.t};
  for (int a = 0; a < 3; ++a) {
    const long long bytes = std::max<long long>(sd.units[a], 1) * SPLIT_UNIT;
    *arena[a] = std::make_shared<DevBuf>((size_t)(bytes / sizeof(double2)), st, a == ARENA_T);
    sd.arenas.a[a] = reinterpret_cast<unsigned char*>((*arena[a])->p);
    sd.arenas.units[a] = std::max<long long>(sd.units[a], 1);
    sd.nviews[a] = (int)views[a].size();
  }
  auto tiles_of = [&](const std::vector<SView>& vs) {
    std::vector<STile> tl;
    for (size_t v = 0; v < vs.size(); ++v)
      for (int t = 0; t < view_tiles_along(vs[v]); ++t)
        for (int ks = 0; ks < vs[v].nks; ++ks) tl.push_back(STile{(int)v, t, ks, 0});
    return tl;
  };
  auto pack = [&](const std::vector<SView>& vs, const std::vector<STile>& tl, DevBufP& buf, const SView*& dv,
                  const STile*& dt) {
    const size_t bv = (vs.size() * sizeof(SView) + 255) / 256 * 256, bt = tl.size() * sizeof(STile);
    buf = std::make_shared<DevBuf>((bv + bt + 15) / 16 + 1, st, false);
    std::vector<char> host(bv + bt, 0);
    if (!vs.empty()) std::memcpy(host.data(), vs.data(), vs.size() * sizeof(SView));
    if (bt) std::memcpy(host.data() + bv, tl.data(), bt);
    cuda_check(cudaMemcpyAsync(buf->p, host.data(), host.size(), cudaMemcpyHostToDevice, st), "split views upload");
    dv = reinterpret_cast<const SView*>(buf->p);
    dt = reinterpret_cast<const STile*>(reinterpret_cast<char*>(buf->p) + bv);
    cuda_check(cudaStreamSynchronize(st), "split views sync");   // the host staging buffer goes out of scope
  };
  {  // operator views: sliced once, here
    std::vector<STile> tl = tiles_of(views[ARENA_FIXED]);
    DevBufP tmp;
    const SView* dv = nullptr;
    const STile* dt = nullptr;
    pack(views[ARENA_FIXED], tl, tmp, dv, dt);
    cuda_check(launch_slice_tiles(dv, dt, (int)tl.size(), nullptr, sd.arenas.a[ARENA_FIXED],
                                  sd.arenas.units[ARENA_FIXED], st),
               "slice operators");
    cuda_check(cudaStreamSynchronize(st), "slice operators sync");
  }
  std::vector<STile> tin = tiles_of(views[ARENA_IN]);
  pack(views[ARENA_IN], tin, sd.in_lists, sd.d_in_views, sd.d_in_tiles);
  sd.n_in_tiles = (int)tin.size();
  p1.arenas = p2.arenas = sd.arenas;
  p1.term_alpha = p2.term_alpha = term_alpha;
}

void slice_input(const SplitData& sd, const double2* d_in, cudaStream_t st) {
  cuda_check(launch_slice_tiles(sd.d_in_views, sd.d_in_tiles, sd.n_in_tiles, d_in, sd.arenas.a[ARENA_IN],
                                sd.arenas.units[ARENA_IN], st),
             "slice input");
}

void TaskList::upload_split(cudaStream_t st) {
  split = true;
  upload(st, 148 * 2, 4);
}

void TaskList::upload(cudaStream_t st, int slots, int waves, int tile_override) {
  tile = tile_override ? tile_override : default_tile();
  int TMt, TNt;
  tile_dims(tile, TMt, TNt);
  if (split) {
    TMt = SPLIT_TILE_M;
    TNt = SPLIT_TILE_N;
  } else {
    slots = slots / 2 * (tile == TILE_32x32 ? 6 : tile == TILE_64x64 ? 2 : 4);   // resident CTAs per SM x SMs
  }
  std::vector<GTerm> terms;
  struct JC {
    GJob j;
    long long cost;
  };
  std::vector<JC> jc;
  std::vector<GReduce> reds;
  exec_flops = 0;
  auto tcost = [](const GTerm& t) -> long long {
    return t.kind == TK_GEMM ? (long long)(t.K + GEMM_TK - 1) / GEMM_TK + 1 : 1;
  };
  // pass 1: flatten terms and total cost
  std::vector<long long> gcost(groups.size(), 0);
  long long total = 0;
  for (size_t gi = 0; gi < groups.size(); ++gi) {
    GGroup& g = groups[gi];
    g.t0 = (int)terms.size();
    long long c = 1;
    for (auto& t : gterms[gi]) {
      terms.push_back(t);
      c += tcost(t);
      if (t.kind == TK_GEMM) exec_flops += 8.0 * g.M * g.N * t.K;
    }
    g.t1 = (int)terms.size();
    gcost[gi] = c;
    if (g.M > 0 && g.N > 0)
      total += c * (long long)((g.M + TMt - 1) / TMt) * ((g.N + TNt - 1) / TNt);
  }
  const long long target = std::max<long long>(8, total / std::max(1, slots * waves));
  part_elems = 0;
  // pass 2: jobs, splitting long groups into term chunks of about `target`
  for (size_t gi = 0; gi < groups.size(); ++gi) {
    const GGroup& g = groups[gi];
    if (g.M <= 0 || g.N <= 0) continue;
    int tm = (g.M + TMt - 1) / TMt, tn = (g.N + TNt - 1) / TNt;
    int nchunk = (int)std::min<long long>((gcost[gi] + target - 1) / target, std::max(1, g.t1 - g.t0));
    if (gcost[gi] <= target + target / 2 || nchunk <= 1) {
      for (int a = 0; a < tm; ++a)
        for (int b = 0; b < tn; ++b) jc.push_back({GJob{(int)gi, a, b, g.t0, g.t1, -1, 0}, gcost[gi]});
      continue;
    }
    // contiguous chunks of roughly equal cost
    std::vector<int> cut{g.t0};
    long long acc = 0, per = (gcost[gi] + nchunk - 1) / nchunk;
    for (int t = g.t0; t < g.t1; ++t) {
      acc += tcost(terms[t]);
      if (acc >= per && t + 1 < g.t1 && (int)cut.size() < nchunk) {
        cut.push_back(t + 1);
        acc = 0;
      }
    }
    cut.push_back(g.t1);
    int P = (int)cut.size() - 1;
    long long base = part_elems;
    long long mn = (long long)g.M * g.N;
    part_elems += P * mn;
    for (int p = 0; p < P; ++p) {
      long long c = 1;
      for (int t = cut[p]; t < cut[p + 1]; ++t) c += tcost(terms[t]);
      for (int a = 0; a < tm; ++a)
        for (int b = 0; b < tn; ++b) jc.push_back({GJob{(int)gi, a, b, cut[p], cut[p + 1], p, base + p * mn}, c});
    }
    reds.push_back(GReduce{(int)gi, P, base});
    max_red_elems = std::max(max_red_elems, mn);
  }
  // longest jobs first: the hardware scheduler then approximates LPT balancing
  std::stable_sort(jc.begin(), jc.end(), [](const JC& a, const JC& b) { return a.cost > b.cost; });
  std::vector<GJob> jobs;
  jobs.reserve(jc.size());
  for (auto& x : jc) jobs.push_back(x.j);
  njobs = (int)jobs.size();
  nreds = (int)reds.size();
  nterms = (long long)terms.size();
  size_t bj = jobs.size() * sizeof(GJob), bg = groups.size() * sizeof(GGroup), bt = terms.size() * sizeof(GTerm),
         br = reds.size() * sizeof(GReduce);
  auto al = [](size_t x) { return (x + 255) / 256 * 256; };
  size_t total_b = al(bj) + al(bg) + al(bt) + al(br) + 256;
  dev = std::make_shared<DevBuf>((total_b + 15) / 16, st, false);
  char* base = reinterpret_cast<char*>(dev->p);
  d_jobs = reinterpret_cast<GJob*>(base);
  d_groups = reinterpret_cast<GGroup*>(base + al(bj));
  d_terms = reinterpret_cast<GTerm*>(base + al(bj) + al(bg));
  d_reds = reinterpret_cast<GReduce*>(base + al(bj) + al(bg) + al(bt));
  std::vector<char> host(total_b, 0);
  if (bj) std::memcpy(host.data(), jobs.data(), bj);
  if (bg) std::memcpy(host.data() + al(bj), groups.data(), bg);
  if (bt) std::memcpy(host.data() + al(bj) + al(bg), terms.data(), bt);
  if (br) std::memcpy(host.data() + al(bj) + al(bg) + al(bt), reds.data(), br);
  cuda_check(cudaMemcpyAsync(base, host.data(), total_b, cudaMemcpyHostToDevice, st), "task upload");
  part = part_elems ? std::make_shared<DevBuf>((size_t)part_elems, st, false) : nullptr;
  cuda_check(cudaStreamSynchronize(st), "task upload sync");
}

void Engine::run_tasks(TaskList& tl, double2* in, double2* out, double2* scr) {
  Bases b;
  b.p[0] = nullptr;
  b.p[1] = in;
  b.p[2] = out;
  b.p[3] = scr;
  b.part = tl.part ? tl.part->p : nullptr;
  if (tl.split)
    cuda_check(launch_grouped_zgemm_split(tl.d_jobs, tl.njobs, tl.d_groups, tl.d_terms, b, tl.arenas, d_fault,
                                          split_wait_limit_, tl.term_alpha ? 1 : 0, st),
               "grouped_zgemm_split");
  else
    cuda_check(launch_grouped_zgemm(tl.d_jobs, tl.njobs, tl.d_groups, tl.d_terms, b, st, tl.tile), "grouped_zgemm");
  if (tl.nreds)
    cuda_check(launch_reduce_partials(tl.d_reds, tl.nreds, tl.d_groups, b, tl.max_red_elems, st), "reduce_partials");
}

// ---- block transfer ----------------------------------------------------------------------
DBlock Engine::upload_block(const int*& ip, const cplx*& dp) {
  DBlock b;
  b.len = *ip++;
  b.num = *ip++;
  b.dim = *ip++;
  b.up_dif = *ip++;
  b.down_dif = *ip++;
  if (b.num < 0 || b.num > 1000000) throw Error(-1, "bad block descriptor");
  long long off = 0;
  for (int i = 0; i < b.num; ++i) {
    SubDesc s;
    s.num_up = *ip++;
    s.num_down = *ip++;
    s.down_dif = *ip++;
    s.row_dim = *ip++;
    s.sdim = *ip++;
    if (s.row_dim < 0 || s.sdim < 0) throw Error(-1, "bad sub-block dims");
    s.off = off;
    off += (long long)s.row_dim * s.sdim;
    b.sub.push_back(s);
  }
  b.buf = std::make_shared<DevBuf>((size_t)off, st, false);
  if (off) cuda_check(cudaMemcpyAsync(b.buf->p, dp, off * sizeof(double2), cudaMemcpyHostToDevice, st), "upload");
  dp += off;
  return b;
}

void Engine::download_block(const DBlock& b, std::vector<int>& ints, std::vector<cplx>& data) const {
  ints.insert(ints.end(), {b.len, b.num, b.dim, b.up_dif, b.down_dif});
  size_t d0 = data.size();
  for (const auto& s : b.sub) ints.insert(ints.end(), {s.num_up, s.num_down, s.down_dif, s.row_dim, s.sdim});
  long long tot = b.total();
  data.resize(d0 + tot);
  for (const auto& s : b.sub) {
    long long n = (long long)s.row_dim * s.sdim;
    if (n)
      cuda_check(cudaMemcpyAsync(&data[d0], b.buf->p + s.off, n * sizeof(double2), cudaMemcpyDeviceToHost, st),
                 "download");
    d0 += n;
  }
  cuda_check(cudaStreamSynchronize(st), "download sync");
}

// ---- stored models: device-resident under a byte limit, host memory beyond it ----
namespace {
template <class F>
void for_blocks(DModel& m, F&& f) {
  f(m.ham);
  for (auto& os : m.sub)
    for (auto& b : os.op) f(b);
}
long long model_bytes(DModel& m) {
  long long n = 0;
  for_blocks(m, [&](DBlock& b) {
    if (b.buf) n += (long long)b.buf->n * (long long)sizeof(double2);
  });
  return n;
}
}  // namespace

long long ModelStore::limit() const {
  if (limit_ >= 0) return limit_;
  size_t fr = 0, tot = 0;
  if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
    cudaGetLastError();
    return 1ll << 62;
  }
  return (long long)(default_frac_ * (double)tot);
}

void ModelStore::spill(Entry& e) {
  if (e.spilled) return;
  auto t0 = std::chrono::steady_clock::now();
  e.host.clear();
  for_blocks(e.m, [&](DBlock& b) {
    e.host.emplace_back();
    if (!b.buf) return;
    auto& h = e.host.back();
    h.resize(b.buf->n);
    if (b.buf->n)
      cuda_check(cudaMemcpyAsync(h.data(), b.buf->p, b.buf->n * sizeof(double2), cudaMemcpyDeviceToHost, st_),
                 "spill d2h");
  });
  cuda_check(cudaStreamSynchronize(st_), "spill sync");
  for_blocks(e.m, [&](DBlock& b) { b.buf.reset(); });
  e.spilled = true;
  resident_ -= e.bytes;
  host_bytes_ += e.bytes;
  spills++;
  moved_bytes += (double)e.bytes;
  moved_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void ModelStore::restore(Entry& e) {
  if (!e.spilled) return;
  if (e.on_disk) from_disk(e);
  auto t0 = std::chrono::steady_clock::now();
  size_t k = 0;
  for_blocks(e.m, [&](DBlock& b) {
    auto& h = e.host[k++];
    if (h.empty()) return;
    b.buf = std::make_shared<DevBuf>(h.size(), st_, false);
    cuda_check(cudaMemcpyAsync(b.buf->p, h.data(), h.size() * sizeof(double2), cudaMemcpyHostToDevice, st_),
               "restore h2d");
  });
  cuda_check(cudaStreamSynchronize(st_), "restore sync");
  e.host.clear();
  e.host.shrink_to_fit();
  e.spilled = false;
  resident_ += e.bytes;
  host_bytes_ -= e.bytes;
  restores++;
  moved_bytes += (double)e.bytes;
  moved_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// spills least recently used models (never `keep`) until the resident ones fit
void ModelStore::enforce(long long keep) {
  const long long lim = limit();
  while (resident_ > lim) {
    Entry* victim = nullptr;
    for (auto& kv : map_)
      if (kv.first != keep && !kv.second.spilled && kv.second.bytes > 0 &&
          (!victim || kv.second.tick < victim->tick))
        victim = &kv.second;
    if (!victim) break;
    spill(*victim);
  }
  enforce_host(keep);
}

void ModelStore::put(int side, int len, const DModel& m) {
  const long long k = key(side, len);
  auto it = map_.find(k);
  if (it != map_.end()) {
    Entry& o = it->second;
    if (!o.spilled) resident_ -= o.bytes;
    else if (!o.on_disk) host_bytes_ -= o.bytes;
    if (o.on_disk) std::remove(o.file.c_str());
  }
  Entry& e = map_[k];
  e.m = m;
  e.host.clear();
  e.spilled = false;
  e.on_disk = false;
  e.file.clear();
  e.bytes = model_bytes(e.m);
  e.tick = ++clock_;
  resident_ += e.bytes;
  enforce(k);
}

DModel ModelStore::get(int side, int len) {
  const long long k = key(side, len);
  auto it = map_.find(k);
  if (it == map_.end()) throw Error(-4, "stored model not found (side " + std::to_string(side) + ", length " +
                                            std::to_string(len) + ")");
  Entry& e = it->second;
  e.tick = ++clock_;
  if (e.spilled) {
    restore(e);
    enforce(k);
  }
  return e.m;
}

// host copies of the least recently used spilled models to files until the
// spilled models' host bytes fit under the host limit
void ModelStore::enforce_host(long long keep) {
  if (host_limit_ < 0 || disk_dir_.empty()) return;
  while (host_bytes_ > host_limit_) {
    long long vk = 0;
    Entry* victim = nullptr;
    for (auto& kv : map_)
      if (kv.first != keep && kv.second.spilled && !kv.second.on_disk && kv.second.bytes > 0 &&
          (!victim || kv.second.tick < victim->tick)) {
        victim = &kv.second;
        vk = kv.first;
      }
    if (!victim) break;
    to_disk(vk, *victim);
  }
}

// one file per model: for every block, its element count (int64) and elements
void ModelStore::to_disk(long long k, Entry& e) {
  auto t0 = std::chrono::steady_clock::now();
  e.file = disk_dir_ + "/tsc_model_" + std::to_string(k >> 32) + "_" + std::to_string(k & 0xffffffff) + "_" +
           std::to_string(reinterpret_cast<uintptr_t>(this)) + ".bin";
  std::FILE* f = std::fopen(e.file.c_str(), "wb");
  if (!f) throw Error(-1, "model spill: cannot create " + e.file);
  bool ok = true;
  for (const auto& h : e.host) {
    const long long n = (long long)h.size();
    ok = ok && std::fwrite(&n, sizeof(n), 1, f) == 1;
    if (n) ok = ok && std::fwrite(h.data(), sizeof(double2), (size_t)n, f) == (size_t)n;
  }
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) {
    std::remove(e.file.c_str());
    throw Error(-1, "model spill: cannot write " + e.file);
  }
  std::vector<std::vector<double2>>().swap(e.host);
  e.on_disk = true;
  host_bytes_ -= e.bytes;
  disk_writes++;
  disk_bytes += (double)e.bytes;
  disk_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void ModelStore::from_disk(Entry& e) {
  auto t0 = std::chrono::steady_clock::now();
  std::FILE* f = std::fopen(e.file.c_str(), "rb");
  if (!f) throw Error(-1, "model spill: cannot open " + e.file);
  e.host.clear();
  bool ok = true;
  size_t nb = 0;
  for_blocks(e.m, [&](DBlock&) { nb++; });
  for (size_t i = 0; i < nb && ok; ++i) {
    long long n = 0;
    ok = std::fread(&n, sizeof(n), 1, f) == 1 && n >= 0;
    e.host.emplace_back();
    if (ok && n) {
      e.host.back().resize((size_t)n);
      ok = std::fread(e.host.back().data(), sizeof(double2), (size_t)n, f) == (size_t)n;
    }
  }
  std::fclose(f);
  if (!ok) throw Error(-1, "model spill: cannot read " + e.file);
  std::remove(e.file.c_str());
  e.file.clear();
  e.on_disk = false;
  host_bytes_ += e.bytes;
  disk_reads++;
  disk_bytes += (double)e.bytes;
  disk_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void ModelStore::clear() {
  for (auto& kv : map_)
    if (kv.second.on_disk) std::remove(kv.second.file.c_str());
  map_.clear();
  resident_ = 0;
  host_bytes_ = 0;
}

DBlock Engine::copy_block(const DBlock& b) {
  DBlock c = b;
  long long off = 0;
  for (auto& s : c.sub) {
    s.off = off;
    off += (long long)s.row_dim * s.sdim;
  }
  c.buf = std::make_shared<DevBuf>((size_t)off, st, false);
  for (int i = 0; i < b.num; ++i) {
    long long n = (long long)b.sub[i].row_dim * b.sub[i].sdim;
    if (n)
      cuda_check(cudaMemcpyAsync(c.buf->p + c.sub[i].off, b.buf->p + b.sub[i].off, n * sizeof(double2),
                                 cudaMemcpyDeviceToDevice, st),
                 "copy");
  }
  return c;
}

double Engine::wave_norm2(const double2* d, long long n) {
  cuda_check(launch_multi_dot(d, 0, 1, d, n, d_red, d_scal + 1900, st), "wave norm");
  cuda_check(cudaMemcpyAsync(h_scal + 1900, d_scal + 1900, sizeof(double), cudaMemcpyDeviceToHost, st), "d2h");
  cuda_check(cudaStreamSynchronize(st), "sync");
  return h_scal[1900];
}

void Engine::normalize(double2* d, long long n) {
  if (n <= 0) return;
  cuda_check(launch_multi_dot(d, 0, 1, d, n, d_red, d_scal + 1901, st), "normalize norm");
  cuda_check(launch_scale(d, d_scal + 1901, n, 1, st), "scale");
}

// random_number stand-in (splitmix64 -> uniform [0,1)), block.f90:1154-1180
double Engine::rand01() {
  uint64_t z = (rng += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z = z ^ (z >> 31);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

void Engine::wave_initialize(const WLayout& wl, double2* d) {
  std::vector<double2> h((size_t)wl.dim);
  for (const auto& s : wl.sec) {
    size_t n = (size_t)s.sys_dim * s.env_dim;
    for (size_t e = 0; e < n; ++e) h[s.off + e].x = rand01();
    for (size_t e = 0; e < n; ++e) h[s.off + e].y = rand01();
  }
  cuda_check(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(double2), cudaMemcpyHostToDevice, st), "upload");
  normalize(d, wl.dim);
  cuda_check(cudaStreamSynchronize(st), "sync");
}

}  // namespace tsc
