// Checkpoint files in the reference's on-disk format, so a run can be stopped,
// moved between this engine and the Fortran code, and continued.
//
// The reference writes, after every DMRG step, one file per stored object
// (names Get_model_name / Get_wave_name, dmrg_sub.f90:657-709):
//   sysblocks<i>, envblocks<i>  model_to_disk   block.f90:1802-1845  (unformatted)
//   systruns<i>,  envtruns<i>   truns_to_disk   block.f90:1936-1956  (unformatted)
//   sysbs<i>,     envbs<i>      basis_to_disk   block.f90:1983-2026  (formatted)
//   eigvec1                     wave_to_disk    block.f90:1547-1576  (unformatted)
// with <i> the block length in decimal.  Unformatted files are sequential
// records, each framed by a 4-byte length before and after it (records longer
// than 2^31-9 bytes split into subrecords whose markers carry a sign: negative
// leading marker = more subrecords follow, negative trailing marker = not the
// first), integers 4 bytes, complex values 16 bytes (re, im), matrices
// column-major: the layout gfortran and ifort both write by default.  A
// Total_Block is the records len, num, dim, up_dif, down_dif and, per
// sub-block, an empty record, (num_up, num_down, down_dif), (row_dim, sdim) and
// the matrix (block_to_disk, block.f90:1713-1737); a model is len, its
// Hamiltonian and, for each of its nleg11(len) boundary sites, elec_up,
// elec_down, spin_sd and num_sn (t-J model, lring = 0).
#include <cerrno>
#include <climits>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/tsc_gpu.h"
#include "tsc_ctx.hpp"
#include "tsc_engine.hpp"

namespace tsc {

namespace {

constexpr long long kMaxSubrecord = 2147483639;   // largest subrecord gfortran writes

struct File {
  FILE* f = nullptr;
  std::string path;
  File(const std::string& p, const char* mode) : path(p) {
    f = std::fopen(p.c_str(), mode);
    if (!f) throw Error(TSC_E_ARG, "checkpoint: cannot open " + p + ": " + std::strerror(errno));
  }
  ~File() {
    if (f) std::fclose(f);
  }
  void put(const void* p, size_t n) {
    if (n && std::fwrite(p, 1, n, f) != n) throw Error(TSC_E_ARG, "checkpoint: write failed on " + path);
  }
  void get(void* p, size_t n) {
    if (n && std::fread(p, 1, n, f) != n) throw Error(TSC_E_ARG, "checkpoint: " + path + " ends early");
  }
};

// ---- unformatted sequential records ----------------------------------------
void put_record(File& F, const void* data, long long n) {
  const char* p = static_cast<const char*>(data);
  long long left = n;
  bool first = true;
  do {
    const long long len = left > kMaxSubrecord ? kMaxSubrecord : left;
    const bool last = len == left;
    const int32_t head = (int32_t)(last ? len : -len), tail = (int32_t)(first ? len : -len);
    F.put(&head, 4);
    F.put(p, (size_t)len);
    F.put(&tail, 4);
    p += len;
    left -= len;
    first = false;
  } while (left > 0);
}
std::vector<char> get_record(File& F) {
  std::vector<char> out;
  while (true) {
    int32_t head = 0, tail = 0;
    F.get(&head, 4);
    const long long len = head < 0 ? -(long long)head : head;
    const size_t at = out.size();
    out.resize(at + (size_t)len);
    F.get(out.data() + at, (size_t)len);
    F.get(&tail, 4);
    if ((tail < 0 ? -(long long)tail : tail) != len) throw Error(TSC_E_ARG, "checkpoint: bad record marker in " + F.path);
    if (head >= 0) return out;
  }
}
void put_ints(File& F, std::initializer_list<int> v) {
  std::vector<int32_t> a(v.begin(), v.end());
  put_record(F, a.data(), (long long)a.size() * 4);
}
std::vector<int> get_ints(File& F, size_t n) {
  std::vector<char> r = get_record(F);
  if (r.size() != 4 * n) throw Error(TSC_E_ARG, "checkpoint: unexpected record length in " + F.path);
  std::vector<int> v(n);
  std::memcpy(v.data(), r.data(), 4 * n);
  return v;
}
int as_int(long long x, const char* what) {
  if (x < INT_MIN || x > INT_MAX) throw Error(TSC_E_LIMIT, std::string("checkpoint: ") + what + " exceeds 32 bits");
  return (int)x;
}

// block_to_disk / block_from_disk (block.f90:1713-1764)
void write_block(Engine& E, File& F, const DBlock& b) {
  std::vector<int> ints;
  std::vector<cplx> data;
  if (b.buf || b.num == 0) E.download_block(b, ints, data);
  else throw Error(TSC_E_STATE, "checkpoint: block without device data");
  put_ints(F, {b.len});
  put_ints(F, {b.num});
  put_ints(F, {b.dim});
  put_ints(F, {b.up_dif});
  put_ints(F, {b.down_dif});
  long long d = 0;
  for (int i = 0; i < b.num; ++i) {
    const int* s = &ints[5 + 5 * i];
    put_record(F, nullptr, 0);
    put_ints(F, {s[0], s[1], s[2]});
    put_ints(F, {s[3], s[4]});
    const long long n = (long long)s[3] * s[4];
    put_record(F, data.data() + d, n * 16);
    d += n;
  }
}
DBlock read_block(Engine& E, File& F) {
  std::vector<int> ints(5);
  for (int k = 0; k < 5; ++k) ints[k] = get_ints(F, 1)[0];
  const int num = ints[1];
  if (num < 0 || num > 1000000) throw Error(TSC_E_ARG, "checkpoint: bad block in " + F.path);
  std::vector<cplx> data;
  for (int i = 0; i < num; ++i) {
    get_record(F);   // the empty record before each sub-block
    std::vector<int> a = get_ints(F, 3), b = get_ints(F, 2);
    ints.insert(ints.end(), {a[0], a[1], a[2], b[0], b[1]});
    std::vector<char> m = get_record(F);
    if ((long long)m.size() != 16ll * b[0] * b[1]) throw Error(TSC_E_ARG, "checkpoint: matrix size in " + F.path);
    const size_t at = data.size();
    data.resize(at + m.size() / 16);
    std::memcpy(data.data() + at, m.data(), m.size());
  }
  const int* ip = ints.data();
  const cplx* dp = data.data();
  return E.upload_block(ip, dp);
}

std::string name(const std::string& dir, const char* stem, int i) { return dir + "/" + stem + std::to_string(i); }

}  // namespace

// model_to_disk (block.f90:1802-1845): len, ham, then the boundary-site operators
static void write_model(Engine& E, const std::string& path, const DModel& m) {
  File F(path, "wb");
  put_ints(F, {m.len});
  write_block(E, F, m.ham);
  for (int ii = 1; ii <= E.L.nleg11[m.len]; ++ii)
    for (int o = 0; o < 4; ++o) write_block(E, F, m.sub[ii].op[o]);
}
static DModel read_model(Engine& E, const std::string& path) {
  File F(path, "rb");
  DModel m;
  m.len = get_ints(F, 1)[0];
  if (m.len < 1 || m.len > E.L.num_site) throw Error(TSC_E_ARG, "checkpoint: bad model length in " + path);
  m.ham = read_block(E, F);
  m.sub.resize(E.L.num_site + 1);
  for (int ii = 1; ii <= E.L.nleg11[m.len]; ++ii)
    for (int o = 0; o < 4; ++o) m.sub[ii].op[o] = read_block(E, F);
  return m;
}

// basis_to_disk / basis_from_disk (block.f90:1983-2083): formats 101 (A4,I6),
// 102 (A11,I4), 103 (A13,I4), 104 (A10,I4,2X,A12,I4); an empty line before each
// sector; idx and num are both the sector's piece count (Get_basis, block.f90:2155-2177)
static void write_basis(const std::string& path, const Basis& b) {
  File F(path, "w");
  std::fprintf(F.f, "len=%6d\nnum=%6d\ndim=%6d\n", b.len, b.num, b.dim);
  for (const auto& s : b.sec) {
    const int np = (int)s.pcs.size();
    std::fprintf(F.f, "\nidx=%6d\nnum=%6d\ndim=%6d\nnew_num_up=%4d\nnew_num_down=%4d\n", np, np, s.dim, s.num_up,
                 s.num_down);
    for (const auto& p : s.pcs)
      std::fprintf(F.f, "pos=%6d\ndim=%6d\nbl_num_up=%4d  bl_num_down=%4d\nst_num_up=%4d  st_num_down=%4d\n", p.spos,
                   p.sdim, p.bl_num_up, p.bl_num_down, p.st_num_up, p.st_num_down);
  }
}
static Basis read_basis(const std::string& path) {
  File F(path, "r");
  char line[256];
  auto next = [&]() -> std::string {
    if (!std::fgets(line, sizeof line, F.f)) throw Error(TSC_E_ARG, "checkpoint: " + path + " ends early");
    std::string s(line);
    while (!s.empty() && (s.back() == '\n' || s.back() == '\r')) s.pop_back();
    return s;
  };
  auto field = [&](const std::string& s, size_t at, size_t w) -> int {
    if (s.size() < at) throw Error(TSC_E_ARG, "checkpoint: short line in " + path);
    return std::stoi(s.substr(at, w));
  };
  Basis b;
  b.len = field(next(), 4, 6);
  b.num = field(next(), 4, 6);
  b.dim = field(next(), 4, 6);
  if (b.num < 0 || b.num > 1000000) throw Error(TSC_E_ARG, "checkpoint: bad basis in " + path);
  b.sec.resize(b.num);
  for (auto& s : b.sec) {
    next();   // the empty line
    field(next(), 4, 6);   // idx
    const int np = field(next(), 4, 6);
    s.dim = field(next(), 4, 6);
    s.num_up = field(next(), 11, 4);
    s.num_down = field(next(), 13, 4);
    for (int x = 0; x < np; ++x) {
      Piece p;
      p.spos = field(next(), 4, 6);
      p.sdim = field(next(), 4, 6);
      std::string a = next();
      p.bl_num_up = field(a, 10, 4);
      p.bl_num_down = field(a, 28, 4);
      std::string c = next();
      p.st_num_up = field(c, 10, 4);
      p.st_num_down = field(c, 28, 4);
      s.pcs.push_back(p);
    }
  }
  return b;
}

// wave_to_disk / wave_from_disk (block.f90:1547-1607)
static void write_wave(Engine& E, const std::string& path, const WLayout& w, const DevBufP& d) {
  File F(path, "wb");
  put_ints(F, {w.sys_len});
  put_ints(F, {w.env_len});
  put_ints(F, {w.num});
  put_ints(F, {as_int(w.dim, "wave dimension")});
  std::vector<cplx> h((size_t)w.dim);
  if (w.dim)
    cuda_check(cudaMemcpyAsync(h.data(), d->p, w.dim * sizeof(double2), cudaMemcpyDeviceToHost, E.st), "d2h");
  cuda_check(cudaStreamSynchronize(E.st), "sync");
  for (const auto& s : w.sec) {
    put_record(F, nullptr, 0);
    put_ints(F, {s.sys_num_up, s.sys_num_down});
    put_ints(F, {s.env_num_up, s.env_num_down});
    put_ints(F, {s.sys_dim, s.env_dim});
    put_record(F, h.data() + s.off, 16ll * s.sys_dim * s.env_dim);
  }
}

int Engine::checkpoint_write(const std::string& dir) {
  if (!disk_wave || disk_layout.num == 0) throw Error(TSC_E_STATE, "checkpoint: no run to save");
  int files = 0;
  for (auto key : models_.keys()) {
    write_model(*this, name(dir, key.first == 0 ? "sysblocks" : "envblocks", key.second), models_.get(key.first, key.second));
    files++;
  }
  for (int side = 0; side < 2; ++side) {
    for (const auto& kv : side ? env_truns : sys_truns) {
      File F(name(dir, side ? "envtruns" : "systruns", kv.first), "wb");
      write_block(*this, F, kv.second);
      files++;
    }
    for (const auto& kv : side ? env_bsm : sys_bsm) {
      write_basis(name(dir, side ? "envbs" : "sysbs", kv.first), kv.second);
      files++;
    }
  }
  write_wave(*this, dir + "/eigvec1", disk_layout, disk_wave);
  return files + 1;
}

void Engine::checkpoint_read(const std::string& dir) {
  models_.clear();
  sys_truns.clear();
  env_truns.clear();
  sys_bsm.clear();
  env_bsm.clear();
  const int N = L.num_site;
  for (int side = 0; side < 2; ++side)
    for (int i = 1; i <= N; ++i) {
      const std::string mb = name(dir, side ? "envblocks" : "sysblocks", i);
      if (FILE* f = std::fopen(mb.c_str(), "rb")) {
        std::fclose(f);
        DModel m = read_model(*this, mb);
        if (m.len != i) throw Error(TSC_E_ARG, "checkpoint: " + mb + " holds length " + std::to_string(m.len));
        models_.put(side, i, m);
      }
      const std::string tr = name(dir, side ? "envtruns" : "systruns", i);
      if (FILE* f = std::fopen(tr.c_str(), "rb")) {
        std::fclose(f);
        File F(tr, "rb");
        (side ? env_truns : sys_truns)[i] = read_block(*this, F);
      }
      const std::string bs = name(dir, side ? "envbs" : "sysbs", i);
      if (FILE* f = std::fopen(bs.c_str(), "r")) {
        std::fclose(f);
        (side ? env_bsm : sys_bsm)[i] = read_basis(bs);
      }
    }
  File F(dir + "/eigvec1", "rb");
  WLayout w;
  w.sys_len = get_ints(F, 1)[0];
  w.env_len = get_ints(F, 1)[0];
  w.num = get_ints(F, 1)[0];
  const int dim = get_ints(F, 1)[0];
  if (w.num < 0 || dim < 0) throw Error(TSC_E_ARG, "checkpoint: bad wave");
  std::vector<cplx> h;
  for (int k = 0; k < w.num; ++k) {
    get_record(F);
    std::vector<int> a = get_ints(F, 2), b = get_ints(F, 2), c = get_ints(F, 2);
    WSec s;
    s.sys_num_up = a[0];
    s.sys_num_down = a[1];
    s.env_num_up = b[0];
    s.env_num_down = b[1];
    s.sys_dim = c[0];
    s.env_dim = c[1];
    s.off = (long long)h.size();
    std::vector<char> v = get_record(F);
    if ((long long)v.size() != 16ll * s.sys_dim * s.env_dim) throw Error(TSC_E_ARG, "checkpoint: wave sector size");
    h.resize(h.size() + v.size() / 16);
    std::memcpy(h.data() + s.off, v.data(), v.size());
    w.sec.push_back(s);
  }
  w.dim = (long long)h.size();
  if (w.dim != dim) throw Error(TSC_E_ARG, "checkpoint: wave dimension mismatch");
  disk_wave = std::make_shared<DevBuf>((size_t)std::max<long long>(w.dim, 1), st, false);
  if (w.dim)
    cuda_check(cudaMemcpyAsync(disk_wave->p, h.data(), w.dim * sizeof(double2), cudaMemcpyHostToDevice, st), "h2d");
  cuda_check(cudaStreamSynchronize(st), "sync");
  disk_layout = w;
  resume_ready_ = true;
}

}  // namespace tsc

using namespace tsc;

extern "C" int tsc_checkpoint_write(tsc_ctx* ctx, const char* dir) {
  int files = 0;
  const int rc = guard(ctx, [&] {
    if (!ctx->eng || !dir) throw Error(TSC_E_ARG, "no engine or directory");
    files = ctx->eng->checkpoint_write(dir);
  });
  return rc == TSC_OK ? files : rc;
}

extern "C" int tsc_checkpoint_read(tsc_ctx* ctx, const char* dir) {
  return guard(ctx, [&] {
    if (!ctx->eng || !dir) throw Error(TSC_E_ARG, "no engine or directory");
    ctx->eng->checkpoint_read(dir);
  });
}
