// tsc_hpsi_noalloc: H.psi for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc (or any allocating library routine) at
// the moment they need H.psi: a host that has handed its whole device-memory
// budget to its own pool, a solver loop that must not change the allocation
// state between iterations, or code running where an allocation would be
// illegal.  tsc_hpsi_device draws its scratch (the phase-1 left products and
// the partial tiles of split output groups) from buffers the context allocated
// when the superblock was set; this variant instead uses one fixed array in
// device global memory and allocates nothing.
//
// The array is a file-scope __device__ variable: every GPU that loads this
// library holds its 64 MiB until the process exits.  Host code may not use its
// name as a device address (on the host it is only a stand-in symbol), so the
// address is resolved with cudaGetSymbolAddress, with the device current, once
// per device and cached.  tsc_create does this for its device: with lazy module
// loading (the CUDA 12 default) that first lookup is what places the array on
// the device, so it happens when the context is created, never inside
// tsc_hpsi_noalloc.  All calls share the array and it keeps the last call's
// contents; nothing in it needs to start at zero (every element a call reads was
// written earlier in the same call).  Calls that overlap on the GPU -- two
// contexts, or two streams of one device, running at the same time -- race on
// the array.
//
// The entry follows the context's precision like tsc_hpsi_device: in the split
// form it runs the split task lists and, like tsc_hpsi_device, waits for them
// and reads the context's status word (into pinned host memory the context
// already holds).
#include <algorithm>
#include <mutex>

#include "../../include/tsc_gpu.h"
#include "tsc_ctx.hpp"
#include "tsc_engine.hpp"

using namespace tsc;

namespace {

constexpr long long kScratchElems = TSC_NOALLOC_SCRATCH_ELEMS;   // complex128 elements (64 MiB)
static __device__ __align__(256) double2 g_scratch[kScratchElems];

std::mutex g_mu;
double2* g_scratch_addr[256] = {};   // per-device address of g_scratch

double2* scratch_address(int device) {
  if (device < 0 || device >= 256) throw Error(TSC_E_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess || !p)
      throw Error(TSC_E_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    g_scratch_addr[device] = static_cast<double2*>(p);
  }
  return g_scratch_addr[device];
}

}  // namespace

double2* tsc::noalloc_scratch_address(int device) { return scratch_address(device); }

extern "C" int tsc_hpsi_noalloc(tsc_ctx* ctx, const void* d_in, void* d_out) {
  return guard(ctx, [&] {
    if (!ctx->eng || !ctx->eng->sb.valid) throw Error(TSC_E_STATE, "no superblock set");
    if (!d_in || !d_out) throw Error(TSC_E_ARG, "null buffers");
    Engine& E = *ctx->eng;
    Engine::Superblock& S = E.sb;
    const bool split = S.p1s.split;   // the context's precision, as tsc_hpsi_device
    TaskList& a = split ? S.p1s : S.p1;
    TaskList& b = split ? S.p2s : S.p2;
    const long long need = S.scratch_elems + std::max(a.part_elems, b.part_elems);
    if (need > kScratchElems)
      throw Error(TSC_E_LIMIT, "tsc_hpsi_noalloc: superblock needs " + std::to_string(need) +
                                   " complex scratch elements, above the fixed maximum of " +
                                   std::to_string(kScratchElems) + " (use tsc_hpsi_device)");
    double2* scr = scratch_address(ctx->device);
    Bases bs;
    bs.p[0] = nullptr;
    bs.p[1] = const_cast<double2*>(static_cast<const double2*>(d_in));
    bs.p[2] = static_cast<double2*>(d_out);
    bs.p[3] = scr;                       // left products at [0, scratch_elems)
    bs.part = scr + S.scratch_elems;     // partial tiles after them (phases run in order)
    if (split) slice_input(S.sv, static_cast<const double2*>(d_in), E.st);   // into the context's arenas
    for (TaskList* tl : {&a, &b}) {
      if (split)
        cuda_check(launch_grouped_zgemm_split(tl->d_jobs, tl->njobs, tl->d_groups, tl->d_terms, bs, tl->arenas,
                                              E.d_fault, E.split_wait_limit_, tl->term_alpha ? 1 : 0, E.st),
                   "grouped_zgemm_split");
      else
        cuda_check(launch_grouped_zgemm(tl->d_jobs, tl->njobs, tl->d_groups, tl->d_terms, bs, E.st, tl->tile),
                   "grouped_zgemm");
      if (tl->nreds)
        cuda_check(launch_reduce_partials(tl->d_reds, tl->nreds, tl->d_groups, bs, tl->max_red_elems, E.st),
                   "reduce_partials");
    }
    if (split) E.check_split_fault();
  });
}
