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
// first call on each device, with that device current, resolves the address
// with cudaGetSymbolAddress and caches it; make that first call before any
// stream capture begins.  All calls share the array and it keeps the last
// call's contents; nothing in it needs to start at zero (every element a call
// reads was written earlier in the same call).  Calls that overlap on the GPU --
// two contexts, or two streams of one device, running at the same time -- race
// on the array.
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

extern "C" int tsc_hpsi_noalloc(tsc_ctx* ctx, const void* d_in, void* d_out) {
  if (!ctx) return TSC_E_ARG;
  try {
    if (!ctx->eng || !ctx->eng->sb.valid) throw Error(TSC_E_STATE, "no superblock set");
    if (!d_in || !d_out) throw Error(TSC_E_ARG, "null buffers");
    Engine& E = *ctx->eng;
    Engine::Superblock& S = E.sb;
    const long long need = S.scratch_elems + std::max(S.p1.part_elems, S.p2.part_elems);
    if (need > kScratchElems)
      throw Error(TSC_E_LIMIT, "tsc_hpsi_noalloc: superblock needs " + std::to_string(need) +
                                   " complex scratch elements, above the fixed maximum of " +
                                   std::to_string(kScratchElems) + " (use tsc_hpsi_device)");
    cuda_check(cudaSetDevice(ctx->device), "cudaSetDevice");
    double2* scr = scratch_address(ctx->device);
    Bases b;
    b.p[0] = nullptr;
    b.p[1] = const_cast<double2*>(static_cast<const double2*>(d_in));
    b.p[2] = static_cast<double2*>(d_out);
    b.p[3] = scr;                       // left products at [0, scratch_elems)
    b.part = scr + S.scratch_elems;     // partial tiles after them (phases run in order)
    for (TaskList* tl : {&S.p1, &S.p2}) {
      cuda_check(launch_grouped_zgemm(tl->d_jobs, tl->njobs, tl->d_groups, tl->d_terms, b, E.st, tl->tile),
                 "grouped_zgemm");
      if (tl->nreds)
        cuda_check(launch_reduce_partials(tl->d_reds, tl->nreds, tl->d_groups, b, tl->max_red_elems, E.st),
                   "reduce_partials");
    }
    ctx->err.clear();
    return TSC_OK;
  } catch (Error& e) {
    ctx->err = e.what();
    return e.code;
  } catch (std::exception& e) {
    ctx->err = e.what();
    return TSC_E_ARG;
  }
}
