// Definition of the opaque C-ABI handle (include/tsc_gpu.h), shared by the
// translation units that implement entry points.
#pragma once
#include <memory>
#include <string>
#include <vector>

#include "tsc_engine.hpp"

struct tsc_ctx {
  std::unique_ptr<tsc::Engine> eng;
  std::string err;
  std::vector<int> out_ints;
  std::vector<tsc::cplx> out_data;
  int device = 0;
};

namespace tsc {

// Runs an entry point's body with the context's device current and turns
// engine exceptions into the status code (and message) of include/tsc_gpu.h.
template <class F>
int guard(tsc_ctx* c, F&& f) {
  if (!c) return -1;
  try {
    if (c->eng) cuda_check(cudaSetDevice(c->device), "cudaSetDevice");
    f();
    c->err.clear();
    return 0;
  } catch (Error& e) {
    c->err = e.what();
    return e.code;
  } catch (std::exception& e) {
    c->err = e.what();
    return -1;
  }
}

// Address of the fixed scratch array of tsc_hpsi_noalloc on `device` (which
// must be current), resolved once per device and cached (tsc_noalloc.cu).
double2* noalloc_scratch_address(int device);

}  // namespace tsc
