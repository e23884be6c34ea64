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
