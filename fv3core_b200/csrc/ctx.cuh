// Context layout shared by the stage sources.
#pragma once
#include "common.cuh"

namespace fv3b {
constexpr int NWS = 24;  // 3-D scratch fields in the workspace
}

struct fv3b_ctx {
  fv3b::Dims d;
  fv3b_metrics m;
  double* ws_base = nullptr;
  double* ws[fv3b::NWS];
};
