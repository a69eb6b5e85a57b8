// mlp.cuh -- learned per-node Newton predictor: device state and kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

struct pfem_ctx;
struct pfem_solve_opts;

namespace pfem {

struct MlpState {
  bool ready = false;
  int used_count = 0;
};

inline void mlp_free(MlpState&) {}

}  // namespace pfem
