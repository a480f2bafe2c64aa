// ct_accel.cuh -- host-side owner of a built acceleration structure.
#pragma once
#include <mutex>
#include <vector>
#include <cuda_runtime.h>
#include "ct_types.cuh"

struct ct_accel {
  DevAccel dev = {};
  std::vector<DevGrid> h_grids;
  DevGrid *d_grids = nullptr;
  uint32_t *d_table = nullptr;
  uint32_t *d_pslot = nullptr;
  uint32_t *d_mask = nullptr;
  uint32_t *d_prim = nullptr;
  uint32_t *d_vcoord = nullptr;
  uint32_t *d_field = nullptr;
  ct_accel_info info = {};
  uint32_t n_primitives = 0;  // AABBs (global primitive indices) the structure was built over
  // scratch of ct_restir_di when the caller passes none (grown on demand)
  std::mutex ws_mu;
  void *ws_ptr = nullptr;
  uint64_t ws_bytes = 0;
  ~ct_accel();
};

void ct_set_cuda_error(cudaError_t e);
