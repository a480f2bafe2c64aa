// ct_accel.cuh -- host-side owner of a built acceleration structure.
#pragma once
#include <vector>
#include <cuda_runtime.h>
#include "ct_types.cuh"

struct ct_accel {
  DevAccel dev = {};
  std::vector<DevGrid> h_grids;
  DevGrid *d_grids = nullptr;
  uint32_t *d_table = nullptr;
  uint32_t *d_occ = nullptr;
  uint32_t *d_prim = nullptr;
  uint32_t *d_vcoord = nullptr;
  ct_accel_info info = {};
  ~ct_accel();
};

void ct_set_cuda_error(cudaError_t e);
