// ct_api.cu -- argument checking and dispatch of the C ABI (include/ct.h).
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstring>
#include "ct_accel.cuh"
#include "ct_kernels.cuh"

static thread_local char g_cuda_err[256] = "";

void ct_set_cuda_error(cudaError_t e) {
  snprintf(g_cuda_err, sizeof(g_cuda_err), "%s: %s", cudaGetErrorName(e), cudaGetErrorString(e));
}

static ct_status cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return CT_OK;
  ct_set_cuda_error(e);
  return CT_ERR_CUDA;
}

extern "C" uint32_t ct_abi_version(void) { return CT_ABI_VERSION; }

extern "C" const char *ct_last_cuda_error(void) { return g_cuda_err; }

extern "C" const char *ct_status_string(ct_status s) {
  switch (s) {
    case CT_OK: return "ok";
    case CT_ERR_INVALID_ARG: return "invalid argument";
    case CT_ERR_CAPACITY: return "capacity exceeded";
    case CT_ERR_CUDA: return "CUDA error";
    case CT_ERR_ITER_LIMIT: return "device loop iteration limit reached";
    case CT_ERR_NAN_INPUT: return "non-finite input";
    case CT_ERR_UNSUPPORTED: return "unsupported feature";
    case CT_ERR_NOT_GRID_ALIGNED: return "AABB is not a grid-aligned voxel";
  }
  return "unknown status";
}

// Reference values: src/shaders/include/defines.glsl:34-48,
// src/shaders/shared.inl:45, src/shaders/glsl/compute/taa.glsl:13.
extern "C" void ct_params_default(ct_params *p) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->struct_size = sizeof(ct_params);
  p->voxel_extent = 0.03125f;
  p->min_ris_point_samples = 1;
  p->max_ris_point_samples = 4;
  p->min_ris_env_samples = 1;
  p->max_ris_env_samples = 4;
  p->min_ris_cube_samples = 4;
  p->max_ris_cube_samples = 32;
  p->min_influence_from_the_past = 10.0f;
  p->max_influence_from_the_past = 20.0f;
  p->min_num_of_neighbors = 3;
  p->max_num_of_neighbors = 4;
  p->min_neighbors_radius = 2.0f;
  p->max_neighbors_radius = 50.0f;
  p->max_distance_to_hit = 1e3f;
  p->spatial_passes = 1;
  p->taa_alpha = 0.8f;
  p->flags = 0;
  p->counters_address = 0;
}

static ct_status check_params(const ct_params *P) {
  if (!P || P->struct_size != sizeof(ct_params)) return CT_ERR_INVALID_ARG;
  if (P->max_num_of_neighbors > CT_MAX_NEIGHBORS || P->min_num_of_neighbors > CT_MAX_NEIGHBORS) return CT_ERR_CAPACITY;
  if (P->spatial_passes < 1 || P->spatial_passes > 16) return CT_ERR_INVALID_ARG;
  if (!std::isfinite(P->taa_alpha) || !std::isfinite(P->max_influence_from_the_past) ||
      !std::isfinite(P->min_neighbors_radius) || !std::isfinite(P->max_neighbors_radius) ||
      !(P->max_distance_to_hit > 0.0f))
    return CT_ERR_NAN_INPUT;
  if ((P->flags & CT_PARAM_COUNT_RAYS) && (P->counters_address == 0 || (P->counters_address & 7u)))
    return CT_ERR_INVALID_ARG;
  return CT_OK;
}

static ct_status check_pc(const ct_push_constant *pc, bool needs_accel) {
  if (!pc) return CT_ERR_INVALID_ARG;
  if (pc->size[0] == 0 || pc->size[1] == 0) return CT_ERR_INVALID_ARG;
  if ((uint64_t)pc->size[0] * pc->size[1] > 0xFFFFFFFFull) return CT_ERR_CAPACITY;
  if (needs_accel && !pc->tlas) return CT_ERR_INVALID_ARG;
  if (!pc->camera_buffer || !pc->status_buffer || !pc->world_buffer || !pc->restir_buffer) return CT_ERR_INVALID_ARG;
  if ((pc->camera_buffer | pc->status_buffer | pc->world_buffer | pc->restir_buffer) & 7u) return CT_ERR_INVALID_ARG;
  if (!pc->swapchain || !pc->taa_frame || !pc->previous_swapchain) return CT_ERR_INVALID_ARG;
  if (((uintptr_t)pc->swapchain | (uintptr_t)pc->taa_frame | (uintptr_t)pc->previous_swapchain) & 15u)
    return CT_ERR_INVALID_ARG;
  return CT_OK;
}

static ct_status check_extent(const ct_push_constant *pc, const ct_params *P) {
  // the scene's voxel edge is fixed when the acceleration structure is built
  if (pc->tlas && pc->tlas->dev.extent != P->voxel_extent) return CT_ERR_INVALID_ARG;
  return CT_OK;
}

extern "C" ct_status ct_trace_frame(const ct_push_constant *pc, const ct_params *P, ct_stream stream) {
  ct_status st = check_pc(pc, true);
  if (st == CT_OK) st = check_params(P);
  if (st == CT_OK) st = check_extent(pc, P);
  if (st != CT_OK) return st;
  return cuda_status(ct_launch_trace(*pc, pc->tlas->dev, *P, (cudaStream_t)stream));
}

extern "C" ct_status ct_restir_di(const ct_push_constant *pc, const ct_params *P, int stage, ct_stream stream) {
  ct_status st = check_pc(pc, true);
  if (st == CT_OK) st = check_params(P);
  if (st == CT_OK) st = check_extent(pc, P);
  if (st != CT_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  const DevAccel &A = pc->tlas->dev;
  if (stage == 0) return cuda_status(ct_launch_di_initial(*pc, A, *P, s));
  if (stage != 1) return CT_ERR_INVALID_ARG;
  // spatial rounds: intermediate -> reservoir -> intermediate ... ; the last
  // round shades.  Extra rounds need the RESTIR.reservoir buffer, whose
  // address the kernels read on the device, so the host only forwards the
  // round's source/destination choice.
  for (uint32_t r = 0; r + 1 < P->spatial_passes; r++) {
    cudaError_t e = ct_launch_di_shade(*pc, A, *P, (int)(r & 1u), 0, (int)((r & 1u) ^ 1u), s);
    if (e != cudaSuccess) return cuda_status(e);
  }
  return cuda_status(ct_launch_di_shade(*pc, A, *P, (int)((P->spatial_passes - 1) & 1u), 1, 0, s));
}

extern "C" ct_status ct_taa(const ct_push_constant *pc, const ct_params *P, ct_stream stream) {
  ct_status st = check_pc(pc, false);
  if (st == CT_OK) st = check_params(P);
  if (st != CT_OK) return st;
  return cuda_status(ct_launch_taa(*pc, *P, (cudaStream_t)stream));
}

extern "C" ct_status ct_render_frame(const ct_push_constant *pc, const ct_params *P, uint32_t is_active,
                                     ct_stream stream) {
  ct_status st = ct_trace_frame(pc, P, stream);
  if (st != CT_OK) return st;
  st = ct_restir_di(pc, P, 0, stream);
  if (st != CT_OK) return st;
  st = ct_restir_di(pc, P, 1, stream);
  if (st != CT_OK) return st;
  if (is_active & CT_TAA_BIT) st = ct_taa(pc, P, stream);
  return st;
}

extern "C" ct_status ct_get_error(ct_stream stream, int reset, ct_error_info *out) {
  if (!out) return CT_ERR_INVALID_ARG;
  uint32_t w[4] = {0, 0, 0, 0};
  cudaError_t e = ct_error_word_read(w, reset, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_status(e);
  out->status = (ct_status)w[0];
  out->detail = w[1];
  out->pixel = w[2];
  out->_pad = 0;
  return CT_OK;
}
