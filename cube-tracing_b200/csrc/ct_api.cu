// ct_api.cu -- argument checking and dispatch of the C ABI (include/ct.h).
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>
#include "ct_accel.cuh"
#include "ct_kernels.cuh"

static thread_local char g_cuda_err[256] = "";

void ct_set_cuda_error(cudaError_t e) {
  snprintf(g_cuda_err, sizeof(g_cuda_err), "%s: %s", cudaGetErrorName(e), cudaGetErrorString(e));
}

ct_status cuda_status(cudaError_t e) {
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
  p->pt_neighbor_count = 3;
  p->pt_neighbor_radius = 1;
  p->pt_max_influence_from_the_past = 20.0f;
  p->counters_address = 0;
  p->workspace_address = 0;
  p->workspace_bytes = 0;
  p->walker_blocks = 0;
  p->pt_shift_mapping = CT_SHIFT_RECONNECTION;
  p->pt_near_field_distance = 0.0f;
  p->_reserved = 0;
}

ct_status check_params(const ct_params *P) {
  if (!P || P->struct_size != sizeof(ct_params)) return CT_ERR_INVALID_ARG;
  if (P->max_num_of_neighbors > CT_MAX_NEIGHBORS || P->min_num_of_neighbors > CT_MAX_NEIGHBORS) return CT_ERR_CAPACITY;
  if (P->spatial_passes < 1 || P->spatial_passes > 16) return CT_ERR_INVALID_ARG;
  if (P->pt_neighbor_count > 64 || P->pt_neighbor_radius < 0 || P->pt_neighbor_radius > 4096) return CT_ERR_INVALID_ARG;
  if (!std::isfinite(P->pt_max_influence_from_the_past)) return CT_ERR_NAN_INPUT;
  if (!std::isfinite(P->taa_alpha) || !std::isfinite(P->max_influence_from_the_past) ||
      !std::isfinite(P->min_neighbors_radius) || !std::isfinite(P->max_neighbors_radius) ||
      !(P->max_distance_to_hit > 0.0f))
    return CT_ERR_NAN_INPUT;
  if ((P->flags & CT_PARAM_COUNT_RAYS) && (P->counters_address == 0 || (P->counters_address & 7u)))
    return CT_ERR_INVALID_ARG;
  if (P->walk_step_limit > (uint32_t)CT_DDA_MAX_STEPS) return CT_ERR_INVALID_ARG;
  if (P->pt_shift_mapping != CT_SHIFT_RECONNECTION && P->pt_shift_mapping != CT_SHIFT_HYBRID) return CT_ERR_INVALID_ARG;
  if (!std::isfinite(P->pt_near_field_distance) || P->pt_near_field_distance < 0.0f) return CT_ERR_NAN_INPUT;
  return CT_OK;
}

ct_status check_pc(const ct_push_constant *pc, bool needs_accel) {
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

// Workspace layout, 256-byte aligned pieces:
//   [counter 256 B][answers W*H*16 B][radiance W*H*16*12 B][neighbours W*H*8*4 B]
//   [neighbour meta W*H*8 B][queue a: cap*16][queue b: cap*16][queue c: cap*8]
// cap = W*H * (most shadow rays one pixel asks for in one wavefront round)
static uint64_t align256(uint64_t v) { return (v + 255u) & ~255ull; }
static uint64_t rays_per_pixel(const ct_params *P) {
  uint32_t nmax = P->max_num_of_neighbors > P->min_num_of_neighbors ? P->max_num_of_neighbors : P->min_num_of_neighbors;
  if (nmax > CT_MAX_NEIGHBORS) nmax = CT_MAX_NEIGHBORS;
  uint64_t r = 2ull * nmax;
  return r < 3 ? 3 : r;
}
// With CT_PARAM_INDIRECT the ReSTIR PT wavefront follows:
//   [path states W*H*CT_PT_STATE_BYTES][closest hits W*H*16][ray queues 2 x W*H*32]
// and with the hybrid shift [replay results W*H*2*64][replay jobs W*H*2*4]
uint64_t workspace_bytes(uint32_t W, uint32_t H, const ct_params *P, uint64_t *cap_out) {
  const uint64_t px = (uint64_t)W * H;
  const uint64_t cap = px * rays_per_pixel(P);
  if (cap_out) *cap_out = cap;
  uint64_t b = 256 + align256(px * 16) + align256(px * 16 * 12) + align256(px * 32) + align256(px * 8) +
               align256(cap * 16) * 2 + align256(cap * 8);
  if (P->flags & CT_PARAM_INDIRECT) b += align256(px * CT_PT_STATE_BYTES) + align256(px * 16) + 2 * align256(px * 32);
  if ((P->flags & CT_PARAM_INDIRECT) && P->pt_shift_mapping == CT_SHIFT_HYBRID) b += align256(px * 128) + align256(px * 8);
  return b;
}
CtWorkspace carve_workspace(void *base, uint32_t W, uint32_t H, const ct_params *P) {
  uint64_t cap = 0;
  workspace_bytes(W, H, P, &cap);
  const uint64_t px = (uint64_t)W * H;
  char *p = (char *)base;
  CtWorkspace w;
  w.counter = (uint32_t *)p;
  p += 256;
  w.vis = (uint8_t *)p;
  p += align256(px * 16);
  w.rad = (float *)p;
  p += align256(px * 16 * 12);
  w.nbr = (uint32_t *)p;
  p += align256(px * 32);
  w.smeta = p;
  p += align256(px * 8);
  w.ray_a = p;
  p += align256(cap * 16);
  w.ray_b = p;
  p += align256(cap * 16);
  w.ray_c = p;
  p += align256(cap * 8);
  w.capacity = (uint32_t)(cap > 0xFFFFFFFFull ? 0xFFFFFFFFull : cap);
  w.pt_state = w.pt_hit = w.pt_q[0] = w.pt_q[1] = w.pt_replay = w.pt_jobs = nullptr;
  w.pt_capacity = 0;
  if (P->flags & CT_PARAM_INDIRECT) {
    w.pt_state = p;
    p += align256(px * CT_PT_STATE_BYTES);
    w.pt_hit = p;
    p += align256(px * 16);
    w.pt_q[0] = p;
    p += align256(px * 32);
    w.pt_q[1] = p;
    p += align256(px * 32);
    w.pt_capacity = (uint32_t)(px > 0xFFFFFFFFull ? 0xFFFFFFFFull : px);
    if (P->pt_shift_mapping == CT_SHIFT_HYBRID) {
      w.pt_replay = p;
      p += align256(px * 128);
      w.pt_jobs = p;
    }
  }
  return w;
}

extern "C" ct_status ct_workspace_size(uint32_t width, uint32_t height, const ct_params *params, uint64_t *out) {
  if (!params || !out || width == 0 || height == 0) return CT_ERR_INVALID_ARG;
  ct_status st = check_params(params);
  if (st != CT_OK) return st;
  *out = workspace_bytes(width, height, params, nullptr);
  return CT_OK;
}

static ct_status get_workspace(const ct_push_constant *pc, const ct_params *P, CtWorkspace *out) {
  const uint32_t W = pc->size[0], H = pc->size[1];
  const uint64_t need = workspace_bytes(W, H, P, nullptr);
  if (P->workspace_address) {
    if (P->workspace_bytes < need || (P->workspace_address & 255u)) return CT_ERR_CAPACITY;
    *out = carve_workspace((void *)(uintptr_t)P->workspace_address, W, H, P);
    return CT_OK;
  }
  ct_accel *acc = const_cast<ct_accel *>(pc->tlas);
  std::lock_guard<std::mutex> lk(acc->ws_mu);
  if (acc->ws_bytes < need) {
    // the old scratch may still be in use by work already queued
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) {
      cudaFree(acc->ws_ptr);
      acc->ws_ptr = nullptr;
      acc->ws_bytes = 0;
      e = cudaMalloc(&acc->ws_ptr, need);
    }
    if (e != cudaSuccess) return cuda_status(e);
    acc->ws_bytes = need;
  }
  *out = carve_workspace(acc->ws_ptr, W, H, P);
  return CT_OK;
}

// the acceleration structure as the kernels see it, with the walk cap of P
DevAccel walk_accel(const ct_accel *a, const ct_params *P) {
  DevAccel A = a->dev;
  if (P->walk_step_limit) A.max_steps = P->walk_step_limit;
  return A;
}

ct_status check_extent(const ct_push_constant *pc, const ct_params *P) {
  // the scene's voxel edge is fixed when the acceleration structure is built
  if (pc->tlas && pc->tlas->dev.extent != P->voxel_extent) return CT_ERR_INVALID_ARG;
  return CT_OK;
}

extern "C" ct_status ct_trace_frame(const ct_push_constant *pc, const ct_params *P, ct_stream stream) {
  ct_status st = check_pc(pc, true);
  if (st == CT_OK) st = check_params(P);
  if (st == CT_OK) st = check_extent(pc, P);
  if (st != CT_OK) return st;
  return cuda_status(ct_launch_trace(*pc, walk_accel(pc->tlas, P), *P, (cudaStream_t)stream));
}

extern "C" ct_status ct_restir_di(const ct_push_constant *pc, const ct_params *P, int stage, ct_stream stream) {
  ct_status st = check_pc(pc, true);
  if (st == CT_OK) st = check_params(P);
  if (st == CT_OK) st = check_extent(pc, P);
  if (st != CT_OK) return st;
  if (stage != 0 && stage != 1) return CT_ERR_INVALID_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const DevAccel A = walk_accel(pc->tlas, P);
  CtWorkspace w;
  st = get_workspace(pc, P, &w);
  if (st != CT_OK) return st;
  const DevAccel A_prev = pc->tlas_previous ? walk_accel(pc->tlas_previous, P) : A;
  if (stage == 0) return cuda_status(ct_launch_di_stage0(*pc, A, A_prev, *P, w, s));
  // spatial rounds: intermediate -> reservoir -> intermediate ... ; the last
  // round shades.  Extra rounds need the RESTIR.reservoir buffer, whose
  // address the kernels read on the device, so the host only forwards the
  // round's source/destination choice.
  for (uint32_t r = 0; r + 1 < P->spatial_passes; r++) {
    cudaError_t e = ct_launch_spatial_round(*pc, A, *P, w, (int)(r & 1u), 0, (int)((r & 1u) ^ 1u), s);
    if (e != cudaSuccess) return cuda_status(e);
  }
  return cuda_status(ct_launch_spatial_round(*pc, A, *P, w, (int)((P->spatial_passes - 1) & 1u), 1, 0, s));
}

extern "C" ct_status ct_restir_pt(const ct_push_constant *pc, const ct_params *P, int stage, ct_stream stream) {
  ct_status st = check_pc(pc, true);
  if (st == CT_OK) st = check_params(P);
  if (st == CT_OK) st = check_extent(pc, P);
  if (st != CT_OK) return st;
  if ((stage != 0 && stage != 1) || !(P->flags & CT_PARAM_INDIRECT)) return CT_ERR_INVALID_ARG;
  CtWorkspace w;
  st = get_workspace(pc, P, &w);
  if (st != CT_OK) return st;
  return cuda_status(ct_launch_pt(*pc, walk_accel(pc->tlas, P), *P, w, stage, (cudaStream_t)stream));
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
  const bool indirect = (P->flags & CT_PARAM_INDIRECT) != 0;
  st = ct_restir_di(pc, P, 0, stream);
  if (st == CT_OK && indirect) st = ct_restir_pt(pc, P, 0, stream);
  if (st != CT_OK) return st;
  st = ct_restir_di(pc, P, 1, stream);
  if (st == CT_OK && indirect) st = ct_restir_pt(pc, P, 1, stream);
  if (st != CT_OK) return st;
  if (is_active & CT_TAA_BIT) st = ct_taa(pc, P, stream);
  return st;
}

// fork/join events of ct_render_views, per device (created on first use)
static std::mutex g_lane_mu;
static std::vector<std::vector<cudaEvent_t>> g_lane_events;

static ct_status lane_events(uint32_t n, cudaEvent_t **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_status(e);
  std::lock_guard<std::mutex> lk(g_lane_mu);
  if ((size_t)dev >= g_lane_events.size()) g_lane_events.resize(dev + 1);
  std::vector<cudaEvent_t> &v = g_lane_events[dev];
  while (v.size() < n) {
    cudaEvent_t ev;
    e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e != cudaSuccess) return cuda_status(e);
    v.push_back(ev);
  }
  *out = v.data();
  return CT_OK;
}

extern "C" ct_status ct_render_views(const ct_view *views, uint32_t n_views, const ct_stream *lanes, uint32_t n_lanes,
                                     ct_stream stream) {
  if (n_views == 0) return CT_OK;
  if (!views || n_lanes > CT_MAX_LANES || (n_lanes && !lanes)) return CT_ERR_INVALID_ARG;
  for (uint32_t i = 0; i < n_views; i++) {
    ct_status st = check_pc(&views[i].pc, true);
    if (st == CT_OK) st = check_params(&views[i].params);
    if (st != CT_OK) return st;
    if (n_lanes) {
      // side by side, every view needs its own scratch
      if (views[i].lane >= n_lanes || views[i].params.workspace_address == 0) return CT_ERR_INVALID_ARG;
      for (uint32_t j = 0; j < i; j++)
        if (views[j].params.workspace_address == views[i].params.workspace_address) return CT_ERR_INVALID_ARG;
    }
  }
  if (n_lanes == 0) {
    for (uint32_t i = 0; i < n_views; i++) {
      ct_status st = ct_render_frame(&views[i].pc, &views[i].params, views[i].is_active, stream);
      if (st != CT_OK) return st;
    }
    return CT_OK;
  }
  cudaEvent_t *ev = nullptr;
  ct_status st = lane_events(n_lanes + 1, &ev);
  if (st != CT_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaEventRecord(ev[n_lanes], s);
  for (uint32_t l = 0; l < n_lanes && e == cudaSuccess; l++) e = cudaStreamWaitEvent((cudaStream_t)lanes[l], ev[n_lanes], 0);
  if (e != cudaSuccess) return cuda_status(e);
  for (uint32_t i = 0; i < n_views; i++) {
    st = ct_render_frame(&views[i].pc, &views[i].params, views[i].is_active, lanes[views[i].lane]);
    if (st != CT_OK) return st;
  }
  for (uint32_t l = 0; l < n_lanes && e == cudaSuccess; l++) {
    e = cudaEventRecord(ev[l], (cudaStream_t)lanes[l]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s, ev[l], 0);
  }
  return cuda_status(e);
}

extern "C" ct_status ct_brush(const ct_push_constant *pc, ct_stream stream) {
  if (!pc || pc->size[0] == 0 || pc->size[1] == 0) return CT_ERR_INVALID_ARG;
  if (!pc->status_buffer || !pc->world_buffer || !pc->restir_buffer) return CT_ERR_INVALID_ARG;
  if ((pc->status_buffer | pc->world_buffer | pc->restir_buffer) & 7u) return CT_ERR_INVALID_ARG;
  return cuda_status(ct_launch_brush(*pc, (cudaStream_t)stream));
}

extern "C" ct_status ct_rearrange(const ct_push_constant *pc, uint32_t instance_count, uint32_t primitive_count,
                                  ct_stream stream) {
  if (!pc || !pc->status_buffer || !pc->world_buffer) return CT_ERR_INVALID_ARG;
  if ((pc->status_buffer | pc->world_buffer) & 7u) return CT_ERR_INVALID_ARG;
  if (instance_count == 0 || instance_count > CT_MAX_INSTANCES || primitive_count > CT_MAX_PRIMITIVES)
    return CT_ERR_INVALID_ARG;
  return cuda_status(ct_launch_rearrange(*pc, instance_count, primitive_count, (cudaStream_t)stream));
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

// ct_adjoint_forward / ct_adjoint_backward: argument checks (include/ct.h)
static ct_status check_adjoint(const ct_accel *accel, const ct_adjoint_desc *d, const float *albedo,
                               const float *emission) {
  if (!accel || !d || !albedo || d->struct_size != sizeof(ct_adjoint_desc)) return CT_ERR_INVALID_ARG;
  if (d->width == 0 || d->height == 0 || d->spp == 0 || d->spp > 65536u) return CT_ERR_INVALID_ARG;
  if (d->max_depth == 0 || d->max_depth > CT_ADJOINT_MAX_DEPTH) return CT_ERR_INVALID_ARG;
  if ((uint64_t)d->width * d->height > 0x10000000ull) return CT_ERR_CAPACITY;
  if (!d->camera_address || (d->camera_address & 3u) || !d->emitter_index_address) return CT_ERR_INVALID_ARG;
  if (d->emitter_count && !emission) return CT_ERR_INVALID_ARG;
  // every global primitive index of the structure must have a row
  if (d->primitive_count < accel->n_primitives) return CT_ERR_CAPACITY;
  if (d->rect[2] != 0) {
    const uint32_t *r = d->rect;
    if (r[0] >= r[2] || r[1] >= r[3] || r[2] > d->width || r[3] > d->height) return CT_ERR_INVALID_ARG;
  }
  return CT_OK;
}

extern "C" ct_status ct_adjoint_forward(const ct_accel *accel, const ct_adjoint_desc *desc, const float *albedo,
                                        const float *emission, void *image, ct_stream stream) {
  ct_status st = check_adjoint(accel, desc, albedo, emission);
  if (st != CT_OK) return st;
  if (!image) return CT_ERR_INVALID_ARG;
  return cuda_status(ct_launch_adjoint(accel->dev, *desc, albedo, emission, image, nullptr, nullptr, nullptr, 0,
                                       (cudaStream_t)stream));
}

extern "C" ct_status ct_nrc_trace(const ct_accel *accel, const ct_adjoint_desc *desc, const float *albedo,
                                  const float *emission, const ct_nrc_frame *f, ct_stream stream) {
  ct_status st = check_adjoint(accel, desc, albedo, emission);
  if (st != CT_OK) return st;
  if (!f || f->struct_size != sizeof(ct_nrc_frame) || !f->base_address || !f->query_address ||
      !f->throughput_address)
    return CT_ERR_INVALID_ARG;
  if ((f->base_address | f->throughput_address) & 3u || (f->query_address & 3u)) return CT_ERR_INVALID_ARG;
  if (f->cache_vertex < 1 || f->cache_vertex > 8 || f->_reserved) return CT_ERR_INVALID_ARG;
  if (f->train_paths) {
    if (f->train_bounces < 1 || f->train_bounces > 8 || f->train_paths > desc->width * desc->height ||
        !f->train_query_address || !f->train_partial_address || !f->train_throughput_address)
      return CT_ERR_INVALID_ARG;
  }
  if (!std::isfinite(desc->miss_radiance)) return CT_ERR_NAN_INPUT;
  return cuda_status(ct_launch_nrc_trace(accel->dev, *desc, albedo, emission, *f, (cudaStream_t)stream));
}

extern "C" ct_status ct_adjoint_backward(const ct_accel *accel, const ct_adjoint_desc *desc, const float *albedo,
                                         const float *emission, const float *d_image, float *d_albedo,
                                         float *d_emission, ct_stream stream) {
  ct_status st = check_adjoint(accel, desc, albedo, emission);
  if (st != CT_OK) return st;
  if (!d_image || !d_albedo || (desc->emitter_count && !d_emission)) return CT_ERR_INVALID_ARG;
  return cuda_status(ct_launch_adjoint(accel->dev, *desc, albedo, emission, nullptr, d_image, d_albedo, d_emission, 1,
                                       (cudaStream_t)stream));
}

extern "C" ct_status ct_trace_visibility(const ct_accel *accel, const ct_ray_query *q, uint32_t n, uint8_t *results,
                                         ct_stream stream) {
  if (!accel || (n && (!q || !results)) || ((uintptr_t)q & 3u)) return CT_ERR_INVALID_ARG;
  return cuda_status(ct_launch_queries(accel->dev, q, n, results, 0, (cudaStream_t)stream));
}

extern "C" ct_status ct_trace_closest(const ct_accel *accel, const ct_ray_query *q, uint32_t n, ct_ray_hit *results,
                                      ct_stream stream) {
  if (!accel || (n && (!q || !results)) || ((uintptr_t)q & 3u) || ((uintptr_t)results & 15u)) return CT_ERR_INVALID_ARG;
  return cuda_status(ct_launch_queries(accel->dev, q, n, results, 1, (cudaStream_t)stream));
}
