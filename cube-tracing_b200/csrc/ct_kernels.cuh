// ct_kernels.cuh -- launchers of the per-pixel frame kernels.
#pragma once
#include <cuda_runtime.h>
#include "ct_types.cuh"

cudaError_t ct_launch_trace(const ct_push_constant &pc, const DevAccel &A, const ct_params &P, cudaStream_t s);
// Scratch of the wavefront ReSTIR passes, carved from one allocation
// (see ct_workspace_size): the shadow-ray queue and one answer byte per
// (pixel, call site).
// bytes of one pixel's path state in the ReSTIR PT workspace
#define CT_PT_STATE_BYTES 256u
// wavefront rounds of the path tracer (paths end within max_depth rounds)
#define CT_PT_MAX_ITER 16
struct CtWorkspace {
  void *pt_state, *pt_hit, *pt_q[2];  // ReSTIR PT (CT_PARAM_INDIRECT only)
  void *pt_replay, *pt_jobs;          // hybrid shift: 2 replay results (64 B) and 2 job slots (4 B) per pixel
  uint32_t pt_capacity;
  uint32_t *counter;
  void *ray_a, *ray_b, *ray_c;
  uint32_t capacity;
  uint8_t *vis;
  float *rad;
  uint32_t *nbr;
  void *smeta;
};
// A_prev: the scene of pc.tlas_previous (previous-frame visibility of
// temporal reuse with CT_REMAP_BIT)
cudaError_t ct_launch_di_stage0(const ct_push_constant &pc, const DevAccel &A, const DevAccel &A_prev,
                                const ct_params &P, const CtWorkspace &w, cudaStream_t s);
cudaError_t ct_launch_spatial_round(const ct_push_constant &pc, const DevAccel &A, const ct_params &P,
                                    const CtWorkspace &w, int src_sel, int final_pass, int dst_sel, cudaStream_t s);
cudaError_t ct_launch_taa(const ct_push_constant &pc, const ct_params &P, cudaStream_t s);
cudaError_t ct_launch_pt(const ct_push_constant &pc, const DevAccel &A, const ct_params &P, const CtWorkspace &w,
                         int stage, cudaStream_t s);
cudaError_t ct_launch_brush(const ct_push_constant &pc, cudaStream_t s);
cudaError_t ct_launch_rearrange(const ct_push_constant &pc, uint32_t instance_count, uint32_t primitive_count,
                                cudaStream_t s);
cudaError_t ct_error_word_read(uint32_t *w, int reset, cudaStream_t s);
cudaError_t ct_launch_queries(const DevAccel &A, const ct_ray_query *q, uint32_t n, void *out, int closest,
                              cudaStream_t s);
// ct_adjoint_forward (backward = 0) / ct_adjoint_backward (backward = 1)
cudaError_t ct_launch_adjoint(const DevAccel &A, const ct_adjoint_desc &d, const float *albedo, const float *emission,
                              void *image, const float *d_image, float *d_albedo, float *d_emission, int backward,
                              cudaStream_t s);
// ct_nrc_trace
cudaError_t ct_launch_nrc_trace(const DevAccel &A, const ct_adjoint_desc &d, const float *albedo,
                                const float *emission, const ct_nrc_frame &f, cudaStream_t s);
