// ct_kernels.cuh -- launchers of the per-pixel frame kernels.
#pragma once
#include <cuda_runtime.h>
#include "ct_types.cuh"

cudaError_t ct_launch_trace(const ct_push_constant &pc, const DevAccel &A, const ct_params &P, cudaStream_t s);
cudaError_t ct_launch_di_initial(const ct_push_constant &pc, const DevAccel &A, const ct_params &P, cudaStream_t s);
cudaError_t ct_launch_di_shade(const ct_push_constant &pc, const DevAccel &A, const ct_params &P, int src_sel,
                               int final_pass, int dst_sel, cudaStream_t s);
cudaError_t ct_launch_taa(const ct_push_constant &pc, const ct_params &P, cudaStream_t s);
cudaError_t ct_error_word_read(uint32_t *w, int reset, cudaStream_t s);
