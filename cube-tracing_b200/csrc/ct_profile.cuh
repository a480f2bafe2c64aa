// ct_profile.cuh -- per-kernel CUDA-event timing behind ct_profile_enable /
// ct_profile_read.  Off by default; when on, every kernel launch of the
// library is bracketed by two events recorded on the launching stream, and
// ct_profile_read waits for them and sums the elapsed times per kernel.
#pragma once
#include <cuda_runtime.h>

enum CtKernelId {
  CT_K_TRACE_PRIMARY = 0,
  CT_K_DI_GEN0,
  CT_K_DI_GEN1,
  CT_K_DI_RESOLVE0,
  CT_K_SPATIAL_SELECT,
  CT_K_SPATIAL_SAMPLE,
  CT_K_SPATIAL_RESOLVE,
  CT_K_TRACE_SHADOW,
  CT_K_TAA,
  CT_K_QUERIES,
  CT_K_PT_START,
  CT_K_PT_EXTEND,
  CT_K_PT_SHADE,
  CT_K_PT_TEMPORAL,
  CT_K_PT_SPATIAL,
  CT_K_EDIT,
  CT_K_PT_FINISH,
  CT_K_TRACE_PREV,
  CT_K_ADJOINT_FORWARD,
  CT_K_ADJOINT_BACKWARD,
  CT_K_PT_REPLAY,
  CT_K_NRC_ENCODE,
  CT_K_NRC_MLP,
  CT_K_NRC_TRACE,
  CT_K_COUNT
};

extern const char *const ct_kernel_names[CT_K_COUNT];

bool ct_profile_on();
// records the start event; returns a token for ct_profile_end (-1 when off)
int ct_profile_begin(int kernel, cudaStream_t s);
void ct_profile_end(int token, cudaStream_t s);

// brackets one launch statement
#define CT_TIMED(kid, stream, ...)                       \
  do {                                                   \
    const int ct_tok_ = ct_profile_begin((kid), (stream)); \
    __VA_ARGS__;                                         \
    ct_profile_end(ct_tok_, (stream));                   \
  } while (0)
