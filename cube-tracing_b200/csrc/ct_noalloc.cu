// ct_noalloc.cu -- ct_restir_di_static: ReSTIR DI with library-resident
// scratch, for callers that cannot allocate device memory.
//
// ct_restir_di needs scratch memory (the shadow-ray queue, one answer byte
// and one radiance per shadow-ray call site, the chosen neighbours).  It
// takes it from ct_params.workspace_address or grows a buffer with
// cudaMalloc.  Some hosts cannot do either at frame time: engines that hand
// out device memory only from a fixed arena set up at start, callers that
// may not introduce the device-wide synchronisation cudaMalloc can cause,
// or plug-in hosts that own all allocations themselves.  This entry point
// runs the same kernels with the scratch carved from a fixed array compiled
// into the library, and calls no allocating routine.
//
// Limits and sharing:
//  * the array holds CT_STATIC_WORKSPACE_BYTES; frames whose scratch
//    (ct_workspace_size) exceeds it are rejected with CT_ERR_CAPACITY;
//  * every GPU that loads the library holds the array until the process
//    exits;
//  * all calls share the one array and it keeps the previous call's
//    contents: the queue counters are cleared on the stream before each use,
//    and nothing else is read before it is written.  Calls that overlap on
//    the GPU (other streams, other host threads) race on it; order them on
//    one stream;
//  * the first call on a device looks up the array's device address for
//    that device (cudaGetSymbolAddress, with the device current); make that
//    first call before capturing the stream into a graph.
#include <cuda_runtime.h>
#include <mutex>
#include "ct_accel.cuh"
#include "ct_kernels.cuh"

static __device__ __align__(256) unsigned char g_ct_static_workspace[CT_STATIC_WORKSPACE_BYTES];

ct_status check_pc(const ct_push_constant *pc, bool needs_accel);
ct_status check_params(const ct_params *P);
ct_status check_extent(const ct_push_constant *pc, const ct_params *P);
ct_status cuda_status(cudaError_t e);
uint64_t workspace_bytes(uint32_t W, uint32_t H, const ct_params *P, uint64_t *cap_out);
CtWorkspace carve_workspace(void *base, uint32_t W, uint32_t H, const ct_params *P);
DevAccel walk_accel(const ct_accel *a, const ct_params *P);

#define CT_MAX_DEVICES 64
static std::mutex g_static_mu;
static void *g_static_ptr[CT_MAX_DEVICES];

// device address of the array on the current device (looked up once per device)
static ct_status static_workspace(void **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_status(e);
  if (dev < 0 || dev >= CT_MAX_DEVICES) return CT_ERR_CAPACITY;
  std::lock_guard<std::mutex> lk(g_static_mu);
  if (!g_static_ptr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_ct_static_workspace);
    if (e != cudaSuccess) return cuda_status(e);
    g_static_ptr[dev] = p;
  }
  *out = g_static_ptr[dev];
  return CT_OK;
}

extern "C" ct_status ct_restir_di_static(const ct_push_constant *pc, const ct_params *P, int stage, ct_stream stream) {
  ct_status st = check_pc(pc, true);
  if (st == CT_OK) st = check_params(P);
  if (st != CT_OK) return st;
  if (stage != 0 && stage != 1) return CT_ERR_INVALID_ARG;
  // the DI scratch only.  With CT_PARAM_INDIRECT, ct_restir_pt keeps its own
  // workspace: every stage of either entry point writes its scratch before
  // reading it within the call, so the two need not share memory.
  ct_params Q = *P;
  Q.flags &= ~CT_PARAM_INDIRECT;
  if (workspace_bytes(pc->size[0], pc->size[1], &Q, nullptr) > (uint64_t)CT_STATIC_WORKSPACE_BYTES)
    return CT_ERR_CAPACITY;
  st = check_extent(pc, P);
  if (st != CT_OK) return st;
  void *base = nullptr;
  st = static_workspace(&base);
  if (st != CT_OK) return st;
  const CtWorkspace w = carve_workspace(base, pc->size[0], pc->size[1], &Q);
  cudaStream_t s = (cudaStream_t)stream;
  // the walk cap of P applies to both scenes, as in ct_restir_di
  const DevAccel A = walk_accel(pc->tlas, P);
  const DevAccel A_prev = pc->tlas_previous ? walk_accel(pc->tlas_previous, P) : A;
  if (stage == 0) return cuda_status(ct_launch_di_stage0(*pc, A, A_prev, *P, w, s));
  for (uint32_t r = 0; r + 1 < P->spatial_passes; r++) {
    cudaError_t e = ct_launch_spatial_round(*pc, A, *P, w, (int)(r & 1u), 0, (int)((r & 1u) ^ 1u), s);
    if (e != cudaSuccess) return cuda_status(e);
  }
  return cuda_status(ct_launch_spatial_round(*pc, A, *P, w, (int)((P->spatial_passes - 1) & 1u), 1, 0, s));
}
