// ct_state.cu -- ct_state_size / ct_state_save / ct_state_load: the frame
// history as one blob (include/ct.h).  Host code only: header, then the
// thirteen sections copied with cudaMemcpyAsync in the layout the buffers
// have.  The reference has no counterpart; its history lives only in the
// GPU buffers of App (main.cpp:96-120).
#include <cuda_runtime.h>
#include <cstring>
#include "ct_accel.cuh"
#include "ct_kernels.cuh"

ct_status cuda_status(cudaError_t e);

namespace {

struct StateHeader {
  uint32_t magic, version, width, height, sections, reserved;
  uint64_t bytes[CT_STATE_SECTIONS];
};
static_assert(sizeof(StateHeader) == CT_STATE_HEADER_BYTES, "state header is 128 bytes");

// bytes per pixel of each section, in blob order
constexpr uint64_t kRecord[CT_STATE_SECTIONS] = {
    sizeof(ct_reservoir), sizeof(ct_reservoir), sizeof(ct_reservoir), sizeof(ct_di_info), sizeof(ct_di_info),
    sizeof(ct_velocity),  sizeof(ct_path_reservoir), sizeof(ct_path_reservoir), 3 * sizeof(float),
    4 * sizeof(float),    4 * sizeof(float), 4 * sizeof(float), 4 * sizeof(float)};

bool pixels(uint32_t w, uint32_t h, uint64_t &n) {
  n = (uint64_t)w * h;
  return w != 0 && h != 0 && n <= 0xFFFFFFFFull;
}

// the device addresses of the sections: the RESTIR table's buffers (read
// from the device) and the push constant's images
ct_status section_pointers(const ct_push_constant *pc, cudaStream_t s, uint64_t ptr[CT_STATE_SECTIONS]) {
  if (!pc || !pc->restir_buffer || (pc->restir_buffer & 7u)) return CT_ERR_INVALID_ARG;
  if (!pc->swapchain || !pc->previous_swapchain || !pc->taa_frame || !pc->taa_prev_frame) return CT_ERR_INVALID_ARG;
  ct_restir r;
  cudaError_t e = cudaMemcpyAsync(&r, (const void *)(uintptr_t)pc->restir_buffer, sizeof(r), cudaMemcpyDefault, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_status(e);
  const uint64_t p[CT_STATE_SECTIONS] = {
      r.previous_reservoir_address, r.intermediate_reservoir_address, r.reservoir_address,
      r.previous_di_address, r.di_address, r.velocity_address, r.output_path_reservoir_address,
      r.temporal_path_reservoir_address, r.indirect_color_address, (uint64_t)(uintptr_t)pc->swapchain,
      (uint64_t)(uintptr_t)pc->previous_swapchain, (uint64_t)(uintptr_t)pc->taa_frame,
      (uint64_t)(uintptr_t)pc->taa_prev_frame};
  for (uint32_t i = 0; i < CT_STATE_SECTIONS; i++) {
    if (!p[i]) return CT_ERR_INVALID_ARG;
    ptr[i] = p[i];
  }
  return CT_OK;
}

}  // namespace

extern "C" ct_status ct_state_size(uint32_t width, uint32_t height, uint64_t *out_bytes) {
  uint64_t n;
  if (!out_bytes) return CT_ERR_INVALID_ARG;
  if (!pixels(width, height, n)) return width && height ? CT_ERR_CAPACITY : CT_ERR_INVALID_ARG;
  uint64_t b = CT_STATE_HEADER_BYTES;
  for (uint32_t i = 0; i < CT_STATE_SECTIONS; i++) b += kRecord[i] * n;
  *out_bytes = b;
  return CT_OK;
}

extern "C" ct_status ct_state_save(const ct_push_constant *pc, void *blob, uint64_t bytes, ct_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  uint64_t need = 0, n = 0;
  if (!pc || !blob) return CT_ERR_INVALID_ARG;
  ct_status st = ct_state_size(pc->size[0], pc->size[1], &need);
  if (st != CT_OK) return st;
  if (bytes != need) return CT_ERR_INVALID_ARG;
  pixels(pc->size[0], pc->size[1], n);
  uint64_t ptr[CT_STATE_SECTIONS];
  if ((st = section_pointers(pc, s, ptr)) != CT_OK) return st;
  StateHeader h;
  memset(&h, 0, sizeof(h));
  h.magic = CT_STATE_MAGIC;
  h.version = CT_STATE_VERSION;
  h.width = pc->size[0];
  h.height = pc->size[1];
  h.sections = CT_STATE_SECTIONS;
  for (uint32_t i = 0; i < CT_STATE_SECTIONS; i++) h.bytes[i] = kRecord[i] * n;
  char *out = (char *)blob;
  cudaError_t e = cudaMemcpyAsync(out, &h, sizeof(h), cudaMemcpyDefault, s);
  uint64_t off = sizeof(h);
  for (uint32_t i = 0; i < CT_STATE_SECTIONS && e == cudaSuccess; i++) {
    e = cudaMemcpyAsync(out + off, (const void *)(uintptr_t)ptr[i], h.bytes[i], cudaMemcpyDefault, s);
    off += h.bytes[i];
  }
  // the header copy reads this stack frame: wait before returning
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return cuda_status(e);
}

extern "C" ct_status ct_state_load(const ct_push_constant *pc, const void *blob, uint64_t bytes, ct_stream stream) {
  cudaStream_t s = (cudaStream_t)stream;
  uint64_t need = 0, n = 0;
  if (!pc || !blob) return CT_ERR_INVALID_ARG;
  ct_status st = ct_state_size(pc->size[0], pc->size[1], &need);
  if (st != CT_OK) return st;
  if (bytes != need) return CT_ERR_INVALID_ARG;
  pixels(pc->size[0], pc->size[1], n);
  uint64_t ptr[CT_STATE_SECTIONS];
  if ((st = section_pointers(pc, s, ptr)) != CT_OK) return st;
  StateHeader h;
  cudaError_t e = cudaMemcpyAsync(&h, blob, sizeof(h), cudaMemcpyDefault, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_status(e);
  if (h.magic != CT_STATE_MAGIC || h.version != CT_STATE_VERSION || h.width != pc->size[0] ||
      h.height != pc->size[1] || h.sections != CT_STATE_SECTIONS)
    return CT_ERR_INVALID_ARG;
  for (uint32_t i = 0; i < CT_STATE_SECTIONS; i++)
    if (h.bytes[i] != kRecord[i] * n) return CT_ERR_INVALID_ARG;
  const char *in = (const char *)blob;
  uint64_t off = sizeof(h);
  for (uint32_t i = 0; i < CT_STATE_SECTIONS && e == cudaSuccess; i++) {
    e = cudaMemcpyAsync((void *)(uintptr_t)ptr[i], in + off, h.bytes[i], cudaMemcpyDefault, s);
    off += h.bytes[i];
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return cuda_status(e);
}
