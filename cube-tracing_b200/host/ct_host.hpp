// ct_host.hpp -- C++ host side of the hot path over the C ABI of include/ct.h.
//
// cube-tracing's host is C++: App keeps the scene and per-pixel buffers
// (src/main.cpp:96-120), fills the WORLD / RESTIR address tables
// (upload_world / upload_restir, main.cpp:560-608, 983-1004) and records one
// frame in App::draw (main.cpp:1436-1703): camera and Status upload, the
// ray-tracing passes, TAA, the swap of the output images.  ct::Renderer is
// that host side for libct: it owns the same buffers in the same layouts,
// uploads the same per-frame state and calls ct_render_frame where App::draw
// records its passes.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

#include "ct.h"

namespace ct {

// A scene as the reference's loaders leave it on the host (the .vox loader,
// map_loader.cpp:106-327; load_materials / load_lights, main.cpp:383-440).
struct Scene {
  std::vector<ct_instance> instances;
  std::vector<ct_primitive> primitives;
  std::vector<ct_aabb> aabbs;
  std::vector<ct_material> materials;
  std::vector<ct_light> point_lights, cube_lights, env_lights;
  ct_light_config light_config{};
  float voxel_extent = 1.0f;
};

// The per-view switches App keeps in Status (shared.inl:73-79, main.cpp:1489-1524).
struct FrameOptions {
  uint32_t width = 0, height = 0;
  uint32_t features = CT_RIS_CUBE_LIGHT_BIT;  // Status.is_active feature bits
  uint32_t max_depth = 3;                     // Status.max_depth (PT)
  bool taa = true;                            // TAA from the second frame on
  float sky_time = 1.0f;                      // Status.time
  uint32_t is_afternoon = 1;                  // Status.is_afternoon
};

// The RESTIR table's buffers, in the table's order.
enum RestirBuffer : int {
  kPreviousReservoir = 0, kIntermediateReservoir, kReservoir, kPreviousDi, kDi, kVelocity,
  kOutputPathReservoir, kTemporalPathReservoir, kIndirectColor, kRestirBufferCount
};

class Renderer {
 public:
  // Uploads the scene, builds the acceleration structure and allocates the
  // per-pixel state on `stream`.  status() reports how that went; a
  // Renderer whose status() is not CT_OK renders nothing.
  Renderer(const Scene &scene, const FrameOptions &options, const ct_params &params, cudaStream_t stream = nullptr);
  ~Renderer();
  Renderer(const Renderer &) = delete;
  Renderer &operator=(const Renderer &) = delete;

  ct_status status() const { return status_; }

  // One frame with the camera's inverse view and projection matrices
  // (column major, Vulkan y flip already in inv_proj as main.cpp:1460 does),
  // recorded on the stream; returns after the calls are enqueued.
  ct_status render(const float inv_view[16], const float inv_proj[16]);

  uint32_t frame() const { return frame_; }                // frames rendered so far
  const float *output() const;                              // device RGBA32F image of the last frame
  ct_status read_output(float *host) const;                 // width*height*4 floats; waits for the stream
  ct_status read_buffer(RestirBuffer which, void *host, size_t bytes) const;  // waits for the stream
  static size_t record_bytes(RestirBuffer which);           // bytes per pixel of a RESTIR buffer

 private:
  ct_status setup(const Scene &scene);
  void *alloc(size_t bytes);
  ct_status upload(void *dst, const void *src, size_t bytes);
  ct_push_constant push_constant() const;

  FrameOptions opt_;
  ct_params params_;
  cudaStream_t stream_;
  ct_status status_ = CT_OK;
  std::vector<void *> owned_;                 // every device allocation
  ct_accel *accel_ = nullptr;
  uint32_t obj_count_ = 0;
  void *light_config_ = nullptr, *world_ = nullptr, *restir_ = nullptr, *camera_ = nullptr, *status_block_ = nullptr;
  void *restir_buf_[kRestirBufferCount] = {};
  float *images_[2] = {nullptr, nullptr};
  float *taa_frame_ = nullptr, *taa_prev_ = nullptr;
  // pinned staging of the per-frame camera + Status upload; a slot is
  // reused only after the copy that read it has completed
  static constexpr int kSlots = 4;
  unsigned char *staging_ = nullptr;
  cudaEvent_t slot_done_[kSlots] = {};
  bool slot_used_[kSlots] = {};
  uint32_t frame_ = 0;
  float prev_view_[16] = {}, prev_proj_[16] = {};
};

}  // namespace ct
