// ct_host.cpp -- ct::Renderer, the C++ host side over include/ct.h (see
// ct_host.hpp).  Host code only; every device call is stream ordered.
#include "ct_host.hpp"

#include <algorithm>
#include <cstring>

namespace ct {

namespace {
constexpr size_t kRecord[kRestirBufferCount] = {
    sizeof(ct_reservoir), sizeof(ct_reservoir),      sizeof(ct_reservoir),      sizeof(ct_di_info),
    sizeof(ct_di_info),   sizeof(ct_velocity),       sizeof(ct_path_reservoir), sizeof(ct_path_reservoir),
    3 * sizeof(float)};
constexpr size_t kStage = sizeof(ct_camera_view) + sizeof(ct_status_block);

template <class T>
const void *data_or_one(const std::vector<T> &v, T &one) {
  // an empty buffer is uploaded as one zero record, as the reference's
  // fixed-capacity buffers always exist
  if (!v.empty()) return v.data();
  memset(&one, 0, sizeof(T));
  return &one;
}
}  // namespace

size_t Renderer::record_bytes(RestirBuffer which) { return which < kRestirBufferCount ? kRecord[which] : 0; }

void *Renderer::alloc(size_t bytes) {
  void *p = nullptr;
  if (cudaMalloc(&p, bytes ? bytes : 1) != cudaSuccess) return nullptr;
  owned_.push_back(p);
  return p;
}

ct_status Renderer::upload(void *dst, const void *src, size_t bytes) {
  if (!dst) return CT_ERR_CUDA;
  if (cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream_) != cudaSuccess) return CT_ERR_CUDA;
  return CT_OK;
}

Renderer::Renderer(const Scene &scene, const FrameOptions &options, const ct_params &params, cudaStream_t stream)
    : opt_(options), params_(params), stream_(stream) {
  status_ = setup(scene);
}

ct_status Renderer::setup(const Scene &sc) {
  if (opt_.width == 0 || opt_.height == 0 || sc.instances.empty() || sc.aabbs.empty()) return CT_ERR_INVALID_ARG;
  if (sc.primitives.size() != sc.aabbs.size()) return CT_ERR_INVALID_ARG;
  const size_t n = (size_t)opt_.width * opt_.height;
  obj_count_ = (uint32_t)sc.aabbs.size();

  // scene buffers and the WORLD table (upload_world, main.cpp:560-608)
  ct_instance i1;
  ct_primitive p1;
  ct_aabb a1;
  ct_material m1;
  ct_light l1, l2, l3;
  struct Buf { const void *src; size_t bytes; void *dev = nullptr; };
  Buf bufs[] = {
      {data_or_one(sc.instances, i1), std::max<size_t>(sc.instances.size(), 1) * sizeof(ct_instance)},
      {data_or_one(sc.primitives, p1), std::max<size_t>(sc.primitives.size(), 1) * sizeof(ct_primitive)},
      {data_or_one(sc.aabbs, a1), std::max<size_t>(sc.aabbs.size(), 1) * sizeof(ct_aabb)},
      {data_or_one(sc.materials, m1), std::max<size_t>(sc.materials.size(), 1) * sizeof(ct_material)},
      {data_or_one(sc.point_lights, l1), std::max<size_t>(sc.point_lights.size(), 1) * sizeof(ct_light)},
      {data_or_one(sc.cube_lights, l2), std::max<size_t>(sc.cube_lights.size(), 1) * sizeof(ct_light)},
      {data_or_one(sc.env_lights, l3), std::max<size_t>(sc.env_lights.size(), 1) * sizeof(ct_light)},
  };
  for (Buf &b : bufs) {
    b.dev = alloc(b.bytes);
    if (upload(b.dev, b.src, b.bytes) != CT_OK) return CT_ERR_CUDA;
  }
  // remap tables of the scene edits, zero outside the frame after an edit
  void *remap_p = alloc(std::max<size_t>(sc.aabbs.size(), 1) * 4);
  void *remap_l = alloc(std::max<size_t>(sc.cube_lights.size(), 1) * 4);
  if (!remap_p || !remap_l) return CT_ERR_CUDA;
  if (cudaMemsetAsync(remap_p, 0, std::max<size_t>(sc.aabbs.size(), 1) * 4, stream_) != cudaSuccess ||
      cudaMemsetAsync(remap_l, 0, std::max<size_t>(sc.cube_lights.size(), 1) * 4, stream_) != cudaSuccess)
    return CT_ERR_CUDA;
  light_config_ = alloc(sizeof(ct_light_config));
  if (upload(light_config_, &sc.light_config, sizeof(ct_light_config)) != CT_OK) return CT_ERR_CUDA;
  ct_world w;
  w.instance_address = w.instance_address_prev = (uint64_t)(uintptr_t)bufs[0].dev;
  w.primitive_address = w.primitive_address_prev = (uint64_t)(uintptr_t)bufs[1].dev;
  w.aabb_address = w.aabb_address_prev = (uint64_t)(uintptr_t)bufs[2].dev;
  w.remapped_primitive_address = (uint64_t)(uintptr_t)remap_p;
  w.remapped_cube_light_address = (uint64_t)(uintptr_t)remap_l;
  w.material_address = (uint64_t)(uintptr_t)bufs[3].dev;
  w.point_light_address = (uint64_t)(uintptr_t)bufs[4].dev;
  w.cube_light_address = (uint64_t)(uintptr_t)bufs[5].dev;
  w.env_light_address = (uint64_t)(uintptr_t)bufs[6].dev;
  world_ = alloc(sizeof(w));
  if (upload(world_, &w, sizeof(w)) != CT_OK) return CT_ERR_CUDA;

  // per-pixel state and the RESTIR table (upload_restir, main.cpp:983-1004)
  ct_restir r;
  uint64_t *addr = &r.previous_reservoir_address;
  for (int i = 0; i < kRestirBufferCount; i++) {
    restir_buf_[i] = alloc(kRecord[i] * n);
    if (!restir_buf_[i] || cudaMemsetAsync(restir_buf_[i], 0, kRecord[i] * n, stream_) != cudaSuccess)
      return CT_ERR_CUDA;
    addr[i] = (uint64_t)(uintptr_t)restir_buf_[i];
  }
  restir_ = alloc(sizeof(r));
  if (upload(restir_, &r, sizeof(r)) != CT_OK) return CT_ERR_CUDA;
  float **imgs[4] = {&images_[0], &images_[1], &taa_frame_, &taa_prev_};
  for (float **im : imgs) {
    *im = (float *)alloc(16 * n);
    if (!*im || cudaMemsetAsync(*im, 0, 16 * n, stream_) != cudaSuccess) return CT_ERR_CUDA;
  }
  camera_ = alloc(sizeof(ct_camera_view));
  status_block_ = alloc(sizeof(ct_status_block));
  if (!camera_ || !status_block_) return CT_ERR_CUDA;

  // the acceleration structure (build_blases / build_tlas)
  ct_scene_desc d;
  memset(&d, 0, sizeof(d));
  d.instance_address = (uint64_t)(uintptr_t)bufs[0].dev;
  d.instance_count = (uint32_t)sc.instances.size();
  d.aabb_address = (uint64_t)(uintptr_t)bufs[2].dev;
  d.aabb_count = (uint32_t)sc.aabbs.size();
  d.voxel_extent = sc.voxel_extent;
  ct_status st = ct_build_accel(&d, &accel_, (ct_stream)stream_);
  if (st != CT_OK) return st;

  // the view's own scratch, so that no call allocates at frame time
  uint64_t ws = 0;
  if ((st = ct_workspace_size(opt_.width, opt_.height, &params_, &ws)) != CT_OK) return st;
  void *wsp = alloc(ws + 256);
  if (!wsp) return CT_ERR_CUDA;
  params_.workspace_address = ((uint64_t)(uintptr_t)wsp + 255u) & ~255ull;
  params_.workspace_bytes = ws;

  if (cudaMallocHost((void **)&staging_, kStage * kSlots) != cudaSuccess) return CT_ERR_CUDA;
  for (int i = 0; i < kSlots; i++)
    if (cudaEventCreateWithFlags(&slot_done_[i], cudaEventDisableTiming) != cudaSuccess) return CT_ERR_CUDA;
  return cudaStreamSynchronize(stream_) == cudaSuccess ? CT_OK : CT_ERR_CUDA;
}

Renderer::~Renderer() {
  cudaStreamSynchronize(stream_);
  if (accel_) ct_accel_free(accel_);
  for (int i = 0; i < kSlots; i++)
    if (slot_done_[i]) cudaEventDestroy(slot_done_[i]);
  if (staging_) cudaFreeHost(staging_);
  for (void *p : owned_) cudaFree(p);
}

ct_push_constant Renderer::push_constant() const {
  // App swaps its two output images every frame; the first frame has no
  // previous image and reads its own
  ct_push_constant pc;
  memset(&pc, 0, sizeof(pc));
  pc.size[0] = opt_.width;
  pc.size[1] = opt_.height;
  pc.tlas = pc.tlas_previous = accel_;
  pc.swapchain = images_[frame_ % 2];
  pc.previous_swapchain = frame_ > 0 ? images_[(frame_ + 1) % 2] : images_[frame_ % 2];
  pc.taa_frame = taa_frame_;
  pc.taa_prev_frame = taa_prev_;
  pc.camera_buffer = (uint64_t)(uintptr_t)camera_;
  pc.status_buffer = (uint64_t)(uintptr_t)status_block_;
  pc.world_buffer = (uint64_t)(uintptr_t)world_;
  pc.restir_buffer = (uint64_t)(uintptr_t)restir_;
  return pc;
}

ct_status Renderer::render(const float inv_view[16], const float inv_proj[16]) {
  if (status_ != CT_OK) return status_;
  if (!inv_view || !inv_proj) return CT_ERR_INVALID_ARG;
  // camera_view with the previous frame's matrices (the first frame
  // reprojects onto itself)
  ct_camera_view cam;
  memset(&cam, 0, sizeof(cam));
  memcpy(cam.inv_view, inv_view, sizeof(cam.inv_view));
  memcpy(cam.inv_proj, inv_proj, sizeof(cam.inv_proj));
  memcpy(cam.prev_inv_view, frame_ > 0 ? prev_view_ : inv_view, sizeof(cam.prev_inv_view));
  memcpy(cam.prev_inv_proj, frame_ > 0 ? prev_proj_ : inv_proj, sizeof(cam.prev_inv_proj));
  // Status (shared.inl:171-189) as App::draw sets it for the frame
  ct_status_block s;
  memset(&s, 0, sizeof(s));
  s.resolution[0] = opt_.width;
  s.resolution[1] = opt_.height;
  s.frame_number = frame_;
  s.is_active = opt_.features | ((opt_.taa && frame_ > 0) ? CT_TAA_BIT : 0u);
  s.light_config_address = (uint64_t)(uintptr_t)light_config_;
  s.obj_count = obj_count_;
  s.time = opt_.sky_time;
  s.is_afternoon = opt_.is_afternoon;
  s.max_depth = opt_.max_depth;
  const int slot = (int)(frame_ % kSlots);
  if (slot_used_[slot] && cudaEventSynchronize(slot_done_[slot]) != cudaSuccess) return CT_ERR_CUDA;
  unsigned char *st = staging_ + (size_t)slot * kStage;
  memcpy(st, &cam, sizeof(cam));
  memcpy(st + sizeof(cam), &s, sizeof(s));
  if (cudaMemcpyAsync(camera_, st, sizeof(cam), cudaMemcpyHostToDevice, stream_) != cudaSuccess ||
      cudaMemcpyAsync(status_block_, st + sizeof(cam), sizeof(s), cudaMemcpyHostToDevice, stream_) != cudaSuccess ||
      cudaEventRecord(slot_done_[slot], stream_) != cudaSuccess)
    return CT_ERR_CUDA;
  slot_used_[slot] = true;
  const ct_push_constant pc = push_constant();
  const ct_status r = ct_render_frame(&pc, &params_, s.is_active, (ct_stream)stream_);
  if (r != CT_OK) return r;
  memcpy(prev_view_, inv_view, sizeof(prev_view_));
  memcpy(prev_proj_, inv_proj, sizeof(prev_proj_));
  frame_++;
  return CT_OK;
}

const float *Renderer::output() const {
  if (frame_ == 0) return nullptr;
  return images_[(frame_ - 1) % 2];
}

ct_status Renderer::read_output(float *host) const {
  const float *img = output();
  if (!host || !img) return CT_ERR_INVALID_ARG;
  const size_t bytes = (size_t)opt_.width * opt_.height * 16;
  if (cudaMemcpyAsync(host, img, bytes, cudaMemcpyDeviceToHost, stream_) != cudaSuccess ||
      cudaStreamSynchronize(stream_) != cudaSuccess)
    return CT_ERR_CUDA;
  return CT_OK;
}

ct_status Renderer::read_buffer(RestirBuffer which, void *host, size_t bytes) const {
  if (which < 0 || which >= kRestirBufferCount || !host || !restir_buf_[which]) return CT_ERR_INVALID_ARG;
  if (bytes != kRecord[which] * (size_t)opt_.width * opt_.height) return CT_ERR_INVALID_ARG;
  if (cudaMemcpyAsync(host, restir_buf_[which], bytes, cudaMemcpyDeviceToHost, stream_) != cudaSuccess ||
      cudaStreamSynchronize(stream_) != cudaSuccess)
    return CT_ERR_CUDA;
  return CT_OK;
}

}  // namespace ct
