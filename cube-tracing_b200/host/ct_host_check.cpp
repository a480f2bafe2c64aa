// ct_host_check.cpp -- runs ct::Renderer on a scene and camera path read
// from a file and writes the last frame's image and per-pixel buffers, so
// that tests can compare the C++ host side with the Python one on the same
// inputs.
//
//   ct_host_check <input> <output>
//
// input (little endian): "CTHI", u32 width, height, frames, features,
// max_depth, taa, is_afternoon; f32 sky_time, voxel_extent; u32 counts of
// instances, primitives, aabbs, materials, point, cube and env lights; u32
// sizeof(ct_params) and the ct_params; ct_light_config; the seven arrays;
// frames x (inv_view[16], inv_proj[16]).
// output: "CTHO", u32 width, height, then the RGBA32F image and the nine
// RESTIR buffers in table order.
#include <cstdio>
#include <cstring>
#include <vector>

#include "ct_host.hpp"

namespace {
struct Reader {
  FILE *f;
  bool ok = true;
  template <class T> void get(T &v) { ok = ok && fread(&v, sizeof(T), 1, f) == 1; }
  template <class T> void get(std::vector<T> &v, uint32_t n) {
    v.resize(n);
    if (n) ok = ok && fread(v.data(), sizeof(T), n, f) == n;
  }
};
}  // namespace

int main(int argc, char **argv) {
  if (argc != 3) {
    fprintf(stderr, "usage: %s <input> <output>\n", argv[0]);
    return 2;
  }
  FILE *in = fopen(argv[1], "rb");
  if (!in) return 2;
  Reader r{in};
  char magic[4];
  r.ok = fread(magic, 1, 4, in) == 4 && memcmp(magic, "CTHI", 4) == 0;
  ct::FrameOptions opt;
  uint32_t frames = 0, taa = 0, counts[7] = {}, psize = 0;
  float voxel_extent = 1.0f;
  r.get(opt.width); r.get(opt.height); r.get(frames); r.get(opt.features); r.get(opt.max_depth); r.get(taa);
  r.get(opt.is_afternoon); r.get(opt.sky_time); r.get(voxel_extent);
  for (uint32_t &c : counts) r.get(c);
  r.get(psize);
  ct_params params;
  if (!r.ok || psize != sizeof(ct_params)) {
    fprintf(stderr, "bad input header\n");
    return 2;
  }
  r.get(params);
  ct::Scene sc;
  sc.voxel_extent = voxel_extent;
  r.get(sc.light_config);
  r.get(sc.instances, counts[0]);
  r.get(sc.primitives, counts[1]);
  r.get(sc.aabbs, counts[2]);
  r.get(sc.materials, counts[3]);
  r.get(sc.point_lights, counts[4]);
  r.get(sc.cube_lights, counts[5]);
  r.get(sc.env_lights, counts[6]);
  std::vector<float> cams;
  r.get(cams, frames * 32u);
  fclose(in);
  if (!r.ok) {
    fprintf(stderr, "truncated input\n");
    return 2;
  }
  opt.taa = taa != 0;
  ct::Renderer ren(sc, opt, params);
  if (ren.status() != CT_OK) {
    fprintf(stderr, "set-up failed: %s\n", ct_status_string(ren.status()));
    return 1;
  }
  for (uint32_t f = 0; f < frames; f++) {
    const ct_status st = ren.render(&cams[32u * f], &cams[32u * f + 16u]);
    if (st != CT_OK) {
      fprintf(stderr, "frame %u: %s %s\n", f, ct_status_string(st), ct_last_cuda_error());
      return 1;
    }
  }
  const size_t n = (size_t)opt.width * opt.height;
  std::vector<unsigned char> img(16 * n);
  if (ren.read_output((float *)img.data()) != CT_OK) return 1;
  ct_error_info err;
  if (ct_get_error(nullptr, 1, &err) != CT_OK || err.status != CT_OK) {
    fprintf(stderr, "device error %d at pixel %u\n", (int)err.status, err.pixel);
    return 1;
  }
  FILE *out = fopen(argv[2], "wb");
  if (!out) return 2;
  fwrite("CTHO", 1, 4, out);
  fwrite(&opt.width, 4, 1, out);
  fwrite(&opt.height, 4, 1, out);
  fwrite(img.data(), 1, img.size(), out);
  for (int b = 0; b < ct::kRestirBufferCount; b++) {
    const ct::RestirBuffer which = (ct::RestirBuffer)b;
    std::vector<unsigned char> buf(ct::Renderer::record_bytes(which) * n);
    if (ren.read_buffer(which, buf.data(), buf.size()) != CT_OK) return 1;
    fwrite(buf.data(), 1, buf.size(), out);
  }
  fclose(out);
  return 0;
}
