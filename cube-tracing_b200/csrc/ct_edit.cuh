// ct_edit.cuh -- scene edits: the voxel brush and the rearrangement that
// removes the brushed primitives (ct_brush / ct_rearrange in ct.h).
// Compiled as part of ct_kernels.cu, whose device status word it shares.
//
// Replaces the brush task graph of cube-tracing:
//   entry_brush        src/shaders/slang/compute/squared_brush.slang:74-133
//   entry_rearragement src/shaders/slang/compute/rearrangement.slang:56-204
// and the host bookkeeping around it (accel_struct_mngr.cpp:607-816,
// 2679-2830).  The reference's rearrangement pairs each marked primitive
// with a replacement by scanning the bitmask per thread; here one CTA per
// instance walks the bitmask word by word, ranking marked primitives below
// the new count and unmarked ones above it with block-wide scans, and moves
// rank j of the second set onto rank j of the first.  The result is the
// reference's swap-with-last for one marked primitive, and a deterministic
// dense compaction for any number.
#pragma once

namespace ct_edit {

constexpr uint32_t kEditThreads = 512;

__device__ __forceinline__ const ct_status_block *status_of(const ct_push_constant &pc) {
  return (const ct_status_block *)(uintptr_t)pc.status_buffer;
}
__device__ __forceinline__ const ct_world *world_of(const ct_push_constant &pc) {
  return (const ct_world *)(uintptr_t)pc.world_buffer;
}

// ---------------------------------------------------------------------------
// entry_brush (squared_brush.slang:74-133) with delete_primitive_from_instance
// (:37-72): one thread per pixel.
__global__ void k_brush(ct_push_constant pc) {
  const ct_status_block *st = status_of(pc);
  const ct_world *w = world_of(pc);
  const ct_restir *r = (const ct_restir *)(uintptr_t)pc.restir_buffer;
  const uint32_t px = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t py = blockIdx.y * blockDim.y + threadIdx.y;
  const uint32_t res_x = st->resolution[0], res_y = st->resolution[1];
  if (px >= res_x || py >= res_y) return;
  const ct_brush_config *bc = (const ct_brush_config *)(uintptr_t)st->brush_config_address;
  const uint32_t window = bc->brush_pixel_size[0];
  const uint32_t cx = st->pixel[0], cy = st->pixel[1];
  if (cx >= res_x || cy >= res_y) {
    if (px == 0 && py == 0) ct_latch_error(CT_ERR_INVALID_ARG, 40, cy * res_x + cx);
    return;
  }
  const ct_di_info *pdi = (const ct_di_info *)(uintptr_t)r->previous_di_address;
  const ct_di_info &centre = pdi[cy * res_x + cx];
  if (!(centre.distance > 0.0f)) return;
  // uint2(pixel - window) and uint2(pixel + window) in 32-bit unsigned
  // arithmetic; max(.., uint2(0)) leaves a wrapped lower corner as it is
  const uint32_t min_x = cx - window, min_y = cy - window;
  const uint32_t max_x = umin(cx + window, res_x ? res_x - 1u : 0u);
  const uint32_t max_y = umin(cy + window, res_y ? res_y - 1u : 0u);
  if (!(px >= min_x && px <= max_x && py >= min_y && py <= max_y)) return;
  const ct_di_info &d = pdi[py * res_x + px];
  if (!(d.distance > 0.0f)) return;
  const uint32_t inst = d.instance_hit.instance_id;
  if (inst != centre.instance_hit.instance_id) return;
  const ct_instance *instances = (const ct_instance *)(uintptr_t)w->instance_address;
  const uint32_t prim = instances[inst].first_primitive_index + d.instance_hit.primitive_id;
  if (prim >= st->obj_count) {  // Status.obj_count: the AABB / PRIMITIVE table size
    ct_latch_error(CT_ERR_INVALID_ARG, 42, py * res_x + px);
    return;
  }
  uint32_t *imask = (uint32_t *)(uintptr_t)st->instance_bitmask_address;
  uint32_t *pmask = (uint32_t *)(uintptr_t)st->primitive_bitmask_address;
  ct_brush_counter *counter = (ct_brush_counter *)(uintptr_t)st->brush_counter_address;
  const uint32_t ib = 1u << (inst & 31u), pb = 1u << (prim & 31u);
  const uint32_t old_i = atomicOr(&imask[inst >> 5], ib);
  const uint32_t old_p = atomicOr(&pmask[prim >> 5], pb);
  if (!(old_p & pb)) atomicAdd(&counter->primitive_count, 1u);
  if (!(old_i & ib)) atomicAdd(&counter->instance_count, 1u);
}

// ---------------------------------------------------------------------------
// block-wide helpers (1-D blocks of kEditThreads)
__device__ uint32_t block_scan_excl(uint32_t v, uint32_t *total) {
  __shared__ uint32_t warp_sum[32];
  __shared__ uint32_t s_total;
  const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
  const uint32_t nwarps = (blockDim.x + 31u) >> 5;
  uint32_t incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= (uint32_t)o) incl += t;
  }
  __syncthreads();  // warp_sum may still be read by the previous call
  if (lane == 31u) warp_sum[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    const uint32_t ws = lane < nwarps ? warp_sum[lane] : 0u;
    uint32_t wi = ws;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, wi, o);
      if (lane >= (uint32_t)o) wi += t;
    }
    if (lane < nwarps) warp_sum[lane] = wi - ws;
    if (lane == nwarps - 1u) s_total = wi;
  }
  __syncthreads();
  *total = s_total;
  return warp_sum[wid] + incl - v;
}

// Cursor of a rank scan: the next word to read and the rank of its first
// matching element.
struct RankCursor {
  uint32_t word, base;
};

// Elements are the bits of a bit space (index e = 32 * word + bit) limited to
// [lo, hi); `flags(word)` returns the word's 32 flags.  Writes into
// out[rank - r0] the index of every flagged element whose rank (order of
// increasing index among flagged elements of [lo, hi)) lies in
// [r0, r0 + n), reading words from the cursor on; leaves the cursor at the
// word holding rank r0 + n.  Called by the whole block with the same
// arguments; `cur` lives in shared memory.
template <class Flags>
__device__ void collect_ranks(Flags flags, uint32_t lo, uint32_t hi, uint32_t r0, uint32_t n, uint32_t *out,
                              RankCursor &cur) {
  __shared__ int s_found;
  __shared__ RankCursor s_next;
  const uint32_t w_end = (hi + 31u) >> 5;
  const uint32_t r1 = r0 + n;
  uint32_t w = cur.word, base = cur.base;
  for (;;) {
    if (base >= r1 || w >= w_end) break;
    const uint32_t wi = w + threadIdx.x;
    uint32_t bits = 0;
    if (wi < w_end) {
      bits = flags(wi);
      const uint32_t e0 = wi << 5;
      if (e0 < lo) bits &= 0xFFFFFFFFu << (lo - e0);
      if (hi - e0 < 32u) bits &= (1u << (hi - e0)) - 1u;
    }
    const uint32_t c = __popc(bits);
    uint32_t total;
    const uint32_t rank = base + block_scan_excl(c, &total);
    if (c && rank < r1 && rank + c > r0) {
      uint32_t b = bits, rr = rank;
      while (b) {
        const uint32_t bit = __ffs(b) - 1u;
        b &= b - 1u;
        if (rr >= r0 && rr < r1) out[rr - r0] = (wi << 5) + bit;
        rr++;
      }
    }
    if (threadIdx.x == 0) s_found = 0;
    __syncthreads();
    if (c && rank <= r1 && r1 < rank + c) {
      s_found = 1;
      s_next.word = wi;
      s_next.base = rank;
    }
    __syncthreads();
    if (s_found) {
      w = s_next.word;
      base = s_next.base;
      break;
    }
    base += total;
    w += blockDim.x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    cur.word = w;
    cur.base = base;
  }
  __syncthreads();
}

// count of flagged elements of [lo, hi)
template <class Flags>
__device__ uint32_t count_flags(Flags flags, uint32_t lo, uint32_t hi) {
  uint32_t sum = 0;
  const uint32_t w_end = (hi + 31u) >> 5;
  for (uint32_t w0 = lo >> 5; w0 < w_end; w0 += blockDim.x) {
    const uint32_t wi = w0 + threadIdx.x;
    uint32_t bits = 0;
    if (wi < w_end) {
      bits = flags(wi);
      const uint32_t e0 = wi << 5;
      if (e0 < lo) bits &= 0xFFFFFFFFu << (lo - e0);
      if (hi - e0 < 32u) bits &= (1u << (hi - e0)) - 1u;
    }
    uint32_t total;
    block_scan_excl(__popc(bits), &total);
    sum += total;
  }
  return sum;
}

struct MaskFlags {
  const uint32_t *mask;
  bool want;
  __device__ uint32_t operator()(uint32_t w) const { return want ? mask[w] : ~mask[w]; }
};

// ---------------------------------------------------------------------------
// Primitive compaction, one CTA per instance (entry_rearragement,
// rearrangement.slang:56-204, with its pairing made deterministic).
__global__ void __launch_bounds__(kEditThreads) k_rearrange_primitives(ct_push_constant pc, uint32_t instance_count) {
  const ct_status_block *st = status_of(pc);
  const ct_world *wd = world_of(pc);
  const uint32_t i = blockIdx.x;
  if (i >= instance_count) return;
  const uint32_t *imask = (const uint32_t *)(uintptr_t)st->instance_bitmask_address;
  if (!((imask[i >> 5] >> (i & 31u)) & 1u)) return;
  const uint32_t *pmask = (const uint32_t *)(uintptr_t)st->primitive_bitmask_address;
  ct_instance *instances = (ct_instance *)(uintptr_t)wd->instance_address;
  ct_primitive *prims = (ct_primitive *)(uintptr_t)wd->primitive_address;
  ct_aabb *aabbs = (ct_aabb *)(uintptr_t)wd->aabb_address;
  uint32_t *remap = (uint32_t *)(uintptr_t)wd->remapped_primitive_address;
  const uint32_t f = instances[i].first_primitive_index;
  const uint32_t n = instances[i].primitive_count;
  if (n == 0) return;
  const MaskFlags marked{pmask, true}, kept{pmask, false};
  const uint32_t k = count_flags(marked, f, f + n);
  if (k == 0) return;
  const uint32_t n2 = n - k;
  // marked primitives below n2 = unmarked ones at or above n2
  const uint32_t pairs = n2 == 0 ? 0u : count_flags(marked, f, f + n2);
  __shared__ uint32_t dst[kEditThreads], src[kEditThreads];
  __shared__ RankCursor cd, cs;
  if (threadIdx.x == 0) {
    cd = RankCursor{f >> 5, 0u};
    cs = RankCursor{(f + n2) >> 5, 0u};
  }
  __syncthreads();
  for (uint32_t r0 = 0; r0 < pairs; r0 += blockDim.x) {
    const uint32_t cnt = umin(blockDim.x, pairs - r0);
    collect_ranks(marked, f, f + n2, r0, cnt, dst, cd);
    collect_ranks(kept, f + n2, f + n, r0, cnt, src, cs);
    if (threadIdx.x < cnt) {
      const uint32_t s = src[threadIdx.x], d = dst[threadIdx.x];
      prims[d] = prims[s];
      aabbs[d] = aabbs[s];
      remap[s] = d - f;
    }
    __syncthreads();
  }
  // every marked primitive: -1
  const uint32_t w_end = (f + n + 31u) >> 5;
  for (uint32_t w0 = f >> 5; w0 < w_end; w0 += blockDim.x) {
    const uint32_t wi = w0 + threadIdx.x;
    if (wi >= w_end) continue;
    uint32_t bits = pmask[wi];
    const uint32_t e0 = wi << 5;
    if (e0 < f) bits &= 0xFFFFFFFFu << (f - e0);
    if (f + n - e0 < 32u) bits &= (1u << (f + n - e0)) - 1u;
    while (bits) {
      const uint32_t b = __ffs(bits) - 1u;
      bits &= bits - 1u;
      remap[e0 + b] = 0xFFFFFFFFu;
    }
  }
  if (threadIdx.x == 0) instances[i].primitive_count = n2;
}

// ---------------------------------------------------------------------------
// Cube-light compaction, one CTA.  A light is removed when its primitive
// (LIGHT.instance_info before the primitive moves) is marked.  The remap
// table doubles as the removal flags: -1 removed, 0 kept, then the new
// index of every moved light.
struct LightRemoved {
  const uint32_t *remap_l;
  uint32_t count;
  __device__ uint32_t operator()(uint32_t w) const {
    uint32_t bits = 0;
    for (uint32_t b = 0; b < 32u; b++) {
      const uint32_t e = (w << 5) + b;
      if (e < count && remap_l[e] == 0xFFFFFFFFu) bits |= 1u << b;
    }
    return bits;
  }
};
struct LightKept {
  LightRemoved r;
  __device__ uint32_t operator()(uint32_t w) const { return ~r(w); }
};

// instance-relative primitive id of a kept light after the primitive moves;
// ids outside the primitive table (the .vox loader's cube lights carry a
// global index, map_loader.cpp:285) are left as they are
__device__ __forceinline__ uint32_t moved_primitive(const ct_instance *instances, uint32_t instance_count,
                                                    uint32_t primitive_total, const uint32_t *remap_p,
                                                    const ct_object_info &o) {
  if (o.instance_id >= instance_count) return o.primitive_id;
  const ct_instance &in = instances[o.instance_id];
  if (o.primitive_id < in.primitive_count) return o.primitive_id;
  const uint64_t g = (uint64_t)in.first_primitive_index + o.primitive_id;
  return g < primitive_total ? remap_p[g] : o.primitive_id;
}

__global__ void __launch_bounds__(kEditThreads) k_rearrange_lights(ct_push_constant pc, uint32_t instance_count,
                                                                   uint32_t primitive_total) {
  const ct_status_block *st = status_of(pc);
  const ct_world *wd = world_of(pc);
  const uint32_t *pmask = (const uint32_t *)(uintptr_t)st->primitive_bitmask_address;
  const ct_instance *instances = (const ct_instance *)(uintptr_t)wd->instance_address;
  ct_primitive *prims = (ct_primitive *)(uintptr_t)wd->primitive_address;
  ct_light *lights = (ct_light *)(uintptr_t)wd->cube_light_address;
  const uint32_t *remap_p = (const uint32_t *)(uintptr_t)wd->remapped_primitive_address;
  uint32_t *remap_l = (uint32_t *)(uintptr_t)wd->remapped_cube_light_address;
  ct_light_config *cfg = (ct_light_config *)(uintptr_t)st->light_config_address;
  const uint32_t L = cfg->cube_light_count;
  if (L == 0) return;
  // removal flags (the primitive bitmask is still the brush's)
  for (uint32_t x = threadIdx.x; x < L; x += blockDim.x) {
    const ct_object_info o = lights[x].instance_info;
    bool removed = false;
    if (o.instance_id < instance_count) {
      const uint64_t g = (uint64_t)instances[o.instance_id].first_primitive_index + o.primitive_id;
      removed = g < primitive_total && ((pmask[g >> 5] >> (g & 31u)) & 1u);
    }
    remap_l[x] = removed ? 0xFFFFFFFFu : 0u;
  }
  __syncthreads();
  const LightRemoved removed{remap_l, L};
  const LightKept kept{removed};
  const uint32_t m = count_flags(removed, 0, L);
  if (m == 0) {
    // primitives may still have moved under their lights
    for (uint32_t x = threadIdx.x; x < L; x += blockDim.x)
      lights[x].instance_info.primitive_id = moved_primitive(instances, instance_count, primitive_total, remap_p, lights[x].instance_info);
    return;
  }
  const uint32_t L2 = L - m;
  // kept lights that stay: follow their primitive
  for (uint32_t x = threadIdx.x; x < L2; x += blockDim.x) {
    if (remap_l[x] == 0xFFFFFFFFu) continue;
    lights[x].instance_info.primitive_id = moved_primitive(instances, instance_count, primitive_total, remap_p, lights[x].instance_info);
  }
  __syncthreads();
  const uint32_t pairs = L2 == 0 ? 0u : count_flags(removed, 0, L2);
  __shared__ uint32_t dst[kEditThreads], src[kEditThreads];
  __shared__ RankCursor cd, cs;
  if (threadIdx.x == 0) {
    cd = RankCursor{0u, 0u};
    cs = RankCursor{L2 >> 5, 0u};
  }
  __syncthreads();
  for (uint32_t r0 = 0; r0 < pairs; r0 += blockDim.x) {
    const uint32_t cnt = umin(blockDim.x, pairs - r0);
    collect_ranks(removed, 0, L2, r0, cnt, dst, cd);
    collect_ranks(kept, L2, L, r0, cnt, src, cs);
    __syncthreads();
    if (threadIdx.x < cnt) {
      const uint32_t s = src[threadIdx.x], d = dst[threadIdx.x];
      ct_light lt = lights[s];
      lt.instance_info.primitive_id = moved_primitive(instances, instance_count, primitive_total, remap_p, lt.instance_info);
      lights[d] = lt;
      remap_l[s] = d;
      if (lt.instance_info.instance_id < instance_count) {
        const uint64_t g =
            (uint64_t)instances[lt.instance_info.instance_id].first_primitive_index + lt.instance_info.primitive_id;
        if (g < primitive_total) prims[g].light_index = d;
      }
    }
    __syncthreads();
  }
  // removed lights above L2 keep their -1; lights above L2 that stayed were
  // all moved (their count equals the removed ones below L2)
  if (threadIdx.x == 0) {
    cfg->cube_light_count = L2;
    cfg->light_count = cfg->light_count >= m ? cfg->light_count - m : 0u;
  }
}

// restore_bitmask_buffers (accel_struct_mngr.cpp:2679-2705) and the counter reset
__global__ void k_clear_marks(ct_push_constant pc, uint32_t instance_words, uint32_t primitive_words) {
  const ct_status_block *st = status_of(pc);
  uint32_t *imask = (uint32_t *)(uintptr_t)st->instance_bitmask_address;
  uint32_t *pmask = (uint32_t *)(uintptr_t)st->primitive_bitmask_address;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < primitive_words; t += stride) pmask[t] = 0u;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < instance_words; t += stride) imask[t] = 0u;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ct_brush_counter *c = (ct_brush_counter *)(uintptr_t)st->brush_counter_address;
    c->instance_count = 0u;
    c->primitive_count = 0u;
  }
}

}  // namespace ct_edit

cudaError_t ct_launch_brush(const ct_push_constant &pc, cudaStream_t s) {
  const dim3 blk(8, 8);  // BRUSH_COMPUTE_X x BRUSH_COMPUTE_Y (shared.inl:82-83)
  const dim3 grid((pc.size[0] + 7u) / 8u, (pc.size[1] + 7u) / 8u);
  CT_TIMED(CT_K_EDIT, s, ct_edit::k_brush<<<grid, blk, 0, s>>>(pc));
  return cudaGetLastError();
}

cudaError_t ct_launch_rearrange(const ct_push_constant &pc, uint32_t instance_count, uint32_t primitive_count,
                                cudaStream_t s) {
  cudaError_t e;
  CT_TIMED(CT_K_EDIT, s, ct_edit::k_rearrange_primitives<<<instance_count, ct_edit::kEditThreads, 0, s>>>(pc, instance_count));
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  CT_TIMED(CT_K_EDIT, s, ct_edit::k_rearrange_lights<<<1, ct_edit::kEditThreads, 0, s>>>(pc, instance_count,
                                                                                   primitive_count));
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  const uint32_t pw = (primitive_count + 31u) / 32u, iw = (instance_count + 31u) / 32u;
  const uint32_t words = pw > iw ? pw : iw;
  const uint32_t blocks = words / 256u + 1u < 1184u ? words / 256u + 1u : 1184u;
  CT_TIMED(CT_K_EDIT, s, ct_edit::k_clear_marks<<<blocks, 256, 0, s>>>(pc, iw, pw));
  return cudaGetLastError();
}
