// ct_nrc.cu -- the neural radiance cache's fully fused MLP on the fifth-
// generation tensor cores (ct_nrc_encode / ct_nrc_infer /
// ct_nrc_infer_encoded, include/ct.h).  No counterpart in the reference,
// whose path tracer has no cache.
//
// Network: 256 inputs (the encoding below, zero padded) -> 5 hidden layers
// of 64 with ReLU -> 16 outputs, of which the first three are RGB radiance.
// Weights are bf16, row-major (output, input); products accumulate in fp32
// in tensor memory; each hidden activation is rounded to bf16 before the
// next layer reads it.
//
// One CTA of 256 threads per SM: two warpgroups, each walking its own tiles
// of 128 queries with its own input tile in shared memory, its own 64
// tensor-memory columns and its own mbarrier, so that one warpgroup's
// encoding and epilogues overlap the other's MMAs.  The weights (66 KB) are
// shared; with the two input tiles the CTA holds 195 KB.  Per tile:
//  * every thread encodes its query into the tile (row = thread), stored
//    K-major in 128-byte-swizzled atoms of 8 rows x 64 bf16, chunk by chunk
//    as it computes them;
//  * one thread of the warpgroup issues tcgen05.mma (M 128, N 64, K 16 per
//    instruction, bf16 inputs, fp32 accumulator) over the layer's K and
//    commits to the warpgroup's mbarrier;
//  * every warp reads its 32 TMEM lanes (tcgen05.ld 32x32b), applies ReLU,
//    rounds to bf16 and writes the next layer's input tile in place;
//  * the last layer (N 16) writes RGB to global memory.
// Warpgroups synchronise on their own named barriers.  Operands are staged
// with ordinary 16-byte shared stores (no TMA).  Every wait is bounded
// (about one second); a warpgroup that gives up latches an error in the
// library's NRC status word and stops; the CTA frees its tensor memory and
// returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cstdint>
#include "ct.h"
#include "ct_profile.cuh"

namespace ct_nrc {

constexpr int kTile = 128;
constexpr int kIn = CT_NRC_INPUT_DIMS;     // 256
constexpr int kWidth = CT_NRC_WIDTH;       // 64
constexpr int kOut = CT_NRC_OUTPUT_DIMS;   // 16
constexpr int kHidden = CT_NRC_HIDDEN_LAYERS;  // 5
constexpr int kGroups = 2;                    // warpgroups per CTA, one tile each
constexpr int kThreads = kTile * kGroups;     // 256
constexpr int kTmemCols = 64 * kGroups;       // 64 accumulator columns per warpgroup

// shared memory regions, each 1024-byte aligned (128-byte swizzle atoms)
constexpr uint32_t kABytes = 4 * 16384;                     // 4 K-blocks of [128 x 64] bf16 = 64 KB
constexpr uint32_t kSmemA = 0;                              // one input tile per warpgroup
constexpr uint32_t kSmemW0 = kSmemA + kGroups * kABytes;    // 4 K-blocks of [64 x 64] = 32 KB
constexpr uint32_t kSmemWh = kSmemW0 + 4 * 8192;            // 4 hidden layers of [64 x 64] = 32 KB
constexpr uint32_t kSmemW5 = kSmemWh + 4 * 8192;            // [16 x 64] = 2 KB
constexpr uint32_t kSmemBar = kSmemW5 + 2048;               // an mbarrier (8 B) per warpgroup + TMEM address
constexpr uint32_t kSmemBytes = kSmemBar + 64 + 1024;       // + slack to align the base to 1024
static_assert(kSmemBytes <= 227 * 1024, "shared memory per CTA");

// weight offsets in the packed bf16 buffer (elements)
constexpr uint32_t kW0 = 0;
constexpr uint32_t kWh = kW0 + kWidth * kIn;
constexpr uint32_t kW5 = kWh + 4 * kWidth * kWidth;
static_assert(kW5 + kOut * kWidth == CT_NRC_WEIGHT_COUNT, "weight packing");

__device__ uint32_t g_nrc_status;  // 0: ok; else the first failure (detail code)

// byte offset of 16-byte chunk `chunk` (8 bf16) of row `row` in a K-major
// region of 64-element rows, 128-byte swizzled: 8-row atoms of 1024 B, the
// chunk index XORed with the row within the atom
__device__ __forceinline__ uint32_t sw128(uint32_t row, uint32_t chunk) {
  return (row >> 3) * 1024u + (row & 7u) * 128u + (((chunk ^ (row & 7u)) & 7u) << 4);
}

// shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 B apart (stride byte offset), version 1 (sm_100)
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)1u << 16;            // leading byte offset: unused with a 128-byte swizzle (16 B)
  d |= (uint64_t)(1024u >> 4) << 32;  // stride byte offset
  d |= (uint64_t)1u << 46;            // descriptor version
  d |= (uint64_t)2u << 61;            // 128-byte swizzle
  return d;
}

// instruction descriptor, kind::f16: bf16 A and B (K-major), fp32 D, M x N
__host__ __device__ constexpr uint32_t instr_desc(uint32_t m, uint32_t n) {
  return (1u << 4)            // D format: f32
         | (1u << 7)          // A format: bf16
         | (1u << 10)         // B format: bf16
         | ((n >> 3) << 17)   // N / 8
         | ((m >> 4) << 24);  // M / 16
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ uint64_t now_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// waits for the mbarrier phase `parity`, for at most about one second
__device__ __forceinline__ bool wait_bar(uint32_t bar, uint32_t parity) {
  const uint64_t t0 = now_ns();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (now_ns() - t0 > 1000000000ull) return false;
  }
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 fp32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t pack2(float a, float b) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t *>(&h);
}

// ---------------------------------------------------------------------------
// The input encoding, 256 values per query:
//   [0, 96)    position q = clamp((p - bbox_min) / bbox_extent, 0, 1): for
//              axis c and band k < 16, t = (q_c * 2^k) mod 2,
//              sin(pi t) at 32c + 2k and cos(pi t) at 32c + 2k + 1;
//   [96, 160)  direction: one-blob of u0 = atan2(w.z, w.x) / 2pi + 1/2 and
//              u1 = w.y / 2 + 1/2, 32 bins each, bin i = exp(-((u - (i +
//              1/2) / 32) * 32)^2 / 2);
//   [160, 224) the normal, the same way;
//   [224, 227) albedo; [227, 256) zero.
__device__ __forceinline__ float onehot_bin(float u, int i) {
  const float d = (u - ((float)i + 0.5f) * (1.0f / 32.0f)) * 32.0f;
  return __expf(-0.5f * d * d);
}

// The encoding in 16-byte chunks of 8 values, emitted as they are computed
// (emit(chunk, v)): chunk 4c + j holds bands 4j .. 4j + 3 of axis c,
// chunks 12 + 8v + j (j < 4) the first angle's bins 8j .. 8j + 7 of vector
// v, chunks 12 + 8v + 4 + j the second angle's, chunk 28 the albedo and
// chunks 29-31 zeros.  (q_c 2^k) mod 2 is s - 2 floor(s / 2) with s = q_c 2^k:
// every step is exact for s < 2^23, as fmod is.
template <class Emit>
__device__ __forceinline__ void encode_chunks(const ct_nrc_query &q, const float *bmin, const float *bext, Emit &&emit) {
#pragma unroll
  for (int c = 0; c < 3; c++) {
    float x = (q.position[c] - bmin[c]) / bext[c];
    x = fminf(fmaxf(x, 0.0f), 1.0f);
#pragma unroll
    for (int j = 0; j < 4; j++) {
      float v[8];
#pragma unroll
      for (int b = 0; b < 4; b++) {
        const float sc = x * (float)(1u << (4 * j + b));
        const float t = sc - 2.0f * floorf(sc * 0.5f);
        sincospif(t, &v[2 * b], &v[2 * b + 1]);
      }
      emit(4 * c + j, v);
    }
  }
  const float *vec[2] = {q.direction, q.normal};
#pragma unroll
  for (int w = 0; w < 2; w++) {
    const float u[2] = {atan2f(vec[w][2], vec[w][0]) * (0.5f / 3.14159265358979323846f) + 0.5f,
                        vec[w][1] * 0.5f + 0.5f};
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
      for (int j = 0; j < 4; j++) {
        float v[8];
#pragma unroll
        for (int i = 0; i < 8; i++) v[i] = onehot_bin(u[a], 8 * j + i);
        emit(12 + 8 * w + 4 * a + j, v);
      }
  }
  float v[8] = {q.albedo[0], q.albedo[1], q.albedo[2], 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
  emit(28, v);
#pragma unroll
  for (int i = 0; i < 3; i++) v[i] = 0.0f;
#pragma unroll
  for (int ch = 29; ch < 32; ch++) emit(ch, v);
}

__device__ __forceinline__ uint4 pack8(const float *v) {
  return make_uint4(pack2(v[0], v[1]), pack2(v[2], v[3]), pack2(v[4], v[5]), pack2(v[6], v[7]));
}

__global__ void __launch_bounds__(256) k_nrc_encode(const ct_nrc_query *q, uint32_t n, float3 bmin, float3 bext,
                                                    __nv_bfloat16 *out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float mn[3] = {bmin.x, bmin.y, bmin.z}, ex[3] = {bext.x, bext.y, bext.z};
  uint4 *dst = reinterpret_cast<uint4 *>(out + 256ull * i);
  encode_chunks(q[i], mn, ex, [&](int ch, const float *v) { dst[ch] = pack8(v); });
}

// warpgroup g's named barrier (ids 1 and 2; 0 is __syncthreads), and the
// same barrier with a vote: true when every thread's `v` is true
__device__ __forceinline__ void group_sync(uint32_t g) { asm volatile("bar.sync %0, 128;" ::"r"(g + 1u) : "memory"); }
__device__ __forceinline__ bool group_all(uint32_t g, bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.and.pred q, %2, 128, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(g + 1u)
      : "memory");
  return r != 0;
}

// one MLP layer: D[128 x N] = A[128 x K] * W[N x K]^T, K in 64-element blocks
__device__ __forceinline__ void layer_mma(uint32_t tmem, uint32_t a_base, uint32_t a_block_bytes, uint32_t w_base,
                                          uint32_t w_block_bytes, int k_blocks, uint32_t idesc, uint32_t bar) {
  fence_after();
  for (int kb = 0; kb < k_blocks; kb++)
    for (int j = 0; j < 4; j++)
      mma(tmem, smem_desc(a_base + kb * a_block_bytes + j * 32), smem_desc(w_base + kb * w_block_bytes + j * 32), idesc,
          (kb | j) != 0);
  commit(bar);
}

template <bool ENCODE>
__global__ void __launch_bounds__(kThreads, 1) k_nrc_mlp(const ct_nrc_query *q, const __nv_bfloat16 *encoded,
                                                         uint32_t n, float3 bmin, float3 bext,
                                                         const __nv_bfloat16 *weights, float *rgb) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t base = smem_u32(smem);
  const uint32_t tid = threadIdx.x, warp = tid >> 5;
  const uint32_t g = tid >> 7, row = tid & (kTile - 1);  // warpgroup, and this thread's row of its tile
  uint32_t *tmem_slot = (uint32_t *)(smem + kSmemBar + 8 * kGroups);

  // weights into their swizzled regions (16-byte chunks)
  for (uint32_t i = tid; i < (uint32_t)(kWidth * (kIn / 8)); i += kThreads) {  // W0: 64 rows x 32 chunks
    const uint32_t r = i / 32u, ch = i % 32u;
    const uint4 v = *reinterpret_cast<const uint4 *>(weights + kW0 + r * kIn + ch * 8u);
    *reinterpret_cast<uint4 *>(smem + kSmemW0 + (ch >> 3) * 8192u + sw128(r, ch & 7u)) = v;
  }
  for (uint32_t i = tid; i < 4u * kWidth * 8u; i += kThreads) {  // W1..W4: 4 x 64 rows x 8 chunks
    const uint32_t l = i / 512u, r = (i / 8u) % 64u, ch = i % 8u;
    const uint4 v = *reinterpret_cast<const uint4 *>(weights + kWh + l * 4096u + r * 64u + ch * 8u);
    *reinterpret_cast<uint4 *>(smem + kSmemWh + l * 8192u + sw128(r, ch)) = v;
  }
  for (uint32_t i = tid; i < (uint32_t)kOut * 8u; i += kThreads) {  // W5: 16 rows x 8 chunks
    const uint32_t r = i / 8u, ch = i % 8u;
    const uint4 v = *reinterpret_cast<const uint4 *>(weights + kW5 + r * 64u + ch * 8u);
    *reinterpret_cast<uint4 *>(smem + kSmemW5 + sw128(r, ch)) = v;
  }
  if (tid == 0) {
    for (uint32_t k = 0; k < (uint32_t)kGroups; k++)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(base + kSmemBar + 8u * k) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem_base = *tmem_slot;
  const uint32_t tmem = tmem_base + 64u * g;                      // this warpgroup's accumulator columns
  const uint32_t lane_addr = tmem + (((warp & 3u) * 32u) << 16);  // a warp reads TMEM lanes 32 (warp % 4) + 0..31
  const uint32_t bar = base + kSmemBar + 8u * g;
  const uint32_t a_off = kSmemA + g * kABytes;
  const float mn[3] = {bmin.x, bmin.y, bmin.z}, ex[3] = {bext.x, bext.y, bext.z};
  uint32_t parity = 0;
  const uint32_t tiles = (n + kTile - 1) / kTile;
  for (uint32_t tile = blockIdx.x * kGroups + g; tile < tiles; tile += gridDim.x * kGroups) {
    const uint32_t qi = tile * kTile + row;
    // layer-0 input tile
    const auto put = [&](int ch, const float *v) {
      *reinterpret_cast<uint4 *>(smem + a_off + (ch >> 3) * 16384u + sw128(row, ch & 7u)) = pack8(v);
    };
    if (ENCODE) {
      if (qi < n) {
        encode_chunks(q[qi], mn, ex, put);
      } else {
        for (uint32_t ch = 0; ch < 32; ch++)
          *reinterpret_cast<uint4 *>(smem + a_off + (ch >> 3) * 16384u + sw128(row, ch & 7u)) = make_uint4(0, 0, 0, 0);
      }
    } else {
      for (uint32_t ch = 0; ch < 32; ch++) {
        uint4 v = make_uint4(0, 0, 0, 0);
        if (qi < n) v = *reinterpret_cast<const uint4 *>(encoded + (uint64_t)qi * kIn + ch * 8u);
        *reinterpret_cast<uint4 *>(smem + a_off + (ch >> 3) * 16384u + sw128(row, ch & 7u)) = v;
      }
    }
    bool ok = true;
    for (int layer = 0; layer <= kHidden; layer++) {
      fence_async_smem();
      fence_before();
      group_sync(g);
      const bool last = layer == kHidden;
      if (row == 0) {
        if (layer == 0)
          layer_mma(tmem, base + a_off, 16384u, base + kSmemW0, 8192u, 4, instr_desc(128, kWidth), bar);
        else if (!last)
          layer_mma(tmem, base + a_off, 16384u, base + kSmemWh + (layer - 1) * 8192u, 8192u, 1,
                    instr_desc(128, kWidth), bar);
        else
          layer_mma(tmem, base + a_off, 16384u, base + kSmemW5, 2048u, 1, instr_desc(128, kOut), bar);
      }
      // the warpgroup's threads leave together when any wait ran out
      if (!group_all(g, wait_bar(bar, parity))) {
        ok = false;
        if (row == 0) atomicCAS(&g_nrc_status, 0u, 1u);
        break;
      }
      parity ^= 1u;
      fence_after();
      if (!last) {
        // ReLU, bf16, next layer's input tile (the first K-block of the warpgroup's tile)
        for (uint32_t c0 = 0; c0 < (uint32_t)kWidth; c0 += 16) {
          float v[16];
          tmem_ld16(lane_addr + c0, v);
#pragma unroll
          for (int k = 0; k < 16; k++) v[k] = fmaxf(v[k], 0.0f);
          *reinterpret_cast<uint4 *>(smem + a_off + sw128(row, c0 >> 3)) = pack8(v);
          *reinterpret_cast<uint4 *>(smem + a_off + sw128(row, (c0 >> 3) + 1)) = pack8(v + 8);
        }
      } else {
        float v[16];
        tmem_ld16(lane_addr, v);
        if (qi < n) {
          rgb[3ull * qi] = v[0];
          rgb[3ull * qi + 1] = v[1];
          rgb[3ull * qi + 2] = v[2];
        }
      }
    }
    if (!ok) break;
    // the next tile's encoding overwrites the input tile: every thread of the
    // warpgroup has read its accumulator rows (tcgen05.wait::ld) by now
    fence_before();
    group_sync(g);
  }
  // every tensor-memory read of this CTA is complete (tcgen05.wait::ld)
  fence_before();
  __syncthreads();
  if (warp == 0) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(kTmemCols) : "memory");
  }
}

}  // namespace ct_nrc

static ct_status nrc_status(cudaError_t e) {
  if (e == cudaSuccess) return CT_OK;
  return CT_ERR_CUDA;
}

static ct_status check_net(const ct_nrc_net *net) {
  if (!net || !net->weights_address || (net->weights_address & 15u)) return CT_ERR_INVALID_ARG;
  for (int c = 0; c < 3; c++)
    if (!(net->bbox_extent[c] > 0.0f) || !isfinite(net->bbox_min[c]) || !isfinite(net->bbox_extent[c]))
      return CT_ERR_INVALID_ARG;
  return CT_OK;
}

static int nrc_grid(uint32_t n) {
  static int sms = 0;
  if (sms == 0) {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    sms = v > 0 ? v : 148;
  }
  const uint32_t pairs = (n + 2u * ct_nrc::kTile - 1) / (2u * ct_nrc::kTile);  // a tile per warpgroup
  return (int)(pairs < (uint32_t)sms ? pairs : (uint32_t)sms);
}

static cudaError_t launch_mlp(bool encode, const ct_nrc_net *net, const ct_nrc_query *q, const void *encoded,
                              uint32_t n, float *rgb, cudaStream_t s) {
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(ct_nrc::k_nrc_mlp<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)ct_nrc::kSmemBytes);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(ct_nrc::k_nrc_mlp<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)ct_nrc::kSmemBytes);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const float3 bmin = make_float3(net->bbox_min[0], net->bbox_min[1], net->bbox_min[2]);
  const float3 bext = make_float3(net->bbox_extent[0], net->bbox_extent[1], net->bbox_extent[2]);
  const __nv_bfloat16 *w = (const __nv_bfloat16 *)(uintptr_t)net->weights_address;
  const int grid = nrc_grid(n);
  if (encode)
    CT_TIMED(CT_K_NRC_MLP, s,
             ct_nrc::k_nrc_mlp<true><<<grid, ct_nrc::kThreads, ct_nrc::kSmemBytes, s>>>(q, nullptr, n, bmin, bext, w, rgb));
  else
    CT_TIMED(CT_K_NRC_MLP, s,
             ct_nrc::k_nrc_mlp<false><<<grid, ct_nrc::kThreads, ct_nrc::kSmemBytes, s>>>(
                 nullptr, (const __nv_bfloat16 *)encoded, n, bmin, bext, w, rgb));
  return cudaGetLastError();
}

extern "C" ct_status ct_nrc_encode(const ct_nrc_net *net, const ct_nrc_query *queries, uint32_t n, void *encoded,
                                   ct_stream stream) {
  ct_status st = check_net(net);
  if (st != CT_OK) return st;
  if (n == 0) return CT_OK;
  if (!queries || !encoded || ((uintptr_t)encoded & 15u)) return CT_ERR_INVALID_ARG;
  const float3 bmin = make_float3(net->bbox_min[0], net->bbox_min[1], net->bbox_min[2]);
  const float3 bext = make_float3(net->bbox_extent[0], net->bbox_extent[1], net->bbox_extent[2]);
  cudaStream_t s = (cudaStream_t)stream;
  CT_TIMED(CT_K_NRC_ENCODE, s,
           ct_nrc::k_nrc_encode<<<(n + 255) / 256, 256, 0, s>>>(queries, n, bmin, bext, (__nv_bfloat16 *)encoded));
  return nrc_status(cudaGetLastError());
}

extern "C" ct_status ct_nrc_infer(const ct_nrc_net *net, const ct_nrc_query *queries, uint32_t n, float *rgb,
                                  ct_stream stream) {
  ct_status st = check_net(net);
  if (st != CT_OK) return st;
  if (n == 0) return CT_OK;
  if (!queries || !rgb) return CT_ERR_INVALID_ARG;
  return nrc_status(launch_mlp(true, net, queries, nullptr, n, rgb, (cudaStream_t)stream));
}

extern "C" ct_status ct_nrc_infer_encoded(const ct_nrc_net *net, const void *encoded, uint32_t n, float *rgb,
                                          ct_stream stream) {
  ct_status st = check_net(net);
  if (st != CT_OK) return st;
  if (n == 0) return CT_OK;
  if (!encoded || !rgb || ((uintptr_t)encoded & 15u)) return CT_ERR_INVALID_ARG;
  return nrc_status(launch_mlp(false, net, nullptr, encoded, n, rgb, (cudaStream_t)stream));
}

extern "C" ct_status ct_nrc_status(int reset, uint32_t *out) {
  if (!out) return CT_ERR_INVALID_ARG;
  cudaError_t e = cudaMemcpyFromSymbol(out, ct_nrc::g_nrc_status, sizeof(uint32_t));
  if (e == cudaSuccess && reset) {
    const uint32_t zero = 0;
    e = cudaMemcpyToSymbol(ct_nrc::g_nrc_status, &zero, sizeof(uint32_t));
  }
  return nrc_status(e);
}
