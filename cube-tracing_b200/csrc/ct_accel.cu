// ct_accel.cu -- ct_build_accel: voxel brick maps from the caller's AABBs.
//
// Replaces the per-instance AABB BLAS + TLAS build of
// ACCEL_STRUCT_MNGR::build_blases / build_tlas (src/accel_struct_mngr.cpp:
// 1362-1504, 1854-1973).  The reference's AABBs are single voxels of a fixed
// grid (src/gvox/map_loader.cpp:264-272), so instead of a BVH over boxes each
// instance gets a dense grid of 8^3 bricks:
//
//   pass 1  per AABB: integer voxel coordinate, alignment check, per-instance
//           bounds (atomic min/max)                        -> host reads bounds
//   pass 2  per AABB: mark the brick as occupied and every brick its
//           26-neighbourhood touches as NEAR
//   pass 3  per brick cell: give NEAR bricks a mask slot and bricks with
//           voxels a primitive slot                       -> host reads counts
//   pass 4  per AABB: set the occupancy bit, keep the lowest primitive id
//           per voxel, record the voxel coordinate of the primitive
//   pass 5  per cell and ray octant: the cell field the walks step by, the
//           edge of the occupied-free cube from the cell (15 Jacobi sweeps)
//
// Device memory held by the result: two 4 B tables per brick cell, 64 B of
// occupancy mask per NEAR brick, 2 KiB of primitive ids per brick with
// voxels, 4 B per primitive, the cell field (4 B per cell), and one
// descriptor per instance.
#include <cuda_runtime.h>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>
#include "ct_accel.cuh"

struct InstBounds {
  int mn[3], mx[3];
  uint32_t inexact;   // any voxel whose centre cannot be recomputed exactly
  uint32_t misaligned;
};

__global__ void k_bounds(const ct_instance *inst, uint32_t n_inst, const ct_aabb *aabb, uint32_t n_aabb, float e,
                         InstBounds *B) {
  const uint32_t i = blockIdx.y;
  if (i >= n_inst) return;
  const uint32_t first = inst[i].first_primitive_index, count = inst[i].primitive_count;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
    const uint32_t gi = first + k;
    if (gi >= n_aabb) { atomicOr(&B[i].misaligned, 2u); continue; }
    const ct_aabb &b = aabb[gi];
    int c[3];
    bool ok = true, exact = true;
    for (int a = 0; a < 3; a++) {
      const float lo = b.minimum[a], hi = b.maximum[a];
      const float v = lo / e;
      const int iv = __float2int_rn(v);
      if (!(fabsf(v - (float)iv) <= 1e-3f) || !(fabsf((hi - lo) / e - 1.0f) <= 1e-3f)) ok = false;
      if (!((float)iv * e == lo && (float)(iv + 1) * e == hi)) exact = false;
      c[a] = iv;
    }
    if (!ok) { atomicOr(&B[i].misaligned, 1u); continue; }
    if (!exact) atomicOr(&B[i].inexact, 1u);
    for (int a = 0; a < 3; a++) {
      atomicMin(&B[i].mn[a], c[a]);
      atomicMax(&B[i].mx[a], c[a]);
    }
  }
}

__device__ __forceinline__ bool voxel_local(const ct_aabb &b, float e, const DevGrid &g, int &x, int &y, int &z) {
  x = __float2int_rn(b.minimum[0] / e) - g.gmin[0];
  y = __float2int_rn(b.minimum[1] / e) - g.gmin[1];
  z = __float2int_rn(b.minimum[2] / e) - g.gmin[2];
  return x >= 0 && y >= 0 && z >= 0 && x < g.bdim[0] * CT_BRICK && y < g.bdim[1] * CT_BRICK && z < g.bdim[2] * CT_BRICK;
}

__device__ __forceinline__ uint32_t *table_at(uint32_t *table, const DevGrid &g, int bx, int by, int bz) {
  return &table[g.table_offset + ((uint32_t)bz * g.bdim[1] + by) * g.bdim[0] + bx];
}

// bit 0 of a table entry marks "has voxels" until slots are assigned
__global__ void k_mark(const DevGrid *grids, uint32_t n_inst, const ct_aabb *aabb, float e, uint32_t *table) {
  const uint32_t i = blockIdx.y;
  if (i >= n_inst) return;
  const DevGrid g = grids[i];
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < g.primitive_count; k += gridDim.x * blockDim.x) {
    int x, y, z;
    if (!voxel_local(aabb[g.first_primitive_index + k], e, g, x, y, z)) continue;
    const int b[3] = {x >> 3, y >> 3, z >> 3};
    const int l[3] = {x & 7, y & 7, z & 7};
    atomicOr(table_at(table, g, b[0], b[1], b[2]), 1u | CT_NEAR_BIT);
    // bricks the voxel's 26-neighbourhood reaches
    int lo[3], hi[3];
    for (int a = 0; a < 3; a++) {
      lo[a] = (l[a] == 0) ? -1 : 0;
      hi[a] = (l[a] == 7) ? 1 : 0;
    }
    for (int dz = lo[2]; dz <= hi[2]; dz++)
      for (int dy = lo[1]; dy <= hi[1]; dy++)
        for (int dx = lo[0]; dx <= hi[0]; dx++) {
          if (!dx && !dy && !dz) continue;
          const int nb[3] = {b[0] + dx, b[1] + dy, b[2] + dz};
          if (nb[0] < 0 || nb[1] < 0 || nb[2] < 0 || nb[0] >= g.bdim[0] || nb[1] >= g.bdim[1] || nb[2] >= g.bdim[2])
            continue;
          atomicOr(table_at(table, g, nb[0], nb[1], nb[2]), CT_NEAR_BIT);
        }
  }
}

// counter[0]: mask slots (NEAR bricks), counter[1]: primitive slots (bricks with voxels)
__global__ void k_assign_slots(uint32_t *table, uint32_t *pslot, uint32_t n_cells, uint32_t *counter) {
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n_cells; c += gridDim.x * blockDim.x) {
    const uint32_t v = table[c];
    uint32_t slot = CT_EMPTY_SLOT, ps = CT_EMPTY_SLOT;
    if (v & CT_NEAR_BIT) slot = atomicAdd(&counter[0], 1u);
    if (v & 1u) ps = atomicAdd(&counter[1], 1u);
    table[c] = (v & CT_NEAR_BIT) | slot;
    pslot[c] = ps;
  }
}

__global__ void k_fill(const DevGrid *grids, uint32_t n_inst, const ct_aabb *aabb, float e, const uint32_t *table,
                       const uint32_t *pslot, uint32_t *mask, uint32_t *prim, uint32_t *vcoord) {
  const uint32_t i = blockIdx.y;
  if (i >= n_inst) return;
  const DevGrid g = grids[i];
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < g.primitive_count; k += gridDim.x * blockDim.x) {
    int x, y, z;
    const uint32_t gi = g.first_primitive_index + k;
    if (!voxel_local(aabb[gi], e, g, x, y, z)) continue;
    const uint32_t cell = g.table_offset + ((uint32_t)(z >> 3) * g.bdim[1] + (y >> 3)) * g.bdim[0] + (x >> 3);
    const uint32_t slot = table[cell] & CT_EMPTY_SLOT;
    const uint32_t local = (uint32_t)(x & 7) + 8u * (uint32_t)(y & 7) + 64u * (uint32_t)(z & 7);
    atomicOr(&mask[slot * CT_MASK_WORDS + (local >> 5)], 1u << (local & 31u));
    atomicMin(&prim[pslot[cell] * 512u + local], k);
    vcoord[gi] = (uint32_t)x | ((uint32_t)y << 10) | ((uint32_t)z << 20);
  }
}

// distinct occupied voxels: the set bits of every NEAR brick's occupancy words
__global__ void k_count_voxels(const uint32_t *mask, uint32_t n_slots, uint32_t *count) {
  uint32_t c = 0;
  for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < (uint64_t)CT_MASK_WORDS * n_slots;
       w += (uint64_t)gridDim.x * blockDim.x)
    c += __popc(mask[w]);
  for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xFFFFFFFFu, c, o);
  if ((threadIdx.x & 31u) == 0u && c) atomicAdd(count, c);
}

// The cell field (cell_field, ct_types.cuh): for every cell of a grid and
// every ray octant, the edge k of the largest cube without occupied cells
// that has the cell as its corner and extends in the octant's directions,
// stored as the largest 4-bit code whose edge (ct_field_edge) is at most k.
// The cube of edge k at c is the cell c and the cubes of edge k - 1 at its 7
// forward neighbours, so k(c) = 0 when c is occupied, else min(15, 1 + min
// over those neighbours), a neighbour beyond the grid counting as 15 (the
// walk clips every box to the grid).  k_field_step runs that rule as a
// Jacobi sweep from k = 15: a value that ends below 15 rests on a chain of
// fewer than 15 cells to an occupied one, so 15 sweeps reach the fixed
// point.  k_field_grow then doubles the cap (15 -> 30) for the cells at it.
// One byte per cell and octant while building.
struct FieldGrid {
  uint64_t cell0;   // first cell in the build buffers
  uint32_t X, Y, Z; // cells per axis
  uint32_t table_offset, bx;
  uint64_t word0;   // first word in cell_field
};

// occupancy of every cell, from the brick table and the NEAR bricks' masks
__global__ void k_occ_cells(const FieldGrid *fg, uint32_t n_inst, const uint32_t *table, const uint32_t *mask,
                            uint8_t *occ) {
  const FieldGrid f = fg[blockIdx.y];
  const uint64_t n = (uint64_t)f.X * f.Y * f.Z;
  for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < n; c += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t x = (uint32_t)(c % f.X), y = (uint32_t)((c / f.X) % f.Y), z = (uint32_t)(c / ((uint64_t)f.X * f.Y));
    const uint32_t e = table[f.table_offset + ((z >> 3) * (f.Y >> 3) + (y >> 3)) * f.bx + (x >> 3)];
    uint8_t v = 0;
    if (e & CT_NEAR_BIT) {
      const uint32_t l = (x & 7u) + 8u * (y & 7u) + 64u * (z & 7u);
      v = (uint8_t)((mask[(e & CT_EMPTY_SLOT) * CT_MASK_WORDS + (l >> 5)] >> (l & 31u)) & 1u);
    }
    occ[f.cell0 + c] = v;
  }
}

__global__ void k_field_step(const FieldGrid *fg, uint32_t octant, const uint8_t *occ, const uint8_t *src,
                             uint8_t *dst, int first) {
  const FieldGrid f = fg[blockIdx.y];
  const uint64_t n = (uint64_t)f.X * f.Y * f.Z;
  const int sx = (octant & 1u) ? -1 : 1, sy = (octant & 2u) ? -1 : 1, sz = (octant & 4u) ? -1 : 1;
  for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < n; c += (uint64_t)gridDim.x * blockDim.x) {
    if (occ[f.cell0 + c]) {
      dst[f.cell0 + c] = 0;
      continue;
    }
    if (first) {
      dst[f.cell0 + c] = 15;
      continue;
    }
    const int x = (int)(c % f.X), y = (int)((c / f.X) % f.Y), z = (int)(c / ((uint64_t)f.X * f.Y));
    int m = 15;
    for (int d = 1; d < 8; d++) {
      const int nx = x + ((d & 1) ? sx : 0), ny = y + ((d & 2) ? sy : 0), nz = z + ((d & 4) ? sz : 0);
      if ((unsigned)nx < f.X && (unsigned)ny < f.Y && (unsigned)nz < f.Z)
        m = min(m, (int)src[f.cell0 + ((uint64_t)nz * f.Y + ny) * f.X + nx]);
    }
    dst[f.cell0 + c] = (uint8_t)min(15, m + 1);
  }
}

// Edges above 15, from the exact edges up to m (m meaning "at least m"):
// the cube of edge e <= 2m at c is the 8 cubes of edge h = ceil(e / 2) at
// c + {0, e - h} per axis (towards the octant), and a cube at a corner beyond
// the grid lies wholly outside it.  An emptiness test is monotone in e, so a
// binary search over (m, min(2m, cap)] finds the largest edge.
__global__ void k_field_grow(const FieldGrid *fg, uint32_t octant, const uint8_t *src, uint8_t *dst, int m, int cap) {
  const FieldGrid f = fg[blockIdx.y];
  const uint64_t n = (uint64_t)f.X * f.Y * f.Z;
  const int sx = (octant & 1u) ? -1 : 1, sy = (octant & 2u) ? -1 : 1, sz = (octant & 4u) ? -1 : 1;
  for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < n; c += (uint64_t)gridDim.x * blockDim.x) {
    const int v = src[f.cell0 + c];
    if (v < m) {
      dst[f.cell0 + c] = (uint8_t)v;
      continue;
    }
    const int x = (int)(c % f.X), y = (int)((c / f.X) % f.Y), z = (int)(c / ((uint64_t)f.X * f.Y));
    int lo = m, hi = min(2 * m, cap);
    while (lo < hi) {
      const int e = (lo + hi + 1) / 2, h = (e + 1) / 2, off = e - h;
      bool empty = true;
      for (int d = 0; d < 8 && empty; d++) {
        const int nx = x + ((d & 1) ? sx * off : 0), ny = y + ((d & 2) ? sy * off : 0),
                  nz = z + ((d & 4) ? sz * off : 0);
        if ((unsigned)nx < f.X && (unsigned)ny < f.Y && (unsigned)nz < f.Z)
          empty = src[f.cell0 + ((uint64_t)nz * f.Y + ny) * f.X + nx] >= h;
      }
      if (empty) lo = e;
      else hi = e - 1;
    }
    dst[f.cell0 + c] = (uint8_t)lo;
  }
}

// 8 cells' edges of one octant into a word of nibbles: the largest code
// whose edge does not exceed the cell's
__global__ void k_field_pack(const FieldGrid *fg, uint32_t octant, const uint8_t *k, uint32_t *field) {
  const FieldGrid f = fg[blockIdx.y];
  const uint64_t n = (uint64_t)f.X * f.Y * f.Z / 8u;
  for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < n; w += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t v = 0;
    for (int i = 0; i < 8; i++) {
      const int e = k[f.cell0 + 8u * w + i];
      uint32_t code = 15u;
      while (ct_field_edge(code) > e) code--;
      v |= code << (4 * i);
    }
    field[f.word0 + (uint64_t)octant * n + w] = v;
  }
}

// Builds the cell field of every grid (see k_field_step): 2 KiB per brick,
// with three bytes per cell of scratch while building.
static cudaError_t build_cell_field(ct_accel *acc, uint64_t total_bricks, cudaStream_t stream) {
  const uint32_t n_inst = (uint32_t)acc->h_grids.size();
  std::vector<FieldGrid> hf(n_inst);
  uint64_t cells = 0, max_cells = 0;
  for (uint32_t i = 0; i < n_inst; i++) {
    DevGrid &g = acc->h_grids[i];
    FieldGrid &f = hf[i];
    f.X = (uint32_t)g.bdim[0] * CT_BRICK;
    f.Y = (uint32_t)g.bdim[1] * CT_BRICK;
    f.Z = (uint32_t)g.bdim[2] * CT_BRICK;
    f.table_offset = g.table_offset;
    f.bx = (uint32_t)g.bdim[0];
    f.cell0 = cells;
    f.word0 = cells;  // 8 octants x (cells / 8) words per grid
    const uint64_t n = (uint64_t)f.X * f.Y * f.Z;
    g.field_offset = cells;
    cells += n;
    max_cells = n > max_cells ? n : max_cells;
  }
  (void)total_bricks;
  cudaError_t e;
  if ((e = cudaMalloc(&acc->d_field, sizeof(uint32_t) * (cells ? cells : 1))) != cudaSuccess) return e;
  if (cells == 0) return cudaSuccess;
  FieldGrid *d_fg = nullptr;
  uint8_t *buf = nullptr;
  if ((e = cudaMalloc(&d_fg, sizeof(FieldGrid) * n_inst)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&buf, 3ull * cells)) != cudaSuccess) { cudaFree(d_fg); return e; }
  uint8_t *occ = buf, *ka = buf + cells, *kb = buf + 2ull * cells;
  if ((e = cudaMemcpyAsync(d_fg, hf.data(), sizeof(FieldGrid) * n_inst, cudaMemcpyHostToDevice, stream)) == cudaSuccess) {
    const uint64_t want = (max_cells + 255) / 256;
    const dim3 grid((uint32_t)(want < 8192 ? (want ? want : 1) : 8192), n_inst);
    k_occ_cells<<<grid, 256, 0, stream>>>(d_fg, n_inst, acc->d_table, acc->d_mask, occ);
    for (uint32_t o = 0; o < 8 && (e = cudaGetLastError()) == cudaSuccess; o++) {
      k_field_step<<<grid, 256, 0, stream>>>(d_fg, o, occ, ka, ka, 1);
      for (int it = 0; it < 15; it++) {
        k_field_step<<<grid, 256, 0, stream>>>(d_fg, o, occ, ka, kb, 0);
        uint8_t *t = ka; ka = kb; kb = t;
      }
      for (int m = 15; m < CT_FIELD_MAX_EDGE; m *= 2) {
        k_field_grow<<<grid, 256, 0, stream>>>(d_fg, o, ka, kb, m, CT_FIELD_MAX_EDGE);
        uint8_t *t = ka; ka = kb; kb = t;
      }
      k_field_pack<<<grid, 256, 0, stream>>>(d_fg, o, ka, acc->d_field);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
  }
  // the grids' field offsets
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(acc->d_grids, acc->h_grids.data(), sizeof(DevGrid) * n_inst, cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);  // the scratch is freed below
  cudaFree(buf);
  cudaFree(d_fg);
  return e;
}

static ct_status cuda_fail(cudaError_t e) {
  ct_set_cuda_error(e);
  return CT_ERR_CUDA;
}

#define CT_TRY(x)                              \
  do {                                         \
    cudaError_t _e = (x);                      \
    if (_e != cudaSuccess) { st = cuda_fail(_e); goto fail; } \
  } while (0)

ct_accel::~ct_accel() {
  cudaFree(d_grids);
  cudaFree(d_table);
  cudaFree(d_pslot);
  cudaFree(d_mask);
  cudaFree(d_prim);
  cudaFree(d_vcoord);
  cudaFree(d_field);
  cudaFree(ws_ptr);
}

extern "C" ct_status ct_build_accel(const ct_scene_desc *scene, ct_accel **out, ct_stream stream_) {
  if (!scene || !out) return CT_ERR_INVALID_ARG;
  *out = nullptr;
  cudaStream_t stream = (cudaStream_t)stream_;
  if (scene->instance_count == 0 || scene->instance_address == 0 || scene->aabb_address == 0) return CT_ERR_INVALID_ARG;
  if (!(scene->voxel_extent > 0.0f) || !isfinite(scene->voxel_extent)) return CT_ERR_INVALID_ARG;
  if (scene->instance_count > CT_MAX_INSTANCES || scene->aabb_count > CT_MAX_PRIMITIVES) return CT_ERR_CAPACITY;
  if ((scene->instance_address & 3u) || (scene->aabb_address & 3u)) return CT_ERR_INVALID_ARG;

  ct_status st = CT_OK;
  const uint32_t n_inst = scene->instance_count;
  const float e = scene->voxel_extent;
  const ct_instance *d_inst = (const ct_instance *)(uintptr_t)scene->instance_address;
  const ct_aabb *d_aabb = (const ct_aabb *)(uintptr_t)scene->aabb_address;
  std::vector<ct_instance> h_inst(n_inst);
  std::vector<InstBounds> h_b(n_inst);
  InstBounds *d_b = nullptr;
  uint32_t *d_counter = nullptr;
  ct_accel *acc = new (std::nothrow) ct_accel();
  if (!acc) return CT_ERR_CAPACITY;
  uint64_t total_cells = 0, max_prims = 0;
  uint32_t n_slots = 0, n_pslots = 0;
  uint32_t counts[2] = {0, 0};

  for (uint32_t i = 0; i < n_inst; i++) {
    h_b[i].mn[0] = h_b[i].mn[1] = h_b[i].mn[2] = INT32_MAX;
    h_b[i].mx[0] = h_b[i].mx[1] = h_b[i].mx[2] = INT32_MIN;
    h_b[i].inexact = h_b[i].misaligned = 0;
  }
  CT_TRY(cudaMemcpyAsync(h_inst.data(), d_inst, sizeof(ct_instance) * n_inst, cudaMemcpyDeviceToHost, stream));
  CT_TRY(cudaMalloc(&d_b, sizeof(InstBounds) * n_inst));
  CT_TRY(cudaMalloc(&d_counter, 2 * sizeof(uint32_t)));
  CT_TRY(cudaMemcpyAsync(d_b, h_b.data(), sizeof(InstBounds) * n_inst, cudaMemcpyHostToDevice, stream));
  CT_TRY(cudaMemsetAsync(d_counter, 0, 2 * sizeof(uint32_t), stream));
  CT_TRY(cudaStreamSynchronize(stream));
  for (uint32_t i = 0; i < n_inst; i++) {
    if ((uint64_t)h_inst[i].first_primitive_index + h_inst[i].primitive_count > scene->aabb_count) {
      st = CT_ERR_INVALID_ARG;
      goto fail;
    }
    max_prims = h_inst[i].primitive_count > max_prims ? h_inst[i].primitive_count : max_prims;
  }
  {
    dim3 grid((uint32_t)((max_prims + 255) / 256 < 4096 ? (max_prims + 255) / 256 : 4096), n_inst);
    if (grid.x == 0) grid.x = 1;
    k_bounds<<<grid, 256, 0, stream>>>(d_inst, n_inst, d_aabb, scene->aabb_count, e, d_b);
    CT_TRY(cudaGetLastError());
    CT_TRY(cudaMemcpyAsync(h_b.data(), d_b, sizeof(InstBounds) * n_inst, cudaMemcpyDeviceToHost, stream));
    CT_TRY(cudaStreamSynchronize(stream));
  }
  acc->h_grids.resize(n_inst);
  acc->info.grid_exact = 1;
  for (uint32_t i = 0; i < n_inst; i++) {
    if (h_b[i].misaligned & 2u) { st = CT_ERR_INVALID_ARG; goto fail; }
    if (h_b[i].misaligned) { st = CT_ERR_NOT_GRID_ALIGNED; goto fail; }
    DevGrid &g = acc->h_grids[i];
    memset(&g, 0, sizeof(g));
    m4 T = load_m4(h_inst[i].transform);
    g.world2obj_inst = ct_inverse(T);
    m4 Tt = T;
    Tt.c[0].w = 0.f; Tt.c[1].w = 0.f; Tt.c[2].w = 0.f; Tt.c[3].w = 1.f;
    g.obj2world_tlas = Tt;
    g.world2obj_tlas = ct_inverse(Tt);
    g.first_primitive_index = h_inst[i].first_primitive_index;
    g.primitive_count = h_inst[i].primitive_count;
    g.grid_exact = h_b[i].inexact ? 0u : 1u;
    if (!g.grid_exact) acc->info.grid_exact = 0;
    int mn[3], mx[3];
    for (int a = 0; a < 3; a++) {
      if (h_inst[i].primitive_count == 0) { mn[a] = 0; mx[a] = 0; }
      else { mn[a] = h_b[i].mn[a]; mx[a] = h_b[i].mx[a]; }
      // one empty voxel of margin on every side, brick aligned
      int lo = mn[a] - 1, hi = mx[a] + 1;
      int glo = (lo >= 0) ? (lo / CT_BRICK) * CT_BRICK : -((-lo + CT_BRICK - 1) / CT_BRICK) * CT_BRICK;
      g.gmin[a] = glo;
      g.bdim[a] = (hi - glo) / CT_BRICK + 1;
      if (g.bdim[a] * CT_BRICK > 1024) { st = CT_ERR_CAPACITY; goto fail; }  // 10-bit voxel coordinates
    }
    g.table_offset = (uint32_t)total_cells;
    total_cells += (uint64_t)g.bdim[0] * g.bdim[1] * g.bdim[2];
    if (total_cells > 0x7FFFFFFFull) { st = CT_ERR_CAPACITY; goto fail; }
    if (i == 0)
      for (int a = 0; a < 3; a++) { acc->info.grid_min[a] = mn[a]; acc->info.grid_dim[a] = mx[a] - mn[a] + 1; }
  }
  CT_TRY(cudaMalloc(&acc->d_grids, sizeof(DevGrid) * n_inst));
  CT_TRY(cudaMemcpyAsync(acc->d_grids, acc->h_grids.data(), sizeof(DevGrid) * n_inst, cudaMemcpyHostToDevice, stream));
  CT_TRY(cudaMalloc(&acc->d_table, sizeof(uint32_t) * total_cells));
  CT_TRY(cudaMemsetAsync(acc->d_table, 0, sizeof(uint32_t) * total_cells, stream));
  CT_TRY(cudaMalloc(&acc->d_pslot, sizeof(uint32_t) * total_cells));
  acc->n_primitives = scene->aabb_count;
  CT_TRY(cudaMalloc(&acc->d_vcoord, sizeof(uint32_t) * (scene->aabb_count > 0 ? scene->aabb_count : 1)));
  CT_TRY(cudaMemsetAsync(acc->d_vcoord, 0xFF, sizeof(uint32_t) * (scene->aabb_count > 0 ? scene->aabb_count : 1), stream));
  {
    dim3 grid((uint32_t)((max_prims + 255) / 256 < 4096 ? (max_prims + 255) / 256 : 4096), n_inst);
    if (grid.x == 0) grid.x = 1;
    k_mark<<<grid, 256, 0, stream>>>(acc->d_grids, n_inst, d_aabb, e, acc->d_table);
    CT_TRY(cudaGetLastError());
    uint32_t cb = (uint32_t)((total_cells + 255) / 256 < 8192 ? (total_cells + 255) / 256 : 8192);
    k_assign_slots<<<cb ? cb : 1, 256, 0, stream>>>(acc->d_table, acc->d_pslot, (uint32_t)total_cells, d_counter);
    CT_TRY(cudaGetLastError());
    CT_TRY(cudaMemcpyAsync(counts, d_counter, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    CT_TRY(cudaStreamSynchronize(stream));
    n_slots = counts[0];
    n_pslots = counts[1];
    const uint32_t ns = n_slots ? n_slots : 1, nps = n_pslots ? n_pslots : 1;
    CT_TRY(cudaMalloc(&acc->d_mask, sizeof(uint32_t) * CT_MASK_WORDS * (uint64_t)ns));
    CT_TRY(cudaMemsetAsync(acc->d_mask, 0, sizeof(uint32_t) * CT_MASK_WORDS * (uint64_t)ns, stream));
    CT_TRY(cudaMalloc(&acc->d_prim, sizeof(uint32_t) * 512ull * nps));
    CT_TRY(cudaMemsetAsync(acc->d_prim, 0xFF, sizeof(uint32_t) * 512ull * nps, stream));
    k_fill<<<grid, 256, 0, stream>>>(acc->d_grids, n_inst, d_aabb, e, acc->d_table, acc->d_pslot, acc->d_mask,
                                     acc->d_prim, acc->d_vcoord);
    CT_TRY(cudaGetLastError());
    CT_TRY(build_cell_field(acc, total_cells, stream));
    CT_TRY(cudaMemsetAsync(d_counter, 0, sizeof(uint32_t), stream));
    const uint64_t words = (uint64_t)CT_MASK_WORDS * n_slots;
    const uint32_t vb = (uint32_t)((words + 255) / 256 < 4096 ? (words + 255) / 256 : 4096);
    k_count_voxels<<<vb ? vb : 1, 256, 0, stream>>>(acc->d_mask, n_slots, d_counter);
    CT_TRY(cudaGetLastError());
    CT_TRY(cudaMemcpyAsync(&acc->info.voxel_count, d_counter, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
  }
  acc->dev.grids = acc->d_grids;
  acc->dev.n_grids = n_inst;
  acc->dev.extent = e;
  acc->dev.brick_table = acc->d_table;
  acc->dev.brick_mask = acc->d_mask;
  acc->dev.brick_pslot = acc->d_pslot;
  acc->dev.brick_prim = acc->d_prim;
  acc->dev.cell_field = acc->d_field;
  acc->dev.voxel_coord = acc->d_vcoord;
  acc->dev.aabbs = d_aabb;
  acc->dev.max_steps = CT_DDA_MAX_STEPS;
  acc->info.instance_count = n_inst;
  acc->info.brick_count = n_pslots;
  acc->info.device_bytes = sizeof(DevGrid) * n_inst + 8ull * total_cells + 2048ull * total_cells + 64ull * n_slots +
                           2048ull * n_pslots +
                           4ull * scene->aabb_count;
  CT_TRY(cudaStreamSynchronize(stream));  // also lands info.voxel_count
  cudaFree(d_b);
  cudaFree(d_counter);
  *out = acc;
  return CT_OK;
fail:
  cudaFree(d_b);
  cudaFree(d_counter);
  delete acc;
  return st;
}

extern "C" ct_status ct_accel_free(ct_accel *acc) {
  if (!acc) return CT_ERR_INVALID_ARG;
  delete acc;
  return CT_OK;
}

extern "C" ct_status ct_accel_get_info(const ct_accel *acc, ct_accel_info *out) {
  if (!acc || !out) return CT_ERR_INVALID_ARG;
  *out = acc->info;
  return CT_OK;
}

// one octant of a grid's cell field, decoded to an edge per cell (the walk's
// cell_field lookup, cell by cell)
__global__ void k_field_unpack(const uint32_t *field, uint64_t word0, uint32_t octant, uint32_t X, uint32_t Y,
                               uint32_t Z, uint8_t *out) {
  const uint64_t n = (uint64_t)X * Y * Z;
  for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < n; c += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t x = (uint32_t)(c % X), y = (uint32_t)((c / X) % Y), z = (uint32_t)(c / ((uint64_t)X * Y));
    const uint64_t w = word0 + (((uint64_t)octant * Z + z) * Y + y) * (X / 8u) + (x >> 3);
    out[c] = (uint8_t)ct_field_edge((field[w] >> ((x & 7u) * 4u)) & 15u);
  }
}

extern "C" ct_status ct_accel_field(const ct_accel *acc, uint32_t instance, uint32_t octant, uint8_t *edges,
                                    int32_t grid_min[3], uint32_t cells[3], ct_stream stream) {
  if (!acc || !grid_min || !cells || octant >= 8u || instance >= acc->h_grids.size()) return CT_ERR_INVALID_ARG;
  const DevGrid &g = acc->h_grids[instance];
  const uint32_t X = (uint32_t)g.bdim[0] * CT_BRICK, Y = (uint32_t)g.bdim[1] * CT_BRICK,
                 Z = (uint32_t)g.bdim[2] * CT_BRICK;
  for (int a = 0; a < 3; a++) grid_min[a] = g.gmin[a];
  cells[0] = X;
  cells[1] = Y;
  cells[2] = Z;
  if (!edges) return CT_OK;
  const uint64_t n = (uint64_t)X * Y * Z;
  if (n == 0) return CT_OK;
  const uint64_t want = (n + 255) / 256;
  k_field_unpack<<<(uint32_t)(want < 8192 ? want : 8192), 256, 0, (cudaStream_t)stream>>>(
      acc->d_field, g.field_offset, octant, X, Y, Z, edges);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CT_OK : cuda_fail(e);
}
