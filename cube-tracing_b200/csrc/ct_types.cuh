// ct_types.cuh -- layout of a built acceleration structure, shared by the
// builder and the frame kernels.
#pragma once
#include <cstdint>
#include "ct.h"
#include "ct_math.cuh"

#define CT_EMPTY_SLOT 0x7FFFFFFFu
#define CT_NEAR_BIT 0x80000000u
#define CT_BRICK 8
#define CT_MASK_WORDS 16u  // occupancy words per NEAR brick
#define CT_DDA_MAX_STEPS (1 << 16)
#define CT_SAMPLER_MAX_TRIES 4096

// ---------------------------------------------------------------------------
// acceleration structure (built by ct_build_accel)
//
// Per instance: a grid of 8x8x8-voxel bricks covering the instance's voxel
// bounds plus a one-voxel empty margin.  A brick is NEAR when a voxel lies
// inside it or touches it (26-neighbourhood); bricks that are not NEAR are
// skipped whole.
//   brick_table[cell]  CT_NEAR_BIT | mask slot (CT_EMPTY_SLOT when not NEAR)
//   brick_mask[slot]   CT_MASK_WORDS words (64 B): the occupancy bits, bit
//                      index = x + 8y + 64z inside the brick
//   brick_pslot[cell]  slot of the brick's 512 primitive ids (CT_EMPTY_SLOT
//                      when the brick has no voxel of its own)
//   brick_prim[pslot*512 + bit]  lowest primitive id of the voxel
//   cell_field[field_offset + ((octant * Z + z) * Y + y) * (X / 8) + x / 8]
//                      for every cell (x, y, z) of the grid (X x Y x Z cells)
//                      and ray octant (bit 0: x decreasing, bit 1: y, bit 2:
//                      z), 4 bits (nibble x & 7): the edge k of the largest
//                      cube without occupied cells that has the cell as its
//                      corner and extends k cells in the octant's
//                      directions, the part beyond the grid not counted,
//                      as a 4-bit code (ct_field_edge: 0 = occupied)
// The edge of each 4-bit cell_field code, one byte per code, codes 4i to
// 4i + 3 in CT_FIELD_EDGES<i>: 0-10, 12, 15, 19, 24, 30.  A cell stores the
// largest code whose edge does not exceed its cube's edge.  Edges up to 30
// instead of 0-15 cut the shadow-ray steps of the DI spatial rounds at 1080p
// from 8.48 to 7.80 per ray, and the walker from 5.06 to 4.86 ms per frame;
// the build's extra pass (k_field_grow) costs 1.4 ms.
#ifndef CT_FIELD_EDGES0
#define CT_FIELD_EDGES0 0x03020100u
#define CT_FIELD_EDGES1 0x07060504u
#define CT_FIELD_EDGES2 0x0C0A0908u
#define CT_FIELD_EDGES3 0x1E18130Fu
#endif
#define CT_FIELD_MAX_EDGE ((int)(CT_FIELD_EDGES3 >> 24))
__device__ __forceinline__ int ct_field_edge(uint32_t code) {
  // byte (code & 7) of the code's half of the table
  const bool lo = code < 8u;
  return (int)(__byte_perm(lo ? CT_FIELD_EDGES0 : CT_FIELD_EDGES2, lo ? CT_FIELD_EDGES1 : CT_FIELD_EDGES3, code & 7u) &
               255u);
}

struct DevGrid {
  m4 world2obj_tlas;   // inverse of the instance transform with row 3 = (0,0,0,1)
  m4 obj2world_tlas;
  m4 world2obj_inst;   // inverse of the full INSTANCE.transform
  int32_t gmin[3];     // voxel coordinate of the grid's first voxel
  int32_t bdim[3];     // bricks per axis
  uint32_t table_offset;
  uint32_t first_primitive_index;
  uint32_t primitive_count;
  uint32_t grid_exact; // voxel centres recomputable from integer coordinates
  uint64_t field_offset;  // first cell_field word of the grid
};

struct DevAccel {
  const DevGrid *grids;
  uint32_t n_grids;
  float extent;
  const uint32_t *brick_table;
  const uint32_t *brick_mask;
  const uint32_t *brick_pslot;
  const uint32_t *brick_prim;
  const uint32_t *cell_field;
  const uint32_t *voxel_coord;  // per primitive (global index): packed local voxel coordinate, for targets
  const ct_aabb *aabbs;         // the caller's AABB buffer (voxel centres of grids that are not exact)
  uint32_t max_steps;           // cells per walk before CT_ERR_ITER_LIMIT (CT_DDA_MAX_STEPS, or a test's cap)
};

