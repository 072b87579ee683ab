// Internal structures shared by the device kernels (lbm_kernels.cu) and the
// host context (octlb_ctx.cu).  Not part of the C ABI.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "lbm_common.cuh"

namespace octlb_gpu {

// One octree level on the device.  Every block is a padded (n+2)^3 box with a
// one-cell halo (the reference's BlockLattice layout, block_lattice.h:294-304),
// stored structure-of-arrays: population i of slot s lives at
// pops[i * qs + s], slot s = b * bstride + (hx * np + hy) * np + hz.  A single
// periodic block drops the halo (np = n) and wraps its pull indices instead.
struct StepArgs {
  const void* src;
  void* dst;
  long long qs;             // elements between population planes
  const uint8_t* flags;     // [slots] kind + role bits
  const int* link_idx;      // [slots] link record index (read if kFlagLink)
  const float* link_rec;    // [n_links][38]: q[19], dw[19]
  const int* save_idx;      // [slots] save slot (read if kFlagSave)
  float* save_buf;          // [n_save][19] pre-collision populations
  const int* open_blocks;   // blocks whose halo is torus-streamed
  const int* halo_map;      // [n_halo] halo slot offsets inside one block
  int n_open, n_halo;
  int nblk, n, np;
  long long bstride, plane; // slots per block, per x-slice
  uint32_t ncore;           // nblk * n^3 core work items
  uint32_t nitems;          // ncore + n_open * n_halo
  FastDiv div_n, div_n2, div_n3, div_halo;
  float omega, scale, inv_scale;
  int off[kQ];              // slot offset of c_i: cx*plane + cy*np + cz
  int* err;                 // device error word (bounded waits that gave up)
};

// Device error codes written to StepArgs::err.
enum : int { kErrNone = 0, kErrBulkTimeout = 1 };

// Rectangular halo copy (same-level face / edge exchange, outflow ghost copy):
// dst(a,b) <- src(a,b) for all 19 populations.
struct CopyDesc {
  long long src, dst;       // first slot
  int n0, n1;
  int s0, s1, d0, d1;       // slot strides along the two region axes
};
// Single-population halo write: pops[pop][dst] = pops[src_pop][src] + add
// (bounce-back wall: src_pop = opp(pop); outflow ghost copy: src_pop = pop).
struct BBOp {
  long long dst, src;
  int pop, src_pop;
  float add;
  int pad;
};

// Lagrava prolongation item (level_coupler.cpp:438-478): a fine core cell
// written from a coarse interface cell's saved pre-collision populations.
struct ProlongItem {
  long long fine_slot;
  int coarse_save;          // row of the coarse level's save buffer
  int prev;                 // row of the prev-macro store (23 floats)
  int fine_kind;
  int pad;
};
// Lagrava restriction item (level_coupler.cpp:613-654).
struct RestrictItem {
  long long coarse_slot;
  int fine_save;            // save row of the fine interface cell
  int nnb;                  // in-block D3Q19 neighbours (<= 18)
  int nb_save[18];
  int coarse_kind;
  int pad;
};
// MEM drag cell: kBulk core cell with at least one obstacle link; bit i of
// mask set when x + c_i is an in-block solid / Bouzidi obstacle cell
// (drag_postprocessor.h:86-110).
struct DragItem {
  long long slot;
  uint32_t mask;
  int pad;
};

}  // namespace octlb_gpu
