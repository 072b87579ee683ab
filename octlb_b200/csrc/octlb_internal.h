// Internal structures shared by the device kernels (lbm_kernels.cu) and the
// host context (octlb_ctx.cu).  Not part of the C ABI.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "lbm_common.cuh"

namespace octlb_gpu {

// One octree level on the device.  Every block's n^3 core cells are stored
// compactly, structure of arrays: population i of slot s at pops[i * qs + s],
// core slot s = block * n^3 + (x * n + y) * n + z.  The reference's one-cell
// halo (block_lattice.h:294-304) is not stored per block: a pull whose source
// lies in the halo is resolved through the block's 27-entry base table to the
// same-level neighbour's core cell that GhostSchedule would have copied there
// (faces, and edges composed from two faces, ghost_schedule.h:56-95).  Blocks
// whose halo is written by a tree-boundary fill, or whose halo carries the
// reference's torus stream because no exchange fills it, own a halo page of
// (n+2)^3 - n^3 slots after all cores (slot halo_base + page * n_halo + hmap).
// A single periodic block resolves every halo direction to itself.
struct StepArgs {
  const void* src;
  void* dst;
  long long qs;             // slots per population plane (cores + halo pages)
  const uint8_t* flags;     // [ncore] kind + role bits
  const int* link_idx;      // [ncore] link record index (read if kFlagLink)
  const float* link_rec;    // [n_links][38]: q[19], dw[19]
  const int* save_idx;      // [ncore] save row (read if kFlagSave)
  float* save_buf;          // [n_save][19] pre-collision populations
  const long long* nbase;   // [nblk][27] slot base of the halo direction (or kOwnPage)
  const int* page_of;       // [nblk] halo page or -1
  const int* hmap;          // [(n+2)^3] padded position -> halo index (-1 in the core)
  const int* hpos;          // [n_halo] halo index -> padded linear position
  const int* open_pages;    // [n_open][4] torus-streamed halo items: page, block, halo index, population
  const int* slot_map;      // [nblk][(n+2)^3] slot of every padded position (k_step_map levels)
  const int* fill_of;       // [n_pages * n_halo][19] boundary fill writing (page slot, population), or -1
  const struct BBOp* fills; // the fills (never materialised: readers take the source, pull_value)
  const float* wall_add;    // [k][19] wall terms of slot-map marker -(2 + k) (moving bounce-back wall)
  const float* wall_dadd;   // [k][19] their derivative by the wall-velocity scale
  const uint8_t* blk_moving; // [nblk] 1 where the block's slot map holds a moving-wall marker
  int n_open, n_halo;       // items, halo slots per page
  int nblk, n, np;          // np = n + 2
  long long halo_base;      // first halo-page slot (= nblk * n^3)
  uint32_t ncore;           // nblk * n^3 core work items
  uint32_t nitems;          // ncore + n_open
  FastDiv div_n, div_n2, div_n3, div_halo, div_np, div_np2;
  float omega, scale, inv_scale;
  int off[kQ];              // core slot offset of c_i: cx*n*n + cy*n + cz
  int off_pad[kQ];          // padded linear offset of c_i: cx*np*np + cy*np + cz
  // ConstRhoBGK (null for BGK): the average density the collide uses, and
  // per-CTA partial sums of rho - 1 over the kBulk cells it collided
  const double* cr_avg;
  double* cr_part;
  int cr_total;             // partials the average update sums
  int* err;                 // device error word (bounded waits that gave up)
  // Periodic block (paired step): the x plane a cell at x = 0 pulls from for
  // c_x = +1 and the one a cell at x = n - 1 pulls from for c_x = -1 -- n - 1
  // and 0 for a block periodic in itself, the two ghost planes after the core
  // (n and n + 1) for an x slab of a periodic box shared over ranks.
  int wrap_lo, wrap_hi;
  unsigned long long wait_ns; // limit of every bounded device wait
  int stall_first_row;      // test of the bounded wait: CTA 0 never issues its first row
  // Readers of an AA-order box after an odd number of steps: population i of
  // cell x sits in plane opp(i) at the periodic neighbour x + c_i.
  int aa_rev;
};

// AA-order box after an odd number of steps: the slot holding population i
// of core slot t, in plane opp(i) -- the periodic neighbour t + c_i of the
// single block.
__device__ __forceinline__ long long aa_rev_slot(const StepArgs& a, int i, uint32_t t) {
  const uint32_t n = a.n;
  const uint32_t x = a.div_n2.div(t), r = t - x * n * n, y = a.div_n.div(r), z = r - y * n;
  const uint32_t xs = cx(i) > 0 ? (x + 1 == n ? 0 : x + 1) : (cx(i) < 0 ? (x == 0 ? n - 1 : x - 1) : x);
  const uint32_t ys = cy(i) > 0 ? (y + 1 == n ? 0 : y + 1) : (cy(i) < 0 ? (y == 0 ? n - 1 : y - 1) : y);
  const uint32_t zs = cz(i) > 0 ? (z + 1 == n ? 0 : z + 1) : (cz(i) < 0 ? (z == 0 ? n - 1 : z - 1) : z);
  return static_cast<long long>(opp(i)) * a.qs + (static_cast<long long>(xs) * n + ys) * n + zs;
}

// Cells flagged kFlagNear with the link rule resolved on the host: for near
// cell k and direction i (arrays [kQ][n]), the slot whose population i the
// rule reads (the pull source, the Bouzidi neighbour x + c_i, or the cell
// itself), and for directions set in mask[k] the link coefficients q (1 =
// half-way bounce-back) and the added moving-wall term (-0 when the cell has
// no link record: an exact no-op).
struct NearTables {
  const int* cells;         // [n] core slot
  const uint32_t* mask;     // [n] bit i: direction i takes the link rule
  const int* slot;          // [kQ][n]
  const float* q;           // [kQ][n]
  const float* add;         // [kQ][n]
  int n;
};

constexpr long long kOwnPage = -(1LL << 62);

// Device error codes written to StepArgs::err.
// kErrBulkDrainTimeout: a CTA that gave up could not see its own copies in
// flight land either, so shared memory may still be written after it exited.
enum : int { kErrNone = 0, kErrBulkTimeout = 1, kErrHalo = 2, kErrBulkDrainTimeout = 3 };

// Tree-boundary fill of one halo-page population: value(dst, pop) =
// g_src_pop(src) + add (bounce-back wall: src_pop = opp(pop); outflow ghost
// copy: src_pop = pop).  Never stored: readers evaluate it (pull_value).
struct BBOp {
  long long dst, src;
  int pop, src_pop;
  float add;
  float dadd;               // d add / d (velocity scale of the moving walls)
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
// Operands of one coupler launch (k_couple): a prolongation and up to two
// restrictions, each on its own range of CTAs (n = 0: absent).
struct ProlongOp {
  const ProlongItem* items;
  int n, half;
  const float* coarse_save;
  float* prev;
  float* rec_prev;          // the adjoint's record of the prev rows read (half time), or null
  void* fine;
  long long fine_qs;
  float scale, omega, fscale;
  // collide of a kBulk target (kCollBgk, kCollNone, or kCollConstRho at
  // *cr_avg with each prolongation CTA's sum of rho - 1 in cr_part[CTA])
  int cmode;
  const double* cr_avg;
  double* cr_part;
};
struct RestrictOp {
  const RestrictItem* items;
  int n;
  const float* fine_save;
  void* coarse;
  long long coarse_qs;
  float scale, omega, cscale;
  int cmode;                // collide of a kBulk target: kCollBgk or kCollNone
};
// MEM drag cell: kBulk core cell with at least one obstacle link; bit i of
// mask set when x + c_i is an in-block solid / Bouzidi obstacle cell
// (drag_postprocessor.h:86-110).
struct DragItem {
  long long slot;
  uint32_t mask;
  int pad;
};

// Finite-difference domain boundary pass (lbm_fd.cu): one record per
// velocity- or pressure-Dirichlet cell (its row), with every read of its
// stencil resolved on the host.  Velocity reads: kFdZero (the overlap padding
// at rest, or a pressure cell on an edge or corner of its block), kFdFluid (idx = slot: the velocity of the populations there),
// kFdPrescribed (idx = row: that boundary cell's prescribed velocity); flip
// bit a negates component a (a mirror image across face a).  Density reads:
// kFdRhoConst (val: a pressure cell's target density, 1 on its block's edges
// and corners and in the padding), 1 + sum f of the populations before the pass (idx =
// slot) or of a rewritten row (idx = row), or velocityBMRho of either with
// face (d, o) and the prescribed velocity of row urow.
enum : int { kFdZero = 0, kFdFluid = 1, kFdPrescribed = 2 };
enum : int { kFdRhoConst = 0, kFdRhoSumPre = 1, kFdRhoSumNew = 2, kFdRhoBmPre = 3, kFdRhoBmNew = 4 };
struct FdURead {
  long long idx;
  int code, flip;
};
struct FdRRead {
  long long idx;
  float val;
  int code, urow, d, o;
};
struct FdCell {
  long long slot;
  int kind, role;             // role 1 plane, 2 edge, 3 corner (faces of its block it lies on)
  int d, o;                   // plane: the face's axis and side (-1 / +1)
  int ax[3];                  // edge: the edge's own axis, then the two normal axes d1, d2
  int nrm[3];                 // edge: sides along d1, d2; corner: sides along x, y, z
  float u_base[3];            // prescribed velocity before the inlet ramp
  float ramp_end;             // inlet ramp length in steps (0: no ramp)
  float rho_target;           // pressure plane cell: the face's target density
  FdURead u[7];               // velocity reads (order fixed per role, lbm_fd.cu)
  FdRRead r[6];               // density reads (edges 4, corners 6)
};

}  // namespace octlb_gpu
