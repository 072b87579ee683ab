// sm_100a kernels of the per-level LBM time step.
//
//   k_step      fused pull-stream + BGK collide over one level (K1), with the
//               reference's two stream rules (torus rotate / per-cell links
//               with half-way bounce-back and Bouzidi, K2), moving-wall term,
//               halo torus-stream of open blocks, and pre-collision save of
//               coupler source cells.
//   (no ghost kernel: a same-level halo position is read from the neighbour's
//               core through the slot map, a tree-boundary fill target from
//               its fill's source, pull_value)
//   k_prolong   Lagrava prolongation (K4), k_restrict Lagrava restriction (K5).
//   k_drag      momentum-exchange force (K6), FP64 with warp shuffles.
//   k_audit     FP64 mass / momentum audit and non-finite check.
//
// Storage is the shifted population g = f - w after collision ("post-collide"
// state): one launch of k_step reads g_n, pulls f_{n+1} = S(g_n), and writes
// g_{n+1} = C(f_{n+1}).  The reference's per-step order collide -> exchange ->
// stream (time_loop.h:201-217) is therefore a ghost fill followed by k_step.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <type_traits>

#include "lbm_device.cuh"

namespace octlb_gpu {

namespace {

// Source slots of the 19 pulls of core cell c (local index tl inside its
// block, global slot t): direction i reads padded position x + 1 - c_i.  The
// halo direction of each source follows from which block faces the cell
// touches, so a boundary cell costs one table read per direction (from the
// CTA's shared copy of the block's 27 bases when `sb` is given).
__device__ __forceinline__ void source_slots(const StepArgs& a, const Cell& c, long long t, long long tl,
                                             const long long* sb, long long (&s)[kQ], uint32_t& halo_mask) {
  const uint32_t n1 = a.n - 1;
  const bool xl = c.x == 0, xh = c.x == n1, yl = c.y == 0, yh = c.y == n1, zl = c.z == 0, zh = c.z == n1;
  halo_mask = 0;
  if (!(xl | xh | yl | yh | zl | zh)) {
#pragma unroll
    for (int i = 0; i < kQ; ++i) s[i] = t - a.off[i];
    return;
  }
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    const int ox = (cx(i) == 1 && xl) ? -1 : ((cx(i) == -1 && xh) ? 1 : 0);
    const int oy = (cy(i) == 1 && yl) ? -1 : ((cy(i) == -1 && yh) ? 1 : 0);
    const int oz = (cz(i) == 1 && zl) ? -1 : ((cz(i) == -1 && zh) ? 1 : 0);
    if ((ox | oy | oz) == 0) {
      s[i] = t - a.off[i];
    } else {
      halo_mask |= 1u << i;
      const int d = (ox + 1) * 9 + (oy + 1) * 3 + (oz + 1);
      const long long base = sb ? sb[d] : a.nbase[c.b * 27 + d];
      s[i] = base != kOwnPage
                 ? base + tl - a.off[i]
                 : page_slot(a, c.b, static_cast<int>(c.x) + 1 - cx(i), static_cast<int>(c.y) + 1 - cy(i),
                             static_cast<int>(c.z) + 1 - cz(i));
    }
  }
}

// The 19 populations of cell t copied unchanged; all loads are issued
// before the first store (for all the compiler knows, a store to row i may
// alias the load from row i + 1, which would cost a round trip each).
template <typename T>
__device__ __forceinline__ void copy_cell(const T* src, T* dst, long long qs, uint32_t t) {
  T v[kQ];
#pragma unroll
  for (int i = 0; i < kQ; ++i) v[i] = src[i * qs + t];
#pragma unroll
  for (int i = 0; i < kQ; ++i) dst[i * qs + t] = v[i];
}

// Torus-streamed halo population of an open block (block_lattice.h:70-89),
// item k: copied without collision.
template <typename T>
__device__ __forceinline__ void rotate_item(const StepArgs& a, uint32_t k) {
  if (k >= static_cast<uint32_t>(a.n_open)) return;
  long long d, sl;
  int i;
  rotate_slots(a, k, d, sl, i);
  const T* src = static_cast<const T*>(a.src);
  T* dst = static_cast<T*>(a.dst);
  if (sl >= a.halo_base && a.fill_of && a.fill_of[(sl - a.halo_base) * kQ + i] >= 0)
    Store<T>::st(dst + i * a.qs + d, pull_value(a, src, i, sl), a.scale);  // source is a boundary fill
  else
    dst[i * a.qs + d] = src[i * a.qs + sl];
}

// ConstRhoBGK statistics of a step launch: this CTA's sum into
// cr_part[blockIdx.x]; CTA 0 also zeroes the partials from `written` (the
// CTAs that write one) up to cr_total, which the average update sums.
__device__ __forceinline__ void cr_store_partial(const StepArgs& a, double v0, uint32_t written) {
  double v[1] = {v0};
  block_reduce<1>(v);
  if (threadIdx.x == 0) a.cr_part[blockIdx.x] = v[0];
  if (blockIdx.x == 0)
    for (int p = static_cast<int>(written) + threadIdx.x; p < a.cr_total; p += kThreads) a.cr_part[p] = 0.0;
}

// One core cell of k_step / k_step_cr: pull, save, collide (kBulk cells:
// BGK, ConstRhoBGK with dr = 1 - average_rho, or none, by CM), store.
// Returns rho - 1 before the collision for a cell the ConstRhoBGK collided
// and a later prolongation does not overwrite, else 0.  CORR: the BGK
// collide removes its own mass / momentum rounding defect (FP32 storage of
// the uniform periodic box, as k_step_pair).
template <typename T, bool LINKS, bool FLAGS, int CM, bool CORR = false>
__device__ __forceinline__ float core_cell(const StepArgs& a, uint32_t t, const long long* sb, float dr) {
  const T* src = static_cast<const T*>(a.src);
  T* dst = static_cast<T*>(a.dst);
  const uint32_t n3 = a.n * a.n * a.n;
  const Cell c = cell_of(a, t);
  const long long tl = t - c.b * n3;
  const uint8_t fl = FLAGS ? a.flags[t] : 0;
  float f[kQ];
  if constexpr (LINKS) {
    if ((fl & kKindMask) == kSolid) {
      // Solid cells are neither streamed nor collided (block_lattice.cpp:581-583).
      copy_cell(src, dst, a.qs, t);
      return 0.f;
    }
  }
  // Cells next to walls take the link rule in k_step_near.
  if constexpr (LINKS) {
    if (fl & kFlagNear) return 0.f;
  }
  long long s[kQ];
  uint32_t halo_mask;
  source_slots(a, c, t, tl, sb, s, halo_mask);
#pragma unroll
  for (int i = 0; i < kQ; ++i) f[i] = pull_value(a, src, i, s[i]);
  float dh = 0.f;
  bool bulk = true;
  if constexpr (FLAGS) {
    if (fl & kFlagSave) {
      float* sv = a.save_buf + static_cast<long long>(a.save_idx[t]) * kQ;
#pragma unroll
      for (int i = 0; i < kQ; ++i) sv[i] = f[i];
    }
    bulk = (fl & kKindMask) == kBulk;
  }
  if (bulk) {
    if constexpr (CM == kCollConstRho) {
      dh = bgk_const_rho(f, a.omega, dr);
      if (fl & kFlagProlong) dh = 0.f;
    } else if constexpr (CM == kCollBgk) {
      bgk<CORR && kBgkCorrect<T>>(f, a.omega);
    }
  }
#pragma unroll
  for (int i = 0; i < kQ; ++i) Store<T>::st(dst + i * a.qs + t, f[i], a.scale);
  return dh;
}

// CM: kCollBgk, or kCollNone for a level whose collide runs after its
// coupling (k_collide_cr).
template <typename T, bool LINKS, bool FLAGS, bool BLOCKED, int CM = kCollBgk, bool CORR = false>
__global__ void __launch_bounds__(kThreads) k_step(const StepArgs a) {
  pdl_wait();
  const uint32_t t = blockIdx.x * kThreads + threadIdx.x;
  const uint32_t cta0 = blockIdx.x * kThreads;
  if (cta0 < a.ncore) {
    // CTAs of core cells (ncore is a multiple of the CTA size when BLOCKED,
    // and then a CTA never straddles two blocks).
    __shared__ long long sb[27];
    if constexpr (BLOCKED) {
      const uint32_t b0 = a.div_n3.div(cta0);
      if (threadIdx.x < 27) sb[threadIdx.x] = a.nbase[b0 * 27 + threadIdx.x];
      __syncthreads();
    }
    if (t >= a.ncore) return;
    core_cell<T, LINKS, FLAGS, CM, CORR>(a, t, BLOCKED ? sb : nullptr, 0.f);
    return;
  }
  // Halo items start at the first CTA after the core CTAs.
  const uint32_t core_end = ((a.ncore + kThreads - 1) / kThreads) * kThreads;
  rotate_item<T>(a, t - core_end);
}

// ConstRhoBGK step (TimeLoop with use_const_rho_bgk, time_loop.h:173-187 and
// 201-222): k_step's cells with the ConstRhoBGK collide at the average density
// *cr_avg, and each core CTA's sum of rho - 1 over the kBulk cells it
// collided in cr_part[blockIdx.x] (a fixed shuffle tree).
template <typename T, bool LINKS, bool FLAGS, bool BLOCKED>
__global__ void __launch_bounds__(kThreads) k_step_cr(const StepArgs a) {
  pdl_wait();
  const uint32_t t = blockIdx.x * kThreads + threadIdx.x;
  const uint32_t cta0 = blockIdx.x * kThreads;
  if (cta0 < a.ncore) {
    __shared__ long long sb[27];
    if constexpr (BLOCKED) {
      const uint32_t b0 = a.div_n3.div(cta0);
      if (threadIdx.x < 27) sb[threadIdx.x] = a.nbase[b0 * 27 + threadIdx.x];
      __syncthreads();
    }
    const float dr = static_cast<float>(1.0 - *a.cr_avg);
    float dh = 0.f;
    if (t < a.ncore) dh = core_cell<T, LINKS, FLAGS, kCollConstRho>(a, t, BLOCKED ? sb : nullptr, dr);
    // the near-cell CTAs of k_step_near_cr write the partials after these
    cr_store_partial(a, static_cast<double>(dh), static_cast<uint32_t>(a.cr_total));
    return;
  }
  const uint32_t core_end = ((a.ncore + kThreads - 1) / kThreads) * kThreads;
  rotate_item<T>(a, t - core_end);
}

// Cells flagged kFlagNear (links stream rule): the per-cell link rule of
// block_lattice.cpp:613-672 with every table lookup done on the host --
// direction i reads population i at nt.slot[i] and, where the rule applies,
// reflects own[opp(i)] (half-way bounce-back, reflect-on-pull at the block
// edge) or interpolates with Bouzidi (bouzidi_pull.h:8-26), then adds the
// moving-wall term.  Then the same save / collide / store as k_step.  One
// warp per cell, lane i on direction i; the collision gathers the 19 values
// so every lane computes the moments exactly as bgk() does.
template <typename T, int CM = kCollBgk>
__device__ __forceinline__ float near_cell(const StepArgs& a, const NearTables& nt, int k, int lane, float dr = 0.f) {
  if (k >= nt.n) return 0.f;
  const T* src = static_cast<const T*>(a.src);
  T* dst = static_cast<T*>(a.dst);
  const LaneDir d = lane_dir(lane);
  const uint32_t t = static_cast<uint32_t>(nt.cells[k]);
  const uint32_t mask = nt.mask[k];
  const uint8_t fl = a.flags[t];
  const int sl = d.act ? nt.slot[lane * nt.n + k] : 0;
  const float q = d.act ? nt.q[lane * nt.n + k] : 1.f, add = d.act ? nt.add[lane * nt.n + k] : 0.f;
  pdl_wait();
  const float val = d.act ? pull_value(a, src, lane, sl) : 0.f;
  const float own = d.act ? LD(src, a.qs, lane, t, a.inv_scale) : 0.f;
  const float own_opp = __shfl_sync(0xffffffffu, own, d.opp);
  float f = val;
  if (d.act && ((mask >> lane) & 1u)) f = (q < 1.0f ? bouzidi(own_opp, val, own, q) : own_opp) + add;
  if ((fl & kFlagSave) && d.act) a.save_buf[static_cast<long long>(a.save_idx[t]) * kQ + lane] = f;
  float dh = 0.f;
  if constexpr (CM != kCollNone) {
    if ((fl & kKindMask) == kBulk) {
      float fa[kQ];
      gather_lanes(f, fa);
      if constexpr (CM == kCollConstRho) {
        f = bgk_lane_const_rho(d, lane, fa, f, a.omega, dr, dh);
        if (fl & kFlagProlong) dh = 0.f;
      } else {
        f = bgk_lane<false>(d, lane, fa, f, a.omega);
      }
    }
  }
  if (d.act) Store<T>::st(dst + lane * a.qs + t, f, a.scale);
  return dh;
}

template <typename T, int CM = kCollBgk>
__global__ void __launch_bounds__(kThreads) k_step_near(const StepArgs a, const NearTables nt) {
  near_cell<T, CM>(a, nt, (blockIdx.x * kThreads + threadIdx.x) >> 5, threadIdx.x & 31);
}

// Near-wall cells under ConstRhoBGK: one warp per cell as k_step_near; each
// CTA's sum of rho - 1 over its collided kBulk cells in
// cr_part[part_off + blockIdx.x].
template <typename T>
__global__ void __launch_bounds__(kThreads) k_step_near_cr(const StepArgs a, const NearTables nt, int part_off) {
  pdl_wait();
  const float dr = static_cast<float>(1.0 - *a.cr_avg);
  const int lane = threadIdx.x & 31;
  const float dh = near_cell<T, kCollConstRho>(a, nt, (blockIdx.x * kThreads + threadIdx.x) >> 5, lane, dr);
  double v[1] = {lane == 0 ? static_cast<double>(dh) : 0.0};
  block_reduce<1>(v);
  if (threadIdx.x == 0) a.cr_part[part_off + blockIdx.x] = v[0];
}

// Two-element vector access for the paired periodic kernel.
template <typename T> struct Pair;
template <> struct Pair<float> {
  using V = float2;
  __device__ static inline void ld(const float* p, float inv, float& a, float& b) {
    const float2 v = *reinterpret_cast<const float2*>(p);
    a = v.x; b = v.y;
  }
  __device__ static inline void st(float* p, float a, float b, float) {
    *reinterpret_cast<float2*>(p) = make_float2(a, b);
  }
};
template <> struct Pair<__half> {
  __device__ static inline void ld(const __half* p, float, float& a, float& b) {
    const float2 v = __half22float2(*reinterpret_cast<const __half2*>(p));
    a = v.x; b = v.y;
  }
  __device__ static inline void st(__half* p, float a, float b, float) {
    *reinterpret_cast<__half2*>(p) = __floats2half2_rn(a, b);
  }
};

// Forest-level step with a per-block slot map: one CTA per block stages the
// block's (n+2)^3 map (padded position -> slot: own core, the neighbour core
// the same-level exchange copies, the source cell of an outflow ghost copy,
// the own halo page, or a bounce-back wall marker) in shared memory, so
// every pull is one shared-memory read and one 32-bit offset, with no
// per-direction branching at block faces.  Each thread takes cells tl and
// tl + 256 together (n^3 a multiple of 512), all 38 pulls issued before the
// two collisions.  Same arithmetic as k_step; kFlagNear cells are left to
// k_step_near, solid cells of the links rule are copied.  CTAs after the
// nblk block CTAs stream the open blocks' halo items.
template <typename T, bool LINKS, bool FLAGS>
__device__ __forceinline__ bool map_cell_prologue(const StepArgs& a, uint32_t t, const T* src, T* dst, uint8_t& fl) {
  fl = FLAGS ? a.flags[t] : 0;
  if constexpr (LINKS) {
    if ((fl & kKindMask) == kSolid) {
      // Solid cells are neither streamed nor collided (block_lattice.cpp:581-583).
      copy_cell(src, dst, a.qs, t);
      return false;
    }
    if (fl & kFlagNear) return false;
  }
  return true;
}

template <typename T, bool FLAGS, int CM = kCollBgk>
__device__ __forceinline__ float map_cell_finish(const StepArgs& a, uint32_t t, uint8_t fl, float (&f)[kQ], T* dst,
                                                 float dr = 0.f) {
  float dh = 0.f;
  bool bulk = true;
  if constexpr (FLAGS) {
    if (fl & kFlagSave) {
      float* sv = a.save_buf + static_cast<long long>(a.save_idx[t]) * kQ;
#pragma unroll
      for (int i = 0; i < kQ; ++i) sv[i] = f[i];
    }
    bulk = (fl & kKindMask) == kBulk;
  }
  if (bulk) {
    if constexpr (CM == kCollConstRho) {
      dh = bgk_const_rho(f, a.omega, dr);
      if (fl & kFlagProlong) dh = 0.f;
    } else if constexpr (CM == kCollBgk) {
      bgk<false>(f, a.omega);
    }
  }
  const uint32_t qs = static_cast<uint32_t>(a.qs);
#pragma unroll
  for (int i = 0; i < kQ; ++i) Store<T>::st(dst + (static_cast<uint32_t>(i) * qs + t), f[i], a.scale);
  return dh;
}

// With one cell per thread (CPT = 1) two CTAs share a block, each over half
// its cells, so small levels still give every SM work.  Under the links rule
// the first CTAs of the launch take the near-wall cells (one warp each), so
// they run beside the bulk instead of in a launch of their own.
//
// CM = kCollConstRho: the ConstRhoBGK collide at average density *cr_avg,
// and per near-cell and block CTA the sum of rho - 1 over its collided kBulk
// cells in cr_part[blockIdx.x] (the halo-item CTAs after them write none);
// kCollNone: no collide.
template <typename T, bool LINKS, bool FLAGS, int CPT, bool GMAP, int CM = kCollBgk>
__global__ void __launch_bounds__(kThreads, CPT == 2 ? 4 : 5) k_step_map(const StepArgs a, const NearTables nt) {
  extern __shared__ int smap_s[];  // (n+2)^3 slots of this block
  constexpr uint32_t kParts = CPT == 1 ? 2 : 1;
  const uint32_t near_ctas = LINKS ? (static_cast<uint32_t>(nt.n) + kThreads / 32 - 1) / (kThreads / 32) : 0;
  if (LINKS && blockIdx.x < near_ctas) {
    if constexpr (CM == kCollConstRho) {
      pdl_wait();
      const float dr = static_cast<float>(1.0 - *a.cr_avg);
      const float dh = near_cell<T, kCollConstRho>(a, nt, static_cast<int>(blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5)),
                                          threadIdx.x & 31, dr);
      cr_store_partial(a, (threadIdx.x & 31) == 0 ? static_cast<double>(dh) : 0.0,
                       near_ctas + static_cast<uint32_t>(a.nblk) * kParts);
    } else {
      near_cell<T, CM>(a, nt, static_cast<int>(blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5)), threadIdx.x & 31);
    }
    return;
  }
  const uint32_t bid = blockIdx.x - near_ctas;
  const uint32_t b = bid / kParts, part = bid % kParts;
  if (b >= static_cast<uint32_t>(a.nblk)) {
    pdl_wait();
    rotate_item<T>(a, (bid - a.nblk * kParts) * kThreads + threadIdx.x);
    return;
  }
  const int np = a.np, np3 = np * np * np;
  const int* gm = a.slot_map + static_cast<long long>(b) * np3;
  if constexpr (!GMAP) {
    for (int k = threadIdx.x; k < np3; k += kThreads) smap_s[k] = gm[k];
    __syncthreads();
  }
  // GMAP: the map is read through the read-only L1 path instead (no staging
  // barrier); 4 KB per block stays L1-resident for the CTA
  const int* smap = GMAP ? gm : smap_s;
  const bool moving = a.blk_moving[b] != 0;  // uniform over the CTA
  pdl_wait();
  const T* src = static_cast<const T*>(a.src);
  T* dst = static_cast<T*>(a.dst);
  const uint32_t n = a.n, n3 = n * n * n, qs = static_cast<uint32_t>(a.qs);
  const uint32_t span = n3 / kParts;
  const float dr = CM == kCollConstRho ? static_cast<float>(1.0 - *a.cr_avg) : 0.f;
  float acc = 0.f;
  for (uint32_t tl0 = part * span + threadIdx.x; tl0 < (part + 1) * span; tl0 += CPT * kThreads) {
    uint32_t t[CPT];
    int P[CPT];
    uint8_t fl[CPT];
    bool go[CPT];
    float f[CPT][kQ];
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      const uint32_t tl = tl0 + c * kThreads;
      t[c] = b * n3 + tl;
      const uint32_t x = a.div_n2.div(tl), r = tl - x * n * n, y = a.div_n.div(r);
      P[c] = (static_cast<int>(x + 1) * np + static_cast<int>(y + 1)) * np + static_cast<int>(r - y * n + 1);
      go[c] = map_cell_prologue<T, LINKS, FLAGS>(a, t[c], src, dst, fl[c]);
    }
#pragma unroll
    for (int i = 0; i < kQ; ++i) {
      const uint32_t row = static_cast<uint32_t>(i) * qs;
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        // bounce-back wall position (marker < 0): the cell's own opposite
        // population; branch-free so the 19 (or 38) loads stay independent
        const int sm = GMAP ? __ldg(smap + P[c] - a.off_pad[i]) : smap[P[c] - a.off_pad[i]];
        const uint32_t off = sm >= 0 ? row + static_cast<uint32_t>(sm) : static_cast<uint32_t>(opp(i)) * qs + t[c];
        const float v = Store<T>::ld(src + off, a.inv_scale);
        // two cells per thread: the moving-wall term inline (a separate pass
        // costs these variants registers)
        if constexpr (CPT == 2) f[c][i] = sm < -1 ? v + a.wall_add[(-sm - 2) * kQ + i] : v;
        else f[c][i] = v;
      }
    }
    if (CPT == 1 && moving) {
      // moving-wall markers (< -1) add the wall term: only blocks flagged in
      // blk_moving hold one, the others skip this pass
#pragma unroll
      for (int i = 0; i < kQ; ++i)
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
          const int sm = GMAP ? __ldg(smap + P[c] - a.off_pad[i]) : smap[P[c] - a.off_pad[i]];
          if (sm < -1) f[c][i] += a.wall_add[(-sm - 2) * kQ + i];
        }
    }
#pragma unroll
    for (int c = 0; c < CPT; ++c)
      if (go[c]) {
        if constexpr (CM == kCollConstRho) acc += map_cell_finish<T, FLAGS, CM>(a, t[c], fl[c], f[c], dst, dr);
        else map_cell_finish<T, FLAGS, CM>(a, t[c], fl[c], f[c], dst);
      }
  }
  if constexpr (CM == kCollConstRho)
    cr_store_partial(a, static_cast<double>(acc), near_ctas + static_cast<uint32_t>(a.nblk) * kParts);
}

// One periodic all-kBulk block, two consecutive z cells per thread: every
// population row is read and written with 2-element vector accesses; a z-shift
// of +-1 takes the two aligned pairs around it.  Same arithmetic as k_step.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_step_pair(const StepArgs a) {
  pdl_wait();
  const uint32_t t = blockIdx.x * kThreads + threadIdx.x;
  const uint32_t n = a.n, half = n >> 1;
  if (t >= a.ncore / 2) return;
  const uint32_t row = a.div_n.div(2 * t);  // = t / (n / 2)
  const uint32_t z = (t - row * half) * 2;
  const uint32_t x = a.div_n.div(row), y = row - x * n;
  const uint32_t xm = x == 0 ? static_cast<uint32_t>(a.wrap_lo) : x - 1;
  const uint32_t xp = x == n - 1 ? static_cast<uint32_t>(a.wrap_hi) : x + 1;
  const uint32_t ym = y == 0 ? n - 1 : y - 1, yp = y == n - 1 ? 0 : y + 1;
  const uint32_t zm2 = z == 0 ? n - 2 : z - 2, zp2 = z + 2 == n ? 0 : z + 2;
  const T* src = static_cast<const T*>(a.src);
  T* dst = static_cast<T*>(a.dst);
  float f0[kQ], f1[kQ];
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    const uint32_t sx = cx(i) == 1 ? xm : (cx(i) == -1 ? xp : x);
    const uint32_t sy = cy(i) == 1 ? ym : (cy(i) == -1 ? yp : y);
    const T* r = src + i * a.qs + (static_cast<long long>(sx) * n + sy) * n;
    if (cz(i) == 0) {
      Pair<T>::ld(r + z, a.inv_scale, f0[i], f1[i]);
    } else if (cz(i) == 1) {  // cells z, z+1 pull z-1, z
      float u, v, w;
      Pair<T>::ld(r + zm2, a.inv_scale, u, v);
      Pair<T>::ld(r + z, a.inv_scale, f1[i], w);
      f0[i] = v;
    } else {                  // cells z, z+1 pull z+1, z+2
      float u, v, w;
      Pair<T>::ld(r + z, a.inv_scale, u, f0[i]);
      Pair<T>::ld(r + zp2, a.inv_scale, f1[i], w);
      (void)u;
      (void)v;
    }
  }
  // populations stay in storage units h = s (f - w); the scale lives in bgk
  bgk<kBgkCorrect<T>>(f0, a.omega, a.scale, a.inv_scale);
  bgk<kBgkCorrect<T>>(f1, a.omega, a.scale, a.inv_scale);
  T* o = dst + static_cast<long long>(row) * n + z;
#pragma unroll
  for (int i = 0; i < kQ; ++i) Pair<T>::st(o + i * a.qs, f0[i], f1[i], a.scale);
}

// The same step for FP16-shifted storage with four consecutive z cells per
// thread: every population row is read and written with 8-byte (four-half)
// accesses, half the memory instructions per cell of the paired kernel; a
// z-shift of +-1 takes the aligned four around the cells and one half beyond
// them.  Per cell the arithmetic is the paired kernel's (conversions to and
// from half are exact / round-to-nearest alike), so the results are bitwise
// equal.  n % 4 == 0 (rows and population planes on 8-byte boundaries).

__global__ void __launch_bounds__(kThreads) k_step_quad_h(const StepArgs a) {
  pdl_wait();
  const uint32_t t = blockIdx.x * kThreads + threadIdx.x;
  const uint32_t n = a.n, q4 = n >> 2;
  if (t >= a.ncore / 4) return;
  const uint32_t row = a.div_n.div(4 * t);  // = t / (n / 4)
  const uint32_t z = (t - row * q4) * 4;
  const uint32_t x = a.div_n.div(row), y = row - x * n;
  const uint32_t xm = x == 0 ? static_cast<uint32_t>(a.wrap_lo) : x - 1;
  const uint32_t xp = x == n - 1 ? static_cast<uint32_t>(a.wrap_hi) : x + 1;
  const uint32_t ym = y == 0 ? n - 1 : y - 1, yp = y == n - 1 ? 0 : y + 1;
  const uint32_t zm1 = z == 0 ? n - 1 : z - 1, zp4 = z + 4 == n ? 0 : z + 4;
  const __half* src = static_cast<const __half*>(a.src);
  __half* dst = static_cast<__half*>(a.dst);
  float f0[kQ], f1[kQ], f2[kQ], f3[kQ];
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    const uint32_t sx = cx(i) == 1 ? xm : (cx(i) == -1 ? xp : x);
    const uint32_t sy = cy(i) == 1 ? ym : (cy(i) == -1 ? yp : y);
    const __half* r = src + i * a.qs + (static_cast<long long>(sx) * n + sy) * n;
    if (cz(i) == 0) {
      ld4h(r + z, f0[i], f1[i], f2[i], f3[i]);
    } else if (cz(i) == 1) {  // cells z..z+3 pull z-1..z+2
      float w;
      ld4h(r + z, f1[i], f2[i], f3[i], w);
      f0[i] = __half2float(r[zm1]);
    } else {                  // cells z..z+3 pull z+1..z+4
      float w;
      ld4h(r + z, w, f0[i], f1[i], f2[i]);
      f3[i] = __half2float(r[zp4]);
    }
  }
  bgk<false>(f0, a.omega, a.scale, a.inv_scale);
  bgk<false>(f1, a.omega, a.scale, a.inv_scale);
  bgk<false>(f2, a.omega, a.scale, a.inv_scale);
  bgk<false>(f3, a.omega, a.scale, a.inv_scale);
  __half* o = dst + static_cast<long long>(row) * n + z;
#pragma unroll
  for (int i = 0; i < kQ; ++i) st4h(o + i * a.qs, f0[i], f1[i], f2[i], f3[i]);
}

// FP16-shifted AA steps with four z cells per thread and 8-byte accesses,
// as k_step_quad_h (n a multiple of 128 for the pull step: a warp's 32
// threads cover 128 cells of one z row; the local step needs n % 4 == 0).
// The pull step writes back with aligned 8-byte stores: for a direction with
// c_z != 0 the thread's four slots sit one cell off its aligned quad, which
// takes three of them and one of the neighbour lane's (a warp shuffle that
// depends on that lane's reads); the warp's edge slots, whose partner lies in
// another warp, take 2-byte stores.  Every slot is still written once.
__global__ void __launch_bounds__(kThreads, 2) k_step_aa_pull_h(const StepArgs a) {
  pdl_wait();
  const uint32_t t = blockIdx.x * kThreads + threadIdx.x;
  const uint32_t n = a.n, q4 = n >> 2;
  if (t >= a.ncore / 4) return;  // whole warps
  const int lane = threadIdx.x & 31;
  const uint32_t row = a.div_n.div(4 * t);
  const uint32_t z = (t - row * q4) * 4;
  const uint32_t x = a.div_n.div(row), y = row - x * n;
  const uint32_t xm = x == 0 ? n - 1 : x - 1, xp = x == n - 1 ? 0 : x + 1;
  const uint32_t ym = y == 0 ? n - 1 : y - 1, yp = y == n - 1 ? 0 : y + 1;
  const uint32_t zm1 = z == 0 ? n - 1 : z - 1, zp4 = z + 4 == n ? 0 : z + 4;
  __half* pops = static_cast<__half*>(a.dst);  // == a.src
  float f0[kQ], f1[kQ], f2[kQ], f3[kQ];
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    const uint32_t sx = cx(i) == 1 ? xm : (cx(i) == -1 ? xp : x);
    const uint32_t sy = cy(i) == 1 ? ym : (cy(i) == -1 ? yp : y);
    const __half* r = pops + i * a.qs + (static_cast<long long>(sx) * n + sy) * n;
    if (cz(i) == 0) {
      ld4h(r + z, f0[i], f1[i], f2[i], f3[i]);
    } else if (cz(i) == 1) {  // cells z..z+3 pull z-1..z+2
      float w;
      ld4h(r + z, f1[i], f2[i], f3[i], w);
      f0[i] = __half2float(r[zm1]);
    } else {                  // cells z..z+3 pull z+1..z+4
      float w;
      ld4h(r + z, w, f0[i], f1[i], f2[i]);
      f3[i] = __half2float(r[zp4]);
    }
  }
  bgk<false>(f0, a.omega, a.scale, a.inv_scale);
  bgk<false>(f1, a.omega, a.scale, a.inv_scale);
  bgk<false>(f2, a.omega, a.scale, a.inv_scale);
  bgk<false>(f3, a.omega, a.scale, a.inv_scale);
#pragma unroll
  for (int k = 0; k < kQ; ++k) {
    const uint32_t sx = cx(k) == 1 ? xm : (cx(k) == -1 ? xp : x);
    const uint32_t sy = cy(k) == 1 ? ym : (cy(k) == -1 ? yp : y);
    __half* r = pops + k * a.qs + (static_cast<long long>(sx) * n + sy) * n;
    const int o = opp(k);
    const float o0 = f0[o], o1 = f1[o], o2 = f2[o], o3 = f3[o];
    if (cz(k) == 0) {         // own slots z..z+3: the aligned quad
      st4h(r + z, o0, o1, o2, o3);
    } else if (cz(k) == 1) {  // own z-1..z+2: quad (z..z+3) = (own[1..3], next lane's own[0])
      const float nx = __shfl_down_sync(0xffffffffu, o0, 1);
      if (lane < 31) {
        st4h(r + z, o1, o2, o3, nx);
      } else {
        r[z] = __float2half_rn(o1);
        r[z + 1] = __float2half_rn(o2);
        r[z + 2] = __float2half_rn(o3);
      }
      if (lane == 0) r[zm1] = __float2half_rn(o0);
    } else {                  // own z+1..z+4: quad (z..z+3) = (previous lane's own[3], own[0..2])
      const float pv = __shfl_up_sync(0xffffffffu, o3, 1);
      if (lane > 0) {
        st4h(r + z, pv, o0, o1, o2);
      } else {
        r[z + 1] = __float2half_rn(o0);
        r[z + 2] = __float2half_rn(o1);
        r[z + 3] = __float2half_rn(o2);
      }
      if (lane == 31) r[zp4] = __float2half_rn(o3);
    }
  }
}

__global__ void __launch_bounds__(kThreads) k_step_aa_local_h(const StepArgs a) {
  pdl_wait();
  const uint32_t t = blockIdx.x * kThreads + threadIdx.x;
  if (t >= a.ncore / 4) return;
  __half* pops = static_cast<__half*>(a.dst);  // == a.src
  const long long s = 4ll * t;
  float f0[kQ], f1[kQ], f2[kQ], f3[kQ];
#pragma unroll
  for (int i = 0; i < kQ; ++i) ld4h(pops + opp(i) * a.qs + s, f0[i], f1[i], f2[i], f3[i]);
  bgk<false>(f0, a.omega, a.scale, a.inv_scale);
  bgk<false>(f1, a.omega, a.scale, a.inv_scale);
  bgk<false>(f2, a.omega, a.scale, a.inv_scale);
  bgk<false>(f3, a.omega, a.scale, a.inv_scale);
#pragma unroll
  for (int i = 0; i < kQ; ++i) st4h(pops + i * a.qs + s, f0[i], f1[i], f2[i], f3[i]);
}

// AA stream order on a uniform periodic box: one population buffer, updated
// in place by two alternating steps (Bailey et al. 2009).  Both pull the
// same values as k_step_pair and collide with the same bgk() call, so the
// results equal the two-buffer order's bitwise.
//
// From the natural layout (plane i at cell x): each cell pulls population i
// from x - c_i in plane i, collides, and writes each result back into a slot
// it read -- the slot read for direction k receives g_opp(k).  Every slot is
// read and written by exactly one cell (x - c_k, plane k belongs to x), so
// the update is race-free in place and leaves the reversed layout: g_i of
// cell x in plane opp(i) at x + c_i.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_step_aa_pull(const StepArgs a) {
  pdl_wait();
  const uint32_t t = blockIdx.x * kThreads + threadIdx.x;
  if (t >= a.ncore) return;
  const uint32_t n = a.n;
  const uint32_t x = a.div_n2.div(t), r = t - x * n * n, y = a.div_n.div(r), z = r - y * n;
  const uint32_t xm = x == 0 ? n - 1 : x - 1, xp = x == n - 1 ? 0 : x + 1;
  const uint32_t ym = y == 0 ? n - 1 : y - 1, yp = y == n - 1 ? 0 : y + 1;
  const uint32_t zm = z == 0 ? n - 1 : z - 1, zp = z == n - 1 ? 0 : z + 1;
  T* pops = static_cast<T*>(a.dst);  // == a.src
  long long at[kQ];
  float f[kQ];
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    const uint32_t sx = cx(i) == 1 ? xm : (cx(i) == -1 ? xp : x);
    const uint32_t sy = cy(i) == 1 ? ym : (cy(i) == -1 ? yp : y);
    const uint32_t sz = cz(i) == 1 ? zm : (cz(i) == -1 ? zp : z);
    at[i] = i * a.qs + (static_cast<long long>(sx) * n + sy) * n + sz;
    f[i] = Store<T>::ld(pops + at[i], 1.0f);  // storage units, as k_step_pair
  }
  bgk<kBgkCorrect<T>>(f, a.omega, a.scale, a.inv_scale);
#pragma unroll
  for (int k = 0; k < kQ; ++k) Store<T>::st(pops + at[k], f[opp(k)], 1.0f);
}

// From the reversed layout: population i of cell x (streamed) is the value
// in plane opp(i) at x itself; collide, and write plane i at x -- the
// natural layout again.  Two z cells per thread with 2-element accesses.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_step_aa_local(const StepArgs a) {
  pdl_wait();
  const uint32_t t = blockIdx.x * kThreads + threadIdx.x;
  if (t >= a.ncore / 2) return;
  T* pops = static_cast<T*>(a.dst);  // == a.src
  const long long s = 2ll * t;
  float f0[kQ], f1[kQ];
#pragma unroll
  for (int i = 0; i < kQ; ++i) Pair<T>::ld(pops + opp(i) * a.qs + s, a.inv_scale, f0[i], f1[i]);
  bgk<kBgkCorrect<T>>(f0, a.omega, a.scale, a.inv_scale);
  bgk<kBgkCorrect<T>>(f1, a.omega, a.scale, a.inv_scale);
#pragma unroll
  for (int i = 0; i < kQ; ++i) Pair<T>::st(pops + i * a.qs + s, f0[i], f1[i], a.scale);
}

// Body force: the forcing term 3 w_i (c_i . F) added to the stored
// (post-collision) populations of kBulk core cells at the start of each level
// step, before the boundary fills read them.  F is SoA [3][ncore].
template <typename T>
__global__ void __launch_bounds__(kThreads) k_add_force(const StepArgs a, T* pops, const float* force) {
  const uint32_t t = blockIdx.x * kThreads + threadIdx.x;
  if (t >= a.ncore) return;
  const int kind = a.flags ? (a.flags[t] & kKindMask) : kBulk;
  const float fx = force[t], fy = force[a.ncore + t], fz = force[2ull * a.ncore + t];
  pdl_wait();
  if (kind != kBulk) return;
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    const float v = LD(pops, a.qs, i, t, a.inv_scale) + 3.0f * wf(i) * (cx(i) * fx + cy(i) * fy + cz(i) * fz);
    Store<T>::st(pops + i * a.qs + t, v, a.scale);
  }
}


// Lagrava prolongation (level_coupler.cpp:455-476), one warp per item, lane
// i on population i: every lane gathers the coarse save row and forms the
// macro state with the same operations as read_macro (so the result does not
// depend on the lane layout), then writes its own population.  Parallel
// lanes keep the item's dependent chain short: the launch is latency-bound
// (a few thousand items).
template <typename T>
__device__ __forceinline__ float prolong_warp(const ProlongOp& op, int w, int lane) {
  if (w >= op.n) return 0.f;  // whole warps
  const ProlongItem it = op.items[w];
  const int half = op.half;
  float* rec_prev = op.rec_prev;
  const float scale = op.scale, omega = op.omega;
  const LaneDir d = lane_dir(lane);
  pdl_wait();
  const float fr = d.act ? op.coarse_save[static_cast<long long>(it.coarse_save) * kQ + lane] : 0.f;
  float* pv = op.prev + static_cast<long long>(it.prev) * 23;
  float p0 = 0.f, p1 = 0.f, p2 = 0.f, p3 = 0.f, pf = 0.f;
  if (half) {
    p0 = pv[0]; p1 = pv[1]; p2 = pv[2]; p3 = pv[3];
    pf = d.act ? pv[4 + lane] : 0.f;
    if (rec_prev) {  // the adjoint's record of the rows read here
      float* rp = rec_prev + static_cast<long long>(it.prev) * 23;
      if (d.act) rp[4 + lane] = pf;
      if (lane == kQ) rp[0] = p0;
      if (lane == kQ + 1) rp[1] = p1;
      if (lane == kQ + 2) rp[2] = p2;
      if (lane == kQ + 3) rp[3] = p3;
    }
  }
  float fa[kQ];
  gather_lanes(fr, fa);
  float drho, jx, jy, jz;
  moments(fa, drho, jx, jy, jz);
  const float rho = 1.0f + drho, inv = 1.0f / rho;
  const float ux = jx * inv, uy = jy * inv, uz = jz * inv;
  const float usq15 = 1.5f * (ux * ux + uy * uy + uz * uz);
  const float cu = d.cx * ux + d.cy * uy + d.cz * uz;
  const float fneq = fr - d.w * (drho + rho * (3.0f * cu + 4.5f * cu * cu - usq15));
  float wd = drho, wx = ux, wy = uy, wz = uz, wn = fneq;
  if (half) {
    // Half-time: average of previous and current coarse macros
    // (level_coupler.cpp:455-465).
    wd = 0.5f * (p0 + drho);
    wx = 0.5f * (p1 + ux); wy = 0.5f * (p2 + uy); wz = 0.5f * (p3 + uz);
    wn = 0.5f * (pf + fneq);
  } else {
    // Full-time: prev <- current (level_coupler.cpp:470-476).
    if (d.act) pv[4 + lane] = fneq;
    if (lane == kQ) pv[0] = drho;
    if (lane == kQ + 1) pv[1] = ux;
    if (lane == kQ + 2) pv[2] = uy;
    if (lane == kQ + 3) pv[3] = uz;
  }
  // feq(w) + scale * f_neq (WriteProlongation, level_coupler.cpp:191-201),
  // collided when the target is kBulk (as write_macro_cell)
  const float wrho = 1.0f + wd;
  const float wusq15 = 1.5f * (wx * wx + wy * wy + wz * wz);
  const float wcu = d.cx * wx + d.cy * wy + d.cz * wz;
  float f = d.w * (wd + wrho * (3.0f * wcu + 4.5f * wcu * wcu - wusq15)) + scale * wn;
  float dh = 0.f;
  if (it.fine_kind == kBulk && op.cmode != kCollNone) {
    gather_lanes(f, fa);
    if (op.cmode == kCollConstRho)
      f = bgk_lane_const_rho(d, lane, fa, f, omega, static_cast<float>(1.0 - *op.cr_avg), dh);
    else
      f = bgk_lane<false>(d, lane, fa, f, omega);
  }
  if (d.act) Store<T>::st(static_cast<T*>(op.fine) + lane * op.fine_qs + it.fine_slot, f, op.fscale);
  return dh;
}

// Lagrava restriction (level_coupler.cpp:613-654), one warp per item: lane
// k <= nnb reads one source row (the fine cell, then its in-block
// neighbours) and forms its macro state; the f_neq rows meet in shared
// memory, where lane i sums population i over the neighbours in the
// reference's order and averages with the centre; then lane i writes
// population i of the coarse target.
template <typename T>
__device__ __forceinline__ void restrict_warp(const RestrictOp& op, int w, int lane, float (*fs)[kQ + 1]) {
  if (w >= op.n) return;  // whole warps
  const RestrictItem& it = op.items[w];
  const float scale = op.scale, omega = op.omega;
  const int nnb = it.nnb;
  const int row = lane == 0 ? it.fine_save : (lane <= nnb ? it.nb_save[lane - 1] : -1);
  pdl_wait();
  Macro m;
  if (row >= 0) {
    read_macro(op.fine_save + static_cast<long long>(row) * kQ, m);
#pragma unroll
    for (int i = 0; i < kQ; ++i) fs[lane][i] = m.fneq[i];
  }
  __syncwarp();
  const LaneDir d = lane_dir(lane);
  float nsum = 0.f;
  for (int r = 1; r <= nnb; ++r) nsum += d.act ? fs[r][lane] : 0.f;
  const float inv = 1.0f / static_cast<float>(nnb + 1);
  const float rn = d.act ? (fs[0][lane] + nsum) * inv : 0.f;
  const float rd = __shfl_sync(0xffffffffu, m.drho, 0), rx = __shfl_sync(0xffffffffu, m.ux, 0);
  const float ry = __shfl_sync(0xffffffffu, m.uy, 0), rz = __shfl_sync(0xffffffffu, m.uz, 0);
  const float rho = 1.0f + rd;
  const float usq15 = 1.5f * (rx * rx + ry * ry + rz * rz);
  const float cu = d.cx * rx + d.cy * ry + d.cz * rz;
  float f = d.w * (rd + rho * (3.0f * cu + 4.5f * cu * cu - usq15)) + scale * rn;
  if (it.coarse_kind == kBulk && op.cmode != kCollNone) {
    float fa[kQ];
    gather_lanes(f, fa);
    f = bgk_lane<false>(d, lane, fa, f, omega);
  }
  if (d.act) Store<T>::st(static_cast<T*>(op.coarse) + lane * op.coarse_qs + it.coarse_slot, f, op.cscale);
}

// One coupler launch: the prolongation's items, then each restriction's, one
// warp per item, each on its own range of CTAs.  Operations that nothing
// between them orders (a restriction into level l and the full-time
// prolongation into level l with disjoint targets; two restrictions) share a
// launch this way.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_couple(const ProlongOp p, const RestrictOp r0, const RestrictOp r1) {
  __shared__ float fneq_s[kThreads / 32][kQ][kQ + 1];  // restriction: [warp][row][population]
  const uint32_t gp = (static_cast<uint32_t>(p.n) * 32 + kThreads - 1) / kThreads;
  const uint32_t g0 = (static_cast<uint32_t>(r0.n) * 32 + kThreads - 1) / kThreads;
  const int lane = threadIdx.x & 31;
  uint32_t b = blockIdx.x;
  if (b < gp) {
    const float dh = prolong_warp<T>(p, static_cast<int>((b * kThreads + threadIdx.x) >> 5), lane);
    if (p.cr_part) {  // ConstRhoBGK statistics of the collided targets (lane 0 of each item)
      double v[1] = {lane == 0 ? static_cast<double>(dh) : 0.0};
      block_reduce<1>(v);
      if (threadIdx.x == 0) p.cr_part[b] = v[0];
    }
    return;
  }
  b -= gp;
  float (*fs)[kQ + 1] = fneq_s[threadIdx.x >> 5];
  if (b < g0) {
    restrict_warp<T>(r0, static_cast<int>((b * kThreads + threadIdx.x) >> 5), lane, fs);
    return;
  }
  b -= g0;
  restrict_warp<T>(r1, static_cast<int>((b * kThreads + threadIdx.x) >> 5), lane, fs);
}

// Momentum-exchange force (drag_postprocessor.h:67-115) from the buffer the
// last step read.  For a link from kBulk cell x to an in-block obstacle cell
// x + c_i: f_out = g_i(x) (the post-collide snapshot) and f_bar is the
// population opp(i) the step pulled from the obstacle: half-way bounce-back
// g_i(x), or the Bouzidi value with the link's q, plus the moving-wall term.
template <typename T, bool LINKS>
__global__ void __launch_bounds__(kThreads)
k_drag(const StepArgs a, const DragItem* items, int nitems, double* partial) {
  // One warp per item, lane i on direction i: the links' dependent lookups
  // (link record, neighbour, its kind, a boundary fill) run side by side.
  const int w = static_cast<int>((blockIdx.x * kThreads + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  double acc[3] = {0.0, 0.0, 0.0};
  pdl_wait();
  if (w < nitems) {
    const DragItem it = items[w];
    const T* src = static_cast<const T*>(a.src);
    const LaneDir d = lane_dir(lane);
    const float own = d.act ? LD(src, a.qs, lane, it.slot, a.inv_scale) : 0.f;  // g_i(x)
    const float own_j = __shfl_sync(0xffffffffu, own, d.opp);                    // g_opp(i)(x)
    const bool link = d.act && lane > 0 && ((it.mask >> lane) & 1u);
    float f_bar = 0.f;
    if (link) {
      const int j = d.opp;
      if constexpr (LINKS) {
        f_bar = own;
        const uint8_t fl = a.flags[it.slot];
        const int li = (fl & kFlagLink) ? a.link_idx[it.slot] : -1;
        if (li >= 0) {
          const float q = a.link_rec[li * 38 + j];
          if (q < 1.0f) {
            const Cell c = cell_of(a, static_cast<uint32_t>(it.slot));
            const int ax = static_cast<int>(d.cx), ay = static_cast<int>(d.cy), az = static_cast<int>(d.cz);
            bool nhalo;
            const long long nb = resolve(a, c.b, static_cast<int>(c.x) + 1 - ax, static_cast<int>(c.y) + 1 - ay,
                                         static_cast<int>(c.z) + 1 - az, nhalo);
            const int nk = nhalo ? kBulk : (a.flags[nb] & kKindMask);
            const float f_q = nk == kBulk ? pull_value(a, src, j, nb) : own_j;
            f_bar = bouzidi(own, f_q, own_j, q);
          }
          f_bar += a.link_rec[li * 38 + kQ + j];
        }
      } else {
        f_bar = LD(src, a.qs, j, it.slot + a.off[lane], a.inv_scale);  // plain pull from x + c_i
      }
    }
    const double sv = link ? static_cast<double>(own) + static_cast<double>(f_bar) : 0.0;
    double v[3] = {sv * d.cx, sv * d.cy, sv * d.cz};
#pragma unroll
    for (int k = 0; k < 3; ++k)
      for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    if (lane == 0) {
      acc[0] = v[0];
      acc[1] = v[1];
      acc[2] = v[2];
    }
  }
  block_reduce<3>(acc);
  if (threadIdx.x == 0) {
    partial[blockIdx.x * 3 + 0] = -acc[0];
    partial[blockIdx.x * 3 + 1] = -acc[1];
    partial[blockIdx.x * 3 + 2] = -acc[2];
  }
}

// Sum of per-CTA partials, `width` doubles each, by one CTA: fixed strided
// per-thread sums then a fixed shuffle tree (deterministic).
__global__ void __launch_bounds__(kThreads)
k_sum_partials(const double* partial, int nparts, int width, double* out, double* accum) {
  pdl_wait();
  for (int k = 0; k < width; ++k) {
    double v[1] = {0.0};
    for (int p = threadIdx.x; p < nparts; p += kThreads) v[0] += partial[p * width + k];
    block_reduce<1>(v);
    if (threadIdx.x == 0) {
      out[k] = v[0];
      if (accum) accum[k] += v[0];
    }
    __syncthreads();
  }
}

// Mass / momentum audit over kBulk core cells (total_mass,
// cylinder3d_case.h:601-622) with a non-finite check over every core cell.
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_audit(const StepArgs a, double* partial) {
  const uint32_t t = blockIdx.x * kThreads + threadIdx.x;
  double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  if (t < a.ncore) {
    const long long slot = t;  // compact core slot
    const T* src = static_cast<const T*>(a.src);
    float f[kQ];
    bool finite = true;
#pragma unroll
    for (int i = 0; i < kQ; ++i) {
      f[i] = LDR(a, src, i, t);
      finite = finite && isfinite(f[i]);
    }
    const int kind = a.flags ? (a.flags[slot] & kKindMask) : kBulk;
    if (!finite) acc[4] = 1.0;
    if (kind == kBulk) {
      double drho = 0, jx = 0, jy = 0, jz = 0;
#pragma unroll
      for (int i = 0; i < kQ; ++i) {
        drho += f[i]; jx += cx(i) * static_cast<double>(f[i]);
        jy += cy(i) * static_cast<double>(f[i]); jz += cz(i) * static_cast<double>(f[i]);
      }
      acc[0] = 1.0 + drho; acc[1] = jx; acc[2] = jy; acc[3] = jz;
    }
  }
  block_reduce<5>(acc);
  if (threadIdx.x == 0)
    for (int k = 0; k < 5; ++k) partial[blockIdx.x * 5 + k] = acc[k];
}

// Core cells <-> dense FP64 host order [block][ix][iy][iz][19].
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_gather(const StepArgs a, double* out, double* out_u, int mode /*0 pops, 1 fields*/) {
  const uint32_t t = blockIdx.x * kThreads + threadIdx.x;
  if (t >= a.ncore) return;
  const long long slot = t;  // compact core slot
  const T* src = static_cast<const T*>(a.src);
  if (mode == 0) {
#pragma unroll
    for (int i = 0; i < kQ; ++i) out[static_cast<long long>(t) * kQ + i] = LDR(a, src, i, t);
  } else {
    double drho = 0, jx = 0, jy = 0, jz = 0;
#pragma unroll
    for (int i = 0; i < kQ; ++i) {
      const double v = LDR(a, src, i, t);
      drho += v; jx += cx(i) * v; jy += cy(i) * v; jz += cz(i) * v;
    }
    const double rho = 1.0 + drho;
    // ConstRhoBGK: the stored state is one collide ahead, which added
    // 1 - average_rho to the density of a kBulk cell and left u unchanged
    const bool cr = a.cr_avg && (a.flags ? (a.flags[slot] & kKindMask) : kBulk) == kBulk;
    out[t] = cr ? rho - (1.0 - *a.cr_avg) : rho;
    out_u[static_cast<long long>(t) * 3 + 0] = jx / rho;
    out_u[static_cast<long long>(t) * 3 + 1] = jy / rho;
    out_u[static_cast<long long>(t) * 3 + 2] = jz / rho;
  }
}

// Reference state f (pre-collision, FP64) -> stored g = C(f) for kBulk cells.
// Under ConstRhoBGK the collide is taken at *cr_avg, and each CTA's sum of
// rho - 1 over its kBulk cells goes to cr_part[blockIdx.x] (the statistics of
// that collide; the near-wall partials after them, near_parts, are zeroed).
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_scatter(const StepArgs a, const double* in, int near_parts) {
  const uint32_t t = blockIdx.x * kThreads + threadIdx.x;
  double v[1] = {0.0};
  if (t < a.ncore) {
    const long long slot = t;  // compact core slot
    float f[kQ];
#pragma unroll
    for (int i = 0; i < kQ; ++i) f[i] = static_cast<float>(in[static_cast<long long>(t) * kQ + i]);
    const uint8_t fl = a.flags ? a.flags[slot] : static_cast<uint8_t>(kBulk);
    if ((fl & kKindMask) == kBulk) {
      if (a.cr_avg) v[0] = (fl & kFlagProlong) ? 0.0 : bgk_const_rho(f, a.omega, static_cast<float>(1.0 - *a.cr_avg));
      else bgk<kBgkCorrect<T>>(f, a.omega);
    }
    T* dst = static_cast<T*>(a.dst);
#pragma unroll
    for (int i = 0; i < kQ; ++i) Store<T>::st(dst + i * a.qs + slot, f[i], a.scale);
  }
  if (a.cr_part) {
    block_reduce<1>(v);
    if (threadIdx.x == 0) a.cr_part[blockIdx.x] = v[0];
    if (blockIdx.x == 0)
      for (int p = threadIdx.x; p < near_parts; p += kThreads) a.cr_part[gridDim.x + p] = 0.0;
  }
}

// Equilibrium state from macroscopic fields (BlockLattice::initialize and
// initialize_from_material with a per-cell rho, u: block_lattice.cpp:273-285,
// lattice_material_init.cpp:11-33): f_i = feq_i(rho, u) - w_i in FP64, then
// the same conversion and collide as k_scatter.  in = [rho | u] (ncore, then
// ncore x 3).  The FP64 operations are rounded one by one in the order
// rho w_i (1 + 3 cu + 4.5 cu cu - 1.5 u.u) - w_i is written (no contraction
// into fused multiply-adds), so the state equals k_scatter's of the same
// equilibrium formed on the host in that order.
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_scatter_eq(const StepArgs a, const double* in, int near_parts) {
  const uint32_t t = blockIdx.x * kThreads + threadIdx.x;
  double v[1] = {0.0};
  if (t < a.ncore) {
    const long long slot = t;
    const double rho = in[t];
    const double* up = in + a.ncore + 3ll * t;
    const double ux = up[0], uy = up[1], uz = up[2];
    const double usq = __dadd_rn(__dadd_rn(__dmul_rn(ux, ux), __dmul_rn(uy, uy)), __dmul_rn(uz, uz));
    const double t6 = __dmul_rn(1.5, usq);
    float f[kQ];
#pragma unroll
    for (int i = 0; i < kQ; ++i) {
      // c_i has at most two nonzero components: cu is exact or one rounding
      double cu = 0.0;
      if (cx(i)) cu = cx(i) > 0 ? ux : -ux;
      if (cy(i)) cu = __dadd_rn(cu, cy(i) > 0 ? uy : -uy);
      if (cz(i)) cu = __dadd_rn(cu, cz(i) > 0 ? uz : -uz);
      const double p = __dsub_rn(__dadd_rn(__dadd_rn(1.0, __dmul_rn(3.0, cu)), __dmul_rn(__dmul_rn(4.5, cu), cu)), t6);
      f[i] = static_cast<float>(__dsub_rn(__dmul_rn(__dmul_rn(rho, wd(i)), p), wd(i)));
    }
    const uint8_t fl = a.flags ? a.flags[slot] : static_cast<uint8_t>(kBulk);
    if ((fl & kKindMask) == kBulk) {
      if (a.cr_avg) v[0] = (fl & kFlagProlong) ? 0.0 : bgk_const_rho(f, a.omega, static_cast<float>(1.0 - *a.cr_avg));
      else bgk<kBgkCorrect<T>>(f, a.omega);
    }
    T* dst = static_cast<T*>(a.dst);
#pragma unroll
    for (int i = 0; i < kQ; ++i) Store<T>::st(dst + i * a.qs + slot, f[i], a.scale);
  }
  if (a.cr_part) {
    block_reduce<1>(v);
    if (threadIdx.x == 0) a.cr_part[blockIdx.x] = v[0];
    if (blockIdx.x == 0)
      for (int p = threadIdx.x; p < near_parts; p += kThreads) a.cr_part[gridDim.x + p] = 0.0;
  }
}

// ConstRhoBGK statistics of a stored state that BGK collided (which keeps
// each cell's density): per CTA the sum of rho - 1 over kBulk core cells
// that no prolongation writes, as k_scatter lays them out.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_cr_seed(const StepArgs a, int near_parts) {
  const uint32_t t = blockIdx.x * kThreads + threadIdx.x;
  double v[1] = {0.0};
  if (t < a.ncore && (a.flags ? (a.flags[t] & (kKindMask | kFlagProlong)) : kBulk) == kBulk) {
    const T* src = static_cast<const T*>(a.src);
    float f[kQ];
#pragma unroll
    for (int i = 0; i < kQ; ++i) f[i] = LD(src, a.qs, i, t, a.inv_scale);
    float dh, jx, jy, jz;
    moments(f, dh, jx, jy, jz);
    v[0] = dh;
  }
  block_reduce<1>(v);
  if (threadIdx.x == 0) a.cr_part[blockIdx.x] = v[0];
  if (blockIdx.x == 0)
    for (int p = threadIdx.x; p < near_parts; p += kThreads) a.cr_part[gridDim.x + p] = 0.0;
}

// The collide of a level above the finest under ConstRhoBGK on a multi-level
// mesh (TimeLoop::collide_level without statistics, time_loop.h:173-187),
// run in place on its pulled populations once its coupling is done: the
// restriction has written its targets, and the average density is the one
// the finest level's last collide gave, which the reference's next collide
// of this level uses.
//
// shift (when not null): the density shift 1 - average_rho the collide puts
// on the level's kBulk cells, which the finite-difference pass removes from
// the densities it reads there.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_collide_cr(const StepArgs a, float* shift) {
  pdl_wait();
  const uint32_t t = blockIdx.x * kThreads + threadIdx.x;
  if (shift && t == 0) *shift = static_cast<float>(1.0 - *a.cr_avg);
  if (t >= a.ncore) return;
  if (a.flags && (a.flags[t] & kKindMask) != kBulk) return;
  T* pops = static_cast<T*>(a.dst);
  float f[kQ];
#pragma unroll
  for (int i = 0; i < kQ; ++i) f[i] = LD(pops, a.qs, i, t, a.inv_scale);
  bgk_const_rho(f, a.omega, static_cast<float>(1.0 - *a.cr_avg));
#pragma unroll
  for (int i = 0; i < kQ; ++i) Store<T>::st(pops + i * a.qs + t, f[i], a.scale);
}

// average_rho <- CollideRhoStats::average() of the last collide
// (block_lattice.h:22-32, time_loop.h:220-222): the statistic of a cell is
// rho + (1 - average_rho) with the average that collide used, so the mean
// over `count` kBulk cells is 2 - average_rho + sum(rho - 1) / count (1 when
// there are none).  The partials are summed in a fixed order.
// With the finite-difference boundary pass (kFluidAndBoundary scope) the
// velocity-Dirichlet cells' collide densities join the statistics:
// (sum(rho - 1) + count (2 - average_rho) + sum rho_b) / (count + count_b).
//
// shift (when not null): 1 - average_rho, the density shift the finest
// level's collide now puts on its kBulk cells.
__global__ void __launch_bounds__(kThreads)
k_cr_update(double* avg, const double* part, int nparts, long long count, const double* bpart, int nbparts,
            long long bcount, float* shift) {
  pdl_wait();
  double v[2] = {0.0, 0.0};
  for (int p = threadIdx.x; p < nparts; p += kThreads) v[0] += part[p];
  for (int p = threadIdx.x; p < nbparts; p += kThreads) v[1] += bpart[p];
  block_reduce<2>(v);
  if (threadIdx.x == 0) {
    if (bcount == 0)
      *avg = count > 0 ? (2.0 - *avg) + v[0] / static_cast<double>(count) : 1.0;
    else
      *avg = (v[0] + static_cast<double>(count) * (2.0 - *avg) + v[1]) / static_cast<double>(count + bcount);
    if (shift) *shift = static_cast<float>(1.0 - *avg);
  }
}

inline uint32_t grid_for(uint32_t items) { return (items + kThreads - 1) / kThreads; }


}  // namespace

// ---------------------------------------------------------------- launchers
// Programmatic launches for the time-step chain on this host thread.
namespace {
thread_local bool g_programmatic = false;
}
void set_programmatic_launch(bool on) { g_programmatic = on; }
bool programmatic_launch() { return g_programmatic; }

template <typename T>
cudaError_t launch_step(const StepArgs& a, bool periodic, bool links, bool flags, cudaStream_t s) {
  cudaError_t e = cudaSuccess;
  if (a.nitems == 0) return cudaSuccess;
  // CTAs aligned to blocks: core cells first (a multiple of the CTA size),
  // then the halo items in CTAs of their own.
  const uint32_t n3 = static_cast<uint32_t>(a.n) * a.n * a.n;
  const bool blocked = n3 % kThreads == 0;
  const uint32_t core_ctas = grid_for(a.ncore);
  const dim3 g(core_ctas + grid_for(a.nitems - a.ncore));
  StepArgs b = a;
  // the flag-free periodic box collides as k_step_pair does (defect removal)
  const bool box = periodic && !flags && !links;
  if (blocked) {
    if (links) e = launch_chain(k_step<T, true, true, true>, dim3(g), dim3(kThreads), 0, s, b);
    else if (flags) e = launch_chain(k_step<T, false, true, true>, dim3(g), dim3(kThreads), 0, s, b);
    else if (box) e = launch_chain(k_step<T, false, false, true, kCollBgk, true>, dim3(g), dim3(kThreads), 0, s, b);
    else e = launch_chain(k_step<T, false, false, true>, dim3(g), dim3(kThreads), 0, s, b);
  } else {
    if (links) e = launch_chain(k_step<T, true, true, false>, dim3(g), dim3(kThreads), 0, s, b);
    else if (flags) e = launch_chain(k_step<T, false, true, false>, dim3(g), dim3(kThreads), 0, s, b);
    else if (box) e = launch_chain(k_step<T, false, false, false, kCollBgk, true>, dim3(g), dim3(kThreads), 0, s, b);
    else e = launch_chain(k_step<T, false, false, false>, dim3(g), dim3(kThreads), 0, s, b);
  }
  return e != cudaSuccess ? e : cudaGetLastError();
}

// Slot-map step: a CTA of 256 threads per block (n^3 a multiple of 512, the
// (n+2)^3 map within 48 KB of shared memory, 32-bit population offsets).
bool map_step_eligible(int n, long long nslots) {
  const long long np = n + 2;
  return n % 8 == 0 && np * np * np * 4 <= 48 * 1024 && nslots * kQ < (1LL << 32);
}
template <typename T>
cudaError_t launch_step_map(const StepArgs& a, const NearTables& nt, bool links, bool flags, int cpt, bool gmap,
                            cudaStream_t s) {
  cudaError_t e = cudaSuccess;
  if (a.nitems == 0) return cudaSuccess;
  const uint32_t near_ctas = links ? grid_for(static_cast<uint32_t>(nt.n) * 32) : 0;
  const dim3 g(near_ctas + static_cast<uint32_t>(a.nblk) * (cpt == 2 ? 1 : 2) + grid_for(static_cast<uint32_t>(a.n_open)));
  const size_t smem = gmap ? 0 : static_cast<size_t>(a.np) * a.np * a.np * sizeof(int);
#define OCTLB_MAP_LAUNCH(C, G)                                                                              \
  if (links) e = launch_chain(k_step_map<T, true, true, C, G>, g, dim3(kThreads), smem, s, a, nt);          \
  else if (flags) e = launch_chain(k_step_map<T, false, true, C, G>, g, dim3(kThreads), smem, s, a, nt);    \
  else e = launch_chain(k_step_map<T, false, false, C, G>, g, dim3(kThreads), smem, s, a, nt);
  if (cpt == 2) {
    if (gmap) { OCTLB_MAP_LAUNCH(2, true) } else { OCTLB_MAP_LAUNCH(2, false) }
  } else {
    if (gmap) { OCTLB_MAP_LAUNCH(1, true) } else { OCTLB_MAP_LAUNCH(1, false) }
  }
#undef OCTLB_MAP_LAUNCH
  return e != cudaSuccess ? e : cudaGetLastError();
}

// ConstRhoBGK slot-map step: the default variants only (one cell per thread
// under the links rule, two otherwise; slot map read through L1).
template <typename T>
cudaError_t launch_step_map_cr(const StepArgs& a, const NearTables& nt, bool links, bool flags, cudaStream_t s) {
  cudaError_t e = cudaSuccess;
  if (a.nitems == 0) return cudaSuccess;
  const uint32_t near_ctas = links ? grid_for(static_cast<uint32_t>(nt.n) * 32) : 0;
  const dim3 g(near_ctas + static_cast<uint32_t>(a.nblk) * (links ? 2 : 1) + grid_for(static_cast<uint32_t>(a.n_open)));
  if (links) e = launch_chain(k_step_map<T, true, true, 1, true, kCollConstRho>, g, dim3(kThreads), 0, s, a, nt);
  else if (flags) e = launch_chain(k_step_map<T, false, true, 2, true, kCollConstRho>, g, dim3(kThreads), 0, s, a, nt);
  else e = launch_chain(k_step_map<T, false, false, 2, true, kCollConstRho>, g, dim3(kThreads), 0, s, a, nt);
  return e != cudaSuccess ? e : cudaGetLastError();
}

// Stream-only steps (no collide) of the levels above the finest under
// ConstRhoBGK on a multi-level mesh: the slot-map form in the variants of
// launch_step_map_cr, else the core / halo-item launch and the near cells.
template <typename T>
cudaError_t launch_step_map_nc(const StepArgs& a, const NearTables& nt, bool links, bool flags, cudaStream_t s) {
  cudaError_t e = cudaSuccess;
  if (a.nitems == 0) return cudaSuccess;
  const uint32_t near_ctas = links ? grid_for(static_cast<uint32_t>(nt.n) * 32) : 0;
  const dim3 g(near_ctas + static_cast<uint32_t>(a.nblk) * (links ? 2 : 1) + grid_for(static_cast<uint32_t>(a.n_open)));
  if (links) e = launch_chain(k_step_map<T, true, true, 1, true, kCollNone>, g, dim3(kThreads), 0, s, a, nt);
  else if (flags) e = launch_chain(k_step_map<T, false, true, 2, true, kCollNone>, g, dim3(kThreads), 0, s, a, nt);
  else e = launch_chain(k_step_map<T, false, false, 2, true, kCollNone>, g, dim3(kThreads), 0, s, a, nt);
  return e != cudaSuccess ? e : cudaGetLastError();
}
template <typename T>
cudaError_t launch_step_nc(const StepArgs& a, const NearTables& nt, bool links, bool flags, cudaStream_t s) {
  cudaError_t e = cudaSuccess;
  if (a.nitems == 0) return cudaSuccess;
  const uint32_t n3 = static_cast<uint32_t>(a.n) * a.n * a.n;
  const bool blocked = n3 % kThreads == 0;
  const uint32_t core_ctas = grid_for(a.ncore);
  const dim3 g(core_ctas + grid_for(a.nitems - a.ncore));
  const StepArgs& b = a;
  if (blocked) {
    if (links) e = launch_chain(k_step<T, true, true, true, kCollNone>, g, dim3(kThreads), 0, s, b);
    else if (flags) e = launch_chain(k_step<T, false, true, true, kCollNone>, g, dim3(kThreads), 0, s, b);
    else e = launch_chain(k_step<T, false, false, true, kCollNone>, g, dim3(kThreads), 0, s, b);
  } else {
    if (links) e = launch_chain(k_step<T, true, true, false, kCollNone>, g, dim3(kThreads), 0, s, b);
    else if (flags) e = launch_chain(k_step<T, false, true, false, kCollNone>, g, dim3(kThreads), 0, s, b);
    else e = launch_chain(k_step<T, false, false, false, kCollNone>, g, dim3(kThreads), 0, s, b);
  }
  if (e == cudaSuccess && nt.n > 0)
    e = launch_chain(k_step_near<T, kCollNone>, dim3(grid_for(static_cast<uint32_t>(nt.n) * 32)), dim3(kThreads), 0,
                     s, a, nt);
  return e != cudaSuccess ? e : cudaGetLastError();
}

template <typename T>
cudaError_t launch_step_near(const StepArgs& a, const NearTables& nt, cudaStream_t s) {
  if (nt.n == 0) return cudaSuccess;
  const cudaError_t e = launch_chain(k_step_near<T>, dim3(grid_for(static_cast<uint32_t>(nt.n) * 32)), dim3(kThreads), 0, s, a, nt);
  return e != cudaSuccess ? e : cudaGetLastError();
}

template <typename T>
cudaError_t launch_step_pair(const StepArgs& a, cudaStream_t s) {
  // FP16 storage: four cells per thread when n % 4 == 0 (OCTLB_FP16_PAIR=1
  // keeps two, for comparison)
  const char* env = std::getenv("OCTLB_FP16_PAIR");
  const bool pair16 = env && env[0] == '1';
  cudaError_t e;
  if (std::is_same<T, __half>::value && a.n % 4 == 0 && !pair16)
    e = launch_chain(k_step_quad_h, dim3(grid_for(a.ncore / 4)), dim3(kThreads), 0, s, a);
  else
    e = launch_chain(k_step_pair<T>, dim3(grid_for(a.ncore / 2)), dim3(kThreads), 0, s, a);
  return e != cudaSuccess ? e : cudaGetLastError();
}
// AA order: the step from the natural layout (reversed = false), or the one
// from the reversed layout.
template <typename T>
cudaError_t launch_step_aa(const StepArgs& a, bool reversed, cudaStream_t s) {
  // The local step takes four FP16 cells per thread where n % 4 == 0, else
  // two.  The pull step takes four FP16 cells per thread where a warp covers
  // a 128-cell row (n % 128 == 0; OCTLB_AA_PULL=scalar keeps one), else one:
  // measured on the 256^3 box, one FP32 cell per thread (80 registers)
  // beats two with shuffled aligned stores (128 registers), and four FP16
  // cells bounded to two CTAs per SM beat one.  (The pull step the context
  // launches by default is the staged k_step_aa_rows<T>; setting
  // OCTLB_AA_PULL selects one of these instead.)
  const char* env = std::getenv("OCTLB_AA_PULL");
  const bool scalar = env && std::string(env) == "scalar";
  const bool half = std::is_same<T, __half>::value;
  cudaError_t e;
  if (reversed) {
    e = half && a.n % 4 == 0 ? launch_chain(k_step_aa_local_h, dim3(grid_for(a.ncore / 4)), dim3(kThreads), 0, s, a)
                             : launch_chain(k_step_aa_local<T>, dim3(grid_for(a.ncore / 2)), dim3(kThreads), 0, s, a);
  } else if (half && a.n % 128 == 0 && !scalar) {
    e = launch_chain(k_step_aa_pull_h, dim3(grid_for(a.ncore / 4)), dim3(kThreads), 0, s, a);
  } else {
    e = launch_chain(k_step_aa_pull<T>, dim3(grid_for(a.ncore)), dim3(kThreads), 0, s, a);
  }
  return e != cudaSuccess ? e : cudaGetLastError();
}
// Paired kernel: even n (aligned pairs), n^3 < 2^31.
bool pair_step_eligible(int n) { return n >= 4 && (n % 2) == 0 && n <= 1024; }

template <typename T>
cudaError_t launch_add_force(const StepArgs& a, T* pops, const float* force, cudaStream_t s) {
  if (a.ncore == 0) return cudaSuccess;
  const cudaError_t e = launch_chain(k_add_force<T>, dim3(grid_for(a.ncore)), dim3(kThreads), 0, s, a, pops, force);
  return e != cudaSuccess ? e : cudaGetLastError();
}


template <typename T>
cudaError_t launch_couple(const ProlongOp& p, const RestrictOp& r0, const RestrictOp& r1, cudaStream_t s) {
  const uint32_t g = grid_for(static_cast<uint32_t>(p.n) * 32) + grid_for(static_cast<uint32_t>(r0.n) * 32) +
                     grid_for(static_cast<uint32_t>(r1.n) * 32);
  if (g == 0) return cudaSuccess;
  const cudaError_t e = launch_chain(k_couple<T>, dim3(g), dim3(kThreads), 0, s, p, r0, r1);
  return e != cudaSuccess ? e : cudaGetLastError();
}

// Drag partials of n items: one per CTA of the warp-per-item launch.
uint32_t drag_partials(int n) { return grid_for(static_cast<uint32_t>(n > 0 ? n : 1) * 32); }

template <typename T>
cudaError_t launch_drag(const StepArgs& a, bool links, const DragItem* items, int n, double* partial,
                        cudaStream_t s) {
  cudaError_t e = cudaSuccess;
  const uint32_t g = drag_partials(n);
  if (links) e = launch_chain(k_drag<T, true>, dim3(g), dim3(kThreads), 0, s, a, items, n, partial);
  else e = launch_chain(k_drag<T, false>, dim3(g), dim3(kThreads), 0, s, a, items, n, partial);
  return e != cudaSuccess ? e : cudaGetLastError();
}
// Force = fixed-order sum of every level's drag partials; accum += force.
cudaError_t launch_drag_total(const double* partial, int nparts, double* out, double* accum, cudaStream_t s) {
  const cudaError_t e = launch_chain(k_sum_partials, dim3(1), dim3(kThreads), 0, s, partial, nparts, 3, out, accum);
  return e != cudaSuccess ? e : cudaGetLastError();
}

template <typename T>
cudaError_t launch_audit(const StepArgs& a, double* partial, double* out, cudaStream_t s) {
  const uint32_t g = grid_for(a.ncore);
  k_audit<T><<<g, kThreads, 0, s>>>(a, partial);
  k_sum_partials<<<1, kThreads, 0, s>>>(partial, static_cast<int>(g), 5, out, nullptr);
  return cudaGetLastError();
}
uint32_t audit_partials(const StepArgs& a) { return grid_for(a.ncore); }

template <typename T>
cudaError_t launch_gather(const StepArgs& a, double* out, double* out_u, int mode, cudaStream_t s) {
  k_gather<T><<<grid_for(a.ncore), kThreads, 0, s>>>(a, out, out_u, mode);
  return cudaGetLastError();
}
template <typename T>
cudaError_t launch_scatter(const StepArgs& a, const double* in, int near_parts, cudaStream_t s) {
  k_scatter<T><<<grid_for(a.ncore), kThreads, 0, s>>>(a, in, near_parts);
  return cudaGetLastError();
}
template <typename T>
cudaError_t launch_scatter_eq(const StepArgs& a, const double* in, int near_parts, cudaStream_t s) {
  k_scatter_eq<T><<<grid_for(a.ncore), kThreads, 0, s>>>(a, in, near_parts);
  return cudaGetLastError();
}

// CTAs of a k_couple launch's prolongation of n items (one warp per item).
uint32_t couple_prolong_ctas(int n) { return grid_for(static_cast<uint32_t>(n) * 32); }

// ConstRhoBGK partials of a level: one per core CTA of k_step_cr (the CTAs of
// k_scatter / k_cr_seed), then one per CTA of k_step_near_cr.
uint32_t cr_core_parts(const StepArgs& a) { return grid_for(a.ncore); }
uint32_t cr_near_parts(const NearTables& nt) { return nt.n > 0 ? grid_for(static_cast<uint32_t>(nt.n) * 32) : 0; }

template <typename T>
cudaError_t launch_step_cr(const StepArgs& a, const NearTables& nt, bool links, bool flags, cudaStream_t s) {
  cudaError_t e = cudaSuccess;
  if (a.nitems == 0) return cudaSuccess;
  const uint32_t n3 = static_cast<uint32_t>(a.n) * a.n * a.n;
  const bool blocked = n3 % kThreads == 0;
  const uint32_t core_ctas = grid_for(a.ncore);
  const dim3 g(core_ctas + grid_for(a.nitems - a.ncore));
  if (blocked) {
    if (links) e = launch_chain(k_step_cr<T, true, true, true>, g, dim3(kThreads), 0, s, a);
    else if (flags) e = launch_chain(k_step_cr<T, false, true, true>, g, dim3(kThreads), 0, s, a);
    else e = launch_chain(k_step_cr<T, false, false, true>, g, dim3(kThreads), 0, s, a);
  } else {
    if (links) e = launch_chain(k_step_cr<T, true, true, false>, g, dim3(kThreads), 0, s, a);
    else if (flags) e = launch_chain(k_step_cr<T, false, true, false>, g, dim3(kThreads), 0, s, a);
    else e = launch_chain(k_step_cr<T, false, false, false>, g, dim3(kThreads), 0, s, a);
  }
  if (e == cudaSuccess && nt.n > 0)
    e = launch_chain(k_step_near_cr<T>, dim3(cr_near_parts(nt)), dim3(kThreads), 0, s, a, nt,
                     static_cast<int>(core_ctas));
  return e != cudaSuccess ? e : cudaGetLastError();
}

template <typename T>
cudaError_t launch_collide_cr(const StepArgs& a, float* shift, cudaStream_t s) {
  if (a.ncore == 0) return cudaSuccess;
  const cudaError_t e = launch_chain(k_collide_cr<T>, dim3(grid_for(a.ncore)), dim3(kThreads), 0, s, a, shift);
  return e != cudaSuccess ? e : cudaGetLastError();
}

template <typename T>
cudaError_t launch_cr_seed(const StepArgs& a, int near_parts, cudaStream_t s) {
  k_cr_seed<T><<<grid_for(a.ncore), kThreads, 0, s>>>(a, near_parts);
  return cudaGetLastError();
}

cudaError_t launch_cr_update(double* avg, const double* part, int nparts, long long count, const double* bpart,
                             int nbparts, long long bcount, float* shift, cudaStream_t s) {
  const cudaError_t e = launch_chain(k_cr_update, dim3(1), dim3(kThreads), 0, s, avg, part, nparts, count, bpart,
                                     nbparts, bcount, shift);
  return e != cudaSuccess ? e : cudaGetLastError();
}

#define OCTLB_INST(T)                                                                              \
  template cudaError_t launch_step<T>(const StepArgs&, bool, bool, bool, cudaStream_t);            \
  template cudaError_t launch_step_pair<T>(const StepArgs&, cudaStream_t);                         \
  template cudaError_t launch_step_aa<T>(const StepArgs&, bool, cudaStream_t);                     \
  template cudaError_t launch_step_near<T>(const StepArgs&, const NearTables&, cudaStream_t);       \
  template cudaError_t launch_add_force<T>(const StepArgs&, T*, const float*, cudaStream_t);         \
  template cudaError_t launch_step_map<T>(const StepArgs&, const NearTables&, bool, bool, int, bool, cudaStream_t); \
  template cudaError_t launch_couple<T>(const ProlongOp&, const RestrictOp&, const RestrictOp&,    \
                                        cudaStream_t);                                             \
  template cudaError_t launch_drag<T>(const StepArgs&, bool, const DragItem*, int, double*,        \
                                      cudaStream_t);                                               \
  template cudaError_t launch_audit<T>(const StepArgs&, double*, double*, cudaStream_t);           \
  template cudaError_t launch_gather<T>(const StepArgs&, double*, double*, int, cudaStream_t);              \
  template cudaError_t launch_scatter<T>(const StepArgs&, const double*, int, cudaStream_t);     \
  template cudaError_t launch_scatter_eq<T>(const StepArgs&, const double*, int, cudaStream_t);  \
  template cudaError_t launch_step_cr<T>(const StepArgs&, const NearTables&, bool, bool, cudaStream_t); \
  template cudaError_t launch_step_map_cr<T>(const StepArgs&, const NearTables&, bool, bool, cudaStream_t); \
  template cudaError_t launch_step_map_nc<T>(const StepArgs&, const NearTables&, bool, bool, cudaStream_t); \
  template cudaError_t launch_step_nc<T>(const StepArgs&, const NearTables&, bool, bool, cudaStream_t); \
  template cudaError_t launch_collide_cr<T>(const StepArgs&, float*, cudaStream_t);                \
  template cudaError_t launch_cr_seed<T>(const StepArgs&, int, cudaStream_t);

OCTLB_INST(float)
OCTLB_INST(__half)

}  // namespace octlb_gpu
