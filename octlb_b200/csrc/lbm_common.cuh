// Shared device/host definitions of the sm_100a per-level LBM step.
//
// D3Q19 lattice in the reference's population order
// (src/solver/lbm/descriptor/definition/common.h:165-197): rest, the nine
// "negative" velocities, then their opposites, opposite(i) = i +- 9.
#pragma once

#include <cstdint>
#include <cuda_fp16.h>

namespace octlb_gpu {

constexpr int kQ = 19;

__host__ __device__ constexpr int cx(int i) {
  constexpr int t[kQ] = {0, -1, 0, 0, -1, -1, -1, -1, 0, 0, 1, 0, 0, 1, 1, 1, 1, 0, 0};
  return t[i];
}
__host__ __device__ constexpr int cy(int i) {
  constexpr int t[kQ] = {0, 0, -1, 0, -1, 1, 0, 0, -1, -1, 0, 1, 0, 1, -1, 0, 0, 1, 1};
  return t[i];
}
__host__ __device__ constexpr int cz(int i) {
  constexpr int t[kQ] = {0, 0, 0, -1, 0, 0, -1, 1, -1, 1, 0, 0, 1, 0, 0, 1, -1, 1, -1};
  return t[i];
}
__host__ __device__ constexpr int opp(int i) { return i == 0 ? 0 : (i <= 9 ? i + 9 : i - 9); }
// Weights t_i: 1/3 rest, 1/18 axis, 1/36 diagonal.
__host__ __device__ constexpr float wf(int i) {
  return i == 0 ? 1.0f / 3.0f : ((cx(i) != 0) + (cy(i) != 0) + (cz(i) != 0) == 1 ? 1.0f / 18.0f : 1.0f / 36.0f);
}
__host__ __device__ constexpr double wd(int i) {
  return i == 0 ? 1.0 / 3.0 : ((cx(i) != 0) + (cy(i) != 0) + (cz(i) != 0) == 1 ? 1.0 / 18.0 : 1.0 / 36.0);
}

// BcKind codes (src/solver/lbm/bc_kind.h:14-23).
enum : uint8_t {
  kBulk = 0, kSolid = 1, kBounceBack = 2, kMovingBounceBack = 3,
  kBouzidi = 4, kVelocityDirichlet = 5, kPressureDirichlet = 6, kOutflow = 7
};
// Per-slot flag byte on the device: bits 0-2 kind, then role bits.
enum : uint8_t {
  kKindMask = 0x07,
  kFlagNear = 0x08,     // core cell whose pull needs the link rule (a solid /
                        // Bouzidi source in the own core, a reflecting kind
                        // with a halo source, or a link record)
  kFlagLink = 0x10,     // core cell with a link record (q / moving-wall term)
  kFlagSave = 0x20,     // save pre-collision populations (coupler source)
  kFlagProlong = 0x40,  // written by a prolongation before it is next read: the
                        // collide a step gives it is replaced, so its ConstRhoBGK
                        // statistic is the prolongation's
};
// Collide of a step launch: BGK, ConstRhoBGK at *cr_avg with per-CTA
// statistics, or none (the populations stored as pulled).
enum : int { kCollBgk = 0, kCollConstRho = 1, kCollNone = 2 };

__host__ __device__ inline bool reflects_on_pull(int k) {
  // BcKindReflectsOnPull (bc_kind.h:30-33)
  return k == kVelocityDirichlet || k == kPressureDirichlet || k == kBouzidi;
}

// Unsigned 32-bit division by a runtime-invariant divisor via multiply-high
// (round-up method of Granlund & Montgomery 1994).
struct FastDiv {
  uint32_t d, m, s;
  FastDiv() : d(1), m(0), s(0) {}
  explicit FastDiv(uint32_t div) : d(div) {
    s = 0;
    while ((1ull << s) < div) ++s;
    m = static_cast<uint32_t>((((1ull << 32) * ((1ull << s) - div)) / div) + 1);
  }
  __host__ __device__ inline uint32_t div(uint32_t n) const {
#ifdef __CUDA_ARCH__
    const uint32_t t = __umulhi(n, m);
#else
    const uint32_t t = static_cast<uint32_t>((static_cast<uint64_t>(n) * m) >> 32);
#endif
    return static_cast<uint32_t>((static_cast<uint64_t>(t) + n) >> s);
  }
};

// Population element access for the two storage types.
// Programmatic dependent launch.  A kernel launched with the programmatic
// stream-serialisation attribute may begin while its predecessor in the
// stream is still finishing: it runs what reads only constant tables, then
// waits for the predecessor's completion and memory before touching anything
// a predecessor writes.  A no-op for a kernel launched without the attribute.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename T> struct Store;
template <> struct Store<float> {
  __device__ static inline float ld(const float* p, float) { return *p; }
  __device__ static inline void st(float* p, float v, float) { *p = v; }
};
template <> struct Store<__half> {
  __device__ static inline float ld(const __half* p, float inv_scale) {
    return __half2float(*p) * inv_scale;
  }
  __device__ static inline void st(__half* p, float v, float scale) {
    *p = __float2half_rn(v * scale);
  }
};

// Moments from opposite pairs: d_i = f_i - f_opp(i) for the nine positive
// directions is nearly exact (the two are close), so the momentum sums carry
// far less rounding than a running sum of mixed-sign terms.
__device__ __forceinline__ void moments(const float (&f)[kQ], float& drho, float& jx, float& jy,
                                        float& jz) {
  // positive directions 10..18 and their opposites 1..9
  const float d10 = f[10] - f[1], d11 = f[11] - f[2], d12 = f[12] - f[3];
  const float d13 = f[13] - f[4], d14 = f[14] - f[5], d15 = f[15] - f[6];
  const float d16 = f[16] - f[7], d17 = f[17] - f[8], d18 = f[18] - f[9];
  // c_10 = +x, c_11 = +y, c_12 = +z, c_13 = (1,1,0), c_14 = (1,-1,0),
  // c_15 = (1,0,1), c_16 = (1,0,-1), c_17 = (0,1,1), c_18 = (0,1,-1)
  jx = ((d10 + d13) + (d14 + d15)) + d16;
  jy = ((d11 + d13) - d14) + ((d17 + d18));
  jz = ((d12 + d15) - d16) + (d17 - d18);
  const float s1 = (f[1] + f[10]) + (f[2] + f[11]) + (f[3] + f[12]);
  const float s2 = ((f[4] + f[13]) + (f[5] + f[14])) + ((f[6] + f[15]) + (f[7] + f[16]));
  const float s3 = (f[8] + f[17]) + (f[9] + f[18]);
  drho = f[0] + (s1 + (s2 + s3));
}

// In-register BGK on populations stored as h = s (f - w) (s = 1 for FP32
// storage): the moments of the shifted populations (rho = 1 + sum f,
// u = sum f c / rho, block_lattice.h:113-125), then f += omega (feq - f) with
// the shifted second-order equilibrium (dynamics/lbm.h:50-64,
// block_lattice.cpp:328-341) rewritten per direction as
//   s (feq_i - w_i) = w_i (c0 + cu (3 A + 4.5 A cu)),  A = s rho,
//   c0 = s (rho - 1) - 1.5 A |u|^2,
// which has no cancellation against w_i and keeps the scale out of the
// per-population work.  The relaxation is applied to the small difference,
// d_i = omega fma(w_i, t, -f), never as (1 - omega) f + omega feq, whose two
// large terms cancel.  Arithmetic is FP32.
//
// In exact arithmetic sum d_i = 0 and sum c_i d_i = 0 (the collide keeps mass
// and momentum); in FP32 the rounded equilibrium leaves a defect of about
// 1e-9 per cell and step that does not average out (it follows the smooth
// local state) and, over a thousand steps, drifts u by ~1e-5 relative against
// FP64.  The defect (e_0 = sum d_i, e = sum c_i d_i, summed in a fixed order)
// is removed along the conserved directions, f_i -= w_i (e_0 + 3 c_i . e),
// which cuts that drift by two orders of magnitude (TGV 64^3, 1,000 steps:
// u 2.1e-5 -> 2.4e-7) at ~7 FP32 ops per population.  cx/cy/cz are +-1 or 0,
// so every product with them is exact; the explicit round-to-nearest
// intrinsics keep the sequence free of contraction, so bgk() and the lane
// form bgk_lane() round identically.  The kernels of the uniform periodic box
// (k_step_pair, k_step_bulk, k_step on a flag-free periodic level) and the
// set-populations collides remove it: HBM-bound, they hide the work (1.7 %
// of the 256^3 step).  The forest kernels (slot map, near cells, coupler)
// are issue-bound, where it costs 13 % of the cylinder's step, and skip it
// (CORRECT = false), as do FP16-shifted kernels, whose 11-bit rounding of
// every population each step lies far above this defect.
struct BgkDefect {
  float e0, ex, ey, ez;
};
__device__ __forceinline__ void defect_add(BgkDefect& e, float d, int ix, int iy, int iz) {
  e.e0 = __fadd_rn(e.e0, d);
  if (ix) e.ex = ix > 0 ? __fadd_rn(e.ex, d) : __fsub_rn(e.ex, d);
  if (iy) e.ey = iy > 0 ? __fadd_rn(e.ey, d) : __fsub_rn(e.ey, d);
  if (iz) e.ez = iz > 0 ? __fadd_rn(e.ez, d) : __fsub_rn(e.ez, d);
}
// f - w (e0 + 3 c . e) for direction (ix, iy, iz) of weight w
__device__ __forceinline__ float defect_remove(const BgkDefect& e, float f, float w, int ix, int iy, int iz) {
  float ce = 0.f;
  if (ix) ce = ix > 0 ? __fadd_rn(ce, e.ex) : __fsub_rn(ce, e.ex);
  if (iy) ce = iy > 0 ? __fadd_rn(ce, e.ey) : __fsub_rn(ce, e.ey);
  if (iz) ce = iz > 0 ? __fadd_rn(ce, e.ez) : __fsub_rn(ce, e.ez);
  return fmaf(-w, fmaf(3.0f, ce, e.e0), f);
}
template <bool CORRECT = true>
__device__ __forceinline__ void bgk(float (&f)[kQ], float omega, float s = 1.0f, float inv_s = 1.0f) {
  float dh, jx, jy, jz;
  moments(f, dh, jx, jy, jz);
  const float rho = 1.0f + dh * inv_s;
  const float k = inv_s / rho;
  const float ux = jx * k, uy = jy * k, uz = jz * k;
  const float A = s * rho;
  const float a3 = 3.0f * A, b45 = 4.5f * A;
  const float c0 = dh - 1.5f * A * (ux * ux + uy * uy + uz * uz);
  BgkDefect e{0.f, 0.f, 0.f, 0.f};
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    const float cu = (cx(i) ? cx(i) * ux : 0.f) + (cy(i) ? cy(i) * uy : 0.f) + (cz(i) ? cz(i) * uz : 0.f);
    const float t = i == 0 ? c0 : fmaf(cu, fmaf(b45, cu, a3), c0);
    if constexpr (CORRECT) {
      const float d = __fmul_rn(omega, fmaf(wf(i), t, -f[i]));
      defect_add(e, d, cx(i), cy(i), cz(i));
      f[i] = __fadd_rn(f[i], d);
    } else {
      f[i] = fmaf(omega, fmaf(wf(i), t, -f[i]), f[i]);
    }
  }
  if constexpr (CORRECT) {
#pragma unroll
    for (int i = 0; i < kQ; ++i) f[i] = defect_remove(e, f[i], wf(i), cx(i), cy(i), cz(i));
  }
}
// The removal where a kernel applies it: FP32 storage, not FP16-shifted.
template <typename T> constexpr bool kBgkCorrect = true;
template <> constexpr bool kBgkCorrect<__half> = false;

// ConstRhoBGK (OpenLB collision::ConstRhoBGK as block_lattice.h:134-151
// restates it, unit scale):
//   f_i <- ratio (feq_i + w_i) - w_i + (1 - omega)(f_i - feq_i),
//   ratio = 1 + dr / rho,  dr = 1 - average_rho (ratio = 1 for rho <= 1e-12).
// With feq_i + w_i = w_i rho P_i, P_i = 1 + 3 c.u + 4.5 (c.u)^2 - 1.5 |u|^2,
// that is the BGK update plus dr w_i P_i: the same relaxation arithmetic as
// bgk() (s = 1) and one extra term.  The term adds dr to the density and
// dr u to the momentum, so u is unchanged.  Returns rho - 1 before the
// collision (the density the reference's statistics sum,
// block_lattice.cpp:441-455).
__device__ __forceinline__ float bgk_const_rho(float (&f)[kQ], float omega, float dr) {
  float dh, jx, jy, jz;
  moments(f, dh, jx, jy, jz);
  const float rho = 1.0f + dh;
  const float k = 1.0f / rho;
  const float ux = jx * k, uy = jy * k, uz = jz * k;
  const float u15 = 1.5f * (ux * ux + uy * uy + uz * uz);
  const float d = rho > 1e-12f ? dr : 0.0f;
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    const float cu = (cx(i) ? cx(i) * ux : 0.f) + (cy(i) ? cy(i) * uy : 0.f) + (cz(i) ? cz(i) * uz : 0.f);
    const float q = i == 0 ? -u15 : fmaf(cu, fmaf(4.5f, cu, 3.0f), -u15);  // P_i - 1
    const float t = fmaf(rho, q, dh);                                       // (feq_i - w_i) / w_i
    f[i] = fmaf(wf(i) * d, 1.0f + q, fmaf(omega, fmaf(wf(i), t, -f[i]), f[i]));
  }
  return dh;
}

// Bouzidi interpolated bounce-back with the reference's argument roles
// (src/solver/lbm/boundary/bouzidi_pull.h:8-26); q in (0,1) guaranteed by the
// caller (q = 1 means plain half-way bounce-back).
__device__ __forceinline__ float bouzidi(float f_bb, float f_q, float f_same, float q) {
  if (q >= 1.0f) return f_bb;
  if (q >= 0.5f) {
    const float inv2q = 0.5f / q;
    return inv2q * f_bb + (1.0f - inv2q) * f_q;
  }
  return 2.0f * q * f_bb + (1.0f - 2.0f * q) * f_same;
}

}  // namespace octlb_gpu
