// sm_100a kernels of the hand-written discrete adjoint of the per-level time
// step (reverse mode).  Each kernel is the vector-Jacobian product of one
// forward kernel of lbm_kernels.cu, evaluated at the forward state that the
// host recomputes from a checkpoint (the step's input after the body force and
// the boundary fills, the save rows, the coupler's prev-macro store):
//
//   k_adj_step     BGK collide + pull stream (+ save rows, halo rotation,
//                  solid copies) -> adjoint of the step's input, scattered to
//                  the pulled slots with FP32 atomics
//                  and, in the same launch, the near-wall link rule:
//                  half-way bounce-back, Bouzidi (bouzidi_pull.h:8-26),
//                  reflect-on-pull, moving-wall term
//   (boundary fills: a cotangent landing on a fill target goes to the fill's
//                  source, with the moving-wall velocity gradient, scatter)
//   k_adj_drag     momentum-exchange force (the objective)
//   k_adj_prolong, k_adj_restrict   Lagrava coupling (one warp per item)
//   k_adj_force    gradient of the per-cell body force
//
// Adjoint populations use the forward slot layout [19][slots] in FP32; the
// parameter gradients (d/d omega, d/d coupler scales, d/d wall velocity) are
// FP64 block sums added with FP64 atomics, the body-force gradient is FP64 per
// cell.  FP32 storage only (the FP16 path is not differentiated).
#include "lbm_device.cuh"

namespace octlb_gpu {
namespace {

// Gradient accumulator slots.
enum : int { kGOmega = 0, kGProlongScale = 1, kGRestrictScale = 2, kGWallVelocity = 3, kGSlots = 4 };

// Lane-parallel feq_vjp: mu_i in lane i; every lane gets P and V.
__device__ __forceinline__ void feq_vjp_lanes(const LaneDir& d, float mu, float rho, float ux, float uy, float uz,
                                              float& P, float& Vx, float& Vy, float& Vz) {
  const float usq = ux * ux + uy * uy + uz * uz;
  const float cu = d.cx * ux + d.cy * uy + d.cz * uz;
  const float mw = d.act ? mu * d.w : 0.f;
  P = warp_sum(mw * (1.0f + 3.0f * cu + 4.5f * cu * cu - 1.5f * usq));
  const float g = mw * (3.0f + 9.0f * cu);
  const float sx = warp_sum(g * d.cx), sy = warp_sum(g * d.cy), sz = warp_sum(g * d.cz), sw = warp_sum(mw);
  Vx = rho * (sx - 3.0f * ux * sw);
  Vy = rho * (sy - 3.0f * uy * sw);
  Vz = rho * (sz - 3.0f * uz * sw);
}

// Lane-parallel read_macro: f_i in lane i -> (drho, u) in every lane, f_neq_i
// in lane i.
__device__ __forceinline__ void read_macro_lanes(const LaneDir& d, float f, float& drho, float& ux, float& uy,
                                                 float& uz, float& fneq) {
  const float fa = d.act ? f : 0.f;
  drho = warp_sum(fa);
  const float jx = warp_sum(fa * d.cx), jy = warp_sum(fa * d.cy), jz = warp_sum(fa * d.cz);
  const float rho = 1.0f + drho, inv = 1.0f / rho;
  ux = jx * inv; uy = jy * inv; uz = jz * inv;
  const float usq = ux * ux + uy * uy + uz * uz;
  const float cu = d.cx * ux + d.cy * uy + d.cz * uz;
  fneq = fa - d.w * (drho + rho * (3.0f * cu + 4.5f * cu * cu - 1.5f * usq));
}

// Lane-parallel write_vjp (see write_vjp): macro (drho, u) in every lane,
// f_neq_i and the cotangent mu_i in lane i -> cotangent of the macro state
// (ldrho, lu in every lane, lfneq_i in lane i), d/d s and d/d omega (every
// lane).
__device__ __forceinline__ void write_vjp_lanes(const LaneDir& d, float drho, float ux, float uy, float uz,
                                                float fneq, float s, int kind, float omega, float mu, float& lfneq,
                                                float& ldrho, float& lux, float& luy, float& luz, float& ds,
                                                float& dom) {
  const float rho = 1.0f + drho;
  const float usq = ux * ux + uy * uy + uz * uz;
  const float cu = d.cx * ux + d.cy * uy + d.cz * uz;
  const float fp = d.act ? d.w * (drho + rho * (3.0f * cu + 4.5f * cu * cu - 1.5f * usq)) + s * fneq : 0.f;
  float lf = mu;
  dom = 0.f;
  if (kind == kBulk) {
    const float dh = warp_sum(fp);
    const float jx = warp_sum(fp * d.cx), jy = warp_sum(fp * d.cy), jz = warp_sum(fp * d.cz);
    const float r2 = 1.0f + dh, k2 = 1.0f / r2;
    const float vx = jx * k2, vy = jy * k2, vz = jz * k2;
    const float vsq = vx * vx + vy * vy + vz * vz;
    const float cv = d.cx * vx + d.cy * vy + d.cz * vz;
    const float feq = d.w * (dh + r2 * (3.0f * cv + 4.5f * cv * cv - 1.5f * vsq));
    dom = warp_sum(d.act ? mu * (feq - fp) : 0.f);
    float P, Vx, Vy, Vz;
    feq_vjp_lanes(d, mu, r2, vx, vy, vz, P, Vx, Vy, Vz);
    lf = (1.0f - omega) * mu + omega * (P + (Vx * (d.cx - vx) + Vy * (d.cy - vy) + Vz * (d.cz - vz)) * k2);
  }
  lf = d.act ? lf : 0.f;
  feq_vjp_lanes(d, lf, rho, ux, uy, uz, ldrho, lux, luy, luz);
  lfneq = s * lf;
  ds = warp_sum(lf * (d.act ? fneq : 0.f));
}

// Lane-parallel body-force gradient of a kBulk coupler target whose stored
// cotangent mu_i (lane i) is about to be cleared.
__device__ __forceinline__ void force_grad_lanes(const LaneDir& d, float mu, double* gF, long long ncore, long long t,
                                                 int lane) {
  const float v = d.act ? 3.0f * d.w * mu : 0.f;
  const float sx = warp_sum(v * d.cx), sy = warp_sum(v * d.cy), sz = warp_sum(v * d.cz);
  if (lane == 0) {  // one contributor per cell and launch: the adds need no return trip
    atomicAdd(gF + t, static_cast<double>(sx));
    atomicAdd(gF + ncore + t, static_cast<double>(sy));
    atomicAdd(gF + 2 * ncore + t, static_cast<double>(sz));
  }
}

// Lane-parallel read_vjp: f_i and the cotangent lfneq_i in lane i, ldrho and
// lu in every lane -> cotangent of f_i in lane i.
__device__ __forceinline__ float read_vjp_lanes(const LaneDir& d, float f, float ldrho, float lux, float luy, float luz,
                                                float lfneq) {
  const float fa = d.act ? f : 0.f;
  const float dh = warp_sum(fa);
  const float jx = warp_sum(fa * d.cx), jy = warp_sum(fa * d.cy), jz = warp_sum(fa * d.cz);
  const float rho = 1.0f + dh, inv = 1.0f / rho;
  const float ux = jx * inv, uy = jy * inv, uz = jz * inv;
  float P, Vx, Vy, Vz;
  feq_vjp_lanes(d, lfneq, rho, ux, uy, uz, P, Vx, Vy, Vz);
  return lfneq + (ldrho - P) + ((lux - Vx) * (d.cx - ux) + (luy - Vy) * (d.cy - uy) + (luz - Vz) * (d.cz - uz)) * inv;
}

// d feq_i / d (drho, u) contracted with a cotangent mu at the moments
// (drho, u) (rho = 1 + drho), feq_i = w_i (drho + rho (3 cu + 4.5 cu^2 - 1.5 u^2)):
//   P   = sum_i mu_i w_i (1 + 3 cu_i + 4.5 cu_i^2 - 1.5 u^2)        (d/d drho)
//   V_a = rho sum_i mu_i w_i (3 c_ia + 9 cu_i c_ia - 3 u_a)         (d/d u_a)
__device__ __forceinline__ void feq_vjp(const float (&mu)[kQ], float rho, float ux, float uy, float uz, float& P,
                                        float& Vx, float& Vy, float& Vz) {
  const float usq = ux * ux + uy * uy + uz * uz;
  float p = 0.f, sx = 0.f, sy = 0.f, sz = 0.f, sw = 0.f;
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    const float cu = cx(i) * ux + cy(i) * uy + cz(i) * uz;
    const float mw = mu[i] * wf(i);
    p += mw * (1.0f + 3.0f * cu + 4.5f * cu * cu - 1.5f * usq);
    const float g = mw * (3.0f + 9.0f * cu);
    sx += g * cx(i);
    sy += g * cy(i);
    sz += g * cz(i);
    sw += mw;
  }
  P = p;
  Vx = rho * (sx - 3.0f * ux * sw);
  Vy = rho * (sy - 3.0f * uy * sw);
  Vz = rho * (sz - 3.0f * uz * sw);
}

// VJP of bgk(f, omega) (unit scale) at the pre-collision f, in place
// (mu -> lam = J^T mu, J = (1 - omega) I + omega d feq / d f), through
// weighted moments of the cotangent: the equilibrium is quadratic in c_i, so every contraction of mu with
// d feq / d(rho, u) is a combination of
//   M0 = sum w_i mu_i,  M1 = sum w_i c_i mu_i,  M2 = sum w_i c_i c_i^T mu_i,
// formed from the opposite-pair sums and differences of mu (D3Q19 order:
// directions 10..18 are c_10 = +x, +y, +z, (1,1,0), (1,-1,0), (1,0,1),
// (1,0,-1), (0,1,1), (0,1,-1), and 1..9 their opposites):
//   P = M0 (1 - 1.5 u^2) + 3 u.M1 + 4.5 u.M2.u,
//   V = rho (3 M1 + 9 M2 u - 3 M0 u),
//   lam_j = (1 - omega) mu_j + omega (P - V.u / rho + V.c_j / rho).
// Returns sum_i mu_i (feq_i - f_i) (d/d omega); fg = 3 M1, the gradient of
// the body-force term 3 w_i c_i.F added to the cell whose cotangent is mu.
__device__ __forceinline__ float bgk_vjp_moments(const float (&f)[kQ], float omega, float (&mu)[kQ], float& fgx,
                                                 float& fgy, float& fgz) {
  float dh, jx, jy, jz;
  moments(f, dh, jx, jy, jz);
  const float rho = 1.0f + dh, k = 1.0f / rho;
  const float ux = jx * k, uy = jy * k, uz = jz * k;
  const float usq = ux * ux + uy * uy + uz * uz;
  constexpr float w0 = 1.0f / 3.0f, wa = 1.0f / 18.0f, wg = 1.0f / 36.0f;  // rest, axis, diagonal
  float sp[10], dp[10];
#pragma unroll
  for (int q = 1; q <= 9; ++q) {
    sp[q] = mu[q + 9] + mu[q];
    dp[q] = mu[q + 9] - mu[q];
  }
  const float m1x = fmaf(wa, dp[1], wg * ((dp[4] + dp[5]) + (dp[6] + dp[7])));
  const float m1y = fmaf(wa, dp[2], wg * ((dp[4] - dp[5]) + (dp[8] + dp[9])));
  const float m1z = fmaf(wa, dp[3], wg * ((dp[6] - dp[7]) + (dp[8] - dp[9])));
  const float mxx = fmaf(wa, sp[1], wg * ((sp[4] + sp[5]) + (sp[6] + sp[7])));
  const float myy = fmaf(wa, sp[2], wg * ((sp[4] + sp[5]) + (sp[8] + sp[9])));
  const float mzz = fmaf(wa, sp[3], wg * ((sp[6] + sp[7]) + (sp[8] + sp[9])));
  const float mxy = wg * (sp[4] - sp[5]), mxz = wg * (sp[6] - sp[7]), myz = wg * (sp[8] - sp[9]);
  const float m0 = fmaf(w0, mu[0], fmaf(wa, (sp[1] + sp[2]) + sp[3],
                                        wg * (((sp[4] + sp[5]) + (sp[6] + sp[7])) + (sp[8] + sp[9]))));
  float sf = 0.f;
#pragma unroll
  for (int i = 0; i < kQ; ++i) sf = fmaf(mu[i], f[i], sf);
  const float mux = mxx * ux + mxy * uy + mxz * uz;  // M2 u
  const float muy = mxy * ux + myy * uy + myz * uz;
  const float muz = mxz * ux + myz * uy + mzz * uz;
  const float um1 = ux * m1x + uy * m1y + uz * m1z;
  const float um2u = ux * mux + uy * muy + uz * muz;
  const float quad = 3.0f * um1 + 4.5f * um2u - 1.5f * usq * m0;
  const float P = m0 + quad;
  const float dom = fmaf(dh, m0, rho * quad) - sf;
  const float vx = rho * (3.0f * m1x + 9.0f * mux - 3.0f * ux * m0);
  const float vy = rho * (3.0f * m1y + 9.0f * muy - 3.0f * uy * m0);
  const float vz = rho * (3.0f * m1z + 9.0f * muz - 3.0f * uz * m0);
  const float oA = omega * (P - (vx * ux + vy * uy + vz * uz) * k);
  const float obx = omega * vx * k, oby = omega * vy * k, obz = omega * vz * k;
  const float om1 = 1.0f - omega;
#pragma unroll
  for (int j = 0; j < kQ; ++j) {
    float t = oA;
    if (cx(j) != 0) t += cx(j) > 0 ? obx : -obx;
    if (cy(j) != 0) t += cy(j) > 0 ? oby : -oby;
    if (cz(j) != 0) t += cz(j) > 0 ? obz : -obz;
    mu[j] = fmaf(om1, mu[j], t);
  }
  fgx = 3.0f * m1x;
  fgy = 3.0f * m1y;
  fgz = 3.0f * m1z;
  return dom;
}

// VJP of read_macro (level_coupler.cpp:183-189) at the saved populations f:
// cotangent lm of (drho, u, f_neq) -> cotangent lf of f.
__device__ __forceinline__ void read_vjp(const float (&f)[kQ], const Macro& lm, float (&lf)[kQ]) {
  float dh, jx, jy, jz;
  moments(f, dh, jx, jy, jz);
  const float rho = 1.0f + dh, inv = 1.0f / rho;
  const float ux = jx * inv, uy = jy * inv, uz = jz * inv;
  float P, Vx, Vy, Vz;
  feq_vjp(lm.fneq, rho, ux, uy, uz, P, Vx, Vy, Vz);
  const float a0 = lm.drho - P;
  const float ax = (lm.ux - Vx) * inv, ay = (lm.uy - Vy) * inv, az = (lm.uz - Vz) * inv;
#pragma unroll
  for (int j = 0; j < kQ; ++j)
    lf[j] = lm.fneq[j] + a0 + ax * (cx(j) - ux) + ay * (cy(j) - uy) + az * (cz(j) - uz);
}



__device__ __forceinline__ void add_grad(double* g, int slot, double v) {
  double a[1] = {v};
  block_reduce<1>(a);
  if (threadIdx.x == 0 && a[0] != 0.0) atomicAdd(g + slot, a[0]);
}

// Cotangent v of population i at slot s of the step's input: a boundary-fill
// target (never stored, see pull_value) passes it to the fill's source and
// to the moving-wall velocity gradient (gw).
__device__ __forceinline__ void scatter(const StepArgs& a, float* lamX, int i, long long s, float v, float& gw) {
  if (s >= a.halo_base && a.fill_of) {
    const int fo = __ldg(a.fill_of + (s - a.halo_base) * kQ + i);
    if (fo >= 0) {
      const BBOp& op = a.fills[fo];
      atomicAdd(lamX + op.src_pop * a.qs + op.src, v);
      gw += v * op.dadd;
      return;
    }
  }
  atomicAdd(lamX + i * a.qs + s, v);
}

// Near-wall cells (the link rule with host-resolved slots, see k_step_near),
// one warp per cell, lane i on direction i.  Every load (tables, the fill
// behind the pulled slot, the input, the cotangents) is issued before the
// first store, so the warp waits for memory about three times, not once per
// dependent access.
__device__ __forceinline__ float adj_near_cell(const StepArgs& a, const NearTables& nt, int k, int lane,
                                               float* __restrict__ lamY, float* lamX, float* __restrict__ lamS,
                                               double* gF, float& gw) {
  float dom = 0.f;
  if (k < nt.n) {
    const float* src = static_cast<const float*>(a.src);
    const long long qs = a.qs;
    const LaneDir d = lane_dir(lane);
    const uint32_t t = static_cast<uint32_t>(__ldg(nt.cells + k));
    const uint32_t mask = __ldg(nt.mask + k);
    const int sl = d.act ? __ldg(nt.slot + lane * nt.n + k) : 0;
    const float q = d.act ? __ldg(nt.q + lane * nt.n + k) : 1.f;
    const float wadd = d.act ? __ldg(nt.add + lane * nt.n + k) : 0.f;
    const bool link = d.act && ((mask >> lane) & 1u);
    // the slot's value (a boundary fill is evaluated from its source) and
    // where its cotangent goes
    long long tgt = lane * qs + sl;
    float fadd = 0.f, fdadd = 0.f;
    bool fill = false;
    if (d.act && sl >= a.halo_base && a.fill_of) {
      const int fo = __ldg(a.fill_of + (sl - a.halo_base) * kQ + lane);
      if (fo >= 0) {
        const BBOp op = a.fills[fo];
        tgt = op.src_pop * qs + op.src;
        fadd = op.add;
        fdadd = op.dadd;
        fill = true;
      }
    }
    const uint8_t fl = __ldg(a.flags + t);
    const float val = d.act ? __ldg(src + tgt) + fadd : 0.f;
    const float own = d.act ? __ldg(src + lane * qs + t) : 0.f;
    const float mu = d.act ? lamY[lane * qs + t] : 0.f;
    float* ls = nullptr;
    float lsv = 0.f;
    if ((fl & kFlagSave) && d.act) {
      ls = lamS + static_cast<long long>(__ldg(a.save_idx + t)) * kQ + lane;
      lsv = *ls;
    }
    if (d.act) lamY[lane * qs + t] = 0.f;
    if (ls) *ls = 0.f;
    const float own_opp = __shfl_sync(0xffffffffu, own, d.opp);
    float f = val;
    if (link) f = (q < 1.0f ? bouzidi(own_opp, val, own, q) : own_opp) + wadd;
    float lam = mu;
    if ((fl & kKindMask) == kBulk) {
      force_grad_lanes(d, mu, gF, a.ncore, t, lane);
      // moments by warp sums (the linearisation point needs no bitwise match)
      const float fa = d.act ? f : 0.f;
      const float dh = warp_sum(fa);
      const float jx = warp_sum(fa * d.cx), jy = warp_sum(fa * d.cy), jz = warp_sum(fa * d.cz);
      const float rho = 1.0f + dh, kr = 1.0f / rho;
      const float ux = jx * kr, uy = jy * kr, uz = jz * kr;
      const float usq = ux * ux + uy * uy + uz * uz;
      const float cu = d.cx * ux + d.cy * uy + d.cz * uz;
      const float feq = d.w * (dh + rho * (3.0f * cu + 4.5f * cu * cu - 1.5f * usq));
      dom = warp_sum(d.act ? mu * (feq - f) : 0.f);
      float P, Vx, Vy, Vz;
      feq_vjp_lanes(d, mu, rho, ux, uy, uz, P, Vx, Vy, Vz);
      lam = (1.0f - a.omega) * mu + a.omega * (P + (Vx * (d.cx - ux) + Vy * (d.cy - uy) + Vz * (d.cz - uz)) * kr);
    }
    lam += lsv;
    // the link rule in reverse: shares to own[opp(i)] (to_opp), own[i]
    // (to_own) and the value read at the slot (to_val)
    float to_opp = 0.f, to_own = 0.f, to_val = d.act ? lam : 0.f;
    if (link) {
      to_val = 0.f;
      if (q >= 1.0f) {
        to_opp = lam;
      } else if (q >= 0.5f) {
        const float inv2q = 0.5f / q;
        to_opp = inv2q * lam;
        to_val = (1.0f - inv2q) * lam;
      } else {
        to_opp = 2.0f * q * lam;
        to_own = (1.0f - 2.0f * q) * lam;
      }
    }
    const float own_total = to_own + __shfl_sync(0xffffffffu, to_opp, d.opp);
    if (d.act) {
      if (to_val != 0.f) {
        atomicAdd(lamX + tgt, to_val);
        if (fill) gw += to_val * fdadd;
      }
      if (own_total != 0.f) atomicAdd(lamX + lane * qs + t, own_total);
    }
  }
  return dom;
}

// Step VJP over the cells the slot-map step streams (one CTA per block, the
// block's slot map in shared memory); CTAs after the nblk block CTAs take the
// halo rotation items.  a.src = the step's input (after force and fills);
// lamY = cotangent of the step's output, lamX += cotangent of its input.
template <bool LINKS, bool FLAGS>
__global__ void __launch_bounds__(kThreads, LINKS ? 3 : 2) k_adj_step(const StepArgs a, const NearTables nt, float* __restrict__ lamY,
                                                      float* lamX, float* __restrict__ lamS, double* g,
                                                      double* gF) {
  extern __shared__ int smap[];
  constexpr uint32_t kParts = 2;  // two CTAs per block, one cell per thread at a time
  // first CTAs: the near-wall cells, one warp each
  const uint32_t near_ctas = LINKS ? (static_cast<uint32_t>(nt.n) + kThreads / 32 - 1) / (kThreads / 32) : 0;
  if (LINKS && blockIdx.x < near_ctas) {
    pdl_wait();
    const int lane = threadIdx.x & 31;
    float gw = 0.f;
    const float dom = adj_near_cell(a, nt, static_cast<int>(blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5)), lane,
                                    lamY, lamX, lamS, gF, gw);
    double a2[2] = {lane == 0 ? static_cast<double>(dom) : 0.0, static_cast<double>(gw)};
    block_reduce<2>(a2);
    if (threadIdx.x == 0) {
      if (a2[0] != 0.0) atomicAdd(g + kGOmega, a2[0]);
      if (a2[1] != 0.0) atomicAdd(g + kGWallVelocity, a2[1]);
    }
    return;
  }
  const uint32_t bid = blockIdx.x - near_ctas;
  const uint32_t b = bid / kParts, part = bid % kParts;
  const long long qs = a.qs;
  if (b >= static_cast<uint32_t>(a.nblk)) {
    pdl_wait();
    const uint32_t k = (bid - a.nblk * kParts) * kThreads + threadIdx.x;
    float gw = 0.f;
    if (k < static_cast<uint32_t>(a.n_open)) {
      long long d, sl;
      int i;
      rotate_slots(a, k, d, sl, i);
      scatter(a, lamX, i, sl, lamY[i * qs + d], gw);
      lamY[i * qs + d] = 0.f;
    }
    add_grad(g, kGWallVelocity, static_cast<double>(gw));
    return;
  }
  const int np = a.np, np3 = np * np * np;
  const int* gm = a.slot_map + static_cast<long long>(b) * np3;
  for (int k = threadIdx.x; k < np3; k += kThreads) smap[k] = gm[k];
  const bool moving = a.blk_moving[b] != 0;  // uniform over the CTA
  __syncthreads();
  pdl_wait();
  const float* src = static_cast<const float*>(a.src);
  const uint32_t n = a.n, n3 = n * n * n, span = n3 / kParts;
  double dom = 0.0;
  float gw = 0.f;
  for (uint32_t tl = part * span + threadIdx.x; tl < (part + 1) * span; tl += kThreads) {
    const uint32_t t = b * n3 + tl;
    const uint32_t x = a.div_n2.div(tl), r = tl - x * n * n, y = a.div_n.div(r);
    const int P = (static_cast<int>(x + 1) * np + static_cast<int>(y + 1)) * np + static_cast<int>(r - y * n + 1);
    const uint8_t fl = FLAGS ? __ldg(a.flags + t) : 0;
    if (LINKS && (fl & kKindMask) == kSolid) {
      float v[kQ];  // loads before stores (see below)
#pragma unroll
      for (int i = 0; i < kQ; ++i) v[i] = lamY[i * qs + t];
#pragma unroll
      for (int i = 0; i < kQ; ++i) {
        atomicAdd(lamX + i * qs + t, v[i]);
        lamY[i * qs + t] = 0.f;
      }
      continue;
    }
    if (LINKS && (fl & kFlagNear)) continue;  // the near-cell CTAs take it
    // All loads are issued before the first store: a warp issues in order,
    // and a load the compiler may not move above a store (lamY[i] and
    // lamY[i + 1] may alias for all it knows) costs a full memory round trip.
    // The recorded input is read through the read-only path.
    float f[kQ], lam[kQ];
#pragma unroll
    for (int i = 0; i < kQ; ++i) {
      const int sm = smap[P - a.off_pad[i]];  // < 0: bounce-back wall position (see k_step_map)
      f[i] = __ldg(src + (sm >= 0 ? i * qs + sm : opp(i) * qs + t));
      lam[i] = lamY[i * qs + t];  // the output's cotangent, turned into the input's below
    }
    if (moving) {  // moving-wall markers: only blocks flagged in blk_moving
#pragma unroll
      for (int i = 0; i < kQ; ++i) {
        const int sm = smap[P - a.off_pad[i]];
        if (sm < -1) f[i] += __ldg(a.wall_add + (-sm - 2) * kQ + i);
      }
    }
    const bool bulk = !FLAGS || (fl & kKindMask) == kBulk;
    float fgx = 0.f, fgy = 0.f, fgz = 0.f;  // body-force gradient of this cell
    if (bulk) dom += bgk_vjp_moments(f, a.omega, lam, fgx, fgy, fgz);
    // no store before this point: the save row's loads need not wait
    const bool save = FLAGS && (fl & kFlagSave);
    float* ls = save ? lamS + static_cast<long long>(__ldg(a.save_idx + t)) * kQ : nullptr;
    if (save) {
#pragma unroll
      for (int i = 0; i < kQ; ++i) lam[i] += ls[i];
    }
#pragma unroll
    for (int i = 0; i < kQ; ++i) lamY[i * qs + t] = 0.f;
    if (save) {
#pragma unroll
      for (int i = 0; i < kQ; ++i) ls[i] = 0.f;
    }
    if (bulk) {  // one contributor per cell and launch: no return trip needed
      atomicAdd(gF + t, static_cast<double>(fgx));
      atomicAdd(gF + a.ncore + t, static_cast<double>(fgy));
      atomicAdd(gF + 2ull * a.ncore + t, static_cast<double>(fgz));
    }
    if (moving) {
#pragma unroll
      for (int i = 0; i < kQ; ++i) {
        const int sm = smap[P - a.off_pad[i]];
        if (sm < -1) gw += lam[i] * __ldg(a.wall_dadd + (-sm - 2) * kQ + i);
      }
    }
#pragma unroll
    for (int i = 0; i < kQ; ++i) {
      const int sm = smap[P - a.off_pad[i]];
      atomicAdd(lamX + (sm >= 0 ? i * qs + sm : opp(i) * qs + t), lam[i]);
    }
  }
  double a2[2] = {dom, static_cast<double>(gw)};
  block_reduce<2>(a2);
  if (threadIdx.x == 0) {
    if (a2[0] != 0.0) atomicAdd(g + kGOmega, a2[0]);
    if (a2[1] != 0.0) atomicAdd(g + kGWallVelocity, a2[1]);
  }
}


// Body-force gradient: the forcing term 3 w_i c_i . F is added to the stored
// populations of kBulk cells at the start of the step whose input cotangent
// is lam.  gF is [3][ncore] FP64.
__global__ void __launch_bounds__(kThreads) k_adj_force(const StepArgs a, const float* __restrict__ lam,
                                                       double* gF) {
  pdl_wait();

  const uint32_t t = blockIdx.x * kThreads + threadIdx.x;
  if (t >= a.ncore) return;
  if (a.flags && (a.flags[t] & kKindMask) != kBulk) return;
  float sx = 0.f, sy = 0.f, sz = 0.f;
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    const float v = 3.0f * wf(i) * lam[i * a.qs + t];
    sx += cx(i) * v;
    sy += cy(i) * v;
    sz += cz(i) * v;
  }
  gF[t] += sx;
  gF[a.ncore + t] += sy;
  gF[2ull * a.ncore + t] += sz;
}

// Momentum-exchange force in reverse (see k_drag): the objective adds
// coef * F[comp], F = -sum (f_out + f_bar) c_i over the item's links.
template <bool LINKS>
__device__ __forceinline__ void adj_drag_item(const StepArgs& a, const DragItem it, float* lamX, float coef, int comp,
                                              float& gw) {
  const float* src = static_cast<const float*>(a.src);
  const long long qs = a.qs;
  float own[kQ], down[kQ];
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    own[i] = src[i * qs + it.slot];
    down[i] = 0.f;
  }
  const uint8_t fl = a.flags[it.slot];
  const int li = (LINKS && (fl & kFlagLink)) ? a.link_idx[it.slot] : -1;
  const Cell c = cell_of(a, static_cast<uint32_t>(it.slot));
#pragma unroll
  for (int i = 1; i < kQ; ++i) {
    if (!(it.mask & (1u << i))) continue;
    const int j = opp(i);
    const int ci = comp == 0 ? cx(i) : (comp == 1 ? cy(i) : cz(i));
    const float gs = -coef * static_cast<float>(ci);  // d J / d (f_out + f_bar)
    if (gs == 0.f) continue;
    down[i] += gs;                                     // f_out = g_i(x)
    if constexpr (LINKS) {
      float qv = 1.0f;
      if (li >= 0) qv = a.link_rec[li * 38 + j];
      if (qv >= 1.0f) {
        down[i] += gs;
      } else {
        bool nhalo;
        const long long nb = resolve(a, c.b, static_cast<int>(c.x) + 1 + cx(j), static_cast<int>(c.y) + 1 + cy(j),
                                     static_cast<int>(c.z) + 1 + cz(j), nhalo);
        const int nk = nhalo ? kBulk : (a.flags[nb] & kKindMask);
        if (qv >= 0.5f) {
          const float inv2q = 0.5f / qv;
          down[i] += inv2q * gs;
          if (nk == kBulk) scatter(a, lamX, j, nb, (1.0f - inv2q) * gs, gw);
          else down[j] += (1.0f - inv2q) * gs;
        } else {
          down[i] += 2.0f * qv * gs;
          down[j] += (1.0f - 2.0f * qv) * gs;
        }
      }
    } else {
      atomicAdd(lamX + j * qs + it.slot + a.off[i], gs);  // plain pull from x + c_i
    }
  }
#pragma unroll
  for (int i = 0; i < kQ; ++i)
    if (down[i] != 0.f) atomicAdd(lamX + i * qs + it.slot, down[i]);
}

template <bool LINKS>
__global__ void __launch_bounds__(kThreads) k_adj_drag(const StepArgs a, const DragItem* items, int nitems,
                                                      float* lamX, float coef, int comp, double* g) {
  pdl_wait();
  const int t = blockIdx.x * kThreads + threadIdx.x;
  float gw = 0.f;
  if (t < nitems) adj_drag_item<LINKS>(a, items[t], lamX, coef, comp, gw);
  add_grad(g, kGWallVelocity, static_cast<double>(gw));
}


// Prolongation in reverse, one warp per item, lane i on population i
// (half = 1: w = (prev + m) / 2; half = 0: w = m and prev <- m).  The fine
// target's cotangent (zeroed: it was overwritten) becomes the cotangent of w;
// lam_m collects d/d m per item and lam_prev is the cotangent of the prev
// store (lanes 0..18 own the f_neq components 4 + i, lanes 19..22 the
// components drho, ux, uy, uz).  The half-time call, the last use of m,
// also takes m's cotangent through read_macro to the coarse save row.
__global__ void __launch_bounds__(kThreads)
k_adj_prolong(const ProlongItem* items, int nitems, const float* coarse_save, const float* prev, int half,
              float* lam_fine, long long fine_qs, float s, float omega, float* lam_m, float* lam_prev,
              float* lam_save, double* g, double* gF_fine, long long fine_ncore) {
  const int w = (blockIdx.x * kThreads + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  ProlongItem it{};
  if (w < nitems) it = items[w];  // constant table: read before the wait
  pdl_wait();
  float ds = 0.f, dom = 0.f;
  if (w < nitems) {
    const LaneDir d = lane_dir(lane);
    // every load first (see adj_near_cell)
    const float* row = coarse_save + static_cast<long long>(it.coarse_save) * kQ;
    const float f = d.act ? __ldg(row + lane) : 0.f;
    const float* pv = prev + static_cast<long long>(it.prev) * 23;
    float pv0 = 0.f, pv1 = 0.f, pv2 = 0.f, pv3 = 0.f, pvf = 0.f;
    if (half) {
      pv0 = __ldg(pv); pv1 = __ldg(pv + 1); pv2 = __ldg(pv + 2); pv3 = __ldg(pv + 3);
      pvf = d.act ? __ldg(pv + 4 + lane) : 0.f;
    }
    float* p = lam_fine + lane * fine_qs + it.fine_slot;
    const float mu = d.act ? *p : 0.f;
    // the component of the prev / m cotangents this lane owns
    const int comp = lane < kQ ? 4 + lane : (lane < kQ + 4 ? lane - kQ : -1);
    float* lm = lam_m + static_cast<long long>(w) * 23;
    float* lp = lam_prev + static_cast<long long>(it.prev) * 23;
    const float lmv = comp >= 0 ? lm[comp] : 0.f, lpv = comp >= 0 ? lp[comp] : 0.f;
    if (d.act) *p = 0.f;
    float drho, ux, uy, uz, fneq;
    read_macro_lanes(d, f, drho, ux, uy, uz, fneq);
    float wd = drho, wx = ux, wy = uy, wz = uz, wf_ = fneq;
    if (half) {
      wd = 0.5f * (pv0 + drho); wx = 0.5f * (pv1 + ux); wy = 0.5f * (pv2 + uy); wz = 0.5f * (pv3 + uz);
      wf_ = d.act ? 0.5f * (pvf + fneq) : 0.f;
    }
    if (it.fine_kind == kBulk) force_grad_lanes(d, mu, gF_fine, fine_ncore, it.fine_slot, lane);
    float lfneq, ldrho, lux, luy, luz;
    write_vjp_lanes(d, wd, wx, wy, wz, wf_, s, it.fine_kind, omega, mu, lfneq, ldrho, lux, luy, luz, ds, dom);
    const float lw = lane < kQ ? lfneq : (lane == kQ ? ldrho : (lane == kQ + 1 ? lux : (lane == kQ + 2 ? luy : luz)));
    float total = 0.f;
    if (comp >= 0) {
      if (half) {
        total = lmv + 0.5f * lw;
        lp[comp] = lpv + 0.5f * lw;
        lm[comp] = 0.f;
      } else {
        lm[comp] = lmv + (lw + lpv);
        lp[comp] = 0.f;
      }
    }
    if (half) {
      // cotangent of m -> coarse save row
      const float tdrho = __shfl_sync(0xffffffffu, total, kQ), tux = __shfl_sync(0xffffffffu, total, kQ + 1);
      const float tuy = __shfl_sync(0xffffffffu, total, kQ + 2), tuz = __shfl_sync(0xffffffffu, total, kQ + 3);
      const float lf = read_vjp_lanes(d, f, tdrho, tux, tuy, tuz, d.act ? total : 0.f);
      if (d.act) atomicAdd(lam_save + static_cast<long long>(it.coarse_save) * kQ + lane, lf);
    }
  }
  double a2[2] = {lane == 0 ? static_cast<double>(dom) : 0.0, lane == 0 ? static_cast<double>(ds) : 0.0};
  block_reduce<2>(a2);
  if (threadIdx.x == 0) {
    if (a2[0] != 0.0) atomicAdd(g + kGOmega, a2[0]);
    if (a2[1] != 0.0) atomicAdd(g + kGProlongScale, a2[1]);
  }
}

// Restriction in reverse, one warp per item as forward: lane 0 recomputes the
// written state, takes the coarse target's cotangent (zeroed), and sends the
// macro cotangent to the fine centre row and the f_neq average to every row.
__global__ void __launch_bounds__(kThreads)
k_adj_restrict(const RestrictItem* items, int nitems, const float* fine_save, float* lam_coarse, long long coarse_qs,
               float s, float omega, float* lam_save, double* g, double* gF_coarse, long long coarse_ncore) {
  const int w = (blockIdx.x * kThreads + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const RestrictItem& it = items[w < nitems ? w : 0];
  // constant table: read before the wait
  const int row = w >= nitems ? -1 : (lane == 0 ? it.fine_save : (lane <= it.nnb ? it.nb_save[lane - 1] : -1));
  const long long cslot = w < nitems ? it.coarse_slot : 0;
  const int ckind = w < nitems ? it.coarse_kind : 0, nnb = w < nitems ? it.nnb : 0;
  pdl_wait();
  float ds = 0.f, dom = 0.f;
  if (w < nitems) {
    const LaneDir d = lane_dir(lane);
    float* p = lam_coarse + lane * coarse_qs + cslot;
    const float mu = d.act ? *p : 0.f;
    Macro m;
    float f[kQ];
    if (row >= 0) {
#pragma unroll
      for (int i = 0; i < kQ; ++i) f[i] = __ldg(fine_save + static_cast<long long>(row) * kQ + i);
      read_macro(f, m);
    }
    if (d.act) *p = 0.f;
    float sum[kQ];
#pragma unroll
    for (int i = 0; i < kQ; ++i) {
      float v = row >= 0 ? m.fneq[i] : 0.f;
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      sum[i] = v;
    }
    const float inv = 1.0f / static_cast<float>(nnb + 1);
    // r = (centre drho, u; f_neq average) spread over the lanes
    float rf = 0.f;
#pragma unroll
    for (int i = 0; i < kQ; ++i) {
      const float v = __shfl_sync(0xffffffffu, sum[i], 0) * inv;
      if (lane == i) rf = v;
    }
    const float rd = __shfl_sync(0xffffffffu, m.drho, 0), rx = __shfl_sync(0xffffffffu, m.ux, 0);
    const float ry = __shfl_sync(0xffffffffu, m.uy, 0), rz = __shfl_sync(0xffffffffu, m.uz, 0);
    if (ckind == kBulk) force_grad_lanes(d, mu, gF_coarse, coarse_ncore, cslot, lane);
    float lfneq, ldrho, lux, luy, luz;
    write_vjp_lanes(d, rd, rx, ry, rz, rf, s, ckind, omega, mu, lfneq, ldrho, lux, luy, luz, ds, dom);
    // row k's cotangent: f_neq part inv * lfneq (all rows), drho / u (centre)
    Macro lm;
    lm.drho = lane == 0 ? ldrho : 0.f;
    lm.ux = lane == 0 ? lux : 0.f;
    lm.uy = lane == 0 ? luy : 0.f;
    lm.uz = lane == 0 ? luz : 0.f;
#pragma unroll
    for (int i = 0; i < kQ; ++i) lm.fneq[i] = __shfl_sync(0xffffffffu, lfneq, i) * inv;
    if (row >= 0) {
      float lf[kQ];
      read_vjp(f, lm, lf);
      float* ls = lam_save + static_cast<long long>(row) * kQ;
#pragma unroll
      for (int i = 0; i < kQ; ++i) atomicAdd(ls + i, lf[i]);
    }
  }
  double a2[2] = {lane == 0 ? static_cast<double>(dom) : 0.0, lane == 0 ? static_cast<double>(ds) : 0.0};
  block_reduce<2>(a2);
  if (threadIdx.x == 0) {
    if (a2[0] != 0.0) atomicAdd(g + kGOmega, a2[0]);
    if (a2[1] != 0.0) atomicAdd(g + kGRestrictScale, a2[1]);
  }
}

inline uint32_t grid_of(long long items, int threads) { return static_cast<uint32_t>((items + threads - 1) / threads); }

}  // namespace

// ---------------------------------------------------------------- launchers
cudaError_t launch_adj_step(const StepArgs& a, const NearTables& nt, bool links, bool flags, float* lamY, float* lamX,
                            float* lamS, double* g, double* gF, cudaStream_t s) {
  cudaError_t e = cudaSuccess;
  const uint32_t near_ctas = links ? grid_of(static_cast<long long>(nt.n) * 32, kThreads) : 0;
  const dim3 grid(near_ctas + static_cast<uint32_t>(a.nblk) * 2 + grid_of(a.n_open, kThreads));
  const size_t smem = static_cast<size_t>(a.np) * a.np * a.np * sizeof(int);
  if (links) e = launch_chain(k_adj_step<true, true>, dim3(grid), dim3(kThreads), smem, s, a, nt, lamY, lamX, lamS, g, gF);
  else if (flags) e = launch_chain(k_adj_step<false, true>, dim3(grid), dim3(kThreads), smem, s, a, nt, lamY, lamX, lamS, g, gF);
  else e = launch_chain(k_adj_step<false, false>, dim3(grid), dim3(kThreads), smem, s, a, nt, lamY, lamX, lamS, g, gF);
  return e != cudaSuccess ? e : cudaGetLastError();
}
cudaError_t launch_adj_force(const StepArgs& a, const float* lam, double* gF, cudaStream_t s) {
  cudaError_t e = cudaSuccess;
  if (a.ncore == 0) return cudaSuccess;
  e = launch_chain(k_adj_force, dim3(grid_of(a.ncore, kThreads)), dim3(kThreads), 0, s, a, lam, gF);
  return e != cudaSuccess ? e : cudaGetLastError();
}
cudaError_t launch_adj_drag(const StepArgs& a, bool links, const DragItem* items, int n, float* lamX, float coef,
                            int comp, double* g, cudaStream_t s) {
  cudaError_t e = cudaSuccess;
  if (n == 0) return cudaSuccess;
  if (links) e = launch_chain(k_adj_drag<true>, dim3(grid_of(n, kThreads)), dim3(kThreads), 0, s, a, items, n, lamX, coef, comp, g);
  else e = launch_chain(k_adj_drag<false>, dim3(grid_of(n, kThreads)), dim3(kThreads), 0, s, a, items, n, lamX, coef, comp, g);
  return e != cudaSuccess ? e : cudaGetLastError();
}
cudaError_t launch_adj_prolong(const ProlongItem* items, int n, const float* coarse_save, const float* prev, int half,
                               float* lam_fine, long long fine_qs, float scale, float omega, float* lam_m,
                               float* lam_prev, float* lam_save, double* g, double* gF_fine, long long fine_ncore,
                               cudaStream_t s) {
  cudaError_t e = cudaSuccess;
  if (n == 0) return cudaSuccess;
  e = launch_chain(k_adj_prolong, dim3(grid_of(static_cast<long long>(n) * 32, kThreads)), dim3(kThreads), 0, s,
      items, n, coarse_save, prev, half, lam_fine, fine_qs, scale, omega, lam_m, lam_prev, lam_save, g, gF_fine,
      fine_ncore);
  return e != cudaSuccess ? e : cudaGetLastError();
}
cudaError_t launch_adj_restrict(const RestrictItem* items, int n, const float* fine_save, float* lam_coarse,
                                long long coarse_qs, float scale, float omega, float* lam_save, double* g,
                                double* gF_coarse, long long coarse_ncore, cudaStream_t s) {
  cudaError_t e = cudaSuccess;
  if (n == 0) return cudaSuccess;
  e = launch_chain(k_adj_restrict, dim3(grid_of(static_cast<long long>(n) * 32, kThreads)), dim3(kThreads), 0, s,
      items, n, fine_save, lam_coarse, coarse_qs, scale, omega, lam_save, g, gF_coarse, coarse_ncore);
  return e != cudaSuccess ? e : cudaGetLastError();
}

}  // namespace octlb_gpu
