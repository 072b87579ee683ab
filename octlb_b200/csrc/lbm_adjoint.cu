// sm_100a kernels of the hand-written discrete adjoint of the per-level time
// step (reverse mode).  Each kernel is the vector-Jacobian product of one
// forward kernel of lbm_kernels.cu, evaluated at the forward state that the
// host recomputes from a checkpoint (the step's input after the body force and
// the boundary fills, the save rows, the coupler's prev-macro store):
//
//   k_adj_step     BGK collide + pull stream (+ save rows, halo rotation,
//                  solid copies) -> adjoint of the step's input, scattered to
//                  the pulled slots with FP32 atomics
//   k_adj_near     the near-wall link rule: half-way bounce-back, Bouzidi
//                  (bouzidi_pull.h:8-26), reflect-on-pull, moving-wall term
//   k_adj_ghost    boundary fills (bounce-back / moving wall / outflow copy)
//   k_adj_drag     momentum-exchange force (the objective)
//   k_adj_prolong, k_adj_read_macro, k_adj_restrict   Lagrava coupling
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

// VJP of bgk(f, omega) (unit scale) at the pre-collision f: lam = J^T mu with
// J = (1 - omega) I + omega d feq / d f; returns sum_i mu_i (feq_i - f_i), the
// derivative with respect to omega.
__device__ __forceinline__ float bgk_vjp(const float (&f)[kQ], float omega, const float (&mu)[kQ],
                                         float (&lam)[kQ]) {
  float dh, jx, jy, jz;
  moments(f, dh, jx, jy, jz);
  const float rho = 1.0f + dh, k = 1.0f / rho;
  const float ux = jx * k, uy = jy * k, uz = jz * k;
  const float usq = ux * ux + uy * uy + uz * uz;
  float dom = 0.f;
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    const float cu = cx(i) * ux + cy(i) * uy + cz(i) * uz;
    const float feq = wf(i) * (dh + rho * (3.0f * cu + 4.5f * cu * cu - 1.5f * usq));
    dom += mu[i] * (feq - f[i]);
  }
  float P, Vx, Vy, Vz;
  feq_vjp(mu, rho, ux, uy, uz, P, Vx, Vy, Vz);
#pragma unroll
  for (int j = 0; j < kQ; ++j)
    lam[j] = (1.0f - omega) * mu[j] +
             omega * (P + (Vx * (cx(j) - ux) + Vy * (cy(j) - uy) + Vz * (cz(j) - uz)) * k);
  return dom;
}

// Macro state -> pre-BGK populations feq(m) + s f_neq (write_macro_cell
// without its collision).
__device__ __forceinline__ void macro_to_f(const Macro& m, float s, float (&f)[kQ]) {
  const float rho = 1.0f + m.drho;
  const float usq15 = 1.5f * (m.ux * m.ux + m.uy * m.uy + m.uz * m.uz);
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    const float cu = cx(i) * m.ux + cy(i) * m.uy + cz(i) * m.uz;
    f[i] = wf(i) * (m.drho + rho * (3.0f * cu + 4.5f * cu * cu - usq15)) + s * m.fneq[i];
  }
}

// VJP of write_macro_cell (level_coupler.cpp:191-201 + the collision of a
// kBulk target): cotangent mu of the written populations -> cotangent of the
// macro state (lm) and d/d s, d/d omega.
__device__ __forceinline__ void write_vjp(const Macro& m, float s, int kind, float omega, const float (&mu)[kQ],
                                          Macro& lm, float& ds, float& dom) {
  float lf[kQ];
  dom = 0.f;
  if (kind == kBulk) {
    float f[kQ];
    macro_to_f(m, s, f);
    dom = bgk_vjp(f, omega, mu, lf);
  } else {
#pragma unroll
    for (int i = 0; i < kQ; ++i) lf[i] = mu[i];
  }
  float P, Vx, Vy, Vz;
  feq_vjp(lf, 1.0f + m.drho, m.ux, m.uy, m.uz, P, Vx, Vy, Vz);
  lm.drho = P;
  lm.ux = Vx;
  lm.uy = Vy;
  lm.uz = Vz;
  ds = 0.f;
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    lm.fneq[i] = s * lf[i];
    ds += lf[i] * m.fneq[i];
  }
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

__device__ __forceinline__ void load_macro_row(const float* row, Macro& m) {
  float f[kQ];
#pragma unroll
  for (int i = 0; i < kQ; ++i) f[i] = row[i];
  read_macro(f, m);
}

__device__ __forceinline__ void macro_from23(const float* p, Macro& m) {
  m.drho = p[0]; m.ux = p[1]; m.uy = p[2]; m.uz = p[3];
#pragma unroll
  for (int i = 0; i < kQ; ++i) m.fneq[i] = p[4 + i];
}

__device__ __forceinline__ void add_grad(double* g, int slot, double v) {
  double a[1] = {v};
  block_reduce<1>(a);
  if (threadIdx.x == 0 && a[0] != 0.0) atomicAdd(g + slot, a[0]);
}

// Step VJP over the cells the slot-map step streams (one CTA per block, the
// block's slot map in shared memory); CTAs after the nblk block CTAs take the
// halo rotation items.  a.src = the step's input (after force and fills);
// lamY = cotangent of the step's output, lamX += cotangent of its input.
template <bool LINKS, bool FLAGS>
__global__ void __launch_bounds__(kThreads) k_adj_step(const StepArgs a, const float* __restrict__ lamY,
                                                      float* lamX, const float* __restrict__ lamS, double* g) {
  extern __shared__ int smap[];
  const uint32_t b = blockIdx.x;
  const long long qs = a.qs;
  if (b >= static_cast<uint32_t>(a.nblk)) {
    const uint32_t k = (b - a.nblk) * kThreads + threadIdx.x;
    if (k < static_cast<uint32_t>(a.n_open)) {
      long long d, sl;
      int i;
      rotate_slots(a, k, d, sl, i);
      atomicAdd(lamX + i * qs + sl, lamY[i * qs + d]);
    }
    return;
  }
  const int np = a.np, np3 = np * np * np;
  const int* gm = a.slot_map + static_cast<long long>(b) * np3;
  for (int k = threadIdx.x; k < np3; k += kThreads) smap[k] = gm[k];
  __syncthreads();
  const float* src = static_cast<const float*>(a.src);
  const uint32_t n = a.n, n3 = n * n * n;
  double dom = 0.0;
  for (uint32_t tl = threadIdx.x; tl < n3; tl += kThreads) {
    const uint32_t t = b * n3 + tl;
    const uint32_t x = a.div_n2.div(tl), r = tl - x * n * n, y = a.div_n.div(r);
    const int P = (static_cast<int>(x + 1) * np + static_cast<int>(y + 1)) * np + static_cast<int>(r - y * n + 1);
    const uint8_t fl = FLAGS ? a.flags[t] : 0;
    if (LINKS && (fl & kKindMask) == kSolid) {
#pragma unroll
      for (int i = 0; i < kQ; ++i) atomicAdd(lamX + i * qs + t, lamY[i * qs + t]);
      continue;
    }
    if (LINKS && (fl & kFlagNear)) continue;  // k_adj_near
    float f[kQ], mu[kQ], lam[kQ];
#pragma unroll
    for (int i = 0; i < kQ; ++i) {
      f[i] = src[i * qs + smap[P - a.off_pad[i]]];
      mu[i] = lamY[i * qs + t];
    }
    if (!FLAGS || (fl & kKindMask) == kBulk) {
      dom += bgk_vjp(f, a.omega, mu, lam);
    } else {
#pragma unroll
      for (int i = 0; i < kQ; ++i) lam[i] = mu[i];
    }
    if (FLAGS && (fl & kFlagSave)) {
      const float* ls = lamS + static_cast<long long>(a.save_idx[t]) * kQ;
#pragma unroll
      for (int i = 0; i < kQ; ++i) lam[i] += ls[i];
    }
#pragma unroll
    for (int i = 0; i < kQ; ++i) atomicAdd(lamX + i * qs + smap[P - a.off_pad[i]], lam[i]);
  }
  add_grad(g, kGOmega, dom);
}

// Near-wall cells (the link rule with host-resolved slots, see k_step_near).
__global__ void __launch_bounds__(kThreads) k_adj_near(const StepArgs a, const NearTables nt,
                                                      const float* __restrict__ lamY, float* lamX,
                                                      const float* __restrict__ lamS, double* g) {
  const int k = blockIdx.x * kThreads + threadIdx.x;
  double dom = 0.0;
  if (k < nt.n) {
    const float* src = static_cast<const float*>(a.src);
    const long long qs = a.qs;
    const uint32_t t = static_cast<uint32_t>(nt.cells[k]);
    const uint32_t mask = nt.mask[k];
    const uint8_t fl = a.flags[t];
    float own[kQ], f[kQ], mu[kQ], lam[kQ];
#pragma unroll
    for (int i = 0; i < kQ; ++i) {
      own[i] = src[i * qs + t];
      f[i] = src[i * qs + nt.slot[i * nt.n + k]];
      mu[i] = lamY[i * qs + t];
    }
#pragma unroll
    for (int i = 1; i < kQ; ++i) {
      if ((mask >> i) & 1u) {
        const float q = nt.q[i * nt.n + k];
        const float v = q < 1.0f ? bouzidi(own[opp(i)], f[i], own[i], q) : own[opp(i)];
        f[i] = v + nt.add[i * nt.n + k];
      }
    }
    if ((fl & kKindMask) == kBulk) {
      dom = bgk_vjp(f, a.omega, mu, lam);
    } else {
#pragma unroll
      for (int i = 0; i < kQ; ++i) lam[i] = mu[i];
    }
    if (fl & kFlagSave) {
      const float* ls = lamS + static_cast<long long>(a.save_idx[t]) * kQ;
#pragma unroll
      for (int i = 0; i < kQ; ++i) lam[i] += ls[i];
    }
    float down[kQ];
#pragma unroll
    for (int i = 0; i < kQ; ++i) down[i] = 0.f;
#pragma unroll
    for (int i = 0; i < kQ; ++i) {
      const long long sl = nt.slot[i * nt.n + k];
      if (i == 0 || !((mask >> i) & 1u)) {
        atomicAdd(lamX + i * qs + sl, lam[i]);
        continue;
      }
      const float q = nt.q[i * nt.n + k];
      if (q >= 1.0f) {
        down[opp(i)] += lam[i];
      } else if (q >= 0.5f) {
        const float inv2q = 0.5f / q;
        down[opp(i)] += inv2q * lam[i];
        atomicAdd(lamX + i * qs + sl, (1.0f - inv2q) * lam[i]);
      } else {
        down[opp(i)] += 2.0f * q * lam[i];
        down[i] += (1.0f - 2.0f * q) * lam[i];
      }
    }
#pragma unroll
    for (int j = 0; j < kQ; ++j)
      if (down[j] != 0.f) atomicAdd(lamX + j * qs + t, down[j]);
  }
  add_grad(g, kGOmega, dom);
}

// Boundary fills in reverse: the fill target's cotangent moves to its source
// (the target was overwritten), and the moving-wall term's velocity
// derivative collects the wall-velocity gradient.
__global__ void __launch_bounds__(kThreads) k_adj_ghost(float* lam, long long qs, const BBOp* bb, uint32_t nbb,
                                                       double* g) {
  const uint32_t u = blockIdx.x * kThreads + threadIdx.x;
  double gv = 0.0;
  if (u < nbb) {
    const BBOp op = bb[u];
    float* d = lam + op.pop * qs + op.dst;
    const float v = *d;
    *d = 0.f;
    if (v != 0.f) atomicAdd(lam + op.src_pop * qs + op.src, v);
    gv = static_cast<double>(v) * op.dadd;
  }
  add_grad(g, kGWallVelocity, gv);
}

// Body-force gradient: the forcing term 3 w_i c_i . F is added to the stored
// populations of kBulk cells at the start of the step whose input cotangent
// is lam.  gF is [3][ncore] FP64.
__global__ void __launch_bounds__(kThreads) k_adj_force(const StepArgs a, const float* __restrict__ lam,
                                                       double* gF) {
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
__global__ void __launch_bounds__(kThreads) k_adj_drag(const StepArgs a, const DragItem* items, int nitems,
                                                      float* lamX, float coef, int comp) {
  const int t = blockIdx.x * kThreads + threadIdx.x;
  if (t >= nitems) return;
  const DragItem it = items[t];
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
          if (nk == kBulk) atomicAdd(lamX + j * qs + nb, (1.0f - inv2q) * gs);
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

// Prolongation in reverse (half = 1: w = (prev + m) / 2; half = 0: w = m and
// prev <- m).  The fine target's cotangent (zeroed: it was overwritten)
// becomes the cotangent of w; lam_m collects d/d m per item, lam_prev is the
// cotangent of the prev store.
constexpr int kAdjCouplerThreads = 64;
__global__ void __launch_bounds__(kAdjCouplerThreads)
k_adj_prolong(const ProlongItem* items, int nitems, const float* coarse_save, const float* prev, int half,
              float* lam_fine, long long fine_qs, float s, float omega, float* lam_m, float* lam_prev, double* g) {
  const int t = blockIdx.x * kAdjCouplerThreads + threadIdx.x;
  float ds = 0.f, dom = 0.f;
  if (t < nitems) {
    const ProlongItem it = items[t];
    Macro m, w;
    load_macro_row(coarse_save + static_cast<long long>(it.coarse_save) * kQ, m);
    w = m;
    if (half) {
      const float* pv = prev + static_cast<long long>(it.prev) * 23;
      w.drho = 0.5f * (pv[0] + m.drho);
      w.ux = 0.5f * (pv[1] + m.ux); w.uy = 0.5f * (pv[2] + m.uy); w.uz = 0.5f * (pv[3] + m.uz);
#pragma unroll
      for (int i = 0; i < kQ; ++i) w.fneq[i] = 0.5f * (pv[4 + i] + m.fneq[i]);
    }
    float mu[kQ];
#pragma unroll
    for (int i = 0; i < kQ; ++i) {
      float* p = lam_fine + i * fine_qs + it.fine_slot;
      mu[i] = *p;
      *p = 0.f;
    }
    Macro lw;
    write_vjp(w, s, it.fine_kind, omega, mu, lw, ds, dom);
    float* lm = lam_m + static_cast<long long>(t) * 23;
    float* lp = lam_prev + static_cast<long long>(it.prev) * 23;
    const float lwv[23] = {lw.drho, lw.ux, lw.uy, lw.uz, lw.fneq[0], lw.fneq[1], lw.fneq[2], lw.fneq[3],
                           lw.fneq[4], lw.fneq[5], lw.fneq[6], lw.fneq[7], lw.fneq[8], lw.fneq[9], lw.fneq[10],
                           lw.fneq[11], lw.fneq[12], lw.fneq[13], lw.fneq[14], lw.fneq[15], lw.fneq[16],
                           lw.fneq[17], lw.fneq[18]};
    if (half) {
#pragma unroll
      for (int k = 0; k < 23; ++k) {
        lm[k] += 0.5f * lwv[k];
        lp[k] += 0.5f * lwv[k];
      }
    } else {
#pragma unroll
      for (int k = 0; k < 23; ++k) {
        lm[k] += lwv[k] + lp[k];
        lp[k] = 0.f;
      }
    }
  }
  double a2[2] = {static_cast<double>(dom), static_cast<double>(ds)};
  __shared__ double sm[kAdjCouplerThreads / 32][2];
  for (int k = 0; k < 2; ++k)
    for (int o = 16; o > 0; o >>= 1) a2[k] += __shfl_down_sync(0xffffffffu, a2[k], o);
  if ((threadIdx.x & 31) == 0) { sm[threadIdx.x >> 5][0] = a2[0]; sm[threadIdx.x >> 5][1] = a2[1]; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double d0 = 0.0, d1 = 0.0;
    for (int w = 0; w < kAdjCouplerThreads / 32; ++w) { d0 += sm[w][0]; d1 += sm[w][1]; }
    if (d0 != 0.0) atomicAdd(g + kGOmega, d0);
    if (d1 != 0.0) atomicAdd(g + kGProlongScale, d1);
  }
}

// Cotangent of the coarse macro states (lam_m per prolongation item) -> the
// coarse save rows; lam_m is cleared for the next coarse step.
__global__ void __launch_bounds__(kAdjCouplerThreads)
k_adj_read_macro(const ProlongItem* items, int nitems, const float* coarse_save, float* lam_m, float* lam_save) {
  const int t = blockIdx.x * kAdjCouplerThreads + threadIdx.x;
  if (t >= nitems) return;
  const ProlongItem it = items[t];
  float* lmv = lam_m + static_cast<long long>(t) * 23;
  Macro lm;
  macro_from23(lmv, lm);
#pragma unroll
  for (int k = 0; k < 23; ++k) lmv[k] = 0.f;
  const float* row = coarse_save + static_cast<long long>(it.coarse_save) * kQ;
  float f[kQ], lf[kQ];
#pragma unroll
  for (int i = 0; i < kQ; ++i) f[i] = row[i];
  read_vjp(f, lm, lf);
  float* ls = lam_save + static_cast<long long>(it.coarse_save) * kQ;
#pragma unroll
  for (int i = 0; i < kQ; ++i) atomicAdd(ls + i, lf[i]);
}

// Restriction in reverse, one warp per item as forward: lane 0 recomputes the
// written state, takes the coarse target's cotangent (zeroed), and sends the
// macro cotangent to the fine centre row and the f_neq average to every row.
__global__ void __launch_bounds__(kThreads)
k_adj_restrict(const RestrictItem* items, int nitems, const float* fine_save, float* lam_coarse, long long coarse_qs,
               float s, float omega, float* lam_save, double* g) {
  const int w = (blockIdx.x * kThreads + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  float ds = 0.f, dom = 0.f;
  if (w < nitems) {
    const RestrictItem& it = items[w];
    const int row = lane == 0 ? it.fine_save : (lane <= it.nnb ? it.nb_save[lane - 1] : -1);
    Macro m;
    float f[kQ];
    if (row >= 0) {
#pragma unroll
      for (int i = 0; i < kQ; ++i) f[i] = fine_save[static_cast<long long>(row) * kQ + i];
      read_macro(f, m);
    }
    float sum[kQ];
#pragma unroll
    for (int i = 0; i < kQ; ++i) {
      float v = row >= 0 ? m.fneq[i] : 0.f;
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      sum[i] = v;
    }
    const float inv = 1.0f / static_cast<float>(it.nnb + 1);
    Macro lr;
    if (lane == 0) {
      Macro r;
      r.drho = m.drho; r.ux = m.ux; r.uy = m.uy; r.uz = m.uz;
#pragma unroll
      for (int i = 0; i < kQ; ++i) r.fneq[i] = sum[i] * inv;
      float mu[kQ];
#pragma unroll
      for (int i = 0; i < kQ; ++i) {
        float* p = lam_coarse + i * coarse_qs + it.coarse_slot;
        mu[i] = *p;
        *p = 0.f;
      }
      write_vjp(r, s, it.coarse_kind, omega, mu, lr, ds, dom);
    }
    // broadcast the cotangent of r
    Macro lm;
    lm.drho = __shfl_sync(0xffffffffu, lr.drho, 0);
    lm.ux = __shfl_sync(0xffffffffu, lr.ux, 0);
    lm.uy = __shfl_sync(0xffffffffu, lr.uy, 0);
    lm.uz = __shfl_sync(0xffffffffu, lr.uz, 0);
#pragma unroll
    for (int i = 0; i < kQ; ++i) lm.fneq[i] = __shfl_sync(0xffffffffu, lr.fneq[i], 0) * inv;
    if (lane != 0) { lm.drho = 0.f; lm.ux = 0.f; lm.uy = 0.f; lm.uz = 0.f; }
    if (row >= 0) {
      float lf[kQ];
      read_vjp(f, lm, lf);
      float* ls = lam_save + static_cast<long long>(row) * kQ;
#pragma unroll
      for (int i = 0; i < kQ; ++i) atomicAdd(ls + i, lf[i]);
    }
  }
  double a2[2] = {static_cast<double>(dom), static_cast<double>(ds)};
  block_reduce<2>(a2);
  if (threadIdx.x == 0) {
    if (a2[0] != 0.0) atomicAdd(g + kGOmega, a2[0]);
    if (a2[1] != 0.0) atomicAdd(g + kGRestrictScale, a2[1]);
  }
}

inline uint32_t grid_of(long long items, int threads) { return static_cast<uint32_t>((items + threads - 1) / threads); }

}  // namespace

// ---------------------------------------------------------------- launchers
cudaError_t launch_adj_step(const StepArgs& a, bool links, bool flags, const float* lamY, float* lamX,
                            const float* lamS, double* g, cudaStream_t s) {
  const dim3 grid(static_cast<uint32_t>(a.nblk) + grid_of(a.n_open, kThreads));
  const size_t smem = static_cast<size_t>(a.np) * a.np * a.np * sizeof(int);
  if (links) k_adj_step<true, true><<<grid, kThreads, smem, s>>>(a, lamY, lamX, lamS, g);
  else if (flags) k_adj_step<false, true><<<grid, kThreads, smem, s>>>(a, lamY, lamX, lamS, g);
  else k_adj_step<false, false><<<grid, kThreads, smem, s>>>(a, lamY, lamX, lamS, g);
  return cudaGetLastError();
}
cudaError_t launch_adj_near(const StepArgs& a, const NearTables& nt, const float* lamY, float* lamX, const float* lamS,
                            double* g, cudaStream_t s) {
  if (nt.n == 0) return cudaSuccess;
  k_adj_near<<<grid_of(nt.n, kThreads), kThreads, 0, s>>>(a, nt, lamY, lamX, lamS, g);
  return cudaGetLastError();
}
cudaError_t launch_adj_ghost(float* lam, long long qs, const BBOp* bb, uint32_t nbb, double* g, cudaStream_t s) {
  if (nbb == 0) return cudaSuccess;
  k_adj_ghost<<<grid_of(nbb, kThreads), kThreads, 0, s>>>(lam, qs, bb, nbb, g);
  return cudaGetLastError();
}
cudaError_t launch_adj_force(const StepArgs& a, const float* lam, double* gF, cudaStream_t s) {
  if (a.ncore == 0) return cudaSuccess;
  k_adj_force<<<grid_of(a.ncore, kThreads), kThreads, 0, s>>>(a, lam, gF);
  return cudaGetLastError();
}
cudaError_t launch_adj_drag(const StepArgs& a, bool links, const DragItem* items, int n, float* lamX, float coef,
                            int comp, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  if (links) k_adj_drag<true><<<grid_of(n, kThreads), kThreads, 0, s>>>(a, items, n, lamX, coef, comp);
  else k_adj_drag<false><<<grid_of(n, kThreads), kThreads, 0, s>>>(a, items, n, lamX, coef, comp);
  return cudaGetLastError();
}
cudaError_t launch_adj_prolong(const ProlongItem* items, int n, const float* coarse_save, const float* prev, int half,
                               float* lam_fine, long long fine_qs, float scale, float omega, float* lam_m,
                               float* lam_prev, double* g, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_adj_prolong<<<grid_of(n, kAdjCouplerThreads), kAdjCouplerThreads, 0, s>>>(
      items, n, coarse_save, prev, half, lam_fine, fine_qs, scale, omega, lam_m, lam_prev, g);
  return cudaGetLastError();
}
cudaError_t launch_adj_read_macro(const ProlongItem* items, int n, const float* coarse_save, float* lam_m,
                                  float* lam_save, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_adj_read_macro<<<grid_of(n, kAdjCouplerThreads), kAdjCouplerThreads, 0, s>>>(items, n, coarse_save, lam_m,
                                                                                  lam_save);
  return cudaGetLastError();
}
cudaError_t launch_adj_restrict(const RestrictItem* items, int n, const float* fine_save, float* lam_coarse,
                                long long coarse_qs, float scale, float omega, float* lam_save, double* g,
                                cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_adj_restrict<<<grid_of(static_cast<long long>(n) * 32, kThreads), kThreads, 0, s>>>(
      items, n, fine_save, lam_coarse, coarse_qs, scale, omega, lam_save, g);
  return cudaGetLastError();
}

}  // namespace octlb_gpu
