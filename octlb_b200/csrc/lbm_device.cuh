// Device helpers shared by the forward kernels (lbm_kernels.cu) and the
// adjoint kernels (lbm_adjoint.cu): slot resolution of padded positions, the
// Lagrava macro state, and a fixed-order FP64 block reduction.
#ifndef OCTLB_LBM_DEVICE_CUH_
#define OCTLB_LBM_DEVICE_CUH_

#include "octlb_internal.h"

namespace octlb_gpu {
// Programmatic dependent launches enabled on this host thread (lbm_kernels.cu).
bool programmatic_launch();
namespace {

constexpr int kThreads = 256;

template <typename T>
__device__ __forceinline__ float LD(const T* base, long long qs, int i, long long slot, float inv) {
  return Store<T>::ld(base + i * qs + slot, inv);
}

// Core coordinates of core work item t (slot t).
struct Cell {
  uint32_t b, x, y, z;
};
__device__ __forceinline__ Cell cell_of(const StepArgs& a, uint32_t t) {
  const uint32_t n = a.n;
  Cell c;
  c.b = a.div_n3.div(t);
  uint32_t r = t - c.b * n * n * n;
  c.x = a.div_n2.div(r);
  r -= c.x * n * n;
  c.y = a.div_n.div(r);
  c.z = r - c.y * n;
  return c;
}

// Population i of core slot t as a reader sees it: plane i at t, or, in an
// AA-order box after an odd number of steps (a.aa_rev), plane opp(i) at the
// periodic neighbour t + c_i of the single block.
template <typename T>
__device__ __forceinline__ float LDR(const StepArgs& a, const T* base, int i, uint32_t t) {
  if (!a.aa_rev) return LD(base, a.qs, i, t, a.inv_scale);
  return Store<T>::ld(base + aa_rev_slot(a, i, t), a.inv_scale);
}

// Own halo-page slot of padded position (X, Y, Z) of block b; positions that
// no table covers are excluded by construction, the check keeps the access in
// bounds and records an error if that ever fails.
__device__ __forceinline__ long long page_slot(const StepArgs& a, uint32_t b, int X, int Y, int Z) {
  const int pg = a.page_of[b];
  const int h = a.hmap[(X * a.np + Y) * a.np + Z];
  if (pg < 0 || h < 0) {
    atomicExch(a.err, kErrHalo);
    return static_cast<long long>(b) * a.n * a.n * a.n;
  }
  return a.halo_base + static_cast<long long>(pg) * a.n_halo + h;
}

// Slot holding padded position (X, Y, Z) in [0, n+1]^3 of block b: the own
// core, the same-level neighbour's core cell the reference's exchange copies
// into that halo position, or the block's own halo page.  in_halo reports a
// position outside the core (the reference sees such sources as kBulk halo
// cells, block_lattice.cpp:510-518).
__device__ __forceinline__ long long resolve(const StepArgs& a, uint32_t b, int X, int Y, int Z,
                                             bool& in_halo) {
  const int n = a.n;
  const int ox = X == 0 ? -1 : (X == n + 1 ? 1 : 0);
  const int oy = Y == 0 ? -1 : (Y == n + 1 ? 1 : 0);
  const int oz = Z == 0 ? -1 : (Z == n + 1 ? 1 : 0);
  const long long lin = (static_cast<long long>(X - 1) * n + (Y - 1)) * n + (Z - 1);
  in_halo = (ox | oy | oz) != 0;
  if (!in_halo) return static_cast<long long>(b) * n * n * n + lin;
  const long long base = a.nbase[b * 27 + (ox + 1) * 9 + (oy + 1) * 3 + (oz + 1)];
  if (base != kOwnPage) return base + lin;
  return page_slot(a, b, X, Y, Z);
}

// Population i at slot s of the step's input.  A halo-page slot that a
// tree-boundary fill writes (the DomainBoundaryHandler::apply() position,
// before the pull) is not stored: its value is the fill's, computed from the
// fill's source (bounce-back: g_opp(i) of the wall-side cell plus the moving
// wall term; outflow: the clamped interior cell's g_i).
template <typename T>
__device__ __forceinline__ float pull_value(const StepArgs& a, const T* src, int i, long long s) {
  if (s >= a.halo_base && a.fill_of) {
    const int fo = a.fill_of[(s - a.halo_base) * kQ + i];
    if (fo >= 0) {
      const BBOp& op = a.fills[fo];
      return Store<T>::ld(src + op.src_pop * a.qs + op.src, a.inv_scale) + op.add;
    }
  }
  return Store<T>::ld(src + i * a.qs + s, a.inv_scale);
}

// Halo item k of an open block (block_lattice.h:70-89): item (page, block,
// halo index, population i); the page slot it writes, and the slot its torus
// pull reads (own core, the neighbour core the exchange copies, or the own
// halo page).
__device__ __forceinline__ void rotate_slots(const StepArgs& a, uint32_t k, long long& dst, long long& src, int& i) {
  const int4 it = reinterpret_cast<const int4*>(a.open_pages)[k];
  i = it.w;
  const int cells = a.np * a.np * a.np;
  int sp = a.hpos[it.z] - a.off_pad[i];
  sp = sp < 0 ? sp + cells : (sp >= cells ? sp - cells : sp);
  const int X = static_cast<int>(a.div_np2.div(static_cast<uint32_t>(sp)));
  const int rem = sp - X * a.np * a.np;
  const int Y = static_cast<int>(a.div_np.div(static_cast<uint32_t>(rem)));
  const int Z = rem - Y * a.np;
  bool halo;
  src = resolve(a, static_cast<uint32_t>(it.y), X, Y, Z, halo);
  dst = a.halo_base + static_cast<long long>(it.x) * a.n_halo + it.z;
}

// Lane-parallel forms (lane i < 19 holds population i): lattice vectors and
// weights by runtime index, packed 2 bits per component.
constexpr uint64_t pack_c(int a) {
  uint64_t v = 0;
  for (int i = 0; i < kQ; ++i) v |= static_cast<uint64_t>((a == 0 ? cx(i) : (a == 1 ? cy(i) : cz(i))) + 1) << (2 * i);
  return v;
}
constexpr uint64_t kPackCx = pack_c(0), kPackCy = pack_c(1), kPackCz = pack_c(2);
struct LaneDir {
  float cx, cy, cz, w;
  int opp;
  bool act;
};
__device__ __forceinline__ LaneDir lane_dir(int lane) {
  LaneDir d;
  d.act = lane < kQ;
  const int i = d.act ? lane : 0;
  const int x = static_cast<int>((kPackCx >> (2 * i)) & 3u) - 1;
  const int y = static_cast<int>((kPackCy >> (2 * i)) & 3u) - 1;
  const int z = static_cast<int>((kPackCz >> (2 * i)) & 3u) - 1;
  d.cx = static_cast<float>(x);
  d.cy = static_cast<float>(y);
  d.cz = static_cast<float>(z);
  const int nn = x * x + y * y + z * z;
  d.w = d.act ? (nn == 0 ? 1.0f / 3.0f : (nn == 1 ? 1.0f / 18.0f : 1.0f / 36.0f)) : 0.f;
  d.opp = d.act ? opp(i) : lane;
  return d;
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Every lane gets the 19 values held by lanes 0..18.
__device__ __forceinline__ void gather_lanes(float v, float (&all)[kQ]) {
#pragma unroll
  for (int i = 0; i < kQ; ++i) all[i] = __shfl_sync(0xffffffffu, v, i);
}

// BGK (unit scale) of population i = lane from the gathered pre-collision
// populations: the same operations and rounding as bgk() for direction i.
template <bool CORRECT = true>
__device__ __forceinline__ float bgk_lane(const LaneDir& d, int lane, const float (&fa)[kQ], float f, float omega) {
  float dh, jx, jy, jz;
  moments(fa, dh, jx, jy, jz);
  const float rho = 1.0f + dh * 1.0f;
  const float k = 1.0f / rho;
  const float ux = jx * k, uy = jy * k, uz = jz * k;
  const float A = 1.0f * rho;
  const float a3 = 3.0f * A, b45 = 4.5f * A;
  const float c0 = dh - 1.5f * A * (ux * ux + uy * uy + uz * uz);
  const float cu = (d.cx != 0.f ? d.cx * ux : 0.f) + (d.cy != 0.f ? d.cy * uy : 0.f) + (d.cz != 0.f ? d.cz * uz : 0.f);
  const float t = lane == 0 ? c0 : fmaf(cu, fmaf(b45, cu, a3), c0);
  if constexpr (!CORRECT) return fmaf(omega, fmaf(d.w, t, -f), f);
  // the collide's defect over all 19 directions, in bgk()'s order (every lane
  // holds the cell's populations fa), so the lane's result is bgk()'s
  BgkDefect e{0.f, 0.f, 0.f, 0.f};
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    const float cui = (cx(i) ? cx(i) * ux : 0.f) + (cy(i) ? cy(i) * uy : 0.f) + (cz(i) ? cz(i) * uz : 0.f);
    const float ti = i == 0 ? c0 : fmaf(cui, fmaf(b45, cui, a3), c0);
    defect_add(e, __fmul_rn(omega, fmaf(wf(i), ti, -fa[i])), cx(i), cy(i), cz(i));
  }
  const float g = __fadd_rn(f, __fmul_rn(omega, fmaf(d.w, t, -f)));
  const int ix = d.cx > 0.f ? 1 : (d.cx < 0.f ? -1 : 0), iy = d.cy > 0.f ? 1 : (d.cy < 0.f ? -1 : 0),
            iz = d.cz > 0.f ? 1 : (d.cz < 0.f ? -1 : 0);
  return defect_remove(e, g, d.w, ix, iy, iz);
}

// ConstRhoBGK of population i = lane (the arithmetic of bgk_const_rho for
// direction i); dh_out = rho - 1 before the collision, on every lane.
__device__ __forceinline__ float bgk_lane_const_rho(const LaneDir& d, int lane, const float (&fa)[kQ], float f,
                                                    float omega, float dr, float& dh_out) {
  float dh, jx, jy, jz;
  moments(fa, dh, jx, jy, jz);
  const float rho = 1.0f + dh;
  const float k = 1.0f / rho;
  const float ux = jx * k, uy = jy * k, uz = jz * k;
  const float u15 = 1.5f * (ux * ux + uy * uy + uz * uz);
  const float dd = rho > 1e-12f ? dr : 0.0f;
  const float cu = (d.cx != 0.f ? d.cx * ux : 0.f) + (d.cy != 0.f ? d.cy * uy : 0.f) + (d.cz != 0.f ? d.cz * uz : 0.f);
  const float q = lane == 0 ? -u15 : fmaf(cu, fmaf(4.5f, cu, 3.0f), -u15);
  const float t = fmaf(rho, q, dh);
  dh_out = dh;
  return fmaf(d.w * dd, 1.0f + q, fmaf(omega, fmaf(d.w, t, -f), f));
}

// Macro state (rho - 1, u, f_neq) of saved pre-collision populations
// (LevelCoupler::ReadMacro, level_coupler.cpp:183-189).
struct Macro {
  float drho, ux, uy, uz;
  float fneq[kQ];
};
__device__ inline void read_macro(const float* f, Macro& m) {
  float fr[kQ];
#pragma unroll
  for (int i = 0; i < kQ; ++i) fr[i] = f[i];
  float drho, jx, jy, jz;
  moments(fr, drho, jx, jy, jz);
  const float rho = 1.0f + drho, inv = 1.0f / rho;
  m.drho = drho; m.ux = jx * inv; m.uy = jy * inv; m.uz = jz * inv;
  const float usq15 = 1.5f * (m.ux * m.ux + m.uy * m.uy + m.uz * m.uz);
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    const float cu = cx(i) * m.ux + cy(i) * m.uy + cz(i) * m.uz;
    m.fneq[i] = fr[i] - wf(i) * (drho + rho * (3.0f * cu + 4.5f * cu * cu - usq15));
  }
}
// feq(rho,u) + scale * f_neq (WriteProlongation, level_coupler.cpp:191-201),
// then BGK if the target cell is kBulk: the written state is collided by the
// next step of its level before it is streamed.
template <bool CORRECT = true>
__device__ inline void write_macro_cell(const Macro& m, float s, int kind, float omega, float (&f)[kQ]) {
  const float rho = 1.0f + m.drho;
  const float usq15 = 1.5f * (m.ux * m.ux + m.uy * m.uy + m.uz * m.uz);
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    const float cu = cx(i) * m.ux + cy(i) * m.uy + cz(i) * m.uz;
    f[i] = wf(i) * (m.drho + rho * (3.0f * cu + 4.5f * cu * cu - usq15)) + s * m.fneq[i];
  }
  if (kind == kBulk) bgk<CORRECT>(f, omega);
}

// FP64 block reduction of N doubles: warp shuffles, then one warp over the
// per-warp partials; thread 0 returns the totals.
template <int N>
__device__ inline void block_reduce(double (&v)[N]) {
  __shared__ double sm[kThreads / 32][N];
#pragma unroll
  for (int k = 0; k < N; ++k)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < N; ++k) sm[wid][k] = v[k];
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int k = 0; k < N; ++k) {
      v[k] = lane < kThreads / 32 ? sm[lane][k] : 0.0;
      for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    }
  }
  __syncthreads();  // sm is reused by the next reduction of the same width
}

// Four consecutive halves (8-byte aligned) to floats, and back with
// round-to-nearest.
__device__ __forceinline__ void ld4h(const __half* p, float& a, float& b, float& c, float& d) {
  const uint2 u = *reinterpret_cast<const uint2*>(p);
  const float2 lo = __half22float2(*reinterpret_cast<const __half2*>(&u.x));
  const float2 hi = __half22float2(*reinterpret_cast<const __half2*>(&u.y));
  a = lo.x; b = lo.y; c = hi.x; d = hi.y;
}
__device__ __forceinline__ void st4h(__half* p, float a, float b, float c, float d) {
  const __half2 lo = __floats2half2_rn(a, b), hi = __floats2half2_rn(c, d);
  uint2 u;
  u.x = *reinterpret_cast<const uint32_t*>(&lo);
  u.y = *reinterpret_cast<const uint32_t*>(&hi);
  *reinterpret_cast<uint2*>(p) = u;
}

// Launches of the time-step chain: with the programmatic stream-serialisation
// attribute when enabled, so each kernel is launched as its predecessor's
// CTAs exit and runs its constant-table prologue before pdl_wait (every such
// kernel calls pdl_wait before its first dependent access).  No kernel
// triggers its dependents early: measured on the forest cases, an early
// trigger gained nothing over the implicit trigger at CTA exit.
template <typename... P, typename... A>
cudaError_t launch_chain(void (*k)(P...), dim3 g, dim3 b, size_t smem, cudaStream_t s, A&&... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = g;
  cfg.blockDim = b;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = programmatic_launch() ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, k, std::forward<A>(args)...);
}
}  // namespace
}  // namespace octlb_gpu

#endif  // OCTLB_LBM_DEVICE_CUH_
