// Finite-difference domain boundary conditions on the device: the post-stream
// reconstruction of velocity- and pressure-Dirichlet cells (Skordos
// InterpolatedVelocity, ApplyInterpolatedVelocityBoundaryCells,
// interpolated_velocity.h:951-1037: plane :571-636, edge :687-752, corner
// :638-685, the BoundaryLatticeView reads :213-445) and their Dirichlet
// collide (BcDispatcher::collide's velocity arm, bc_dispatcher.h:55-72 with
// BoundaryCellStatisticRho, interpolated_velocity.h:815-884).
//
// After a level step the state buffer holds, for a boundary cell, its
// post-stream populations f (the step leaves non-kBulk cells uncollided) and,
// for a fluid cell, its post-collision populations, whose velocity is the
// post-stream one (the collide keeps rho u).  The reference rewrites the
// boundary cells in place in (ix, iy, iz) order; a cell's stencil reads the
// densities of boundary cells one and two cells inward, rewritten or not by
// that order.  Edge cells read plane cells and corners read edge cells, so the
// pass runs as three launches -- planes, edges, corners -- each writing the
// rewritten populations to its own rows and reading an earlier phase's row
// where the reference's walk would have rewritten the cell already (one warp
// per cell, lane = population, every read of the stencil loaded at once).  A fourth
// launch collides the rewritten cells (velocity cells at the prescribed
// velocity, the next step's time; pressure cells are not collided) into the
// state buffer.  Every read a cell makes is resolved on the host into a table
// (FdCell): which slot or row, the velocity source (fluid populations, the
// prescribed velocity of a boundary cell, the overlap padding at rest, or a
// mirror image with flipped normal components), the density source.
// Arithmetic FP32; storage FP32 or FP16-shifted.
#include "octlb_internal.h"

namespace octlb_gpu {

namespace {

constexpr int kFdThreads = 128;

// PolynomialStartScale: 10 x^3 - 15 x^4 + 6 x^5, x = t / t_end clamped to [0, 1].
__device__ __forceinline__ float ramp(float t, float t_end) {
  if (t_end <= 0.f) return 1.f;
  const float x = fminf(fmaxf(t / t_end, 0.f), 1.f);
  return x * x * x * (10.f + x * (-15.f + 6.f * x));
}

__device__ __forceinline__ void prescribed(const FdCell* cells, int row, float t, float u[3]) {
  const FdCell& b = cells[row];
  const float r = ramp(t, b.ramp_end);
  u[0] = r * b.u_base[0];
  u[1] = r * b.u_base[1];
  u[2] = r * b.u_base[2];
}

template <typename T>
__device__ __forceinline__ void load_pops(const T* state, long long qs, long long slot, float inv_s, float f[kQ]) {
#pragma unroll
  for (int i = 0; i < kQ; ++i) f[i] = Store<T>::ld(state + i * qs + slot, inv_s);
}

__device__ __forceinline__ float sum_pops(const float f[kQ]) {
  float s = 0.f;
#pragma unroll
  for (int i = 0; i < kQ; ++i) s += f[i];
  return s;
}

// velocityBMRho: (2 sum_{c_d = o} f + sum_{c_d = 0} f + 1) / (1 + o u_d).
__device__ __forceinline__ float bm_rho(const float f[kQ], int d, int o, const float u[3]) {
  float out = 0.f, wall = 0.f;
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    const int c = d == 0 ? cx(i) : (d == 1 ? cy(i) : cz(i));
    if (c == 0) wall += f[i];
    else if (c == o) out += f[i];
  }
  return (2.f * out + wall + 1.f) / (1.f + o * u[d]);
}

// Shifted second-order equilibrium, rho w (1 + 3 cu + 4.5 cu^2 - 1.5 u^2) - w.
__device__ __forceinline__ float feq_i(int i, float rho, const float u[3], float usq) {
  const float cu = cx(i) * u[0] + cy(i) * u[1] + cz(i) * u[2];
  return rho * wf(i) * (1.f + 3.f * cu + 4.5f * cu * cu - 1.5f * usq) - wf(i);
}

// Gradient along `axis` by the one-sided second-order stencil
// -n (-3 u0 + 4 u1 - u2) / 2 (u1, u2 one and two cells inward).
__device__ __forceinline__ void normal_grad(const float u0[3], const float u1[3], const float u2[3], int n,
                                            float g[3]) {
#pragma unroll
  for (int b = 0; b < 3; ++b) g[b] = -n * (-3.f * u0[b] + 4.f * u1[b] - u2[b]) * 0.5f;
}

// Direction components and weight of a population index known only at run
// time (one lane per population), from bit masks of the D3Q19 table.
__host__ __device__ constexpr uint32_t fd_mask(int axis, int sign) {
  uint32_t m = 0;
  for (int i = 0; i < kQ; ++i)
    if ((axis == 0 ? cx(i) : axis == 1 ? cy(i) : cz(i)) == sign) m |= 1u << i;
  return m;
}
constexpr uint32_t kFdPx = fd_mask(0, 1), kFdNx = fd_mask(0, -1), kFdPy = fd_mask(1, 1), kFdNy = fd_mask(1, -1),
                   kFdPz = fd_mask(2, 1), kFdNz = fd_mask(2, -1);
__device__ __forceinline__ int c_rt(int axis, int i) {
  const uint32_t pos = axis == 0 ? kFdPx : (axis == 1 ? kFdPy : kFdPz);
  const uint32_t neg = axis == 0 ? kFdNx : (axis == 1 ? kFdNy : kFdNz);
  return static_cast<int>((pos >> i) & 1u) - static_cast<int>((neg >> i) & 1u);
}
__device__ __forceinline__ float w_rt(const int c[3]) {
  const int m = (c[0] != 0) + (c[1] != 0) + (c[2] != 0);
  return m == 0 ? 1.0f / 3.0f : (m == 1 ? 1.0f / 18.0f : 1.0f / 36.0f);
}
// Sum over the warp, every lane receiving it.
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// One boundary cell of role `role` (1 plane, 2 edge, 3 corner) per warp,
// lane i holding population i of every cell the stencil reads: all of them
// are loaded up front (independent loads, one memory latency), the moments
// and densities summed over the warp.  Rewritten populations feq(rho, u) +
// f_neq(Pi), Pi = -rho / (3 omega) (du + du^T), into the cell's row of fnew.
template <typename T>
__global__ void __launch_bounds__(kFdThreads)
k_fd_reconstruct(const T* state, long long qs, float inv_s, const FdCell* cells, const int* list, int n,
                 float* fnew, const double* time, float omega, const float* cr_shift) {
  const int w = static_cast<int>((blockIdx.x * kFdThreads + threadIdx.x) >> 5);
  if (w >= n) return;  // whole warps
  const int lane = threadIdx.x & 31;
  const bool act = lane < kQ;
  const int i = act ? lane : 0;
  const int ci[3] = {c_rt(0, i), c_rt(1, i), c_rt(2, i)};
  const int row = list[w];
  const FdCell& cell = cells[row];
  const float t = static_cast<float>(*time);
  const int nr = cell.role == 2 ? 4 : (cell.role == 3 ? 6 : 0);
  const bool own = cell.role == 1 && cell.kind != kPressureDirichlet;
  float fu[7], fr[6];
#pragma unroll
  for (int j = 0; j < 7; ++j) {
    const FdURead& r = cell.u[j];
    fu[j] = act && r.code == kFdFluid ? Store<T>::ld(state + i * qs + r.idx, inv_s) : 0.f;
  }
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    const FdRRead& r = cell.r[j];
    float v = 0.f;
    if (act && j < nr && r.code != kFdRhoConst)
      v = r.code == kFdRhoSumPre || r.code == kFdRhoBmPre ? Store<T>::ld(state + i * qs + r.idx, inv_s)
                                                          : fnew[r.idx * kQ + i];
    fr[j] = v;
  }
  const float fo = act && own ? Store<T>::ld(state + i * qs + cell.slot, inv_s) : 0.f;
  // the seven velocities
  float uu[7][3];
#pragma unroll
  for (int j = 0; j < 7; ++j) {
    const FdURead& r = cell.u[j];
    if (r.code == kFdZero) {
      uu[j][0] = uu[j][1] = uu[j][2] = 0.f;
    } else if (r.code == kFdFluid) {
      const float dh = warp_sum(fu[j]);
      const float k = 1.f / (1.f + dh);
#pragma unroll
      for (int a = 0; a < 3; ++a) uu[j][a] = warp_sum(ci[a] * fu[j]) * k;
    } else {
      prescribed(cells, static_cast<int>(r.idx), t, uu[j]);
    }
#pragma unroll
    for (int a = 0; a < 3; ++a)
      if (r.flip >> a & 1) uu[j][a] = -uu[j][a];
  }
  // velocityBMRho of values v held one population per lane
  auto bm = [&](float v, int d, int o, const float u[3]) {
    const float out = warp_sum(ci[d] == o ? v : 0.f), wall = warp_sum(ci[d] == 0 ? v : 0.f);
    return (2.f * out + wall + 1.f) / (1.f + o * u[d]);
  };
  float rr[6];
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    rr[j] = 0.f;
    if (j >= nr) continue;
    const FdRRead& r = cell.r[j];
    if (r.code == kFdRhoConst) {
      rr[j] = r.val;
    } else if (r.code == kFdRhoSumPre || r.code == kFdRhoSumNew) {
      // a kBulk cell's stored density under ConstRhoBGK carries the 1 -
      // average_rho its level's last collide added, if that collide came
      // after the level's stream (urow = 1 marks a kBulk cell)
      const float shift = (r.code == kFdRhoSumPre && r.urow == 1 && cr_shift) ? *cr_shift : 0.f;
      rr[j] = 1.f + warp_sum(fr[j]) - shift;
    } else {
      float u[3];
      prescribed(cells, r.urow, t, u);
      rr[j] = bm(fr[j], r.d, r.o, u);
    }
  }
  float du[3][3];
  float rho;
  if (cell.role == 1) {
    const int d = cell.d, o = cell.o;
    rho = cell.kind == kPressureDirichlet ? cell.rho_target : bm(fo, d, o, uu[0]);
    normal_grad(uu[0], uu[1], uu[2], o, du[d]);
    const int t0 = (d + 1) % 3 < (d + 2) % 3 ? (d + 1) % 3 : (d + 2) % 3;
    const int t1 = 3 - d - t0;
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      du[t0][b] = (uu[3][b] - uu[4][b]) * 0.5f;
      du[t1][b] = (uu[5][b] - uu[6][b]) * 0.5f;
    }
  } else if (cell.role == 2) {
    const int p = cell.ax[0], d1 = cell.ax[1], d2 = cell.ax[2];
#pragma unroll
    for (int b = 0; b < 3; ++b) du[p][b] = (uu[1][b] - uu[2][b]) * 0.5f;
    normal_grad(uu[0], uu[3], uu[4], cell.nrm[0], du[d1]);
    normal_grad(uu[0], uu[5], uu[6], cell.nrm[1], du[d2]);
    rho = 2.f / 3.f * (rr[0] + rr[1]) - 1.f / 6.f * (rr[2] + rr[3]);
  } else {
#pragma unroll
    for (int a = 0; a < 3; ++a) normal_grad(uu[0], uu[1 + 2 * a], uu[2 + 2 * a], cell.nrm[a], du[a]);
    rho = 4.f / 9.f * (rr[0] + rr[1] + rr[2]) - 1.f / 9.f * (rr[3] + rr[4] + rr[5]);
  }
  if (!act) return;
  const float s = -rho / 3.f / omega;
  const float pi[6] = {2.f * du[0][0] * s, (du[0][1] + du[1][0]) * s, (du[0][2] + du[2][0]) * s,
                       2.f * du[1][1] * s, (du[1][2] + du[2][1]) * s, 2.f * du[2][2] * s};
  const float* u = uu[0];
  const float usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
  const float c3[3] = {static_cast<float>(ci[0]), static_cast<float>(ci[1]), static_cast<float>(ci[2])};
  // f_neq from the symmetric stress (lbm.h:248-270): sum over a <= b of
  // (c_a c_b - delta_ab / 3) (x2 off the diagonal) Pi_ab, times w 9 / 2
  float q = 0.f;
  int m = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b, ++m) {
      float qq = c3[a] * c3[b] - (a == b ? 1.f / 3.f : 0.f);
      if (a != b) qq *= 2.f;
      q += qq * pi[m];
    }
  const float wi = w_rt(ci);
  const float cu = c3[0] * u[0] + c3[1] * u[1] + c3[2] * u[2];
  const float feq = rho * wi * (1.f + 3.f * cu + 4.5f * cu * cu - 1.5f * usq) - wi;
  fnew[static_cast<long long>(row) * kQ + i] = feq + q * wi * 4.5f;
}

// The collide of the boundary cells into the state buffer, at the start of
// their level's step: velocity cells f (1 - omega) + omega feq(rho,
// u_presc(t)), rho = velocityBMRho on plane cells and 1 + sum f on edges and
// corners; bounce-back cells the full-way swap of their streamed state (kept
// in their row); pressure cells unchanged.  Source: the rows (the last
// pass's, or the initial state's), or the state itself when fnew is null.
template <typename T>
__global__ void __launch_bounds__(kFdThreads)
k_fd_collide(T* state, long long qs, float scale, float inv_s, const FdCell* cells, int n, float* fnew,
             const double* time, double time_shift, float omega, double* cr_part) {
  const int row = blockIdx.x * kFdThreads + threadIdx.x;
  double stat = 0.0;  // ConstRhoBGK statistics: the velocity cell's collide density
  if (row < n) {
  const FdCell& cell = cells[row];
  float f[kQ];
  if (cell.role == 0) {
    // a bounce-back cell (the dispatcher's kBounceBack arm, bc_dispatcher.h:
    // 55-67): its streamed populations are its row (the state after the
    // step), then the full-way swap f_i <- f_opp(i)
    load_pops(state, qs, cell.slot, inv_s, f);
    float g[kQ];
#pragma unroll
    for (int i = 0; i < kQ; ++i) {
      if (fnew) fnew[static_cast<long long>(row) * kQ + i] = f[i];
      g[i] = f[i];
    }
#pragma unroll
    for (int i = 0; i < kQ; ++i) f[i] = g[opp(i)];
  } else if (fnew) {
#pragma unroll
    for (int i = 0; i < kQ; ++i) f[i] = fnew[static_cast<long long>(row) * kQ + i];
  } else {
    load_pops(state, qs, cell.slot, inv_s, f);
  }
  if (cell.kind == kVelocityDirichlet) {
    float u[3];
    prescribed(cells, row, static_cast<float>(*time + time_shift), u);
    const float rho = cell.role == 1 ? bm_rho(f, cell.d, cell.o, u) : 1.f + sum_pops(f);
    stat = rho;
    const float usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
#pragma unroll
    for (int i = 0; i < kQ; ++i) f[i] = f[i] * (1.f - omega) + omega * feq_i(i, rho, u, usq);
  }
#pragma unroll
  for (int i = 0; i < kQ; ++i) Store<T>::st(state + i * qs + cell.slot, f[i], scale);
  }
  if (cr_part) {  // this CTA's sum, in a fixed order
    for (int o = 16; o > 0; o >>= 1) stat += __shfl_down_sync(0xffffffffu, stat, o);
    __shared__ double ws[kFdThreads / 32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = stat;
    __syncthreads();
    if (threadIdx.x == 0) {
      double sum = 0.0;
      for (int w = 0; w < kFdThreads / 32; ++w) sum += ws[w];
      cr_part[blockIdx.x] = sum;
    }
  }
}

__global__ void k_fd_tick(double* time) { *time += 1.0; }

// The pass's rewritten rows into the state (velocity and pressure cells; the
// bounce-back cells keep their streamed populations until their collide).
template <typename T>
__global__ void __launch_bounds__(kFdThreads)
k_fd_store(T* state, long long qs, float scale, const FdCell* cells, int n, const float* fnew, double* tick) {
  const int row = blockIdx.x * kFdThreads + threadIdx.x;
  // the boundary clock's tick, where this is the step's last pass (no kernel
  // of the pass reads the clock after the reconstruction)
  if (tick && row == 0) *tick += 1.0;
  if (row >= n || cells[row].role == 0) return;
#pragma unroll
  for (int i = 0; i < kQ; ++i)
    Store<T>::st(state + i * qs + cells[row].slot, fnew[static_cast<long long>(row) * kQ + i], scale);
}

// The Dirichlet cells' populations before their collide (the initial state)
// into their rows: what the reference holds for them after a step.
template <typename T>
__global__ void __launch_bounds__(kFdThreads)
k_fd_rows_from_state(const T* state, long long qs, float inv_s, const FdCell* cells, int n, float* fnew) {
  const int row = blockIdx.x * kFdThreads + threadIdx.x;
  if (row >= n) return;
#pragma unroll
  for (int i = 0; i < kQ; ++i)
    fnew[static_cast<long long>(row) * kQ + i] = Store<T>::ld(state + i * qs + cells[row].slot, inv_s);
}

// rho and u of the Dirichlet cells from their rows (the populations after the
// pass, before the next collide -- the reference's state after the step),
// over the fields the gather wrote; the bounce-back cells' fields are the
// gathered ones (their streamed state).
__global__ void __launch_bounds__(kFdThreads)
k_fd_fields(const FdCell* cells, int n, const float* fnew, double* rho, double* u) {
  const int row = blockIdx.x * kFdThreads + threadIdx.x;
  if (row >= n || cells[row].role == 0) return;
  double dr = 0, jx = 0, jy = 0, jz = 0;
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    const double v = fnew[static_cast<long long>(row) * kQ + i];
    dr += v; jx += cx(i) * v; jy += cy(i) * v; jz += cz(i) * v;
  }
  const double r = 1.0 + dr;
  const long long s = cells[row].slot;
  rho[s] = r;
  u[3 * s] = jx / r;
  u[3 * s + 1] = jy / r;
  u[3 * s + 2] = jz / r;
}

inline unsigned fd_grid(int n) { return static_cast<unsigned>((n + kFdThreads - 1) / kFdThreads); }

}  // namespace

unsigned fd_collide_parts(int n) { return fd_grid(n); }

namespace {

}  // namespace

template <typename T>
cudaError_t launch_fd_reconstruct(const void* state, long long qs, float inv_s, const FdCell* cells, const int* list,
                                  int n, float* fnew, const double* time, float omega, const float* cr_shift,
                                  cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const unsigned grid = static_cast<unsigned>((static_cast<long long>(n) * 32 + kFdThreads - 1) / kFdThreads);
  k_fd_reconstruct<T><<<grid, kFdThreads, 0, s>>>(static_cast<const T*>(state), qs, inv_s, cells, list, n, fnew,
                                                  time, omega, cr_shift);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_fd_collide(void* state, long long qs, float scale, float inv_s, const FdCell* cells, int n,
                              float* fnew, const double* time, double time_shift, float omega, double* cr_part,
                              cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_fd_collide<T><<<fd_grid(n), kFdThreads, 0, s>>>(static_cast<T*>(state), qs, scale, inv_s, cells, n, fnew, time,
                                                     time_shift, omega, cr_part);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_fd_rows_from_state(const void* state, long long qs, float inv_s, const FdCell* cells, int n,
                                     float* fnew, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_fd_rows_from_state<T><<<fd_grid(n), kFdThreads, 0, s>>>(static_cast<const T*>(state), qs, inv_s, cells, n, fnew);
  return cudaGetLastError();
}

cudaError_t launch_fd_fields(const FdCell* cells, int n, const float* fnew, double* rho, double* u, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_fd_fields<<<fd_grid(n), kFdThreads, 0, s>>>(cells, n, fnew, rho, u);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_fd_store(void* state, long long qs, float scale, const FdCell* cells, int n, const float* fnew,
                            double* tick, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_fd_store<T><<<fd_grid(n), kFdThreads, 0, s>>>(static_cast<T*>(state), qs, scale, cells, n, fnew, tick);
  return cudaGetLastError();
}
template cudaError_t launch_fd_store<float>(void*, long long, float, const FdCell*, int, const float*, double*,
                                           cudaStream_t);
template cudaError_t launch_fd_store<__half>(void*, long long, float, const FdCell*, int, const float*, double*,
                                            cudaStream_t);

cudaError_t launch_fd_tick(double* time, cudaStream_t s) {
  k_fd_tick<<<1, 1, 0, s>>>(time);
  return cudaGetLastError();
}

#define OCTLB_FD_INST(T)                                                                                      \
  template cudaError_t launch_fd_reconstruct<T>(const void*, long long, float, const FdCell*, const int*, int, \
                                                float*, const double*, float, const float*, cudaStream_t);  \
  template cudaError_t launch_fd_collide<T>(void*, long long, float, float, const FdCell*, int, float*,        \
                                            const double*, double, float, double*, cudaStream_t);
template cudaError_t launch_fd_rows_from_state<float>(const void*, long long, float, const FdCell*, int, float*,
                                                     cudaStream_t);
template cudaError_t launch_fd_rows_from_state<__half>(const void*, long long, float, const FdCell*, int, float*,
                                                      cudaStream_t);
OCTLB_FD_INST(float)
OCTLB_FD_INST(__half)

}  // namespace octlb_gpu
