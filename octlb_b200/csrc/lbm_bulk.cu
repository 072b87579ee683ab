// Pipelined fused steps for one periodic block fed by bulk async copies:
// k_step_bulk (one cell per thread, FP32 or FP16, an option),
// k_step_rows_h (four FP16 cells per thread: the FP16 default, and the AA
// order's local step) and k_step_aa_rows<T> (the AA order's pull step,
// drained by bulk stores too).
//
// A persistent CTA of n threads walks z-rows (x, y).  For each row it needs
// the 19 source rows (x - cx_i, y - cy_i) of the 19 population planes; an
// elected thread streams them into shared memory with 1D bulk async copies
// (cp.async.bulk, TMA engine, 16-byte aligned rows) completing on a per-stage
// mbarrier, STAGES rows ahead of the compute.  Thread z then reads
// f_i = S[i][(z - cz_i) mod n], collides in registers (BGK) and stores the
// row of post-collision populations with coalesced stores.  Every source
// element is read exactly once per step, so the shared-memory staging buys
// latency hiding (many KB in flight per SM with few threads), not reuse.
//
// Every mbarrier wait is bounded (StepArgs::wait_ns of %globaltimer, 1 s by
// default): on expiry the CTA agrees via __syncthreads_and, records
// kErrBulkTimeout in *err, drains the copies it has issued and not yet seen
// land (again bounded; kErrBulkDrainTimeout if that expires too) and returns;
// the host reports OCTLB_ETIMEOUT (OCTLB_ECUDA after a failed drain).
// StepArgs::stall_first_row makes CTA 0 skip issuing its first row, so its
// first wait runs out: the test of this path (no fault, no hang).
#include "lbm_device.cuh"

namespace octlb_gpu {
namespace {

constexpr int kStages = 4;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the phase with the given parity.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, unsigned long long limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (global_ns() - t0 > limit_ns) return false;
  }
  return true;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Bulk async stores (shared -> global) of this thread's bulk group, and the
// proxy fence that orders a CTA's generic shared-memory writes before them.
__device__ __forceinline__ void bulk_s2g(void* dst, const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_u32(src)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// this thread's committed stores have finished reading shared memory
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// ... and are complete in global memory
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_smem_to_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

template <typename T>
__device__ __forceinline__ void issue_row(const StepArgs& a, const T* src, T* stage, uint64_t* bar,
                                          uint32_t row) {
  const uint32_t n = a.n;
  const uint32_t x = a.div_n.div(row), y = row - x * n;
  const uint32_t bytes = n * sizeof(T);
  mbar_expect_tx(bar, bytes * kQ);
#pragma unroll
  for (int i = 0; i < kQ; ++i) {
    const uint32_t xs = cx(i) == 1 ? (x == 0 ? n - 1 : x - 1) : (cx(i) == -1 ? (x == n - 1 ? 0 : x + 1) : x);
    const uint32_t ys = cy(i) == 1 ? (y == 0 ? n - 1 : y - 1) : (cy(i) == -1 ? (y == n - 1 ? 0 : y + 1) : y);
    const T* g = src + i * a.qs + (static_cast<long long>(xs) * n + ys) * n;
    bulk_g2s(stage + i * n, g, bytes, bar);
  }
}

template <typename T>
__global__ void __launch_bounds__(1024) k_step_bulk(const StepArgs a) {
  // Dynamic shared memory only: kStages stage buffers of 19 rows, then the
  // kStages mbarriers (stage bytes are a multiple of 16).
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const uint32_t n = a.n;
  T* stages = reinterpret_cast<T*>(smem_raw);
  const uint32_t stage_elems = kQ * n;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + static_cast<size_t>(kStages) * stage_elems * sizeof(T));
  const T* src = static_cast<const T*>(a.src);
  T* dst = static_cast<T*>(a.dst);
  const uint32_t rows = n * n;
  const uint32_t z = threadIdx.x;
  const uint32_t zm = z == 0 ? n - 1 : z - 1, zp = z == n - 1 ? 0 : z + 1;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) mbar_init(&bars[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  // rows of this CTA: blockIdx.x + k * gridDim.x, k = 0..my_rows-1
  const uint32_t my_rows = blockIdx.x < rows ? (rows - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  // Thread 0's record of which rows it issued (rows k .. k + kStages - 2 are
  // in flight while row k is consumed): bit j % kStages.
  uint32_t issued = 0;
  if (threadIdx.x == 0) {
    for (uint32_t k = 0; k < my_rows && k < kStages - 1; ++k) {
      if (k == 0 && a.stall_first_row && blockIdx.x == 0) continue;
      issue_row<T>(a, src, stages + k * stage_elems, &bars[k], blockIdx.x + k * gridDim.x);
      issued |= 1u << k;
    }
  }
  for (uint32_t k = 0; k < my_rows; ++k) {
    const uint32_t s = k % kStages;
    bool ok = mbar_wait_bounded(&bars[s], (k / kStages) & 1, a.wait_ns);
    ok = __syncthreads_and(ok) != 0;
    if (!ok) {
      if (threadIdx.x == 0) {
        int code = kErrBulkTimeout;
        // drain the copies this CTA issued and has not seen land (bounded)
        for (uint32_t j = k; j < my_rows && j < k + kStages - 1; ++j)
          if ((issued >> (j % kStages)) & 1u)
            if (!mbar_wait_bounded(&bars[j % kStages], (j / kStages) & 1, a.wait_ns)) code = kErrBulkDrainTimeout;
        atomicMax(a.err, code);
      }
      return;
    }
    if (threadIdx.x == 0) issued &= ~(1u << s);
    // every thread has finished reading stage (k-1) % kStages: refill it
    if (threadIdx.x == 0 && k + kStages - 1 < my_rows) {
      const uint32_t kk = k + kStages - 1;
      issue_row<T>(a, src, stages + (kk % kStages) * stage_elems, &bars[kk % kStages],
                   blockIdx.x + kk * gridDim.x);
      issued |= 1u << (kk % kStages);
    }
    const T* S = stages + s * stage_elems;
    float f[kQ];
#pragma unroll
    for (int i = 0; i < kQ; ++i) {
      const uint32_t zs = cz(i) == 1 ? zm : (cz(i) == -1 ? zp : z);
      f[i] = Store<T>::ld(S + i * n + zs, 1.0f);
    }
    bgk<kBgkCorrect<T>>(f, a.omega, a.scale, a.inv_scale);  // storage units h = s (f - w)
    const uint32_t row = blockIdx.x + k * gridDim.x;
    T* o = dst + static_cast<long long>(row) * n + z;
#pragma unroll
    for (int i = 0; i < kQ; ++i) Store<T>::st(o + i * a.qs, f[i], 1.0f);
  }
}

// FP16-shifted step of one periodic all-kBulk block, four z cells per
// thread, fed by bulk async copies.  A CTA of THREADS threads computes
// stages of 4 THREADS consecutive cells: R = 4 THREADS / n whole z rows
// (x, y0 .. y0 + R - 1) of one x plane.  For each population a lane of warp
// 0 copies the R source rows (x - cx_i, y0 - cy_i ..), one contiguous run or
// two at the y wrap, into the stage's shared-memory buffer, STAGES - 1
// stages ahead of the compute, so the loads stay in flight through the
// arithmetic without the occupancy the register-heavy four-cell collide
// lacks.  Per cell the values read, the arithmetic and the 8-byte stores
// are k_step_quad_h's, so the results are bitwise equal.  Waits are bounded
// as in k_step_bulk.  n a power of two dividing 4 THREADS, n >= 8; the
// population stride qs a multiple of 8 (16-byte aligned rows).
// Direction components as bit masks, for a population index known only at
// run time (one lane per population).
__host__ __device__ constexpr uint32_t dir_mask(int axis, int sign) {
  uint32_t m = 0;
  for (int i = 0; i < kQ; ++i)
    if ((axis == 0 ? cx(i) : axis == 1 ? cy(i) : cz(i)) == sign) m |= 1u << i;
  return m;
}
constexpr uint32_t kXPos = dir_mask(0, 1), kXNeg = dir_mask(0, -1);
constexpr uint32_t kYPos = dir_mask(1, 1), kYNeg = dir_mask(1, -1);
__device__ __forceinline__ int dir_rt(int axis, int i) {
  const uint32_t pos = axis == 0 ? kXPos : kYPos, neg = axis == 0 ? kXNeg : kYNeg;
  return static_cast<int>((pos >> i) & 1u) - static_cast<int>((neg >> i) & 1u);
}

// The R source rows of population i of a stage -- rows (x - cx_i, y0 - cy_i
// .. y0 - cy_i + R - 1) of plane i, one contiguous run or two at the y wrap --
// as (global, shared, bytes) runs handed to f.
// Unshifted (the AA order's local step): rows (x, y0 .. y0 + R - 1) of
// plane i, one run.
template <typename E, typename F>
__device__ __forceinline__ void pop_runs_h(const StepArgs& a, E* pops, E* stage, uint32_t row0, uint32_t R,
                                           uint32_t cells, int i, F&& f, bool shifted = true) {
  const uint32_t n = a.n;
  const int ci = shifted ? dir_rt(0, i) : 0, cj = shifted ? dir_rt(1, i) : 0;
  const uint32_t x = a.div_n.div(row0), y0 = row0 - x * n;
  const uint32_t xs = ci == 1 ? (x == 0 ? static_cast<uint32_t>(a.wrap_lo) : x - 1)
                              : (ci == -1 ? (x == n - 1 ? static_cast<uint32_t>(a.wrap_hi) : x + 1) : x);
  E* plane = pops + i * a.qs + static_cast<long long>(xs) * n * n;
  E* d = stage + i * cells;
  const int ys = static_cast<int>(y0) - cj;
  const uint32_t rb = n * sizeof(E);
  if (ys >= 0 && ys + static_cast<int>(R) <= static_cast<int>(n)) {
    f(plane + static_cast<long long>(ys) * n, d, R * rb);
  } else if (ys < 0) {  // rows n - 1, 0 .. R - 2
    f(plane + static_cast<long long>(n - 1) * n, d, rb);
    if (R > 1) f(plane, d + n, (R - 1) * rb);
  } else {              // rows y0 + 1 .. n - 1, 0
    if (R > 1) f(plane + static_cast<long long>(ys) * n, d, (R - 1) * rb);
    f(plane, d + (R - 1) * n, rb);
  }
}
template <typename E>
__device__ __forceinline__ void issue_pop_h(const StepArgs& a, const E* src, E* stage, uint64_t* bar, uint32_t row0,
                                            uint32_t R, uint32_t cells, int i, bool shifted) {
  pop_runs_h(
      a, const_cast<E*>(src), stage, row0, R, cells, i,
      [&](E* g, E* sm, uint32_t bytes) { bulk_g2s(sm, g, bytes, bar); }, shifted);
}

// Warp 0 requests a stage: lane 0 arms the barrier with the stage's bytes,
// then lanes 0..18 copy one population each.  (Measured on the 256^3 box:
// one lane issuing all 19 made the step 0.2385 ms instead of 0.2077.)
template <typename E>
__device__ __forceinline__ void issue_stage_h(const StepArgs& a, const E* src, E* stage, uint64_t* bar, uint32_t row0,
                                              uint32_t R, uint32_t cells, uint32_t lane, bool shifted = true) {
  if (lane == 0) mbar_expect_tx(bar, static_cast<uint32_t>(kQ * cells * sizeof(E)));
  __syncwarp();
  if (lane < static_cast<uint32_t>(kQ))
    issue_pop_h(a, src, stage, bar, row0, R, cells, static_cast<int>(lane), shifted);
}

// A thread's CPT consecutive FP16 cells: four (8-byte accesses) or two
// (4-byte accesses), converted to and from float as ld4h / st4h do.
template <int CPT> struct HalfCells;
template <> struct HalfCells<4> {
  __device__ static void ld(const __half* p, float (&v)[4]) { ld4h(p, v[0], v[1], v[2], v[3]); }
  __device__ static void st(__half* p, const float (&v)[4]) { st4h(p, v[0], v[1], v[2], v[3]); }
};
template <> struct HalfCells<2> {
  __device__ static void ld(const __half* p, float (&v)[2]) {
    const float2 u = __half22float2(*reinterpret_cast<const __half2*>(p));
    v[0] = u.x;
    v[1] = u.y;
  }
  __device__ static void st(__half* p, const float (&v)[2]) {
    *reinterpret_cast<__half2*>(p) = __floats2half2_rn(v[0], v[1]);
  }
};

// LOCAL: the AA order's step from the reversed layout -- each cell's own
// slots, population i from plane opp(i), written to plane i; no shifts, the
// same values and arithmetic as k_step_aa_local_h (in place: every stage
// reads and writes only its own cells' slots).  CPT: cells per thread.
template <int THREADS, int STAGES, int MINB, bool LOCAL, int CPT>
__global__ void __launch_bounds__(THREADS, MINB) k_step_rows_h(const StepArgs a) {
  using V = HalfCells<CPT>;
  constexpr uint32_t kCells = CPT * THREADS;
  constexpr uint32_t kStageElems = kQ * kCells;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __half* stages = reinterpret_cast<__half*>(smem_raw);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + static_cast<size_t>(STAGES) * kStageElems * sizeof(__half));
  const __half* src = static_cast<const __half*>(a.src);
  __half* dst = static_cast<__half*>(a.dst);
  const uint32_t n = a.n;
  const uint32_t R = kCells / n;
  const uint32_t nst = static_cast<uint32_t>(a.ncore / kCells);
  // this thread's cells within a stage: row r, z .. z + CPT - 1
  const uint32_t c = CPT * threadIdx.x;
  const uint32_t lg = static_cast<uint32_t>(__ffs(static_cast<int>(n)) - 1);
  const uint32_t r = c >> lg, z = c & (n - 1);
  const uint32_t zm1 = z == 0 ? n - 1 : z - 1, zpc = z + CPT == n ? 0 : z + CPT;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(&bars[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  pdl_wait();

  const uint32_t mine = blockIdx.x < nst ? (nst - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const uint32_t lane = threadIdx.x;  // < 32: warp 0, the requesting warp
  uint32_t issued = 0;                // warp 0: stages in flight, bit k % STAGES
  if (threadIdx.x < 32) {
    for (uint32_t k = 0; k < mine && k < STAGES - 1; ++k) {
      if (k == 0 && a.stall_first_row && blockIdx.x == 0) continue;
      issue_stage_h(a, src, stages + k * kStageElems, &bars[k], (blockIdx.x + k * gridDim.x) * R, R, kCells, lane,
                    !LOCAL);
      issued |= 1u << k;
    }
  }
  for (uint32_t k = 0; k < mine; ++k) {
    const uint32_t s = k % STAGES;
    bool ok = mbar_wait_bounded(&bars[s], (k / STAGES) & 1, a.wait_ns);
    ok = __syncthreads_and(ok) != 0;
    if (!ok) {
      if (threadIdx.x == 0) {
        int code = kErrBulkTimeout;
        for (uint32_t j = k; j < mine && j < k + STAGES - 1; ++j)
          if ((issued >> (j % STAGES)) & 1u)
            if (!mbar_wait_bounded(&bars[j % STAGES], (j / STAGES) & 1, a.wait_ns)) code = kErrBulkDrainTimeout;
        atomicMax(a.err, code);
      }
      return;
    }
    if (threadIdx.x < 32) {
      issued &= ~(1u << s);
      // every thread has finished reading stage (k - 1) % STAGES: refill it
      if (k + STAGES - 1 < mine) {
        const uint32_t kk = k + STAGES - 1;
        issue_stage_h(a, src, stages + (kk % STAGES) * kStageElems, &bars[kk % STAGES],
                      (blockIdx.x + kk * gridDim.x) * R, R, kCells, lane, !LOCAL);
        issued |= 1u << (kk % STAGES);
      }
    }
    const __half* S = stages + s * kStageElems + r * n;
    float f[CPT][kQ];
#pragma unroll
    for (int i = 0; i < kQ; ++i) {
      float v[CPT];
      if constexpr (LOCAL) {
        V::ld(S + opp(i) * kCells + z, v);
#pragma unroll
        for (int j = 0; j < CPT; ++j) f[j][i] = v[j];
        continue;
      }
      const __half* p = S + i * kCells;
      V::ld(p + z, v);
#pragma unroll
      for (int j = 0; j < CPT; ++j) {
        if (cz(i) == 0) f[j][i] = v[j];
        else if (cz(i) == 1) f[j][i] = j == 0 ? __half2float(p[zm1]) : v[j - 1];  // cells pull z-1 ..
        else f[j][i] = j == CPT - 1 ? __half2float(p[zpc]) : v[j + 1];             // cells pull z+1 ..
      }
    }
#pragma unroll
    for (int j = 0; j < CPT; ++j) bgk<false>(f[j], a.omega, a.scale, a.inv_scale);
    __half* o = dst + static_cast<long long>(blockIdx.x + k * gridDim.x) * kCells + c;
#pragma unroll
    for (int i = 0; i < kQ; ++i) {
      float v[CPT];
#pragma unroll
      for (int j = 0; j < CPT; ++j) v[j] = f[j][i];
      V::st(o + i * a.qs, v);
    }
  }
}

// Vector access of a thread's CPT consecutive cells (8 bytes: four halves
// or two floats), as k_step_aa_pull_h and k_step_pair read them.
template <typename T> struct Cells8;
template <> struct Cells8<__half> {
  static constexpr int kCpt = 4;
  __device__ static void ld(const __half* p, float (&v)[4]) { ld4h(p, v[0], v[1], v[2], v[3]); }
  __device__ static float ld1(const __half* p) { return __half2float(*p); }
  __device__ static void st1(__half* p, float v) { *p = __float2half_rn(v); }
  __device__ static void st(__half* p, const float (&v)[4]) { st4h(p, v[0], v[1], v[2], v[3]); }
};
template <> struct Cells8<float> {
  static constexpr int kCpt = 2;
  __device__ static void ld(const float* p, float (&v)[2]) {
    const float2 u = *reinterpret_cast<const float2*>(p);
    v[0] = u.x;
    v[1] = u.y;
  }
  __device__ static float ld1(const float* p) { return *p; }
  __device__ static void st1(float* p, float v) { *p = v; }
  __device__ static void st(float* p, const float (&v)[2]) { *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]); }
};

// The AA order's pull step (natural -> reversed layout), staged the same
// way: the 19 source rows of a stage come in by bulk copies; each cell
// collides its pulled values and writes g_opp(k) back into the
// shared-memory slot it read for direction k; the stage's rows then go back
// by bulk stores to the global rows they came from.  Every slot belongs to
// one cell (a thread's 8-byte read may include a neighbour's slot, whose
// value it does not use), and a population's source rows of different
// stages are disjoint, so the in-place update needs no ordering between
// threads before the write-back or between CTAs.  Per cell the values and
// the arithmetic are the unstaged pull steps' (k_step_aa_pull_h,
// k_step_aa_pull<float>): bitwise equal.  A buffer is refilled once the lane
// that stored a population's rows from it has seen its stores read out.
// CPT = 4 FP16 or 2 FP32 cells per thread.
template <typename T, int THREADS, int STAGES, int MINB>
__global__ void __launch_bounds__(THREADS, MINB) k_step_aa_rows(const StepArgs a) {
  using V = Cells8<T>;
  constexpr int CPT = V::kCpt;
  constexpr uint32_t kCells = CPT * THREADS;
  constexpr uint32_t kStageElems = kQ * kCells;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T* stages = reinterpret_cast<T*>(smem_raw);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + static_cast<size_t>(STAGES) * kStageElems * sizeof(T));
  T* pops = static_cast<T*>(a.dst);  // == a.src
  const uint32_t n = a.n;
  const uint32_t R = kCells / n;
  const uint32_t nst = static_cast<uint32_t>(a.ncore / kCells);
  const uint32_t c = CPT * threadIdx.x;
  const uint32_t lg = static_cast<uint32_t>(__ffs(static_cast<int>(n)) - 1);
  const uint32_t r = c >> lg, z = c & (n - 1);
  const uint32_t zm1 = z == 0 ? n - 1 : z - 1, zpc = z + CPT == n ? 0 : z + CPT;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(&bars[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  pdl_wait();

  const uint32_t mine = blockIdx.x < nst ? (nst - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const uint32_t lane = threadIdx.x;  // < 32: warp 0, the copying warp
  uint32_t issued = 0;                // warp 0: loads in flight, bit k % STAGES
  if (threadIdx.x < 32) {
    for (uint32_t k = 0; k < mine && k < STAGES - 1; ++k) {
      if (k == 0 && a.stall_first_row && blockIdx.x == 0) continue;
      issue_stage_h(a, pops, stages + k * kStageElems, &bars[k], (blockIdx.x + k * gridDim.x) * R, R, kCells, lane);
      issued |= 1u << k;
    }
  }
  for (uint32_t k = 0; k < mine; ++k) {
    const uint32_t s = k % STAGES;
    if (threadIdx.x < 32 && k + STAGES - 1 < mine) {
      // the buffer of stage k - 1: every thread wrote it before that stage's
      // stores were issued; refill it once they have read it out
      const uint32_t kk = k + STAGES - 1, b = kk % STAGES;
      bulk_wait_read_all();
      issue_stage_h(a, pops, stages + b * kStageElems, &bars[b], (blockIdx.x + kk * gridDim.x) * R, R, kCells, lane);
      issued |= 1u << b;
    }
    bool ok = mbar_wait_bounded(&bars[s], (k / STAGES) & 1, a.wait_ns);
    ok = __syncthreads_and(ok) != 0;
    if (!ok) {
      if (threadIdx.x < 32) bulk_wait_all();
      if (threadIdx.x == 0) {
        int code = kErrBulkTimeout;
        for (uint32_t j = k; j < mine && j < k + STAGES; ++j)
          if ((issued >> (j % STAGES)) & 1u)
            if (!mbar_wait_bounded(&bars[j % STAGES], (j / STAGES) & 1, a.wait_ns)) code = kErrBulkDrainTimeout;
        atomicMax(a.err, code);
      }
      return;
    }
    if (threadIdx.x < 32) issued &= ~(1u << s);
    T* S = stages + s * kStageElems + r * n;
    float f[CPT][kQ];
#pragma unroll
    for (int i = 0; i < kQ; ++i) {
      const T* p = S + i * kCells;
      float v[CPT];
      V::ld(p + z, v);
#pragma unroll
      for (int j = 0; j < CPT; ++j) {
        if (cz(i) == 0) f[j][i] = v[j];
        else if (cz(i) == 1) f[j][i] = j == 0 ? V::ld1(p + zm1) : v[j - 1];  // cells pull z-1 ..
        else f[j][i] = j == CPT - 1 ? V::ld1(p + zpc) : v[j + 1];             // cells pull z+1 ..
      }
    }
#pragma unroll
    for (int j = 0; j < CPT; ++j) bgk<kBgkCorrect<T>>(f[j], a.omega, a.scale, a.inv_scale);
#pragma unroll
    for (int k2 = 0; k2 < kQ; ++k2) {
      T* p = S + k2 * kCells;
      const int o = opp(k2);
      if (cz(k2) == 0) {  // slots z .. z + CPT - 1
        float v[CPT];
#pragma unroll
        for (int j = 0; j < CPT; ++j) v[j] = f[j][o];
        V::st(p + z, v);
      } else if (cz(k2) == 1) {  // slots z - 1, z .. z + CPT - 2
        V::st1(p + zm1, f[0][o]);
        if constexpr (CPT == 4) {
          *reinterpret_cast<__half2*>(p + z) = __floats2half2_rn(f[1][o], f[2][o]);
          V::st1(p + z + 2, f[3][o]);
        } else {
          V::st1(p + z, f[1][o]);
        }
      } else {  // slots z + 1 .. z + CPT - 1, z + CPT
        if constexpr (CPT == 4) {
          V::st1(p + z + 1, f[0][o]);
          *reinterpret_cast<__half2*>(p + z + 2) = __floats2half2_rn(f[1][o], f[2][o]);
        } else {
          V::st1(p + z + 1, f[0][o]);
        }
        V::st1(p + zpc, f[CPT - 1][o]);
      }
    }
    fence_smem_to_async();
    __syncthreads();
    if (threadIdx.x < static_cast<uint32_t>(kQ)) {
      pop_runs_h(a, pops, stages + s * kStageElems, (blockIdx.x + k * gridDim.x) * R, R, kCells,
                 static_cast<int>(lane), [](T* g, T* sm, uint32_t bytes) { bulk_s2g(g, sm, bytes); });
      bulk_commit();
    }
  }
  if (threadIdx.x < 32) bulk_wait_all();
}

}  // namespace

// Eligible: one periodic all-kBulk block, n threads per CTA, rows of 16-byte
// multiples.
bool bulk_step_eligible(int n, int elem_bytes) {
  return n >= 32 && n <= 1024 && (n % 32) == 0 && (n * elem_bytes) % 16 == 0;
}
size_t bulk_step_smem(int n, int elem_bytes) {
  return static_cast<size_t>(kStages) * kQ * n * elem_bytes + kStages * sizeof(uint64_t);
}

// Raises the dynamic shared-memory limit for this instantiation and returns
// the resident CTAs per SM (0 when the kernel cannot run with n threads).
template <typename T>
int bulk_prepare(int n) {
  const size_t smem = bulk_step_smem(n, sizeof(T));
  if (cudaFuncSetAttribute(k_step_bulk<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(smem)) != cudaSuccess)
    return 0;
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_step_bulk<T>, n, smem) != cudaSuccess) return 0;
  return b;
}

template <typename T>
cudaError_t launch_step_bulk(const StepArgs& a, int grid, cudaStream_t s) {
  k_step_bulk<T><<<grid, a.n, bulk_step_smem(a.n, sizeof(T)), s>>>(a);
  return cudaGetLastError();
}

// The staged FP16 step's launch shapes: threads, stages, the CTAs per SM
// the register budget is set for, cells per thread.  Per step on the 256^3
// box, two boxes: 0 (256 x 2, four cells) 0.2077 / 0.2058 ms, 1 (128 x 2)
// 0.2070 / 0.2169, 2 (128 x 3) 0.2129 / 0.2306, 3 (64 x 2) 0.2130, 4 (64 x 3)
// 0.2521; k_step_quad_h 0.2210 / 0.2213.  5-7 take two cells per thread
// (79 registers, more warps): on a third box, where 0 took 0.2053 ms, 5
// (256 x 3) took 0.2265, 6 (256 x 2) 0.2475 and 7 (128 x 3) 0.2231.
namespace {
constexpr int kRowsVariants = 8;
constexpr int kRowsThreads[kRowsVariants] = {256, 128, 128, 64, 64, 256, 256, 128};
constexpr int kRowsStages[kRowsVariants] = {2, 2, 3, 2, 3, 3, 2, 3};
constexpr int kRowsCpt[kRowsVariants] = {4, 4, 4, 4, 4, 2, 2, 2};
constexpr int rows_threads(int v) { return kRowsThreads[v]; }
constexpr int rows_stages(int v) { return kRowsStages[v]; }
size_t rows_smem(int v) {
  return static_cast<size_t>(rows_stages(v)) * kQ * kRowsCpt[v] * rows_threads(v) * sizeof(__half) +
         rows_stages(v) * sizeof(uint64_t);
}
template <bool LOCAL, typename F>
auto with_rows_kernel_t(int v, F&& f) {
  switch (v) {
    case 1: return f(k_step_rows_h<128, 2, 4, LOCAL, 4>);
    case 2: return f(k_step_rows_h<128, 3, 3, LOCAL, 4>);
    case 3: return f(k_step_rows_h<64, 2, 8, LOCAL, 4>);
    case 4: return f(k_step_rows_h<64, 3, 7, LOCAL, 4>);
    case 5: return f(k_step_rows_h<256, 3, 3, LOCAL, 2>);
    case 6: return f(k_step_rows_h<256, 2, 3, LOCAL, 2>);
    case 7: return f(k_step_rows_h<128, 3, 6, LOCAL, 2>);
    default: return f(k_step_rows_h<256, 2, 2, LOCAL, 4>);
  }
}
template <typename F>
auto with_rows_kernel(int v, bool local, F&& f) {
  return local ? with_rows_kernel_t<true>(v, f) : with_rows_kernel_t<false>(v, f);
}
}  // namespace

long long rows_stage_cells(int variant) { return static_cast<long long>(kRowsCpt[variant]) * rows_threads(variant); }

bool rows_step_eligible(int n, long long ncore, long long qs, int variant) {
  if (variant < 0 || variant >= kRowsVariants) return false;
  const long long cells = rows_stage_cells(variant);
  return n >= 32 && (n & (n - 1)) == 0 && cells % n == 0 &&
         static_cast<long long>(n) * n >= cells && ncore % cells == 0 && qs % 8 == 0;
}

// Raises the shared-memory limit of the variant and returns its resident
// CTAs per SM (0: it cannot run).
int rows_prepare(int variant, bool local) {
  const size_t smem = rows_smem(variant);
  const int th = rows_threads(variant);
  return with_rows_kernel(variant, local, [&](void (*k)(StepArgs)) {
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) != cudaSuccess)
      return 0;
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k, th, smem) != cudaSuccess) return 0;
    return b;
  });
}

// The staged AA pull step's launch shapes: 0 = 128 threads x 2 stages, 1 =
// 256 x 2, 2 = 128 x 3 (stages of 8 bytes x threads per population, either
// precision).  AA steps (pull + local) on the 256^3 box: FP16 on two boxes
// 0.2240 / 0.2167 ms, 0.2314 / 0.2224, 0.2339 / 0.2288, with the unstaged
// pull (k_step_aa_pull_h) 0.2763 / 0.2677; FP32 0.3933, 0.4061, 0.4215, with
// the unstaged one-cell pull 0.4224 (AB step 0.3813).
namespace {
constexpr int kAaVariants = 3;
constexpr int kAaThreads[kAaVariants] = {128, 256, 128};
constexpr int kAaStages[kAaVariants] = {2, 2, 3};
size_t aa_rows_smem(int v) {
  return static_cast<size_t>(kAaStages[v]) * kQ * 8 * kAaThreads[v] + kAaStages[v] * sizeof(uint64_t);
}
template <typename T, typename F>
auto with_aa_rows_kernel(int v, F&& f) {
  switch (v) {
    case 1: return f(k_step_aa_rows<T, 256, 2, 2>);
    case 2: return f(k_step_aa_rows<T, 128, 3, 3>);
    default: return f(k_step_aa_rows<T, 128, 2, 4>);
  }
}
}  // namespace

long long aa_rows_stage_cells(int variant, int elem_bytes) { return 8LL / elem_bytes * kAaThreads[variant]; }
bool aa_rows_eligible(int n, long long ncore, long long qs, int elem_bytes, int variant) {
  if (variant < 0 || variant >= kAaVariants || (elem_bytes != 2 && elem_bytes != 4)) return false;
  const long long cells = aa_rows_stage_cells(variant, elem_bytes);
  return n >= 32 && (n & (n - 1)) == 0 && cells % n == 0 && static_cast<long long>(n) * n >= cells &&
         ncore % cells == 0 && (qs * elem_bytes) % 16 == 0;
}
template <typename T>
int aa_rows_prepare(int variant) {
  const size_t smem = aa_rows_smem(variant);
  const int th = kAaThreads[variant];
  return with_aa_rows_kernel<T>(variant, [&](void (*k)(StepArgs)) {
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) != cudaSuccess)
      return 0;
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k, th, smem) != cudaSuccess) return 0;
    return b;
  });
}
template <typename T>
cudaError_t launch_step_aa_rows(const StepArgs& a, int variant, int grid, cudaStream_t s) {
  const size_t smem = aa_rows_smem(variant);
  const int th = kAaThreads[variant];
  const cudaError_t e = with_aa_rows_kernel<T>(variant, [&](void (*k)(StepArgs)) {
    return launch_chain(k, dim3(grid), dim3(th), smem, s, a);
  });
  return e != cudaSuccess ? e : cudaGetLastError();
}
template int aa_rows_prepare<float>(int);
template int aa_rows_prepare<__half>(int);
template cudaError_t launch_step_aa_rows<float>(const StepArgs&, int, int, cudaStream_t);
template cudaError_t launch_step_aa_rows<__half>(const StepArgs&, int, int, cudaStream_t);

cudaError_t launch_step_rows_h(const StepArgs& a, int variant, int grid, bool local, cudaStream_t s) {
  const size_t smem = rows_smem(variant);
  const int th = rows_threads(variant);
  const cudaError_t e = with_rows_kernel(variant, local, [&](void (*k)(StepArgs)) {
    return launch_chain(k, dim3(grid), dim3(th), smem, s, a);
  });
  return e != cudaSuccess ? e : cudaGetLastError();
}

template cudaError_t launch_step_bulk<float>(const StepArgs&, int, cudaStream_t);
template cudaError_t launch_step_bulk<__half>(const StepArgs&, int, cudaStream_t);
template int bulk_prepare<float>(int);
template int bulk_prepare<__half>(int);

}  // namespace octlb_gpu
