// Pipelined fused step for one periodic block (the throughput path).
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
#include "octlb_internal.h"

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

template cudaError_t launch_step_bulk<float>(const StepArgs&, int, cudaStream_t);
template cudaError_t launch_step_bulk<__half>(const StepArgs&, int, cudaStream_t);
template int bulk_prepare<float>(int);
template int bulk_prepare<__half>(int);

}  // namespace octlb_gpu
