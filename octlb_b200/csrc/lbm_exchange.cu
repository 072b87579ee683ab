// Pack / unpack kernels of the cross-rank exchange (rank contexts of
// octlb_gpu_create_part).
//
// The same-level ghost exchange of the reference (GhostSchedule::exchange,
// ghost_schedule.h:121-255: face layers of N^2 and edge rows of N cells, all
// 19 populations, post-collision) becomes, per level step, one gather of the
// owned cells the peers mirror into a staging buffer, the transport, and one
// scatter of the received cells into this rank's mirror blocks.  Items are
// [item][19] in the staging buffer (each peer's run contiguous); a thread
// takes one (population, item) pair, items fastest, so the reads and writes
// of the state array are coalesced along the face's contiguous z rows.
//
// The coupler's payloads (LevelCoupler's MPI batches, level_coupler.cpp:
// 325-436 and 492-585: macros and f_neq of interface cells) are the save rows
// here -- the pre-collision populations of the interface cells -- gathered
// the same way after the source level's step; a peer receives them straight
// into its save-row buffer.
#include "octlb_internal.h"

namespace octlb_gpu {
namespace {

constexpr int kXThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kXThreads)
k_pack_cells(const T* __restrict__ src, long long qs, const long long* __restrict__ slots, long long items,
             T* __restrict__ buf) {
  const long long t = static_cast<long long>(blockIdx.x) * kXThreads + threadIdx.x;
  if (t >= items * kQ) return;
  const int i = static_cast<int>(t / items);
  const long long j = t - i * items;
  buf[j * kQ + i] = src[i * qs + slots[j]];
}

template <typename T>
__global__ void __launch_bounds__(kXThreads)
k_unpack_cells(T* __restrict__ dst, long long qs, const long long* __restrict__ slots, long long items,
               const T* __restrict__ buf) {
  const long long t = static_cast<long long>(blockIdx.x) * kXThreads + threadIdx.x;
  if (t >= items * kQ) return;
  const int i = static_cast<int>(t / items);
  const long long j = t - i * items;
  dst[i * qs + slots[j]] = buf[j * kQ + i];
}

// Save rows are [row][19] floats already: item j copies row rows[j].
__global__ void __launch_bounds__(kXThreads)
k_pack_rows(const float* __restrict__ save, const long long* __restrict__ rows, long long items,
            float* __restrict__ buf) {
  const long long t = static_cast<long long>(blockIdx.x) * kXThreads + threadIdx.x;
  if (t >= items * kQ) return;
  const long long j = t / kQ;
  const int i = static_cast<int>(t - j * kQ);
  buf[t] = save[rows[j] * kQ + i];
}

inline unsigned grid_of(long long work) { return static_cast<unsigned>((work + kXThreads - 1) / kXThreads); }

}  // namespace

template <typename T>
cudaError_t launch_pack_cells(const void* src, long long qs, const long long* slots, long long items, void* buf,
                              cudaStream_t s) {
  if (items == 0) return cudaSuccess;
  k_pack_cells<T><<<grid_of(items * kQ), kXThreads, 0, s>>>(static_cast<const T*>(src), qs, slots, items,
                                                             static_cast<T*>(buf));
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_unpack_cells(void* dst, long long qs, const long long* slots, long long items, const void* buf,
                                cudaStream_t s) {
  if (items == 0) return cudaSuccess;
  k_unpack_cells<T><<<grid_of(items * kQ), kXThreads, 0, s>>>(static_cast<T*>(dst), qs, slots, items,
                                                               static_cast<const T*>(buf));
  return cudaGetLastError();
}

cudaError_t launch_pack_rows(const float* save, const long long* rows, long long items, float* buf, cudaStream_t s) {
  if (items == 0) return cudaSuccess;
  k_pack_rows<<<grid_of(items * kQ), kXThreads, 0, s>>>(save, rows, items, buf);
  return cudaGetLastError();
}

template cudaError_t launch_pack_cells<float>(const void*, long long, const long long*, long long, void*, cudaStream_t);
template cudaError_t launch_pack_cells<__half>(const void*, long long, const long long*, long long, void*,
                                               cudaStream_t);
template cudaError_t launch_unpack_cells<float>(void*, long long, const long long*, long long, const void*,
                                                cudaStream_t);
template cudaError_t launch_unpack_cells<__half>(void*, long long, const long long*, long long, const void*,
                                                 cudaStream_t);

}  // namespace octlb_gpu
