// blockscan.cuh -- exclusive prefix sums of the time step's short count arrays (hash-grid
// buckets, per-body slave lists, per-pair contact counts) by one CTA: one graph node
// instead of cub's two (an init and a decoupled look-back scan), each of which costs its
// launch latency in a replayed step.  Longer arrays go to cub's device-wide scan.
#pragma once
#include <cub/cub.cuh>

#include "pdl.cuh"

#include <cstdint>

namespace delta {

constexpr int kBlockScanThreads = 1024, kBlockScanItems = 8;
// one tile: a CTA that loops over two or more tiles was slower than cub's two kernels (the
// hopper's 10,001-entry slave lists: 8% of its replayed step)
constexpr int64_t kBlockScanMax = (int64_t)kBlockScanThreads * kBlockScanItems;

// out[i] = in[0] + ... + in[i-1] over tiles of 8192 entries, the running total carried
// from tile to tile (integer sums: exact in any order).
template <class T>
__global__ void __launch_bounds__(kBlockScanThreads) k_block_exclusive_scan(const T *__restrict__ in,
                                                                            T *__restrict__ out, int64_t n) {
  dep_sync();
  using Scan = cub::BlockScan<T, kBlockScanThreads>;
  __shared__ typename Scan::TempStorage tmp;
  __shared__ T carry;
  if (threadIdx.x == 0) carry = T(0);
  __syncthreads();
  for (int64_t base = 0; base < n; base += (int64_t)kBlockScanThreads * kBlockScanItems) {
    T v[kBlockScanItems];
#pragma unroll
    for (int j = 0; j < kBlockScanItems; ++j) {
      const int64_t i = base + (int64_t)threadIdx.x * kBlockScanItems + j;
      v[j] = i < n ? in[i] : T(0);
    }
    T total;
    Scan(tmp).ExclusiveSum(v, v, total);
    const T c = carry;
#pragma unroll
    for (int j = 0; j < kBlockScanItems; ++j) {
      const int64_t i = base + (int64_t)threadIdx.x * kBlockScanItems + j;
      if (i < n) out[i] = v[j] + c;
    }
    __syncthreads();  // every thread has read carry and tmp
    if (threadIdx.x == 0) carry = c + total;
    __syncthreads();
  }
}

// Exclusive sum of n entries: one CTA for n <= kBlockScanMax, else cub's device scan with
// the given temporary storage (sized by cub for n).
template <class T>
inline cudaError_t exclusive_sum(void *temp, size_t &temp_bytes, const T *in, T *out, int64_t n, cudaStream_t s,
                                 bool dep = false) {
  if (n <= kBlockScanMax) return launch_dep(dep, k_block_exclusive_scan<T>, 1, kBlockScanThreads, 0, s, in, out, n);
  return cub::DeviceScan::ExclusiveSum(temp, temp_bytes, in, out, n, s);
}

}  // namespace delta
