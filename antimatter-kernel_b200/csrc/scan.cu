// Exclusive prefix sum of int32 counts (multi-CTA: per-block sums -> one
// CTA scans the block sums -> per-block downsweep). Used by the octree
// builder to number nodes.
#include "amk_internal.cuh"

namespace amk {
namespace {

constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int block_exclusive_scan(int v, int* sh, int* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = lane < kScanThreads / 32 ? sh[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < kScanThreads / 32) sh[lane] = w;
  }
  __syncthreads();
  const int before = (warp > 0 ? sh[warp - 1] : 0) + x - v;
  if (total) *total = sh[kScanThreads / 32 - 1];
  __syncthreads();
  return before;
}

__global__ void __launch_bounds__(kScanThreads) scan_block_sums(const int* in, long n, int* sums) {
  __shared__ int sh[32];
  const long base = static_cast<long>(blockIdx.x) * kScanTile + static_cast<long>(threadIdx.x) * kScanItems;
  int s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k)
    if (base + k < n) s += in[base + k];
  int total = 0;
  block_exclusive_scan(s, sh, &total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads) scan_sums_kernel(int* sums, int nb, int* grand_total) {
  __shared__ int sh[32];
  int carry = 0;
  for (int base = 0; base < nb; base += kScanThreads) {
    const int i = base + threadIdx.x;
    const int v = i < nb ? sums[i] : 0;
    int total = 0;
    const int ex = block_exclusive_scan(v, sh, &total);
    if (i < nb) sums[i] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0) *grand_total = carry;
}

__global__ void __launch_bounds__(kScanThreads)
scan_down_kernel(const int* in, long n, const int* sums, int* out) {
  __shared__ int sh[32];
  const long base = static_cast<long>(blockIdx.x) * kScanTile + static_cast<long>(threadIdx.x) * kScanItems;
  int v[kScanItems];
  int s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = (base + k < n) ? in[base + k] : 0;
    s += v[k];
  }
  int run = block_exclusive_scan(s, sh, nullptr) + sums[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) out[base + k] = run;
    run += v[k];
  }
}

}  // namespace

// out[i] = sum_{j < i} in[i]; *total_dev = sum of all (device pointer).
// out may equal in (each thread reads its items before writing them).
int exclusive_scan_int(amk_ctx* c, const int* in, long n, int* out, int* total_dev) {
  if (n <= 0) {
    AMK_CUDA_TRY(cudaMemsetAsync(total_dev, 0, sizeof(int), c->stream));
    return AMK_OK;
  }
  const int nb = static_cast<int>((n + kScanTile - 1) / kScanTile);
  int rc = AMK_OK;
  int* sums = slot<int>(c, kSlotScanSums, static_cast<size_t>(nb) + 1, &rc);
  AMK_TRY(rc);
  scan_block_sums<<<nb, kScanThreads, 0, c->stream>>>(in, n, sums);
  AMK_TRY(check_launch(c, "scan_block_sums"));
  scan_sums_kernel<<<1, kScanThreads, 0, c->stream>>>(sums, nb, total_dev);
  AMK_TRY(check_launch(c, "scan_sums_kernel"));
  scan_down_kernel<<<nb, kScanThreads, 0, c->stream>>>(in, n, sums, out);
  return check_launch(c, "scan_down_kernel");
}

}  // namespace amk
