// Stable LSD radix sort of (uint64 key, uint32 value) pairs, 8 bits per
// pass: per-tile digit histograms -> one exclusive scan (digit-major, so the
// result is stable across tiles) -> scatter with in-tile stable ranks from
// warp match masks (the context's sort stages each tile in digit order in
// shared memory first, so that a digit's writes are contiguous). HBM-bound:
// each pass reads 12 B and writes 12 B per element plus the key read of the
// histogram pass.
#include <algorithm>

#include "amk_internal.cuh"

namespace amk {
namespace {

constexpr int kSortThreads = 256;
constexpr int kItems = 16;
constexpr int kTile = kSortThreads * kItems;
constexpr int kWarps = kSortThreads / 32;
// counters the one-CTA scan_kernel handles (64 per thread; the bound of the
// allocation-free sort, which has no scratch for the multi-CTA scan)
constexpr long kSingleScanCounters = 65536;
// the context's sort scans more than this many counters (n > 32,768 keys)
// with the multi-CTA scan: the one-CTA scan of 65,536 counters takes about
// 100 us per pass, the multi-CTA one about 15 us
constexpr long kCtxSingleScanCounters = 2048;

__global__ void __launch_bounds__(kSortThreads)
hist_kernel(const uint64_t* __restrict__ keys, long n, int shift, int nb, uint32_t* __restrict__ hist) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const long base = static_cast<long>(blockIdx.x) * kTile;
#pragma unroll 4
  for (int k = 0; k < kItems; ++k) {
    const long i = base + k * kSortThreads + threadIdx.x;
    if (i < n) atomicAdd(&h[(keys[i] >> shift) & 0xFF], 1u);
  }
  __syncthreads();
  hist[static_cast<long>(threadIdx.x) * nb + blockIdx.x] = h[threadIdx.x];
}

// Exclusive scan of `len` counters with one CTA of 1024 threads.
__global__ void __launch_bounds__(1024) scan_kernel(uint32_t* __restrict__ data, long len) {
  __shared__ uint32_t s[1024];
  const long per = (len + 1023) / 1024;
  const long b = threadIdx.x * per;
  const long e = min(len, b + per);
  uint32_t sum = 0;
  for (long i = b; i < e; ++i) sum += data[i];
  s[threadIdx.x] = sum;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    uint32_t v = threadIdx.x >= off ? s[threadIdx.x - off] : 0u;
    __syncthreads();
    s[threadIdx.x] += v;
    __syncthreads();
  }
  uint32_t run = s[threadIdx.x] - sum;
  for (long i = b; i < e; ++i) {
    const uint32_t v = data[i];
    data[i] = run;
    run += v;
  }
}

__global__ void __launch_bounds__(kSortThreads)
scatter_kernel(const uint64_t* __restrict__ kin, const uint32_t* __restrict__ vin, long n, int shift, int nb,
               const uint32_t* __restrict__ offs, uint64_t* __restrict__ kout, uint32_t* __restrict__ vout) {
  __shared__ uint32_t cnt[kWarps][256];
  __shared__ uint32_t running[256];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  running[threadIdx.x] = 0;
  const uint32_t base_off = 0;
  (void)base_off;
  const long base = static_cast<long>(blockIdx.x) * kTile;
  const uint32_t lt_mask = (1u << lane) - 1u;
  for (int k = 0; k < kItems; ++k) {
    const long i = base + k * kSortThreads + threadIdx.x;
    const bool valid = i < n;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) cnt[w][threadIdx.x] = 0;
    __syncthreads();
    uint64_t key = 0;
    uint32_t val = 0;
    int d = 0;
    uint32_t rank = 0;
    const uint32_t active = __ballot_sync(0xffffffffu, valid);
    if (valid) {
      key = kin[i];
      val = vin[i];
      d = static_cast<int>((key >> shift) & 0xFF);
      const uint32_t peers = __match_any_sync(active, d);
      rank = __popc(peers & lt_mask);
      if ((peers & lt_mask) == 0) cnt[warp][d] = __popc(peers);
    }
    __syncthreads();
    if (valid) {
      uint32_t pre = running[d] + rank;
      for (int w = 0; w < warp; ++w) pre += cnt[w][d];
      const long pos = static_cast<long>(offs[static_cast<long>(d) * nb + blockIdx.x]) + pre;
      kout[pos] = key;
      vout[pos] = val;
    }
    __syncthreads();
    uint32_t add = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) add += cnt[w][threadIdx.x];
    running[threadIdx.x] += add;
    __syncthreads();
  }
}

// The same scatter with the tile staged in shared memory in digit order, so
// that the global writes of one digit are contiguous. Warp w ranks the
// contiguous chunk [w * kWarpChunk, (w + 1) * kWarpChunk) of the tile with
// counters of its own (match masks per round, no block barrier), which keeps
// the ranks stable; one block pass then turns the per-warp digit counts into
// tile positions, the elements are placed in shared memory in sorted order
// and written out in that order. Element j of the staged tile goes to
// offs[d][tile] + j - (tile start of digit d).
constexpr int kWarpChunk = kTile / kWarps;  // 512 consecutive elements per warp
constexpr size_t kStagedSmem = static_cast<size_t>(kTile) * (sizeof(uint64_t) + sizeof(uint32_t)) +
                               sizeof(uint32_t) * (kWarps * 256 + 256 + kWarps);

__global__ void __launch_bounds__(kSortThreads)
scatter_staged_kernel(const uint64_t* __restrict__ kin, const uint32_t* __restrict__ vin, long n, int shift,
                      int nb, const uint32_t* __restrict__ offs, uint64_t* __restrict__ kout,
                      uint32_t* __restrict__ vout) {
  extern __shared__ __align__(16) unsigned char sort_smem[];
  uint64_t* sk = reinterpret_cast<uint64_t*>(sort_smem);
  uint32_t* sv = reinterpret_cast<uint32_t*>(sk + kTile);
  uint32_t* wc = sv + kTile;                 // [kWarps][256]: counts, then tile positions
  uint32_t* dstart = wc + kWarps * 256;      // [256]
  uint32_t* wsum = dstart + 256;             // [kWarps]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long base = static_cast<long>(blockIdx.x) * kTile;
  const long wbase = base + static_cast<long>(warp) * kWarpChunk;
  const uint32_t lt_mask = (1u << lane) - 1u;
  uint32_t* mine = wc + warp * 256;
  for (int d = lane; d < 256; d += 32) mine[d] = 0;
  __syncwarp();
  uint64_t key[kItems];
  uint32_t val[kItems], dr[kItems];  // dr: digit | rank in the warp's chunk << 8
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    const long i = wbase + k * 32 + lane;
    const bool valid = i < n;
    key[k] = 0;
    val[k] = 0;
    dr[k] = 0;
    const uint32_t active = __ballot_sync(0xffffffffu, valid);
    if (valid) {
      key[k] = kin[i];
      val[k] = vin[i];
      const int d = static_cast<int>((key[k] >> shift) & 0xFF);
      const uint32_t peers = __match_any_sync(active, d);
      const int leader = __ffs(peers) - 1;
      uint32_t old = lane == leader ? mine[d] : 0u;
      old = __shfl_sync(active, old, leader);
      if (lane == leader) mine[d] = old + __popc(peers);
      dr[k] = static_cast<uint32_t>(d) | ((old + __popc(peers & lt_mask)) << 8);
    }
    __syncwarp();
  }
  __syncthreads();
  // digit d (thread d): the per-warp starts within the digit and the digit's total
  {
    const int d = threadIdx.x;
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      const uint32_t c = wc[w * 256 + d];
      wc[w * 256 + d] = run;
      run += c;
    }
    uint32_t incl = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    uint32_t before = 0;
    for (int w = 0; w < warp; ++w) before += wsum[w];
    const uint32_t start = before + incl - run;
    dstart[d] = start;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) wc[w * 256 + d] += start;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    const long i = wbase + k * 32 + lane;
    if (i < n) {
      const uint32_t pos = mine[dr[k] & 0xFF] + (dr[k] >> 8);
      sk[pos] = key[k];
      sv[pos] = val[k];
    }
  }
  __syncthreads();
  const int tile_n = static_cast<int>(min(static_cast<long>(kTile), n - base));
  for (int j = threadIdx.x; j < tile_n; j += kSortThreads) {
    const uint64_t kk = sk[j];
    const int d = static_cast<int>((kk >> shift) & 0xFF);
    const long pos = static_cast<long>(offs[static_cast<long>(d) * nb + blockIdx.x]) + (j - dstart[d]);
    kout[pos] = kk;
    vout[pos] = sv[j];
  }
}

}  // namespace

int radix_sort_pairs(amk_ctx* c, const uint64_t* keys_in, const uint32_t* vals_in, uint64_t* keys_out,
                     uint32_t* vals_out, long n, int key_bits) {
  if (n <= 0) return AMK_OK;
  if (n > 0xFFFFFFF0L) return fail(AMK_ERR_LIMIT, "radix sort of %ld elements exceeds 32-bit ranks", n);
  const int passes = std::max(1, (key_bits + 7) / 8);
  const int nb = static_cast<int>((n + kTile - 1) / kTile);
  int rc = AMK_OK;
  uint64_t* kt = slot<uint64_t>(c, kSlotKeysB, static_cast<size_t>(n), &rc);
  AMK_TRY(rc);
  uint32_t* vt = slot<uint32_t>(c, kSlotValsB, static_cast<size_t>(n), &rc);
  AMK_TRY(rc);
  uint32_t* hist = slot<uint32_t>(c, kSlotSortHist, static_cast<size_t>(256) * nb, &rc);
  AMK_TRY(rc);
  int* total = slot<int>(c, kSlotSortFlags, 8, &rc);
  AMK_TRY(rc);
  // the staged scatter's shared memory is above the 48 KB default (set per call: per device)
  AMK_CUDA_TRY(cudaFuncSetAttribute(scatter_staged_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(kStagedSmem)));
  const uint64_t* ksrc = keys_in;
  const uint32_t* vsrc = vals_in;
  for (int p = 0; p < passes; ++p) {
    const bool to_out = ((passes - 1 - p) % 2) == 0;
    uint64_t* kdst = to_out ? keys_out : kt;
    uint32_t* vdst = to_out ? vals_out : vt;
    const int shift = 8 * p;
    hist_kernel<<<nb, kSortThreads, 0, c->stream>>>(ksrc, n, shift, nb, hist);
    AMK_TRY(check_launch(c, "hist_kernel"));
    if (static_cast<long>(256) * nb > kCtxSingleScanCounters) {
      // many tiles: the multi-CTA scan (in place; counts stay below 2^31)
      AMK_TRY(exclusive_scan_int(c, reinterpret_cast<const int*>(hist), static_cast<long>(256) * nb,
                                 reinterpret_cast<int*>(hist), total));
    } else {
      scan_kernel<<<1, 1024, 0, c->stream>>>(hist, static_cast<long>(256) * nb);
      AMK_TRY(check_launch(c, "scan_kernel"));
    }
    scatter_staged_kernel<<<nb, kSortThreads, kStagedSmem, c->stream>>>(ksrc, vsrc, n, shift, nb, hist, kdst, vdst);
    AMK_TRY(check_launch(c, "scatter_staged_kernel"));
    ksrc = kdst;
    vsrc = vdst;
  }
  return AMK_OK;
}

}  // namespace amk

namespace amk {

// The same sort on caller-provided buffers (no context, no allocation):
// ktmp/vtmp hold n elements, hist holds 256 * ceil(n / 4096) counters. The
// digit scan is the one-CTA scan_kernel, so 256 * ceil(n / 4096) must stay
// within kSingleScanCounters (n <= 1,048,576): larger n is refused with
// cudaErrorInvalidValue before anything is launched.
cudaError_t radix_sort_pairs_buffers(cudaStream_t stream, const uint64_t* keys_in, const uint32_t* vals_in,
                                     uint64_t* keys_out, uint32_t* vals_out, uint64_t* ktmp, uint32_t* vtmp,
                                     uint32_t* hist, long n, int key_bits) {
  if (n <= 0) return cudaSuccess;
  const int passes = std::max(1, (key_bits + 7) / 8);
  const int nb = static_cast<int>((n + kTile - 1) / kTile);
  if (static_cast<long>(256) * nb > kSingleScanCounters) return cudaErrorInvalidValue;
  const uint64_t* ksrc = keys_in;
  const uint32_t* vsrc = vals_in;
  for (int p = 0; p < passes; ++p) {
    const bool to_out = ((passes - 1 - p) % 2) == 0;
    uint64_t* kdst = to_out ? keys_out : ktmp;
    uint32_t* vdst = to_out ? vals_out : vtmp;
    const int shift = 8 * p;
    hist_kernel<<<nb, kSortThreads, 0, stream>>>(ksrc, n, shift, nb, hist);
    scan_kernel<<<1, 1024, 0, stream>>>(hist, static_cast<long>(256) * nb);
    scatter_kernel<<<nb, kSortThreads, 0, stream>>>(ksrc, vsrc, n, shift, nb, hist, kdst, vdst);
    ksrc = kdst;
    vsrc = vdst;
  }
  return cudaGetLastError();
}

}  // namespace amk
