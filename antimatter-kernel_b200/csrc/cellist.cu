// Uniform-grid cell list (cell edge >= the interaction radius) built by
// Morton-keying the live particles and radix-sorting the keys, and the two
// kernels that walk it:
//   * the cutoff direct sum of ComputeStandardCoulombForces
//     (interaction/coulomb_interaction.cc:23-80) with the shifted-cutoff pair
//     energy of ComputeStandardEnergy (analysis/energy_analysis.cc:16-43);
//   * the annihilation contact search of AnnihilationInteraction::Run
//     (interaction/annihilation.cc:21-61), made deterministic: candidate
//     directed contacts (owner -> partner) with a Philox draw below p are
//     matched greedily in ascending (owner id, partner id) order, which is
//     the result of visiting owners one at a time in id order. The greedy
//     matching is computed in parallel by repeatedly selecting every contact
//     that has the smallest priority at both of its endpoints.
// Pair geometry is FP64 with contraction-free arithmetic so that contact
// decisions are bit-identical to a scalar FP64 evaluation.
#include <algorithm>

#include "amk_internal.cuh"
#include "philox.cuh"

namespace amk {
namespace {

constexpr uint64_t kDeadKey = ~0ull;
constexpr int kCellBits = 21;
constexpr double kCellMax = 2097150.0;  // 2^21 - 2

__device__ __forceinline__ uint64_t spread3(uint64_t v) {
  v &= 0x1fffffull;
  v = (v | (v << 32)) & 0x1f00000000ffffull;
  v = (v | (v << 16)) & 0x1f0000ff0000ffull;
  v = (v | (v << 8)) & 0x100f00f00f00f00full;
  v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
  v = (v | (v << 2)) & 0x1249249249249249ull;
  return v;
}

__device__ __forceinline__ uint64_t morton3(uint32_t x, uint32_t y, uint32_t z) {
  return spread3(x) | (spread3(y) << 1) | (spread3(z) << 2);
}

__device__ __forceinline__ unsigned long long order_bits(double v) {
  const unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(v));
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double from_order_bits(unsigned long long b) {
  const unsigned long long r = (b >> 63) ? (b & 0x7fffffffffffffffull) : ~b;
  return __longlong_as_double(static_cast<long long>(r));
}

__device__ __forceinline__ bool usable(const View& v, long i) {
  return (v.alive == nullptr || v.alive[i]) && isfinite(v.x[i]) && isfinite(v.y[i]) && isfinite(v.z[i]);
}

// bb[0..2] = ordered-bits min, bb[3..5] = ordered-bits of -max.
__global__ void bbox_kernel(View v, unsigned long long* bb) {
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < v.n;
       i += static_cast<long>(gridDim.x) * blockDim.x) {
    if (!usable(v, i)) continue;
    const double p[3] = {v.x[i], v.y[i], v.z[i]};
    for (int d = 0; d < 3; ++d) {
      lo[d] = fmin(lo[d], p[d]);
      hi[d] = fmax(hi[d], p[d]);
    }
  }
  for (int d = 0; d < 3; ++d) {
    for (int o = 16; o > 0; o >>= 1) {
      lo[d] = fmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
      hi[d] = fmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
    }
  }
  if ((threadIdx.x & 31) == 0) {
    for (int d = 0; d < 3; ++d) {
      atomicMin(&bb[d], order_bits(lo[d]));
      atomicMin(&bb[3 + d], order_bits(-hi[d]));
    }
  }
}

struct Grid {
  double ox, oy, oz, inv_cs;
  uint32_t nmax;  // largest valid cell coordinate
};

__device__ __forceinline__ Grid grid_from(const unsigned long long* bb, double radius) {
  Grid g;
  const double lo0 = from_order_bits(bb[0]), lo1 = from_order_bits(bb[1]), lo2 = from_order_bits(bb[2]);
  const double hi0 = -from_order_bits(bb[3]), hi1 = -from_order_bits(bb[4]), hi2 = -from_order_bits(bb[5]);
  double ext = fmax(hi0 - lo0, fmax(hi1 - lo1, hi2 - lo2));
  if (!(ext >= 0.0)) ext = 0.0;  // no live particle
  double cs = radius * (1.0 + 1e-9);
  cs = fmax(cs, ext / kCellMax);
  if (!(cs > 0.0)) cs = 1.0;
  g.ox = isfinite(lo0) ? lo0 : 0.0;
  g.oy = isfinite(lo1) ? lo1 : 0.0;
  g.oz = isfinite(lo2) ? lo2 : 0.0;
  g.inv_cs = 1.0 / cs;
  g.nmax = (1u << kCellBits) - 1u;
  return g;
}

__device__ __forceinline__ void cell_of(const Grid& g, double x, double y, double z, int c[3]) {
  c[0] = static_cast<int>(fmin(floor((x - g.ox) * g.inv_cs), static_cast<double>(g.nmax)));
  c[1] = static_cast<int>(fmin(floor((y - g.oy) * g.inv_cs), static_cast<double>(g.nmax)));
  c[2] = static_cast<int>(fmin(floor((z - g.oz) * g.inv_cs), static_cast<double>(g.nmax)));
  c[0] = max(c[0], 0);
  c[1] = max(c[1], 0);
  c[2] = max(c[2], 0);
}

__global__ void cell_key_kernel(View v, const unsigned long long* bb, double radius, uint64_t* keys,
                                uint32_t* vals) {
  const long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  if (i >= v.n) return;
  vals[i] = static_cast<uint32_t>(i);
  if (!usable(v, i)) {
    keys[i] = kDeadKey;
    return;
  }
  const Grid g = grid_from(bb, radius);
  int c[3];
  cell_of(g, v.x[i], v.y[i], v.z[i], c);
  keys[i] = morton3(c[0], c[1], c[2]);
}

__device__ __forceinline__ long lower_bound(const uint64_t* keys, long n, uint64_t k) {
  long lo = 0, hi = n;
  while (lo < hi) {
    const long mid = (lo + hi) >> 1;
    if (keys[mid] < k)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

__device__ __forceinline__ double dist2_exact(double rx, double ry, double rz) {
  return __dadd_rn(__dadd_rn(__dmul_rn(rx, rx), __dmul_rn(ry, ry)), __dmul_rn(rz, rz));
}

// One thread per sorted particle. Forces in SI (N), potential sums in
// e_i = sum_j q_j (1/r - 1/rc) for the energy.
__global__ void __launch_bounds__(128)
cutoff_kernel(View v, const unsigned long long* bb, double rc, const uint64_t* __restrict__ skeys,
              const uint32_t* __restrict__ sidx, double* __restrict__ epart) {
  const long s = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  if (s >= v.n) return;
  const long i = sidx[s];
  double fx = 0.0, fy = 0.0, fz = 0.0, ei = 0.0;
  const double qi = v.q[i];
  if (skeys[s] != kDeadKey && qi != 0.0) {
    const Grid g = grid_from(bb, rc);
    const double xi = v.x[i], yi = v.y[i], zi = v.z[i];
    int c[3];
    cell_of(g, xi, yi, zi, c);
    const double rc2 = rc * rc;
    const double inv_rc = 1.0 / rc;
    for (int dz = -1; dz <= 1; ++dz) {
      const int cz = c[2] + dz;
      if (cz < 0 || cz > static_cast<int>(g.nmax)) continue;
      for (int dy = -1; dy <= 1; ++dy) {
        const int cy = c[1] + dy;
        if (cy < 0 || cy > static_cast<int>(g.nmax)) continue;
        for (int dx = -1; dx <= 1; ++dx) {
          const int cx = c[0] + dx;
          if (cx < 0 || cx > static_cast<int>(g.nmax)) continue;
          const uint64_t key = morton3(cx, cy, cz);
          for (long k = lower_bound(skeys, v.n, key); k < v.n && skeys[k] == key; ++k) {
            const long j = sidx[k];
            if (j == i) continue;
            const double qj = v.q[j];
            if (qj == 0.0) continue;
            const double rx = xi - v.x[j], ry = yi - v.y[j], rz = zi - v.z[j];
            const double d2 = dist2_exact(rx, ry, rz);
            if (d2 < kMinSquaredDistance) continue;
            if (d2 < rc2) {  // coulomb_interaction.cc:60-73
              const double dist = sqrt(d2);
              const double mag = kCoulombConstant * qi * qj / d2;
              const double w = mag / dist;
              fx += rx * w;
              fy += ry * w;
              fz += rz * w;
            }
            if (epart && d2 <= rc2) ei += qj * (1.0 / sqrt(d2) - inv_rc);  // energy_analysis.cc:30-40
          }
        }
      }
    }
  }
  v.fx[i] = fx;
  v.fy[i] = fy;
  v.fz[i] = fz;
  if (epart) epart[i] = qi * ei;
}

__global__ void zero_forces_kernel(View v) {
  const long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  if (i >= v.n) return;
  v.fx[i] = 0.0;
  v.fy[i] = 0.0;
  v.fz[i] = 0.0;
}

}  // namespace
}  // namespace amk
#include "contacts.cuh"
namespace amk {
namespace {
__global__ void __launch_bounds__(128)
contact_kernel(View v, const uint8_t* __restrict__ species, const uint32_t* __restrict__ ids,
               const unsigned long long* bb, double rc, double prob, uint32_t seed, uint64_t step,
               const uint64_t* __restrict__ skeys, const uint32_t* __restrict__ sidx, Contact* out,
               unsigned long long* count, long cap) {
  const long s = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  if (s >= v.n) return;
  if (skeys[s] == kDeadKey) return;
  const long i = sidx[s];
  const int si = species[i];
  const bool has_partner = si == AMK_POSITRON || si == AMK_ELECTRON || si == AMK_PROTON || si == AMK_ANTIPROTON;
  if (!has_partner) return;
  const Grid g = grid_from(bb, rc);
  const double xi = v.x[i], yi = v.y[i], zi = v.z[i];
  int c[3];
  cell_of(g, xi, yi, zi, c);
  const double rc2 = rc * rc;
  for (int dz = -1; dz <= 1; ++dz) {
    const int cz = c[2] + dz;
    if (cz < 0 || cz > static_cast<int>(g.nmax)) continue;
    for (int dy = -1; dy <= 1; ++dy) {
      const int cy = c[1] + dy;
      if (cy < 0 || cy > static_cast<int>(g.nmax)) continue;
      for (int dx = -1; dx <= 1; ++dx) {
        const int cx = c[0] + dx;
        if (cx < 0 || cx > static_cast<int>(g.nmax)) continue;
        const uint64_t key = morton3(cx, cy, cz);
        for (long k = lower_bound(skeys, v.n, key); k < v.n && skeys[k] == key; ++k) {
          const long j = sidx[k];
          if (j == i) continue;
          const int sj = species[j];
          const bool pair = (si == AMK_ANTIPROTON && sj == AMK_PROTON) || (si == AMK_PROTON && sj == AMK_ANTIPROTON) ||
                            (si == AMK_POSITRON && sj == AMK_ELECTRON) || (si == AMK_ELECTRON && sj == AMK_POSITRON);
          if (!pair) continue;
          const double d2 = dist2_exact(xi - v.x[j], yi - v.y[j], zi - v.z[j]);
          if (!(d2 < rc2)) continue;
          const Philox4 w = philox4x32(seed, kTagAnnihilation, ids[i], ids[j], static_cast<uint32_t>(step),
                                       static_cast<uint32_t>(step >> 32));
          if (!(u01(w.w[0]) < prob)) continue;
          const unsigned long long slot_i = atomicAdd(count, 1ull);
          if (static_cast<long>(slot_i) < cap) {
            Contact e;
            e.a = static_cast<uint32_t>(i);
            e.b = static_cast<uint32_t>(j);
            e.prio = (static_cast<uint64_t>(ids[i]) << 32) | ids[j];
            out[slot_i] = e;
          }
        }
      }
    }
  }
}

struct CellList {
  unsigned long long* bb;
  uint64_t* skeys;
  uint32_t* sidx;
};

int build_cell_list(amk_ctx* c, const View& v, double radius, CellList* out) {
  int rc = AMK_OK;
  const long n = v.n;
  unsigned long long* bb = slot<unsigned long long>(c, kSlotCellStart, 8, &rc);
  AMK_TRY(rc);
  uint64_t* keys = slot<uint64_t>(c, kSlotKeysA, n, &rc);
  AMK_TRY(rc);
  uint32_t* vals = slot<uint32_t>(c, kSlotValsA, n, &rc);
  AMK_TRY(rc);
  uint64_t* skeys = slot<uint64_t>(c, kSlotTreeKeys, n, &rc);
  AMK_TRY(rc);
  uint32_t* sidx = slot<uint32_t>(c, kSlotSorted0, n, &rc);
  AMK_TRY(rc);
  AMK_CUDA_TRY(cudaMemsetAsync(bb, 0xFF, 6 * sizeof(unsigned long long), c->stream));
  bbox_kernel<<<148, 256, 0, c->stream>>>(v, bb);
  AMK_TRY(check_launch(c, "bbox_kernel"));
  cell_key_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, c->stream>>>(v, bb, radius, keys, vals);
  AMK_TRY(check_launch(c, "cell_key_kernel"));
  AMK_TRY(phase_begin(c, AMK_PHASE_SORT));
  AMK_TRY(radix_sort_pairs(c, keys, vals, skeys, sidx, n, 64));
  AMK_TRY(phase_end(c, AMK_PHASE_SORT));
  out->bb = bb;
  out->skeys = skeys;
  out->sidx = sidx;
  return AMK_OK;
}

}  // namespace

int cutoff_forces(amk_ctx* c, const View& v, double cutoff, double* energy_out) {
  if (energy_out) *energy_out = 0.0;
  const long n = v.n;
  if (n == 0) return AMK_OK;
  if (!(cutoff > 0.0)) {  // coulomb_interaction.cc:33-37
    zero_forces_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, c->stream>>>(v);
    return check_launch(c, "zero_forces_kernel");
  }
  CellList cl;
  AMK_TRY(build_cell_list(c, v, cutoff, &cl));
  int rc = AMK_OK;
  double* epart = nullptr;
  if (energy_out) {
    epart = slot<double>(c, kSlotAuxState2, static_cast<size_t>(n) + 8, &rc);
    AMK_TRY(rc);
  }
  AMK_TRY(phase_begin(c, AMK_PHASE_CUTOFF));
  cutoff_kernel<<<static_cast<unsigned>((n + 127) / 128), 128, 0, c->stream>>>(v, cl.bb, cutoff, cl.skeys, cl.sidx,
                                                                               epart);
  AMK_TRY(check_launch(c, "cutoff_kernel"));
  AMK_TRY(phase_end(c, AMK_PHASE_CUTOFF));
  if (energy_out) {
    double* res = slot<double>(c, kSlotAuxState4, 8, &rc);
    AMK_TRY(rc);
    AMK_TRY(reduce_sum(c, epart, n, res));
    double h = 0.0;
    AMK_CUDA_TRY(cudaMemcpyAsync(&h, res, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
    *energy_out = 0.5 * kCoulombConstant * h;  // each pair counted from both ends
  }
  return AMK_OK;
}

int annihilate_view(amk_ctx* c, const View& v, const uint8_t* species, const uint32_t* ids, double radius,
                    double probability, uint32_t seed, uint64_t step_index, long* marked) {
  if (marked) *marked = 0;
  if (!(radius > 0.0) || v.n == 0) return AMK_OK;  // annihilation.cc:34-35
  CellList cl;
  AMK_TRY(build_cell_list(c, v, radius, &cl));
  int rc = AMK_OK;
  unsigned long long* counters = slot<unsigned long long>(c, kSlotAnnAux, 8, &rc);
  AMK_TRY(rc);
  long cap = std::max<long>(1024, v.n / 16);
  for (int attempt = 0; attempt < 3; ++attempt) {
    Contact* edges = slot<Contact>(c, kSlotAnnEdges, static_cast<size_t>(cap), &rc);
    AMK_TRY(rc);
    AMK_CUDA_TRY(cudaMemsetAsync(counters, 0, 4 * sizeof(unsigned long long), c->stream));
    contact_kernel<<<static_cast<unsigned>((v.n + 127) / 128), 128, 0, c->stream>>>(
        v, species, ids, cl.bb, radius, probability, seed, step_index, cl.skeys, cl.sidx, edges, counters, cap);
    AMK_TRY(check_launch(c, "contact_kernel"));
    unsigned long long m = 0;
    AMK_CUDA_TRY(cudaMemcpyAsync(&m, counters, sizeof(m), cudaMemcpyDeviceToHost, c->stream));
    AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (static_cast<long>(m) > cap) {
      cap = static_cast<long>(m) + 1024;
      continue;
    }
    if (m == 0) break;
    // two per-particle priority arrays, then the matching state
    unsigned long long* best = slot<unsigned long long>(
        c, kSlotAnnBest, 2 * static_cast<size_t>(v.n) + sizeof(MatchState) / 8 + 1, &rc);
    AMK_TRY(rc);
    uint8_t* flags = slot<uint8_t>(c, kSlotAuxState1, static_cast<size_t>(v.n) + static_cast<size_t>(m) + 16, &rc);
    AMK_TRY(rc);
    AMK_TRY(queue_matching(c, c->stream, edges, static_cast<long>(m), nullptr, best, best + v.n, flags, flags + v.n,
                           v.alive, reinterpret_cast<MatchState*>(best + 2 * v.n), counters + 2));
    unsigned long long res[2] = {0, 0};
    AMK_CUDA_TRY(cudaMemcpyAsync(res, counters + 2, sizeof(res), cudaMemcpyDeviceToHost, c->stream));
    AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (res[1]) return fail(AMK_ERR_TIMEOUT, "annihilation matching did not converge");
    if (marked) *marked = static_cast<long>(res[0]);
    break;
  }
  return AMK_OK;
}

int annihilate_step(amk_ctx* c, uint64_t step_index, long* marked) {
  if (marked) *marked = 0;
  const amk_params& p = c->p;
  if (!(p.contact_radius > 0.0)) return AMK_OK;  // annihilation.cc:34-35
  AMK_TRY(phase_begin(c, AMK_PHASE_ANNIHILATION));
  AMK_TRY(annihilate_view(c, main_view(c), c->species.as<uint8_t>(), c->ids.as<uint32_t>(), p.contact_radius,
                          p.annihilation_probability, static_cast<uint32_t>(p.seed), step_index, marked));
  AMK_TRY(phase_end(c, AMK_PHASE_ANNIHILATION));
  return AMK_OK;
}

}  // namespace amk

// ======================================================================
// Allocation-free cutoff solver.
//
// Some callers cannot let a library allocate device memory: a host code
// whose device memory is already owned by its own pool allocator (a
// library cudaMalloc could fail there, or fragment the pool), or a
// per-step loop that cannot take the implicit device-wide synchronisation
// of cudaMalloc/cudaFree. For them this variant of the cutoff solver keeps
// all of its scratch (cell keys, sort buffers, histograms: about 2.4 MB)
// in one file-scope device array sized for kNoAllocMaxParticles. Every GPU
// that loads this library holds that array until the process exits.
//
// Set-up: the first call on a device (with that device current) looks up
// the array's device address with cudaGetSymbolAddress and caches it; make
// that first call during set-up, before any stream capture. Later calls
// allocate nothing and call no allocating routine.
//
// Every call uses the same array and it keeps the last call's contents:
// only the bounding-box words must start cleared and they are reset at the
// start of each call. Calls that overlap on the GPU (different streams, or
// different host threads without ordering) race on the array.
// ======================================================================
#include <mutex>

namespace amk {
namespace {

constexpr long kNoAllocMaxParticles = 65536;
constexpr long kNoAllocSortTile = 4096;  // the sort's tile (256 threads x 16)
// radix_sort_pairs_buffers scans its digit histogram (256 counters per tile)
// with one CTA, which handles at most 65,536 counters
static_assert(256 * ((kNoAllocMaxParticles + kNoAllocSortTile - 1) / kNoAllocSortTile) <= 65536,
              "the allocation-free sort's histogram exceeds the one-CTA scan");
constexpr size_t align256(size_t b) { return (b + 255) / 256 * 256; }
constexpr size_t kNaBbox = 0;
constexpr size_t kNaKeys = align256(kNaBbox + 8 * sizeof(unsigned long long));
constexpr size_t kNaVals = align256(kNaKeys + kNoAllocMaxParticles * sizeof(uint64_t));
constexpr size_t kNaSKeys = align256(kNaVals + kNoAllocMaxParticles * sizeof(uint32_t));
constexpr size_t kNaSIdx = align256(kNaSKeys + kNoAllocMaxParticles * sizeof(uint64_t));
constexpr size_t kNaTKeys = align256(kNaSIdx + kNoAllocMaxParticles * sizeof(uint32_t));
constexpr size_t kNaTVals = align256(kNaTKeys + kNoAllocMaxParticles * sizeof(uint64_t));
constexpr size_t kNaHist = align256(kNaTVals + kNoAllocMaxParticles * sizeof(uint32_t));
constexpr size_t kNaBytes =
    align256(kNaHist + 256 * ((kNoAllocMaxParticles + kNoAllocSortTile - 1) / kNoAllocSortTile) * sizeof(uint32_t));

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
unsigned char* g_noalloc_addr[kNoAllocMaxDevices] = {};

}  // namespace

cudaError_t radix_sort_pairs_buffers(cudaStream_t stream, const uint64_t* keys_in, const uint32_t* vals_in,
                                     uint64_t* keys_out, uint32_t* vals_out, uint64_t* ktmp, uint32_t* vtmp,
                                     uint32_t* hist, long n, int key_bits);

}  // namespace amk

extern "C" int amk_coulomb_standard_noalloc(const double* x, const double* y, const double* z, const double* q,
                                            const uint8_t* alive, long n, double cutoff_radius, double* fx,
                                            double* fy, double* fz, void* stream) {
  using namespace amk;
  if (n < 0) return fail(AMK_ERR_INVALID, "amk_coulomb_standard_noalloc: n < 0");
  if (n > kNoAllocMaxParticles)
    return fail(AMK_ERR_LIMIT,
                "amk_coulomb_standard_noalloc: %ld particles exceed the allocation-free maximum of %ld", n,
                kNoAllocMaxParticles);
  if (n == 0) return AMK_OK;
  if (!x || !y || !z || !q || !fx || !fy || !fz) return fail(AMK_ERR_INVALID, "amk_coulomb_standard_noalloc: null array");
  int dev = 0;
  AMK_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(AMK_ERR_LIMIT, "device %d beyond the supported range", dev);
  unsigned char* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[dev]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || p == nullptr)
        return fail(AMK_ERR_CUDA, "cudaGetSymbolAddress of the allocation-free scratch failed: %s",
                    cudaGetErrorString(e));
      g_noalloc_addr[dev] = static_cast<unsigned char*>(p);
    }
    base = g_noalloc_addr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  View v;
  v.n = n;
  v.x = const_cast<double*>(x);
  v.y = const_cast<double*>(y);
  v.z = const_cast<double*>(z);
  v.q = const_cast<double*>(q);
  v.alive = const_cast<uint8_t*>(alive);
  v.fx = fx;
  v.fy = fy;
  v.fz = fz;
  const unsigned blocks = static_cast<unsigned>((n + 255) / 256);
  if (!(cutoff_radius > 0.0)) {  // coulomb_interaction.cc:33-37
    zero_forces_kernel<<<blocks, 256, 0, s>>>(v);
    AMK_CUDA_TRY(cudaGetLastError());
    return AMK_OK;
  }
  unsigned long long* bb = reinterpret_cast<unsigned long long*>(base + kNaBbox);
  uint64_t* keys = reinterpret_cast<uint64_t*>(base + kNaKeys);
  uint32_t* vals = reinterpret_cast<uint32_t*>(base + kNaVals);
  uint64_t* skeys = reinterpret_cast<uint64_t*>(base + kNaSKeys);
  uint32_t* sidx = reinterpret_cast<uint32_t*>(base + kNaSIdx);
  uint64_t* ktmp = reinterpret_cast<uint64_t*>(base + kNaTKeys);
  uint32_t* vtmp = reinterpret_cast<uint32_t*>(base + kNaTVals);
  uint32_t* hist = reinterpret_cast<uint32_t*>(base + kNaHist);
  AMK_CUDA_TRY(cudaMemsetAsync(bb, 0xFF, 6 * sizeof(unsigned long long), s));
  bbox_kernel<<<148, 256, 0, s>>>(v, bb);
  cell_key_kernel<<<blocks, 256, 0, s>>>(v, bb, cutoff_radius, keys, vals);
  AMK_CUDA_TRY(cudaGetLastError());
  AMK_CUDA_TRY(radix_sort_pairs_buffers(s, keys, vals, skeys, sidx, ktmp, vtmp, hist, n, 64));
  cutoff_kernel<<<static_cast<unsigned>((n + 127) / 128), 128, 0, s>>>(v, bb, cutoff_radius, skeys, sidx, nullptr);
  AMK_CUDA_TRY(cudaGetLastError());
  return AMK_OK;
}
