// Tiled all-pairs Coulomb direct sum (no cutoff) on the FP32 pipes.
//
// The reference's exact all-pairs force is Barnes-Hut at theta = 0
// (barnes-hut.h:22-24, barnes-hut.cc:183-221): F_i = sum_{j != i} k q_i q_j
// r_ij / r^3, skipping q_j = 0 and r^2 < 1e-30. Here:
//   * positions are scaled by a power of two L and split into a float pair
//     (hi, lo); the pair difference (xi_hi - xj_hi) + (xi_lo - xj_lo) is
//     exact to FP32 rounding of |r_ij| even for close pairs (Sterbenz), so no
//     absolute position rounding enters the 1/r^2 force;
//   * the pair math is FP32 with one MUFU.RSQ; r^2 gets eps2 = 1e-30 m^2 / L^2
//     added so that the self pair (r = 0, q_j r_ij = 0) contributes exactly 0
//     without a per-pair branch (pairs closer than 1e-15 m are skipped by the
//     reference and are not bit-compatible here);
//   * each 256-source tile is summed in FP32 and folded into a (hi, lo) float
//     pair with TwoSum, so accumulated rounding stays O(eps) per tile rather
//     than O(N eps) (compensated accumulation);
//   * a persistent grid of (SM count x resident CTAs) walks contiguous
//     ranges of (target block, source chunk) units, keeping a target block's
//     sums in registers across its chunks; the finalize kernel adds the
//     partial runs in a fixed order in FP64 (deterministic).
#include <algorithm>

#include "amk_internal.cuh"

namespace amk {
namespace {

constexpr int kThreads = 256;  // threads per CTA = sources per tile
constexpr int kR = 2;          // targets per thread

__device__ __forceinline__ void two_sum_fold(float& hi, float& lo, float p) {
  const float s = hi + p;
  const float bp = s - hi;
  const float e = (hi - (s - bp)) + (p - bp);
  hi = s;
  lo += e;
}

// Work decomposition: units = (target block tb, source chunk) in tb-major
// order; CTA c owns the contiguous unit range [start(c), start(c+1)) with
// start(c) = floor(c * units / grid). Consecutive units of one target block
// accumulate in registers; a run is flushed to partial slot
// (first chunk of the run, tb) when the target block changes.
__device__ __forceinline__ long unit_start(long c, long units, long grid) { return (c * units) / grid; }

template <bool kPhi>
__global__ void __launch_bounds__(kThreads, 3)
allpairs_kernel(const float4* __restrict__ hq, const float4* __restrict__ lo, int n, int n_tb,
                int n_split, int chunk, float eps2, float4* __restrict__ part) {
  __shared__ float4 sh[2][kThreads];
  __shared__ float4 sl[2][kThreads];
  const int tid = threadIdx.x;
  const long units = static_cast<long>(n_tb) * n_split;
  const long u_begin = unit_start(blockIdx.x, units, gridDim.x);
  const long u_end = unit_start(blockIdx.x + 1, units, gridDim.x);
  // the self pair (and pairs closer than 1e-15 m) have d2 < 2 eps2: they are
  // left out of the potential (barnes-hut.cc:242-246)
  const float self_cut = 2.0f * eps2;

  float tx[kR], ty[kR], tz[kR], ux[kR], uy[kR], uz[kR];
  float ahx[kR], ahy[kR], ahz[kR], ahp[kR], alx[kR], aly[kR], alz[kR], alp[kR];
  int run_tb = -1, run_split = 0;

  auto flush = [&]() {
#pragma unroll
    for (int r = 0; r < kR; ++r) {
      const int i = run_tb * (kThreads * kR) + r * kThreads + tid;
      if (i < n) {
        part[(static_cast<size_t>(run_split) * 2 + 0) * n + i] = make_float4(ahx[r], ahy[r], ahz[r], ahp[r]);
        part[(static_cast<size_t>(run_split) * 2 + 1) * n + i] = make_float4(alx[r], aly[r], alz[r], alp[r]);
      }
    }
  };

  for (long u = u_begin; u < u_end; ++u) {
    const int tb = static_cast<int>(u / n_split);
    const int split = static_cast<int>(u - static_cast<long>(tb) * n_split);
    if (tb != run_tb) {
      if (run_tb >= 0) flush();
      run_tb = tb;
      run_split = split;
#pragma unroll
      for (int r = 0; r < kR; ++r) {
        const int i = tb * (kThreads * kR) + r * kThreads + tid;
        float4 h = make_float4(0.f, 0.f, 0.f, 0.f), l = h;
        if (i < n) {
          h = hq[i];
          l = lo[i];
        }
        tx[r] = h.x; ty[r] = h.y; tz[r] = h.z;
        ux[r] = l.x; uy[r] = l.y; uz[r] = l.z;
        ahx[r] = ahy[r] = ahz[r] = ahp[r] = 0.f;
        alx[r] = aly[r] = alz[r] = alp[r] = 0.f;
      }
    }
    const int src_begin = split * chunk;
    const int src_end = min(n, src_begin + chunk);

    // prefetch the first tile into registers
    float4 nh = make_float4(0.f, 0.f, 0.f, 0.f), nl = nh;
    {
      const int j = src_begin + tid;
      if (j < src_end) {
        nh = hq[j];
        nl = lo[j];
      }
    }
    int buf = 0;
    __syncthreads();  // the previous unit's readers are done with both buffers
    sh[buf][tid] = nh;
    sl[buf][tid] = nl;
    __syncthreads();
    for (int t0 = src_begin; t0 < src_end; t0 += kThreads) {
      // prefetch the next tile while this one is consumed
      const int jn = t0 + kThreads + tid;
      nh = make_float4(0.f, 0.f, 0.f, 0.f);
      nl = nh;
      if (jn < src_end) {
        nh = hq[jn];
        nl = lo[jn];
      }
      float px[kR], py[kR], pz[kR], pp[kR];
#pragma unroll
      for (int r = 0; r < kR; ++r) px[r] = py[r] = pz[r] = pp[r] = 0.f;
#pragma unroll 8
      for (int k = 0; k < kThreads; ++k) {
        const float4 s = sh[buf][k];
        const float4 l = sl[buf][k];
#pragma unroll
        for (int r = 0; r < kR; ++r) {
          const float dx = (tx[r] - s.x) + (ux[r] - l.x);
          const float dy = (ty[r] - s.y) + (uy[r] - l.y);
          const float dz = (tz[r] - s.z) + (uz[r] - l.z);
          const float d2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
          const float rinv = rsqrtf(d2);
          const float qr = s.w * rinv;
          const float w = qr * (rinv * rinv);
          px[r] = fmaf(w, dx, px[r]);
          py[r] = fmaf(w, dy, py[r]);
          pz[r] = fmaf(w, dz, pz[r]);
          if (kPhi) pp[r] += (d2 >= self_cut) ? qr : 0.0f;
        }
      }
#pragma unroll
      for (int r = 0; r < kR; ++r) {
        two_sum_fold(ahx[r], alx[r], px[r]);
        two_sum_fold(ahy[r], aly[r], py[r]);
        two_sum_fold(ahz[r], alz[r], pz[r]);
        if (kPhi) two_sum_fold(ahp[r], alp[r], pp[r]);
      }
      buf ^= 1;
      sh[buf][tid] = nh;
      sl[buf][tid] = nl;
      __syncthreads();
    }
  }
  if (run_tb >= 0) flush();
}

// Sums the partial runs of each target in chunk order (FP64) and converts to
// SI: F_i = k e q_i / L^2 * sum, phi_i = e / L * sum_phi. The runs of target
// block tb start at chunk 0 and at every CTA boundary inside tb's units.
__global__ void allpairs_finalize_kernel(int n, int n_tb, int n_split, int grid, const float4* __restrict__ part,
                                         const double* __restrict__ q, const uint8_t* __restrict__ alive,
                                         const float4* __restrict__ hq, double force_coef, double phi_coef,
                                         double* __restrict__ fx, double* __restrict__ fy,
                                         double* __restrict__ fz, double* __restrict__ phi) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const long units = static_cast<long>(n_tb) * n_split;
  const int tb = i / (kThreads * kR);
  const long ub = static_cast<long>(tb) * n_split, ue = ub + n_split;
  long c = (ub * grid) / units;
  while (c + 1 < grid && unit_start(c + 1, units, grid) <= ub) ++c;
  while (c > 0 && unit_start(c, units, grid) > ub) --c;
  double sx = 0.0, sy = 0.0, sz = 0.0, sp = 0.0;
  for (; c < grid; ++c) {
    const long st = unit_start(c, units, grid);
    if (st >= ue) break;
    if (unit_start(c + 1, units, grid) <= st) continue;  // CTA without units
    const int s = static_cast<int>((st > ub ? st : ub) - ub);
    const float4 h = part[(static_cast<size_t>(s) * 2 + 0) * n + i];
    const float4 l = part[(static_cast<size_t>(s) * 2 + 1) * n + i];
    sx += static_cast<double>(h.x) + static_cast<double>(l.x);
    sy += static_cast<double>(h.y) + static_cast<double>(l.y);
    sz += static_cast<double>(h.z) + static_cast<double>(l.z);
    sp += static_cast<double>(h.w) + static_cast<double>(l.w);
  }
  // Targets that are dead, neutral or non-finite were staged with q_e = 0.
  const bool live = hq[i].w != 0.0f;
  const double cq = live ? force_coef * q[i] : 0.0;
  fx[i] = cq * sx;
  fy[i] = cq * sy;
  fz[i] = cq * sz;
  if (phi) phi[i] = (alive == nullptr || alive[i]) ? phi_coef * sp : 0.0;
}

int g_ctas_per_sm[2] = {0, 0};
int g_num_sms = 0;

}  // namespace

int allpairs_forces(amk_ctx* c, const View& v) {
  const int n = static_cast<int>(v.n);
  if (n == 0) return AMK_OK;
  const bool want_phi = v.phi != nullptr;
  if (g_num_sms == 0) {
    AMK_CUDA_TRY(cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, c->device));
    AMK_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&g_ctas_per_sm[0], allpairs_kernel<false>, kThreads, 0));
    AMK_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&g_ctas_per_sm[1], allpairs_kernel<true>, kThreads, 0));
  }
  const int grid_cap = g_num_sms * std::max(1, g_ctas_per_sm[want_phi ? 1 : 0]);
  const int per_tb = kThreads * kR;
  const int n_tb = (n + per_tb - 1) / per_tb;
  // Source chunks of whole tiles; aim for >= 32 units per CTA so that the
  // contiguous per-CTA ranges balance to within ~3%.
  const int tiles = (n + kThreads - 1) / kThreads;
  int n_split = std::min(tiles, std::max(1, (32 * grid_cap + n_tb - 1) / n_tb));
  const int chunk = ((tiles + n_split - 1) / n_split) * kThreads;
  n_split = (n + chunk - 1) / chunk;
  const long units = static_cast<long>(n_tb) * n_split;
  const int grid = static_cast<int>(std::min<long>(units, grid_cap));

  int rc = AMK_OK;
  float4* part = slot<float4>(c, kSlotPartial, static_cast<size_t>(n_split) * 2 * n, &rc);
  AMK_TRY(rc);
  const double l = v.length_scale;
  const float eps2 = static_cast<float>(kMinSquaredDistance / (l * l));

  AMK_TRY(phase_begin(c, AMK_PHASE_ALLPAIRS));
  if (want_phi)
    allpairs_kernel<true><<<grid, kThreads, 0, c->stream>>>(v.hq, v.lo, n, n_tb, n_split, chunk, eps2, part);
  else
    allpairs_kernel<false><<<grid, kThreads, 0, c->stream>>>(v.hq, v.lo, n, n_tb, n_split, chunk, eps2, part);
  AMK_TRY(check_launch(c, "allpairs_kernel"));
  AMK_TRY(phase_end(c, AMK_PHASE_ALLPAIRS));
  AMK_TRY(phase_begin(c, AMK_PHASE_STAGE));
  allpairs_finalize_kernel<<<(n + 255) / 256, 256, 0, c->stream>>>(
      n, n_tb, n_split, grid, part, v.q, v.alive, v.hq, kCoulombConstant * kElementaryCharge / (l * l),
      kElementaryCharge / l, v.fx, v.fy, v.fz, v.phi);
  AMK_TRY(check_launch(c, "allpairs_finalize_kernel"));
  AMK_TRY(phase_end(c, AMK_PHASE_STAGE));
  return AMK_OK;
}

}  // namespace amk
