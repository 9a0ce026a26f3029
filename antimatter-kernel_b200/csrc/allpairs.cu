// Tiled all-pairs Coulomb direct sum (no cutoff) on the FP32 pipes.
//
// The reference's exact all-pairs force is Barnes-Hut at theta = 0
// (barnes-hut.h:22-24, barnes-hut.cc:183-221): F_i = sum_{j != i} k q_i q_j
// r_ij / r^3, skipping q_j = 0 and r^2 < 1e-30. Design:
//   * particles are ordered along a 30-bit Morton curve (radix sort; the
//     order is reused for 16 calls on a context's own particle set -- boxes
//     are rebuilt on every call, so a stale order costs speed only); every
//     32 consecutive sorted particles form a sub-tile with an axis-aligned
//     box, and each warp owns 64 consecutive targets (two sub-tiles);
//   * positions are scaled by a power of two L. The near/far decision is
//     made per (warp, 32-source sub-tile), uniform across the warp. Near
//     pairs (the warp's box and the sub-tile's box closer than a quarter of
//     their summed half-extent norms) use a float pair (hi, lo):
//     r_ij = (xi_hi - xj_hi) + (xi_lo - xj_lo), exact to FP32 rounding of
//     |r_ij| (Sterbenz) -- 18 FP32 ops per pair, issued as packed FP32x2
//     operations over a lane's two targets (9 issue slots per pair); the
//     self pair and exact duplicates give r = 0 exactly;
//   * far pairs: each source carries its FP32 offset u_j from its sub-tile
//     centre (stored negated) and each target forms a_i = x_i - c_sub once
//     per sub-tile, so r_ij = a_i + (-u_j) costs one FADD per component --
//     12 FP32 ops per pair, issued as packed FP32x2 operations over a lane's
//     two targets (one instruction per two pairs, two MUFU.RSQ);
//     Its relative error is at most eps (1 + 1.5 / 0.25) = 7 eps of |r_ij|
//     for the closest far pairs (gap >= 0.25 (|h_w| + |h_s|)) and ~eps for
//     the bulk; about 5 % of the sub-tile pairs of a 65,536-particle cloud
//     are near;
//   * r^2 gets eps2 = max(1e-30 m^2 / L^2, 1e-25) added so that the self pair
//     (r = 0) contributes exactly 0 without a branch and rinv^3 cannot
//     overflow (the reference skips pairs closer than 1e-15 m; such pairs,
//     and pairs closer than 3e-13 L, are softened here instead);
//   * each 256-source chunk (8 sub-tiles) is summed in FP32 and folded into a
//     (hi, lo) float pair with TwoSum (compensated accumulation);
//   * a persistent grid of (SM count x resident CTAs) walks contiguous
//     ranges of (target block, source chunk) units, keeping a target block's
//     sums in registers across its chunks; the finalize kernel adds the
//     partial runs in a fixed order in FP64 (deterministic).
// Compiled with -ftz=true: every operand is a normal float by construction.
#include <algorithm>

#include "amk_internal.cuh"
#include "morton.cuh"

namespace amk {
namespace {

constexpr int kThreads = 256;  // threads per CTA = sources per chunk
constexpr int kR = 2;          // targets per thread (a warp owns 64 consecutive targets)
constexpr int kSub = 32;       // particles per sub-tile (box granularity)
constexpr int kSubPerChunk = kThreads / kSub;
constexpr float kNearFactor = 0.25f;
constexpr int kResortEvery = 16;

__device__ __forceinline__ void two_sum_fold(float& hi, float& lo, float p) {
  const float s = hi + p;
  const float bp = s - hi;
  const float e = (hi - (s - bp)) + (p - bp);
  hi = s;
  lo += e;
}

__device__ __forceinline__ bool usable(const View& v, long i) {
  return (v.alive == nullptr || v.alive[i]) && v.q[i] != 0.0 && isfinite(v.x[i]) && isfinite(v.y[i]) &&
         isfinite(v.z[i]);
}

// ------------------------------------------------------------ ordering
__global__ void ap_bbox_kernel(View v, unsigned long long* bb) {
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
      atomicMin(&bb[d], double_order_bits(lo[d]));
      atomicMin(&bb[3 + d], double_order_bits(-hi[d]));
    }
  }
}

// 30-bit Morton key (10 bits per axis) inside the live bounding box; unusable
// particles sort last.
__global__ void ap_key_kernel(View v, const unsigned long long* bb, uint64_t* keys, uint32_t* vals) {
  const long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  if (i >= v.n) return;
  vals[i] = static_cast<uint32_t>(i);
  if (!usable(v, i)) {
    keys[i] = 0xFFFFFFFFull;
    return;
  }
  const double p[3] = {v.x[i], v.y[i], v.z[i]};
  uint32_t c[3];
  for (int d = 0; d < 3; ++d) {
    const double lo = double_from_order_bits(bb[d]);
    const double hi = -double_from_order_bits(bb[3 + d]);
    const double ext = hi - lo;
    const double f = ext > 0.0 ? (p[d] - lo) / ext : 0.0;
    c[d] = static_cast<uint32_t>(fmin(fmax(f * 1024.0, 0.0), 1023.0));
  }
  keys[i] = morton3_21(c[0], c[1], c[2]);
}

// ------------------------------------------------------------ staging
struct TileBox {
  float4 c;   // centre (scaled, float hi part); w = 1 when the tile has sources
  float4 cl;  // centre low part
  float4 h;   // half-extent per axis (rounded up); w = |h|
};

// One warp per sub-tile of 32 sorted particles: double-float positions,
// offsets from the sub-tile centre, and the box of its usable particles.
__global__ void __launch_bounds__(kThreads)
ap_stage_kernel(View v, const uint32_t* __restrict__ perm, double inv_l, float4* __restrict__ hq,
                float4* __restrict__ lo, float4* __restrict__ rel, TileBox* __restrict__ boxes) {
  const long k = static_cast<long>(blockIdx.x) * kThreads + threadIdx.x;
  const long sub = k / kSub;
  double xs = 0.0, ys = 0.0, zs = 0.0, qe = 0.0;
  bool ok = false;
  if (k < v.n) {
    const long i = perm[k];
    ok = usable(v, i);
    if (ok) {
      xs = v.x[i] * inv_l;
      ys = v.y[i] * inv_l;
      zs = v.z[i] * inv_l;
      qe = v.q[i] / kElementaryCharge;
    }
  }
  double m[6] = {ok ? xs : INFINITY, ok ? ys : INFINITY, ok ? zs : INFINITY,
                 ok ? -xs : INFINITY, ok ? -ys : INFINITY, ok ? -zs : INFINITY};
#pragma unroll
  for (int d = 0; d < 6; ++d)
    for (int o = 16; o > 0; o >>= 1) m[d] = fmin(m[d], __shfl_xor_sync(0xffffffffu, m[d], o));
  const bool any = isfinite(m[0]);
  const double cx = any ? 0.5 * (m[0] - m[3]) : 0.0;
  const double cy = any ? 0.5 * (m[1] - m[4]) : 0.0;
  const double cz = any ? 0.5 * (m[2] - m[5]) : 0.0;
  float4 h = make_float4(0.f, 0.f, 0.f, 0.f), l = h, u = h;
  if (ok) {
    h.x = __double2float_rn(xs);
    h.y = __double2float_rn(ys);
    h.z = __double2float_rn(zs);
    h.w = __double2float_rn(qe);
    l.x = __double2float_rn(xs - static_cast<double>(h.x));
    l.y = __double2float_rn(ys - static_cast<double>(h.y));
    l.z = __double2float_rn(zs - static_cast<double>(h.z));
    u.x = -__double2float_rn(xs - cx);  // negated: the far loop adds it
    u.y = -__double2float_rn(ys - cy);
    u.z = -__double2float_rn(zs - cz);
    u.w = h.w;
  }
  if (k < v.n) {
    hq[k] = h;
    lo[k] = l;
    rel[k] = u;
  }
  if ((threadIdx.x & 31) == 0) {
    TileBox b;
    b.c = make_float4(__double2float_rn(cx), __double2float_rn(cy), __double2float_rn(cz), any ? 1.f : 0.f);
    b.cl = make_float4(__double2float_rn(cx - static_cast<double>(b.c.x)),
                       __double2float_rn(cy - static_cast<double>(b.c.y)),
                       __double2float_rn(cz - static_cast<double>(b.c.z)), 0.f);
    const double hx = any ? 0.5 * (-m[3] - m[0]) : 0.0;
    const double hy = any ? 0.5 * (-m[4] - m[1]) : 0.0;
    const double hz = any ? 0.5 * (-m[5] - m[2]) : 0.0;
    b.h = make_float4(__double2float_ru(hx), __double2float_ru(hy), __double2float_ru(hz),
                      __double2float_ru(sqrt(hx * hx + hy * hy + hz * hz)));
    boxes[sub] = b;
  }
}

// ------------------------------------------------------------ pair kernel
__device__ __forceinline__ long unit_start(long c, long units, long grid) { return (c * units) / grid; }

// Work: units = (target block tb, chunk of source tiles), tb-major; CTA c owns
// units [start(c), start(c+1)), start(c) = floor(c * units / grid). A target
// block's sums stay in registers over its consecutive units; a run is
// flushed to partial slot (first chunk of the run) when the block changes.
// Target block tb = sorted targets [512 tb, 512 tb + 512); warp w owns
// [512 tb + 64 w, + 64): lane l holds targets +l (r = 0) and +32+l (r = 1).
template <bool kPhi>
__global__ void __launch_bounds__(kThreads, 2)
allpairs_kernel(const float4* __restrict__ hq, const float4* __restrict__ lo, const float4* __restrict__ rel,
                const TileBox* __restrict__ boxes, int n, int n_tiles, int n_tb, int n_split,
                int tiles_per_chunk, float eps2, float4* __restrict__ part) {
  __shared__ float4 sa[kThreads];
  __shared__ float4 sb[kThreads];
  __shared__ float4 sc[kThreads];
  __shared__ TileBox sbox[kSubPerChunk];
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int n_sub = (n + kSub - 1) / kSub;
  const long units = static_cast<long>(n_tb) * n_split;
  const long u_begin = unit_start(blockIdx.x, units, gridDim.x);
  const long u_end = unit_start(blockIdx.x + 1, units, gridDim.x);
  const float self_cut = 2.0f * eps2;  // self pair and r < 1e-15 m: not in phi

  float tx[kR], ty[kR], tz[kR], ux[kR], uy[kR], uz[kR];
  float ahx[kR], ahy[kR], ahz[kR], ahp[kR], alx[kR], aly[kR], alz[kR], alp[kR];
  __shared__ float4 swc[kThreads / 32], swh[kThreads / 32];  // each warp's target box
  bool warp_live = false;
  int run_tb = -1, run_split = 0;

  auto target = [&](int tb, int r) { return tb * (kThreads * kR) + warp * (kSub * kR) + r * kSub + lane; };
  auto flush = [&]() {
#pragma unroll
    for (int r = 0; r < kR; ++r) {
      const int i = target(run_tb, r);
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
        const int i = target(tb, r);
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
      // union box of the warp's two target sub-tiles (warp-uniform loads)
      const int s0 = (tb * (kThreads * kR) + warp * (kSub * kR)) / kSub;
      TileBox b0 = s0 < n_sub ? boxes[s0] : TileBox{};
      TileBox b1 = s0 + 1 < n_sub ? boxes[s0 + 1] : TileBox{};
      if (b1.c.w == 0.f) b1 = b0;
      if (b0.c.w == 0.f) b0 = b1;
      warp_live = b0.c.w != 0.f;
      const float lx = fminf(b0.c.x - b0.h.x, b1.c.x - b1.h.x), hx = fmaxf(b0.c.x + b0.h.x, b1.c.x + b1.h.x);
      const float ly = fminf(b0.c.y - b0.h.y, b1.c.y - b1.h.y), hy = fmaxf(b0.c.y + b0.h.y, b1.c.y + b1.h.y);
      const float lz = fminf(b0.c.z - b0.h.z, b1.c.z - b1.h.z), hz = fmaxf(b0.c.z + b0.h.z, b1.c.z + b1.h.z);
      float4 wh = make_float4(0.5001f * (hx - lx), 0.5001f * (hy - ly), 0.5001f * (hz - lz), 0.f);
      wh.w = 1.0001f * sqrtf(wh.x * wh.x + wh.y * wh.y + wh.z * wh.z);
      __syncwarp();
      if (lane == 0) {
        swc[warp] = make_float4(0.5f * (lx + hx), 0.5f * (ly + hy), 0.5f * (lz + hz), 0.f);
        swh[warp] = wh;
      }
      __syncwarp();
    }
    const int t_begin = split * tiles_per_chunk;
    const int t_end = min(n_tiles, t_begin + tiles_per_chunk);

    for (int t = t_begin; t < t_end; ++t) {
      const int j = t * kThreads + tid;
      __syncthreads();  // the previous chunk's readers are done with the buffers
      if (j < n) {
        sa[tid] = hq[j];
        sb[tid] = lo[j];
        sc[tid] = rel[j];
      } else {
        sa[tid] = sb[tid] = sc[tid] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
      if (tid < kSubPerChunk) {
        const int sidx = t * kSubPerChunk + tid;
        sbox[tid] = sidx < n_sub ? boxes[sidx] : TileBox{};
      }
      __syncthreads();
      if (!warp_live) continue;  // no usable target in this warp (uniform)
      float px[kR], py[kR], pz[kR], pp[kR];
#pragma unroll
      for (int r = 0; r < kR; ++r) px[r] = py[r] = pz[r] = pp[r] = 0.f;
      const float4 wc = swc[warp], wh = swh[warp];
      for (int q = 0; q < kSubPerChunk; ++q) {
        const TileBox sbx = sbox[q];
        if (sbx.c.w == 0.f) continue;  // no usable sources (uniform)
        const float gx = fmaxf(fabsf(wc.x - sbx.c.x) - (wh.x + sbx.h.x), 0.f);
        const float gy = fmaxf(fabsf(wc.y - sbx.c.y) - (wh.y + sbx.h.y), 0.f);
        const float gz = fmaxf(fabsf(wc.z - sbx.c.z) - (wh.z + sbx.h.z), 0.f);
        const float lim = kNearFactor * (wh.w + sbx.h.w);
        const int base = q * kSub;
        if (gx * gx + gy * gy + gz * gz <= lim * lim) {
          // near: double-float differences (t_hi - s_hi) + (t_lo - s_lo) for
          // the lane's two targets in the two halves of packed FP32x2
          // operations; t - s is formed as fma(s, -1, t), the same rounding
          // as the subtraction, so the sums equal the scalar form bit for bit
          const float2 m1 = make_float2(-1.f, -1.f), e2 = make_float2(eps2, eps2);
          const float2 thx = make_float2(tx[0], tx[1]), thy = make_float2(ty[0], ty[1]),
                       thz = make_float2(tz[0], tz[1]);
          const float2 tlx = make_float2(ux[0], ux[1]), tly = make_float2(uy[0], uy[1]),
                       tlz = make_float2(uz[0], uz[1]);
          float2 fx = make_float2(px[0], px[1]), fy = make_float2(py[0], py[1]),
                 fz = make_float2(pz[0], pz[1]);
#pragma unroll 8
          for (int k = 0; k < kSub; ++k) {
            const float4 s = sa[base + k];
            const float4 l = sb[base + k];
            const float2 dx = __fadd2_rn(__ffma2_rn(make_float2(s.x, s.x), m1, thx),
                                         __ffma2_rn(make_float2(l.x, l.x), m1, tlx));
            const float2 dy = __fadd2_rn(__ffma2_rn(make_float2(s.y, s.y), m1, thy),
                                         __ffma2_rn(make_float2(l.y, l.y), m1, tly));
            const float2 dz = __fadd2_rn(__ffma2_rn(make_float2(s.z, s.z), m1, thz),
                                         __ffma2_rn(make_float2(l.z, l.z), m1, tlz));
            const float2 d2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, e2)));
            const float2 rinv = make_float2(rsqrtf(d2.x), rsqrtf(d2.y));
            const float2 qr = __fmul2_rn(make_float2(s.w, s.w), rinv);
            const float2 w = __fmul2_rn(qr, __fmul2_rn(rinv, rinv));
            fx = __ffma2_rn(w, dx, fx);
            fy = __ffma2_rn(w, dy, fy);
            fz = __ffma2_rn(w, dz, fz);
            if (kPhi) {
              pp[0] += (d2.x >= self_cut) ? qr.x : 0.0f;
              pp[1] += (d2.y >= self_cut) ? qr.y : 0.0f;
            }
          }
          px[0] = fx.x;
          px[1] = fx.y;
          py[0] = fy.x;
          py[1] = fy.y;
          pz[0] = fz.x;
          pz[1] = fz.y;
        } else {
          // far: the warp's two targets per lane in the two halves of packed
          // FP32x2 operations (same operations and association as the
          // scalar form, half the issue slots)
          static_assert(kR == 2, "packed far path holds two targets per lane");
          float2 ax, ay, az;
          ax.x = (tx[0] - sbx.c.x) + (ux[0] - sbx.cl.x);
          ax.y = (tx[1] - sbx.c.x) + (ux[1] - sbx.cl.x);
          ay.x = (ty[0] - sbx.c.y) + (uy[0] - sbx.cl.y);
          ay.y = (ty[1] - sbx.c.y) + (uy[1] - sbx.cl.y);
          az.x = (tz[0] - sbx.c.z) + (uz[0] - sbx.cl.z);
          az.y = (tz[1] - sbx.c.z) + (uz[1] - sbx.cl.z);
          const float2 e2 = make_float2(eps2, eps2);
          float2 fx = make_float2(px[0], px[1]), fy = make_float2(py[0], py[1]),
                 fz = make_float2(pz[0], pz[1]), fp = make_float2(pp[0], pp[1]);
#pragma unroll 16
          for (int k = 0; k < kSub; ++k) {
            const float4 s = sc[base + k];  // -u_j, q_j
            const float2 dx = __fadd2_rn(ax, make_float2(s.x, s.x));
            const float2 dy = __fadd2_rn(ay, make_float2(s.y, s.y));
            const float2 dz = __fadd2_rn(az, make_float2(s.z, s.z));
            const float2 d2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, e2)));
            const float2 rinv = make_float2(rsqrtf(d2.x), rsqrtf(d2.y));
            const float2 qr = __fmul2_rn(make_float2(s.w, s.w), rinv);
            const float2 w = __fmul2_rn(qr, __fmul2_rn(rinv, rinv));
            fx = __ffma2_rn(w, dx, fx);
            fy = __ffma2_rn(w, dy, fy);
            fz = __ffma2_rn(w, dz, fz);
            if (kPhi) fp = __fadd2_rn(fp, qr);
          }
          px[0] = fx.x;
          px[1] = fx.y;
          py[0] = fy.x;
          py[1] = fy.y;
          pz[0] = fz.x;
          pz[1] = fz.y;
          pp[0] = fp.x;
          pp[1] = fp.y;
        }
      }
#pragma unroll
      for (int r = 0; r < kR; ++r) {
        two_sum_fold(ahx[r], alx[r], px[r]);
        two_sum_fold(ahy[r], aly[r], py[r]);
        two_sum_fold(ahz[r], alz[r], pz[r]);
        if (kPhi) two_sum_fold(ahp[r], alp[r], pp[r]);
      }
    }
  }
  if (run_tb >= 0) flush();
}

// Sums the partial runs of each (sorted) target in chunk order in FP64 and
// scatters to the caller's order: F_i = k e q_i / L^2 * sum,
// phi_i = e / L * sum_phi. The runs of target block tb start at chunk 0 and
// at every CTA boundary inside tb's units.
__global__ void allpairs_finalize_kernel(int n, int n_tb, int n_split, int grid, const float4* __restrict__ part,
                                         const uint32_t* __restrict__ perm, const float4* __restrict__ hq,
                                         const double* __restrict__ q, const uint8_t* __restrict__ alive,
                                         double force_coef, double phi_coef, double* __restrict__ fx,
                                         double* __restrict__ fy, double* __restrict__ fz, double* __restrict__ phi) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const long units = static_cast<long>(n_tb) * n_split;
  const int tb = k / (kThreads * kR);
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
    const float4 h = part[(static_cast<size_t>(s) * 2 + 0) * n + k];
    const float4 l = part[(static_cast<size_t>(s) * 2 + 1) * n + k];
    sx += static_cast<double>(h.x) + static_cast<double>(l.x);
    sy += static_cast<double>(h.y) + static_cast<double>(l.y);
    sz += static_cast<double>(h.z) + static_cast<double>(l.z);
    sp += static_cast<double>(h.w) + static_cast<double>(l.w);
  }
  const long i = perm[k];
  // Targets that are dead, neutral or non-finite were staged with q_e = 0.
  const bool live = hq[k].w != 0.0f;
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
  int rc = AMK_OK;
  const int n_tiles = (n + kThreads - 1) / kThreads;

  // ---- Morton order (reused for kResortEvery calls on the context's own set)
  const bool main_set = v.x == c->x.as<double>() && v.n == c->n;
  uint32_t* perm = nullptr;
  bool resort = true;
  if (main_set) {
    AMK_TRY(c->ap_perm.reserve(static_cast<size_t>(n) * sizeof(uint32_t)));
    perm = c->ap_perm.as<uint32_t>();
    resort = c->ap_perm_n != n || c->ap_perm_age >= kResortEvery;
  } else {
    perm = slot<uint32_t>(c, kSlotSorted0, static_cast<size_t>(n), &rc);
    AMK_TRY(rc);
  }
  AMK_TRY(phase_begin(c, AMK_PHASE_STAGE));
  if (resort) {
    unsigned long long* bb = slot<unsigned long long>(c, kSlotCellStart, 8, &rc);
    AMK_TRY(rc);
    uint64_t* keys = slot<uint64_t>(c, kSlotKeysA, n, &rc);
    AMK_TRY(rc);
    uint32_t* vals = slot<uint32_t>(c, kSlotValsA, n, &rc);
    AMK_TRY(rc);
    uint64_t* skeys = slot<uint64_t>(c, kSlotTreeKeys, n, &rc);
    AMK_TRY(rc);
    AMK_CUDA_TRY(cudaMemsetAsync(bb, 0xFF, 6 * sizeof(unsigned long long), c->stream));
    ap_bbox_kernel<<<148, 256, 0, c->stream>>>(v, bb);
    AMK_TRY(check_launch(c, "ap_bbox_kernel"));
    ap_key_kernel<<<(n + 255) / 256, 256, 0, c->stream>>>(v, bb, keys, vals);
    AMK_TRY(check_launch(c, "ap_key_kernel"));
    AMK_TRY(radix_sort_pairs(c, keys, vals, skeys, perm, n, 32));
    if (main_set) {
      c->ap_perm_n = n;
      c->ap_perm_age = 0;
    }
  }
  if (main_set) c->ap_perm_age++;

  // ---- sorted staging + tile boxes
  float4* hq = slot<float4>(c, kSlotSorted1, n, &rc);
  AMK_TRY(rc);
  float4* lo = slot<float4>(c, kSlotSorted2, n, &rc);
  AMK_TRY(rc);
  float4* rel = slot<float4>(c, kSlotTreeAux0, n, &rc);
  AMK_TRY(rc);
  // one box per sub-tile of every staged chunk (the stage kernel's warps past
  // n write empty boxes)
  TileBox* boxes = slot<TileBox>(c, kSlotTreeAux1, static_cast<size_t>(n_tiles) * kSubPerChunk, &rc);
  AMK_TRY(rc);
  const double l = v.length_scale;
  ap_stage_kernel<<<n_tiles, kThreads, 0, c->stream>>>(v, perm, 1.0 / l, hq, lo, rel, boxes);
  AMK_TRY(check_launch(c, "ap_stage_kernel"));
  AMK_TRY(phase_end(c, AMK_PHASE_STAGE));

  // ---- work split: chunks of whole tiles, >= 32 units per CTA
  const int grid_cap = g_num_sms * std::max(1, g_ctas_per_sm[want_phi ? 1 : 0]);
  const int n_tb = (n_tiles + kR - 1) / kR;
  int n_split = std::min(n_tiles, std::max(1, (32 * grid_cap + n_tb - 1) / n_tb));
  const int tiles_per_chunk = (n_tiles + n_split - 1) / n_split;
  n_split = (n_tiles + tiles_per_chunk - 1) / tiles_per_chunk;
  const long units = static_cast<long>(n_tb) * n_split;
  const int grid = static_cast<int>(std::min<long>(units, grid_cap));
  float4* part = slot<float4>(c, kSlotPartial, static_cast<size_t>(n_split) * 2 * n, &rc);
  AMK_TRY(rc);
  // r^2 floor: 1e-30 m^2 (the reference's skip radius), raised to 1e-25 in
  // scaled units so that rinv^3 stays finite in FP32 for any length scale.
  const float eps2 = static_cast<float>(std::max(kMinSquaredDistance / (l * l), 1e-25));

  AMK_TRY(phase_begin(c, AMK_PHASE_ALLPAIRS));
  if (want_phi)
    allpairs_kernel<true><<<grid, kThreads, 0, c->stream>>>(hq, lo, rel, boxes, n, n_tiles, n_tb, n_split,
                                                            tiles_per_chunk, eps2, part);
  else
    allpairs_kernel<false><<<grid, kThreads, 0, c->stream>>>(hq, lo, rel, boxes, n, n_tiles, n_tb, n_split,
                                                             tiles_per_chunk, eps2, part);
  AMK_TRY(check_launch(c, "allpairs_kernel"));
  AMK_TRY(phase_end(c, AMK_PHASE_ALLPAIRS));
  AMK_TRY(phase_begin(c, AMK_PHASE_STAGE));
  allpairs_finalize_kernel<<<(n + 255) / 256, 256, 0, c->stream>>>(
      n, n_tb, n_split, grid, part, perm, hq, v.q, v.alive, kCoulombConstant * kElementaryCharge / (l * l),
      kElementaryCharge / l, v.fx, v.fy, v.fz, v.phi);
  AMK_TRY(check_launch(c, "allpairs_finalize_kernel"));
  AMK_TRY(phase_end(c, AMK_PHASE_STAGE));
  return AMK_OK;
}

}  // namespace amk
