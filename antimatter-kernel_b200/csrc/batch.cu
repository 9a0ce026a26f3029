// Batched multi-instance sweep: many independent trap instances of uneven
// population stepped together. The reference runs one instance per process
// (antimatter-kernel.cc:153-162 is its step loop); a sweep over temperature,
// field and population is many such runs. Here the instances share one
// particle set: instance i owns [offset[i], offset[i+1]) and has its own
// trap, time step, cooling, annihilation and Coulomb parameters.
//
// One batched step is:
//   * all-pairs instances: ONE persistent launch over (instance, 128-target
//     block) units taken from a queue ordered by cost (largest instances
//     first). Double-float pair differences, FP32 pair math, TwoSum-folded
//     tile sums: each target's result depends only on its own instance, in
//     a fixed order, so it is deterministic and independent of the batch;
//   * cutoff, Barnes-Hut and FMM instances: the single-instance solver on
//     the instance's view;
//   * one push kernel (Boris + cooling, per-instance parameters, the same
//     per-particle code as the single-instance push);
//   * annihilation: one cell list whose keys start with the instance id (so
//     contacts never cross instances), one contact kernel, and one matching
//     kernel that reads the contact count on the device.
// When no instance uses Barnes-Hut or the FMM a step has no host
// synchronisation, and chunks of steps are captured in a CUDA graph and
// replayed. Random streams use the instance's seed and the particle's index
// within its instance, so an instance gives the same result in any batch.
#include <algorithm>
#include <cmath>
#include <vector>

#include "amk_internal.cuh"
#include "contacts.cuh"
#include "push.cuh"

namespace amk {

int push_range(amk_ctx* c, const PushParams& P, long begin, long end, bool stagger, uint64_t step_index);

namespace {

constexpr int kBT = 128;           // threads per all-pairs CTA = sources per staged chunk
constexpr int kBR = 2;             // targets per thread: a warp owns 64 consecutive targets
constexpr int kBUnit = kBT * kBR;  // targets per work unit
constexpr int kBSub = 32;          // particles per sub-tile (box granularity)
constexpr int kBSubPerChunk = kBT / kBSub;
constexpr int kBSubPerUnit = kBUnit / kBSub;
constexpr float kBNearFactor = 0.25f;
constexpr int kGridBits = 10;      // annihilation cells per axis per instance: 2^10
constexpr int kInstBits = 9;       // up to 512 instances
constexpr int kMaxInstances = 1 << kInstBits;
static_assert(kMaxInstances == AMK_BATCH_MAX_INSTANCES, "instance key bits");
constexpr double kGridMax = (1 << kGridBits) - 1;

struct InstanceDev {
  PushParams push;
  double contact_radius, probability;  // annihilation
  double inv_l;                        // 1 / length scale (a power of two)
  double origin[3], inv_cell;          // annihilation grid (cells >= the contact radius)
  double inv_sort_cell;                // all-pairs ordering grid: 1022 cells over the same cube
  long offset, count;
  long sub0;                           // first all-pairs sub-tile slot of the instance
  int annihilation;
  uint32_t seed;
};

__device__ __forceinline__ void fold(float& hi, float& lo, float p) {
  const float s = hi + p;
  const float bp = s - hi;
  lo += (hi - (s - bp)) + (p - bp);
  hi = s;
}

__global__ void batch_local_ids_kernel(long n, const uint16_t* __restrict__ inst_of,
                                       const InstanceDev* __restrict__ inst, uint32_t* __restrict__ ids) {
  const long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  ids[i] = static_cast<uint32_t>(i - inst[inst_of[i]].offset);
}

// ---------------------------------------------------------------- all-pairs
// Per step, every particle gets the key (instance << 30 | 30-bit Morton cell
// in its instance's grid); usable particles (alive, charged, finite) sort
// before the others of their instance. The stable sort keeps each instance
// inside its own [offset, offset + count) range, so sorted position k holds
// a particle of the same instance as original index k. Every 32 sorted
// positions of an instance form a sub-tile with a box; a warp owns 64
// consecutive targets and decides near/far per 32-source sub-tile, uniform
// across the warp: sub-tiles farther than a quarter of the summed
// half-extent norms use FP32 offsets from the sub-tile centre (12 FP32 ops
// per pair, relative error <= 7 eps of |r|), the others exact double-float
// differences (18 ops per pair; the self pair gives exactly 0).
__global__ void batch_sort_key_kernel(long n, const double* __restrict__ x, const double* __restrict__ y,
                                      const double* __restrict__ z, const double* __restrict__ q,
                                      const uint8_t* __restrict__ alive, const uint16_t* __restrict__ inst_of,
                                      const InstanceDev* __restrict__ inst, uint64_t* __restrict__ keys,
                                      uint32_t* __restrict__ vals) {
  const long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  vals[i] = static_cast<uint32_t>(i);
  const uint16_t k = inst_of[i];
  const InstanceDev& I = inst[k];
  const uint64_t prefix = static_cast<uint64_t>(k) << 30;
  if (!alive[i] || q[i] == 0.0 || !isfinite(x[i]) || !isfinite(y[i]) || !isfinite(z[i])) {
    keys[i] = prefix | ((1ull << 30) - 1ull);
    return;
  }
  const double p[3] = {x[i], y[i], z[i]};
  uint32_t c[3];
#pragma unroll
  for (int d = 0; d < 3; ++d)
    c[d] = static_cast<uint32_t>(fmin(fmax(floor((p[d] - I.origin[d]) * I.inv_sort_cell), 0.0), 1022.0));
  keys[i] = prefix | morton3_21(c[0], c[1], c[2]);
}

struct TileBox {
  float4 c;   // centre (scaled, hi part); w = 1 when the tile has usable particles
  float4 cl;  // centre, lo part
  float4 h;   // half-extents (rounded up); w = |h|
};

// One CTA of 256 threads per all-pairs unit (256 sorted positions of one
// instance); each warp stages its 32-position sub-tile: double-float
// positions, offsets from the sub-tile centre and the sub-tile box. Slots of
// sub-tiles past the instance's end receive empty boxes.
__global__ void __launch_bounds__(kBUnit)
batch_tile_stage_kernel(const int2* __restrict__ units, const InstanceDev* __restrict__ inst,
                        const uint32_t* __restrict__ perm, const double* __restrict__ x,
                        const double* __restrict__ y, const double* __restrict__ z, const double* __restrict__ q,
                        const uint8_t* __restrict__ alive, float4* __restrict__ hq, float4* __restrict__ lo,
                        float4* __restrict__ rel, TileBox* __restrict__ boxes) {
  const int2 un = units[blockIdx.x];
  const InstanceDev& I = inst[un.x];
  const long e = I.offset + I.count;
  const long k = I.offset + static_cast<long>(un.y) * kBUnit + threadIdx.x;
  double xs = 0.0, ys = 0.0, zs = 0.0, qe = 0.0;
  bool ok = false;
  if (k < e) {
    const long i = perm[k];
    xs = x[i] * I.inv_l;
    ys = y[i] * I.inv_l;
    zs = z[i] * I.inv_l;
    ok = alive[i] && q[i] != 0.0 && isfinite(xs) && isfinite(ys) && isfinite(zs);
    qe = q[i] / kElementaryCharge;
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
    h = make_float4(__double2float_rn(xs), __double2float_rn(ys), __double2float_rn(zs), __double2float_rn(qe));
    l = make_float4(__double2float_rn(xs - static_cast<double>(h.x)), __double2float_rn(ys - static_cast<double>(h.y)),
                    __double2float_rn(zs - static_cast<double>(h.z)), 0.f);
    u = make_float4(-__double2float_rn(xs - cx), -__double2float_rn(ys - cy), -__double2float_rn(zs - cz),
                    h.w);  // negated offsets: the far loop adds them
  }
  if (k < e) {
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
    boxes[I.sub0 + static_cast<long>(un.y) * kBSubPerUnit + (threadIdx.x >> 5)] = b;
  }
}

// Persistent all-pairs over (instance, 256-target block) units taken from a
// queue (`queue` zeroed before every launch): F_i = k e q_i / L^2 * sum_j q_j
// (r_i - r_j) / |r_i - r_j|^3 in scaled units, written to the particle's
// original index. Warp w of a unit owns targets [64 w, 64 w + 64) of the
// block: lane l holds +l (r = 0) and +32+l (r = 1).
__global__ void __launch_bounds__(kBT, 4)
batch_allpairs_kernel(const int2* __restrict__ units, int n_units, const InstanceDev* __restrict__ inst,
                      const float4* __restrict__ hq, const float4* __restrict__ lo, const float4* __restrict__ rel,
                      const TileBox* __restrict__ boxes, const uint32_t* __restrict__ perm,
                      const double* __restrict__ q, double* __restrict__ fx, double* __restrict__ fy,
                      double* __restrict__ fz, int* __restrict__ queue) {
  __shared__ float4 sa[kBT], sb[kBT], sc[kBT];
  __shared__ TileBox sbox[kBSubPerChunk];
  __shared__ float4 swc[kBT / 32], swh[kBT / 32];
  __shared__ int s_unit;
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  for (;;) {
    __syncthreads();  // the previous unit's readers are done with s_unit and the buffers
    if (tid == 0) s_unit = atomicAdd(queue, 1);
    __syncthreads();
    const int u = s_unit;
    if (u >= n_units) return;
    const int2 un = units[u];
    const long b = inst[un.x].offset, e = b + inst[un.x].count;
    const long sub0 = inst[un.x].sub0;
    const long n_sub = (e - b + kBSub - 1) / kBSub;
    const double inv_l = inst[un.x].inv_l;
    const float eps2 = static_cast<float>(fmax(kMinSquaredDistance * inv_l * inv_l, 1e-25));
    const long kw = b + static_cast<long>(un.y) * kBUnit + warp * (kBSub * kBR);  // the warp's first target
    float tx[kBR], ty[kBR], tz[kBR], ux[kBR], uy[kBR], uz[kBR];
    float ahx[kBR], ahy[kBR], ahz[kBR], alx[kBR], aly[kBR], alz[kBR];
    bool live_t[kBR];
#pragma unroll
    for (int r = 0; r < kBR; ++r) {
      const long k = kw + r * kBSub + lane;
      float4 h = make_float4(0.f, 0.f, 0.f, 0.f), l = h;
      if (k < e) {
        h = hq[k];
        l = lo[k];
      }
      live_t[r] = h.w != 0.f;
      tx[r] = h.x; ty[r] = h.y; tz[r] = h.z;
      ux[r] = l.x; uy[r] = l.y; uz[r] = l.z;
      ahx[r] = ahy[r] = ahz[r] = alx[r] = aly[r] = alz[r] = 0.f;
    }
    // union box of the warp's two target sub-tiles
    const long s_loc = (kw - b) / kBSub;
    TileBox b0 = s_loc < n_sub ? boxes[sub0 + s_loc] : TileBox{};
    TileBox b1 = s_loc + 1 < n_sub ? boxes[sub0 + s_loc + 1] : TileBox{};
    if (b1.c.w == 0.f) b1 = b0;
    if (b0.c.w == 0.f) b0 = b1;
    const bool warp_live = b0.c.w != 0.f;
    if (lane == 0) {
      const float lx = fminf(b0.c.x - b0.h.x, b1.c.x - b1.h.x), hx = fmaxf(b0.c.x + b0.h.x, b1.c.x + b1.h.x);
      const float ly = fminf(b0.c.y - b0.h.y, b1.c.y - b1.h.y), hy = fmaxf(b0.c.y + b0.h.y, b1.c.y + b1.h.y);
      const float lz = fminf(b0.c.z - b0.h.z, b1.c.z - b1.h.z), hz = fmaxf(b0.c.z + b0.h.z, b1.c.z + b1.h.z);
      float4 wh = make_float4(0.5001f * (hx - lx), 0.5001f * (hy - ly), 0.5001f * (hz - lz), 0.f);
      wh.w = 1.0001f * sqrtf(wh.x * wh.x + wh.y * wh.y + wh.z * wh.z);
      swc[warp] = make_float4(0.5f * (lx + hx), 0.5f * (ly + hy), 0.5f * (lz + hz), 0.f);
      swh[warp] = wh;
    }
    for (long c0 = b; c0 < e; c0 += kBT) {
      const long j = c0 + tid;
      __syncthreads();  // the previous chunk's readers are done with the buffers
      if (j < e) {
        sa[tid] = hq[j];
        sb[tid] = lo[j];
        sc[tid] = rel[j];
      } else {
        sa[tid] = sb[tid] = sc[tid] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
      if (tid < kBSubPerChunk) {
        const long s = (c0 - b) / kBSub + tid;
        sbox[tid] = s < n_sub ? boxes[sub0 + s] : TileBox{};
      }
      __syncthreads();
      if (!warp_live) continue;  // no usable target in this warp (uniform)
      const float4 wc = swc[warp], wh = swh[warp];
      float px[kBR], py[kBR], pz[kBR];
#pragma unroll
      for (int r = 0; r < kBR; ++r) px[r] = py[r] = pz[r] = 0.f;
      for (int qd = 0; qd < kBSubPerChunk; ++qd) {
        const TileBox sbx = sbox[qd];
        if (sbx.c.w == 0.f) continue;  // no usable sources (uniform)
        const float gx = fmaxf(fabsf(wc.x - sbx.c.x) - (wh.x + sbx.h.x), 0.f);
        const float gy = fmaxf(fabsf(wc.y - sbx.c.y) - (wh.y + sbx.h.y), 0.f);
        const float gz = fmaxf(fabsf(wc.z - sbx.c.z) - (wh.z + sbx.h.z), 0.f);
        const float lim = kBNearFactor * (wh.w + sbx.h.w);
        const int base = qd * kBSub;
        if (gx * gx + gy * gy + gz * gz <= lim * lim) {
          // near: double-float differences for the lane's two targets in
          // packed FP32x2 operations (t - s as fma(s, -1, t): the scalar
          // form's rounding, so the sums are bit-identical to it)
          const float2 m1 = make_float2(-1.f, -1.f), e2 = make_float2(eps2, eps2);
          const float2 thx = make_float2(tx[0], tx[1]), thy = make_float2(ty[0], ty[1]),
                       thz = make_float2(tz[0], tz[1]);
          const float2 tlx = make_float2(ux[0], ux[1]), tly = make_float2(uy[0], uy[1]),
                       tlz = make_float2(uz[0], uz[1]);
          float2 fx2 = make_float2(px[0], px[1]), fy2 = make_float2(py[0], py[1]), fz2 = make_float2(pz[0], pz[1]);
#pragma unroll 8
          for (int k = 0; k < kBSub; ++k) {
            const float4 sh = sa[base + k], sl = sb[base + k];
            const float2 dx = __fadd2_rn(__ffma2_rn(make_float2(sh.x, sh.x), m1, thx),
                                         __ffma2_rn(make_float2(sl.x, sl.x), m1, tlx));
            const float2 dy = __fadd2_rn(__ffma2_rn(make_float2(sh.y, sh.y), m1, thy),
                                         __ffma2_rn(make_float2(sl.y, sl.y), m1, tly));
            const float2 dz = __fadd2_rn(__ffma2_rn(make_float2(sh.z, sh.z), m1, thz),
                                         __ffma2_rn(make_float2(sl.z, sl.z), m1, tlz));
            const float2 d2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, e2)));
            const float2 rinv = make_float2(rsqrtf(d2.x), rsqrtf(d2.y));
            const float2 w = __fmul2_rn(__fmul2_rn(make_float2(sh.w, sh.w), rinv), __fmul2_rn(rinv, rinv));
            fx2 = __ffma2_rn(w, dx, fx2);
            fy2 = __ffma2_rn(w, dy, fy2);
            fz2 = __ffma2_rn(w, dz, fz2);
          }
          px[0] = fx2.x;
          px[1] = fx2.y;
          py[0] = fy2.x;
          py[1] = fy2.y;
          pz[0] = fz2.x;
          pz[1] = fz2.y;
        } else {
          // far: a lane's two targets in the halves of packed FP32x2
          // operations (same operations and association as the scalar form)
          static_assert(kBR == 2, "packed far path holds two targets per lane");
          float2 ax, ay, az;
          ax.x = (tx[0] - sbx.c.x) + (ux[0] - sbx.cl.x);
          ax.y = (tx[1] - sbx.c.x) + (ux[1] - sbx.cl.x);
          ay.x = (ty[0] - sbx.c.y) + (uy[0] - sbx.cl.y);
          ay.y = (ty[1] - sbx.c.y) + (uy[1] - sbx.cl.y);
          az.x = (tz[0] - sbx.c.z) + (uz[0] - sbx.cl.z);
          az.y = (tz[1] - sbx.c.z) + (uz[1] - sbx.cl.z);
          const float2 e2 = make_float2(eps2, eps2);
          float2 fx2 = make_float2(px[0], px[1]), fy2 = make_float2(py[0], py[1]), fz2 = make_float2(pz[0], pz[1]);
#pragma unroll 16
          for (int k = 0; k < kBSub; ++k) {
            const float4 sr = sc[base + k];  // -u_j, q_j
            const float2 dx = __fadd2_rn(ax, make_float2(sr.x, sr.x));
            const float2 dy = __fadd2_rn(ay, make_float2(sr.y, sr.y));
            const float2 dz = __fadd2_rn(az, make_float2(sr.z, sr.z));
            const float2 d2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, e2)));
            const float2 rinv = make_float2(rsqrtf(d2.x), rsqrtf(d2.y));
            const float2 w = __fmul2_rn(__fmul2_rn(make_float2(sr.w, sr.w), rinv), __fmul2_rn(rinv, rinv));
            fx2 = __ffma2_rn(w, dx, fx2);
            fy2 = __ffma2_rn(w, dy, fy2);
            fz2 = __ffma2_rn(w, dz, fz2);
          }
          px[0] = fx2.x;
          px[1] = fx2.y;
          py[0] = fy2.x;
          py[1] = fy2.y;
          pz[0] = fz2.x;
          pz[1] = fz2.y;
        }
      }
#pragma unroll
      for (int r = 0; r < kBR; ++r) {
        fold(ahx[r], alx[r], px[r]);
        fold(ahy[r], aly[r], py[r]);
        fold(ahz[r], alz[r], pz[r]);
      }
    }
#pragma unroll
    for (int r = 0; r < kBR; ++r) {
      const long k = kw + r * kBSub + lane;
      if (k < e) {
        const long i = perm[k];
        const double coef = live_t[r] ? kCoulombConstant * kElementaryCharge * inv_l * inv_l * q[i] : 0.0;
        fx[i] = coef * (static_cast<double>(ahx[r]) + static_cast<double>(alx[r]));
        fy[i] = coef * (static_cast<double>(ahy[r]) + static_cast<double>(aly[r]));
        fz[i] = coef * (static_cast<double>(ahz[r]) + static_cast<double>(alz[r]));
      }
    }
  }
}

// LorentzForce + CyclotronCooling with each particle's instance parameters;
// the step index is read on the device so that graph replays advance it.
__global__ void __launch_bounds__(256)
batch_push_kernel(long n, double* __restrict__ x, double* __restrict__ y, double* __restrict__ z,
                  double* __restrict__ vx, double* __restrict__ vy, double* __restrict__ vz, double* __restrict__ fx,
                  double* __restrict__ fy, double* __restrict__ fz, const double* __restrict__ q,
                  const double* __restrict__ m, const uint8_t* __restrict__ alive, const uint32_t* __restrict__ ids,
                  const uint16_t* __restrict__ inst_of, const InstanceDev* __restrict__ inst,
                  const unsigned long long* __restrict__ step_dev, int stagger) {
  const long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const PushParams P = inst[inst_of[i]].push;
  push_particle(i, x, y, z, vx, vy, vz, fx, fy, fz, q, m, alive, P, stagger, *step_dev, ids[i]);
}

// Step counter (advanced at the start of every batched step) and the
// queue / contact-count reset.
__global__ void batch_begin_step_kernel(unsigned long long* step_dev, int* queue, unsigned long long* contacts) {
  *step_dev += 1ull;
  *queue = 0;
  contacts[0] = 0;
}

__device__ __forceinline__ void batch_cell(const InstanceDev& I, double x, double y, double z, uint32_t c[3]) {
  const double p[3] = {x, y, z};
#pragma unroll
  for (int d = 0; d < 3; ++d)
    c[d] = static_cast<uint32_t>(fmin(fmax(floor((p[d] - I.origin[d]) * I.inv_cell), 0.0), kGridMax));
}

__device__ __forceinline__ bool has_partner(int s) {
  return s == AMK_POSITRON || s == AMK_ELECTRON || s == AMK_PROTON || s == AMK_ANTIPROTON;
}

// Annihilation cell keys: instance id above a 30-bit Morton cell index
// (10 bits per axis); particles that cannot annihilate sort last. Cells
// are clamped to the instance's grid, which keeps neighbours within one
// cell of each other, so a particle outside the grid is still found.
__global__ void batch_cell_key_kernel(long n, const double* __restrict__ x, const double* __restrict__ y,
                                      const double* __restrict__ z, const uint8_t* __restrict__ alive,
                                      const uint8_t* __restrict__ species, const uint16_t* __restrict__ inst_of,
                                      const InstanceDev* __restrict__ inst, uint64_t* __restrict__ keys,
                                      uint32_t* __restrict__ vals) {
  const long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  vals[i] = static_cast<uint32_t>(i);
  const InstanceDev& I = inst[inst_of[i]];
  if (!alive[i] || !I.annihilation || !has_partner(species[i]) || !isfinite(x[i]) || !isfinite(y[i]) ||
      !isfinite(z[i])) {
    keys[i] = ~0ull;
    return;
  }
  uint32_t c[3];
  batch_cell(I, x[i], y[i], z[i], c);
  keys[i] = (static_cast<uint64_t>(inst_of[i]) << (3 * kGridBits)) | morton3_21(c[0], c[1], c[2]);
}

__device__ __forceinline__ long lower_bound_key(const uint64_t* keys, long n, uint64_t k) {
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

// Directed contacts owner -> partner within the contact radius whose Philox
// draw is below the instance's probability (annihilation.cc:21-61 made
// deterministic; the same rule as the single-instance contact kernel).
__global__ void __launch_bounds__(128)
batch_contact_kernel(long n, const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z,
                     const uint8_t* __restrict__ species, const uint32_t* __restrict__ ids,
                     const uint16_t* __restrict__ inst_of, const InstanceDev* __restrict__ inst,
                     const uint64_t* __restrict__ skeys, const uint32_t* __restrict__ sidx,
                     const unsigned long long* __restrict__ step_dev, Contact* __restrict__ out,
                     unsigned long long* count, long cap) {
  const long s = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  if (s >= n || skeys[s] == ~0ull) return;
  const long i = sidx[s];
  const uint64_t prefix = skeys[s] & ~((1ull << (3 * kGridBits)) - 1ull);
  const InstanceDev& I = inst[inst_of[i]];
  const int si = species[i];
  const double xi = x[i], yi = y[i], zi = z[i];
  uint32_t c[3];
  batch_cell(I, xi, yi, zi, c);
  const double rc2 = I.contact_radius * I.contact_radius;
  const double prob = I.probability;
  const uint32_t seed = I.seed;
  const uint64_t st = *step_dev;
  for (int dz = -1; dz <= 1; ++dz) {
    const int cz = static_cast<int>(c[2]) + dz;
    if (cz < 0 || cz > static_cast<int>(kGridMax)) continue;
    for (int dy = -1; dy <= 1; ++dy) {
      const int cy = static_cast<int>(c[1]) + dy;
      if (cy < 0 || cy > static_cast<int>(kGridMax)) continue;
      for (int dx = -1; dx <= 1; ++dx) {
        const int cx = static_cast<int>(c[0]) + dx;
        if (cx < 0 || cx > static_cast<int>(kGridMax)) continue;
        const uint64_t key = prefix | morton3_21(cx, cy, cz);
        for (long k = lower_bound_key(skeys, n, key); k < n && skeys[k] == key; ++k) {
          const long j = sidx[k];
          if (j == i) continue;
          const int sj = species[j];
          const bool pair = (si == AMK_ANTIPROTON && sj == AMK_PROTON) || (si == AMK_PROTON && sj == AMK_ANTIPROTON) ||
                            (si == AMK_POSITRON && sj == AMK_ELECTRON) || (si == AMK_ELECTRON && sj == AMK_POSITRON);
          if (!pair) continue;
          const double rx = xi - x[j], ry = yi - y[j], rz = zi - z[j];
          const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(rx, rx), __dmul_rn(ry, ry)), __dmul_rn(rz, rz));
          if (!(d2 < rc2)) continue;
          const Philox4 w = philox4x32(seed, kTagAnnihilation, ids[i], ids[j], static_cast<uint32_t>(st),
                                       static_cast<uint32_t>(st >> 32));
          if (!(u01(w.w[0]) < prob)) continue;
          const unsigned long long slot_i = atomicAdd(count, 1ull);
          if (static_cast<long>(slot_i) < cap) {
            Contact e;
            e.a = static_cast<uint32_t>(i);
            e.b = static_cast<uint32_t>(j);
            // instance id above the local ids: within an instance the greedy
            // order is the single-instance order, and instances are disjoint
            e.prio = (static_cast<uint64_t>(inst_of[i]) << 54) | (static_cast<uint64_t>(ids[i]) << 27) | ids[j];
            out[slot_i] = e;
          }
        }
      }
    }
  }
}

// Records a contact-buffer overflow in the sticky status word and in the
// per-call word.
__global__ void batch_overflow_kernel(const unsigned long long* contacts, long cap, unsigned long long* status) {
  if (contacts[0] > static_cast<unsigned long long>(cap)) {
    status[0] = 1ull;
    status[1] = 1ull;
  }
}

// Kinetic energy, trap potential energy and live count of each instance:
// one CTA per instance, fixed reduction order (energy_analysis.cc:84-125
// per instance; trap potential q U (2 z^2 - rho^2) / (4 d^2),
// penning_trap.cc:35-43).
__global__ void __launch_bounds__(256)
batch_energy_kernel(const InstanceDev* __restrict__ inst, const double* __restrict__ x, const double* __restrict__ y,
                    const double* __restrict__ z, const double* __restrict__ vx, const double* __restrict__ vy,
                    const double* __restrict__ vz, const double* __restrict__ q, const double* __restrict__ m,
                    const uint8_t* __restrict__ alive, double* __restrict__ out) {
  __shared__ double s[3][256];
  const InstanceDev& I = inst[blockIdx.x];
  const double trap_coef = 0.5 * I.push.radial;  // U / (4 d^2)
  double ke = 0.0, pe = 0.0, cnt = 0.0;
  for (long i = I.offset + threadIdx.x; i < I.offset + I.count; i += 256) {
    if (!alive[i]) continue;
    ke += 0.5 * m[i] * (vx[i] * vx[i] + vy[i] * vy[i] + vz[i] * vz[i]);
    pe += q[i] * (trap_coef * (2.0 * z[i] * z[i] - (x[i] * x[i] + y[i] * y[i])));
    cnt += 1.0;
  }
  s[0][threadIdx.x] = ke;
  s[1][threadIdx.x] = pe;
  s[2][threadIdx.x] = cnt;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int k = 0; k < 3; ++k) s[k][threadIdx.x] += s[k][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 3) out[3 * blockIdx.x + threadIdx.x] = s[threadIdx.x][0];
}

__global__ void batch_alive_count_kernel(long n, const uint8_t* __restrict__ alive,
                                         const uint16_t* __restrict__ inst_of, unsigned long long* counts) {
  const long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  if (i >= n || !alive[i]) return;
  atomicAdd(&counts[inst_of[i]], 1ull);
}

}  // namespace

struct Batch {
  int n_inst = 0;
  std::vector<amk_params> params;
  std::vector<long> offsets;
  std::vector<double> scale;
  std::vector<PushParams> push;
  std::vector<int> solver_instances;  // instances with a per-instance solver call
  std::vector<int> leaf;              // leaf capacity of each instance's tree solver
  bool any_annihilation = false;
  bool graphable = true;
  DevBuf inst, inst_of, units, counters, contacts, best, flags, keys, vals, skeys, sidx;
  DevBuf perm, rel, boxes;  // all-pairs order, tile offsets, tile boxes
  long n_units = 0;
  long contact_cap = 0;
  unsigned long long max_contacts = 0;  // largest contact count seen by a synchronised step
  int grid = 0;
  uint64_t step = 0;  // host mirror of the device step counter
  bool warm = false;  // one uncaptured step done (scratch reserved)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int graph_steps = 0;
  // energy time-centring history per instance (EnergyHistory, energy_analysis.h:23-28)
  std::vector<double> prev_trap, prev_coulomb;
  bool energy_has_previous = false;
  long graph_launches = 0;
  ~Batch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
  }
  // counters (64-bit words): [0] queue head (int), [1] step, [2] contact
  // count, [3..4] match result, [5] sticky overflow status, [6] overflow
  // inside the current call's graph replays
  int* queue() const { return counters.as<int>(); }
  unsigned long long* step_dev() const { return counters.as<unsigned long long>() + 1; }
  unsigned long long* contact_count() const { return counters.as<unsigned long long>() + 2; }
  unsigned long long* match_result() const { return counters.as<unsigned long long>() + 3; }
  unsigned long long* overflow() const { return counters.as<unsigned long long>() + 5; }
  unsigned long long* call_overflow() const { return counters.as<unsigned long long>() + 6; }
  void drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
    graph_steps = 0;
  }
  // Contact buffer of at least `cap` entries (drops a captured graph, which
  // holds the old addresses).
  int reserve_contacts(long cap, long n) {
    if (cap <= contact_cap) return AMK_OK;
    drop_graph();
    AMK_TRY(contacts.reserve(static_cast<size_t>(cap) * sizeof(Contact)));
    AMK_TRY(flags.reserve(static_cast<size_t>(std::max<long>(n, 1)) + static_cast<size_t>(cap)));
    contact_cap = cap;
    return AMK_OK;
  }
};

void batch_destroy(amk_ctx* c) {
  delete c->batch;
  c->batch = nullptr;
}

namespace {

View instance_view(amk_ctx* c, const Batch& B, int i) {
  View v = main_view(c);
  const long off = B.offsets[i];
  v.n = B.offsets[i + 1] - off;
  v.x += off;
  v.y += off;
  v.z += off;
  v.q += off;
  v.alive += off;
  v.hq += off;
  v.lo += off;
  v.fx += off;
  v.fy += off;
  v.fz += off;
  v.phi = nullptr;
  v.length_scale = B.scale[i];
  return v;
}

// The single-instance solver of instance i on its view.
int instance_coulomb(amk_ctx* c, const Batch& B, int i) {
  const amk_params& p = B.params[i];
  View v = instance_view(c, B, i);
  if (v.n == 0 || !p.coulomb_forces_enabled) return AMK_OK;
  switch (p.coulomb_method) {
    case AMK_METHOD_ALLPAIRS: return allpairs_forces(c, v);
    case AMK_METHOD_STANDARD: return cutoff_forces(c, v, p.cutoff_radius, nullptr);
    case AMK_METHOD_BARNES_HUT: return barnes_hut_forces(c, v, p.barnes_hut_theta, B.leaf[i]);
    case AMK_METHOD_FAST_MULTIPOLE:
      return fmm_forces(c, v, static_cast<int>(p.fast_multipole_order), p.fast_multipole_theta, B.leaf[i], false,
                        nullptr);
    default: return fail(AMK_ERR_INVALID, "unknown coulomb method %d", p.coulomb_method);
  }
}

// `sync`: read the contact count back and enlarge the buffer and redo the
// search when it overflowed (not possible inside a graph capture, where an
// overflow is only recorded).
int batch_annihilate(amk_ctx* c, Batch& B, bool sync) {
  const long n = c->n;
  const unsigned gb = static_cast<unsigned>((n + 255) / 256);
  AMK_TRY(phase_begin(c, AMK_PHASE_ANNIHILATION));
  batch_cell_key_kernel<<<gb, 256, 0, c->stream>>>(n, c->x.as<double>(), c->y.as<double>(), c->z.as<double>(),
                                                   c->alive.as<uint8_t>(), c->species.as<uint8_t>(),
                                                   B.inst_of.as<uint16_t>(), B.inst.as<InstanceDev>(),
                                                   B.keys.as<uint64_t>(), B.vals.as<uint32_t>());
  AMK_TRY(check_launch(c, "batch_cell_key_kernel"));
  AMK_TRY(radix_sort_pairs(c, B.keys.as<uint64_t>(), B.vals.as<uint32_t>(), B.skeys.as<uint64_t>(),
                           B.sidx.as<uint32_t>(), n, kInstBits + 3 * kGridBits));
  for (int attempt = 0; attempt < 2; ++attempt) {
    batch_contact_kernel<<<static_cast<unsigned>((n + 127) / 128), 128, 0, c->stream>>>(
        n, c->x.as<double>(), c->y.as<double>(), c->z.as<double>(), c->species.as<uint8_t>(),
        c->ids.as<uint32_t>(), B.inst_of.as<uint16_t>(), B.inst.as<InstanceDev>(), B.skeys.as<uint64_t>(),
        B.sidx.as<uint32_t>(), B.step_dev(), B.contacts.as<Contact>(), B.contact_count(), B.contact_cap);
    AMK_TRY(check_launch(c, "batch_contact_kernel"));
    if (!sync) break;
    unsigned long long m = 0;
    AMK_CUDA_TRY(cudaMemcpyAsync(&m, B.contact_count(), sizeof(m), cudaMemcpyDeviceToHost, c->stream));
    AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
    B.max_contacts = std::max(B.max_contacts, m);
    if (m <= static_cast<unsigned long long>(B.contact_cap)) break;
    AMK_TRY(B.reserve_contacts(static_cast<long>(m + m / 4 + 65536), n));
    AMK_CUDA_TRY(cudaMemsetAsync(B.contact_count(), 0, sizeof(unsigned long long), c->stream));
  }
  unsigned long long* best = B.best.as<unsigned long long>();
  AMK_TRY(queue_matching(c, c->stream, B.contacts.as<Contact>(), B.contact_cap, B.contact_count(), best, best + n,
                         B.flags.as<uint8_t>(), B.flags.as<uint8_t>() + n, c->alive.as<uint8_t>(),
                         reinterpret_cast<MatchState*>(best + 2 * n), B.match_result()));
  batch_overflow_kernel<<<1, 1, 0, c->stream>>>(B.contact_count(), B.contact_cap, B.overflow());
  AMK_TRY(check_launch(c, "batch_overflow_kernel"));
  return phase_end(c, AMK_PHASE_ANNIHILATION);
}

// Coulomb forces of every instance into the context's force arrays.
int batch_coulomb(amk_ctx* c, Batch& B) {
  const long n = c->n;
  if (B.n_units > 0) {
    AMK_TRY(phase_begin(c, AMK_PHASE_STAGE));
    batch_sort_key_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, c->stream>>>(
        n, c->x.as<double>(), c->y.as<double>(), c->z.as<double>(), c->q.as<double>(), c->alive.as<uint8_t>(),
        B.inst_of.as<uint16_t>(), B.inst.as<InstanceDev>(), B.keys.as<uint64_t>(), B.vals.as<uint32_t>());
    AMK_TRY(check_launch(c, "batch_sort_key_kernel"));
    AMK_TRY(radix_sort_pairs(c, B.keys.as<uint64_t>(), B.vals.as<uint32_t>(), B.skeys.as<uint64_t>(),
                             B.perm.as<uint32_t>(), n, kInstBits + 30));
    batch_tile_stage_kernel<<<static_cast<unsigned>(B.n_units), kBUnit, 0, c->stream>>>(
        B.units.as<int2>(), B.inst.as<InstanceDev>(), B.perm.as<uint32_t>(), c->x.as<double>(), c->y.as<double>(),
        c->z.as<double>(), c->q.as<double>(), c->alive.as<uint8_t>(), c->hq.as<float4>(), c->lo.as<float4>(),
        B.rel.as<float4>(), B.boxes.as<TileBox>());
    AMK_TRY(check_launch(c, "batch_tile_stage_kernel"));
    AMK_TRY(phase_end(c, AMK_PHASE_STAGE));
    AMK_TRY(phase_begin(c, AMK_PHASE_ALLPAIRS));
    batch_allpairs_kernel<<<B.grid, kBT, 0, c->stream>>>(
        B.units.as<int2>(), static_cast<int>(B.n_units), B.inst.as<InstanceDev>(), c->hq.as<float4>(),
        c->lo.as<float4>(), B.rel.as<float4>(), B.boxes.as<TileBox>(), B.perm.as<uint32_t>(), c->q.as<double>(),
        c->fx.as<double>(), c->fy.as<double>(), c->fz.as<double>(), B.queue());
    AMK_TRY(check_launch(c, "batch_allpairs_kernel"));
    AMK_TRY(phase_end(c, AMK_PHASE_ALLPAIRS));
  }
  for (int i : B.solver_instances) AMK_TRY(instance_coulomb(c, B, i));
  return AMK_OK;
}

// One batched step; `sync` = false (graph capture) runs it without host
// synchronisation, which needs every instance's solver to run without
// (all-pairs, cutoff).
int batch_step_once(amk_ctx* c, Batch& B, bool stagger, bool sync) {
  const long n = c->n;
  batch_begin_step_kernel<<<1, 1, 0, c->stream>>>(B.step_dev(), B.queue(), B.contact_count());
  AMK_TRY(check_launch(c, "batch_begin_step_kernel"));
  if (n == 0) return AMK_OK;
  AMK_TRY(batch_coulomb(c, B));
  AMK_TRY(phase_begin(c, AMK_PHASE_PUSH));
  batch_push_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, c->stream>>>(
      n, c->x.as<double>(), c->y.as<double>(), c->z.as<double>(), c->vx.as<double>(), c->vy.as<double>(),
      c->vz.as<double>(), c->fx.as<double>(), c->fy.as<double>(), c->fz.as<double>(), c->q.as<double>(),
      c->m.as<double>(), c->alive.as<uint8_t>(), c->ids.as<uint32_t>(), B.inst_of.as<uint16_t>(),
      B.inst.as<InstanceDev>(), B.step_dev(), stagger ? 1 : 0);
  AMK_TRY(check_launch(c, "batch_push_kernel"));
  AMK_TRY(phase_end(c, AMK_PHASE_PUSH));
  if (B.any_annihilation) AMK_TRY(batch_annihilate(c, B, sync));
  return AMK_OK;
}

// The same step with every instance run on its own, one after the other,
// through the single-instance kernels (solver on the view, push on the
// range, annihilation on the view): the comparison baseline for the batch.
int serial_step_once(amk_ctx* c, Batch& B, bool stagger) {
  batch_begin_step_kernel<<<1, 1, 0, c->stream>>>(B.step_dev(), B.queue(), B.contact_count());
  AMK_TRY(check_launch(c, "batch_begin_step_kernel"));
  const uint64_t st = B.step + 1;
  for (int i = 0; i < B.n_inst; ++i) {
    const long off = B.offsets[i], cnt = B.offsets[i + 1] - off;
    if (cnt == 0) continue;
    const amk_params& p = B.params[i];
    AMK_TRY(instance_coulomb(c, B, i));
    AMK_TRY(push_range(c, B.push[i], off, off + cnt, stagger, st));
    if (p.annihilation_enabled && p.contact_radius > 0.0) {
      View v = instance_view(c, B, i);
      AMK_TRY(annihilate_view(c, v, c->species.as<uint8_t>() + off, c->ids.as<uint32_t>() + off, p.contact_radius,
                              p.annihilation_probability, static_cast<uint32_t>(p.seed), st, nullptr));
    }
  }
  return AMK_OK;
}

}  // namespace
}  // namespace amk

using namespace amk;

extern "C" int amk_batch_set(amk_ctx* c, int n_inst, const amk_params* params, const long* offsets) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  if (n_inst <= 0 || !params || !offsets) return fail(AMK_ERR_INVALID, "amk_batch_set: no instances");
  if (n_inst > kMaxInstances) return fail(AMK_ERR_LIMIT, "%d instances exceed the maximum of %d", n_inst, kMaxInstances);
  if (offsets[0] != 0 || offsets[n_inst] != c->n)
    return fail(AMK_ERR_INVALID, "instance offsets must run from 0 to the particle count %ld", c->n);
  for (int i = 0; i < n_inst; ++i) {
    if (offsets[i + 1] < offsets[i]) return fail(AMK_ERR_INVALID, "instance offsets must not decrease");
    if (offsets[i + 1] - offsets[i] >= (1L << 27))
      return fail(AMK_ERR_LIMIT, "instance %d: more than 2^27 particles", i);
    if (amk_params_validate(&params[i], 0) != AMK_OK) return AMK_ERR_INVALID;
    if (!(params[i].dt > 0.0)) return fail(AMK_ERR_INVALID, "instance %d: dt must be positive", i);
    if (params[i].coulomb_forces_enabled && params[i].coulomb_method == AMK_METHOD_FAST_MULTIPOLE &&
        params[i].fmm_learned)
      return fail(AMK_ERR_UNSUPPORTED, "instance %d: the learned correction is not available in batches", i);
  }
  AMK_CUDA_TRY(cudaSetDevice(c->device));
  batch_destroy(c);
  Batch* B = new Batch();
  c->batch = B;
  B->n_inst = n_inst;
  B->params.assign(params, params + n_inst);
  B->offsets.assign(offsets, offsets + n_inst + 1);
  B->step = static_cast<uint64_t>(c->step);
  const long n = c->n;
  // host copies of the positions for the per-instance scales and grids
  std::vector<double> hx(n), hy(n), hz(n);
  if (n > 0) {
    AMK_CUDA_TRY(cudaMemcpyAsync(hx.data(), c->x.ptr, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    AMK_CUDA_TRY(cudaMemcpyAsync(hy.data(), c->y.ptr, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    AMK_CUDA_TRY(cudaMemcpyAsync(hz.data(), c->z.ptr, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
  }
  std::vector<InstanceDev> inst(n_inst);
  std::vector<uint16_t> inst_of(n);
  std::vector<std::pair<long, int2>> units;  // (instance size, unit)
  long n_tiles = 0;  // all-pairs sub-tile slots (kBSubPerUnit per unit)
  for (int i = 0; i < n_inst; ++i) {
    const amk_params& p = params[i];
    const long off = offsets[i], cnt = offsets[i + 1] - off;
    double mx = 0.0;
    for (long k = off; k < off + cnt; ++k) {
      inst_of[k] = static_cast<uint16_t>(i);
      const double a = std::max(std::fabs(hx[k]), std::max(std::fabs(hy[k]), std::fabs(hz[k])));
      if (std::isfinite(a)) mx = std::max(mx, a);
    }
    InstanceDev& d = inst[i];
    d.push = push_params_for(p);
    B->push.push_back(d.push);
    B->scale.push_back(length_scale_for(mx));
    d.inv_l = 1.0 / B->scale.back();
    d.annihilation = (p.annihilation_enabled && p.contact_radius > 0.0) ? 1 : 0;
    B->any_annihilation = B->any_annihilation || d.annihilation;
    d.contact_radius = p.contact_radius;
    d.probability = p.annihilation_probability;
    // grid over [-reach, reach)^3 with cells no smaller than the contact radius
    const double reach = std::max(4.0 * mx, 1e-12);
    const double cs = std::max(p.contact_radius * (1.0 + 1e-9), 2.0 * reach / (kGridMax - 1.0));
    for (int k = 0; k < 3; ++k) d.origin[k] = -reach;
    d.inv_cell = 1.0 / cs;
    d.inv_sort_cell = 1022.0 / (2.0 * reach);
    d.sub0 = n_tiles;
    if (p.coulomb_forces_enabled && p.coulomb_method == AMK_METHOD_ALLPAIRS)
      n_tiles += (cnt + kBUnit - 1) / kBUnit * kBSubPerUnit;
    d.seed = static_cast<uint32_t>(p.seed);
    B->leaf.push_back(p.coulomb_method == AMK_METHOD_BARNES_HUT ? 8 : 32);
    d.offset = off;
    d.count = cnt;
    if (!p.coulomb_forces_enabled || cnt == 0) continue;
    if (p.coulomb_method == AMK_METHOD_ALLPAIRS) {
      for (long b = 0; b * kBUnit < cnt; ++b) units.push_back({cnt, make_int2(i, static_cast<int>(b))});
    } else {
      B->solver_instances.push_back(i);
      if (p.coulomb_method == AMK_METHOD_BARNES_HUT || p.coulomb_method == AMK_METHOD_FAST_MULTIPOLE)
        B->graphable = false;  // their tree builds read sizes back to the host
    }
  }
  std::stable_sort(units.begin(), units.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
  std::vector<int2> hu(units.size());
  for (size_t k = 0; k < units.size(); ++k) hu[k] = units[k].second;
  B->n_units = static_cast<long>(hu.size());
  B->contact_cap = 0;
  int sms = 148, per_sm = 1;
  AMK_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
  AMK_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_allpairs_kernel, kBT, 0));
  B->grid = static_cast<int>(std::max<long>(1, std::min<long>(B->n_units, static_cast<long>(sms) * std::max(1, per_sm))));
  const size_t nn = static_cast<size_t>(std::max<long>(n, 1));
  AMK_TRY(B->inst.reserve(n_inst * sizeof(InstanceDev)));
  AMK_TRY(B->inst_of.reserve(nn * sizeof(uint16_t)));
  AMK_TRY(B->units.reserve(std::max<size_t>(1, hu.size()) * sizeof(int2)));
  AMK_TRY(B->counters.reserve(64));
  AMK_TRY(B->reserve_contacts(std::max<long>(65536, n / 8), n));
  AMK_TRY(B->best.reserve((2 * nn + sizeof(MatchState) / 8 + 1) * sizeof(unsigned long long)));  // two arrays + state
  AMK_TRY(B->keys.reserve(nn * sizeof(uint64_t)));
  AMK_TRY(B->vals.reserve(nn * sizeof(uint32_t)));
  AMK_TRY(B->skeys.reserve(nn * sizeof(uint64_t)));
  AMK_TRY(B->sidx.reserve(nn * sizeof(uint32_t)));
  AMK_TRY(B->perm.reserve(nn * sizeof(uint32_t)));
  AMK_TRY(B->rel.reserve(nn * sizeof(float4)));
  AMK_TRY(B->boxes.reserve(static_cast<size_t>(std::max<long>(n_tiles, 1)) * sizeof(TileBox)));
  AMK_CUDA_TRY(cudaMemcpyAsync(B->inst.ptr, inst.data(), n_inst * sizeof(InstanceDev), cudaMemcpyHostToDevice,
                               c->stream));
  if (n > 0)
    AMK_CUDA_TRY(cudaMemcpyAsync(B->inst_of.ptr, inst_of.data(), n * sizeof(uint16_t), cudaMemcpyHostToDevice,
                                 c->stream));
  if (!hu.empty())
    AMK_CUDA_TRY(cudaMemcpyAsync(B->units.ptr, hu.data(), hu.size() * sizeof(int2), cudaMemcpyHostToDevice, c->stream));
  const unsigned long long init[8] = {0, B->step, 0, 0, 0, 0, 0, 0};
  AMK_CUDA_TRY(cudaMemcpyAsync(B->counters.ptr, init, sizeof(init), cudaMemcpyHostToDevice, c->stream));
  if (n > 0) {
    // random streams and contact priorities use the index within the instance
    batch_local_ids_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, c->stream>>>(
        n, B->inst_of.as<uint16_t>(), B->inst.as<InstanceDev>(), c->ids.as<uint32_t>());
    AMK_TRY(check_launch(c, "batch_local_ids_kernel"));
  }
  AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return AMK_OK;
}

extern "C" int amk_batch_step(amk_ctx* c, int nsteps, int graph_chunk, int serial) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  if (!c->batch) return fail(AMK_ERR_STATE, "no batch: call amk_batch_set first");
  if (nsteps < 0) return fail(AMK_ERR_INVALID, "nsteps < 0");
  Batch& B = *c->batch;
  AMK_CUDA_TRY(cudaSetDevice(c->device));
  const bool use_graph = graph_chunk > 0 && !serial && B.graphable && !c->profiling;
  int done = 0;
  bool graphed = false;
  while (done < nsteps) {
    const bool stagger = !c->staggered;
    if (!use_graph || !B.warm || stagger || nsteps - done < graph_chunk) {
      AMK_TRY(serial ? serial_step_once(c, B, stagger) : batch_step_once(c, B, stagger, true));
      c->staggered = true;
      B.warm = true;
      B.step++;
      c->step++;
      ++done;
      continue;
    }
    if (!B.exec || B.graph_steps != graph_chunk) {
      B.drop_graph();
      // head room over the largest contact count seen so far: inside the
      // graph an overflow can only be recorded
      AMK_TRY(B.reserve_contacts(static_cast<long>(2 * B.max_contacts), c->n));
      const long launches0 = c->kernel_launches;
      AMK_CUDA_TRY(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
      int rc = AMK_OK;
      for (int s = 0; s < graph_chunk && rc == AMK_OK; ++s) rc = batch_step_once(c, B, false, false);
      cudaGraph_t g = nullptr;
      const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
      B.graph_launches = c->kernel_launches - launches0;
      c->kernel_launches = launches0;  // captured, not run
      if (rc != AMK_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
      }
      if (e != cudaSuccess) return fail(AMK_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
      B.graph = g;
      AMK_CUDA_TRY(cudaGraphInstantiate(&B.exec, B.graph, 0));
      B.graph_steps = graph_chunk;
    }
    if (!graphed) AMK_CUDA_TRY(cudaMemsetAsync(B.call_overflow(), 0, sizeof(unsigned long long), c->stream));
    graphed = true;
    AMK_CUDA_TRY(cudaGraphLaunch(B.exec, c->stream));
    c->kernel_launches += B.graph_launches;
    B.step += static_cast<uint64_t>(graph_chunk);
    c->step += graph_chunk;
    done += graph_chunk;
  }
  c->stage_dirty = true;
  if (graphed) {
    unsigned long long ov = 0;
    AMK_CUDA_TRY(cudaMemcpyAsync(&ov, B.call_overflow(), sizeof(ov), cudaMemcpyDeviceToHost, c->stream));
    AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (ov) {
      AMK_TRY(B.reserve_contacts(2 * B.contact_cap, c->n));  // the next capture gets a larger buffer
      return fail(AMK_ERR_LIMIT,
                  "annihilation contacts overflowed the contact buffer inside a CUDA graph chunk: the "
                  "steps of this call dropped contacts (the buffer is now larger; step without graphs "
                  "to avoid it)");
    }
  }
  return AMK_OK;
}

extern "C" int amk_batch_coulomb(amk_ctx* c) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  if (!c->batch) return fail(AMK_ERR_STATE, "no batch: call amk_batch_set first");
  AMK_CUDA_TRY(cudaSetDevice(c->device));
  Batch& B = *c->batch;
  if (c->n == 0) return AMK_OK;
  // the all-pairs queue head is reset by the step prologue; reset it here
  AMK_CUDA_TRY(cudaMemsetAsync(B.queue(), 0, sizeof(int), c->stream));
  AMK_TRY(batch_coulomb(c, B));
  return AMK_OK;
}

extern "C" int amk_batch_status(amk_ctx* c, int* overflow, long* alive_counts) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  if (!c->batch) return fail(AMK_ERR_STATE, "no batch: call amk_batch_set first");
  Batch& B = *c->batch;
  AMK_CUDA_TRY(cudaSetDevice(c->device));
  unsigned long long ov = 0;
  AMK_CUDA_TRY(cudaMemcpyAsync(&ov, B.overflow(), sizeof(ov), cudaMemcpyDeviceToHost, c->stream));
  std::vector<unsigned long long> h(B.n_inst, 0ull);
  if (alive_counts) {
    int rc = AMK_OK;
    unsigned long long* cnt = slot<unsigned long long>(c, kSlotStatus, B.n_inst, &rc);
    AMK_TRY(rc);
    AMK_CUDA_TRY(cudaMemsetAsync(cnt, 0, B.n_inst * sizeof(unsigned long long), c->stream));
    if (c->n > 0) {
      batch_alive_count_kernel<<<static_cast<unsigned>((c->n + 255) / 256), 256, 0, c->stream>>>(
          c->n, c->alive.as<uint8_t>(), B.inst_of.as<uint16_t>(), cnt);
      AMK_TRY(check_launch(c, "batch_alive_count_kernel"));
    }
    AMK_CUDA_TRY(cudaMemcpyAsync(h.data(), cnt, B.n_inst * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                 c->stream));
  }
  AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (alive_counts)
    for (int i = 0; i < B.n_inst; ++i) alive_counts[i] = static_cast<long>(h[i]);
  if (overflow) *overflow = ov ? 1 : 0;
  return AMK_OK;
}

extern "C" int amk_batch_info(const amk_ctx* c, long* n_instances, long* work_units, int* graphable) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  if (!c->batch) return fail(AMK_ERR_STATE, "no batch: call amk_batch_set first");
  if (n_instances) *n_instances = c->batch->n_inst;
  if (work_units) *work_units = c->batch->n_units;
  if (graphable) *graphable = c->batch->graphable ? 1 : 0;
  return AMK_OK;
}

// Per-instance method choice by measurement: the batched all-pairs launch is
// timed once (its cost split over instances in proportion to N_i^2); the FMM
// configurations (orders 4/6/8, theta 0.5/0.35, leaf 32/64; higher orders
// skipped once a lower one meets the budget) are timed and audited on the
// largest instance; the best one that meets the budget then replaces
// all-pairs on every instance, largest first, where its measured time is
// below the instance's all-pairs share and its audit meets the budget. The
// batch is rebuilt with the chosen methods.
extern "C" int amk_batch_autotune(amk_ctx* c, double error_budget, long samples, int* methods_out) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  if (!c->batch) return fail(AMK_ERR_STATE, "no batch: call amk_batch_set first");
  if (!(error_budget > 0.0)) return fail(AMK_ERR_INVALID, "error budget must be positive");
  AMK_CUDA_TRY(cudaSetDevice(c->device));
  const int n_inst = c->batch->n_inst;
  std::vector<amk_params> P = c->batch->params;
  const std::vector<long> offsets = c->batch->offsets;
  std::vector<int> leaf(n_inst, 32);
  for (int i = 0; i < n_inst; ++i)
    if (P[i].coulomb_forces_enabled) P[i].coulomb_method = AMK_METHOD_ALLPAIRS;
  AMK_TRY(amk_batch_set(c, n_inst, P.data(), offsets.data()));
  Batch* B = c->batch;
  // 1. the batched all-pairs launch and its cost share per instance
  double ap_ms = 0.0;
  AMK_TRY(time_solver(c, [&]() -> int {
    AMK_CUDA_TRY(cudaMemsetAsync(B->queue(), 0, sizeof(int), c->stream));
    return batch_coulomb(c, *B);
  }, 3, &ap_ms));
  std::vector<int> order;
  double total_pairs = 0.0;
  for (int i = 0; i < n_inst; ++i) {
    const double ni = static_cast<double>(offsets[i + 1] - offsets[i]);
    if (P[i].coulomb_forces_enabled && ni > 1) {
      order.push_back(i);
      total_pairs += ni * ni;
    }
  }
  if (order.empty()) {
    if (methods_out)
      for (int i = 0; i < n_inst; ++i) methods_out[i] = P[i].coulomb_method;
    return AMK_OK;
  }
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    return offsets[a + 1] - offsets[a] > offsets[b + 1] - offsets[b];
  });
  auto ap_share = [&](int i) {
    const double ni = static_cast<double>(offsets[i + 1] - offsets[i]);
    return ap_ms * ni * ni / total_pairs;
  };
  // all-pairs must itself meet the budget (on the largest instance)
  double ap_err = 0.0;
  AMK_TRY(force_error(c, instance_view(c, *B, order[0]), samples, &ap_err, nullptr));
  // 2. FMM configurations on the largest instance
  const int big = order[0];
  const View vb = instance_view(c, *B, big);
  int best_order = 0, best_leaf = 32;
  double best_theta = 0.5, best_ms = INFINITY;
  for (double theta : {0.5, 0.35})
    for (int lf : {32, 64})
      for (int p : {4, 6, 8}) {
        double ms = 0.0, err = 0.0;
        AMK_TRY(time_solver(c, [&]() { return fmm_forces(c, vb, p, theta, lf, false, nullptr); }, 1, &ms));
        AMK_TRY(force_error(c, vb, samples, &err, nullptr));
        if (err <= error_budget) {
          if (ms < best_ms) {
            best_ms = ms;
            best_order = p;
            best_theta = theta;
            best_leaf = lf;
          }
          break;  // higher orders at this theta and leaf cost more
        }
      }
  // 3. instances, largest first, switch to that FMM where it is faster
  int losses = 0;
  if (best_order > 0)
    for (int i : order) {
      if (losses >= 2) break;
      const View v = instance_view(c, *B, i);
      double ms = 0.0, err = 0.0;
      AMK_TRY(time_solver(c, [&]() { return fmm_forces(c, v, best_order, best_theta, best_leaf, false, nullptr); },
                          1, &ms));
      AMK_TRY(force_error(c, v, samples, &err, nullptr));
      if ((ms < ap_share(i) || ap_err > error_budget) && err <= error_budget) {
        P[i].coulomb_method = AMK_METHOD_FAST_MULTIPOLE;
        P[i].fast_multipole_order = best_order;
        P[i].fast_multipole_theta = best_theta;
        P[i].fmm_learned = 0;
        leaf[i] = best_leaf;
        losses = 0;
      } else {
        ++losses;
      }
    }
  AMK_TRY(amk_batch_set(c, n_inst, P.data(), offsets.data()));
  for (int i = 0; i < n_inst; ++i)
    if (P[i].coulomb_method == AMK_METHOD_FAST_MULTIPOLE) c->batch->leaf[i] = leaf[i];
  if (methods_out)
    for (int i = 0; i < n_inst; ++i) methods_out[i] = P[i].coulomb_forces_enabled ? P[i].coulomb_method : -1;
  if (ap_err > error_budget && best_order == 0)
    return fail(AMK_ERR_LIMIT, "neither all-pairs (%g) nor the FMM met the error budget %g", ap_err, error_budget);
  return AMK_OK;
}

// Energies of every instance (amk_energy per instance): kinetic and trap
// terms from one CTA per instance, the Coulomb term from the instance's
// energy method on its own slice, and per-instance time-centring.
extern "C" int amk_batch_energy(amk_ctx* c, int time_centre, amk_energy_out* out) {
  if (!c || !out) return fail(AMK_ERR_INVALID, "null argument");
  if (!c->batch) return fail(AMK_ERR_STATE, "no batch: call amk_batch_set first");
  AMK_CUDA_TRY(cudaSetDevice(c->device));
  Batch& B = *c->batch;
  const int ni = B.n_inst;
  int rc = AMK_OK;
  double* part = slot<double>(c, kSlotAuxState3, 3 * static_cast<size_t>(ni) + 8, &rc);
  AMK_TRY(rc);
  AMK_TRY(phase_begin(c, AMK_PHASE_ENERGY));
  batch_energy_kernel<<<ni, 256, 0, c->stream>>>(B.inst.as<InstanceDev>(), c->x.as<double>(), c->y.as<double>(),
                                                 c->z.as<double>(), c->vx.as<double>(), c->vy.as<double>(),
                                                 c->vz.as<double>(), c->q.as<double>(), c->m.as<double>(),
                                                 c->alive.as<uint8_t>(), part);
  AMK_TRY(check_launch(c, "batch_energy_kernel"));
  std::vector<double> h(3 * static_cast<size_t>(ni));
  AMK_CUDA_TRY(cudaMemcpyAsync(h.data(), part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (B.prev_trap.size() != static_cast<size_t>(ni)) {
    B.prev_trap.assign(ni, 0.0);
    B.prev_coulomb.assign(ni, 0.0);
  }
  for (int i = 0; i < ni; ++i) {
    const amk_params& p = B.params[i];
    double coul = 0.0;
    if (p.coulomb_forces_enabled && B.offsets[i + 1] > B.offsets[i])
      AMK_TRY(coulomb_energy_view(c, instance_view(c, B, i), p, p.energy_method, &coul));
    amk_energy_out& o = out[i];
    o.kinetic = h[3 * i];
    o.trap_potential = h[3 * i + 1];
    o.coulomb_potential = coul;
    o.num_active = static_cast<long>(h[3 * i + 2]);
    if (time_centre) {  // energy_analysis.cc:126-142
      const double raw_trap = o.trap_potential, raw_coul = o.coulomb_potential;
      if (B.energy_has_previous) {
        o.trap_potential = 0.5 * (B.prev_trap[i] + raw_trap);
        o.coulomb_potential = 0.5 * (B.prev_coulomb[i] + raw_coul);
      }
      B.prev_trap[i] = raw_trap;
      B.prev_coulomb[i] = raw_coul;
    }
    o.total = o.kinetic + o.trap_potential + o.coulomb_potential;
  }
  if (time_centre) B.energy_has_previous = true;
  return phase_end(c, AMK_PHASE_ENERGY);
}
