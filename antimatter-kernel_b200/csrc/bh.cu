// Barnes-Hut forces and potentials on the GPU octree.
//
// Monopoles (barnes-hut.cc:76-159): every node keeps the positive charge sum
// and the |negative| charge sum with their charge centres; leaves sum their
// particles, internal nodes merge their children in octant order, level by
// level from the deepest.
//
// Walk (barnes-hut.cc:183-269): a warp takes 32 consecutive targets in tree
// order and walks one shared depth-first stack. Each entry carries the mask
// of lanes that still need that node. A lane accepts an internal node when
// (2h)^2 < theta^2 |x - c|^2 (the reference's test, evaluated in FP64
// without contraction, so the accepted-node set of every target is the
// reference's); accepting lanes add the two monopoles, the others push the
// children for themselves. Leaves are summed directly, skipping the target
// itself and q = 0 sources. Pairs closer than 1e-30 m^2 are skipped
// (barnes-hut.cc:33-41). All arithmetic is FP64 (leaf sums FP32 in the
// tensor precision mode, below); inverse distances use rsqrt where the
// reference divides by sqrt (an ulp-level difference).
#include <algorithm>
#include <vector>

#include "amk_internal.cuh"

namespace amk {
namespace {

constexpr int kWalkWarps = 4;
constexpr int kStack = 176;  // >= 1 + 7 * 21 + 8

__device__ __forceinline__ double dot_rn(double a, double b, double c) {
  // ((0 + a*a) + b*b) + c*c without contraction (the reference's Real3 dot)
  return __dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)), __dmul_rn(c, c));
}

// BH node charges: pos = (Q+, centre+), neg = (|Q-|, centre-).
__global__ void bh_leaf_kernel(const Octree t, double4* __restrict__ pos, double4* __restrict__ neg) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= t.n_nodes) return;
  if (!t.meta[id].y) return;
  const int2 r = t.range[id];
  double qp = 0.0, qn = 0.0, mp[3] = {0.0, 0.0, 0.0}, mn[3] = {0.0, 0.0, 0.0};
  for (int k = r.x; k < r.y; ++k) {
    const double4 s = t.src[k];
    if (s.w > 0.0) {
      qp += s.w;
      mp[0] = __dadd_rn(mp[0], __dmul_rn(s.x, s.w));
      mp[1] = __dadd_rn(mp[1], __dmul_rn(s.y, s.w));
      mp[2] = __dadd_rn(mp[2], __dmul_rn(s.z, s.w));
    } else if (s.w < 0.0) {
      qn += -s.w;
      mn[0] = __dadd_rn(mn[0], __dmul_rn(s.x, -s.w));
      mn[1] = __dadd_rn(mn[1], __dmul_rn(s.y, -s.w));
      mn[2] = __dadd_rn(mn[2], __dmul_rn(s.z, -s.w));
    }
  }
  const double4 c = t.center[id];
  pos[id] = qp > 0.0 ? make_double4(mp[0] * (1.0 / qp), mp[1] * (1.0 / qp), mp[2] * (1.0 / qp), qp)
                     : make_double4(c.x, c.y, c.z, 0.0);
  neg[id] = qn > 0.0 ? make_double4(mn[0] * (1.0 / qn), mn[1] * (1.0 / qn), mn[2] * (1.0 / qn), qn)
                     : make_double4(c.x, c.y, c.z, 0.0);
}

__global__ void bh_merge_kernel(const Octree t, int depth, double4* __restrict__ pos, double4* __restrict__ neg) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= t.n_nodes) return;
  const uchar2 mt = t.meta[id];
  if (mt.y || mt.x != depth) return;
  double qp = 0.0, qn = 0.0, mp[3] = {0.0, 0.0, 0.0}, mn[3] = {0.0, 0.0, 0.0};
  for (int o = 0; o < 8; ++o) {
    const int ch = t.child[8 * id + o];
    if (ch < 0) continue;
    const double4 a = pos[ch], b = neg[ch];
    if (a.w > 0.0) {
      qp += a.w;
      mp[0] = __dadd_rn(mp[0], __dmul_rn(a.x, a.w));
      mp[1] = __dadd_rn(mp[1], __dmul_rn(a.y, a.w));
      mp[2] = __dadd_rn(mp[2], __dmul_rn(a.z, a.w));
    }
    if (b.w > 0.0) {
      qn += b.w;
      mn[0] = __dadd_rn(mn[0], __dmul_rn(b.x, b.w));
      mn[1] = __dadd_rn(mn[1], __dmul_rn(b.y, b.w));
      mn[2] = __dadd_rn(mn[2], __dmul_rn(b.z, b.w));
    }
  }
  const double4 c = t.center[id];
  pos[id] = qp > 0.0 ? make_double4(mp[0] * (1.0 / qp), mp[1] * (1.0 / qp), mp[2] * (1.0 / qp), qp)
                     : make_double4(c.x, c.y, c.z, 0.0);
  neg[id] = qn > 0.0 ? make_double4(mn[0] * (1.0 / qn), mn[1] * (1.0 / qn), mn[2] * (1.0 / qn), qn)
                     : make_double4(c.x, c.y, c.z, 0.0);
}

// AddPointCharge, barnes-hut.cc:20-28: force += r * (k qt qs / r^2 / r).
__device__ __forceinline__ void add_point(double tx, double ty, double tz, double tq, double sx, double sy,
                                          double sz, double sq, double* f) {
  const double rx = tx - sx, ry = ty - sy, rz = tz - sz;
  const double d2 = dot_rn(rx, ry, rz);
  if (d2 < kMinSquaredDistance) return;
  const double inv = rsqrt(d2);
  const double w = kCoulombConstant * tq * sq * (inv * inv * inv);
  f[0] += rx * w;
  f[1] += ry * w;
  f[2] += rz * w;
}

__device__ __forceinline__ void add_phi(double tx, double ty, double tz, double sx, double sy, double sz,
                                        double sq, double* phi) {
  const double rx = tx - sx, ry = ty - sy, rz = tz - sz;
  const double d2 = dot_rn(rx, ry, rz);
  if (d2 < kMinSquaredDistance) return;
  *phi += sq * rsqrt(d2);
}

// Leaf sums in FP32 (the tensor precision mode): sources as double-float
// pairs x = hi + lo (hi = float(x), lo = float(x - hi)) relative to the
// tree frame; a pair's difference (x_i,hi - x_j,hi) + (x_i,lo - x_j,lo) is
// exact to FP32 rounding of |r| for particles of neighbouring cells
// (Sterbenz), the per-leaf sums of q_j r / r^3 are FP32 and are added to the
// FP64 accumulators once per leaf. The opening test and the node monopoles
// stay FP64, so the accepted-node sets are the reference's.
struct BhF32 {
  const float4* hi;  // (x, y, z, q) hi parts, q as float
  const float4* lo;  // lo parts
  double qs;         // charges were divided by this before the float conversion
};

__global__ void bh_stage_kernel(const Octree t, double qs, float4* __restrict__ hi, float4* __restrict__ lo) {
  const long k = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  if (k >= t.m) return;
  const double4 s = t.src[k];
  const float hx = static_cast<float>(s.x), hy = static_cast<float>(s.y), hz = static_cast<float>(s.z);
  hi[k] = make_float4(hx, hy, hz, static_cast<float>(s.w / qs));
  lo[k] = make_float4(static_cast<float>(s.x - hx), static_cast<float>(s.y - hy), static_cast<float>(s.z - hz), 0.f);
}

template <bool kPhi, bool kF32>
__global__ void __launch_bounds__(32 * kWalkWarps)
bh_walk_kernel(const Octree t, const double4* __restrict__ pos, const double4* __restrict__ neg, double theta2,
               BhF32 f32, double* __restrict__ out, int* __restrict__ status) {
  __shared__ int s_node[kWalkWarps][kStack];
  __shared__ unsigned s_mask[kWalkWarps][kStack];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const long k = (static_cast<long>(blockIdx.x) * kWalkWarps + w) * 32 + lane;
  const bool valid = k < t.m;
  double4 me = make_double4(0.0, 0.0, 0.0, 0.0);
  if (valid) me = t.src[k];
  // ComputeForce returns 0 for q = 0 (barnes-hut.cc:169); potentials walk anyway
  const bool want = valid && (kPhi || me.w != 0.0);
  const unsigned lanes = __ballot_sync(0xffffffffu, want);
  double f[3] = {0.0, 0.0, 0.0};
  double phi = 0.0;
  int sp = 0;
  if (lanes) {
    if (lane == 0) {
      s_node[w][0] = 0;
      s_mask[w][0] = lanes;
    }
    sp = 1;
  }
  __syncwarp();
  while (sp > 0) {
    --sp;
    const int nd = s_node[w][sp];
    const unsigned mask = s_mask[w][sp];
    __syncwarp();
    const bool act = (mask >> lane) & 1u;
    const double4 pq = pos[nd], nq = neg[nd];
    if (pq.w == 0.0 && nq.w == 0.0) continue;  // barnes-hut.cc:186
    if (t.meta[nd].y) {
      const int2 r = t.range[nd];
      if (act) {
        if (kF32) {
          // sum over the leaf of (q_j / qs) r / r^3 (or / r) in FP32
          const float4 mh = f32.hi[k], ml = f32.lo[k];
          const float min_sq = 1e-30f;  // kMinSquaredDistance (m^2), a normal float
          float ax = 0.f, ay = 0.f, az = 0.f, ap = 0.f;
          for (int j = r.x; j < r.y; ++j) {
            const float4 s = f32.hi[j], q = f32.lo[j];
            const float rx = fmaf(s.x, -1.f, mh.x) + fmaf(q.x, -1.f, ml.x);
            const float ry = fmaf(s.y, -1.f, mh.y) + fmaf(q.y, -1.f, ml.y);
            const float rz = fmaf(s.z, -1.f, mh.z) + fmaf(q.z, -1.f, ml.z);
            const float r2 = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
            // the target itself (r = 0), closer pairs and neutral sources add zero
            const float inv = (j != k && r2 >= min_sq) ? rsqrtf(r2) : 0.f;
            const float qr = s.w * inv;
            if (kPhi) {
              ap += qr;
            } else {
              const float w = qr * (inv * inv);
              ax = fmaf(rx, w, ax);
              ay = fmaf(ry, w, ay);
              az = fmaf(rz, w, az);
            }
          }
          if (kPhi) {
            phi += f32.qs * static_cast<double>(ap);
          } else {
            const double sc = kCoulombConstant * me.w * f32.qs;
            f[0] += sc * static_cast<double>(ax);
            f[1] += sc * static_cast<double>(ay);
            f[2] += sc * static_cast<double>(az);
          }
        } else {
          for (int j = r.x; j < r.y; ++j) {
            if (j == k) continue;
            const double4 s = t.src[j];
            if (s.w == 0.0) continue;
            if (kPhi)
              add_phi(me.x, me.y, me.z, s.x, s.y, s.z, s.w, &phi);
            else
              add_point(me.x, me.y, me.z, me.w, s.x, s.y, s.z, s.w, f);
          }
        }
      }
      continue;
    }
    const double4 c = t.center[nd];
    const double dx = me.x - c.x, dy = me.y - c.y, dz = me.z - c.z;
    const double d2 = dot_rn(dx, dy, dz);
    const double width = 2.0 * c.w;
    const bool accept = act && (__dmul_rn(width, width) < __dmul_rn(theta2, d2));
    const unsigned acc = __ballot_sync(0xffffffffu, accept);
    if (accept) {
      if (kPhi) {
        if (pq.w > 0.0) add_phi(me.x, me.y, me.z, pq.x, pq.y, pq.z, pq.w, &phi);
        if (nq.w > 0.0) add_phi(me.x, me.y, me.z, nq.x, nq.y, nq.z, -nq.w, &phi);
      } else {
        if (pq.w > 0.0) add_point(me.x, me.y, me.z, me.w, pq.x, pq.y, pq.z, pq.w, f);
        if (nq.w > 0.0) add_point(me.x, me.y, me.z, me.w, nq.x, nq.y, nq.z, -nq.w, f);
      }
    }
    const unsigned open = mask & ~acc;
    if (open) {
      // push children 7..0 (lane 0 holds child 7) so that octant 0 pops first
      const int ch = lane < 8 ? t.child[8 * nd + (7 - lane)] : -1;
      const unsigned has = __ballot_sync(0xffffffffu, ch >= 0);
      const int pushed = __popc(has);
      if (sp + pushed > kStack) {  // cannot happen for depth <= 21; guarded anyway
        if (lane == 0) atomicExch(status, 1);
        break;
      }
      if (ch >= 0) {
        const int slot_i = sp + __popc(has & ((1u << lane) - 1u));
        s_node[w][slot_i] = ch;
        s_mask[w][slot_i] = open;
      }
      sp += pushed;
      __syncwarp();
    }
  }
  if (valid) {
    if (kPhi) {
      out[k] = phi;
    } else {
      out[3 * k + 0] = f[0];
      out[3 * k + 1] = f[1];
      out[3 * k + 2] = f[2];
    }
  }
}

__global__ void bh_scatter_kernel(const Octree t, const double* __restrict__ fo, const double* __restrict__ po,
                                  View v) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= t.m) return;
  const long i = t.order[k];
  if (fo) {
    v.fx[i] = fo[3 * k + 0];
    v.fy[i] = fo[3 * k + 1];
    v.fz[i] = fo[3 * k + 2];
  }
  if (po && v.phi) v.phi[i] = po[k];
}

__global__ void zero_outputs_kernel(View v, bool forces) {
  const long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  if (i >= v.n) return;
  if (forces) {
    v.fx[i] = 0.0;
    v.fy[i] = 0.0;
    v.fz[i] = 0.0;
  }
  if (v.phi) v.phi[i] = 0.0;
}

int bh_monopoles(amk_ctx* c, const Octree& t, double4** pos_out, double4** neg_out) {
  int rc = AMK_OK;
  double4* pos = slot<double4>(c, kSlotBhPos, t.n_nodes, &rc);
  AMK_TRY(rc);
  double4* neg = slot<double4>(c, kSlotBhNeg, t.n_nodes, &rc);
  AMK_TRY(rc);
  const unsigned g = static_cast<unsigned>((t.n_nodes + 255) / 256);
  bh_leaf_kernel<<<g, 256, 0, c->stream>>>(t, pos, neg);
  AMK_TRY(check_launch(c, "bh_leaf_kernel"));
  for (int d = t.max_depth; d >= 0; --d) {
    bh_merge_kernel<<<g, 256, 0, c->stream>>>(t, d, pos, neg);
    AMK_TRY(check_launch(c, "bh_merge_kernel"));
  }
  *pos_out = pos;
  *neg_out = neg;
  return AMK_OK;
}

}  // namespace

int barnes_hut_forces(amk_ctx* c, const View& v, double theta, long leaf_capacity) {
  const long n = v.n;
  if (n == 0) return AMK_OK;
  zero_outputs_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, c->stream>>>(v, true);
  AMK_TRY(check_launch(c, "zero_outputs_kernel"));
  Octree t;
  AMK_TRY(phase_begin(c, AMK_PHASE_TREE));
  AMK_TRY(build_octree(c, v, static_cast<int>(std::min<long>(leaf_capacity, 1 << 20)), 0, &t));
  if (t.m == 0) return phase_end(c, AMK_PHASE_TREE);
  double4 *pos = nullptr, *neg = nullptr;
  AMK_TRY(bh_monopoles(c, t, &pos, &neg));
  AMK_TRY(phase_end(c, AMK_PHASE_TREE));
  int rc = AMK_OK;
  double* fo = slot<double>(c, kSlotWalkOut, 3 * static_cast<size_t>(t.m), &rc);
  AMK_TRY(rc);
  double* po = v.phi ? slot<double>(c, kSlotFmmWork5, static_cast<size_t>(t.m), &rc) : nullptr;
  AMK_TRY(rc);
  int* status = slot<int>(c, kSlotStatus, 8, &rc) + 4;
  AMK_TRY(rc);
  AMK_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(int), c->stream));
  const unsigned blocks = static_cast<unsigned>((t.m + 32 * kWalkWarps - 1) / (32 * kWalkWarps));
  const double theta2 = theta * theta;  // squared_theta_, barnes-hut.cc:36
  const bool f32 = c->fmm_precision == AMK_FMM_TENSOR;
  BhF32 fs{nullptr, nullptr, kElementaryCharge};
  if (f32) {  // sources as double-float pairs, charges in units of e
    float4* stage = slot<float4>(c, kSlotP2PStage, 2 * static_cast<size_t>(t.m), &rc);
    AMK_TRY(rc);
    bh_stage_kernel<<<static_cast<unsigned>((t.m + 255) / 256), 256, 0, c->stream>>>(t, fs.qs, stage, stage + t.m);
    AMK_TRY(check_launch(c, "bh_stage_kernel"));
    fs.hi = stage;
    fs.lo = stage + t.m;
  }
  AMK_TRY(phase_begin(c, AMK_PHASE_BH_WALK));
  if (f32)
    bh_walk_kernel<false, true><<<blocks, 32 * kWalkWarps, 0, c->stream>>>(t, pos, neg, theta2, fs, fo, status);
  else
    bh_walk_kernel<false, false><<<blocks, 32 * kWalkWarps, 0, c->stream>>>(t, pos, neg, theta2, fs, fo, status);
  AMK_TRY(check_launch(c, "bh_walk_kernel"));
  if (po) {
    if (f32)
      bh_walk_kernel<true, true><<<blocks, 32 * kWalkWarps, 0, c->stream>>>(t, pos, neg, theta2, fs, po, status);
    else
      bh_walk_kernel<true, false><<<blocks, 32 * kWalkWarps, 0, c->stream>>>(t, pos, neg, theta2, fs, po, status);
    AMK_TRY(check_launch(c, "bh_walk_kernel"));
  }
  AMK_TRY(phase_end(c, AMK_PHASE_BH_WALK));
  bh_scatter_kernel<<<static_cast<unsigned>((t.m + 255) / 256), 256, 0, c->stream>>>(t, fo, po, v);
  AMK_TRY(check_launch(c, "bh_scatter_kernel"));
  int st = 0;
  AMK_CUDA_TRY(cudaMemcpyAsync(&st, status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (st) return fail(AMK_ERR_LIMIT, "Barnes-Hut walk stack exceeded %d entries", kStack);
  return AMK_OK;
}

}  // namespace amk

using namespace amk;

// Tree introspection for tests: node arrays in the reference's layout
// (BarnesHutTree::Node, barnes-hut.h:49-61).
extern "C" long amk_bh_tree_dump(amk_ctx* c, long n, const double* x, const double* y, const double* z,
                                 const double* q, long leaf_capacity, long max_nodes, double* node_f64,
                                 long* node_i64) {
  if (!c || n < 0) return fail(AMK_ERR_INVALID, "bad argument");
  if (n == 0) return 0;
  View v;
  AMK_TRY(load_aux_view(c, n, x, y, z, q, &v));
  Octree t;
  AMK_TRY(build_octree(c, v, static_cast<int>(leaf_capacity), 0, &t));
  if (t.n_nodes > max_nodes) return fail(AMK_ERR_LIMIT, "tree has %ld nodes, buffer holds %ld", t.n_nodes, max_nodes);
  double4 *pos = nullptr, *neg = nullptr;
  AMK_TRY(bh_monopoles(c, t, &pos, &neg));
  const long nn = t.n_nodes;
  std::vector<double4> hc(nn), hp(nn), hn(nn);
  std::vector<int> hch(8 * nn);
  std::vector<int2> hr(nn);
  std::vector<uchar2> hm(nn);
  AMK_CUDA_TRY(cudaMemcpyAsync(hc.data(), t.center, nn * sizeof(double4), cudaMemcpyDeviceToHost, c->stream));
  AMK_CUDA_TRY(cudaMemcpyAsync(hp.data(), pos, nn * sizeof(double4), cudaMemcpyDeviceToHost, c->stream));
  AMK_CUDA_TRY(cudaMemcpyAsync(hn.data(), neg, nn * sizeof(double4), cudaMemcpyDeviceToHost, c->stream));
  AMK_CUDA_TRY(cudaMemcpyAsync(hch.data(), t.child, 8 * nn * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  AMK_CUDA_TRY(cudaMemcpyAsync(hr.data(), t.range, nn * sizeof(int2), cudaMemcpyDeviceToHost, c->stream));
  AMK_CUDA_TRY(cudaMemcpyAsync(hm.data(), t.meta, nn * sizeof(uchar2), cudaMemcpyDeviceToHost, c->stream));
  AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
  for (long k = 0; k < nn; ++k) {
    double* f = node_f64 + 12 * k;
    f[0] = hc[k].x;
    f[1] = hc[k].y;
    f[2] = hc[k].z;
    f[3] = hc[k].w;
    f[4] = hp[k].w;
    f[5] = hn[k].w;
    f[6] = hp[k].x;
    f[7] = hp[k].y;
    f[8] = hp[k].z;
    f[9] = hn[k].x;
    f[10] = hn[k].y;
    f[11] = hn[k].z;
    long* g = node_i64 + 11 * k;
    for (int o = 0; o < 8; ++o) g[o] = hch[8 * k + o];
    g[8] = hr[k].x;
    g[9] = hr[k].y;
    g[10] = hm[k].y;
  }
  return nn;
}
