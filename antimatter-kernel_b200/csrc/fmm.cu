// Cartesian fast multipole method on the GPU octree (fast-multipole.cc).
//
// Same mathematics as the reference (all in unit-cube coordinates,
// fast-multipole.cc:91-113): multipoles M_a = sum q (y - c)^a / a!, local
// expansions L_g = 1/g! sum_a (-1)^|a| M_a D_{a+g}(t - s) with D = d^a (1/r)
// from the recurrence r^2 d_i f = -x_i f, L2L/M2M shifts by the binomial
// tables, L2P as E = -grad phi, near field by direct sums. Order P in [1, 8],
// leaf capacity 32, theta acceptance (r_T + r_S)^2 < theta^2 d^2.
//
// GPU mapping:
//   radii, P2M      leaves in parallel (a thread per leaf / a warp per leaf)
//   M2M, L2L        level-synchronous, a warp per node, lanes over coefficients
//   lists           the reference's dual-tree recursion run breadth-first over
//                   (target, source) pairs; M2L and P2P pairs are radix-sorted
//                   by (target, source), so every sum has a fixed order
//                   (run-to-run deterministic)
//   M2L             a warp per target cell; per source the derivative tensor
//                   is built degree by degree in shared memory (lanes over the
//                   multi-indices of one degree) and contracted with the
//                   source's multipole, lanes over local coefficients
//   L2P + P2P       work items of (target leaf, <= 8 source leaves); a warp
//                   per item with lanes split into groups over the sources;
//                   partials added in a fixed order
// Arithmetic is FP64 throughout, as in the reference; inverse distances use
// rsqrt (the reference divides by sqrt), a difference of an ulp.
#include <algorithm>
#include <array>
#include <functional>
#include <map>
#include <memory>
#include <type_traits>
#include <vector>

#include "amk_internal.cuh"
#include "tcgen05.cuh"

namespace amk {

// ------------------------------------------------------------ tables
// The expansion tables (the reference keeps the same quantities in its
// FmmTables, fast-multipole.cc:41-178), generated here from their
// definitions.
//
// Multi-indices (a, b, c) of degree d = a + b + c <= 2p are numbered in
// graded order -- by degree, then a descending, then b descending -- with
// the closed form
//   pos(a, b, c) = d(d+1)(d+2)/6 + e(e+1)/2 + (e - b),   e = d - a,
// where the first term counts the multi-indices of lower degree and the
// second those of degree d with a larger first component. The first
// n_m = (p+1)(p+2)(p+3)/6 positions are the expansion coefficients.
__host__ __device__ constexpr int graded_index(int a, int b, int c) {
  return (a < 0 || b < 0 || c < 0)
             ? -1
             : (a + b + c) * (a + b + c + 1) * (a + b + c + 2) / 6 + (b + c) * (b + c + 1) / 2 + c;
}
static_assert(graded_index(0, 0, 0) == 0 && graded_index(1, 0, 0) == 1 && graded_index(0, 0, 1) == 3 &&
                  graded_index(2, 0, 0) == 4 && graded_index(0, 2, 0) == 7 && graded_index(0, 0, 2) == 9,
              "graded order");

struct FmmHostTables {
  int p = 0, n_m = 0, n_d = 0;
  std::vector<int4> multi;  // a, b, c, degree
  std::vector<double> fact, inv_fact, sign;
  std::vector<int> deg_start;                // n_d entries grouped by degree
  std::vector<int> rec_axis;                 // per k
  std::vector<int> rec_delta, rec_m1, rec_m2;  // 3 per k
  std::vector<int> m2l_index;                // [g * n_m + a]
  std::vector<short> m2l_index_t;            // [a * n_m + g]
  std::vector<int> m2m_off, m2m_b, m2m_c;    // CSR by a
  std::vector<int> l2l_off, l2l_b, l2l_c;    // CSR by a
  std::vector<int> grad;                     // 3 per g, -1 none

  explicit FmmHostTables(int order) : p(order) {
    const int dmax = 2 * p;
    n_d = graded_index(0, 0, dmax) + 1;
    n_m = graded_index(0, 0, p) + 1;
    auto pos = [](const int m[3]) { return graded_index(m[0], m[1], m[2]); };
    multi.resize(n_d);
    for (int d = 0; d <= dmax + 1; ++d) deg_start.push_back(d * (d + 1) * (d + 2) / 6);
    for (int d = 0; d <= dmax; ++d)
      for (int a = 0; a <= d; ++a)
        for (int b = 0; a + b <= d; ++b) multi[graded_index(a, b, d - a - b)] = make_int4(a, b, d - a - b, d);
    auto factorial = [](int n) {
      double f = 1.0;
      for (int i = 2; i <= n; ++i) f *= i;
      return f;
    };
    for (const int4& m : multi) {
      fact.push_back(factorial(m.x) * factorial(m.y) * factorial(m.z));
      inv_fact.push_back(1.0 / fact.back());
      sign.push_back(m.w % 2 == 0 ? 1.0 : -1.0);
    }
    // Derivatives of 1/r by r^2 d_k f = -(...) along one axis i with k_i >= 1:
    // the axis with the largest component (lowest index among equals); each
    // entry lists k_j and the positions of k - e_j and k - 2 e_j per axis.
    rec_axis.assign(n_d, 0);
    rec_delta.assign(3 * n_d, 0);
    rec_m1.assign(3 * n_d, -1);
    rec_m2.assign(3 * n_d, -1);
    for (int k = 1; k < n_d; ++k) {
      const int m[3] = {multi[k].x, multi[k].y, multi[k].z};
      int axis = 0;
      for (int j = 1; j < 3; ++j)
        if (m[j] > m[axis]) axis = j;
      rec_axis[k] = axis;
      for (int j = 0; j < 3; ++j) {
        rec_delta[3 * k + j] = m[j];
        int t[3] = {m[0], m[1], m[2]};
        t[j] -= 1;
        if (m[j] >= 1) rec_m1[3 * k + j] = pos(t);
        t[j] -= 1;
        if (m[j] >= 2) rec_m2[3 * k + j] = pos(t);
      }
    }
    // M2L: D_{g+a}; transposed copy for the class products
    m2l_index.resize(static_cast<size_t>(n_m) * n_m);
    m2l_index_t.resize(static_cast<size_t>(n_m) * n_m);
    for (int g = 0; g < n_m; ++g)
      for (int a = 0; a < n_m; ++a) {
        const int s3[3] = {multi[g].x + multi[a].x, multi[g].y + multi[a].y, multi[g].z + multi[a].z};
        m2l_index[static_cast<size_t>(g) * n_m + a] = pos(s3);
        m2l_index_t[static_cast<size_t>(a) * n_m + g] = static_cast<short>(pos(s3));
      }
    // M2M (child -> parent): M_a += M_b * d^(a-b) / (a-b)! over b <= a;
    // L2L (parent -> child): L_a += L_b * (b!/a!) d^(b-a) / (b-a)! over b >= a
    // with |b| <= p. Both enumerated componentwise.
    m2m_off.push_back(0);
    l2l_off.push_back(0);
    for (int a = 0; a < n_m; ++a) {
      const int4 ma = multi[a];
      for (int b0 = 0; b0 <= ma.x; ++b0)
        for (int b1 = 0; b1 <= ma.y; ++b1)
          for (int b2 = 0; b2 <= ma.z; ++b2) {
            m2m_b.push_back(graded_index(b0, b1, b2));
            m2m_c.push_back(graded_index(ma.x - b0, ma.y - b1, ma.z - b2));
          }
      m2m_off.push_back(static_cast<int>(m2m_b.size()));
      for (int c = 0; c < n_m; ++c) {
        const int4 mc = multi[c];
        if (ma.w + mc.w > p) break;  // graded order: every later c has a higher degree
        l2l_b.push_back(graded_index(ma.x + mc.x, ma.y + mc.y, ma.z + mc.z));
        l2l_c.push_back(c);
      }
      l2l_off.push_back(static_cast<int>(l2l_b.size()));
    }
    // gradient of the local expansion: d/dx_k of x^g is g_k x^(g - e_k)
    grad.assign(3 * n_m, -1);
    for (int g = 0; g < n_m; ++g) {
      const int m[3] = {multi[g].x, multi[g].y, multi[g].z};
      for (int k = 0; k < 3; ++k)
        if (m[k] >= 1) {
          int t[3] = {m[0], m[1], m[2]};
          t[k] -= 1;
          grad[3 * g + k] = pos(t);
        }
    }
  }
};

// Device copy of one order's tables.
struct FmmDevTables {
  int p, n_m, n_d;
  const int4* multi;
  const double* fact;
  const double* inv_fact;
  const double* sign;
  const int* deg_start;
  const int* rec_axis;
  const int* rec_delta;
  const int* rec_m1;
  const int* rec_m2;
  const int* m2l_index;
  const short* m2l_index_t;
  const int* m2m_off;
  const int* m2m_b;
  const int* m2m_c;
  const int* l2l_off;
  const int* l2l_b;
  const int* l2l_c;
  const int* grad;
};

struct FmmLists {
  DevBuf cur, next, m2l, p2p;
  // list lengths the last traversal needed (the next one reserves them)
  long need_front = 0, need_m2l = 0, need_p2p = 0;
};

struct Fmm {
  std::map<int, std::pair<DevBuf*, FmmDevTables>> tables;
  FmmLists lists;
  DevBuf m2l_out[2];  // per-pair M2L products of two chunks in flight
  // the per-target M2L sums of one chunk run on `side` while the products
  // of the next chunk run on the context stream
  cudaStream_t side = nullptr;
  cudaEvent_t products_done[2] = {nullptr, nullptr}, sums_done[2] = {nullptr, nullptr};
  // FP32 near field (tensor mode): its pair kernel runs on `near` after the
  // last M2L products, concurrently with the per-target sums and L2L
  cudaStream_t near = nullptr;
  cudaEvent_t near_start = nullptr, near_done = nullptr;
  // P2M / M2M run on `up` concurrently with the traversal, which needs only
  // the cell radii
  cudaStream_t up = nullptr;
  cudaEvent_t up_start = nullptr, up_done = nullptr;
  // statistics of the last evaluation (amk_fmm_stats)
  long stats[11] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  ~Fmm() {
    for (auto& kv : tables) delete kv.second.first;
    for (int i = 0; i < 2; ++i) {
      if (products_done[i]) cudaEventDestroy(products_done[i]);
      if (sums_done[i]) cudaEventDestroy(sums_done[i]);
    }
    if (near_start) cudaEventDestroy(near_start);
    if (near_done) cudaEventDestroy(near_done);
    if (near) cudaStreamDestroy(near);
    if (side) cudaStreamDestroy(side);
    if (up_start) cudaEventDestroy(up_start);
    if (up_done) cudaEventDestroy(up_done);
    if (up) cudaStreamDestroy(up);
  }
};

namespace {

constexpr int kMaxOrder = 8;
constexpr int kMaxNm = 165;  // n_m(8)
constexpr int kFmmWarps = 4;

template <typename T>
size_t append(std::vector<char>& blob, const std::vector<T>& v) {
  while (blob.size() % 16) blob.push_back(0);
  const size_t off = blob.size();
  const char* p = reinterpret_cast<const char*>(v.data());
  blob.insert(blob.end(), p, p + v.size() * sizeof(T));
  return off;
}

int get_tables(amk_ctx* c, int order, FmmDevTables* out) {
  if (!c->fmm) c->fmm = new Fmm();
  auto it = c->fmm->tables.find(order);
  if (it != c->fmm->tables.end()) {
    *out = it->second.second;
    return AMK_OK;
  }
  FmmHostTables h(order);
  std::vector<char> blob;
  const size_t o_multi = append(blob, h.multi), o_fact = append(blob, h.fact), o_if = append(blob, h.inv_fact),
               o_sign = append(blob, h.sign), o_ds = append(blob, h.deg_start), o_ax = append(blob, h.rec_axis),
               o_de = append(blob, h.rec_delta), o_m1 = append(blob, h.rec_m1), o_m2 = append(blob, h.rec_m2),
               o_idx = append(blob, h.m2l_index), o_idt = append(blob, h.m2l_index_t), o_mo = append(blob, h.m2m_off), o_mb = append(blob, h.m2m_b),
               o_mc = append(blob, h.m2m_c), o_lo = append(blob, h.l2l_off), o_lb = append(blob, h.l2l_b),
               o_lc = append(blob, h.l2l_c), o_g = append(blob, h.grad);
  DevBuf* buf = new DevBuf();
  int rc = buf->reserve(blob.size());
  if (rc != AMK_OK) {
    delete buf;
    return rc;
  }
  AMK_CUDA_TRY(cudaMemcpy(buf->ptr, blob.data(), blob.size(), cudaMemcpyHostToDevice));
  const char* b = static_cast<const char*>(buf->ptr);
  FmmDevTables t;
  t.p = h.p;
  t.n_m = h.n_m;
  t.n_d = h.n_d;
  t.multi = reinterpret_cast<const int4*>(b + o_multi);
  t.fact = reinterpret_cast<const double*>(b + o_fact);
  t.inv_fact = reinterpret_cast<const double*>(b + o_if);
  t.sign = reinterpret_cast<const double*>(b + o_sign);
  t.deg_start = reinterpret_cast<const int*>(b + o_ds);
  t.rec_axis = reinterpret_cast<const int*>(b + o_ax);
  t.rec_delta = reinterpret_cast<const int*>(b + o_de);
  t.rec_m1 = reinterpret_cast<const int*>(b + o_m1);
  t.rec_m2 = reinterpret_cast<const int*>(b + o_m2);
  t.m2l_index = reinterpret_cast<const int*>(b + o_idx);
  t.m2l_index_t = reinterpret_cast<const short*>(b + o_idt);
  t.m2m_off = reinterpret_cast<const int*>(b + o_mo);
  t.m2m_b = reinterpret_cast<const int*>(b + o_mb);
  t.m2m_c = reinterpret_cast<const int*>(b + o_mc);
  t.l2l_off = reinterpret_cast<const int*>(b + o_lo);
  t.l2l_b = reinterpret_cast<const int*>(b + o_lb);
  t.l2l_c = reinterpret_cast<const int*>(b + o_lc);
  t.grad = reinterpret_cast<const int*>(b + o_g);
  c->fmm->tables[order] = {buf, t};
  *out = t;
  return AMK_OK;
}

// powers x^i, y^i, z^i for i <= p, then mono[k] = x^a y^b z^c (Monomials,
// fast-multipole.cc:190-204)
__device__ __forceinline__ void powers(int p, double x, double y, double z, double* px, double* py, double* pz) {
  px[0] = py[0] = pz[0] = 1.0;
  for (int i = 1; i <= p; ++i) {
    px[i] = px[i - 1] * x;
    py[i] = py[i - 1] * y;
    pz[i] = pz[i - 1] * z;
  }
}

// ------------------------------------------------------------ radii
__global__ void fmm_leaf_radius_kernel(const Octree t, double* __restrict__ radius) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= t.n_nodes || !t.meta[id].y) return;
  const double4 c = t.center[id];
  const int2 r = t.range[id];
  double r2 = 0.0;
  for (int k = r.x; k < r.y; ++k) {
    const double4 s = t.src[k];
    const double dx = s.x - c.x, dy = s.y - c.y, dz = s.z - c.z;
    r2 = fmax(r2, __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
  }
  radius[id] = sqrt(r2);
}

__global__ void fmm_parent_radius_kernel(const Octree t, int depth, double* __restrict__ radius) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= t.n_nodes) return;
  const uchar2 mt = t.meta[id];
  if (mt.y || mt.x != depth) return;
  const double4 c = t.center[id];
  double r = 0.0;
  for (int o = 0; o < 8; ++o) {
    const int ch = t.child[8 * id + o];
    if (ch < 0) continue;
    const double4 cc = t.center[ch];
    const double dx = cc.x - c.x, dy = cc.y - c.y, dz = cc.z - c.z;
    r = fmax(r, sqrt(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz))) + radius[ch]);
  }
  radius[id] = r;
}

// ------------------------------------------------------------ P2M, M2M
// P2M (fast-multipole.cc:443-461): M_a = sum_j q_j d_j^a / a!, d_j = x_j - c.
// A warp per leaf; lanes over particles (up to kP2mPer per lane per round).
// The multi-indices a are visited in the lexicographic order of three
// nested loops with running powers, so each monomial of each particle costs
// one multiply; the lanes' partial sums of a coefficient are added by a
// shuffle tree (fixed order: run-to-run deterministic) and lane 0 keeps the
// leaf's sums in shared memory across rounds.
constexpr int kP2mPer = 4;

__global__ void __launch_bounds__(32 * kFmmWarps)
fmm_p2m_kernel(const Octree t, FmmDevTables T, double* __restrict__ M) {
  __shared__ double acc_s[kFmmWarps][kMaxNm];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int id = blockIdx.x * kFmmWarps + w;
  if (id >= t.n_nodes || !t.meta[id].y) return;
  const double4 c = t.center[id];
  const int2 r = t.range[id];
  const int P = T.p;
  double* acc = acc_s[w];
  for (int a = lane; a < T.n_m; a += 32) acc[a] = 0.0;
  __syncwarp();
  for (int r0 = r.x; r0 < r.y; r0 += 32 * kP2mPer) {
    double dx[kP2mPer], dy[kP2mPer], dz[kP2mPer], qx[kP2mPer];
#pragma unroll
    for (int u = 0; u < kP2mPer; ++u) {
      const int k = r0 + lane + 32 * u;
      const double4 s = k < r.y ? t.src[k] : make_double4(c.x, c.y, c.z, 0.0);
      dx[u] = s.x - c.x;
      dy[u] = s.y - c.y;
      dz[u] = s.z - c.z;
      qx[u] = s.w;  // q x^i, running
    }
    for (int i = 0; i <= P; ++i) {
      double qy[kP2mPer];
#pragma unroll
      for (int u = 0; u < kP2mPer; ++u) qy[u] = qx[u];  // q x^i y^j, running
      for (int j = 0; i + j <= P; ++j) {
        double m[kP2mPer];
#pragma unroll
        for (int u = 0; u < kP2mPer; ++u) m[u] = qy[u];  // q x^i y^j z^k, running
        for (int k = 0; i + j + k <= P; ++k) {
          double v = 0.0;
#pragma unroll
          for (int u = 0; u < kP2mPer; ++u) {
            v += m[u];
            m[u] *= dz[u];
          }
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
          if (lane == 0) acc[graded_index(i, j, k)] += v;
        }
#pragma unroll
        for (int u = 0; u < kP2mPer; ++u) qy[u] *= dy[u];
      }
#pragma unroll
      for (int u = 0; u < kP2mPer; ++u) qx[u] *= dx[u];
    }
  }
  __syncwarp();
  for (int a = lane; a < T.n_m; a += 32) M[static_cast<size_t>(id) * T.n_m + a] = acc[a] * T.inv_fact[a];
}

// M2M for parents at `depth` (fast-multipole.cc:463-482). A warp per
// parent, lanes over the parent's coefficients; per child the lanes first
// write the offset's monomials d^c / c! (c over all multi-indices) into
// shared memory, then each term of coefficient a is one product
// M_child[b] * mono[a - b] with b and a - b from the table.
__global__ void __launch_bounds__(32 * kFmmWarps)
fmm_m2m_kernel(const Octree t, FmmDevTables T, int depth, double* __restrict__ M) {
  __shared__ double mono_s[kFmmWarps][kMaxNm];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int id = blockIdx.x * kFmmWarps + w;
  if (id >= t.n_nodes) return;
  const uchar2 mt = t.meta[id];
  if (mt.y || mt.x != depth) return;
  const double4 c = t.center[id];
  double* mono = mono_s[w];
  double acc[(kMaxNm + 31) / 32];
  for (int u = 0; u < (kMaxNm + 31) / 32; ++u) acc[u] = 0.0;
  double px[kMaxOrder + 1], py[kMaxOrder + 1], pz[kMaxOrder + 1];
  for (int o = 0; o < 8; ++o) {
    const int ch = t.child[8 * id + o];
    if (ch < 0) continue;
    const double4 cc = t.center[ch];
    powers(T.p, cc.x - c.x, cc.y - c.y, cc.z - c.z, px, py, pz);
    __syncwarp();  // the previous child's monomials are no longer read
    for (int a = lane; a < T.n_m; a += 32) {
      const int4 m = T.multi[a];
      mono[a] = (px[m.x] * py[m.y] * pz[m.z]) * T.inv_fact[a];
    }
    __syncwarp();
    const double* mc = M + static_cast<size_t>(ch) * T.n_m;
    for (int u = 0, a = lane; a < T.n_m; ++u, a += 32) {
      double s = acc[u];
      for (int e = T.m2m_off[a]; e < T.m2m_off[a + 1]; ++e) s += mc[T.m2m_b[e]] * mono[T.m2m_c[e]];
      acc[u] = s;
    }
  }
  for (int u = 0, a = lane; a < T.n_m; ++u, a += 32) M[static_cast<size_t>(id) * T.n_m + a] = acc[u];
}

// ------------------------------------------------------------ dual traversal
// One level of the dual-tree recursion (fast-multipole.cc:484-526): each
// pair is accepted for M2L, kept for P2P, or split into its children. The
// emissions of a warp are reserved with one atomic per list (ballot / warp
// prefix sums); the order of the lists is irrelevant, they are sorted after.
// The level's pair count is read on the device (lv[0]), the children are
// counted into lv[1]; a slot past a list's capacity is not written and
// raises cnt[2], so the host can grow the lists and run the traversal again
// (counts keep growing past the capacity, and every slot below it is
// written). A pair that is not a pair of nodes raises cnt[3] and is
// skipped. Warps stride over the level's pairs, so one grid size serves
// every level.
// Per node, what the traversal reads of it in one 32-byte record: the
// centre and the radius, negated for a leaf (a leaf of radius 0 stores -0.0;
// the sign bit is the leaf flag, the magnitude the radius).
__global__ void fmm_node_record_kernel(const Octree t, const double* __restrict__ radius,
                                       double4* __restrict__ rec) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= t.n_nodes) return;
  const double4 c = t.center[id];
  const double r = radius[id];
  rec[id] = make_double4(c.x, c.y, c.z, t.meta[id].y ? -r : r);
}

__global__ void fmm_traverse_root_kernel(int2* __restrict__ cur, int* __restrict__ lv) {
  if (threadIdx.x == 0) {
    cur[0] = make_int2(0, 0);
    lv[0] = 1;
  }
}

struct TraverseLists {
  int2* m2l;
  int2* p2p;
  long cap_m2l, cap_p2p, cap_front;
};

__global__ void fmm_traverse_kernel(const Octree t, const double4* __restrict__ rec, double theta2,
                                    const int2* __restrict__ cur, int2* __restrict__ next, TraverseLists out,
                                    int* __restrict__ lv, int* __restrict__ cnt) {
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  const long n_cur = min(static_cast<long>(lv[0]), out.cap_front);
  const long warp0 = (blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x) >> 5;
  const long n_warps = (static_cast<long>(gridDim.x) * blockDim.x) >> 5;
  for (long base = warp0 * 32; base < n_cur; base += n_warps * 32) {
    const long i = base + lane;
    int2 pr = make_int2(0, 0);
    int kind = -1;  // 0 M2L, 1 P2P, 2 split
    int kids[8], nk = 0;
    bool split_target = false;
    if (i < n_cur) pr = cur[i];
    if (i < n_cur && (static_cast<unsigned>(pr.x) >= static_cast<unsigned>(t.n_nodes) ||
                      static_cast<unsigned>(pr.y) >= static_cast<unsigned>(t.n_nodes))) {
      cnt[3] = 1;  // not a node pair: recorded and skipped
    } else if (i < n_cur) {
      const int ti = pr.x, si = pr.y;
      const double4 tc = rec[ti], sc = rec[si];
      const double dx = tc.x - sc.x, dy = tc.y - sc.y, dz = tc.z - sc.z;
      const double dist2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
      const double rt = fabs(tc.w), rs = fabs(sc.w);
      const double rsum = rt + rs;
      if (__dmul_rn(rsum, rsum) < __dmul_rn(theta2, dist2)) {
        kind = 0;
      } else {
        const bool tleaf = signbit(tc.w), sleaf = signbit(sc.w);
        if (tleaf && sleaf) {
          kind = 1;
        } else {
          kind = 2;
          split_target = sleaf || (!tleaf && rt >= rs);
          const int node = split_target ? ti : si;
          for (int o = 0; o < 8; ++o) {
            const int ch = t.child[8 * node + o];
            if (ch >= 0) kids[nk++] = ch;
          }
        }
      }
    }
    // M2L and P2P: one slot per lane
    for (int list = 0; list < 2; ++list) {
      const unsigned m = __ballot_sync(0xffffffffu, kind == list);
      if (m == 0) continue;
      int b = 0;
      if (lane == __ffs(m) - 1) b = atomicAdd(&cnt[list], __popc(m));
      b = __shfl_sync(0xffffffffu, b, __ffs(m) - 1);
      const long slot = static_cast<long>(b) + __popc(m & below);
      if (kind == list) {
        if (slot < (list == 0 ? out.cap_m2l : out.cap_p2p))
          (list == 0 ? out.m2l : out.p2p)[slot] = pr;
        else
          cnt[2] = 1;
      }
    }
    // children: a warp prefix sum of the counts
    int incl = nk;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    if (total == 0) continue;
    int b = 0;
    if (lane == 31) b = atomicAdd(&lv[1], total);
    const long first = static_cast<long>(__shfl_sync(0xffffffffu, b, 31)) + incl - nk;
    // every slot below the capacity is written (the reservations are
    // contiguous), so the next level reads only pairs of this one
    for (int k = 0; k < nk; ++k) {
      if (first + k < out.cap_front)
        next[first + k] = split_target ? make_int2(kids[k], pr.y) : make_int2(pr.x, kids[k]);
      else
        cnt[2] = 1;
    }
  }
}

// Group pairs by target: pack (target, source) into one key and radix-sort
// it, so each target's sources are contiguous and in ascending source order
// (a fixed summation order, independent of the emission order).
__global__ void pair_pack_kernel(const int2* __restrict__ pairs, int n, int bits, uint64_t* __restrict__ keys,
                                 uint32_t* __restrict__ vals) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int2 p = pairs[i];
  keys[i] = (static_cast<uint64_t>(p.x) << bits) | static_cast<uint64_t>(p.y);
  vals[i] = static_cast<uint32_t>(i);
}

// Sorted keys: a warp's lanes with the same target add their count once.
__global__ void pair_unpack_kernel(const uint64_t* __restrict__ keys, int n, int bits, int* __restrict__ src,
                                   int* __restrict__ count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  int target = -1;
  if (i < n) {
    const uint64_t k = keys[i];
    src[i] = static_cast<int>(k & ((1ull << bits) - 1ull));
    target = static_cast<int>(k >> bits);
  }
  const unsigned same = __match_any_sync(0xffffffffu, target);
  if (target >= 0 && lane == __ffs(same) - 1) atomicAdd(&count[target], __popc(same));
}

struct Grouped {
  int* off = nullptr;
  int* count = nullptr;
  int* src = nullptr;
};

// ------------------------------------------------------------ M2L
// L_g(t) = 1/g! sum_a (-1)^|a| M_a(s) D_{g+a}(c_t - c_s) for every M2L pair
// (fast-multipole.cc:528-555), evaluated as dense products per displacement
// class.
//
// Cube centres lie on a lattice: for a pair with depths d_t, d_s and half
// edges h_t, h_s, c_t - c_s = u v with u = min(h_t, h_s) and v an integer
// vector (up to the rounding of the centres, ~1e-15 relative). D is
// homogeneous, D_k(u v) = u^{-|k|-1} D_k(v), so with per-cell rescaled
// expansions
//     Mh_a(s) = (-1)^|a| M_a(s) h_s^{-|a|},   L_g(t) = h_t^{-|g|-1} Lh_g(t)
// a pair contributes Lh(t) += A_{v,dd} Mh(s) with the n_m x n_m matrix
//     A_{v,dd}[g][a] = 1/g! (h_t/u)^{|g|+1} (h_s/u)^{|a|} D_{g+a}(v),
// which depends only on the class (v, dd = d_t - d_s): h_t/u and h_s/u are
// powers of two. Pairs are sorted by class and each class is one FP64
// product A (n_m x n_m) x [Mh of its sources] (n_m x k), in tiles of 64
// pairs, up to 8 tiles of one class per block. The products are written per pair and summed per target in the
// pairs' (target, source) order, so the result is run-to-run deterministic.
// A class is found through an open-addressing hash of (d_t - d_s, v) with
// bounded probing; pairs off the lattice, beyond the class reach or left
// without a hash slot take a per-pair path with the derivative recurrence.
// The pairs are processed in chunks that bound the per-pair scratch.
constexpr int kM2lTileP = 64;      // pairs per product tile
constexpr int kM2lUnitTiles = 8;   // tiles of one class per block
constexpr int kM2lUnitPairs = kM2lUnitTiles * kM2lTileP;
// classes below this size take the per-pair path in both precision modes (in
// tensor-core mode a class-matrix build per tiny class costs more than the
// per-pair path: measured at 1,048,576 particles, leaf 128)
constexpr int kM2lMinClass = 4;
constexpr size_t kM2lChunkBytes = size_t(4) << 30;  // per-pair products of one chunk
// tensor-core mode: larger chunks (a class split across chunks costs one
// more class-matrix build per chunk; two buffers of this size at most)
constexpr size_t kM2lTcChunkBytes = size_t(12) << 30;
constexpr int kM2lHashBits = 21;
constexpr long kM2lHashSlots = 1L << kM2lHashBits;
constexpr int kM2lHashProbes = 64;
constexpr int kM2lVBias = 1 << 18;             // v components biased into 19 bits
constexpr int kM2lMaxReach = kM2lVBias - 1;    // |v_i| covered by the classes
constexpr unsigned long long kM2lEmpty = ~0ull;

__host__ __device__ __forceinline__ unsigned long long m2l_key(int dd, int vx, int vy, int vz) {
  return (static_cast<unsigned long long>(dd + 32) << 57) |
         (static_cast<unsigned long long>(vx + kM2lVBias) << 38) |
         (static_cast<unsigned long long>(vy + kM2lVBias) << 19) | static_cast<unsigned long long>(vz + kM2lVBias);
}
__device__ __forceinline__ int m2l_key_dd(unsigned long long k) { return static_cast<int>(k >> 57) - 32; }
__device__ __forceinline__ int m2l_key_v(unsigned long long k, int axis) {
  return static_cast<int>((k >> (38 - 19 * axis)) & ((1u << 19) - 1)) - kM2lVBias;
}

// Class key of a pair, kM2lEmpty = off the lattice or out of reach. The
// centres are sums of power-of-two fractions of the root half edge, rounded
// to FP64 at every level, so a lattice offset v carries a rounding error of
// a few dozen ulp of max|c| / u; the acceptance tolerance tracks that bound
// (256 ulp), and a pair further off the lattice takes the per-pair path,
// where D is built from the actual centres as in the reference.
__device__ __forceinline__ unsigned long long m2l_class_key(const Octree& t, int ti, int si, int reach, bool fold,
                                                            int* refl) {
  const double4 tc = t.center[ti], sc = t.center[si];
  const int dd = static_cast<int>(t.meta[ti].x) - static_cast<int>(t.meta[si].x);
  const double u = fmin(tc.w, sc.w);
  const double vx = (tc.x - sc.x) / u, vy = (tc.y - sc.y) / u, vz = (tc.z - sc.z) / u;
  const double rx = rint(vx), ry = rint(vy), rz = rint(vz);
  const double cmax = fmax(fmax(fmax(fabs(tc.x), fabs(tc.y)), fmax(fabs(tc.z), fabs(sc.x))),
                           fmax(fabs(sc.y), fabs(sc.z)));
  const double tol = 256.0 * 2.220446049250313e-16 * (cmax / u + fabs(rx) + fabs(ry) + fabs(rz) + 1.0);
  if (fabs(vx - rx) > tol || fabs(vy - ry) > tol || fabs(vz - rz) > tol) return kM2lEmpty;
  if (fabs(rx) > reach || fabs(ry) > reach || fabs(rz) > reach) return kM2lEmpty;
  int ix = static_cast<int>(rx), iy = static_cast<int>(ry), iz = static_cast<int>(rz), r = 0;
  if (fold) {  // the class of |v|; the reflection that maps |v| to v in bits x, y, z
    if (ix < 0) ix = -ix, r |= 1;
    if (iy < 0) iy = -iy, r |= 2;
    if (iz < 0) iz = -iz, r |= 4;
  }
  *refl = r;
  return m2l_key(dd, ix, iy, iz);
}

// Slot of a key in the class hash (inserted if absent), -1 if no slot
// within the probe limit.
__device__ __forceinline__ int m2l_hash_slot(unsigned long long* keys, unsigned long long key) {
  unsigned long long h = key;  // splitmix64 finaliser
  h = (h ^ (h >> 30)) * 0xbf58476d1ce4e5b9ull;
  h = (h ^ (h >> 27)) * 0x94d049bb133111ebull;
  h ^= h >> 31;
  long slot = static_cast<long>(h & (kM2lHashSlots - 1));
  for (int probe = 0; probe < kM2lHashProbes; ++probe) {
    const unsigned long long k = keys[slot];
    if (k == key) return static_cast<int>(slot);
    if (k == kM2lEmpty) {
      const unsigned long long old = atomicCAS(keys + slot, kM2lEmpty, key);
      if (old == kM2lEmpty || old == key) return static_cast<int>(slot);
    }
    slot = (slot + 1) & (kM2lHashSlots - 1);
  }
  return -1;
}

// Mh[s][a] = (-1)^|a| M[s][a] h_s^{-|a|}
__global__ void m2l_rescale_kernel(const Octree t, FmmDevTables T, const double* __restrict__ M,
                                   double* __restrict__ Mh) {
  const long e = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  if (e >= t.n_nodes * T.n_m) return;
  const int s = static_cast<int>(e / T.n_m), a = static_cast<int>(e - static_cast<long>(s) * T.n_m);
  const double ih = 1.0 / t.center[s].w;
  double f = T.sign[a];
  for (int d = 0; d < T.multi[a].w; ++d) f *= ih;
  Mh[e] = M[e] * f;
}

// Class slot (-1: per-pair path) and target of every pair (a warp per target);
// refl (tensor-core mode) is cleared: every pair starts unreflected.
__global__ void m2l_classify_kernel(const Octree t, const int* __restrict__ off, const int* __restrict__ count,
                                    const int* __restrict__ src, int reach, unsigned long long* __restrict__ keys,
                                    int* __restrict__ codes, int* __restrict__ tgt,
                                    unsigned char* __restrict__ refl) {
  const int lane = threadIdx.x & 31;
  const long w0 = (blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x) >> 5;
  const long nw = (static_cast<long>(gridDim.x) * blockDim.x) >> 5;
  for (long ti = w0; ti < t.n_nodes; ti += nw) {
    const int b = off[ti], n = count[ti];
    for (int e = b + lane; e < b + n; e += 32) {
      int r = 0;
      const unsigned long long key = m2l_class_key(t, static_cast<int>(ti), src[e], reach, false, &r);
      codes[e] = key == kM2lEmpty ? -1 : m2l_hash_slot(keys, key);
      tgt[e] = static_cast<int>(ti);
      if (refl) refl[e] = 0;
    }
  }
}

// Tensor-core mode: a pair of a class smaller than min_class (over all
// pairs) is moved to the class of |v| with its reflection in refl[e] (bit i:
// v_i < 0). D is even in each coordinate, D_k(R w) = s^k D_k(w) with
// s^k = prod_i s_i^k_i, so the class matrix of v is S_g A(|v|) S_a: the
// source expansion is read with the signs s^a (a sign-flipped copy of its
// split rows) and the product's row g gets s^g (m2l_refl_sign_kernel).
// Folding the 8 reflections merges most of the small classes into classes
// large enough for a class product (or into the class of |v| itself when
// that one exists), while the pairs of large classes keep their own.
__global__ void m2l_refold_kernel(const Octree t, const int* __restrict__ hist, int min_class,
                                  const int* __restrict__ tgt, const int* __restrict__ src, int reach, long n,
                                  unsigned long long* __restrict__ keys, int* __restrict__ codes,
                                  unsigned char* __restrict__ refl) {
  const long e = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  if (e >= n) return;
  const int code = codes[e];
  if (code < 0 || hist[code] >= min_class) return;
  int r = 0;
  const unsigned long long key = m2l_class_key(t, tgt[e], src[e], reach, true, &r);
  if (key == kM2lEmpty || r == 0) return;
  const int folded = m2l_hash_slot(keys, key);
  if (folded < 0) return;  // no slot: the pair stays in its own (small) class
  codes[e] = folded;
  refl[e] = static_cast<unsigned char>(r);
}

// Pairs per class code over all pairs (tensor-core mode, before folding).
__global__ void m2l_code_count_kernel(const int* __restrict__ codes, long n, int* __restrict__ hist) {
  const long e = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  if (e < n && codes[e] >= 0) atomicAdd(hist + codes[e], 1);
}

// Pairs per class code in [e0, e1); off-lattice pairs listed for the per-pair path.
__global__ void m2l_histogram_kernel(const int* __restrict__ codes, long e0, long e1, int* __restrict__ hist,
                                     int* __restrict__ fallback, int* __restrict__ n_fallback) {
  const long e = e0 + blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  if (e >= e1) return;
  const int code = codes[e];
  if (code >= 0)
    atomicAdd(hist + code, 1);
  else
    fallback[atomicAdd(n_fallback, 1)] = static_cast<int>(e);
}

// Classes of fewer than min_class pairs go the per-pair path; their counts
// are cleared, so the scan of hist places the pairs of the classes taken
// contiguously at the start of the chunk's permutation.
__global__ void m2l_code_flags_kernel(int* __restrict__ hist, long n_codes, int min_class,
                                      int* __restrict__ used, int* __restrict__ units) {
  const long code = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  if (code >= n_codes) return;
  const int n = hist[code];
  const bool take = n > 0 && n >= min_class;
  used[code] = take;
  units[code] = take ? (n + kM2lUnitPairs - 1) / kM2lUnitPairs : 0;
  if (!take) hist[code] = 0;
}

// Class list and product units (<= 8 tiles of one class) from the scanned
// per-code counts.
__global__ void m2l_class_fill_kernel(const int* __restrict__ hist, const int* __restrict__ start,
                                      const int* __restrict__ cls_index, const int* __restrict__ unit_start,
                                      long n_codes, const int* __restrict__ used, int* __restrict__ cls_code,
                                      int* __restrict__ cls_end, int* __restrict__ unit_cls,
                                      int* __restrict__ unit_pos) {
  const long code = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  if (code >= n_codes) return;
  const int n = hist[code];
  if (!used[code]) return;
  const int cls = cls_index[code];
  cls_code[cls] = static_cast<int>(code);
  cls_end[cls] = start[code] + n;
  const int nu = (n + kM2lUnitPairs - 1) / kM2lUnitPairs;
  for (int k = 0; k < nu; ++k) {
    unit_cls[unit_start[code] + k] = cls;
    unit_pos[unit_start[code] + k] = start[code] + k * kM2lUnitPairs;
  }
}

// Pair positions grouped by class (order inside a class is irrelevant: every
// pair's product is computed on its own); pairs of small classes join the
// per-pair list. Consumes hist.
__global__ void m2l_scatter_kernel(const int* __restrict__ codes, long e0, long e1, const int* __restrict__ start,
                                   const int* __restrict__ used, int* __restrict__ hist, int* __restrict__ perm,
                                   int* __restrict__ fallback, int* __restrict__ n_fallback,
                                   unsigned char* __restrict__ refl) {
  const long e = e0 + blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  if (e >= e1) return;
  const int code = codes[e];
  if (code < 0) return;
  if (used[code]) {
    perm[start[code] + atomicSub(hist + code, 1) - 1] = static_cast<int>(e);
  } else {
    fallback[atomicAdd(n_fallback, 1)] = static_cast<int>(e);
    if (refl) refl[e] = 0;  // the per-pair path works from the actual centres
  }
}

// D recurrence (fast-multipole.cc:207-232) for displacement xs into D[0, n_d), one warp.
__device__ __forceinline__ void m2l_derivatives(const FmmDevTables& T, int lane, const double xs[3], double* D) {
  const double inv_r2 = 1.0 / (xs[0] * xs[0] + xs[1] * xs[1] + xs[2] * xs[2]);
  if (lane == 0) D[0] = sqrt(inv_r2);
  __syncwarp();
  for (int deg = 1; deg <= 2 * T.p; ++deg) {
    for (int k = T.deg_start[deg] + lane; k < T.deg_start[deg + 1]; k += 32) {
      const int i = T.rec_axis[k];
      const int di = T.rec_delta[3 * k + i];
      double sum = (2 * di - 1) * xs[i] * D[T.rec_m1[3 * k + i]];
      if (T.rec_m2[3 * k + i] >= 0) sum += (di - 1) * (di - 1) * D[T.rec_m2[3 * k + i]];
      for (int j = 0; j < 3; ++j) {
        const int dj = T.rec_delta[3 * k + j];
        if (j == i || dj == 0) continue;
        sum += 2.0 * dj * xs[j] * D[T.rec_m1[3 * k + j]];
        if (T.rec_m2[3 * k + j] >= 0) sum += dj * (dj - 1) * D[T.rec_m2[3 * k + j]];
      }
      D[k] = -sum * inv_r2;
    }
    __syncwarp();
  }
}

__device__ __forceinline__ void split3_bf16(double v, __nv_bfloat16* t);

// D(v) of every class: a warp per class, into table[class * n_d + k], or
// (tensor-core mode, table3 given) split into three BF16 terms packed as
// {t0 | t1 << 16, t2} into table3[class * nd3 + k], zero for k >= n_d.
__global__ void __launch_bounds__(32 * kFmmWarps)
m2l_table_kernel(FmmDevTables T, const int* __restrict__ cls_code, int n_classes,
                 const unsigned long long* __restrict__ keys, double* __restrict__ table,
                 uint2* __restrict__ table3, int nd3) {
  extern __shared__ __align__(16) unsigned char tab_smem[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double* D = reinterpret_cast<double*>(tab_smem) + static_cast<size_t>(w) * T.n_d;
  const int cls = blockIdx.x * kFmmWarps + w;
  if (cls >= n_classes) return;
  const unsigned long long key = keys[cls_code[cls]];
  const double xs[3] = {static_cast<double>(m2l_key_v(key, 0)), static_cast<double>(m2l_key_v(key, 1)),
                        static_cast<double>(m2l_key_v(key, 2))};
  m2l_derivatives(T, lane, xs, D);
  if (table3 == nullptr) {
    for (int k = lane; k < T.n_d; k += 32) table[static_cast<size_t>(cls) * T.n_d + k] = D[k];
    return;
  }
  for (int k = lane; k < nd3; k += 32) {
    __nv_bfloat16 t3[3];
    split3_bf16(k < T.n_d ? D[k] : 0.0, t3);
    table3[static_cast<size_t>(cls) * nd3 + k] =
        make_uint2(static_cast<uint32_t>(__bfloat16_as_ushort(t3[0])) |
                       (static_cast<uint32_t>(__bfloat16_as_ushort(t3[1])) << 16),
                   __bfloat16_as_ushort(t3[2]));
  }
}

constexpr int kM2lBs = kM2lTileP + 2;   // B row stride (doubles): 16-byte rows, 2-way store conflicts
constexpr int kM2lStages = 3;           // B pipeline depth (k chunks)

__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool valid) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  const int n = valid ? 8 : 0;  // 0: zero fill, nothing read
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Tensor-core form of the class product: mma.m8n8k4 with FP64 operands
// (256 FMAs per warp instruction, the same FP64 rate as FMA instructions but
// an eighth of the issue slots). A block covers 8 * kGb >= n_m rows and 64
// pairs; warp (wr, wc) owns kWr x kWc 8 x 8 output tiles. A fragments are
// gathered from the class's D(v) through the transposed index map (both in
// shared memory) and scaled by the source factor; B fragments come from the
// cp.async pipeline ([k][pair] rows, k padded to a multiple of 4 with zeros,
// so padded A entries only need to be finite).
template <int P>
struct M2lMma;
#define AMK_M2L_MMA(P, WR, WC, KC)                                                               \
  template <>                                                                                    \
  struct M2lMma<P> {                                                                             \
    static constexpr int kNm = (P + 1) * (P + 2) * (P + 3) / 6;                                  \
    static constexpr int kNd = (2 * P + 1) * (2 * P + 2) * (2 * P + 3) / 6;                      \
    static constexpr int kGb = (kNm + 7) / 8, kNg = 8 * kGb, kNk = 4 * ((kNm + 3) / 4);           \
    static constexpr int kWr = WR, kWc = WC, kKc = KC;                                           \
    static constexpr int kWarpsR = kGb / WR, kWarps = kWarpsR * (8 / WC), kThreads = 32 * kWarps; \
    static_assert(kGb % WR == 0 && 8 % WC == 0 && kNk % KC == 0 && KC % 4 == 0, "M2L mma shape"); \
  };
AMK_M2L_MMA(1, 1, 8, 4)
AMK_M2L_MMA(2, 2, 4, 12)
AMK_M2L_MMA(3, 3, 4, 20)
AMK_M2L_MMA(4, 5, 4, 12)
AMK_M2L_MMA(5, 7, 4, 8)
AMK_M2L_MMA(6, 11, 2, 12)
AMK_M2L_MMA(7, 5, 4, 24)
AMK_M2L_MMA(8, 7, 4, 24)
#undef AMK_M2L_MMA

template <int P>
size_t m2l_mma_smem() {
  using S = M2lMma<P>;
  return sizeof(double) * (static_cast<size_t>(kM2lStages) * S::kKc * kM2lBs + S::kNd + S::kNg + S::kNk) +
         sizeof(short) * static_cast<size_t>(S::kNk) * S::kNg + 2 * kM2lUnitPairs * sizeof(int) + 16;
}

__device__ __forceinline__ void mma_f64(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// Persistent blocks: the index map is built once per block, then units are
// taken from a counter; within a tile, warps skip the 8-pair column blocks
// past the tile's last pair, so a class of a few pairs costs a fraction of a
// tile.
template <int P>
__global__ void __launch_bounds__(M2lMma<P>::kThreads)
m2l_class_mma_kernel(FmmDevTables T, int n_units, int* __restrict__ unit_counter,
                     const int* __restrict__ unit_cls, const int* __restrict__ unit_pos,
                     const int* __restrict__ cls_code, const int* __restrict__ cls_end,
                     const int* __restrict__ perm, const int* __restrict__ src, const double* __restrict__ Mh,
                     const double* __restrict__ table, const unsigned long long* __restrict__ keys, long e0,
                     double* __restrict__ out) {
  using S = M2lMma<P>;
  constexpr int kNm = S::kNm, kNg = S::kNg, kNk = S::kNk, kKc = S::kKc, kTh = S::kThreads;
  constexpr int kChunks = kNk / kKc;
  extern __shared__ __align__(16) unsigned char mma_smem[];
  double* Bs = reinterpret_cast<double*>(mma_smem);  // [kM2lStages][kKc][kM2lBs]
  double* Ds = Bs + kM2lStages * kKc * kM2lBs;        // [kNd]
  double* rowf = Ds + S::kNd;                         // [kNg]
  double* colf = rowf + kNg;                          // [kNk]
  int* pe = reinterpret_cast<int*>(colf + kNk);       // [kM2lUnitPairs]
  int* ps = pe + kM2lUnitPairs;                       // [kM2lUnitPairs]
  short* idx = reinterpret_cast<short*>(ps + kM2lUnitPairs);  // [kNk][kNg]
  __shared__ int s_unit;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wr = warp % S::kWarpsR, wc = warp / S::kWarpsR;
  const int lr = lane >> 2, lc = lane & 3;  // fragment row / column within a tile
  const int g_base = 8 * S::kWr * wr + lr, p_base = 8 * S::kWc * wc + lr;
  for (int x = tid; x < kNk * kNg; x += kTh) {
    const int a = x / kNg, g = x - a * kNg;
    idx[x] = (a < kNm && g < kNm) ? T.m2l_index_t[a * kNm + g] : 0;
  }
  for (;;) {
    if (tid == 0) s_unit = atomicAdd(unit_counter, 1);
    __syncthreads();  // also: the previous unit is done with the shared arrays
    const int unit = s_unit;
    if (unit >= n_units) break;
    const int cls = unit_cls[unit], pos0 = unit_pos[unit];
    const int np = min(kM2lUnitPairs, cls_end[cls] - pos0);
    const int n_tiles = (np + kM2lTileP - 1) / kM2lTileP, n_steps = n_tiles * kChunks;
    const int dd = m2l_key_dd(keys[cls_code[cls]]);
    const int et = dd < 0 ? -dd : 0, es = dd > 0 ? dd : 0;  // log2(h_t / u), log2(h_s / u)
    for (int k = tid; k < S::kNd; k += kTh) Ds[k] = table[static_cast<size_t>(cls) * S::kNd + k];
    for (int g = tid; g < kNg; g += kTh) rowf[g] = g < kNm ? ldexp(T.inv_fact[g], (T.multi[g].w + 1) * et) : 0.0;
    for (int a = tid; a < kNk; a += kTh) colf[a] = a < kNm ? ldexp(1.0, T.multi[a].w * es) : 0.0;
    for (int p = tid; p < n_tiles * kM2lTileP; p += kTh) {
      const int e = p < np ? perm[pos0 + p] : -1;
      pe[p] = e;
      ps[p] = e >= 0 ? src[e] : -1;
    }
    __syncthreads();
    auto issue = [&](int step) {
      if (step < n_steps) {
        const int tile = step / kChunks, chunk = step - tile * kChunks;
        const int live = min(kM2lTileP, np - tile * kM2lTileP);
        double* B = Bs + (step % kM2lStages) * kKc * kM2lBs;
        for (int x = tid; x < kKc * kM2lTileP; x += kTh) {
          const int p = x / kKc, kk = x - p * kKc, a = chunk * kKc + kk;
          if (p >= ((live + 7) & ~7)) continue;  // column blocks no warp reads
          const int sp = ps[tile * kM2lTileP + p];
          const bool ok = sp >= 0 && a < kNm;
          cp_async8(B + kk * kM2lBs + p, ok ? Mh + static_cast<size_t>(sp) * kNm + a : Mh, ok);
        }
      }
      cp_async_commit();
    };
    for (int st = 0; st < kM2lStages - 1; ++st) issue(st);
    double acc[S::kWr][S::kWc][2];
#pragma unroll
    for (int i = 0; i < S::kWr; ++i)
#pragma unroll
      for (int j = 0; j < S::kWc; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
#pragma unroll 1
    for (int step = 0; step < n_steps; ++step) {
      const int tile = step / kChunks, chunk = step - tile * kChunks;
      const int live = min(kM2lTileP, np - tile * kM2lTileP);  // pairs in this tile
      const int jn = min(S::kWc, max(0, (live - 8 * S::kWc * wc + 7) / 8));  // this warp's live column blocks
      cp_async_wait<kM2lStages - 2>();
      __syncthreads();
      issue(step + kM2lStages - 1);
      // k chunk: A fragments from D(v) (scaled by the source factor when the
      // source is the larger cell), B fragments from the staged rows
      auto chunk_products = [&](auto scaled) {
        const double* B = Bs + (step % kM2lStages) * kKc * kM2lBs;
#pragma unroll
        for (int ks = 0; ks < kKc / 4; ++ks) {
          const int a = chunk * kKc + 4 * ks + lc;
          const short* irow = idx + a * kNg + g_base;
          double af[S::kWr], bf[S::kWc];
#pragma unroll
          for (int i = 0; i < S::kWr; ++i) af[i] = Ds[irow[8 * i]];
          if (decltype(scaled)::value) {
            const double cf = colf[a];
#pragma unroll
            for (int i = 0; i < S::kWr; ++i) af[i] *= cf;
          }
#pragma unroll
          for (int j = 0; j < S::kWc; ++j)
            if (j < jn) bf[j] = B[(4 * ks + lc) * kM2lBs + p_base + 8 * j];
#pragma unroll
          for (int j = 0; j < S::kWc; ++j)
            if (j < jn)
#pragma unroll
              for (int i = 0; i < S::kWr; ++i) mma_f64(acc[i][j], af[i], bf[j]);
        }
      };
      if (jn > 0) {
        if (es > 0)
          chunk_products(std::true_type());
        else
          chunk_products(std::false_type());
      }
      if (chunk == kChunks - 1) {
#pragma unroll
        for (int j = 0; j < S::kWc; ++j)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int e = pe[tile * kM2lTileP + 8 * S::kWc * wc + 8 * j + 2 * lc + h];
#pragma unroll
            for (int i = 0; i < S::kWr; ++i) {
              const int g = 8 * S::kWr * wr + 8 * i + lr;
              if (e >= 0 && g < kNm) out[static_cast<size_t>(e - e0) * kNm + g] = acc[i][j][h] * rowf[g];
              acc[i][j][h] = 0.0;
            }
          }
      }
    }
    cp_async_wait<0>();
  }
}

// Split-BF16 tensor-core form of the class product (FMM precision mode
// AMK_FMM_TENSOR). The class matrix A (rows g padded to 128, K = a padded
// to a multiple of 32) and the tile's rescaled source expansions B (64
// pairs, K-major) are each split into three BF16 terms, x = x0 + x1 + x2
// (24 significant bits), and the six products x0y0 + x0y1 + x1y0 + x0y2 +
// x1y1 + x2y0 accumulate into one FP32 accumulator in tensor memory
// (tcgen05.mma, M = 128, N = 64, K = 16, A from tensor memory). The
// per-pair products are written as FP32 (n_m floats per pair) and summed
// per target in FP64 by the same reduction as the FP64 path. Relative error
// of a product: about 2^-22, far below the FMM's truncation error at p >= 5.
//
// Before the kernel, per evaluation chunk: the cells' rescaled expansions
// are split into BF16 rows of kKp elements (m2l_split_kernel), each class's
// D(v) into packed BF16 terms (m2l_table_kernel), and every unit gets a
// descriptor {class, first pair, pairs, depth difference} and every pair its
// source cell (m2l_tc_prep_kernel), so each role reads one value where it
// would otherwise follow a chain of dependent loads.
//
// Roles (one CTA per SM, units of one class taken in a fixed stride; every
// role prefetches the next unit's descriptor and the next tile's indices):
//  - warps 0-3 drain the accumulators (tcgen05.ld, FP32 stores), row g =
//    TMEM lane of the warp's quarter;
//  - warps 4-11 build A for the next unit straight into tensor memory
//    (tcgen05.st, two K halves per lane quarter, A double-buffered) from the
//    class's split D(v), staged in shared memory by cp.async one unit ahead;
//  - warps 12-15 stream B: a pair's column is 3 * kKp / 8 16-byte
//    core-matrix rows copied with cp.async into one of 3-4 stages, each
//    thread's arrival on the stage's barrier triggered by the completion of
//    its copies (cp.async.mbarrier.arrive.noinc);
//  - one thread of warp 16 issues the MMAs into one of two accumulators.
// The roles meet at mbarriers (stage full / empty, accumulator full /
// empty, A full / empty). Every wait is bounded in time; a wait that runs out
// sets an abort flag that ends every other wait at once, the roles run
// through their loops without work, and the kernel reports the status.
constexpr int kM2lTcN = 64;          // pairs per tensor-core tile (MMA N)
constexpr int kM2lTcAcc = 2;         // FP32 accumulators in tensor memory
constexpr int kM2lTcEpiWarps = 4;    // accumulator readers
constexpr int kM2lTcBldWarps = 8;    // A builders (two per TMEM lane quarter)
constexpr int kM2lTcProdWarps = 4;   // B producers
constexpr int kM2lTcBldThreads = 32 * kM2lTcBldWarps;
constexpr int kM2lTcProdThreads = 32 * kM2lTcProdWarps;
constexpr int kM2lTcBld0 = kM2lTcEpiWarps;                      // first builder warp
constexpr int kM2lTcProd0 = kM2lTcBld0 + kM2lTcBldWarps;        // first producer warp
constexpr int kM2lTcMmaWarp = kM2lTcProd0 + kM2lTcProdWarps;
constexpr int kM2lTcThreads = 32 * (kM2lTcMmaWarp + 1);
constexpr unsigned long long kM2lTcWaitNs = 2000000000ull;  // a wait gives up after 2 s
constexpr uint32_t kM2lTcCols = 512;                         // TMEM columns the block allocates

template <int P>
struct M2lTc {
  static constexpr int kNm = (P + 1) * (P + 2) * (P + 3) / 6;
  static constexpr int kNd = (2 * P + 1) * (2 * P + 2) * (2 * P + 3) / 6;
  static constexpr int kNd3 = (kNd + 2) & ~1;              // packed D row: zero at kNd, 16-byte multiple
  static constexpr int kKp = 32 * ((kNm + 31) / 32);
  static constexpr int kChunks = kKp / 8;                  // 16-byte rows of one split of a pair
  static constexpr uint32_t kACols = kKp / 2;              // TMEM columns of one split of A (2 BF16 per column)
  static constexpr uint32_t kABuf = 3 * kACols;            // one A buffer
  static constexpr uint32_t kAccCol = 2 * kABuf;           // first accumulator column
  static constexpr uint32_t kBSplit = static_cast<uint32_t>(kM2lTcN) * kKp * 2u;
  static constexpr uint32_t kBStage = 3u * kBSplit;
  static constexpr int kStages = kBStage > 40u * 1024u ? 3 : 4;      // B stages
  static constexpr int kIdxStride = kKp + 2;  // index-map row pitch: an odd number of words, rows in distinct banks
  static constexpr uint32_t kOffIdx = kStages * kBStage;             // idx [kNm][kIdxStride] (u16)
  static constexpr uint32_t kOffD = kOffIdx + ((2u * kNm * kIdxStride + 15u) & ~15u);  // Ds3 [2][kNd3]
  static constexpr uint32_t kOffCol = kOffD + 2u * 8u * kNd3;        // column scales [2][kKp] (float)
  static constexpr uint32_t kOffStg = kOffCol + 2u * 4u * kKp;       // output staging [kN][kNm] (float)
  static constexpr uint32_t kOffPe = kOffStg + 4u * kM2lTcN * kNm;    // the tile's pair ids [kN]
  static constexpr int kBars = 2 * kStages + 2 * kM2lTcAcc + 5;       // + A full x2, A empty x2, done
  static constexpr uint32_t kOffBar = kOffPe + 4u * kM2lTcN;
  static constexpr uint32_t kOffSlot = kOffBar + 8u * kBars;         // TMEM address, abort flag
  static constexpr uint32_t kUsed = kOffSlot + 16u;
  // one CTA per SM: the block allocates all of tensor memory
  static constexpr uint32_t kSmem = kUsed > 120u * 1024u ? kUsed : 120u * 1024u;
  static_assert(kNm <= 128, "the tensor-core class product covers n_m <= 128 (orders up to 7)");
  static_assert(kAccCol + kM2lTcAcc * kM2lTcN <= kM2lTcCols, "tensor memory columns");
  static_assert(kUsed <= 226u * 1024u, "tensor-core class product shared memory");
  static_assert(kKp % 32 == 0 && kNd3 < 65535, "K halves of 16-column chunks; 16-bit derivative indices");
  static_assert(kNm % 4 == 0, "per-pair product rows are whole 16-byte vectors");
};

__device__ __forceinline__ void split3_bf16(double v, __nv_bfloat16* t) {
  const __nv_bfloat16 a0 = __double2bfloat16(v);
  const double r1 = v - static_cast<double>(__bfloat162float(a0));
  const __nv_bfloat16 a1 = __double2bfloat16(r1);
  const double r2 = r1 - static_cast<double>(__bfloat162float(a1));
  t[0] = a0;
  t[1] = a1;
  t[2] = __double2bfloat16(r2);
}

// Mh3[(cell * 3 + q) * kp + a] = term q of the split of Mh[cell][a] (zero for
// a >= n_m): a cell's three rows are 3 * kp contiguous BF16 values.
// With copies = 8 (reflection-folded classes), copy R holds the rows with the
// signs s^a of reflection R: Mh3[((R * n_cells + cell) * 3 + q) * kp + a]
// (a sign flip of a BF16 term is exact).
__global__ void m2l_split_kernel(long n_cells, int nm, int kp, const int4* __restrict__ multi, int copies,
                                 const double* __restrict__ Mh, __nv_bfloat16* __restrict__ Mh3) {
  const long e = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  if (e >= n_cells * kp) return;
  const long cell = e / kp;
  const int a = static_cast<int>(e - cell * kp);
  __nv_bfloat16 t[3];
  split3_bf16(a < nm ? Mh[cell * nm + a] : 0.0, t);
  const int4 ma = a < nm ? multi[a] : make_int4(0, 0, 0, 0);
  for (int R = 0; R < copies; ++R) {
    const int odd = ((R & 1) ? ma.x : 0) + ((R & 2) ? ma.y : 0) + ((R & 4) ? ma.z : 0);
    const size_t row = (static_cast<size_t>(R) * n_cells + cell) * 3;
#pragma unroll
    for (int q = 0; q < 3; ++q) Mh3[(row + q) * kp + a] = (odd & 1) ? __hneg(t[q]) : t[q];
  }
}

// Unit descriptors {class, first pair, pairs, depth difference} and the
// source cell of every class pair.
__global__ void m2l_tc_prep_kernel(int n_units, const int* __restrict__ unit_cls, const int* __restrict__ unit_pos,
                                   const int* __restrict__ cls_code, const int* __restrict__ cls_end,
                                   const unsigned long long* __restrict__ keys, int n_pairs,
                                   const int* __restrict__ perm, const int* __restrict__ src,
                                   const unsigned char* __restrict__ refl, int n_cells, int4* __restrict__ ud,
                                   int* __restrict__ psrc) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x < n_units) {
    const int cls = unit_cls[x], pos0 = unit_pos[x];
    ud[x] = make_int4(cls, pos0, min(kM2lUnitPairs, cls_end[cls] - pos0), m2l_key_dd(keys[cls_code[cls]]));
  }
  if (x < n_pairs) {  // the source's row in the split expansions (its reflected copy when folded)
    const int e = perm[x];
    psrc[x] = (refl ? static_cast<int>(refl[e]) * n_cells : 0) + src[e];
  }
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  const int n = valid ? 16 : 0;  // 0: zero fill, nothing read
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(n) : "memory");
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait for the phase of parity `parity` of an mbarrier. Returns
// false (and raises the block's abort flag) when the flag is already up or
// the wait runs past kM2lTcWaitNs.
__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag) {
  if (*abort_flag) return false;
  unsigned long long t0 = 0;
  for (long spins = 1;; ++spins) {
    if (tc::mbar_try_wait(bar, parity)) return true;
    if ((spins & 63) == 0) {
      if (*abort_flag) return false;
      const unsigned long long now = global_ns();
      if (t0 == 0) {
        t0 = now;
      } else if (now - t0 > kM2lTcWaitNs || spins > (1L << 34)) {
        *abort_flag = 1;
        return false;
      }
    }
  }
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// One MMA with A in tensor memory and B in shared memory.
__device__ __forceinline__ void mma_bf16_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t bdesc, uint32_t idesc,
                                            int accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(tmem_d), "r"(tmem_a), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t (&r)[8]) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(taddr), "r"(r[0]),
               "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
               : "memory");
}

// A BF16 value (bit pattern) times 2^s, exact for the exponents of the
// class matrices (no overflow or subnormal results).
__device__ __forceinline__ uint32_t bf16_scale(uint32_t bits, float scale) {
  const float f = __uint_as_float(bits << 16) * scale;
  return __bfloat16_as_ushort(__float2bfloat16_rn(f));
}

// The block's units in order: unit = blockIdx.x + k * gridDim.x.
struct TcUnits {
  const int4* ud;
  int n_units;
  __device__ int4 load(int unit) const { return unit < n_units ? ud[unit] : make_int4(0, 0, 0, 0); }
};

template <int P>
__global__ void __launch_bounds__(kM2lTcThreads, 1)
m2l_class_tc_kernel(FmmDevTables T, int n_units, const int4* __restrict__ ud, const int* __restrict__ perm,
                    const int* __restrict__ psrc, const __nv_bfloat16* __restrict__ Mh3,
                    const uint2* __restrict__ table3, long e0, float* __restrict__ out, int* __restrict__ status) {
  using S = M2lTc<P>;
  constexpr int kNm = S::kNm, kKp = S::kKp, kN = kM2lTcN, kSt = S::kStages, kAc = kM2lTcAcc;
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  unsigned char* b_img = tc_smem;
  uint16_t* idx = reinterpret_cast<uint16_t*>(tc_smem + S::kOffIdx);  // [g][a]; kNd where g or a >= n_m
  uint2* Ds3 = reinterpret_cast<uint2*>(tc_smem + S::kOffD);           // [2][kNd3]: x = t0 | t1 << 16, y = t2
  float* colsc = reinterpret_cast<float*>(tc_smem + S::kOffCol);       // [2][kKp]
  const uint32_t bar0 = tc::smem_u32(tc_smem + S::kOffBar);
  // barrier addresses: full[s], empty[s], accf[b], acce[b], afull[2], aempty[2], done
  auto full_bar = [&](int s) { return bar0 + 8u * s; };
  auto empty_bar = [&](int s) { return bar0 + 8u * (kSt + s); };
  auto accf_bar = [&](int b) { return bar0 + 8u * (2 * kSt + b); };
  auto acce_bar = [&](int b) { return bar0 + 8u * (2 * kSt + kAc + b); };
  auto afull_bar = [&](int h) { return bar0 + 8u * (2 * kSt + 2 * kAc + h); };
  auto aempty_bar = [&](int h) { return bar0 + 8u * (2 * kSt + 2 * kAc + 2 + h); };
  const uint32_t done_bar = bar0 + 8u * (2 * kSt + 2 * kAc + 4);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tc_smem + S::kOffSlot);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tc_smem + S::kOffSlot + 4);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int stride = gridDim.x;
  const TcUnits units{ud, n_units};
  if (tid == 0) {
    auto init = [](uint32_t b, int count) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(b), "r"(count));
    };
    for (int s = 0; s < kSt; ++s) {
      init(full_bar(s), kM2lTcProdThreads);
      init(empty_bar(s), 1);
    }
    for (int b = 0; b < kAc; ++b) {
      init(accf_bar(b), 1);
      init(acce_bar(b), 32 * kM2lTcEpiWarps);
    }
    for (int h = 0; h < 2; ++h) {
      init(afull_bar(h), kM2lTcBldThreads);
      init(aempty_bar(h), 1);
    }
    init(done_bar, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == kM2lTcMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc::smem_u32(tmem_slot)),
                 "r"(kM2lTcCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  for (int x = tid; x < kNm * S::kIdxStride; x += kM2lTcThreads) {
    const int g = x / S::kIdxStride, a = x - g * S::kIdxStride;
    idx[x] = a < kNm ? static_cast<uint16_t>(T.m2l_index_t[a * kNm + g]) : static_cast<uint16_t>(S::kNd);
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp < kM2lTcEpiWarps) {
    // ---- accumulator readers: row g of the accumulator (all kN pairs of a
    // tile) scaled into the staging tile [pair][g], then whole 16-byte
    // vectors of the pairs' product rows to global memory
    const int g = 32 * warp + lane, et_ = tid;  // et_: thread index among the readers
    const uint32_t lane_addr = static_cast<uint32_t>(32 * warp) << 16;
    float* stg = reinterpret_cast<float*>(tc_smem + S::kOffStg);
    int* pe_s = reinterpret_cast<int*>(tc_smem + S::kOffPe);
    const double ifact = g < kNm ? T.inv_fact[g] : 0.0;
    const int wg1 = g < kNm ? T.multi[g].w + 1 : 0;
    constexpr int kVec = kNm / 4;  // 16-byte vectors per pair row
    long i = 0;
    int4 u = units.load(blockIdx.x);
    for (int unit = blockIdx.x; unit < n_units; unit += stride) {
      const int4 un = units.load(unit + stride);  // next unit, in flight
      const int pos0 = u.y, np = u.z, et = u.w < 0 ? -u.w : 0;  // log2(h_t / u)
      const float rf = static_cast<float>(ldexp(ifact, wg1 * et));
      int pe_next = et_ < kN && et_ < np ? perm[pos0 + et_] : 0;
      for (int tile0 = 0; tile0 < np; tile0 += kN, ++i) {
        const int b = static_cast<int>(i % kAc);
        const int pe_cur = pe_next;  // this tile's pair id of reader et_ (< kN)
        pe_next = et_ < kN && tile0 + kN + et_ < np ? perm[pos0 + tile0 + kN + et_] : 0;  // in flight
        const bool ok = tc_wait(accf_bar(b), static_cast<uint32_t>((i / kAc) & 1), abort_flag);
        tc::fence_after();
        float v0[32], v1[32];
        tc::tmem_ld32(tmem + lane_addr + S::kAccCol + b * kN, v0);
        tc::tmem_ld32(tmem + lane_addr + S::kAccCol + b * kN + 32, v1);
        tc::fence_before();
        mbar_arrive(acce_bar(b));
        const int live = min(kN, np - tile0);
        asm volatile("bar.sync 2, %0;" ::"n"(32 * kM2lTcEpiWarps) : "memory");  // the last tile's rows are out
        if (et_ < kN) pe_s[et_] = pe_cur;
        if (g < kNm) {
#pragma unroll
          for (int j = 0; j < 32; ++j) stg[j * kNm + g] = v0[j] * rf;
#pragma unroll
          for (int j = 0; j < 32; ++j) stg[(32 + j) * kNm + g] = v1[j] * rf;
        }
        asm volatile("bar.sync 2, %0;" ::"n"(32 * kM2lTcEpiWarps) : "memory");
        if (ok)
          for (int x = et_; x < live * kVec; x += 32 * kM2lTcEpiWarps) {
            const int j = x / kVec, cv = x - j * kVec;
            const float4 val = *reinterpret_cast<const float4*>(stg + j * kNm + 4 * cv);
            *reinterpret_cast<float4*>(out + static_cast<size_t>(pe_s[j] - e0) * kNm + 4 * cv) = val;
          }
      }
      u = un;
    }
  } else if (warp < kM2lTcProd0) {
    // ---- A builders: row g of A, half c2 of its K range
    const int bt = tid - 32 * kM2lTcBld0, q4 = warp & 3, c2 = (warp - kM2lTcBld0) >> 2, g = 32 * q4 + lane;
    const uint32_t lane_addr = static_cast<uint32_t>(32 * q4) << 16;
    const uint32_t* irow = reinterpret_cast<const uint32_t*>(idx + (g < kNm ? g : 0) * S::kIdxStride);
    constexpr int kCopies = S::kNd3 * 8 / 16;  // 16-byte copies of one packed D row
    auto stage_d = [&](int4 uu, int h) {     // the packed D row of unit uu's class into Ds3[h]
      const unsigned char* srcp = reinterpret_cast<const unsigned char*>(table3 + static_cast<size_t>(uu.x) * S::kNd3);
      unsigned char* dst = reinterpret_cast<unsigned char*>(Ds3 + h * S::kNd3);
      for (int x = bt; x < kCopies; x += kM2lTcBldThreads) cp_async16(dst + 16 * x, srcp + 16 * x, true);
      cp_async_commit();
    };
    int4 u = units.load(blockIdx.x);
    if (blockIdx.x < n_units) stage_d(u, 0);
    for (int k = 0, unit = blockIdx.x; unit < n_units; ++k, unit += stride) {
      const int4 un = units.load(unit + stride);
      const int es = u.w > 0 ? u.w : 0;  // log2(h_s / u)
      const int h = k & 1;
      float* cs = colsc + h * kKp;
      if (es > 0)
        for (int x = bt; x < kKp; x += kM2lTcBldThreads)
          cs[x] = x < kNm ? __uint_as_float(static_cast<uint32_t>(127 + T.multi[x].w * es) << 23) : 0.0f;
      if (unit + stride < n_units) {
        stage_d(un, h ^ 1);  // the next unit's row: its buffer was released by the barrier ending the last build
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
      asm volatile("bar.sync 1, %0;" ::"n"(kM2lTcBldThreads) : "memory");  // Ds3[h], colsc[h] complete
      // A buffer h was last read by unit k - 2
      const bool ok = k < 2 || tc_wait(aempty_bar(h), static_cast<uint32_t>(((k - 2) >> 1) & 1), abort_flag);
      if (!__any_sync(0xFFFFFFFFu, !ok)) {  // warp-uniform: tcgen05.st is .aligned
        const uint2* D3 = Ds3 + h * S::kNd3;
        const uint32_t abase = tmem + lane_addr + h * S::kABuf;
#pragma unroll 1
        for (int a0 = c2 * (kKp / 2); a0 < (c2 + 1) * (kKp / 2); a0 += 16) {
          uint32_t r[3][8];
#pragma unroll
          for (int c = 0; c < 8; ++c) {
            // two derivative indices per 32-bit load; even k in the low half of a column
            const uint32_t ip = g < kNm ? irow[(a0 >> 1) + c] : (S::kNd | (S::kNd << 16));
            uint2 d0 = D3[ip & 0xFFFFu], d1 = D3[ip >> 16];
            if (es > 0) {
              const float s0 = cs[a0 + 2 * c], s1 = cs[a0 + 2 * c + 1];
              d0 = make_uint2(bf16_scale(d0.x & 0xFFFFu, s0) | (bf16_scale(d0.x >> 16, s0) << 16),
                              bf16_scale(d0.y, s0));
              d1 = make_uint2(bf16_scale(d1.x & 0xFFFFu, s1) | (bf16_scale(d1.x >> 16, s1) << 16),
                              bf16_scale(d1.y, s1));
            }
            r[0][c] = __byte_perm(d0.x, d1.x, 0x5410);
            r[1][c] = __byte_perm(d0.x, d1.x, 0x7632);
            r[2][c] = __byte_perm(d0.y, d1.y, 0x5410);
          }
#pragma unroll
          for (int q = 0; q < 3; ++q) tmem_st8(abase + q * S::kACols + a0 / 2, r[q]);
        }
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
      }
      tc::fence_before();
      mbar_arrive(afull_bar(h));
      asm volatile("bar.sync 1, %0;" ::"n"(kM2lTcBldThreads) : "memory");  // Ds3[h], colsc[h] free
      u = un;
    }
    cp_async_wait<0>();
  } else if (warp < kM2lTcMmaWarp) {
    // ---- B producers: thread pt copies half of pair j's 3 * kChunks rows
    const int pt = tid - 32 * kM2lTcProd0, j = pt >> 1, hh = pt & 1;
    long i = 0;
    int unit = blockIdx.x, tile0 = 0;
    int4 u = units.load(unit);
    int cur = unit < n_units && j < u.z ? psrc[u.y + j] : -1;
    while (unit < n_units) {
      // the next tile (possibly of the next unit): its source cell, in flight
      int nunit = unit, ntile0 = tile0 + kN;
      int4 nu = u;
      if (ntile0 >= u.z) {
        nunit = unit + stride;
        ntile0 = 0;
        nu = units.load(nunit);
      }
      const int nxt = nunit < n_units && ntile0 + j < nu.z ? psrc[nu.y + ntile0 + j] : -1;
      const int s = static_cast<int>(i % kSt);
      const bool ok = i < kSt || tc_wait(empty_bar(s), static_cast<uint32_t>((i / kSt - 1) & 1), abort_flag);
      if (ok) {
        const bool live = cur >= 0;
        const unsigned char* sp =
            reinterpret_cast<const unsigned char*>(Mh3) + (live ? static_cast<size_t>(cur) * (3u * kKp * 2u) : 0);
        unsigned char* dst = b_img + s * S::kBStage;
#pragma unroll 4
        for (int r = hh; r < 3 * S::kChunks; r += 2) {
          const int q = r / S::kChunks, ch = r - q * S::kChunks;
          cp_async16(dst + q * S::kBSplit + tc::op_offset(j, 8 * ch, kN), sp + 16 * r, live);
        }
      }
      // full[s] counts this thread's arrival once all of its copies so far
      // have landed (the MMA thread orders them for the tensor core)
      asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(full_bar(s)) : "memory");
      ++i;
      unit = nunit;
      tile0 = ntile0;
      u = nu;
      cur = nxt;
    }
    cp_async_wait<0>();
  } else if (lane == 0) {
    // ---- MMA issue: six split products per K step of 16, smallest terms first
    constexpr int kCombo[6][2] = {{2, 0}, {1, 1}, {0, 2}, {1, 0}, {0, 1}, {0, 0}};
    const uint32_t idesc = tc::make_idesc(kN), b_base = tc::smem_u32(b_img);
    long i = 0;
    int4 u = units.load(blockIdx.x);
    for (int k = 0, unit = blockIdx.x; unit < n_units; ++k, unit += stride) {
      const int4 un = units.load(unit + stride);
      const int h = k & 1;
      const bool a_ok = tc_wait(afull_bar(h), static_cast<uint32_t>((k >> 1) & 1), abort_flag);
      const uint32_t abuf = tmem + h * S::kABuf;
      for (int tile0 = 0; tile0 < u.z; tile0 += kN, ++i) {
        const int s = static_cast<int>(i % kSt), b = static_cast<int>(i % kAc);
        bool ok = a_ok && tc_wait(full_bar(s), static_cast<uint32_t>((i / kSt) & 1), abort_flag);
        ok = ok && (i < kAc || tc_wait(acce_bar(b), static_cast<uint32_t>((i / kAc - 1) & 1), abort_flag));
        tc::fence_proxy_async();  // the stage's cp.async writes, for the tensor core's reads
        tc::fence_after();
        if (ok) {
          const uint32_t bb = b_base + s * S::kBStage, d = tmem + S::kAccCol + b * kN;
          uint64_t bd[3];
#pragma unroll
          for (int q = 0; q < 3; ++q) bd[q] = tc::make_sdesc(bb + q * S::kBSplit);
#pragma unroll
          for (int st = 0; st < kKp / 16; ++st)
#pragma unroll
            for (int c = 0; c < 6; ++c)  // descriptor start address advances by 16-byte units
              mma_bf16_ts(d, abuf + kCombo[c][0] * S::kACols + st * 8,
                          bd[kCombo[c][1]] + static_cast<uint64_t>((st * kN * 32) >> 4), idesc, (st | c) != 0);
        }
        tc::mma_commit(empty_bar(s));  // arrives once the products above have read the stage
        tc::mma_commit(accf_bar(b));
      }
      tc::mma_commit(aempty_bar(h));  // every product of this unit has read A buffer h
      u = un;
    }
    // every product has completed before tensor memory is released
    tc::mma_commit(done_bar);
    const unsigned long long t0 = global_ns();
    while (!tc::mbar_try_wait(done_bar, 0) && global_ns() - t0 < kM2lTcWaitNs) {
    }
  }
  __syncwarp();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  if (warp == kM2lTcMmaWarp)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kM2lTcCols));
  if (tid == 0 && *abort_flag) atomicExch(status, 1);
}

// Pairs outside the classes: a warp per pair (persistent blocks), the
// derivative tensor by the recurrence, the product through the transposed
// index map staged once per block, written in the rescaled form
// Lh = h_t^{|g|+1} L.
template <typename OutT>
__global__ void __launch_bounds__(32 * kFmmWarps)
m2l_pair_kernel(const Octree t, FmmDevTables T, const int* __restrict__ list, int n, const int* __restrict__ tgt,
                const int* __restrict__ src, const double* __restrict__ M, long e0, OutT* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char pair_smem[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nm = T.n_m;
  double* D = reinterpret_cast<double*>(pair_smem) + static_cast<size_t>(w) * (T.n_d + nm);
  double* Ms = D + T.n_d;
  short* idx = reinterpret_cast<short*>(reinterpret_cast<double*>(pair_smem) +
                                        static_cast<size_t>(kFmmWarps) * (T.n_d + nm));  // [a][g]
  for (int x = threadIdx.x; x < nm * nm; x += blockDim.x) idx[x] = T.m2l_index_t[x];
  __syncthreads();
  for (int k = blockIdx.x * kFmmWarps + w; k < n; k += gridDim.x * kFmmWarps) {
    const int e = list[k], ti = tgt[e], si = src[e];
    const double4 tc = t.center[ti], sc = t.center[si];
    for (int a = lane; a < nm; a += 32) Ms[a] = T.sign[a] * M[static_cast<size_t>(si) * nm + a];
    const double xs[3] = {tc.x - sc.x, tc.y - sc.y, tc.z - sc.z};
    m2l_derivatives(T, lane, xs, D);  // ends with __syncwarp
    for (int g = lane; g < nm; g += 32) {
      double s = 0.0;
      for (int a = 0; a < nm; ++a) s += Ms[a] * D[idx[a * nm + g]];
      double f = T.inv_fact[g];
      for (int d = 0; d <= T.multi[g].w; ++d) f *= tc.w;
      out[static_cast<size_t>(e - e0) * nm + g] = static_cast<OutT>(s * f);
    }
    __syncwarp();
  }
}

// L(t) += h_t^{-|g|-1} sum over the target's pairs in [e0, e1) in pair order;
// a warp per target, lanes over coefficients (R rows of 32), four pairs'
// rows in flight.
template <int R, typename InT>
__global__ void __launch_bounds__(256)
m2l_reduce_kernel(const Octree t, FmmDevTables T, const int* __restrict__ off, const int* __restrict__ count,
                  int t_first, int n_targets, long e0, long e1, const InT* __restrict__ out,
                  double* __restrict__ L) {
  constexpr int kU = 4;
  const int lane = threadIdx.x & 31;
  const int k = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (k >= n_targets) return;
  const int ti = t_first + k, nm = T.n_m;
  const long b = max(static_cast<long>(off[ti]), e0), end = min(static_cast<long>(off[ti]) + count[ti], e1);
  if (b >= end) return;
  double s[R];
#pragma unroll
  for (int r = 0; r < R; ++r) s[r] = 0.0;
  const InT* o = out + static_cast<size_t>(b - e0) * nm;
  long e = b;
  for (; e + kU <= end; e += kU, o += kU * nm) {
    double v[kU][R];
#pragma unroll
    for (int u = 0; u < kU; ++u)
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int g = lane + 32 * r;
        v[u][r] = g < nm ? o[u * nm + g] : 0.0;
      }
#pragma unroll
    for (int u = 0; u < kU; ++u)
#pragma unroll
      for (int r = 0; r < R; ++r) s[r] += v[u][r];
  }
  for (; e < end; ++e, o += nm)
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int g = lane + 32 * r;
      if (g < nm) s[r] += o[g];
    }
  const double ih = 1.0 / t.center[ti].w;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int g = lane + 32 * r;
    if (g >= nm) continue;
    double f = s[r];
    for (int d = 0; d <= T.multi[g].w; ++d) f *= ih;
    L[static_cast<size_t>(ti) * nm + g] += f;
  }
}

// The same sum over FP32 per-pair products (tensor-core mode, n_m a multiple
// of 4): lane l holds coefficients 4l..4l+3 and reads them as one 16-byte
// vector, eight pairs' rows in flight per warp. The sum per coefficient is
// the FP64 sum in pair order, as in m2l_reduce_kernel.
// Reflection-folded class pairs (tensor-core mode): the product row of a
// pair with reflection R gets s^g on coefficient g, in place (refl = 0 for
// every other pair, the per-pair path's included). A warp takes 32 pairs and
// rewrites the rows of those with R != 0 together, lane l holding
// coefficients 4l..4l+3 (n_m a multiple of 4, at most 128).
__global__ void __launch_bounds__(256)
m2l_refl_sign_kernel(FmmDevTables T, long e0, long e1, const unsigned char* __restrict__ refl,
                     float* __restrict__ out) {
  const int lane = threadIdx.x & 31, nv = T.n_m >> 2;
  const long e = e0 + blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  const uint32_t r = e < e1 ? refl[e] : 0u;
  uint32_t todo = __ballot_sync(0xffffffffu, r != 0);
  if (todo == 0) return;
  uint32_t neg[4] = {0u, 0u, 0u, 0u};  // bit R: s^g = -1 under reflection R, for g = 4 lane + c
  if (lane < nv)
    for (int c = 0; c < 4; ++c) {
      const int4 mg = T.multi[4 * lane + c];
      for (int R = 1; R < 8; ++R)
        if ((((R & 1) ? mg.x : 0) + ((R & 2) ? mg.y : 0) + ((R & 4) ? mg.z : 0)) & 1) neg[c] |= 1u << R;
    }
  const long warp_e = e - lane;
  while (todo) {
    const int src_lane = __ffs(todo) - 1;
    todo &= todo - 1;
    const uint32_t rr = __shfl_sync(0xffffffffu, r, src_lane);
    if (lane < nv) {
      float4* row = reinterpret_cast<float4*>(out + static_cast<size_t>(warp_e + src_lane - e0) * T.n_m) + lane;
      float4 v = *row;
      if ((neg[0] >> rr) & 1u) v.x = -v.x;
      if ((neg[1] >> rr) & 1u) v.y = -v.y;
      if ((neg[2] >> rr) & 1u) v.z = -v.z;
      if ((neg[3] >> rr) & 1u) v.w = -v.w;
      *row = v;
    }
  }
}

__global__ void __launch_bounds__(256)
m2l_reduce_f4_kernel(const Octree t, FmmDevTables T, const int* __restrict__ off, const int* __restrict__ count,
                     int t_first, int n_targets, long e0, long e1, const float* __restrict__ out,
                     double* __restrict__ L) {
  constexpr int kU = 8;
  const int lane = threadIdx.x & 31;
  const int k = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (k >= n_targets) return;
  const int ti = t_first + k, nm = T.n_m, nv = nm >> 2;
  const long b = max(static_cast<long>(off[ti]), e0), end = min(static_cast<long>(off[ti]) + count[ti], e1);
  if (b >= end || lane >= nv) return;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  const float4* o = reinterpret_cast<const float4*>(out + static_cast<size_t>(b - e0) * nm) + lane;
  long e = b;
  for (; e + kU <= end; e += kU, o += kU * nv) {
    float4 v[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) v[u] = o[u * nv];
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      s0 += v[u].x;
      s1 += v[u].y;
      s2 += v[u].z;
      s3 += v[u].w;
    }
  }
  for (; e < end; ++e, o += nv) {
    const float4 v = *o;
    s0 += v.x;
    s1 += v.y;
    s2 += v.z;
    s3 += v.w;
  }
  const double ih = 1.0 / t.center[ti].w;
  const double sv[4] = {s0, s1, s2, s3};
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const int g = 4 * lane + c;
    double f = sv[c];
    for (int d = 0; d <= T.multi[g].w; ++d) f *= ih;
    L[static_cast<size_t>(ti) * nm + g] += f;
  }
}

template <typename InT>
int m2l_reduce(amk_ctx* c, cudaStream_t stream, const Octree& t, const FmmDevTables& T, const int* off,
               const int* count, int t_first, int n_targets, long e0, long e1, const InT* out, double* L) {
  const unsigned grid = static_cast<unsigned>((n_targets + 7) / 8);
  if constexpr (std::is_same<InT, float>::value) {
    if (T.n_m % 4 == 0 && T.n_m <= 128) {
      m2l_reduce_f4_kernel<<<grid, 256, 0, stream>>>(t, T, off, count, t_first, n_targets, e0, e1, out, L);
      return check_launch(c, "m2l_reduce_f4_kernel");
    }
  }
  switch ((T.n_m + 31) / 32) {
    case 1:
      m2l_reduce_kernel<1, InT><<<grid, 256, 0, stream>>>(t, T, off, count, t_first, n_targets, e0, e1, out, L);
      break;
    case 2:
      m2l_reduce_kernel<2, InT><<<grid, 256, 0, stream>>>(t, T, off, count, t_first, n_targets, e0, e1, out, L);
      break;
    case 3:
      m2l_reduce_kernel<3, InT><<<grid, 256, 0, stream>>>(t, T, off, count, t_first, n_targets, e0, e1, out, L);
      break;
    case 4:
      m2l_reduce_kernel<4, InT><<<grid, 256, 0, stream>>>(t, T, off, count, t_first, n_targets, e0, e1, out, L);
      break;
    default:
      static_assert((kMaxNm + 31) / 32 == 6, "rows per lane");
      m2l_reduce_kernel<6, InT><<<grid, 256, 0, stream>>>(t, T, off, count, t_first, n_targets, e0, e1, out, L);
      break;
  }
  return check_launch(c, "m2l_reduce_kernel");
}

template <int P>
int launch_class_product(amk_ctx* c, const FmmDevTables& T, int n_units, int* unit_counter, const int* unit_cls, const int* unit_pos,
                         const int* cls_code, const int* cls_end, const int* perm, const int* src, const double* Mh,
                         const double* table, const unsigned long long* keys, long e0, double* out) {
  const size_t smem = m2l_mma_smem<P>();
  AMK_CUDA_TRY(cudaFuncSetAttribute(m2l_class_mma_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(smem)));
  int per_sm = 0;
  AMK_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, m2l_class_mma_kernel<P>, M2lMma<P>::kThreads,
                                                             smem));
  int sms = 0;
  AMK_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
  const int grid = std::max(1, std::min(n_units, std::max(1, per_sm) * sms));
  AMK_CUDA_TRY(cudaMemsetAsync(unit_counter, 0, sizeof(int), c->stream));
  m2l_class_mma_kernel<P><<<grid, M2lMma<P>::kThreads, smem, c->stream>>>(
      T, n_units, unit_counter, unit_cls, unit_pos, cls_code, cls_end, perm, src, Mh, table, keys, e0, out);
  return check_launch(c, "m2l_class_mma_kernel");
}

int class_product(amk_ctx* c, int order, const FmmDevTables& T, int n_units, int* unit_counter, const int* unit_cls,
                  const int* unit_pos, const int* cls_code, const int* cls_end, const int* perm, const int* src,
                  const double* Mh, const double* table, const unsigned long long* keys, long e0, double* out) {
#define AMK_M2L_CASE(P)                                                                                         \
  case P:                                                                                                     \
    return launch_class_product<P>(c, T, n_units, unit_counter, unit_cls, unit_pos, cls_code, cls_end, perm, src, Mh, table, \
                                   keys, e0, out);
  switch (order) {
    AMK_M2L_CASE(1)
    AMK_M2L_CASE(2)
    AMK_M2L_CASE(3)
    AMK_M2L_CASE(4)
    AMK_M2L_CASE(5)
    AMK_M2L_CASE(6)
    AMK_M2L_CASE(7)
    AMK_M2L_CASE(8)
    default:
      return fail(AMK_ERR_INVALID, "FMM order %d outside [1, %d]", order, kMaxOrder);
  }
#undef AMK_M2L_CASE
}

template <int P>
int launch_class_tc(amk_ctx* c, const FmmDevTables& T, int n_units, const int4* ud, const int* perm,
                    const int* psrc, const __nv_bfloat16* Mh3, const uint2* table3, long e0, float* out,
                    int* status) {
  const size_t smem = M2lTc<P>::kSmem;
  AMK_CUDA_TRY(cudaFuncSetAttribute(m2l_class_tc_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(smem)));
  int sms = 0;
  AMK_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
  const int grid = std::max(1, std::min(n_units, sms));  // one CTA per SM (shared memory and TMEM)
  m2l_class_tc_kernel<P><<<grid, kM2lTcThreads, smem, c->stream>>>(T, n_units, ud, perm, psrc, Mh3, table3, e0,
                                                                   out, status);
  return check_launch(c, "m2l_class_tc_kernel");
}

// Orders the tensor-core class product covers (n_m <= 128; below p = 5 the
// FP64 products are already cheap next to the rest of the evaluation).
inline bool tc_order(int order) { return order >= 5 && order <= 7; }

// Packed D row length of the tensor-core product for an order.
inline int tc_nd3(int n_d) { return (n_d + 2) & ~1; }

int class_tc(amk_ctx* c, int order, const FmmDevTables& T, int n_units, const int4* ud, const int* perm,
             const int* psrc, const __nv_bfloat16* Mh3, const uint2* table3, long e0, float* out, int* status) {
  switch (order) {
    case 5: return launch_class_tc<5>(c, T, n_units, ud, perm, psrc, Mh3, table3, e0, out, status);
    case 6: return launch_class_tc<6>(c, T, n_units, ud, perm, psrc, Mh3, table3, e0, out, status);
    case 7: return launch_class_tc<7>(c, T, n_units, ud, perm, psrc, Mh3, table3, e0, out, status);
    default: return fail(AMK_ERR_INVALID, "no tensor-core class product for order %d", order);
  }
}

// Class reach; AMK_FMM_M2L_REACH narrows it, which sends the pairs beyond it
// through the per-pair path (tests of that path).
int m2l_reach() {
  const char* s = getenv("AMK_FMM_M2L_REACH");
  if (!s || !*s) return kM2lMaxReach;
  const int r = atoi(s);
  return r < 0 ? 0 : (r > kM2lMaxReach ? kM2lMaxReach : r);
}

// All M2L pairs (grouped by target in gm) into L. after_products (may be
// empty) runs once the last chunk's products are enqueued on the context
// stream, before their per-target sums and the final status read.
int m2l_products(amk_ctx* c, int order, const Octree& t, const FmmDevTables& T, const Grouped& gm, long n_m2l,
                 const double* M, double* L, const std::function<int()>& after_products) {
  int rc = AMK_OK;
  const long nn = t.n_nodes;
  const int reach = m2l_reach();
  const long n_codes = kM2lHashSlots;
  unsigned long long* keys = slot<unsigned long long>(c, kSlotM2lHash, kM2lHashSlots, &rc);
  AMK_TRY(rc);
  double* Mh = slot<double>(c, kSlotFmmWork5, static_cast<size_t>(nn) * T.n_m, &rc);
  AMK_TRY(rc);
  int* codes = slot<int>(c, kSlotM2lCodes, n_m2l, &rc);
  AMK_TRY(rc);
  int* tgt = slot<int>(c, kSlotM2lTarget, n_m2l, &rc);
  AMK_TRY(rc);
  int* hist = slot<int>(c, kSlotM2lHist, n_codes + 1, &rc);
  AMK_TRY(rc);
  int* start = slot<int>(c, kSlotM2lStart, n_codes + 1, &rc);
  AMK_TRY(rc);
  int* used = slot<int>(c, kSlotM2lUsed, n_codes + 1, &rc);
  AMK_TRY(rc);
  int* cls_index = slot<int>(c, kSlotM2lClassIndex, n_codes + 1, &rc);
  AMK_TRY(rc);
  int* nunit = slot<int>(c, kSlotM2lTiles, n_codes + 1, &rc);
  AMK_TRY(rc);
  int* unit_start = slot<int>(c, kSlotM2lTileStart, n_codes + 1, &rc);
  AMK_TRY(rc);
  int* counters = slot<int>(c, kSlotM2lCounters, 8, &rc);  // pairs, classes, units, fallback pairs
  AMK_TRY(rc);
  const long total = nn * T.n_m;
  m2l_rescale_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, c->stream>>>(t, T, M, Mh);
  AMK_TRY(check_launch(c, "m2l_rescale_kernel"));
  // the tensor-core products (split BF16) write FP32 per-pair products and
  // take classes folded over the 8 reflections
  const bool tc = c->fmm_precision == AMK_FMM_TENSOR && tc_order(order);
  unsigned char* refl = nullptr;
  if (tc) {
    refl = slot<unsigned char>(c, kSlotM2lRefl, n_m2l, &rc);
    AMK_TRY(rc);
  }
  AMK_CUDA_TRY(cudaMemsetAsync(keys, 0xff, kM2lHashSlots * sizeof(unsigned long long), c->stream));
  m2l_classify_kernel<<<4 * 148, 256, 0, c->stream>>>(t, gm.off, gm.count, gm.src, reach, keys, codes, tgt, refl);
  AMK_TRY(check_launch(c, "m2l_classify_kernel"));
  if (tc) {  // class sizes over all pairs, then the small classes folded by reflection
    AMK_CUDA_TRY(cudaMemsetAsync(hist, 0, n_codes * sizeof(int), c->stream));
    const unsigned ga = static_cast<unsigned>((n_m2l + 255) / 256);
    m2l_code_count_kernel<<<ga, 256, 0, c->stream>>>(codes, n_m2l, hist);
    AMK_TRY(check_launch(c, "m2l_code_count_kernel"));
    m2l_refold_kernel<<<ga, 256, 0, c->stream>>>(t, hist, kM2lMinClass, tgt, gm.src, reach, n_m2l, keys, codes,
                                                  refl);
    AMK_TRY(check_launch(c, "m2l_refold_kernel"));
  }
  const size_t esz = tc ? sizeof(float) : sizeof(double);
  long cap = std::max<long>(1L << 20, static_cast<long>((tc ? kM2lTcChunkBytes : kM2lChunkBytes) / (esz * T.n_m)));
  if (const char* env = getenv("AMK_FMM_M2L_CHUNK_PAIRS")) {  // smaller chunks (tests of the chunk seams)
    const long v = atol(env);
    if (v > 0) cap = std::min(cap, v);
  }
  Fmm* f = c->fmm;
  if (!f->side) {
    AMK_CUDA_TRY(cudaStreamCreateWithFlags(&f->side, cudaStreamNonBlocking));
    for (int i = 0; i < 2; ++i) {
      AMK_CUDA_TRY(cudaEventCreateWithFlags(&f->products_done[i], cudaEventDisableTiming));
      AMK_CUDA_TRY(cudaEventCreateWithFlags(&f->sums_done[i], cudaEventDisableTiming));
    }
  }
  const long max_cls = std::min<long>(cap, n_codes) + 1, max_units = cap / kM2lUnitPairs + max_cls + 1;
  int* perm = slot<int>(c, kSlotM2lPerm, std::min(cap, n_m2l), &rc);
  AMK_TRY(rc);
  int* fallback = slot<int>(c, kSlotM2lFallback, std::min(cap, n_m2l), &rc);
  AMK_TRY(rc);
  int* cls_code = slot<int>(c, kSlotM2lClassCode, max_cls, &rc);
  AMK_TRY(rc);
  int* cls_end = slot<int>(c, kSlotM2lClassEnd, max_cls, &rc);
  AMK_TRY(rc);
  int* unit_cls = slot<int>(c, kSlotM2lTileClass, max_units, &rc);
  AMK_TRY(rc);
  int* unit_pos = slot<int>(c, kSlotM2lTilePos, max_units, &rc);
  AMK_TRY(rc);
  int* tc_status = counters + 6;
  __nv_bfloat16* Mh3 = nullptr;
  if (tc) {
    AMK_CUDA_TRY(cudaMemsetAsync(tc_status, 0, sizeof(int), c->stream));
    const int kp = 32 * ((T.n_m + 31) / 32);  // M2lTc<P>::kKp
    Mh3 = slot<__nv_bfloat16>(c, kSlotM2lSplit, static_cast<size_t>(8) * nn * 3 * kp, &rc);  // 8 signed copies
    AMK_TRY(rc);
    m2l_split_kernel<<<static_cast<unsigned>((nn * kp + 255) / 256), 256, 0, c->stream>>>(nn, T.n_m, kp, T.multi, 8,
                                                                                        Mh, Mh3);
    AMK_TRY(check_launch(c, "m2l_split_kernel"));
  }
  const int n_buf = n_m2l > cap ? 2 : 1;
  for (int i = 0; i < n_buf; ++i)
    AMK_TRY(f->m2l_out[i].reserve(static_cast<size_t>(std::min(cap, n_m2l)) * T.n_m * esz));
  int chunk = 0;
  for (long e0 = 0; e0 < n_m2l; e0 += cap, ++chunk) {
    const long e1 = std::min(n_m2l, e0 + cap), ne = e1 - e0;
    const int buf = chunk & 1;
    void* out = f->m2l_out[buf].ptr;
    AMK_CUDA_TRY(cudaMemsetAsync(hist, 0, n_codes * sizeof(int), c->stream));
    AMK_CUDA_TRY(cudaMemsetAsync(counters, 0, 6 * sizeof(int), c->stream));  // [6]: the tensor-core status
    const unsigned ge = static_cast<unsigned>((ne + 255) / 256), gc = static_cast<unsigned>((n_codes + 255) / 256);
    m2l_histogram_kernel<<<ge, 256, 0, c->stream>>>(codes, e0, e1, hist, fallback, counters + 3);
    AMK_TRY(check_launch(c, "m2l_histogram_kernel"));
    m2l_code_flags_kernel<<<gc, 256, 0, c->stream>>>(hist, n_codes, kM2lMinClass, used, nunit);
    AMK_TRY(check_launch(c, "m2l_code_flags_kernel"));
    AMK_TRY(exclusive_scan_int(c, hist, n_codes, start, counters));
    AMK_TRY(exclusive_scan_int(c, used, n_codes, cls_index, counters + 1));
    AMK_TRY(exclusive_scan_int(c, nunit, n_codes, unit_start, counters + 2));
    m2l_class_fill_kernel<<<gc, 256, 0, c->stream>>>(hist, start, cls_index, unit_start, n_codes, used, cls_code,
                                                     cls_end, unit_cls, unit_pos);
    AMK_TRY(check_launch(c, "m2l_class_fill_kernel"));
    m2l_scatter_kernel<<<ge, 256, 0, c->stream>>>(codes, e0, e1, start, used, hist, perm, fallback, counters + 3,
                                                  refl);
    AMK_TRY(check_launch(c, "m2l_scatter_kernel"));
    int h[4] = {0, 0, 0, 0}, tr[2] = {0, 0};
    AMK_CUDA_TRY(cudaMemcpyAsync(h, counters, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    AMK_CUDA_TRY(cudaMemcpyAsync(tr, tgt + e0, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    AMK_CUDA_TRY(cudaMemcpyAsync(tr + 1, tgt + e1 - 1, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
    const int n_cls = h[1], n_units = h[2], n_fb = h[3];
    // the classes' pairs fill perm[0, h[0]) and every other pair is on the per-pair list
    if (static_cast<long>(h[0]) + n_fb != ne)
      return fail(AMK_ERR_STATE, "M2L chunk: %d class pairs + %d per-pair != %ld", h[0], n_fb, ne);
    f->stats[8] += ne - n_fb;
    f->stats[9] += n_cls;
    f->stats[10] += 1;
    // the sums of the chunk before the previous one still read this buffer
    if (chunk >= 2) AMK_CUDA_TRY(cudaStreamWaitEvent(c->stream, f->sums_done[buf], 0));
    if (n_cls > 0) {
      // D(v) per class: FP64 rows for the FP64 product, split BF16 rows for
      // the tensor-core product
      const int nd3 = tc_nd3(T.n_d);
      double* table = nullptr;
      uint2* table3 = nullptr;
      if (tc)
        table3 = slot<uint2>(c, kSlotM2lTable3, static_cast<size_t>(n_cls) * nd3, &rc);
      else
        table = slot<double>(c, kSlotM2lTable, static_cast<size_t>(n_cls) * T.n_d, &rc);
      AMK_TRY(rc);
      const size_t tsm = static_cast<size_t>(kFmmWarps) * T.n_d * sizeof(double);
      AMK_CUDA_TRY(cudaFuncSetAttribute(m2l_table_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(tsm)));
      m2l_table_kernel<<<(n_cls + kFmmWarps - 1) / kFmmWarps, 32 * kFmmWarps, tsm, c->stream>>>(
          T, cls_code, n_cls, keys, table, table3, nd3);
      AMK_TRY(check_launch(c, "m2l_table_kernel"));
      int4* ud = nullptr;
      int* psrc = nullptr;
      if (tc) {  // the tensor-core product's other inputs: unit descriptors, pair sources
        const long n_cp = ne - n_fb;  // pairs in classes: perm[0, n_cp)
        ud = slot<int4>(c, kSlotM2lUnitDesc, static_cast<size_t>(n_units), &rc);
        AMK_TRY(rc);
        psrc = slot<int>(c, kSlotM2lPairSrc, static_cast<size_t>(std::max<long>(1, n_cp)), &rc);
        AMK_TRY(rc);
        const long np_ = std::max<long>(n_units, n_cp);
        m2l_tc_prep_kernel<<<static_cast<unsigned>((np_ + 255) / 256), 256, 0, c->stream>>>(
            n_units, unit_cls, unit_pos, cls_code, cls_end, keys, static_cast<int>(n_cp), perm, gm.src, refl,
            static_cast<int>(nn), ud, psrc);
        AMK_TRY(check_launch(c, "m2l_tc_prep_kernel"));
      }
      AMK_TRY(phase_begin(c, AMK_PHASE_FMM_M2L_PRODUCTS));
      if (tc)
        AMK_TRY(class_tc(c, order, T, n_units, ud, perm, psrc, Mh3, table3, e0, static_cast<float*>(out),
                         tc_status));
      else
        AMK_TRY(class_product(c, order, T, n_units, counters + 4, unit_cls, unit_pos, cls_code, cls_end, perm,
                              gm.src, Mh, table, keys, e0, static_cast<double*>(out)));
      AMK_TRY(phase_end(c, AMK_PHASE_FMM_M2L_PRODUCTS));
      if (tc) {  // the signs s^g of the reflection-folded pairs
        m2l_refl_sign_kernel<<<static_cast<unsigned>((ne + 255) / 256), 256, 0, c->stream>>>(
            T, e0, e1, refl, static_cast<float*>(out));
        AMK_TRY(check_launch(c, "m2l_refl_sign_kernel"));
      }
    }
    if (n_fb > 0) {
      const size_t psm = static_cast<size_t>(kFmmWarps) * (T.n_d + T.n_m) * sizeof(double) +
                         static_cast<size_t>(T.n_m) * T.n_m * sizeof(short);
      auto launch_pairs = [&](auto kernel, auto* dst) -> int {
        AMK_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(psm)));
        int per_sm = 0, sms = 0;
        AMK_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 32 * kFmmWarps, psm));
        AMK_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
        const int grid = std::max(1, std::min((n_fb + kFmmWarps - 1) / kFmmWarps, std::max(1, per_sm) * sms));
        kernel<<<grid, 32 * kFmmWarps, psm, c->stream>>>(t, T, fallback, n_fb, tgt, gm.src, M, e0, dst);
        return check_launch(c, "m2l_pair_kernel");
      };
      if (tc)
        AMK_TRY(launch_pairs(m2l_pair_kernel<float>, static_cast<float*>(out)));
      else
        AMK_TRY(launch_pairs(m2l_pair_kernel<double>, static_cast<double*>(out)));
    }
    // after the per-pair products (run concurrently with them, the near
    // field took longer than both in sequence)
    if (e1 >= n_m2l && after_products) AMK_TRY(after_products());
    // per-target sums on the side stream, in chunk order
    AMK_CUDA_TRY(cudaEventRecord(f->products_done[buf], c->stream));
    AMK_CUDA_TRY(cudaStreamWaitEvent(f->side, f->products_done[buf], 0));
    if (tc)
      AMK_TRY(m2l_reduce(c, f->side, t, T, gm.off, gm.count, tr[0], tr[1] - tr[0] + 1, e0, e1,
                         static_cast<const float*>(out), L));
    else
      AMK_TRY(m2l_reduce(c, f->side, t, T, gm.off, gm.count, tr[0], tr[1] - tr[0] + 1, e0, e1,
                         static_cast<const double*>(out), L));
    AMK_CUDA_TRY(cudaEventRecord(f->sums_done[buf], f->side));
  }
  // the context stream resumes after the last sums
  AMK_CUDA_TRY(cudaStreamWaitEvent(c->stream, f->sums_done[(chunk - 1) & 1], 0));
  if (tc) {  // a tensor-core wait that timed out leaves its flag
    int st = 0;
    AMK_CUDA_TRY(cudaMemcpyAsync(&st, tc_status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (st) return fail(AMK_ERR_TIMEOUT, "tensor-core M2L product: an mbarrier wait timed out");
  }
  return AMK_OK;
}

// ------------------------------------------------------------ L2L
// Children at `depth` receive their parent's expansion (fast-multipole.cc:557-578).
// A warp per child, lanes over its coefficients; the offset's monomials
// d^c / c! and the parent's L_b b! are staged in shared memory first, so a
// term is one product; 1/a! is applied once per coefficient.
__global__ void __launch_bounds__(32 * kFmmWarps)
fmm_l2l_kernel(const Octree t, FmmDevTables T, int depth, double* __restrict__ L) {
  __shared__ double mono_s[kFmmWarps][kMaxNm], lps_s[kFmmWarps][kMaxNm];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int id = blockIdx.x * kFmmWarps + w;
  if (id >= t.n_nodes) return;
  if (t.meta[id].x != depth) return;
  const int par = t.parent[id];
  if (par < 0) return;
  const double4 c = t.center[id], pc = t.center[par];
  double px[kMaxOrder + 1], py[kMaxOrder + 1], pz[kMaxOrder + 1];
  powers(T.p, c.x - pc.x, c.y - pc.y, c.z - pc.z, px, py, pz);
  const double* lp = L + static_cast<size_t>(par) * T.n_m;
  double* lc = L + static_cast<size_t>(id) * T.n_m;
  double* mono = mono_s[w];
  double* lps = lps_s[w];
  for (int a = lane; a < T.n_m; a += 32) {
    const int4 m = T.multi[a];
    mono[a] = (px[m.x] * py[m.y] * pz[m.z]) * T.inv_fact[a];
    lps[a] = lp[a] * T.fact[a];
  }
  __syncwarp();
  for (int a = lane; a < T.n_m; a += 32) {
    double s = 0.0;
    for (int e = T.l2l_off[a]; e < T.l2l_off[a + 1]; ++e) s += lps[T.l2l_b[e]] * mono[T.l2l_c[e]];
    lc[a] += s * T.inv_fact[a];
  }
}

// ------------------------------------------------------------ L2P + P2P
// Work items = (target leaf, chunk of <= kP2PChunk source leaves of its P2P
// list; kP2P32Chunk in the FP32 near field); every leaf has at least one item (its L2P). A warp takes one item;
// its lanes are split into G = 32 / n_targets groups, group g summing every
// G-th source particle for all the leaf's targets, so small leaves still
// fill the warp. Group sums are added in group order and item partials in
// chunk order (fast-multipole.cc:580-661), so results do not depend on
// scheduling.
constexpr int kP2PChunk = 8;

__global__ void p2p_items_count_kernel(const Octree t, const int* __restrict__ count, int chunk,
                                       int* __restrict__ items, int* __restrict__ psize) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= t.n_nodes) return;
  int it = 0;
  if (t.meta[id].y) it = max(1, (count[id] + chunk - 1) / chunk);
  const int2 r = t.range[id];
  items[id] = it;
  psize[id] = it * (r.y - r.x);
}

__global__ void p2p_items_fill_kernel(const Octree t, const int* __restrict__ items, const int* __restrict__ ibase,
                                      int2* __restrict__ work, int* __restrict__ leaf_of) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= t.n_nodes || !t.meta[id].y) return;
  const int b = ibase[id];
  for (int c = 0; c < items[id]; ++c) work[b + c] = make_int2(id, c);
  const int2 r = t.range[id];
  for (int k = r.x; k < r.y; ++k) leaf_of[k] = id;
}

__global__ void __launch_bounds__(32 * kFmmWarps)
fmm_p2p_kernel(const Octree t, FmmDevTables T, const int2* __restrict__ work, int n_work,
               const int* __restrict__ off, const int* __restrict__ count, const int* __restrict__ src,
               const int* __restrict__ pbase, const double* __restrict__ L, double min_sq, bool want_phi,
               double4* __restrict__ part) {
  __shared__ double4 red[kFmmWarps][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int wi = blockIdx.x * kFmmWarps + w;
  if (wi >= n_work) return;
  const int2 item = work[wi];
  const int ti = item.x, chunk = item.y;
  const double4 tc = t.center[ti];
  const int2 tr = t.range[ti];
  const int nt_all = tr.y - tr.x;
  const int sb = off[ti] + chunk * kP2PChunk;
  const int se = min(off[ti] + count[ti], sb + kP2PChunk);
  double4* out = part + pbase[ti] + static_cast<size_t>(chunk) * nt_all;
  for (int base = tr.x; base < tr.y; base += 32) {
    const int nt = min(32, tr.y - base);
    const int groups = 32 / nt;
    const int g = lane / nt, tl = lane - g * nt;
    const bool active = g < groups;
    const int i = base + tl;
    double4 me = make_double4(0.0, 0.0, 0.0, 0.0);
    if (active) me = t.src[i];
    double pot = 0.0, fx = 0.0, fy = 0.0, fz = 0.0;
    if (active && g == 0 && chunk == 0) {  // L2P, once per target
      const double* l = L + static_cast<size_t>(ti) * T.n_m;
      double px[kMaxOrder + 1], py[kMaxOrder + 1], pz[kMaxOrder + 1];
      powers(T.p, me.x - tc.x, me.y - tc.y, me.z - tc.z, px, py, pz);
      if (want_phi)
        for (int gg = 0; gg < T.n_m; ++gg) {
          const int4 m = T.multi[gg];
          pot += l[gg] * (px[m.x] * py[m.y] * pz[m.z]);
        }
      double gx = 0.0, gy = 0.0, gz = 0.0;
      for (int gg = 1; gg < T.n_m; ++gg) {
        const int4 m = T.multi[gg];
        const int g0 = T.grad[3 * gg], g1 = T.grad[3 * gg + 1], g2 = T.grad[3 * gg + 2];
        if (g0 >= 0) {
          const int4 q = T.multi[g0];
          gx += m.x * l[gg] * (px[q.x] * py[q.y] * pz[q.z]);
        }
        if (g1 >= 0) {
          const int4 q = T.multi[g1];
          gy += m.y * l[gg] * (px[q.x] * py[q.y] * pz[q.z]);
        }
        if (g2 >= 0) {
          const int4 q = T.multi[g2];
          gz += m.z * l[gg] * (px[q.x] * py[q.y] * pz[q.z]);
        }
      }
      fx = -gx;
      fy = -gy;
      fz = -gz;
    }
    if (active) {
      for (int e = sb; e < se; ++e) {
        const int2 sr = t.range[src[e]];
        for (int j = sr.x + g; j < sr.y; j += groups) {
          const double4 s = t.src[j];
          if (j == i || s.w == 0.0) continue;
          const double rx = me.x - s.x, ry = me.y - s.y, rz = me.z - s.z;
          const double r2 = rx * rx + ry * ry + rz * rz;
          if (r2 < min_sq) continue;
          const double inv_r = rsqrt(r2);
          const double f = s.w * (inv_r * inv_r * inv_r);
          fx += rx * f;
          fy += ry * f;
          fz += rz * f;
          pot += s.w * inv_r;
        }
      }
    }
    red[w][lane] = make_double4(fx, fy, fz, pot);
    __syncwarp();
    if (active && g == 0) {
      double4 a = red[w][tl];
      for (int gg = 1; gg < groups; ++gg) {
        const double4 b = red[w][gg * nt + tl];
        a.x += b.x;
        a.y += b.y;
        a.z += b.z;
        a.w += b.w;
      }
      out[i - tr.x] = a;
    }
    __syncwarp();
  }
}

// Near field in FP32 (the tensor precision mode): the sorted sources in
// unit-cube coordinates as double-float pairs x = hi + lo (hi = float(x),
// lo = float(x - hi)) plus the charge; a pair's difference
// (x_i,hi - x_j,hi) + (x_i,lo - x_j,lo) is exact to FP32 rounding of |r_ij|
// for the neighbouring leaves of a P2P list (Sterbenz), so the pair terms
// carry FP32 relative error. Per-source-leaf partial sums are FP32 and are
// added to FP64 accumulators once per leaf.
__global__ void p2p_stage_kernel(const Octree t, float4* __restrict__ hi, float4* __restrict__ lo) {
  const long k = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  if (k >= t.m) return;
  const double4 s = t.src[k];
  const float hx = static_cast<float>(s.x), hy = static_cast<float>(s.y), hz = static_cast<float>(s.z);
  hi[k] = make_float4(hx, hy, hz, static_cast<float>(s.w));
  lo[k] = make_float4(static_cast<float>(s.x - hx), static_cast<float>(s.y - hy), static_cast<float>(s.z - hz),
                      0.f);
}

constexpr int kP2PStage = 64;  // source particles staged per warp at a time
constexpr int kP2P32Chunk = 16;  // source leaves per work item of the FP32 near field

// L2P in FP64 for particle i of leaf ti (centre tc): force and potential of
// the leaf's local expansion at the particle.
__device__ __forceinline__ double4 l2p_fp64(const Octree& t, const FmmDevTables& T, const double* __restrict__ L,
                                            int ti, const double4& tc, int i, bool want_phi) {
  const double4 me = t.src[i];
  const double* l = L + static_cast<size_t>(ti) * T.n_m;
  double px[kMaxOrder + 1], py[kMaxOrder + 1], pz[kMaxOrder + 1];
  powers(T.p, me.x - tc.x, me.y - tc.y, me.z - tc.z, px, py, pz);
  double pot = 0.0;
  if (want_phi)
    for (int gg = 0; gg < T.n_m; ++gg) {
      const int4 m = T.multi[gg];
      pot += l[gg] * (px[m.x] * py[m.y] * pz[m.z]);
    }
  double gx = 0.0, gy = 0.0, gz = 0.0;
  for (int gg = 1; gg < T.n_m; ++gg) {
    const int4 m = T.multi[gg];
    const int g0 = T.grad[3 * gg], g1 = T.grad[3 * gg + 1], g2 = T.grad[3 * gg + 2];
    if (g0 >= 0) {
      const int4 q = T.multi[g0];
      gx += m.x * l[gg] * (px[q.x] * py[q.y] * pz[q.z]);
    }
    if (g1 >= 0) {
      const int4 q = T.multi[g1];
      gy += m.y * l[gg] * (px[q.x] * py[q.y] * pz[q.z]);
    }
    if (g2 >= 0) {
      const int4 q = T.multi[g2];
      gz += m.z * l[gg] * (px[q.x] * py[q.y] * pz[q.z]);
    }
  }
  return make_double4(-gx, -gy, -gz, pot);
}

// Near-field pair sums of one work item (target leaf, up to kP2P32Chunk
// source leaves); the FP64 L2P runs in fmm_l2p_add_kernel.
// The arithmetic is packed over pairs of SOURCES: a lane holds its target's
// coordinates duplicated in both halves of FP32x2 registers and each packed
// operation evaluates the pair terms of two consecutive sources, so every
// pass is packed whatever the leaf's size. The sources of a leaf are staged
// by the warp in shared memory 64 at a time as pairs {x_hi, y_hi} {z_hi, q}
// {x_lo, y_lo} {z_lo} of two sources each (broadcast reads; an odd count is
// padded with a neutral source). Targets: two per lane while more than 48
// remain, else up to 32 at one per lane, with the lanes split into groups
// over the source pairs when 16 or fewer remain. A pair term is
//   r = (t_hi - s_hi) + (t_lo - s_lo)  (t - s formed as fma(s, -1, t)),
// exact to FP32 rounding of |r| for neighbouring leaves (Sterbenz), and is
// zero for a pair closer than the minimum distance (r^2 := +inf, so 1/r = 0;
// the particle itself included) or a neutral source. Each lane keeps FP32
// sums of its even and odd sources per source leaf, added to FP64 once per
// leaf in a fixed order, so results do not depend on scheduling.
struct P2PPairs {
  float4 a[kP2PStage / 2];  // {x_hi, x_hi'}, {y_hi, y_hi'}
  float4 b[kP2PStage / 2];  // {z_hi, z_hi'}, {q, q'}
  float4 c[kP2PStage / 2];  // {x_lo, x_lo'}, {y_lo, y_lo'}
  float2 d[kP2PStage / 2];  // {z_lo, z_lo'}
};

struct P2PTarget {
  float2 hx, hy, hz, lx, ly, lz;  // duplicated in both halves
  float2 ox, oy, oz;              // offset from a separated source leaf's centre (duplicated)
  float2 ax, ay, az, ap;          // even / odd source sums of the current leaf
  double4 acc;
};

// A source leaf separated from the target leaf: gap between their spheres
// (centre, radius) of at least half the summed radii. Its pairs use FP32
// offsets from the source leaf's centre c: r = (x_i - c) + (-(x_j - c)),
// each offset formed once from the double-float positions. The relative
// error of r is then at most 2 eps (1 + r_s / |r|) <= 6 eps, and r > 0
// (no pair below the minimum distance: the spheres are apart).
struct P2PCentre {
  float hx, hy, hz, lx, ly, lz;
};

__device__ __forceinline__ float2 dup2(float v) { return make_float2(v, v); }

__device__ __forceinline__ void p2p32_far_begin(P2PTarget& t, const P2PCentre& c) {
  t.ox = dup2((t.hx.x - c.hx) + (t.lx.x - c.lx));
  t.oy = dup2((t.hy.x - c.hy) + (t.ly.x - c.ly));
  t.oz = dup2((t.hz.x - c.hz) + (t.lz.x - c.lz));
}

// Far pair term of two sources: a = {-u_x, -u_x'} {-u_y, -u_y'}, b = {-u_z, -u_z'} {q, q'}.
__device__ __forceinline__ void p2p32_far_term(P2PTarget& t, const float4& a, const float4& b) {
  const float2 rx = __fadd2_rn(t.ox, make_float2(a.x, a.y));
  const float2 ry = __fadd2_rn(t.oy, make_float2(a.z, a.w));
  const float2 rz = __fadd2_rn(t.oz, make_float2(b.x, b.y));
  const float2 r2 = __ffma2_rn(rx, rx, __ffma2_rn(ry, ry, __fmul2_rn(rz, rz)));
  const float2 inv = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
  const float2 qr = __fmul2_rn(make_float2(b.z, b.w), inv);
  const float2 f = __fmul2_rn(qr, __fmul2_rn(inv, inv));
  t.ax = __ffma2_rn(rx, f, t.ax);
  t.ay = __ffma2_rn(ry, f, t.ay);
  t.az = __ffma2_rn(rz, f, t.az);
  t.ap = __fadd2_rn(t.ap, qr);
}

__device__ __forceinline__ void p2p32_load_target(P2PTarget& t, const float4* __restrict__ shi,
                                                  const float4* __restrict__ slo, int i) {
  const float4 h = shi[i], l = slo[i];
  t.hx = make_float2(h.x, h.x);
  t.hy = make_float2(h.y, h.y);
  t.hz = make_float2(h.z, h.z);
  t.lx = make_float2(l.x, l.x);
  t.ly = make_float2(l.y, l.y);
  t.lz = make_float2(l.z, l.z);
  t.acc = make_double4(0.0, 0.0, 0.0, 0.0);
}

__device__ __forceinline__ void p2p32_term(P2PTarget& t, const float4& a, const float4& b, const float4& c,
                                           const float2& d, float min_sq32) {
  const float2 m1 = make_float2(-1.f, -1.f);
  const float inf32 = __int_as_float(0x7f800000);
  const float2 rx = __fadd2_rn(__ffma2_rn(make_float2(a.x, a.y), m1, t.hx), __ffma2_rn(make_float2(c.x, c.y), m1, t.lx));
  const float2 ry = __fadd2_rn(__ffma2_rn(make_float2(a.z, a.w), m1, t.hy), __ffma2_rn(make_float2(c.z, c.w), m1, t.ly));
  const float2 rz = __fadd2_rn(__ffma2_rn(make_float2(b.x, b.y), m1, t.hz), __ffma2_rn(d, m1, t.lz));
  float2 r2 = __ffma2_rn(rx, rx, __ffma2_rn(ry, ry, __fmul2_rn(rz, rz)));
  r2.x = r2.x >= min_sq32 ? r2.x : inf32;
  r2.y = r2.y >= min_sq32 ? r2.y : inf32;
  const float2 inv = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
  const float2 qr = __fmul2_rn(make_float2(b.z, b.w), inv);
  const float2 f = __fmul2_rn(qr, __fmul2_rn(inv, inv));
  t.ax = __ffma2_rn(rx, f, t.ax);
  t.ay = __ffma2_rn(ry, f, t.ay);
  t.az = __ffma2_rn(rz, f, t.az);
  t.ap = __fadd2_rn(t.ap, qr);
}

__device__ __forceinline__ void p2p32_leaf_begin(P2PTarget& t) {
  t.ax = t.ay = t.az = t.ap = make_float2(0.f, 0.f);
}

__device__ __forceinline__ void p2p32_leaf_end(P2PTarget& t) {
  t.acc.x += static_cast<double>(t.ax.x) + static_cast<double>(t.ax.y);
  t.acc.y += static_cast<double>(t.ay.x) + static_cast<double>(t.ay.y);
  t.acc.z += static_cast<double>(t.az.x) + static_cast<double>(t.az.y);
  t.acc.w += static_cast<double>(t.ap.x) + static_cast<double>(t.ap.y);
}

// Stages sources [s0, s0 + ns) (ns <= kP2PStage) as pairs; returns the pairs.
__device__ __forceinline__ int p2p32_stage(P2PPairs& sp, const float4* __restrict__ shi,
                                           const float4* __restrict__ slo, int s0, int ns, int lane) {
  const int np = (ns + 1) >> 1;
  __syncwarp();
  if (lane < np) {
    const int j0 = s0 + 2 * lane;
    const bool two = 2 * lane + 1 < ns;
    const float4 h0 = shi[j0], l0 = slo[j0];
    float4 h1 = h0, l1 = l0;
    if (two) {
      h1 = shi[j0 + 1];
      l1 = slo[j0 + 1];
    } else {
      h1.w = 0.f;  // neutral padding source at the same position: a zero term
    }
    sp.a[lane] = make_float4(h0.x, h1.x, h0.y, h1.y);
    sp.b[lane] = make_float4(h0.z, h1.z, h0.w, h1.w);
    sp.c[lane] = make_float4(l0.x, l1.x, l0.y, l1.y);
    sp.d[lane] = make_float2(l0.z, l1.z);
  }
  __syncwarp();
  return np;
}

// Stages sources [s0, s0 + ns) of a separated leaf as negated FP32 offsets
// from its centre; returns the pairs (padding: a neutral source).
__device__ __forceinline__ int p2p32_stage_far(P2PPairs& sp, const float4* __restrict__ shi,
                                               const float4* __restrict__ slo, int s0, int ns, int lane,
                                               const P2PCentre& c) {
  const int np = (ns + 1) >> 1;
  __syncwarp();
  if (lane < np) {
    const int j0 = s0 + 2 * lane;
    const bool two = 2 * lane + 1 < ns;
    const float4 h0 = shi[j0], l0 = slo[j0];
    float4 h1 = h0, l1 = l0;
    if (two) {
      h1 = shi[j0 + 1];
      l1 = slo[j0 + 1];
    } else {
      h1.w = 0.f;
    }
    auto neg_off = [&](const float4& h, const float4& l, float& x, float& y, float& z) {
      x = -((h.x - c.hx) + (l.x - c.lx));
      y = -((h.y - c.hy) + (l.y - c.ly));
      z = -((h.z - c.hz) + (l.z - c.lz));
    };
    float x0, y0, z0, x1, y1, z1;
    neg_off(h0, l0, x0, y0, z0);
    neg_off(h1, l1, x1, y1, z1);
    sp.a[lane] = make_float4(x0, x1, y0, y1);
    sp.b[lane] = make_float4(z0, z1, h0.w, h1.w);
  }
  __syncwarp();
  return np;
}

__global__ void __launch_bounds__(32 * kFmmWarps, 6)  // 6 blocks per SM (80 registers): measured best of 4-6
fmm_p2p32_kernel(const Octree t, const int2* __restrict__ work, int n_work, const int* __restrict__ off,
                 const int* __restrict__ count, const int* __restrict__ src, const int* __restrict__ pbase,
                 double min_sq, const float4* __restrict__ shi, const float4* __restrict__ slo,
                 const double* __restrict__ radius, double4* __restrict__ part) {
  __shared__ double4 red[kFmmWarps][32];
  __shared__ P2PPairs stg[kFmmWarps];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int wi = blockIdx.x * kFmmWarps + w;
  if (wi >= n_work) return;
  const int2 item = work[wi];
  const int ti = item.x, chunk = item.y;
  const int2 tr = t.range[ti];
  const int nt_all = tr.y - tr.x;
  const int sb = off[ti] + chunk * kP2P32Chunk;
  const int se = min(off[ti] + count[ti], sb + kP2P32Chunk);
  double4* out = part + pbase[ti] + static_cast<size_t>(chunk) * nt_all;
  const float min_sq32 = fmaxf(static_cast<float>(min_sq), 1.17549435e-38f);
  P2PPairs& sp = stg[w];
  const double4 ct = t.center[ti];
  const double rt = radius[ti];
  // whether source leaf sl is separated (warp-uniform), and its centre
  auto separated = [&](int sl, P2PCentre& c) {
    const double4 cs = t.center[sl];
    const double dx = ct.x - cs.x, dy = ct.y - cs.y, dz = ct.z - cs.z;
    const double rs = radius[sl];
    const double gap = sqrt(dx * dx + dy * dy + dz * dz) - rt - rs;
    c.hx = static_cast<float>(cs.x);
    c.hy = static_cast<float>(cs.y);
    c.hz = static_cast<float>(cs.z);
    c.lx = static_cast<float>(cs.x - c.hx);
    c.ly = static_cast<float>(cs.y - c.hy);
    c.lz = static_cast<float>(cs.z - c.hz);
    return gap >= 0.5 * (rt + rs);
  };
  for (int base = tr.x; base < tr.y;) {
    const int rem = tr.y - base;
    if (rem > 48) {
      // ---- two targets per lane (the second may be past the leaf: computed, not written);
      // with 33-48 left, a one-per-lane pass of 32 and a grouped pass of the
      // rest cost less than the idle second slots (measured: 19.5 -> 19.3 ms
      // per 1M step)
      const int i0 = base + lane, i1 = min(base + 32 + lane, tr.y - 1);
      P2PTarget t0, t1;
      p2p32_load_target(t0, shi, slo, i0);
      p2p32_load_target(t1, shi, slo, i1);
      for (int e = sb; e < se; ++e) {
        const int sl = src[e];
        const int2 sr = t.range[sl];
        P2PCentre cc;
        const bool far = separated(sl, cc);
        p2p32_leaf_begin(t0);
        p2p32_leaf_begin(t1);
        if (far) {
          p2p32_far_begin(t0, cc);
          p2p32_far_begin(t1, cc);
          for (int s0 = sr.x; s0 < sr.y; s0 += kP2PStage) {
            const int np = p2p32_stage_far(sp, shi, slo, s0, min(kP2PStage, sr.y - s0), lane, cc);
#pragma unroll 2
            for (int q = 0; q < np; ++q) {
              const float4 a = sp.a[q], b = sp.b[q];
              p2p32_far_term(t0, a, b);
              p2p32_far_term(t1, a, b);
            }
          }
        } else {
          for (int s0 = sr.x; s0 < sr.y; s0 += kP2PStage) {
            const int np = p2p32_stage(sp, shi, slo, s0, min(kP2PStage, sr.y - s0), lane);
#pragma unroll 2
            for (int q = 0; q < np; ++q) {
              const float4 a = sp.a[q], b = sp.b[q], c = sp.c[q];
              const float2 d = sp.d[q];
              p2p32_term(t0, a, b, c, d, min_sq32);
              p2p32_term(t1, a, b, c, d, min_sq32);
            }
          }
        }
        p2p32_leaf_end(t0);
        p2p32_leaf_end(t1);
      }
      out[i0 - tr.x] = t0.acc;
      if (base + 32 + lane < tr.y) out[base + 32 + lane - tr.x] = t1.acc;
      base += 64;
      continue;
    }
    // ---- at most 32 targets: one per lane, lanes in groups over the source pairs
    const int nt = min(rem, 32);
    const int groups = 32 / nt;
    const int g = lane / nt, tl = lane - g * nt;
    const bool active = g < groups;
    const int i = base + tl;
    P2PTarget t0;
    p2p32_load_target(t0, shi, slo, active ? i : base);
    for (int e = sb; e < se; ++e) {
      const int sl = src[e];
      const int2 sr = t.range[sl];
      P2PCentre cc;
      const bool far = separated(sl, cc);
      p2p32_leaf_begin(t0);
      if (far) {
        p2p32_far_begin(t0, cc);
        for (int s0 = sr.x; s0 < sr.y; s0 += kP2PStage) {
          const int np = p2p32_stage_far(sp, shi, slo, s0, min(kP2PStage, sr.y - s0), lane, cc);
          if (active) {
#pragma unroll 2
            for (int q = g; q < np; q += groups) p2p32_far_term(t0, sp.a[q], sp.b[q]);
          }
        }
      } else {
        for (int s0 = sr.x; s0 < sr.y; s0 += kP2PStage) {
          const int np = p2p32_stage(sp, shi, slo, s0, min(kP2PStage, sr.y - s0), lane);
          if (active) {
#pragma unroll 2
            for (int q = g; q < np; q += groups) p2p32_term(t0, sp.a[q], sp.b[q], sp.c[q], sp.d[q], min_sq32);
          }
        }
      }
      p2p32_leaf_end(t0);
    }
    red[w][lane] = t0.acc;
    __syncwarp();
    if (active && g == 0) {
      double4 a = red[w][tl];
      for (int gg = 1; gg < groups; ++gg) {
        const double4 b = red[w][gg * nt + tl];
        a.x += b.x;
        a.y += b.y;
        a.z += b.z;
        a.w += b.w;
      }
      out[i - tr.x] = a;
    }
    __syncwarp();
    base += nt;
  }
}

// Per particle: item partials in chunk order.
__global__ void fmm_p2p_reduce_kernel(const Octree t, const int* __restrict__ leaf_of, const int* __restrict__ items,
                                      const int* __restrict__ pbase, const double4* __restrict__ part,
                                      double4* __restrict__ ef) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= t.m) return;
  const int leaf = leaf_of[k];
  const int2 r = t.range[leaf];
  const int nt = r.y - r.x;
  const double4* p = part + pbase[leaf] + (k - r.x);
  double4 a = p[0];
  for (int c = 1; c < items[leaf]; ++c) {
    const double4 b = p[static_cast<size_t>(c) * nt];
    a.x += b.x;
    a.y += b.y;
    a.z += b.z;
    a.w += b.w;
  }
  ef[k] = a;
}

// FP32 near-field path: the FP64 L2P of every particle added to its summed
// near field (a thread per particle; the table indices are the same on every
// lane and a leaf's coefficients are shared by its particles' lanes).
__global__ void fmm_l2p_add_kernel(const Octree t, FmmDevTables T, const int* __restrict__ leaf_of,
                                   const double* __restrict__ L, bool want_phi, double4* __restrict__ ef) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= t.m) return;
  const int leaf = leaf_of[k];
  const double4 l = l2p_fp64(t, T, L, leaf, t.center[leaf], k, want_phi);
  double4 a = ef[k];
  a.x += l.x;
  a.y += l.y;
  a.z += l.z;
  a.w += l.w;
  ef[k] = a;
}

__global__ void fmm_output_kernel(const Octree t, const double4* __restrict__ ef, double force_scale, View v,
                                  double* __restrict__ qphi) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= t.m) return;
  const double4 e = ef[k];
  const double q = t.src[k].w;
  const long i = t.order[k];
  const double s = force_scale * q;  // fast-multipole.cc:663-673
  v.fx[i] = s * e.x;
  v.fy[i] = s * e.y;
  v.fz[i] = s * e.z;
  if (qphi) qphi[k] = q * e.w;
}

// sum over P2P leaf pairs of |T| * |S| (particle pairs before self/min_sq skips)
__global__ void p2p_pair_count_kernel(const Octree t, const int2* __restrict__ pairs, const int* __restrict__ count,
                                      long cap, unsigned long long* out) {
  const long n = min(static_cast<long>(*count), cap);
  unsigned long long s = 0;
  for (long i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int2 p = pairs[i];
    const int2 a = t.range[p.x], b = t.range[p.y];
    s += static_cast<unsigned long long>(a.y - a.x) * static_cast<unsigned long long>(b.y - b.x);
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

__global__ void leaf_count_kernel(const Octree t, unsigned long long* out) {
  unsigned long long s = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < t.n_nodes; i += gridDim.x * blockDim.x)
    s += t.meta[i].y ? 1 : 0;
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

__global__ void zero_forces_kernel(View v) {
  const long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  if (i >= v.n) return;
  v.fx[i] = 0.0;
  v.fy[i] = 0.0;
  v.fz[i] = 0.0;
}

int group_pairs(amk_ctx* c, const int2* pairs, long n_pairs, long n_nodes, int slot_off, int slot_cnt, int slot_src,
                int slot_cursor, Grouped* g) {
  (void)slot_cursor;
  int rc = AMK_OK;
  g->off = slot<int>(c, slot_off, n_nodes + 1, &rc);
  AMK_TRY(rc);
  g->count = slot<int>(c, slot_cnt, n_nodes + 1, &rc);
  AMK_TRY(rc);
  g->src = slot<int>(c, slot_src, std::max<long>(n_pairs, 1), &rc);
  AMK_TRY(rc);
  int* total = slot<int>(c, kSlotStatus, 8, &rc) + 6;
  AMK_TRY(rc);
  AMK_CUDA_TRY(cudaMemsetAsync(g->count, 0, (n_nodes + 1) * sizeof(int), c->stream));
  if (n_pairs > 0) {
    int bits = 1;
    while ((1L << bits) < n_nodes) ++bits;
    uint64_t* keys = slot<uint64_t>(c, kSlotKeysA, n_pairs, &rc);
    AMK_TRY(rc);
    uint32_t* vals = slot<uint32_t>(c, kSlotValsA, n_pairs, &rc);
    AMK_TRY(rc);
    uint64_t* skeys = slot<uint64_t>(c, kSlotTreeKeys, n_pairs, &rc);
    AMK_TRY(rc);
    uint32_t* svals = slot<uint32_t>(c, kSlotSorted0, n_pairs, &rc);
    AMK_TRY(rc);
    const unsigned gp = static_cast<unsigned>((n_pairs + 255) / 256);
    pair_pack_kernel<<<gp, 256, 0, c->stream>>>(pairs, static_cast<int>(n_pairs), bits, keys, vals);
    AMK_TRY(check_launch(c, "pair_pack_kernel"));
    AMK_TRY(radix_sort_pairs(c, keys, vals, skeys, svals, n_pairs, 2 * bits));
    pair_unpack_kernel<<<gp, 256, 0, c->stream>>>(skeys, static_cast<int>(n_pairs), bits, g->src, g->count);
    AMK_TRY(check_launch(c, "pair_unpack_kernel"));
  }
  return exclusive_scan_int(c, g->count, n_nodes, g->off, total);
}

}  // namespace

// State of one FMM evaluation kept for the output, learned-correction and
// audit steps (all device pointers into the context's scratch).
struct FmmRun {
  Octree t;
  FmmDevTables T;
  TreeFrame hf;
  double* M = nullptr;
  double* L = nullptr;
  double* radius = nullptr;
  double4* ef = nullptr;      // per sorted source: E (unit-cube units, per unit charge), phi
  int* leaf_of = nullptr;     // sorted source -> leaf node
  int* p2p_count = nullptr;   // per node: P2P source leaves
};

int fmm_run(amk_ctx* c, const View& v, int order, double theta, long leaf_capacity, bool want_phi, FmmRun* run) {
  run->t = Octree{};
  const long n = v.n;
  if (n == 0) return AMK_OK;
  order = std::min(std::max(order, 1), kMaxOrder);  // fast-multipole.cc:324-328
  zero_forces_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, c->stream>>>(v);
  AMK_TRY(check_launch(c, "zero_forces_kernel"));
  FmmDevTables T;
  AMK_TRY(get_tables(c, order, &T));
  Octree t;
  AMK_TRY(phase_begin(c, AMK_PHASE_TREE));
  AMK_TRY(build_octree(c, v, static_cast<int>(std::min<long>(leaf_capacity, 1 << 20)), 1, &t));
  AMK_TRY(phase_end(c, AMK_PHASE_TREE));
  if (t.m == 0) return AMK_OK;
  const long nn = t.n_nodes;
  int rc = AMK_OK;
  double* radius = slot<double>(c, kSlotFmmRadius, nn, &rc);
  AMK_TRY(rc);
  double* M = slot<double>(c, kSlotFmmM, static_cast<size_t>(nn) * T.n_m, &rc);
  AMK_TRY(rc);
  double* Lx = slot<double>(c, kSlotFmmL, static_cast<size_t>(nn) * T.n_m, &rc);
  AMK_TRY(rc);
  const unsigned gn = static_cast<unsigned>((nn + 255) / 256);
  const unsigned gw = static_cast<unsigned>((nn + kFmmWarps - 1) / kFmmWarps);

  // ---- upward pass: the radii on the context stream, then P2M / M2M on
  // their own stream while the traversal (radii only) runs
  Fmm* f = c->fmm;
  if (!f->up) {
    AMK_CUDA_TRY(cudaStreamCreateWithFlags(&f->up, cudaStreamNonBlocking));
    AMK_CUDA_TRY(cudaEventCreateWithFlags(&f->up_start, cudaEventDisableTiming));
    AMK_CUDA_TRY(cudaEventCreateWithFlags(&f->up_done, cudaEventDisableTiming));
  }
  AMK_TRY(phase_begin(c, AMK_PHASE_FMM_UP));
  fmm_leaf_radius_kernel<<<gn, 256, 0, c->stream>>>(t, radius);
  AMK_TRY(check_launch(c, "fmm_leaf_radius_kernel"));
  for (int d = t.max_depth; d >= 0; --d) {
    fmm_parent_radius_kernel<<<gn, 256, 0, c->stream>>>(t, d, radius);
    AMK_TRY(check_launch(c, "fmm_parent_radius_kernel"));
  }
  AMK_CUDA_TRY(cudaEventRecord(f->up_start, c->stream));
  AMK_CUDA_TRY(cudaStreamWaitEvent(f->up, f->up_start, 0));
  fmm_p2m_kernel<<<gw, 32 * kFmmWarps, 0, f->up>>>(t, T, M);
  AMK_TRY(check_launch(c, "fmm_p2m_kernel"));
  for (int d = t.max_depth; d >= 0; --d) {
    fmm_m2m_kernel<<<gw, 32 * kFmmWarps, 0, f->up>>>(t, T, d, M);
    AMK_TRY(check_launch(c, "fmm_m2m_kernel"));
  }
  AMK_CUDA_TRY(cudaEventRecord(f->up_done, f->up));
  AMK_TRY(phase_end(c, AMK_PHASE_FMM_UP));

  // ---- interaction lists: every level of the traversal is launched without
  // reading its size back (a pair's depth sum grows by one per level, so
  // there are at most 2 max_depth + 1 levels); one read-back at the end
  // checks the capacities, and a traversal that overflowed one runs again
  // with larger lists
  AMK_TRY(phase_begin(c, AMK_PHASE_FMM_LISTS));
  FmmLists& lists = c->fmm->lists;
  const int n_levels = 2 * t.max_depth + 1;
  const int n_tv = 8 + n_levels + 1;  // m2l, p2p, overflow, -, -, -, -, -, pairs per level
  int* tv = slot<int>(c, kSlotFmmAux0, n_tv, &rc);
  AMK_TRY(rc);
  unsigned long long* cnt64 = slot<unsigned long long>(c, kSlotFmmAux1, 4, &rc);
  AMK_TRY(rc);
  const double theta2 = theta * theta;
  double4* rec = slot<double4>(c, kSlotFmmNodeRec, nn, &rc);
  AMK_TRY(rc);
  fmm_node_record_kernel<<<gn, 256, 0, c->stream>>>(t, radius, rec);
  AMK_TRY(check_launch(c, "fmm_node_record_kernel"));
  long n_m2l = 0, n_p2p = 0;
  std::vector<int> hv(n_tv);
  unsigned long long h64[2] = {0, 0};
  TreeFrame hf;
  long want_front = std::max({lists.need_front, 8 * nn, 1024L});
  long want_m2l = std::max({lists.need_m2l, 64 * nn, 1024L}), want_p2p = std::max({lists.need_p2p, 16 * nn, 1024L});
  if (const char* env = getenv("AMK_FMM_LIST_CAP")) {  // small first capacities (tests of the overflow retry)
    const long v = atol(env);
    if (v > 0) {
      lists.cur.release();
      lists.next.release();
      lists.m2l.release();
      lists.p2p.release();
      want_front = want_m2l = want_p2p = v;
    }
  }
  for (int attempt = 0;; ++attempt) {
    if (attempt > 12) return fail(AMK_ERR_LIMIT, "FMM traversal: interaction lists did not fit");
    AMK_TRY(lists.cur.reserve(static_cast<size_t>(want_front) * sizeof(int2)));
    AMK_TRY(lists.next.reserve(static_cast<size_t>(want_front) * sizeof(int2)));
    AMK_TRY(lists.m2l.reserve(static_cast<size_t>(want_m2l) * sizeof(int2)));
    AMK_TRY(lists.p2p.reserve(static_cast<size_t>(want_p2p) * sizeof(int2)));
    TraverseLists tl;
    tl.m2l = lists.m2l.as<int2>();
    tl.p2p = lists.p2p.as<int2>();
    tl.cap_front = static_cast<long>(std::min(lists.cur.bytes, lists.next.bytes) / sizeof(int2));
    tl.cap_m2l = static_cast<long>(lists.m2l.bytes / sizeof(int2));
    tl.cap_p2p = static_cast<long>(lists.p2p.bytes / sizeof(int2));
    AMK_CUDA_TRY(cudaMemsetAsync(tv, 0, n_tv * sizeof(int), c->stream));
    fmm_traverse_root_kernel<<<1, 32, 0, c->stream>>>(lists.cur.as<int2>(), tv + 8);
    AMK_TRY(check_launch(c, "fmm_traverse_root_kernel"));
    const unsigned grid = static_cast<unsigned>(std::min<long>((tl.cap_front + 255) / 256, 148L * 8));
    for (int level = 0; level < n_levels; ++level) {
      int2* a = (level & 1) ? lists.next.as<int2>() : lists.cur.as<int2>();
      int2* b = (level & 1) ? lists.cur.as<int2>() : lists.next.as<int2>();
      fmm_traverse_kernel<<<grid, 256, 0, c->stream>>>(t, rec, theta2, a, b, tl, tv + 8 + level, tv);
      AMK_TRY(check_launch(c, "fmm_traverse_kernel"));
    }
    // statistics: leaves and P2P particle pairs (before self / min_sq skips)
    AMK_CUDA_TRY(cudaMemsetAsync(cnt64, 0, 2 * sizeof(unsigned long long), c->stream));
    p2p_pair_count_kernel<<<148, 256, 0, c->stream>>>(t, tl.p2p, tv + 1, tl.cap_p2p, cnt64);
    AMK_TRY(check_launch(c, "p2p_pair_count_kernel"));
    leaf_count_kernel<<<148, 256, 0, c->stream>>>(t, cnt64 + 1);
    AMK_TRY(check_launch(c, "leaf_count_kernel"));
    AMK_CUDA_TRY(cudaMemcpyAsync(hv.data(), tv, n_tv * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    AMK_CUDA_TRY(cudaMemcpyAsync(h64, cnt64, sizeof(h64), cudaMemcpyDeviceToHost, c->stream));
    AMK_CUDA_TRY(cudaMemcpyAsync(&hf, t.frame, sizeof(hf), cudaMemcpyDeviceToHost, c->stream));
    AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
    long max_front = 1;
    for (int level = 0; level <= n_levels; ++level) max_front = std::max<long>(max_front, hv[8 + level]);
    if (hv[3] != 0) return fail(AMK_ERR_STATE, "FMM traversal: a list entry is not a pair of nodes");
    if (hv[2] == 0) {
      if (hv[8 + n_levels] != 0) return fail(AMK_ERR_STATE, "FMM traversal: pairs left after the deepest level");
      n_m2l = hv[0];
      n_p2p = hv[1];
      lists.need_front = max_front;
      lists.need_m2l = n_m2l;
      lists.need_p2p = n_p2p;
      break;
    }
    // counts past a capacity keep growing, so they bound the sizes from below
    want_front = std::max(2 * tl.cap_front, max_front);
    want_m2l = hv[0] > tl.cap_m2l ? std::max(2 * tl.cap_m2l, static_cast<long>(hv[0])) : tl.cap_m2l;
    want_p2p = hv[1] > tl.cap_p2p ? std::max(2 * tl.cap_p2p, static_cast<long>(hv[1])) : tl.cap_p2p;
  }
  {  // statistics: nodes, leaves, M2L pairs, P2P leaf pairs, P2P particle pairs, depth
    long* st = c->fmm->stats;
    st[0] = nn;
    st[8] = st[9] = st[10] = 0;  // filled by the M2L products
    st[1] = static_cast<long>(h64[1]);
    st[2] = n_m2l;
    st[3] = n_p2p;
    st[4] = static_cast<long>(h64[0]);
    st[5] = t.max_depth;
    st[6] = t.m;
    st[7] = order;
  }
  Grouped gm, gp;
  AMK_TRY(group_pairs(c, lists.m2l.as<int2>(), n_m2l, nn, kSlotFmmLists0, kSlotFmmLists1, kSlotFmmWork0,
                      kSlotFmmWork1, &gm));
  AMK_TRY(group_pairs(c, lists.p2p.as<int2>(), n_p2p, nn, kSlotFmmLists2, kSlotFmmLists3, kSlotFmmWork2,
                      kSlotFmmWork3, &gp));
  AMK_TRY(phase_end(c, AMK_PHASE_FMM_LISTS));

  // ---- near-field set-up: work items (a target leaf and up to kP2PChunk
  // source leaves of its list, kP2P32Chunk in the FP32 near field) and the
  // per-item partial sums' layout
  double4* ef = slot<double4>(c, kSlotFmmWork4, t.m, &rc);
  AMK_TRY(rc);
  const double min_sq = kMinSquaredDistance / (hf.length * hf.length);
  const bool f32 = c->fmm_precision == AMK_FMM_TENSOR;
  AMK_TRY(phase_begin(c, AMK_PHASE_FMM_P2P));
  int* items = slot<int>(c, kSlotFmmAux2, nn + 1, &rc);
  AMK_TRY(rc);
  int* psize = slot<int>(c, kSlotTreeCount, nn + 1, &rc);  // tree build scratch, free again
  AMK_TRY(rc);
  int* ibase = slot<int>(c, kSlotTreeBase, nn + 1, &rc);
  AMK_TRY(rc);
  int* pbase = slot<int>(c, kSlotTreeL, nn + 1, &rc);
  AMK_TRY(rc);
  int* totals = slot<int>(c, kSlotFmmAux1, 8, &rc);
  AMK_TRY(rc);
  p2p_items_count_kernel<<<gn, 256, 0, c->stream>>>(t, gp.count, f32 ? kP2P32Chunk : kP2PChunk, items, psize);
  AMK_TRY(check_launch(c, "p2p_items_count_kernel"));
  AMK_TRY(exclusive_scan_int(c, items, nn, ibase, totals));
  AMK_TRY(exclusive_scan_int(c, psize, nn, pbase, totals + 1));
  int ht[2] = {0, 0};
  AMK_CUDA_TRY(cudaMemcpyAsync(ht, totals, sizeof(ht), cudaMemcpyDeviceToHost, c->stream));
  AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
  int2* work = slot<int2>(c, kSlotP2PWork, ht[0] + 1, &rc);
  AMK_TRY(rc);
  int* leaf_of = slot<int>(c, kSlotTreeLeafDepth, t.m + 1, &rc);
  AMK_TRY(rc);
  double4* part = slot<double4>(c, kSlotP2PPart, static_cast<size_t>(ht[1]) + 1, &rc);
  AMK_TRY(rc);
  float4* stage = nullptr;
  if (f32) {
    stage = slot<float4>(c, kSlotP2PStage, 2 * static_cast<size_t>(t.m), &rc);
    AMK_TRY(rc);
  }
  p2p_items_fill_kernel<<<gn, 256, 0, c->stream>>>(t, items, ibase, work, leaf_of);
  AMK_TRY(check_launch(c, "p2p_items_fill_kernel"));
  AMK_TRY(phase_end(c, AMK_PHASE_FMM_P2P));
  const unsigned gwork = static_cast<unsigned>((ht[0] + kFmmWarps - 1) / kFmmWarps);
  // FP32 near field: its pair sums need no expansion, so they run on their
  // own stream once the last M2L products are enqueued (the product kernel
  // holds every SM's shared memory), concurrently with the per-target M2L
  // sums and L2L; the FP64 L2P is added after L2L on the context stream
  auto launch_near = [&]() -> int {
    if (!f->near) {
      AMK_CUDA_TRY(cudaStreamCreateWithFlags(&f->near, cudaStreamNonBlocking));
      AMK_CUDA_TRY(cudaEventCreateWithFlags(&f->near_start, cudaEventDisableTiming));
      AMK_CUDA_TRY(cudaEventCreateWithFlags(&f->near_done, cudaEventDisableTiming));
    }
    AMK_CUDA_TRY(cudaEventRecord(f->near_start, c->stream));
    AMK_CUDA_TRY(cudaStreamWaitEvent(f->near, f->near_start, 0));
    p2p_stage_kernel<<<static_cast<unsigned>((t.m + 255) / 256), 256, 0, f->near>>>(t, stage, stage + t.m);
    AMK_TRY(check_launch(c, "p2p_stage_kernel"));
    AMK_TRY(phase_begin_on(c, AMK_PHASE_FMM_NEAR, f->near));
    fmm_p2p32_kernel<<<gwork, 32 * kFmmWarps, 0, f->near>>>(t, work, ht[0], gp.off, gp.count, gp.src, pbase, min_sq,
                                                            stage, stage + t.m, radius, part);
    AMK_TRY(check_launch(c, "fmm_p2p32_kernel"));
    AMK_TRY(phase_end_on(c, AMK_PHASE_FMM_NEAR, f->near));
    fmm_p2p_reduce_kernel<<<static_cast<unsigned>((t.m + 255) / 256), 256, 0, f->near>>>(t, leaf_of, items, pbase,
                                                                                       part, ef);
    AMK_TRY(check_launch(c, "fmm_p2p_reduce_kernel"));
    AMK_CUDA_TRY(cudaEventRecord(f->near_done, f->near));
    return AMK_OK;
  };
  const std::function<int()> no_hook;

  // ---- M2L (the multipoles: join the upward pass)
  AMK_CUDA_TRY(cudaStreamWaitEvent(c->stream, f->up_done, 0));
  AMK_CUDA_TRY(cudaMemsetAsync(Lx, 0, static_cast<size_t>(nn) * T.n_m * sizeof(double), c->stream));
  AMK_TRY(phase_begin(c, AMK_PHASE_FMM_M2L));
  if (n_m2l > 0) {
    const std::function<int()> hook(launch_near);
    AMK_TRY(m2l_products(c, order, t, T, gm, n_m2l, M, Lx, f32 ? hook : no_hook));
  } else if (f32) {
    AMK_TRY(launch_near());
  }
  AMK_TRY(phase_end(c, AMK_PHASE_FMM_M2L));

  // ---- L2L
  AMK_TRY(phase_begin(c, AMK_PHASE_FMM_DOWN));
  for (int d = 1; d <= t.max_depth; ++d) {
    fmm_l2l_kernel<<<gw, 32 * kFmmWarps, 0, c->stream>>>(t, T, d, Lx);
    AMK_TRY(check_launch(c, "fmm_l2l_kernel"));
  }
  AMK_TRY(phase_end(c, AMK_PHASE_FMM_DOWN));

  // ---- L2P + P2P
  AMK_TRY(phase_begin(c, AMK_PHASE_FMM_P2P));
  if (f32) {  // join the near-field stream, then the FP64 L2P
    AMK_CUDA_TRY(cudaStreamWaitEvent(c->stream, f->near_done, 0));
    fmm_l2p_add_kernel<<<static_cast<unsigned>((t.m + 127) / 128), 128, 0, c->stream>>>(t, T, leaf_of, Lx, want_phi,
                                                                                        ef);
    AMK_TRY(check_launch(c, "fmm_l2p_add_kernel"));
  } else {
    fmm_p2p_kernel<<<gwork, 32 * kFmmWarps, 0, c->stream>>>(t, T, work, ht[0], gp.off, gp.count, gp.src, pbase, Lx,
                                                            min_sq, want_phi, part);
    AMK_TRY(check_launch(c, "fmm_p2p_kernel"));
    fmm_p2p_reduce_kernel<<<static_cast<unsigned>((t.m + 255) / 256), 256, 0, c->stream>>>(t, leaf_of, items, pbase,
                                                                                          part, ef);
    AMK_TRY(check_launch(c, "fmm_p2p_reduce_kernel"));
  }
  run->leaf_of = leaf_of;
  AMK_TRY(phase_end(c, AMK_PHASE_FMM_P2P));
  run->t = t;
  run->T = T;
  run->hf = hf;
  run->M = M;
  run->L = Lx;
  run->radius = radius;
  run->ef = ef;
  run->p2p_count = gp.count;
  return AMK_OK;
}

int fmm_apply_learned(amk_ctx* c, const FmmRun& r);  // below

int fmm_forces(amk_ctx* c, const View& v, int order, double theta, long leaf_capacity, bool learned,
               double* energy_out) {
  if (energy_out) *energy_out = 0.0;
  if (v.n == 0) return AMK_OK;
  FmmRun r;
  AMK_TRY(fmm_run(c, v, learned ? 2 : order, theta, leaf_capacity, energy_out != nullptr, &r));
  if (r.t.m == 0) return AMK_OK;
  if (learned) AMK_TRY(fmm_apply_learned(c, r));
  const Octree& t = r.t;
  int rc = AMK_OK;
  double* qphi = nullptr;
  if (energy_out) {
    qphi = slot<double>(c, kSlotFmmWork5, t.m, &rc);
    AMK_TRY(rc);
  }
  const double force_scale = kCoulombConstant / (r.hf.length * r.hf.length);
  fmm_output_kernel<<<static_cast<unsigned>((t.m + 255) / 256), 256, 0, c->stream>>>(t, r.ef, force_scale, v, qphi);
  AMK_TRY(check_launch(c, "fmm_output_kernel"));
  if (energy_out) {
    double* res = slot<double>(c, kSlotAuxState4, 8, &rc);
    AMK_TRY(rc);
    AMK_TRY(reduce_sum(c, qphi, t.m, res));
    double h = 0.0;
    AMK_CUDA_TRY(cudaMemcpyAsync(&h, res, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
    *energy_out = 0.5 * kCoulombConstant / r.hf.length * h;  // fast-multipole.cc:676-680
  }
  return AMK_OK;
}

// ====================================================================== learned
// Per-particle features of the learned far-field correction (35 values, all
// dimensionless; x in unit-cube coordinates, leaf centre c, half edge h,
// E = E_far + E_near the p=2 FMM field at the particle):
//   0-2   u = (x - c) / h                    3-5   2 c (position in the cloud)
//   6-8   E_far / |E|                        9-11  E_near / |E|
//   12-14 degree-1 local coefficients / |E|  15-20 degree-2 local coefficients * h / |E|
//   21    log2(h) / 10                       22-24 leaf charge centroid offset / h
//   25-30 leaf second moments / (Q h^2)      31    leaf particle count / 32
//   32    leaf radius / h                    33    P2P source leaves / 64
//   34    1
// The neglected far-field terms (higher derivatives of the far potential,
// higher source moments) vary smoothly with position in the cloud, which is
// what the network learns. It predicts 100 (E_exact - E_fmm) / |E|: the
// relative far-field error, scaled to order one.
constexpr int kFeat = 35;
constexpr double kTargetScale = 100.0;
// The correction is bounded: a predicted relative error above 20 % of |E|
// (far beyond the p=2 truncation error) or not finite is scaled back to it,
// so a network queried outside its training distribution cannot inject an
// unbounded force. Features are clipped to +-64 for the same reason.
constexpr double kMaxPred = 0.2 * kTargetScale;
constexpr float kMaxFeature = 64.0f;

__global__ void fmm_features_kernel(const Octree t, FmmDevTables T, const double* __restrict__ L,
                                    const double* __restrict__ M, const double* __restrict__ radius,
                                    const int* __restrict__ p2p_count, const int* __restrict__ leaf_of,
                                    const double4* __restrict__ ef, const int* __restrict__ sel, int n_sel,
                                    float* __restrict__ feat, double* __restrict__ scale) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_sel) return;
  const int k = sel ? sel[s] : s;
  const int leaf = leaf_of[k];
  const double4 cc = t.center[leaf];
  const double h = cc.w;
  const double4 me = t.src[k];
  const double dx = me.x - cc.x, dy = me.y - cc.y, dz = me.z - cc.z;
  const double* l = L + static_cast<size_t>(leaf) * T.n_m;  // p = 2: 10 coefficients
  // E_far = -grad sum_g L_g d^g for degree <= 2 (index order of FmmTables)
  // indices: 0:(000) 1:(100) 2:(010) 3:(001) 4:(200) 5:(110) 6:(101) 7:(020) 8:(011) 9:(002)
  const double efx = -(l[1] + 2.0 * l[4] * dx + l[5] * dy + l[6] * dz);
  const double efy = -(l[2] + l[5] * dx + 2.0 * l[7] * dy + l[8] * dz);
  const double efz = -(l[3] + l[6] * dx + l[8] * dy + 2.0 * l[9] * dz);
  const double4 e = ef[k];
  const double se = sqrt(e.x * e.x + e.y * e.y + e.z * e.z) + 1e-300;
  float* f = feat + static_cast<size_t>(s) * kFeat;
  f[0] = static_cast<float>(dx / h);
  f[1] = static_cast<float>(dy / h);
  f[2] = static_cast<float>(dz / h);
  f[3] = static_cast<float>(2.0 * cc.x);
  f[4] = static_cast<float>(2.0 * cc.y);
  f[5] = static_cast<float>(2.0 * cc.z);
  f[6] = static_cast<float>(efx / se);
  f[7] = static_cast<float>(efy / se);
  f[8] = static_cast<float>(efz / se);
  f[9] = static_cast<float>((e.x - efx) / se);
  f[10] = static_cast<float>((e.y - efy) / se);
  f[11] = static_cast<float>((e.z - efz) / se);
  for (int g = 1; g <= 3; ++g) f[11 + g] = static_cast<float>(l[g] / se);
  for (int g = 4; g <= 9; ++g) f[11 + g] = static_cast<float>(l[g] * h / se);
  f[21] = static_cast<float>(log2(h) / 10.0);
  const double* mm = M + static_cast<size_t>(leaf) * T.n_m;
  const double q0 = mm[0];
  const bool has_q = q0 != 0.0;
  for (int g = 1; g <= 3; ++g) f[21 + g] = has_q ? static_cast<float>(mm[g] / (q0 * h)) : 0.f;
  for (int g = 4; g <= 9; ++g) f[21 + g] = has_q ? static_cast<float>(mm[g] / (q0 * h * h)) : 0.f;
  const int2 rr = t.range[leaf];
  f[31] = static_cast<float>(rr.y - rr.x) / 32.f;
  f[32] = static_cast<float>(radius[leaf] / h);
  f[33] = static_cast<float>(p2p_count[leaf]) / 64.f;
  f[34] = 1.f;
  for (int i = 0; i < kFeat; ++i) f[i] = isfinite(f[i]) ? fminf(fmaxf(f[i], -kMaxFeature), kMaxFeature) : 0.f;
  scale[s] = se / kTargetScale;
}

__global__ void fmm_correct_kernel(const float* __restrict__ pred, const double* __restrict__ scale, int m,
                                   double4* __restrict__ ef) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  double4 e = ef[k];
  const double px = pred[3 * k + 0], py = pred[3 * k + 1], pz = pred[3 * k + 2];
  const double n2 = px * px + py * py + pz * pz;
  const double lim = n2 <= kMaxPred * kMaxPred ? 1.0 : (isfinite(n2) ? kMaxPred / sqrt(n2) : 0.0);
  e.x += scale[k] * lim * px;
  e.y += scale[k] * lim * py;
  e.z += scale[k] * lim * pz;
  ef[k] = e;
}

int fmm_apply_learned(amk_ctx* c, const FmmRun& r) {
  const int m = static_cast<int>(r.t.m);
  int rc = AMK_OK;
  float* feat = slot<float>(c, kSlotMlp5, static_cast<size_t>(m) * kFeat, &rc);
  AMK_TRY(rc);
  double* scale = slot<double>(c, kSlotAuxState0, m, &rc);
  AMK_TRY(rc);
  float* pred = slot<float>(c, kSlotMlp4, static_cast<size_t>(m) * 3, &rc);
  AMK_TRY(rc);
  fmm_features_kernel<<<(m + 255) / 256, 256, 0, c->stream>>>(r.t, r.T, r.L, r.M, r.radius, r.p2p_count, r.leaf_of,
                                                               r.ef, nullptr, m, feat, scale);
  AMK_TRY(check_launch(c, "fmm_features_kernel"));
  AMK_TRY(mlp_forward_device(c, feat, m, pred));
  fmm_correct_kernel<<<(m + 255) / 256, 256, 0, c->stream>>>(pred, scale, m, r.ef);
  return check_launch(c, "fmm_correct_kernel");
}

// Exact FP64 field (unit-cube units, per unit charge) at selected sorted
// sources from all sources: a thread per target, sources staged in tiles.
__global__ void __launch_bounds__(256)
exact_field_kernel(const Octree t, const int* __restrict__ sel, int n_sel, double min_sq, double4* __restrict__ out) {
  __shared__ double4 tile[256];
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = s < n_sel ? sel[s] : -1;
  double4 me = make_double4(0.0, 0.0, 0.0, 0.0);
  if (k >= 0) me = t.src[k];
  double ex = 0.0, ey = 0.0, ez = 0.0;
  for (long base = 0; base < t.m; base += 256) {
    __syncthreads();
    const long j = base + threadIdx.x;
    tile[threadIdx.x] = j < t.m ? t.src[j] : make_double4(0.0, 0.0, 0.0, 0.0);
    __syncthreads();
    const int cnt = static_cast<int>(min(256L, t.m - base));
    if (k < 0) continue;
    for (int u = 0; u < cnt; ++u) {
      const double4 q = tile[u];
      if (base + u == k || q.w == 0.0) continue;
      const double rx = me.x - q.x, ry = me.y - q.y, rz = me.z - q.z;
      const double r2 = rx * rx + ry * ry + rz * rz;
      if (r2 < min_sq) continue;
      const double inv = rsqrt(r2);
      const double f = q.w * inv * inv * inv;
      ex += rx * f;
      ey += ry * f;
      ez += rz * f;
    }
  }
  if (k >= 0) out[s] = make_double4(ex, ey, ez, 0.0);
}

// Particles of every `stride`-th leaf (deterministic sample of leaves).
__global__ void select_leaf_particles_kernel(const Octree t, const int* __restrict__ leaf_of, int stride,
                                             int* __restrict__ flag) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= t.m) return;
  const unsigned h = static_cast<unsigned>(leaf_of[k]) * 2654435761u;
  flag[k] = (h % static_cast<unsigned>(stride)) == 0 ? 1 : 0;
}

__global__ void compact_kernel(const int* __restrict__ flag, const int* __restrict__ pos, int m, int* __restrict__ sel) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < m && flag[k]) sel[pos[k]] = k;
}

__global__ void residual_targets_kernel(const int* __restrict__ sel, int n_sel, const double4* __restrict__ exact,
                                        const double4* __restrict__ ef, const double* __restrict__ scale,
                                        float* __restrict__ target) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_sel) return;
  const double4 a = exact[s], b = ef[sel[s]];
  const double sc = scale[s];
  target[3 * s + 0] = static_cast<float>((a.x - b.x) / sc);
  target[3 * s + 1] = static_cast<float>((a.y - b.y) / sc);
  target[3 * s + 2] = static_cast<float>((a.z - b.z) / sc);
}

__global__ void audit_error_kernel(const int* __restrict__ sel, int n_sel, const double4* __restrict__ exact,
                                   const double4* __restrict__ ef, double* __restrict__ err) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_sel) return;
  const double4 a = exact[s], b = ef[sel[s]];
  const double num = (a.x - b.x) * (a.x - b.x) + (a.y - b.y) * (a.y - b.y) + (a.z - b.z) * (a.z - b.z);
  const double den = a.x * a.x + a.y * a.y + a.z * a.z;
  err[s] = den > 0.0 ? num / den : 0.0;
}

__global__ void stride_select_kernel(int m, int n_sel, int* __restrict__ sel) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n_sel) sel[s] = static_cast<int>((static_cast<long>(s) * m) / n_sel);
}

// Trains the correction on the context's particles: p=2 FMM, particles of a
// deterministic sample of about `sample_leaves` leaves, exact FP64 fields for
// them, Adam on (features, 100 (E_exact - E_p2) / |E_p2|).
int fmm_train_learned(amk_ctx* c, const View& v, double theta, int sample_leaves, int steps, long batch, float lr,
                      float* loss_out, long* samples_out) {
  FmmRun r;
  AMK_TRY(fmm_run(c, v, 2, theta, 32, false, &r));
  const int m = static_cast<int>(r.t.m);
  if (m == 0) return fail(AMK_ERR_STATE, "no charged particles to train on");
  const long leaves = c->fmm->stats[1];
  const int stride = static_cast<int>(std::max<long>(1, leaves / std::max(1, sample_leaves)));
  int rc = AMK_OK;
  int* flag = slot<int>(c, kSlotFmmWork0, m + 1, &rc);
  AMK_TRY(rc);
  int* pos = slot<int>(c, kSlotFmmWork1, m + 1, &rc);
  AMK_TRY(rc);
  int* total = slot<int>(c, kSlotStatus, 8, &rc) + 7;
  AMK_TRY(rc);
  select_leaf_particles_kernel<<<(m + 255) / 256, 256, 0, c->stream>>>(r.t, r.leaf_of, stride, flag);
  AMK_TRY(check_launch(c, "select_leaf_particles_kernel"));
  AMK_TRY(exclusive_scan_int(c, flag, m, pos, total));
  int n_sel = 0;
  AMK_CUDA_TRY(cudaMemcpyAsync(&n_sel, total, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (n_sel == 0) return fail(AMK_ERR_STATE, "empty training sample");
  int* sel = slot<int>(c, kSlotFmmWork2, n_sel, &rc);
  AMK_TRY(rc);
  compact_kernel<<<(m + 255) / 256, 256, 0, c->stream>>>(flag, pos, m, sel);
  AMK_TRY(check_launch(c, "compact_kernel"));
  float* feat = slot<float>(c, kSlotMlp5, static_cast<size_t>(n_sel) * kFeat, &rc);
  AMK_TRY(rc);
  double* scale = slot<double>(c, kSlotAuxState0, n_sel, &rc);
  AMK_TRY(rc);
  double4* exact = slot<double4>(c, kSlotAuxState1, n_sel, &rc);
  AMK_TRY(rc);
  float* target = slot<float>(c, kSlotMlp4, static_cast<size_t>(n_sel) * 3, &rc);
  AMK_TRY(rc);
  fmm_features_kernel<<<(n_sel + 255) / 256, 256, 0, c->stream>>>(r.t, r.T, r.L, r.M, r.radius, r.p2p_count,
                                                                   r.leaf_of, r.ef, sel, n_sel, feat, scale);
  AMK_TRY(check_launch(c, "fmm_features_kernel"));
  const double min_sq = kMinSquaredDistance / (r.hf.length * r.hf.length);
  exact_field_kernel<<<(n_sel + 255) / 256, 256, 0, c->stream>>>(r.t, sel, n_sel, min_sq, exact);
  AMK_TRY(check_launch(c, "exact_field_kernel"));
  residual_targets_kernel<<<(n_sel + 255) / 256, 256, 0, c->stream>>>(sel, n_sel, exact, r.ef, scale, target);
  AMK_TRY(check_launch(c, "residual_targets_kernel"));
  if (samples_out) *samples_out = n_sel;
  return mlp_train_device(c, feat, target, n_sel, steps, batch, lr, loss_out);
}

// RMS of |E - E_exact| / |E_exact| over `samples` evenly spaced particles for
// plain FMM of `order` or (learned) p=2 plus the correction.
int fmm_audit(amk_ctx* c, const View& v, int order, double theta, bool learned, long samples, double* rms) {
  FmmRun r;
  AMK_TRY(fmm_run(c, v, learned ? 2 : order, theta, 32, false, &r));
  const int m = static_cast<int>(r.t.m);
  *rms = 0.0;
  if (m == 0) return AMK_OK;
  if (learned) AMK_TRY(fmm_apply_learned(c, r));
  const int n_sel = static_cast<int>(std::min<long>(std::max<long>(1, samples), m));
  int rc = AMK_OK;
  int* sel = slot<int>(c, kSlotFmmWork2, n_sel, &rc);
  AMK_TRY(rc);
  double4* exact = slot<double4>(c, kSlotAuxState1, n_sel, &rc);
  AMK_TRY(rc);
  double* err = slot<double>(c, kSlotAuxState2, n_sel, &rc);
  AMK_TRY(rc);
  double* res = slot<double>(c, kSlotAuxState4, 8, &rc);
  AMK_TRY(rc);
  stride_select_kernel<<<(n_sel + 255) / 256, 256, 0, c->stream>>>(m, n_sel, sel);
  AMK_TRY(check_launch(c, "stride_select_kernel"));
  const double min_sq = kMinSquaredDistance / (r.hf.length * r.hf.length);
  exact_field_kernel<<<(n_sel + 255) / 256, 256, 0, c->stream>>>(r.t, sel, n_sel, min_sq, exact);
  AMK_TRY(check_launch(c, "exact_field_kernel"));
  audit_error_kernel<<<(n_sel + 255) / 256, 256, 0, c->stream>>>(sel, n_sel, exact, r.ef, err);
  AMK_TRY(check_launch(c, "audit_error_kernel"));
  AMK_TRY(reduce_sum(c, err, n_sel, res));
  double h = 0.0;
  AMK_CUDA_TRY(cudaMemcpyAsync(&h, res, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
  AMK_TRY(mlp_check_status(c));
  *rms = std::sqrt(h / n_sel);
  return AMK_OK;
}

}  // namespace amk

extern "C" int amk_set_fmm_precision(amk_ctx* c, int mode) {
  if (!c) return amk::fail(AMK_ERR_INVALID, "null context");
  if (mode != AMK_FMM_FP64 && mode != AMK_FMM_TENSOR) return amk::fail(AMK_ERR_INVALID, "unknown FMM precision %d", mode);
  c->fmm_precision = mode;
  return AMK_OK;
}

extern "C" int amk_get_fmm_precision(const amk_ctx* c) { return c ? c->fmm_precision : AMK_ERR_INVALID; }

// Counts of the last FMM evaluation on this context: out[0] cells, [1] leaves,
// [2] M2L pairs, [3] P2P leaf pairs, [4] P2P particle pairs, [5] depth,
// [6] sources, [7] order.
extern "C" int amk_fmm_stats(amk_ctx* c, long* out, int n) {
  if (!c || !out) return amk::fail(AMK_ERR_INVALID, "null argument");
  for (int k = 0; k < n && k < 11; ++k) out[k] = c->fmm ? c->fmm->stats[k] : 0;
  return AMK_OK;
}

void fmm_destroy(amk_ctx* c) {
  delete c->fmm;
  c->fmm = nullptr;
}
