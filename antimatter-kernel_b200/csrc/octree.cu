// GPU octree identical to the reference's recursive builds.
//
// The reference splits every cube at its geometric centre with the tests
// x >= cx, y >= cy, z >= cz (barnes-hut.cc:30-33, fast-multipole.cc:234-237),
// children in octant order (bit 0 = x, 1 = y, 2 = z), a node is a leaf when it
// holds <= leaf_capacity particles (barnes-hut.cc:83, fast-multipole.cc:268),
// and nodes are numbered in depth-first pre-order (index taken on entry,
// barnes-hut.cc:69-75, fast-multipole.cc:258-266). Here:
//   1. each source descends 21 levels from the root cube with exactly the
//      reference's FP64 centre updates (c +- h/2) and comparisons, giving a
//      63-bit key whose 3-bit digits are the octants -- so sorted keys list
//      the particles in the reference's tree order;
//   2. with L_k = common leading digits of keys k-1 and k, the node of depth
//      d holding k is [max{s<=k: L_s<d}, min{e>k: L_e<d}); the leaf depth of
//      k is the smallest d whose node holds <= cap particles, found from a
//      +-cap window of L values;
//   3. particle k opens the nodes of depths L_k+1 .. leafdepth(k); an
//      exclusive scan of those counts numbers all nodes in pre-order -- the
//      reference's indices;
//   4. each node replays its key prefix for centre and half edge (same FP64
//      operations as the reference) and links itself into its parent.
// Limitation: keys hold 21 levels (reference: 32). A node deeper than 21
// levels with more than `cap` particles (particles closer than root/2^21) is
// a leaf here; θ = 0 results are unaffected and θ > 0 results differ only by
// the monopole error of such sub-nanometre cells.
#include <algorithm>

#include "amk_internal.cuh"

namespace amk {
namespace {

constexpr uint64_t kNoKey = ~0ull;

__device__ __forceinline__ bool is_source(const View& v, long i, int mode) {
  if (v.alive && !v.alive[i]) return false;
  if (mode == 1 && v.q[i] == 0.0) return false;  // fast-multipole.cc:687-696
  return isfinite(v.x[i]) && isfinite(v.y[i]) && isfinite(v.z[i]);
}

__global__ void tree_bbox_kernel(View v, int mode, unsigned long long* bb) {
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < v.n;
       i += static_cast<long>(gridDim.x) * blockDim.x) {
    if (!is_source(v, i, mode)) continue;
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

// Root cube: barnes-hut.cc:46-61 (Barnes-Hut) / fast-multipole.cc:355-397.
__global__ void tree_root_kernel(const unsigned long long* bb, int mode, TreeFrame* f) {
  const double low[3] = {double_from_order_bits(bb[0]), double_from_order_bits(bb[1]),
                         double_from_order_bits(bb[2])};
  const double high[3] = {-double_from_order_bits(bb[3]), -double_from_order_bits(bb[4]),
                          -double_from_order_bits(bb[5])};
  const double extent = fmax(fmax(high[0] - low[0], high[1] - low[1]), high[2] - low[2]);
  TreeFrame t;
  if (mode == 0) {
    for (int d = 0; d < 3; ++d) {
      t.mid[d] = 0.0;
      t.root_c[d] = 0.5 * (low[d] + high[d]);
    }
    t.length = 1.0;
    double half = 0.5 * extent * (1.0 + 1e-9);
    if (half < 1e-30) half = 1e-30;
    t.root_h = half;
  } else {
    for (int d = 0; d < 3; ++d) {
      t.mid[d] = 0.5 * (low[d] + high[d]);
      t.root_c[d] = 0.0;
    }
    t.length = fmax(extent, 1e-15);
    t.root_h = 0.5 * (1.0 + 1e-9);
  }
  *f = t;
}

__device__ __forceinline__ void tree_coords(const TreeFrame& f, int mode, double x, double y, double z, double* p) {
  if (mode == 0) {
    p[0] = x;
    p[1] = y;
    p[2] = z;
  } else {  // fast-multipole.cc:460-462
    p[0] = (x - f.mid[0]) / f.length;
    p[1] = (y - f.mid[1]) / f.length;
    p[2] = (z - f.mid[2]) / f.length;
  }
}

__global__ void tree_key_kernel(View v, int mode, const TreeFrame* __restrict__ fp, uint64_t* keys, uint32_t* vals) {
  const long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  if (i >= v.n) return;
  vals[i] = static_cast<uint32_t>(i);
  if (!is_source(v, i, mode)) {
    keys[i] = kNoKey;
    return;
  }
  const TreeFrame f = *fp;
  double p[3];
  tree_coords(f, mode, v.x[i], v.y[i], v.z[i], p);
  double c0 = f.root_c[0], c1 = f.root_c[1], c2 = f.root_c[2], h = f.root_h;
  uint64_t key = 0;
  for (int l = 0; l < kTreeLevels; ++l) {
    const int o = (p[0] >= c0 ? 1 : 0) | (p[1] >= c1 ? 2 : 0) | (p[2] >= c2 ? 4 : 0);
    key = (key << 3) | static_cast<uint64_t>(o);
    const double ch = 0.5 * h;
    c0 = c0 + ((o & 1) ? ch : -ch);
    c1 = c1 + ((o & 2) ? ch : -ch);
    c2 = c2 + ((o & 4) ? ch : -ch);
    h = ch;
  }
  keys[i] = key;
}

__global__ void tree_count_sources_kernel(const uint64_t* keys, long n, int* m_out) {
  long lo = 0, hi = n;
  while (lo < hi) {
    const long mid = (lo + hi) >> 1;
    if (keys[mid] < kNoKey)
      lo = mid + 1;
    else
      hi = mid;
  }
  *m_out = static_cast<int>(lo);
}

__device__ __forceinline__ int common_levels(uint64_t a, uint64_t b) {
  const uint64_t x = a ^ b;
  if (x == 0) return kTreeLevels;
  return (__clzll(static_cast<long long>(x)) - 1) / 3;
}

__global__ void tree_L_kernel(const uint64_t* __restrict__ keys, int m, int* __restrict__ L) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  L[k] = (k == 0) ? -1 : common_levels(keys[k - 1], keys[k]);
}

// leafdepth(k) = min over runs [s, e) containing k with e - s <= cap of
// max(L_s, L_e) + 1 (L_0 = L_m = -1), capped at the key depth.
__global__ void tree_leafdepth_kernel(const int* __restrict__ L, int m, int cap, int* __restrict__ ld,
                                      int* __restrict__ count) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  int best = kTreeLevels;
  const int s0 = max(0, k - cap + 1);
  int emin = 1 << 30;
  int ehi = k;  // e range [k+1, ehi] scanned so far
  for (int s = s0; s <= k; ++s) {
    const int lim = min(m, s + cap);
    while (ehi < lim) {
      ++ehi;
      const int le = (ehi == m) ? -1 : L[ehi];
      emin = min(emin, le);
    }
    if (ehi >= k + 1) best = min(best, max(L[s], emin) + 1);
  }
  ld[k] = best;
  const int lk = L[k];
  count[k] = (lk < best) ? best - lk : 0;
}

__device__ __forceinline__ int digit(uint64_t key, int level) {
  return static_cast<int>((key >> (3 * (kTreeLevels - 1 - level))) & 7ull);
}

// first position in [lo, hi) whose key prefix of `depth` digits exceeds `prefix`
__device__ __forceinline__ int prefix_upper(const uint64_t* keys, int lo, int hi, uint64_t prefix, int depth) {
  const int shift = 3 * (kTreeLevels - depth);
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    const uint64_t p = depth == 0 ? 0 : (keys[mid] >> shift);
    if (p <= prefix)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// first position in [lo, hi) whose key prefix of `depth` digits is >= `prefix`
__device__ __forceinline__ int prefix_lower(const uint64_t* keys, int lo, int hi, uint64_t prefix, int depth) {
  const int shift = 3 * (kTreeLevels - depth);
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    const uint64_t p = depth == 0 ? 0 : (keys[mid] >> shift);
    if (p < prefix)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

__global__ void tree_fill_kernel(const uint64_t* __restrict__ keys, int m, const int* __restrict__ L,
                                 const int* __restrict__ ld, const int* __restrict__ base,
                                 const TreeFrame* __restrict__ fp, double4* __restrict__ center,
                                 int* __restrict__ child, int2* __restrict__ range, uchar2* __restrict__ meta,
                                 int* __restrict__ parent) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const int lk = L[k], lf = ld[k];
  if (lk >= lf) return;
  const uint64_t key = keys[k];
  const TreeFrame f = *fp;
  double c0 = f.root_c[0], c1 = f.root_c[1], c2 = f.root_c[2], h = f.root_h;
  int id = base[k];
  for (int d = 0; d <= lf; ++d) {
    if (d > lk) {
      center[id] = make_double4(c0, c1, c2, h);
      const uint64_t prefix = d == 0 ? 0 : (key >> (3 * (kTreeLevels - d)));
      range[id] = make_int2(k, prefix_upper(keys, k + 1, m, prefix, d));
      meta[id] = make_uchar2(static_cast<unsigned char>(d), d == lf ? 1 : 0);
      if (d == 0) {
        parent[id] = -1;
      } else {
        int pid;
        if (lk < d - 1) {
          pid = id - 1;
        } else {
          const uint64_t pp = d - 1 == 0 ? 0 : (key >> (3 * (kTreeLevels - d + 1)));
          const int kp = prefix_lower(keys, 0, k, pp, d - 1);
          pid = base[kp] + (d - 1 - (L[kp] + 1));
        }
        parent[id] = pid;
        child[8 * pid + digit(key, d - 1)] = id;
      }
      ++id;
    }
    if (d < kTreeLevels) {  // descend along this particle's digit
      const int o = digit(key, d);
      const double ch = 0.5 * h;
      c0 = c0 + ((o & 1) ? ch : -ch);
      c1 = c1 + ((o & 2) ? ch : -ch);
      c2 = c2 + ((o & 4) ? ch : -ch);
      h = ch;
    }
  }
}

__global__ void tree_sources_kernel(View v, int mode, const TreeFrame* __restrict__ fp,
                                    const uint32_t* __restrict__ order, int m, double4* __restrict__ src) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const TreeFrame f = *fp;
  const long i = order[k];
  double p[3];
  tree_coords(f, mode, v.x[i], v.y[i], v.z[i], p);
  src[k] = make_double4(p[0], p[1], p[2], v.q[i]);
}

__global__ void tree_max_depth_kernel(const int* __restrict__ ld, int m, int* out) {
  int d = 0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) d = max(d, ld[k]);
  for (int o = 16; o > 0; o >>= 1) d = max(d, __shfl_xor_sync(0xffffffffu, d, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, d);
}

}  // namespace

int build_octree(amk_ctx* c, const View& v, int leaf_cap, int mode, Octree* t) {
  *t = Octree{};
  t->leaf_cap = std::max(1, leaf_cap);
  const long n = v.n;
  if (n == 0) return AMK_OK;
  int rc = AMK_OK;
  unsigned long long* bb = slot<unsigned long long>(c, kSlotCellStart, 8, &rc);
  AMK_TRY(rc);
  TreeFrame* frame = slot<TreeFrame>(c, kSlotTreeFrame, 1, &rc);
  AMK_TRY(rc);
  uint64_t* keys = slot<uint64_t>(c, kSlotKeysA, n, &rc);
  AMK_TRY(rc);
  uint32_t* vals = slot<uint32_t>(c, kSlotValsA, n, &rc);
  AMK_TRY(rc);
  uint64_t* skeys = slot<uint64_t>(c, kSlotTreeSortedKeys, n, &rc);
  AMK_TRY(rc);
  uint32_t* order = slot<uint32_t>(c, kSlotTreeOrder, n, &rc);
  AMK_TRY(rc);
  int* small = slot<int>(c, kSlotStatus, 8, &rc);
  AMK_TRY(rc);

  AMK_CUDA_TRY(cudaMemsetAsync(bb, 0xFF, 6 * sizeof(unsigned long long), c->stream));
  tree_bbox_kernel<<<148, 256, 0, c->stream>>>(v, mode, bb);
  AMK_TRY(check_launch(c, "tree_bbox_kernel"));
  tree_root_kernel<<<1, 1, 0, c->stream>>>(bb, mode, frame);
  AMK_TRY(check_launch(c, "tree_root_kernel"));
  tree_key_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, c->stream>>>(v, mode, frame, keys, vals);
  AMK_TRY(check_launch(c, "tree_key_kernel"));
  AMK_TRY(phase_begin(c, AMK_PHASE_SORT));
  AMK_TRY(radix_sort_pairs(c, keys, vals, skeys, order, n, 64));
  AMK_TRY(phase_end(c, AMK_PHASE_SORT));
  tree_count_sources_kernel<<<1, 1, 0, c->stream>>>(skeys, n, small);
  AMK_TRY(check_launch(c, "tree_count_sources_kernel"));
  int m = 0;
  AMK_CUDA_TRY(cudaMemcpyAsync(&m, small, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
  t->frame = frame;
  t->order = order;
  t->keys = skeys;
  t->m = m;
  if (m == 0) return AMK_OK;

  AMK_TRY(phase_begin(c, AMK_PHASE_TREE));
  int* L = slot<int>(c, kSlotTreeL, m + 1, &rc);
  AMK_TRY(rc);
  int* ld = slot<int>(c, kSlotTreeLeafDepth, m + 1, &rc);
  AMK_TRY(rc);
  int* cnt = slot<int>(c, kSlotTreeCount, m + 1, &rc);
  AMK_TRY(rc);
  int* base = slot<int>(c, kSlotTreeBase, m + 1, &rc);
  AMK_TRY(rc);
  const unsigned gm = static_cast<unsigned>((m + 255) / 256);
  tree_L_kernel<<<gm, 256, 0, c->stream>>>(skeys, m, L);
  AMK_TRY(check_launch(c, "tree_L_kernel"));
  tree_leafdepth_kernel<<<gm, 256, 0, c->stream>>>(L, m, t->leaf_cap, ld, cnt);
  AMK_TRY(check_launch(c, "tree_leafdepth_kernel"));
  AMK_TRY(exclusive_scan_int(c, cnt, m, base, small + 1));
  AMK_CUDA_TRY(cudaMemsetAsync(small + 2, 0, sizeof(int), c->stream));
  tree_max_depth_kernel<<<std::min(gm, 148u), 256, 0, c->stream>>>(ld, m, small + 2);
  AMK_TRY(check_launch(c, "tree_max_depth_kernel"));
  int hs[2] = {0, 0};
  AMK_CUDA_TRY(cudaMemcpyAsync(hs, small + 1, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
  const int nn = hs[0];
  t->n_nodes = nn;
  t->max_depth = hs[1];

  t->center = slot<double4>(c, kSlotTreeCenter, nn, &rc);
  AMK_TRY(rc);
  t->child = slot<int>(c, kSlotTreeChild, 8 * static_cast<size_t>(nn), &rc);
  AMK_TRY(rc);
  t->range = slot<int2>(c, kSlotTreeRange, nn, &rc);
  AMK_TRY(rc);
  t->meta = slot<uchar2>(c, kSlotTreeMeta, nn, &rc);
  AMK_TRY(rc);
  t->parent = slot<int>(c, kSlotTreeParent, nn, &rc);
  AMK_TRY(rc);
  t->src = slot<double4>(c, kSlotTreeSrc, m, &rc);
  AMK_TRY(rc);
  AMK_CUDA_TRY(cudaMemsetAsync(t->child, 0xFF, 8 * static_cast<size_t>(nn) * sizeof(int), c->stream));
  tree_fill_kernel<<<gm, 256, 0, c->stream>>>(skeys, m, L, ld, base, frame, t->center, t->child, t->range,
                                              t->meta, t->parent);
  AMK_TRY(check_launch(c, "tree_fill_kernel"));
  tree_sources_kernel<<<gm, 256, 0, c->stream>>>(v, mode, frame, order, m, t->src);
  AMK_TRY(check_launch(c, "tree_sources_kernel"));
  AMK_TRY(phase_end(c, AMK_PHASE_TREE));
  return AMK_OK;
}

}  // namespace amk
