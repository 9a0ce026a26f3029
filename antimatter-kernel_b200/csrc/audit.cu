// Force audit and autotuner.
//
// amk_force_error: RMS and maximum relative error of the context's current
// forces against an FP64 exact Coulomb sum (the reference's exact all-pairs
// force, barnes-hut.h:22-24 at theta = 0: F_i = k q_i sum_j q_j r_ij / r^3,
// pairs closer than 1e-15 m skipped) for evenly spaced sampled targets.
//
// amk_autotune: measures candidate solver configurations on the context's
// own particles -- the all-pairs solver, the FMM over orders, opening angles
// and leaf sizes, Barnes-Hut over opening angles -- times each on the
// device (CUDA events), audits its force error, and configures the context
// with the fastest one whose RMS error is within the budget.
#include <algorithm>
#include <cmath>
#include <functional>
#include <vector>

#include "amk_internal.cuh"

namespace amk {
namespace {

// One thread per sampled target; sources staged in shared-memory tiles.
__global__ void __launch_bounds__(256)
exact_force_kernel(View v, const long* __restrict__ targets, int n_t, double4* __restrict__ out) {
  __shared__ double4 tile[256];
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const long i = s < n_t ? targets[s] : -1;
  double xi = 0.0, yi = 0.0, zi = 0.0;
  if (i >= 0) {
    xi = v.x[i];
    yi = v.y[i];
    zi = v.z[i];
  }
  double ex = 0.0, ey = 0.0, ez = 0.0;
  for (long base = 0; base < v.n; base += 256) {
    __syncthreads();
    const long j = base + threadIdx.x;
    double4 src = make_double4(0.0, 0.0, 0.0, 0.0);
    if (j < v.n && (v.alive == nullptr || v.alive[j]) && isfinite(v.x[j]) && isfinite(v.y[j]) && isfinite(v.z[j]))
      src = make_double4(v.x[j], v.y[j], v.z[j], v.q[j]);
    tile[threadIdx.x] = src;
    __syncthreads();
    if (i < 0) continue;
    const int cnt = static_cast<int>(min(256L, v.n - base));
    for (int u = 0; u < cnt; ++u) {
      const double4 q = tile[u];
      if (base + u == i || q.w == 0.0) continue;
      const double rx = xi - q.x, ry = yi - q.y, rz = zi - q.z;
      const double r2 = rx * rx + ry * ry + rz * rz;
      if (r2 < kMinSquaredDistance) continue;
      const double inv = 1.0 / sqrt(r2);
      const double f = q.w * inv * inv * inv;
      ex += rx * f;
      ey += ry * f;
      ez += rz * f;
    }
  }
  if (i >= 0) {
    const double k = kCoulombConstant * v.q[i];
    out[s] = make_double4(k * ex, k * ey, k * ez, 0.0);
  }
}

}  // namespace

// Evenly spaced usable (alive, charged, finite) targets of the view, at most
// `samples`; the view's force arrays hold the forces under audit.
int force_error(amk_ctx* c, const View& v, long samples, double* rms, double* max_rel) {
  *rms = 0.0;
  if (max_rel) *max_rel = 0.0;
  const long n = v.n;
  if (n == 0 || samples <= 0) return AMK_OK;
  std::vector<double> x(n), y(n), z(n), q(n), fx(n), fy(n), fz(n);
  std::vector<uint8_t> alive(n);
  AMK_CUDA_TRY(cudaMemcpyAsync(x.data(), v.x, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  AMK_CUDA_TRY(cudaMemcpyAsync(y.data(), v.y, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  AMK_CUDA_TRY(cudaMemcpyAsync(z.data(), v.z, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  AMK_CUDA_TRY(cudaMemcpyAsync(q.data(), v.q, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  AMK_CUDA_TRY(cudaMemcpyAsync(alive.data(), v.alive, n, cudaMemcpyDeviceToHost, c->stream));
  AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
  std::vector<long> usable;
  usable.reserve(n);
  for (long i = 0; i < n; ++i)
    if (alive[i] && q[i] != 0.0 && std::isfinite(x[i]) && std::isfinite(y[i]) && std::isfinite(z[i]))
      usable.push_back(i);
  if (usable.empty()) return AMK_OK;
  const long m = std::min<long>(samples, static_cast<long>(usable.size()));
  std::vector<long> targets(m);
  for (long k = 0; k < m; ++k) targets[k] = usable[(k * static_cast<long>(usable.size())) / m];
  int rc = AMK_OK;
  long* dt = slot<long>(c, kSlotAuxState5, m, &rc);
  AMK_TRY(rc);
  double4* dex = slot<double4>(c, kSlotAuxState6, m, &rc);
  AMK_TRY(rc);
  AMK_CUDA_TRY(cudaMemcpyAsync(dt, targets.data(), m * sizeof(long), cudaMemcpyHostToDevice, c->stream));
  exact_force_kernel<<<static_cast<unsigned>((m + 255) / 256), 256, 0, c->stream>>>(v, dt, static_cast<int>(m), dex);
  AMK_TRY(check_launch(c, "exact_force_kernel"));
  std::vector<double4> ex(m);
  AMK_CUDA_TRY(cudaMemcpyAsync(ex.data(), dex, m * sizeof(double4), cudaMemcpyDeviceToHost, c->stream));
  AMK_CUDA_TRY(cudaMemcpyAsync(fx.data(), v.fx, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  AMK_CUDA_TRY(cudaMemcpyAsync(fy.data(), v.fy, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  AMK_CUDA_TRY(cudaMemcpyAsync(fz.data(), v.fz, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
  double sum = 0.0, mx = 0.0;
  long cnt = 0;
  for (long k = 0; k < m; ++k) {
    const long i = targets[k];
    const double den = std::sqrt(ex[k].x * ex[k].x + ex[k].y * ex[k].y + ex[k].z * ex[k].z);
    if (!(den > 0.0)) continue;
    const double dx = fx[i] - ex[k].x, dy = fy[i] - ex[k].y, dz = fz[i] - ex[k].z;
    const double e = std::sqrt(dx * dx + dy * dy + dz * dz) / den;
    sum += e * e;
    mx = std::max(mx, e);
    ++cnt;
  }
  *rms = cnt ? std::sqrt(sum / cnt) : 0.0;
  if (max_rel) *max_rel = mx;
  return AMK_OK;
}

}  // namespace amk

using namespace amk;

extern "C" int amk_force_error(amk_ctx* c, long samples, double* rms, double* max_rel) {
  if (!c || !rms) return fail(AMK_ERR_INVALID, "null argument");
  AMK_CUDA_TRY(cudaSetDevice(c->device));
  return force_error(c, main_view(c), samples, rms, max_rel);
}

namespace amk {

// Device time of one solver call (ms): one warm call, then the median of
// `reps` timed calls.
template <typename F>
int time_call(amk_ctx* c, F&& call, int reps, double* ms) {
  AMK_TRY(call());
  cudaEvent_t a, b;
  AMK_CUDA_TRY(cudaEventCreate(&a));
  AMK_CUDA_TRY(cudaEventCreate(&b));
  std::vector<double> t;
  int rc = AMK_OK;
  for (int r = 0; r < reps && rc == AMK_OK; ++r) {
    cudaEventRecord(a, c->stream);
    rc = call();
    cudaEventRecord(b, c->stream);
    if (cudaEventSynchronize(b) != cudaSuccess) rc = fail(AMK_ERR_CUDA, "event synchronisation failed");
    float f = 0.f;
    if (rc == AMK_OK) cudaEventElapsedTime(&f, a, b);
    t.push_back(f);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  AMK_TRY(rc);
  std::sort(t.begin(), t.end());
  *ms = t[t.size() / 2];
  return AMK_OK;
}

int time_solver(amk_ctx* c, const std::function<int()>& call, int reps, double* ms) {
  return time_call(c, call, reps, ms);
}

}  // namespace amk

extern "C" int amk_autotune(amk_ctx* c, double error_budget, long samples, int flags, amk_tune_candidate* out,
                            int max_out, int* n_out, int* chosen) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  if (!(error_budget > 0.0)) return fail(AMK_ERR_INVALID, "error budget must be positive");
  if (c->batch) return fail(AMK_ERR_STATE, "the context holds a batch");
  AMK_CUDA_TRY(cudaSetDevice(c->device));
  if (n_out) *n_out = 0;
  if (chosen) *chosen = -1;
  if (c->n == 0) return AMK_OK;
  std::vector<amk_tune_candidate> cand;
  if (!(flags & AMK_TUNE_NO_ALLPAIRS)) cand.push_back({AMK_METHOD_ALLPAIRS, 0, 0.0, 0, 0.0, 0.0, 0});
  if (!(flags & AMK_TUNE_NO_FMM))
    for (double theta : {0.6, 0.55, 0.5375, 0.525, 0.5, 0.475, 0.45, 0.4})
      for (int leaf : {16, 32, 64, 128, 256})
        for (int order : {4, 5, 6, 7, 8}) cand.push_back({AMK_METHOD_FAST_MULTIPOLE, order, theta, leaf, 0.0, 0.0, 0});
  if (!(flags & AMK_TUNE_NO_BARNES_HUT))
    for (double theta : {0.5, 0.3, 0.2}) cand.push_back({AMK_METHOD_BARNES_HUT, 0, theta, 8, 0.0, 0.0, 0});
  double best_ms = INFINITY;
  int best = -1;
  for (size_t k = 0; k < cand.size(); ++k) {
    amk_tune_candidate& d = cand[k];
    d.ms = -1.0;
    d.rms = -1.0;
    // skip FMM orders above one that already met the budget at this theta and leaf
    bool skip = false;
    for (size_t j = 0; j < k; ++j)
      if (cand[j].method == d.method && d.method == AMK_METHOD_FAST_MULTIPOLE && cand[j].theta == d.theta &&
          cand[j].leaf == d.leaf && cand[j].order < d.order && cand[j].meets)
        skip = true;
    // ... and Barnes-Hut angles below one that met it
    for (size_t j = 0; j < k; ++j)
      if (d.method == AMK_METHOD_BARNES_HUT && cand[j].method == d.method && cand[j].theta > d.theta && cand[j].meets)
        skip = true;
    if (skip) continue;
    auto call = [&]() -> int {
      switch (d.method) {
        case AMK_METHOD_ALLPAIRS: return allpairs_forces(c, main_view(c));
        case AMK_METHOD_FAST_MULTIPOLE: return fmm_forces(c, main_view(c), d.order, d.theta, d.leaf, false, nullptr);
        default: return barnes_hut_forces(c, main_view(c), d.theta, d.leaf);
      }
    };
    AMK_TRY(time_call(c, call, 3, &d.ms));
    AMK_TRY(force_error(c, main_view(c), samples, &d.rms, nullptr));
    d.meets = d.rms <= error_budget ? 1 : 0;
    if (d.meets && d.ms < best_ms) {
      best_ms = d.ms;
      best = static_cast<int>(k);
    }
  }
  if (out)
    for (int k = 0; k < static_cast<int>(cand.size()) && k < max_out; ++k) out[k] = cand[k];
  if (n_out) *n_out = static_cast<int>(cand.size());
  if (chosen) *chosen = best;
  if (best < 0) return fail(AMK_ERR_LIMIT, "no candidate met the error budget %g", error_budget);
  const amk_tune_candidate& w = cand[best];
  c->p.coulomb_forces_enabled = 1;
  c->p.coulomb_method = w.method;
  if (w.method == AMK_METHOD_FAST_MULTIPOLE) {
    c->p.fast_multipole_order = w.order;
    c->p.fast_multipole_theta = w.theta;
    c->p.fmm_learned = 0;
    c->fmm_leaf = w.leaf;
  } else if (w.method == AMK_METHOD_BARNES_HUT) {
    c->p.barnes_hut_theta = w.theta;
    c->bh_leaf = w.leaf;
  }
  return AMK_OK;
}
