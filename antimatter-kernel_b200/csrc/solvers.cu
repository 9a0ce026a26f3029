// Stateless mirrors of the reference's solver classes on caller host
// buffers (BarnesHutTree, FastMultipoleSolver, the cutoff and all-pairs
// direct sums). The sources are copied into the context's auxiliary
// particle set; the context's own particle state is not touched.
#include <cmath>

#include "amk_internal.cuh"

namespace amk {

int load_aux_view(amk_ctx* c, long n, const double* x, const double* y, const double* z, const double* q,
                    View* out) {
  if (n < 0 || n > 0x7fffffffL) return fail(AMK_ERR_LIMIT, "source count %ld outside [0, 2^31)", n);
  if (n > 0 && (!x || !y || !z || !q)) return fail(AMK_ERR_INVALID, "null source array");
  AMK_CUDA_TRY(cudaSetDevice(c->device));
  if (n > c->aux_capacity) {
    const size_t nd = static_cast<size_t>(n) * sizeof(double);
    for (DevBuf* b : {&c->ax, &c->ay, &c->az, &c->aq, &c->afx, &c->afy, &c->afz, &c->aphi}) AMK_TRY(b->reserve(nd));
    AMK_TRY(c->ahq.reserve(static_cast<size_t>(n) * sizeof(float4)));
    AMK_TRY(c->alo.reserve(static_cast<size_t>(n) * sizeof(float4)));
    c->aux_capacity = n;
  }
  const size_t nd = static_cast<size_t>(n) * sizeof(double);
  double mx = 0.0;
  for (long i = 0; i < n; ++i) {
    const double a = std::fmax(std::fabs(x[i]), std::fmax(std::fabs(y[i]), std::fabs(z[i])));
    if (std::isfinite(a)) mx = std::fmax(mx, a);
  }
  if (n > 0) {
    AMK_CUDA_TRY(cudaMemcpyAsync(c->ax.ptr, x, nd, cudaMemcpyHostToDevice, c->stream));
    AMK_CUDA_TRY(cudaMemcpyAsync(c->ay.ptr, y, nd, cudaMemcpyHostToDevice, c->stream));
    AMK_CUDA_TRY(cudaMemcpyAsync(c->az.ptr, z, nd, cudaMemcpyHostToDevice, c->stream));
    AMK_CUDA_TRY(cudaMemcpyAsync(c->aq.ptr, q, nd, cudaMemcpyHostToDevice, c->stream));
  }
  View v;
  v.n = n;
  v.x = c->ax.as<double>();
  v.y = c->ay.as<double>();
  v.z = c->az.as<double>();
  v.q = c->aq.as<double>();
  v.alive = nullptr;
  v.hq = c->ahq.as<float4>();
  v.lo = c->alo.as<float4>();
  v.fx = c->afx.as<double>();
  v.fy = c->afy.as<double>();
  v.fz = c->afz.as<double>();
  v.phi = nullptr;
  v.length_scale = length_scale_for(mx);
  AMK_TRY(stage_view(c, v));
  *out = v;
  return AMK_OK;
}

static int copy_out(amk_ctx* c, const View& v, double* fx, double* fy, double* fz, double* phi) {
  const size_t nd = static_cast<size_t>(v.n) * sizeof(double);
  if (v.n > 0) {
    if (fx) AMK_CUDA_TRY(cudaMemcpyAsync(fx, v.fx, nd, cudaMemcpyDeviceToHost, c->stream));
    if (fy) AMK_CUDA_TRY(cudaMemcpyAsync(fy, v.fy, nd, cudaMemcpyDeviceToHost, c->stream));
    if (fz) AMK_CUDA_TRY(cudaMemcpyAsync(fz, v.fz, nd, cudaMemcpyDeviceToHost, c->stream));
    if (phi && v.phi) AMK_CUDA_TRY(cudaMemcpyAsync(phi, v.phi, nd, cudaMemcpyDeviceToHost, c->stream));
  }
  AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return AMK_OK;
}

}  // namespace amk

using namespace amk;

extern "C" int amk_solve_allpairs(amk_ctx* c, long n, const double* x, const double* y, const double* z,
                                  const double* q, double* fx, double* fy, double* fz, double* phi) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  View v;
  AMK_TRY(load_aux_view(c, n, x, y, z, q, &v));
  if (n == 0) return AMK_OK;
  if (phi) v.phi = c->aphi.as<double>();
  AMK_TRY(allpairs_forces(c, v));
  return copy_out(c, v, fx, fy, fz, phi);
}

extern "C" int amk_solve_cutoff(amk_ctx* c, long n, const double* x, const double* y, const double* z,
                                const double* q, double cutoff, double* fx, double* fy, double* fz) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  View v;
  AMK_TRY(load_aux_view(c, n, x, y, z, q, &v));
  if (n == 0) return AMK_OK;
  AMK_TRY(cutoff_forces(c, v, cutoff, nullptr));
  return copy_out(c, v, fx, fy, fz, nullptr);
}

extern "C" int amk_solve_barnes_hut(amk_ctx* c, long n, const double* x, const double* y, const double* z,
                                    const double* q, double theta, long leaf_capacity, double* fx, double* fy,
                                    double* fz, double* phi) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  View v;
  AMK_TRY(load_aux_view(c, n, x, y, z, q, &v));
  if (n == 0) return AMK_OK;
  if (phi) v.phi = c->aphi.as<double>();
  AMK_TRY(barnes_hut_forces(c, v, theta, leaf_capacity < 1 ? 1 : leaf_capacity));
  return copy_out(c, v, fx, fy, fz, phi);
}

extern "C" int amk_solve_fmm(amk_ctx* c, long n, const double* x, const double* y, const double* z,
                             const double* q, int order, double theta, long leaf_capacity, double* fx, double* fy,
                             double* fz, double* energy) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  if (energy) *energy = 0.0;
  View v;
  AMK_TRY(load_aux_view(c, n, x, y, z, q, &v));
  if (n == 0) return AMK_OK;
  AMK_TRY(fmm_forces(c, v, order, theta, leaf_capacity < 1 ? 1 : leaf_capacity, false, energy));
  return copy_out(c, v, fx, fy, fz, nullptr);
}
