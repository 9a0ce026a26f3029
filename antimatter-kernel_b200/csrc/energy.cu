// FP64 energy diagnostics, analysis/energy_analysis.cc:84-145.
//
// Kinetic and trap-potential sums are deterministic two-pass block
// reductions (fixed tree order). The Coulomb term comes from the solver the
// energy method names, each producing per-particle potentials (or the pair
// energy directly) that are reduced the same way.
#include <cmath>
#include <vector>

#include "amk_internal.cuh"

namespace amk {
namespace {

constexpr int kRedThreads = 256;
constexpr int kRedBlocks = 296;  // 2 x 148 SMs

// out[b*3 + {0,1,2}] = per-block sums of (1/2 m v^2, q phi_trap, alive count).
__global__ void __launch_bounds__(kRedThreads)
ke_trap_kernel(long n, const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z,
               const double* __restrict__ vx, const double* __restrict__ vy, const double* __restrict__ vz,
               const double* __restrict__ q, const double* __restrict__ m, const uint8_t* __restrict__ alive,
               double trap_coef, double* __restrict__ out) {
  __shared__ double s[3][kRedThreads];
  double ke = 0.0, pe = 0.0, cnt = 0.0;
  for (long i = blockIdx.x * static_cast<long>(kRedThreads) + threadIdx.x; i < n;
       i += static_cast<long>(gridDim.x) * kRedThreads) {
    if (!alive[i]) continue;
    ke += 0.5 * m[i] * (vx[i] * vx[i] + vy[i] * vy[i] + vz[i] * vz[i]);
    const double rho2 = x[i] * x[i] + y[i] * y[i];
    pe += q[i] * (trap_coef * (2.0 * z[i] * z[i] - rho2));  // penning_trap.cc:35-43
    cnt += 1.0;
  }
  s[0][threadIdx.x] = ke;
  s[1][threadIdx.x] = pe;
  s[2][threadIdx.x] = cnt;
  __syncthreads();
  for (int w = kRedThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int k = 0; k < 3; ++k) s[k][threadIdx.x] += s[k][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; ++k) out[blockIdx.x * 3 + k] = s[k][0];
}

// q_i * phi_i per block (phi in C/m, i.e. sum q_j / r_ij).
__global__ void __launch_bounds__(kRedThreads)
q_phi_kernel(long n, const double* __restrict__ q, const double* __restrict__ phi,
             const uint8_t* __restrict__ alive, double* __restrict__ out) {
  __shared__ double s[kRedThreads];
  double acc = 0.0;
  for (long i = blockIdx.x * static_cast<long>(kRedThreads) + threadIdx.x; i < n;
       i += static_cast<long>(gridDim.x) * kRedThreads) {
    if (alive && !alive[i]) continue;
    acc += q[i] * phi[i];
  }
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int w = kRedThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = s[0];
}

__global__ void __launch_bounds__(kRedThreads)
sum_kernel(long n, const double* __restrict__ in, double* __restrict__ out) {
  __shared__ double s[kRedThreads];
  double acc = 0.0;
  for (long i = blockIdx.x * static_cast<long>(kRedThreads) + threadIdx.x; i < n;
       i += static_cast<long>(gridDim.x) * kRedThreads)
    acc += in[i];
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int w = kRedThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = s[0];
}

}  // namespace

int reduce_sum(amk_ctx* c, const double* in, long n, double* out_dev) {
  int rc = AMK_OK;
  double* tmp = slot<double>(c, kSlotReduce, kRedBlocks + 8, &rc);
  AMK_TRY(rc);
  sum_kernel<<<kRedBlocks, kRedThreads, 0, c->stream>>>(n, in, tmp);
  AMK_TRY(check_launch(c, "sum_kernel"));
  sum_kernel<<<1, kRedThreads, 0, c->stream>>>(kRedBlocks, tmp, out_dev);
  return check_launch(c, "sum_kernel");
}

// Coulomb potential energy (J) of a view under the energy method and the
// parameters p (cutoff radius, opening angles, FMM order). The view's force
// outputs are redirected to scratch: the force slots are not touched.
int coulomb_energy_view(amk_ctx* c, View v, const amk_params& p, int method, double* out_host) {
  *out_host = 0.0;
  if (v.n == 0) return AMK_OK;
  int rc = AMK_OK;
  // per-particle potential buffer
  double* phi = slot<double>(c, kSlotAuxState6, static_cast<size_t>(v.n) + 8, &rc);
  AMK_TRY(rc);
  double* tf = slot<double>(c, kSlotAuxState5, 3 * static_cast<size_t>(v.n) + 8, &rc);
  AMK_TRY(rc);
  v.fx = tf;
  v.fy = tf + v.n;
  v.fz = tf + 2 * v.n;
  v.phi = phi;
  switch (method) {
    case AMK_METHOD_STANDARD: {
      double e = 0.0;
      AMK_TRY(cutoff_forces(c, v, p.cutoff_radius, &e));
      *out_host = e;
      return AMK_OK;
    }
    case AMK_METHOD_FAST_MULTIPOLE: {
      double e = 0.0;
      AMK_TRY(fmm_forces(c, v, static_cast<int>(p.fast_multipole_order), p.fast_multipole_theta, 32, false, &e));
      *out_host = e;
      return AMK_OK;
    }
    case AMK_METHOD_BARNES_HUT:
      AMK_TRY(barnes_hut_forces(c, v, p.barnes_hut_theta, 8));
      break;
    case AMK_METHOD_ALLPAIRS:
      AMK_TRY(allpairs_forces(c, v));
      break;
    default:
      return fail(AMK_ERR_INVALID, "unknown energy method %d", method);
  }
  double* part = slot<double>(c, kSlotReduce, kRedBlocks + 8, &rc);
  AMK_TRY(rc);
  double* res = slot<double>(c, kSlotAuxState4, 8, &rc);
  AMK_TRY(rc);
  q_phi_kernel<<<kRedBlocks, kRedThreads, 0, c->stream>>>(v.n, v.q, phi, v.alive, part);
  AMK_TRY(check_launch(c, "q_phi_kernel"));
  sum_kernel<<<1, kRedThreads, 0, c->stream>>>(kRedBlocks, part, res);
  AMK_TRY(check_launch(c, "sum_kernel"));
  double h = 0.0;
  AMK_CUDA_TRY(cudaMemcpyAsync(&h, res, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
  *out_host = 0.5 * kCoulombConstant * h;  // energy_analysis.cc:66
  return AMK_OK;
}

}  // namespace amk

using namespace amk;

extern "C" int amk_energy(amk_ctx* c, int time_centre, amk_energy_out* out) {
  if (!c || !out) return fail(AMK_ERR_INVALID, "null argument");
  *out = amk_energy_out{};
  if (c->n == 0) return AMK_OK;
  AMK_CUDA_TRY(cudaSetDevice(c->device));
  AMK_TRY(phase_begin(c, AMK_PHASE_ENERGY));
  int rc = AMK_OK;
  double* part = slot<double>(c, kSlotAuxState3, 3 * static_cast<size_t>(kRedBlocks) + 8, &rc);
  AMK_TRY(rc);
  const double d = sqrt((c->p.z0 * c->p.z0) / 2.0 + (c->p.rho0 * c->p.rho0) / 4.0);
  const double trap_coef = c->p.trap_voltage / (4.0 * (d * d));
  ke_trap_kernel<<<kRedBlocks, kRedThreads, 0, c->stream>>>(
      c->n, c->x.as<double>(), c->y.as<double>(), c->z.as<double>(), c->vx.as<double>(), c->vy.as<double>(),
      c->vz.as<double>(), c->q.as<double>(), c->m.as<double>(), c->alive.as<uint8_t>(), trap_coef, part);
  AMK_TRY(check_launch(c, "ke_trap_kernel"));
  std::vector<double> h(3 * kRedBlocks);
  AMK_CUDA_TRY(cudaMemcpyAsync(h.data(), part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
  double ke = 0.0, pe = 0.0, cnt = 0.0;
  for (int b = 0; b < kRedBlocks; ++b) {
    ke += h[3 * b];
    pe += h[3 * b + 1];
    cnt += h[3 * b + 2];
  }
  double coul = 0.0;
  if (c->p.coulomb_forces_enabled) {
    if (c->stage_dirty) {
      AMK_TRY(stage_view(c, main_view(c)));
      c->stage_dirty = false;
    }
    AMK_TRY(coulomb_energy_view(c, main_view(c), c->p, c->p.energy_method, &coul));
  }
  AMK_TRY(phase_end(c, AMK_PHASE_ENERGY));
  out->kinetic = ke;
  out->trap_potential = pe;
  out->coulomb_potential = coul;
  out->num_active = static_cast<long>(cnt);
  if (time_centre) {  // energy_analysis.cc:126-142
    const double raw_trap = out->trap_potential, raw_coul = out->coulomb_potential;
    if (c->energy_has_previous) {
      out->trap_potential = 0.5 * (c->prev_trap + raw_trap);
      out->coulomb_potential = 0.5 * (c->prev_coulomb + raw_coul);
    }
    c->prev_trap = raw_trap;
    c->prev_coulomb = raw_coul;
    c->energy_has_previous = true;
  }
  out->total = out->kinetic + out->trap_potential + out->coulomb_potential;
  return AMK_OK;
}
