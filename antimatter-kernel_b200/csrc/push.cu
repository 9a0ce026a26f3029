// Fused per-particle behaviours: LorentzForce::Run followed by
// CyclotronCooling::Run (push.cuh holds the per-particle arithmetic). The
// kernel is HBM-bound: x, v read and written, F read and zeroed, q, m, alive
// and id read: 165 B per particle-step.
#include "push.cuh"

namespace amk {
namespace {

__global__ void __launch_bounds__(256)
push_kernel(long begin, long end, double* __restrict__ x, double* __restrict__ y, double* __restrict__ z,
            double* __restrict__ vx, double* __restrict__ vy, double* __restrict__ vz, double* __restrict__ fx,
            double* __restrict__ fy, double* __restrict__ fz, const double* __restrict__ q,
            const double* __restrict__ m, const uint8_t* __restrict__ alive, const uint32_t* __restrict__ ids,
            PushParams P, int stagger, uint64_t step) {
  const long i = begin + blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  if (i >= end) return;
  push_particle(i, x, y, z, vx, vy, vz, fx, fy, fz, q, m, alive, P, stagger, step, ids[i]);
}

}  // namespace

PushParams push_params_for(const amk_params& p) {
  const double d = sqrt((p.z0 * p.z0) / 2.0 + (p.rho0 * p.rho0) / 4.0);
  const double d2 = d * d;
  PushParams P;
  P.radial = p.trap_voltage / (2.0 * d2);
  P.axial = p.trap_voltage / d2;
  P.b0 = p.b0;
  P.dt = p.dt;
  P.cooling = p.cooling_enabled ? 1 : 0;
  P.tau_scale = p.cooling_scale;
  P.bath_temp = p.bath_temperature;
  P.seed = static_cast<uint32_t>(p.seed);
  return P;
}

int push_range(amk_ctx* c, const PushParams& P, long begin, long end, bool stagger, uint64_t step_index) {
  if (end <= begin) return AMK_OK;
  push_kernel<<<static_cast<unsigned>((end - begin + 255) / 256), 256, 0, c->stream>>>(
      begin, end, c->x.as<double>(), c->y.as<double>(), c->z.as<double>(), c->vx.as<double>(), c->vy.as<double>(),
      c->vz.as<double>(), c->fx.as<double>(), c->fy.as<double>(), c->fz.as<double>(), c->q.as<double>(),
      c->m.as<double>(), c->alive.as<uint8_t>(), c->ids.as<uint32_t>(), P, stagger ? 1 : 0, step_index);
  return check_launch(c, "push_kernel");
}

int push_step(amk_ctx* c, uint64_t step_index) {
  AMK_TRY(phase_begin(c, AMK_PHASE_PUSH));
  AMK_TRY(push_range(c, push_params_for(c->p), 0, c->n, !c->staggered, step_index));
  AMK_TRY(phase_end(c, AMK_PHASE_PUSH));
  c->staggered = true;
  return AMK_OK;
}

}  // namespace amk
