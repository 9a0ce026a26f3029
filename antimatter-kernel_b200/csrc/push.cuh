// Per-particle LorentzForce::Run (Boris push in the ideal Penning-trap field)
// followed by CyclotronCooling::Run (exact exponential damping of v_perp plus
// Langevin noise), shared by the single-instance and batched push kernels so
// that both give bit-identical results. FP64 in the reference's operation
// order.
#pragma once
#include "amk_internal.cuh"
#include "philox.cuh"

namespace amk {

struct PushParams {
  double radial;     // U / (2 d^2)      penning_trap.cc:22-33
  double axial;      // U / d^2
  double b0;         // B = (0, 0, b0)   penning_trap.cc:45-48
  double dt;
  double tau_scale;  // cooling_scale
  double bath_temp;  // bath_temperature
  int cooling;       // CyclotronCooling attached
  uint32_t seed;
};

// Trap and behaviour constants of one parameter set (host).
PushParams push_params_for(const amk_params& p);

// BorisVelocity, lorentz.cc:18-35 (same operation order).
__device__ __forceinline__ void boris(double v[3], const double f[3], const double b[3], double q, double m,
                                      double dt) {
  const double half_dt = 0.5 * dt;
  double kick[3], vm[3], t[3], vp[3], s[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) kick[d] = f[d] * (half_dt / m);
#pragma unroll
  for (int d = 0; d < 3; ++d) vm[d] = v[d] + kick[d];
#pragma unroll
  for (int d = 0; d < 3; ++d) t[d] = b[d] * (q * half_dt / m);
  vp[0] = vm[0] + (vm[1] * t[2] - vm[2] * t[1]);
  vp[1] = vm[1] + (vm[2] * t[0] - vm[0] * t[2]);
  vp[2] = vm[2] + (vm[0] * t[1] - vm[1] * t[0]);
  const double t2 = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
#pragma unroll
  for (int d = 0; d < 3; ++d) s[d] = t[d] * (2.0 / (1.0 + t2));
  const double px = vm[0] + (vp[1] * s[2] - vp[2] * s[1]);
  const double py = vm[1] + (vp[2] * s[0] - vp[0] * s[2]);
  const double pz = vm[2] + (vp[0] * s[1] - vp[1] * s[0]);
  v[0] = px + kick[0];
  v[1] = py + kick[1];
  v[2] = pz + kick[2];
}

// One particle's step; `stagger` applies the first call's -dt/2 velocity
// offset (lorentz.cc:56-60), `step` and `id` select the Philox noise stream.
__device__ __forceinline__ void push_particle(long i, double* __restrict__ x, double* __restrict__ y,
                                              double* __restrict__ z, double* __restrict__ vx,
                                              double* __restrict__ vy, double* __restrict__ vz,
                                              double* __restrict__ fx, double* __restrict__ fy,
                                              double* __restrict__ fz, const double* __restrict__ q,
                                              const double* __restrict__ m, const uint8_t* __restrict__ alive,
                                              const PushParams& P, int stagger, uint64_t step, uint32_t id) {
  const bool live = alive[i] != 0;
  const double qi = q[i], mi = m[i];
  double px = x[i], py = y[i], pz = z[i];
  if (!(live && mi > 0.0 && P.dt > 0.0)) return;
  // ---- LorentzForce::Run, lorentz.cc:37-71
  const double e[3] = {P.radial * px, P.radial * py, -P.axial * pz};
  const double f[3] = {e[0] * qi + fx[i], e[1] * qi + fy[i], e[2] * qi + fz[i]};
  const double b[3] = {0.0, 0.0, P.b0};
  double v[3] = {vx[i], vy[i], vz[i]};
  if (stagger) boris(v, f, b, qi, mi, -0.5 * P.dt);
  boris(v, f, b, qi, mi, P.dt);
  px = px + v[0] * P.dt;
  py = py + v[1] * P.dt;
  pz = pz + v[2] * P.dt;
  fx[i] = 0.0;
  fy[i] = 0.0;
  fz[i] = 0.0;
  // ---- CyclotronCooling::Run, cooling.cc:24-66
  const double bmag = sqrt(P.b0 * P.b0);
  if (P.cooling && qi != 0.0 && P.tau_scale > 0.0 && bmag > 0.0) {
    const double aq = fabs(qi);
    const double q2 = aq * aq;
    const double denom = q2 * q2 * bmag * bmag;
    const double tau_e =
        (0.75 / kCoulombConstant) * mi * mi * mi * kSpeedOfLight * kSpeedOfLight * kSpeedOfLight / denom;
    const double tau = P.tau_scale * tau_e;
    if (isfinite(tau)) {
      const double bh[3] = {0.0, 0.0, P.b0 / bmag};
      const double vpar = v[0] * bh[0] + v[1] * bh[1] + v[2] * bh[2];
      const double vpv[3] = {bh[0] * vpar, bh[1] * vpar, bh[2] * vpar};
      double vperp[3] = {v[0] - vpv[0], v[1] - vpv[1], v[2] - vpv[2]};
      const double decay = exp(-P.dt / (2.0 * tau));
#pragma unroll
      for (int d = 0; d < 3; ++d) vperp[d] = vperp[d] * decay;
      if (P.bath_temp > 0.0) {
        const double sigma = sqrt(kBoltzmann * P.bath_temp / mi * (1.0 - decay * decay));
        const Philox4 w = philox4x32(P.seed, kTagCooling, id, static_cast<uint32_t>(step),
                                     static_cast<uint32_t>(step >> 32), 0u);
        const double u1 = u01(w.w[0]), u2 = u01(w.w[1]), u3 = u01(w.w[2]), u4 = u01(w.w[3]);
        const double r1 = sqrt(-2.0 * log(u1));
        const double r2 = sqrt(-2.0 * log(u3));
        double noise[3] = {sigma * (r1 * cos(2.0 * kPi * u2)), sigma * (r1 * sin(2.0 * kPi * u2)),
                           sigma * (r2 * cos(2.0 * kPi * u4))};
        const double nb = noise[0] * bh[0] + noise[1] * bh[1] + noise[2] * bh[2];
#pragma unroll
        for (int d = 0; d < 3; ++d) noise[d] = noise[d] - bh[d] * nb;
#pragma unroll
        for (int d = 0; d < 3; ++d) vperp[d] = vperp[d] + noise[d];
      }
      v[0] = vpv[0] + vperp[0];
      v[1] = vpv[1] + vperp[1];
      v[2] = vpv[2] + vperp[2];
    }
  }
  x[i] = px;
  y[i] = py;
  z[i] = pz;
  vx[i] = v[0];
  vy[i] = v[1];
  vz[i] = v[2];
}

}  // namespace amk
