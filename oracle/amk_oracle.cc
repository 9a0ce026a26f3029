// CPU oracle for the antimatter-kernel per-step particle path.
//
// TEST INFRASTRUCTURE ONLY. This file restates, in plain FP64 C++, the
// reference's per-step arithmetic so that the CUDA library can be checked
// against it. Only tests/, __graft_entry__.smoke() and the CPU-baseline legs
// of bench.py load it. It is never the thing measured or shipped.
//
// Each function cites the reference file:line it restates (paths relative to
// the antimatter-kernel source tree). Where the reference depends on
// BioDynaMo's racy scheduler or its ROOT RNG, the oracle states the
// deterministic rule the CUDA library implements instead (see philox.h).
//
// Parity pins: the initial-condition generators and the step-0 energies are
// checked against the reference's stored notebook values and against the
// reference's own penning_trap.cc compiled in place (oracle/_ref).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <random>
#include <vector>

#include "philox.h"

namespace {

// utils/constants.h:11-38
constexpr double kPi = 3.14159265358979323846;
constexpr double kE = 1.602176634e-19;
constexpr double kMe = 9.1093837015e-31;
constexpr double kMp = 1.67262192369e-27;
constexpr double kMn = 1.67492749804e-27;
constexpr double kK = 8.9875517923e9;
constexpr double kKb = 1.380649e-23;
constexpr double kC = 2.99792458e8;
constexpr double kMinSq = 1e-30;  // coulomb_interaction.cc:19, barnes-hut.cc:17

// agents/particle_species.h:27-46
void SpeciesProps(int s, double* m, double* q) {
  switch (s) {
    case 0: *m = kMp; *q = -kE; return;
    case 1: *m = kMe; *q = kE; return;
    case 2: *m = kMp + kMe; *q = 0.0; return;
    case 3: *m = kMe; *q = -kE; return;
    case 4: *m = kMp; *q = kE; return;
    case 5: *m = 2 * (kMp + kMn); *q = 0.0; return;
    default: *m = 0.0; *q = 0.0; return;
  }
}

// interaction/annihilation.cc:12-19
bool IsAntiparticlePair(int a, int b) {
  auto is_pair = [](int x, int y, int p, int q) { return (x == p && y == q) || (x == q && y == p); };
  return is_pair(a, b, 0, 4) || is_pair(a, b, 1, 3);
}

// Neumaier (improved Kahan) compensated accumulator.
struct Acc {
  double s = 0.0, c = 0.0;
  void add(double v) {
    const double t = s + v;
    if (std::fabs(s) >= std::fabs(v))
      c += (s - t) + v;
    else
      c += (v - t) + s;
    s = t;
  }
  double value() const { return s + c; }
};

}  // namespace

extern "C" {

void orc_species_props(int species, double* mass, double* charge) { SpeciesProps(species, mass, charge); }

int orc_is_antiparticle_pair(int a, int b) { return IsAntiparticlePair(a, b) ? 1 : 0; }

void orc_philox4x32(uint32_t k0, uint32_t k1, const uint32_t* ctr, uint32_t* out) {
  const orc::U32x4 r = orc::Philox4x32(k0, k1, ctr[0], ctr[1], ctr[2], ctr[3]);
  for (int i = 0; i < 4; ++i) out[i] = r.v[i];
}

// params/physics_params.cc:60-74 (dt = pi * min(1e-6, min m/|q|) / (2 b0)).
// Species with zero charge give m/0 = inf and never lower the minimum.
double orc_dt(int n_species, const int* species, double b0) {
  double ratio = 1e-6;
  for (int k = 0; k < n_species; ++k) {
    double m, q;
    SpeciesProps(species[k], &m, &q);
    ratio = std::min(ratio, m / std::fabs(q));
  }
  return (ratio * kPi) / (b0 * 2);
}

// Exact FP64 all-pairs Coulomb force (the theta=0 limit of
// barnes-hut.cc:183-221 / fast-multipole.cc:580-661): F_i = sum_j k q_i q_j
// r_ij / r^3, skipping self, dead particles, q=0 and r^2 < 1e-30
// (barnes-hut.cc:33-41). Sums are Neumaier-compensated. phi (optional) is
// sum_j q_j / r_ij without the Coulomb constant, as barnes-hut.cc:223-269.
void orc_allpairs(long n, const double* x, const double* y, const double* z, const double* q,
                  const unsigned char* alive, double* fx, double* fy, double* fz, double* phi) {
#pragma omp parallel for schedule(dynamic, 16)
  for (long i = 0; i < n; ++i) {
    Acc ax, ay, az, ap;
    const bool live_i = !alive || alive[i];
    if (live_i) {
      for (long j = 0; j < n; ++j) {
        if (j == i || (alive && !alive[j]) || q[j] == 0.0) continue;
        const double rx = x[i] - x[j], ry = y[i] - y[j], rz = z[i] - z[j];
        const double d2 = rx * rx + ry * ry + rz * rz;
        if (d2 < kMinSq) continue;
        const double inv = 1.0 / std::sqrt(d2);
        const double mag = kK * q[i] * q[j] / d2;
        ax.add(rx * (mag * inv));
        ay.add(ry * (mag * inv));
        az.add(rz * (mag * inv));
        ap.add(q[j] * inv);
      }
    }
    if (fx) {
      fx[i] = (live_i && q[i] != 0.0) ? ax.value() : 0.0;
      fy[i] = (live_i && q[i] != 0.0) ? ay.value() : 0.0;
      fz[i] = (live_i && q[i] != 0.0) ? az.value() : 0.0;
    }
    if (phi) phi[i] = live_i ? ap.value() : 0.0;
  }
}

// All-pairs forces on a subset of targets (bounded CPU samples).
void orc_allpairs_subset(long n, const double* x, const double* y, const double* z,
                         const double* q, long n_targets, const long* targets, double* fx,
                         double* fy, double* fz) {
#pragma omp parallel for schedule(dynamic, 16)
  for (long k = 0; k < n_targets; ++k) {
    const long i = targets[k];
    Acc ax, ay, az;
    for (long j = 0; j < n; ++j) {
      if (j == i || q[j] == 0.0) continue;
      const double rx = x[i] - x[j], ry = y[i] - y[j], rz = z[i] - z[j];
      const double d2 = rx * rx + ry * ry + rz * rz;
      if (d2 < kMinSq) continue;
      const double inv = 1.0 / std::sqrt(d2);
      const double mag = kK * q[i] * q[j] / d2;
      ax.add(rx * (mag * inv));
      ay.add(ry * (mag * inv));
      az.add(rz * (mag * inv));
    }
    fx[k] = ax.value();
    fy[k] = ay.value();
    fz[k] = az.value();
  }
}

// Cutoff direct sum, interaction/coulomb_interaction.cc:23-80. Neighbours
// are j != i, alive, q_j != 0 with r^2 < rc^2 (BioDynaMo's neighbour query
// is strict); pairs with r^2 < 1e-30 are skipped (:67); targets with q=0 or
// a non-finite position get no force (:52-56); rc <= 0 gives zero forces
// (:33-37).
void orc_cutoff(long n, const double* x, const double* y, const double* z, const double* q,
                const unsigned char* alive, double rc, double* fx, double* fy, double* fz) {
  const double rc2 = rc * rc;
#pragma omp parallel for schedule(dynamic, 16)
  for (long i = 0; i < n; ++i) {
    Acc ax, ay, az;
    const bool ok = (!alive || alive[i]) && q[i] != 0.0 && rc > 0.0 && std::isfinite(x[i]) &&
                    std::isfinite(y[i]) && std::isfinite(z[i]);
    if (ok) {
      for (long j = 0; j < n; ++j) {
        if (j == i || (alive && !alive[j]) || q[j] == 0.0) continue;
        const double rx = x[i] - x[j], ry = y[i] - y[j], rz = z[i] - z[j];
        const double d2 = rx * rx + ry * ry + rz * rz;
        if (!(d2 < rc2)) continue;
        if (d2 < kMinSq) continue;
        const double dist = std::sqrt(d2);
        const double mag = kK * q[i] * q[j] / d2;
        ax.add(rx * (mag / dist));
        ay.add(ry * (mag / dist));
        az.add(rz * (mag / dist));
      }
    }
    fx[i] = ax.value();
    fy[i] = ay.value();
    fz[i] = az.value();
  }
}

// Boris velocity update, forces/lorentz.cc:18-35.
static void BorisVelocity(const double v[3], const double f[3], const double b[3], double q,
                          double m, double dt, double out[3]) {
  const double half_dt = 0.5 * dt;
  double kick[3], vm[3], t[3], vp[3], s[3], vplus[3];
  for (int d = 0; d < 3; ++d) kick[d] = f[d] * (half_dt / m);
  for (int d = 0; d < 3; ++d) vm[d] = v[d] + kick[d];
  for (int d = 0; d < 3; ++d) t[d] = b[d] * (q * half_dt / m);
  const double cx = vm[1] * t[2] - vm[2] * t[1];
  const double cy = vm[2] * t[0] - vm[0] * t[2];
  const double cz = vm[0] * t[1] - vm[1] * t[0];
  vp[0] = vm[0] + cx;
  vp[1] = vm[1] + cy;
  vp[2] = vm[2] + cz;
  const double t2 = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
  for (int d = 0; d < 3; ++d) s[d] = t[d] * (2.0 / (1.0 + t2));
  const double c2x = vp[1] * s[2] - vp[2] * s[1];
  const double c2y = vp[2] * s[0] - vp[0] * s[2];
  const double c2z = vp[0] * s[1] - vp[1] * s[0];
  vplus[0] = vm[0] + c2x;
  vplus[1] = vm[1] + c2y;
  vplus[2] = vm[2] + c2z;
  for (int d = 0; d < 3; ++d) out[d] = vplus[d] + kick[d];
}

// LorentzForce::Run, forces/lorentz.cc:37-71 with the ideal trap of
// fields/penning_trap.cc:15-48 (d = sqrt(z0^2/2 + rho0^2/4)). On the first
// call (stagger != 0) v is moved back by dt/2 first (:56-60). Coulomb forces
// are consumed and zeroed (:70).
void orc_boris_push(long n, double* x, double* y, double* z, double* vx, double* vy,
                    double* vz, double* fx, double* fy, double* fz, const double* q,
                    const double* m, const unsigned char* alive, double b0, double voltage,
                    double z0, double rho0, double dt, int stagger) {
  const double d = std::sqrt((z0 * z0) / 2.0 + (rho0 * rho0) / 4.0);
  const double d2 = d * d;
  const double radial = voltage / (2.0 * d2);
  const double axial = voltage / d2;
  const double b[3] = {0.0, 0.0, b0};
  for (long i = 0; i < n; ++i) {
    if (alive && !alive[i]) continue;
    if (m[i] <= 0.0 || dt <= 0.0) continue;
    const double e[3] = {radial * x[i], radial * y[i], -axial * z[i]};
    const double f[3] = {e[0] * q[i] + fx[i], e[1] * q[i] + fy[i], e[2] * q[i] + fz[i]};
    double v[3] = {vx[i], vy[i], vz[i]};
    if (stagger) {
      double vb[3];
      BorisVelocity(v, f, b, q[i], m[i], -0.5 * dt, vb);
      v[0] = vb[0];
      v[1] = vb[1];
      v[2] = vb[2];
    }
    double vn[3];
    BorisVelocity(v, f, b, q[i], m[i], dt, vn);
    vx[i] = vn[0];
    vy[i] = vn[1];
    vz[i] = vn[2];
    x[i] = x[i] + vn[0] * dt;
    y[i] = y[i] + vn[1] * dt;
    z[i] = z[i] + vn[2] * dt;
    fx[i] = 0.0;
    fy[i] = 0.0;
    fz[i] = 0.0;
  }
}

// CyclotronCooling::CoolingTime, forces/cooling.cc:16-22.
double orc_cooling_time(double charge, double mass, double b_mag) {
  const double q2 = charge * charge;
  const double denom = q2 * q2 * b_mag * b_mag;
  if (denom <= 0.0) return INFINITY;
  return (0.75 / kK) * mass * mass * mass * kC * kC * kC / denom;
}

// Three N(0,1) draws for particle `id` at step `step` (philox.h stream rule).
void orc_cooling_normals(uint32_t seed, uint32_t id, uint64_t step, double* out3) {
  orc::CoolingNormals(seed, id, step, out3);
}

// CyclotronCooling::Run, forces/cooling.cc:24-66 with B = (0, 0, b0). The
// Gaussian noise uses the Philox rule of philox.h in place of BioDynaMo's
// Random::Gaus; ids[i] is the particle's stable id.
void orc_cooling(long n, double* vx, double* vy, double* vz, const double* q, const double* m,
                 const unsigned char* alive, const uint32_t* ids, double b0, double dt,
                 double tau_scale, double bath_temp, uint32_t seed, uint64_t step) {
  for (long i = 0; i < n; ++i) {
    if (alive && !alive[i]) continue;
    if (q[i] == 0.0 || m[i] <= 0.0 || dt <= 0.0 || tau_scale <= 0.0) continue;
    const double b_mag = std::sqrt(b0 * b0);
    if (b_mag <= 0.0) continue;
    const double tau = tau_scale * orc_cooling_time(std::fabs(q[i]), m[i], b_mag);
    if (!std::isfinite(tau)) continue;
    const double bh[3] = {0.0, 0.0, b0 / b_mag};
    const double v[3] = {vx[i], vy[i], vz[i]};
    const double vpar = v[0] * bh[0] + v[1] * bh[1] + v[2] * bh[2];
    const double vpv[3] = {bh[0] * vpar, bh[1] * vpar, bh[2] * vpar};
    double vperp[3] = {v[0] - vpv[0], v[1] - vpv[1], v[2] - vpv[2]};
    const double decay = std::exp(-dt / (2.0 * tau));
    for (int d = 0; d < 3; ++d) vperp[d] = vperp[d] * decay;
    if (bath_temp > 0.0) {
      const double sigma = std::sqrt(kKb * bath_temp / m[i] * (1.0 - decay * decay));
      double g[3];
      orc_cooling_normals(seed, ids ? ids[i] : static_cast<uint32_t>(i), step, g);
      double noise[3] = {sigma * g[0], sigma * g[1], sigma * g[2]};
      const double nb = noise[0] * bh[0] + noise[1] * bh[1] + noise[2] * bh[2];
      for (int d = 0; d < 3; ++d) noise[d] = noise[d] - bh[d] * nb;
      for (int d = 0; d < 3; ++d) vperp[d] = vperp[d] + noise[d];
    }
    vx[i] = vpv[0] + vperp[0];
    vy[i] = vpv[1] + vperp[1];
    vz[i] = vpv[2] + vperp[2];
  }
}

// Annihilation draw for the ordered pair (owner -> partner) at `step`.
double orc_annihilation_uniform(uint32_t seed, uint32_t owner, uint32_t partner, uint64_t step) {
  const orc::U32x4 w = orc::Philox4x32(seed, orc::kTagAnnihilation, owner, partner,
                                       static_cast<uint32_t>(step),
                                       static_cast<uint32_t>(step >> 32));
  return orc::U01(w.v[0]);
}

// AnnihilationInteraction::Run, interaction/annihilation.cc:21-61, made
// deterministic: the agents are visited one at a time in ascending id order
// and each scans its neighbours in ascending id order (the reference does the
// same visit in parallel, in scheduler order, drawing from a shared RNG). An
// alive agent i pairs with the first alive antiparticle partner j (j != i,
// r^2 < rc^2) whose Philox draw u(i -> j) < p; both are marked annihilated and
// i stops scanning (:37-58). Pairs are looked up on the positions given.
// Returns the number of particles marked this call.
long orc_annihilation(long n, const double* x, const double* y, const double* z,
                      const unsigned char* species, unsigned char* alive, const uint32_t* ids,
                      double contact_radius, double probability, uint32_t seed, uint64_t step) {
  if (contact_radius <= 0.0) return 0;
  const double rc2 = contact_radius * contact_radius;
  // order visited = ascending id
  std::vector<long> order(static_cast<size_t>(n));
  for (long i = 0; i < n; ++i) order[i] = i;
  if (ids) {
    std::sort(order.begin(), order.end(), [&](long a, long b) { return ids[a] < ids[b]; });
  }
  long marked = 0;
  for (long oi = 0; oi < n; ++oi) {
    const long i = order[oi];
    if (!alive[i]) continue;
    for (long oj = 0; oj < n; ++oj) {
      const long j = order[oj];
      if (j == i || !alive[j]) continue;
      if (!IsAntiparticlePair(species[i], species[j])) continue;
      const double rx = x[i] - x[j], ry = y[i] - y[j], rz = z[i] - z[j];
      const double d2 = rx * rx + ry * ry + rz * rz;
      if (!(d2 < rc2)) continue;
      const uint32_t idi = ids ? ids[i] : static_cast<uint32_t>(i);
      const uint32_t idj = ids ? ids[j] : static_cast<uint32_t>(j);
      if (orc_annihilation_uniform(seed, idi, idj, step) < probability) {
        alive[i] = 0;
        alive[j] = 0;
        marked += 2;
        break;
      }
    }
  }
  return marked;
}

// Raw energy terms of analysis/energy_analysis.cc:84-145 for the alive set:
// out[0] = kinetic sum 0.5 m v^2 (:102-111), out[1] = trap potential
// sum q phi(x) (:110, penning_trap.cc:35-43), out[2] = shifted-cutoff Coulomb
// energy sum_{i<j, r^2<=rc^2, r^2>=1e-30} k q_i q_j (1/r - 1/rc) (:16-43),
// out[3] = number of alive particles.
void orc_energy_standard(long n, const double* x, const double* y, const double* z,
                         const double* vx, const double* vy, const double* vz, const double* q,
                         const double* m, const unsigned char* alive, double voltage, double z0,
                         double rho0, double cutoff, double* out) {
  const double d = std::sqrt((z0 * z0) / 2.0 + (rho0 * rho0) / 4.0);
  const double dd = d * d;
  Acc ke, pe;
  long count = 0;
  std::vector<long> live;
  for (long i = 0; i < n; ++i) {
    if (alive && !alive[i]) continue;
    ++count;
    live.push_back(i);
    ke.add(0.5 * m[i] * (vx[i] * vx[i] + vy[i] * vy[i] + vz[i] * vz[i]));
    const double rho2 = x[i] * x[i] + y[i] * y[i];
    pe.add(q[i] * ((voltage / (4.0 * dd)) * (2.0 * z[i] * z[i] - rho2)));
  }
  const double rc2 = cutoff * cutoff;
  const long nl = static_cast<long>(live.size());
  double coul = 0.0;
#pragma omp parallel
  {
    Acc local;
#pragma omp for schedule(dynamic, 16)
    for (long a = 0; a < nl; ++a) {
      const long i = live[a];
      if (q[i] == 0.0) continue;
      for (long b = a + 1; b < nl; ++b) {
        const long j = live[b];
        if (q[j] == 0.0) continue;
        const double rx = x[i] - x[j], ry = y[i] - y[j], rz = z[i] - z[j];
        const double d2 = rx * rx + ry * ry + rz * rz;
        if (d2 > rc2) continue;
        if (d2 < kMinSq) continue;
        local.add(kK * q[i] * q[j] * (1.0 / std::sqrt(d2) - 1.0 / cutoff));
      }
    }
#pragma omp critical
    coul += local.value();
  }
  out[0] = ke.value();
  out[1] = pe.value();
  out[2] = coul;
  out[3] = static_cast<double>(count);
}

// Initial positions, fields/penning_trap.cc:118-160: one
// std::default_random_engine(seed) over all species in enum order, each
// point drawn x, y, z from uniform(-r, r) and kept when inside the ellipsoid.
int orc_initial_positions(int n_species, const int* species, const long* counts,
                          const double* radii, int seed, double* out_xyz) {
  std::map<int, long> pops;
  for (int k = 0; k < n_species; ++k) pops[species[k]] = counts[k];
  std::default_random_engine rng(seed);
  std::uniform_real_distribution<double> ux(-radii[0], radii[0]);
  std::uniform_real_distribution<double> uy(-radii[1], radii[1]);
  std::uniform_real_distribution<double> uz(-radii[2], radii[2]);
  long w = 0;
  for (const auto& kv : pops) {
    for (long i = 0; i < kv.second; ++i) {
      double p[3];
      for (;;) {
        p[0] = ux(rng);
        p[1] = uy(rng);
        p[2] = uz(rng);
        const double a = p[0] / radii[0], b = p[1] / radii[1], c = p[2] / radii[2];
        if ((a * a) + (b * b) + (c * c) <= 1.0) break;
      }
      out_xyz[3 * w + 0] = p[0];
      out_xyz[3 * w + 1] = p[1];
      out_xyz[3 * w + 2] = p[2];
      ++w;
    }
  }
  return 0;
}

// Initial velocities, fields/penning_trap.cc:51-115: per species a fresh
// std::mt19937(seed) with normal(0, sqrt(kT/m)) for 3*count draws, mean
// removed and rescaled by sqrt(n/(n-1)) when count >= 2; T = 0 gives rest.
int orc_initial_velocities(int n_species, const int* species, const long* counts,
                           const double* temperatures, int seed, double* out_xyz) {
  std::map<int, long> pops;
  std::map<int, double> temps;
  for (int k = 0; k < n_species; ++k) {
    pops[species[k]] = counts[k];
    temps[species[k]] = temperatures[k];
  }
  long w = 0;
  for (const auto& kv : pops) {
    const long count = kv.second;
    const double temp = temps[kv.first];
    if (temp == 0.0) {
      for (long i = 0; i < count; ++i, ++w) out_xyz[3 * w] = out_xyz[3 * w + 1] = out_xyz[3 * w + 2] = 0.0;
      continue;
    }
    double mass, charge;
    SpeciesProps(kv.first, &mass, &charge);
    const double sigma = std::sqrt(kKb * temp / mass);
    std::mt19937 rng(seed);
    std::normal_distribution<double> gauss(0.0, sigma);
    std::vector<double> raw(static_cast<size_t>(3 * count));
    for (auto& r : raw) r = gauss(rng);
    if (count >= 2) {
      double mean[3] = {0.0, 0.0, 0.0};
      for (long i = 0; i < count; ++i)
        for (int d = 0; d < 3; ++d) mean[d] += raw[3 * i + d];
      for (int d = 0; d < 3; ++d) mean[d] /= static_cast<double>(count);
      const double rescale = std::sqrt(static_cast<double>(count) / static_cast<double>(count - 1));
      for (long i = 0; i < count; ++i)
        for (int d = 0; d < 3; ++d) raw[3 * i + d] = (raw[3 * i + d] - mean[d]) * rescale;
    }
    for (long i = 0; i < count; ++i, ++w)
      for (int d = 0; d < 3; ++d) out_xyz[3 * w + d] = raw[3 * i + d];
  }
  return 0;
}

}  // extern "C"
