// C entry points over the reference's own solver sources, compiled in place
// from the reference tree (src/interaction/barnes-hut.cc,
// src/interaction/fast-multipole.cc, src/fields/penning_trap.cc) against the
// headers in oracle/shim. TEST INFRASTRUCTURE ONLY: the oracle is the checker
// for the CUDA library and the timed CPU reference arm of bench.py; nothing
// in the product links it.
//
// Every function returns 0 on success and a negative value on bad input.

#include <cstring>
#include <map>
#include <vector>

#include "fields/penning_trap.h"
#include "interaction/barnes-hut.h"
#include "interaction/fast-multipole.h"
#include "core/resource_manager.h"

using bdm::BarnesHutTree;
using bdm::FastMultipoleSolver;
using bdm::ParticleSpecies;
using bdm::Real3;

namespace {

std::vector<BarnesHutTree::Source> BhSources(long n, const double* x, const double* y,
                                             const double* z, const double* q) {
  std::vector<BarnesHutTree::Source> s(static_cast<size_t>(n));
  for (long i = 0; i < n; ++i) {
    s[i].position = Real3{{x[i], y[i], z[i]}};
    s[i].charge = q[i];
  }
  return s;
}

}  // namespace

extern "C" {

// Reference BarnesHutTree forces for every source (barnes-hut.cc:271-299):
// target i excludes itself (self_index = i). Parallel over targets with
// OpenMP exactly as ComputeBarnesHutCoulombForces does.
int amkref_bh_forces(long n, const double* x, const double* y, const double* z,
                     const double* q, double theta, long leaf_capacity, double* fx,
                     double* fy, double* fz) {
  if (n < 0) return -1;
  if (n == 0) return 0;
  auto sources = BhSources(n, x, y, z, q);
  BarnesHutTree tree(theta, static_cast<size_t>(leaf_capacity));
  tree.Build(sources);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; ++i) {
    const Real3 f = tree.ComputeForce(sources[i].position, sources[i].charge,
                                      static_cast<size_t>(i));
    fx[i] = f[0];
    fy[i] = f[1];
    fz[i] = f[2];
  }
  return 0;
}

// Same tree, forces on a subset of targets only (the bounded CPU sample used
// for timing): targets[k] is a source index.
int amkref_bh_forces_subset(long n, const double* x, const double* y, const double* z,
                            const double* q, double theta, long leaf_capacity,
                            long n_targets, const long* targets, double* fx, double* fy,
                            double* fz, double* build_seconds_out) {
  if (n <= 0 || n_targets < 0) return -1;
  auto sources = BhSources(n, x, y, z, q);
  BarnesHutTree tree(theta, static_cast<size_t>(leaf_capacity));
  tree.Build(sources);
  (void)build_seconds_out;
#pragma omp parallel for schedule(static)
  for (long k = 0; k < n_targets; ++k) {
    const long i = targets[k];
    const Real3 f = tree.ComputeForce(sources[i].position, sources[i].charge,
                                      static_cast<size_t>(i));
    fx[k] = f[0];
    fy[k] = f[1];
    fz[k] = f[2];
  }
  return 0;
}

// Reference potential walk (barnes-hut.cc:223-269): phi_i = sum_j q_j / r_ij
// (no Coulomb constant), self excluded.
int amkref_bh_potentials(long n, const double* x, const double* y, const double* z,
                         const double* q, double theta, long leaf_capacity, double* phi) {
  if (n < 0) return -1;
  if (n == 0) return 0;
  auto sources = BhSources(n, x, y, z, q);
  BarnesHutTree tree(theta, static_cast<size_t>(leaf_capacity));
  tree.Build(sources);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; ++i) {
    phi[i] = tree.ComputePotential(sources[i].position, static_cast<size_t>(i));
  }
  return 0;
}

// Dumps the reference octree (barnes-hut.cc:38-164) in its own node order.
// node_f64: 12 doubles per node = center xyz, half, positive_charge,
// negative_charge, positive_center xyz, negative_center xyz.
// node_i64: 11 per node = children[8], begin, end, is_leaf.
// Returns the node count, or -1 when max_nodes is too small.
long amkref_bh_tree(long n, const double* x, const double* y, const double* z,
                    const double* q, long leaf_capacity, long max_nodes, double* node_f64,
                    long* node_i64, long* order_out) {
  if (n <= 0) return 0;
  auto sources = BhSources(n, x, y, z, q);
  BarnesHutTree tree(0.5, static_cast<size_t>(leaf_capacity));
  tree.Build(sources);
  const long nn = static_cast<long>(tree.nodes_.size());
  if (nn > max_nodes) return -1;
  for (long k = 0; k < nn; ++k) {
    const auto& nd = tree.nodes_[k];
    double* f = node_f64 + 12 * k;
    f[0] = nd.center[0];
    f[1] = nd.center[1];
    f[2] = nd.center[2];
    f[3] = nd.half_size;
    f[4] = nd.positive_charge;
    f[5] = nd.negative_charge;
    f[6] = nd.positive_center[0];
    f[7] = nd.positive_center[1];
    f[8] = nd.positive_center[2];
    f[9] = nd.negative_center[0];
    f[10] = nd.negative_center[1];
    f[11] = nd.negative_center[2];
    long* g = node_i64 + 11 * k;
    for (int o = 0; o < 8; ++o) g[o] = nd.children[o];
    g[8] = static_cast<long>(nd.begin);
    g[9] = static_cast<long>(nd.end);
    g[10] = nd.is_leaf ? 1 : 0;
  }
  if (order_out) {
    for (long i = 0; i < n; ++i) order_out[i] = static_cast<long>(tree.order_[i]);
  }
  return nn;
}

// Reference FMM (fast-multipole.cc:342-682). Either output may be null.
int amkref_fmm(long n, const double* x, const double* y, const double* z, const double* q,
               int order, double theta, long leaf_capacity, double* fx, double* fy,
               double* fz, double* energy) {
  if (n < 0) return -1;
  std::vector<FastMultipoleSolver::Source> s(static_cast<size_t>(n));
  for (long i = 0; i < n; ++i) {
    s[i].position = Real3{{x[i], y[i], z[i]}};
    s[i].charge = q[i];
  }
  FastMultipoleSolver solver(order, theta, static_cast<size_t>(leaf_capacity));
  std::vector<Real3> forces;
  double u = 0.0;
  solver.Compute(s, fx ? &forces : nullptr, energy ? &u : nullptr);
  if (fx) {
    for (long i = 0; i < n; ++i) {
      fx[i] = forces[i][0];
      fy[i] = forces[i][1];
      fz[i] = forces[i][2];
    }
  }
  if (energy) *energy = u;
  return 0;
}

// The reference's drop-in driver ComputeBarnesHutCoulombForces over a flat
// agent list (annihilated agents skipped, as barnes-hut.cc:274-278 does).
int amkref_compute_barnes_hut_coulomb_forces(long n, const double* x, const double* y,
                                             const double* z, const double* q,
                                             const unsigned char* alive, double theta,
                                             double* fx, double* fy, double* fz) {
  std::vector<bdm::ChargedAntiparticle> parts(static_cast<size_t>(n));
  bdm::ResourceManager rm;
  for (long i = 0; i < n; ++i) {
    parts[i].position_ = Real3{{x[i], y[i], z[i]}};
    parts[i].charge_ = q[i];
    parts[i].annihilated_ = alive ? (alive[i] == 0) : false;
    rm.agents.push_back(&parts[i]);
  }
  bdm::ComputeBarnesHutCoulombForces(&rm, theta);
  for (long i = 0; i < n; ++i) {
    fx[i] = parts[i].coulomb_force_[0];
    fy[i] = parts[i].coulomb_force_[1];
    fz[i] = parts[i].coulomb_force_[2];
  }
  return 0;
}

// The reference's drop-in driver ComputeFastMultipoleCoulombForces.
int amkref_compute_fast_multipole_coulomb_forces(long n, const double* x, const double* y,
                                                 const double* z, const double* q,
                                                 const unsigned char* alive, int order,
                                                 double theta, double* fx, double* fy,
                                                 double* fz) {
  std::vector<bdm::ChargedAntiparticle> parts(static_cast<size_t>(n));
  bdm::ResourceManager rm;
  for (long i = 0; i < n; ++i) {
    parts[i].position_ = Real3{{x[i], y[i], z[i]}};
    parts[i].charge_ = q[i];
    parts[i].annihilated_ = alive ? (alive[i] == 0) : false;
    rm.agents.push_back(&parts[i]);
  }
  bdm::ComputeFastMultipoleCoulombForces(&rm, order, theta);
  for (long i = 0; i < n; ++i) {
    fx[i] = parts[i].coulomb_force_[0];
    fy[i] = parts[i].coulomb_force_[1];
    fz[i] = parts[i].coulomb_force_[2];
  }
  return 0;
}

// Reference initial conditions (penning_trap.cc:118-160 and :51-115). The
// species map is iterated in enum order, exactly as std::map does in the
// reference. species[k] are ParticleSpecies enum values; counts[k] >= 0.
int amkref_initial_positions(int n_species, const int* species, const long* counts,
                             const double* radii, int seed, double* out_xyz) {
  std::map<ParticleSpecies, size_t> pops;
  for (int k = 0; k < n_species; ++k)
    pops[static_cast<ParticleSpecies>(species[k])] = static_cast<size_t>(counts[k]);
  const Real3 r{{radii[0], radii[1], radii[2]}};
  auto pos = bdm::PenningTrapField::SetParticlePositions(pops, r, seed);
  for (size_t i = 0; i < pos.size(); ++i) {
    out_xyz[3 * i + 0] = pos[i][0];
    out_xyz[3 * i + 1] = pos[i][1];
    out_xyz[3 * i + 2] = pos[i][2];
  }
  return 0;
}

int amkref_initial_velocities(int n_species, const int* species, const long* counts,
                              const double* temperatures, int seed, double* out_xyz) {
  std::map<ParticleSpecies, size_t> pops;
  std::map<ParticleSpecies, bdm::real_t> temps;
  for (int k = 0; k < n_species; ++k) {
    pops[static_cast<ParticleSpecies>(species[k])] = static_cast<size_t>(counts[k]);
    temps[static_cast<ParticleSpecies>(species[k])] = temperatures[k];
  }
  try {
    auto vel = bdm::PenningTrapField::SetParticleVelocities(pops, temps, seed);
    for (size_t i = 0; i < vel.size(); ++i) {
      out_xyz[3 * i + 0] = vel[i][0];
      out_xyz[3 * i + 1] = vel[i][1];
      out_xyz[3 * i + 2] = vel[i][2];
    }
  } catch (const std::exception&) {
    return -2;
  }
  return 0;
}

// Reference trap field (penning_trap.cc:15-48): e_out = E(x), *phi_out = phi(x).
int amkref_trap_field(double b0, double voltage, double z0, double rho0, const double* pos,
                      double* e_out, double* b_out, double* phi_out) {
  auto field = bdm::PenningTrapField::MakeFromGeometry(b0, voltage, z0, rho0);
  const Real3 p{{pos[0], pos[1], pos[2]}};
  const Real3 e = field.GetElectricField(p);
  const Real3 b = field.GetMagneticField(p);
  for (int d = 0; d < 3; ++d) {
    e_out[d] = e[d];
    b_out[d] = b[d];
  }
  *phi_out = field.GetPotential(p);
  return 0;
}

}  // extern "C"
