// Initial clouds generated on the GPU (the reference's generators,
// penning_trap.cc:51-160, restated for large clouds): species laid out in
// the reference's order (populations by species enum, creation order),
// positions uniform in the ellipsoid with the given radii or Gaussian with
// those radii as standard deviations, velocities Maxwellian per species
// (sigma = sqrt(kT / m) per component) with the reference's mean-drift
// removal and sqrt(n / (n - 1)) rescale (penning_trap.cc:82-105).
//
// The draws come from Philox (key {seed, kTagCloud + generator}, counter
// {index within the cloud, 0, 0, 0}), not from the reference's std::
// engines: amk_init_particles keeps the host path that reproduces those
// bit for bit; this one is for clouds of millions of particles and for
// the many instances of a sweep. Each index's draws depend only on (seed,
// index), so an instance generated inside a batch equals the same instance
// generated on its own context.
//
// Uniform ellipsoid without rejection: a direction from three normals and a
// radius u^(1/3), scaled by the radii. Per-species velocity means are FP64
// block reductions in a fixed order (deterministic).
#include <algorithm>
#include <cstring>
#include <map>
#include <vector>

#include "amk_internal.cuh"
#include "philox.cuh"

namespace amk {
namespace {

constexpr uint32_t kGenPosition = 1, kGenVelocity = 2;

__device__ __forceinline__ void normals4(uint32_t seed, uint32_t gen, uint32_t index, double* z) {
  const Philox4 w = philox4x32(seed, kTagCloud + gen, index, 0u, 0u, 0u);
  const double r1 = sqrt(-2.0 * log(u01(w.w[0]))), r2 = sqrt(-2.0 * log(u01(w.w[2])));
  double s1, c1, s2, c2;
  sincospi(2.0 * u01(w.w[1]), &s1, &c1);
  sincospi(2.0 * u01(w.w[3]), &s2, &c2);
  z[0] = r1 * c1;
  z[1] = r1 * s1;
  z[2] = r2 * c2;
  z[3] = r2 * s2;
}

struct SpeciesRange {
  long begin, end;  // particle range of one species (creation order)
  double sigma;     // sqrt(kT / m)
};

// Positions and raw velocities of particles [base, base + n) of a cloud:
// `first` is the index of particle `base` within its cloud (the counter).
__global__ void cloud_kernel(long n, long base, long first, uint32_t seed, int gaussian, double ra, double rb,
                             double rc, const SpeciesRange* __restrict__ ranges, int n_ranges,
                             double* __restrict__ x, double* __restrict__ y, double* __restrict__ z,
                             double* __restrict__ vx, double* __restrict__ vy, double* __restrict__ vz,
                             uint8_t* __restrict__ species, const uint8_t* __restrict__ codes) {
  const long k = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  if (k >= n) return;
  const uint32_t idx = static_cast<uint32_t>(first + k);
  double g[4];
  normals4(seed, kGenPosition, idx, g);
  double px, py, pz;
  if (gaussian) {
    px = g[0] * ra;
    py = g[1] * rb;
    pz = g[2] * rc;
  } else {
    const double nrm = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
    const Philox4 w = philox4x32(seed, kTagCloud + kGenPosition, idx, 1u, 0u, 0u);
    const double rad = cbrt(u01(w.w[0])) / fmax(nrm, 1e-300);
    px = g[0] * rad * ra;
    py = g[1] * rad * rb;
    pz = g[2] * rad * rc;
  }
  const long i = base + k;
  x[i] = px;
  y[i] = py;
  z[i] = pz;
  int s = 0;
  while (s + 1 < n_ranges && first + k >= ranges[s].end) ++s;
  normals4(seed, kGenVelocity, idx, g);
  const double sig = ranges[s].sigma;
  vx[i] = g[0] * sig;
  vy[i] = g[1] * sig;
  vz[i] = g[2] * sig;
  species[i] = codes[s];
}

// One block per species: mean velocity (fixed-order FP64 tree) removed and
// the spread rescaled by sqrt(n / (n - 1)), as penning_trap.cc:82-105.
__global__ void __launch_bounds__(256)
drift_kernel(long base, const SpeciesRange* __restrict__ ranges, double* vx, double* vy, double* vz) {
  __shared__ double s[3][256];
  const SpeciesRange r = ranges[blockIdx.x];
  const long cnt = r.end - r.begin;
  if (cnt < 2 || r.sigma == 0.0) return;
  double a[3] = {0.0, 0.0, 0.0};
  for (long i = r.begin + threadIdx.x; i < r.end; i += blockDim.x) {
    a[0] += vx[base + i];
    a[1] += vy[base + i];
    a[2] += vz[base + i];
  }
  for (int d = 0; d < 3; ++d) s[d][threadIdx.x] = a[d];
  __syncthreads();
  for (int off = 128; off > 0; off >>= 1) {
    if (threadIdx.x < off)
      for (int d = 0; d < 3; ++d) s[d][threadIdx.x] += s[d][threadIdx.x + off];
    __syncthreads();
  }
  const double inv = 1.0 / static_cast<double>(cnt);
  const double mx = s[0][0] * inv, my = s[1][0] * inv, mz = s[2][0] * inv;
  const double scale = sqrt(static_cast<double>(cnt) / static_cast<double>(cnt - 1));
  for (long i = r.begin + threadIdx.x; i < r.end; i += blockDim.x) {
    vx[base + i] = (vx[base + i] - mx) * scale;
    vy[base + i] = (vy[base + i] - my) * scale;
    vz[base + i] = (vz[base + i] - mz) * scale;
  }
}

// Species ranges of a parameter set in the reference's order (std::map by
// species code, penning_trap.cc:129-157).
int cloud_ranges(const amk_params& p, std::vector<SpeciesRange>* out, std::vector<uint8_t>* codes, long* total) {
  std::map<int, std::pair<long, double>> pops;
  for (int k = 0; k < p.n_species; ++k) {
    if (p.species[k] < 0 || p.species[k] >= AMK_MAX_SPECIES || p.populations[k] < 0)
      return fail(AMK_ERR_INVALID, "bad population entry %d", k);
    pops[p.species[k]] = {p.populations[k], p.temperatures[k]};
  }
  long at = 0;
  out->clear();
  codes->clear();
  for (auto& kv : pops) {
    if (kv.second.first == 0) continue;
    double mass, charge;
    species_properties(kv.first, &mass, &charge);
    const double temp = kv.second.second;
    out->push_back({at, at + kv.second.first, temp > 0.0 && mass > 0.0 ? std::sqrt(kBoltzmann * temp / mass) : 0.0});
    codes->push_back(static_cast<uint8_t>(kv.first));
    at += kv.second.first;
  }
  *total = at;
  return AMK_OK;
}

// Generates one cloud into x..species at offset `base` (device arrays).
int generate_cloud(amk_ctx* c, const amk_params& p, int distribution, long base, double* x, double* y, double* z,
                   double* vx, double* vy, double* vz, uint8_t* species, long* count) {
  std::vector<SpeciesRange> ranges;
  std::vector<uint8_t> codes;
  long total = 0;
  AMK_TRY(cloud_ranges(p, &ranges, &codes, &total));
  *count = total;
  if (total == 0) return AMK_OK;
  // ranges and species codes travel as one small host-to-device copy
  const size_t rb = ranges.size() * sizeof(SpeciesRange);
  std::vector<char> blob(rb + codes.size() + 16);
  std::memcpy(blob.data(), ranges.data(), rb);
  std::memcpy(blob.data() + rb, codes.data(), codes.size());
  DevBuf dev;
  AMK_TRY(dev.reserve(blob.size()));
  AMK_CUDA_TRY(cudaMemcpyAsync(dev.ptr, blob.data(), blob.size(), cudaMemcpyHostToDevice, c->stream));
  const SpeciesRange* dr = dev.as<SpeciesRange>();
  const uint8_t* dc = static_cast<const uint8_t*>(dev.ptr) + rb;
  cloud_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, c->stream>>>(
      total, base, 0, static_cast<uint32_t>(p.seed), distribution == AMK_CLOUD_GAUSSIAN ? 1 : 0, p.cloud_radii[0],
      p.cloud_radii[1], p.cloud_radii[2], dr, static_cast<int>(ranges.size()), x, y, z, vx, vy, vz, species, dc);
  AMK_TRY(check_launch(c, "cloud_kernel"));
  drift_kernel<<<static_cast<unsigned>(ranges.size()), 256, 0, c->stream>>>(base, dr, vx, vy, vz);
  AMK_TRY(check_launch(c, "drift_kernel"));
  AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));  // `dev` is released on return
  return AMK_OK;
}

}  // namespace
}  // namespace amk

using namespace amk;

extern "C" int amk_init_particles_gpu(amk_ctx* c, int distribution) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  if (distribution != AMK_CLOUD_UNIFORM_ELLIPSOID && distribution != AMK_CLOUD_GAUSSIAN)
    return fail(AMK_ERR_INVALID, "unknown cloud distribution %d", distribution);
  AMK_CUDA_TRY(cudaSetDevice(c->device));
  std::vector<SpeciesRange> ranges;
  std::vector<uint8_t> codes;
  long total = 0;
  AMK_TRY(cloud_ranges(c->p, &ranges, &codes, &total));
  if (total <= 0) return fail(AMK_ERR_INVALID, "PenningTrapField: Total particles in PenningTrap should be > 0");
  if (total > 0x7fffffffL) return fail(AMK_ERR_LIMIT, "particle count %ld outside [0, 2^31)", total);
  DevBuf x, y, z, vx, vy, vz, sp;
  const size_t nd = static_cast<size_t>(total) * sizeof(double);
  for (DevBuf* b : {&x, &y, &z, &vx, &vy, &vz}) AMK_TRY(b->reserve(nd));
  AMK_TRY(sp.reserve(static_cast<size_t>(total)));
  long count = 0;
  AMK_TRY(generate_cloud(c, c->p, distribution, 0, x.as<double>(), y.as<double>(), z.as<double>(), vx.as<double>(),
                         vy.as<double>(), vz.as<double>(), sp.as<uint8_t>(), &count));
  AMK_TRY(amk_set_particles_device(c, total, x.as<double>(), y.as<double>(), z.as<double>(), vx.as<double>(),
                                   vy.as<double>(), vz.as<double>(), sp.as<uint8_t>()));
  AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return AMK_OK;
}

extern "C" int amk_batch_init_particles(amk_ctx* c, int n_inst, const amk_params* params, int distribution) {
  if (!c || !params || n_inst <= 0) return fail(AMK_ERR_INVALID, "amk_batch_init_particles: bad argument");
  if (distribution != AMK_CLOUD_UNIFORM_ELLIPSOID && distribution != AMK_CLOUD_GAUSSIAN)
    return fail(AMK_ERR_INVALID, "unknown cloud distribution %d", distribution);
  AMK_CUDA_TRY(cudaSetDevice(c->device));
  std::vector<long> offsets(static_cast<size_t>(n_inst) + 1, 0);
  for (int i = 0; i < n_inst; ++i) {
    std::vector<SpeciesRange> r;
    std::vector<uint8_t> codes;
    long t = 0;
    AMK_TRY(cloud_ranges(params[i], &r, &codes, &t));
    offsets[i + 1] = offsets[i] + t;
  }
  const long total = offsets[n_inst];
  if (total > 0x7fffffffL) return fail(AMK_ERR_LIMIT, "particle count %ld outside [0, 2^31)", total);
  DevBuf x, y, z, vx, vy, vz, sp;
  const size_t nd = static_cast<size_t>(std::max<long>(total, 1)) * sizeof(double);
  for (DevBuf* b : {&x, &y, &z, &vx, &vy, &vz}) AMK_TRY(b->reserve(nd));
  AMK_TRY(sp.reserve(static_cast<size_t>(std::max<long>(total, 1))));
  for (int i = 0; i < n_inst; ++i) {
    long count = 0;
    AMK_TRY(generate_cloud(c, params[i], distribution, offsets[i], x.as<double>(), y.as<double>(), z.as<double>(),
                           vx.as<double>(), vy.as<double>(), vz.as<double>(), sp.as<uint8_t>(), &count));
  }
  AMK_TRY(amk_set_particles_device(c, total, x.as<double>(), y.as<double>(), z.as<double>(), vx.as<double>(),
                                   vy.as<double>(), vz.as<double>(), sp.as<uint8_t>()));
  AMK_TRY(amk_batch_set(c, n_inst, params, offsets.data()));
  AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return AMK_OK;
}
