// Context life cycle, particle transfer, parameter helpers, error reporting,
// phase timing and the per-step driver of the C ABI (include/amk.h).
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <map>
#include <random>
#include <vector>

#include "amk_internal.cuh"

namespace amk {

namespace {
thread_local char g_error[1024] = "no error";

struct EventPool {
  std::vector<cudaEvent_t> start, stop;
  size_t used = 0;
  int open = 0;  // nesting depth: an inner begin/end of the same phase is not timed twice
};
std::map<const amk_ctx*, std::vector<EventPool>> g_events;
}  // namespace

void set_error(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  int off = std::snprintf(g_error, sizeof(g_error), "[amk %d] ", code);
  if (off < 0) off = 0;
  std::vsnprintf(g_error + off, sizeof(g_error) - static_cast<size_t>(off), fmt, ap);
  va_end(ap);
}

int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  int off = std::snprintf(g_error, sizeof(g_error), "[amk %d] ", code);
  if (off < 0) off = 0;
  std::vsnprintf(g_error + off, sizeof(g_error) - static_cast<size_t>(off), fmt, ap);
  va_end(ap);
  return code;
}

void species_properties(int s, double* m, double* q) {
  switch (s) {
    case AMK_ANTIPROTON: *m = kProtonMass; *q = -kElementaryCharge; return;
    case AMK_POSITRON: *m = kElectronMass; *q = kElementaryCharge; return;
    case AMK_ANTIHYDROGEN: *m = kProtonMass + kElectronMass; *q = 0.0; return;
    case AMK_ELECTRON: *m = kElectronMass; *q = -kElementaryCharge; return;
    case AMK_PROTON: *m = kProtonMass; *q = kElementaryCharge; return;
    case AMK_ANTIHELIUM: *m = 2 * (kProtonMass + kNeutronMass); *q = 0.0; return;
    default: *m = 0.0; *q = 0.0; return;
  }
}

bool is_antiparticle_pair(int a, int b) {
  auto is_pair = [](int x, int y, int p, int q) { return (x == p && y == q) || (x == q && y == p); };
  return is_pair(a, b, AMK_ANTIPROTON, AMK_PROTON) || is_pair(a, b, AMK_POSITRON, AMK_ELECTRON);
}

double length_scale_for(double max_abs) {
  if (!(max_abs > 0.0) || !std::isfinite(max_abs)) return 1.0;
  int e = 0;
  std::frexp(max_abs, &e);  // max_abs = f * 2^e, f in [0.5, 1)
  return std::ldexp(1.0, e);
}

View main_view(amk_ctx* c) {
  View v;
  v.n = c->n;
  v.x = c->x.as<double>();
  v.y = c->y.as<double>();
  v.z = c->z.as<double>();
  v.q = c->q.as<double>();
  v.alive = c->alive.as<uint8_t>();
  v.hq = c->hq.as<float4>();
  v.lo = c->lo.as<float4>();
  v.fx = c->fx.as<double>();
  v.fy = c->fy.as<double>();
  v.fz = c->fz.as<double>();
  v.length_scale = c->length_scale;
  return v;
}

// x / L split into a float pair: hi = fl(x/L), lo = fl(x/L - hi). Dead,
// neutral and non-finite particles get q_e = 0 and a zero position so that
// they drop out of every pair sum (coulomb_interaction.cc:52-56,64-66).
__global__ void stage_kernel(long n, const double* __restrict__ x, const double* __restrict__ y,
                             const double* __restrict__ z, const double* __restrict__ q,
                             const uint8_t* __restrict__ alive, double inv_l, float4* __restrict__ hq,
                             float4* __restrict__ lo) {
  const long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const double xs = x[i] * inv_l, ys = y[i] * inv_l, zs = z[i] * inv_l;
  const bool ok = (alive == nullptr || alive[i]) && q[i] != 0.0 && isfinite(xs) && isfinite(ys) &&
                  isfinite(zs);
  float4 h, l;
  if (ok) {
    h.x = __double2float_rn(xs);
    h.y = __double2float_rn(ys);
    h.z = __double2float_rn(zs);
    h.w = __double2float_rn(q[i] / kElementaryCharge);
    l.x = __double2float_rn(xs - static_cast<double>(h.x));
    l.y = __double2float_rn(ys - static_cast<double>(h.y));
    l.z = __double2float_rn(zs - static_cast<double>(h.z));
    l.w = 0.0f;
  } else {
    h = make_float4(0.f, 0.f, 0.f, 0.f);
    l = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  hq[i] = h;
  lo[i] = l;
}

int stage_view(amk_ctx* c, const View& v) {
  if (v.n == 0) return AMK_OK;
  const int threads = 256;
  const long blocks = (v.n + threads - 1) / threads;
  stage_kernel<<<static_cast<unsigned>(blocks), threads, 0, c->stream>>>(
      v.n, v.x, v.y, v.z, v.q, v.alive, 1.0 / v.length_scale, v.hq, v.lo);
  return check_launch(c, "stage_kernel");
}

int phase_begin(amk_ctx* c, int phase) { return phase_begin_on(c, phase, c->stream); }

int phase_end(amk_ctx* c, int phase) { return phase_end_on(c, phase, c->stream); }

int phase_begin_on(amk_ctx* c, int phase, cudaStream_t stream) {
  if (!c->profiling) return AMK_OK;
  auto& pools = g_events[c];
  if (pools.size() < AMK_NUM_PHASES) pools.resize(AMK_NUM_PHASES);
  EventPool& p = pools[phase];
  if (p.open++ > 0) return AMK_OK;
  if (p.used == p.start.size()) {
    cudaEvent_t a, b;
    AMK_CUDA_TRY(cudaEventCreate(&a));
    AMK_CUDA_TRY(cudaEventCreate(&b));
    p.start.push_back(a);
    p.stop.push_back(b);
  }
  AMK_CUDA_TRY(cudaEventRecord(p.start[p.used], stream));
  return AMK_OK;
}

int phase_end_on(amk_ctx* c, int phase, cudaStream_t stream) {
  if (!c->profiling) return AMK_OK;
  auto& pools = g_events[c];
  if (pools.size() < AMK_NUM_PHASES) return AMK_OK;
  EventPool& p = pools[phase];
  if (p.open == 0) return AMK_OK;
  if (--p.open > 0) return AMK_OK;
  AMK_CUDA_TRY(cudaEventRecord(p.stop[p.used], stream));
  p.used++;
  return AMK_OK;
}

static int harvest_events(amk_ctx* c) {
  auto it = g_events.find(c);
  if (it == g_events.end()) return AMK_OK;
  for (int ph = 0; ph < static_cast<int>(it->second.size()); ++ph) {
    EventPool& p = it->second[ph];
    for (size_t k = 0; k < p.used; ++k) {
      AMK_CUDA_TRY(cudaEventSynchronize(p.stop[k]));
      float ms = 0.f;
      AMK_CUDA_TRY(cudaEventElapsedTime(&ms, p.start[k], p.stop[k]));
      c->clock.ms[ph] += ms;
      c->clock.launches[ph] += 1;
    }
    p.used = 0;
  }
  return AMK_OK;
}

static void destroy_events(const amk_ctx* c) {
  auto it = g_events.find(c);
  if (it == g_events.end()) return;
  for (auto& p : it->second) {
    for (auto e : p.start) cudaEventDestroy(e);
    for (auto e : p.stop) cudaEventDestroy(e);
  }
  g_events.erase(it);
}

}  // namespace amk

using namespace amk;

// ============================================================== parameters
extern "C" int amk_params_default(amk_params* p) {
  if (!p) return fail(AMK_ERR_INVALID, "amk_params_default: null");
  std::memset(p, 0, sizeof(*p));
  p->seed = 42;
  p->b0 = 1.0;
  p->trap_voltage = 10.0;
  p->z0 = 0.01;
  p->rho0 = 0.01;
  p->dt = 1e-9;
  p->num_steps = 5000;
  p->bath_temperature = 0.5;
  p->cooling_scale = 10;
  p->cooling_enabled = 1;
  p->coulomb_forces_enabled = 1;
  p->coulomb_method = AMK_METHOD_STANDARD;
  p->energy_method = AMK_METHOD_STANDARD;
  p->cutoff_radius = 0.0;
  p->barnes_hut_theta = 0.5;
  p->fast_multipole_order = 4;
  p->fast_multipole_theta = 0.5;
  p->annihilation_enabled = 0;
  p->contact_radius = 1e-9;
  p->annihilation_probability = 0.1;
  p->n_species = 1;
  p->species[0] = AMK_POSITRON;
  p->populations[0] = 10;
  p->temperatures[0] = 4;
  p->cloud_radii[0] = p->cloud_radii[1] = p->cloud_radii[2] = 1e-4;
  p->learned_audit_interval = 100;
  p->learned_error_budget = 1e-5;
  p->learned_fallback_order = 6;
  p->learned_audit_samples = 1024;
  return AMK_OK;
}

extern "C" double amk_dt_for_species(int n_species, const int* species, double b0) {
  double ratio = 1e-6;
  for (int k = 0; k < n_species; ++k) {
    double m, q;
    species_properties(species[k], &m, &q);
    ratio = std::min(ratio, m / std::fabs(q));
  }
  return (ratio * kPi) / (b0 * 2);
}

extern "C" int amk_species_properties(int s, double* mass, double* charge) {
  if (s < 0 || s >= AMK_MAX_SPECIES || !mass || !charge)
    return fail(AMK_ERR_INVALID, "unknown species %d", s);
  species_properties(s, mass, charge);
  return AMK_OK;
}

extern "C" double amk_trap_dimension(double z0, double rho0) {
  return std::sqrt((z0 * z0) / 2.0 + (rho0 * rho0) / 4.0);
}

extern "C" double amk_cooling_time(double charge, double mass, double b_mag) {
  const double q2 = charge * charge;
  const double denom = q2 * q2 * b_mag * b_mag;
  if (denom <= 0.0) return INFINITY;
  return (0.75 / kCoulombConstant) * mass * mass * mass * kSpeedOfLight * kSpeedOfLight *
         kSpeedOfLight / denom;
}

extern "C" int amk_params_validate(const amk_params* p, int strict) {
  if (!p) return fail(AMK_ERR_INVALID, "null params");
  // physics_params.cc:126-160
  if (p->b0 <= 0.0) return fail(AMK_ERR_INVALID, "PhysicsParams: b0 must be > 0");
  if (p->z0 <= 0.0 || p->rho0 <= 0.0) return fail(AMK_ERR_INVALID, "PhysicsParams: z0 and rho0 must be > 0");
  if (p->num_steps <= 0) return fail(AMK_ERR_INVALID, "PhysicsParams: num_steps must be > 0");
  for (int k = 0; k < p->n_species; ++k)
    if (p->temperatures[k] < 0)
      return fail(AMK_ERR_INVALID, "PhysicsParams: initial temperature of particles count must be >= 0");
  if (p->bath_temperature < 0.0) return fail(AMK_ERR_INVALID, "PhysicsParams: bath_temperature must be > 0");
  if (strict && p->cooling_scale > 1.0) return fail(AMK_ERR_INVALID, "PhysicsParams: cooling_scale must be <= 1");
  if (p->n_species <= 0) return fail(AMK_ERR_INVALID, "PhysicsParams: populations must not be empty");
  for (int k = 0; k < p->n_species; ++k) {
    if (p->populations[k] < 0) return fail(AMK_ERR_INVALID, "PhysicsParams: every population count must be >= 0");
    if (p->species[k] < 0 || p->species[k] >= AMK_MAX_SPECIES)
      return fail(AMK_ERR_INVALID, "PhysicsParams: unrecognized species %d", p->species[k]);
  }
  if (p->cloud_radii[0] <= 0.0 || p->cloud_radii[1] <= 0.0 || p->cloud_radii[2] <= 0.0)
    return fail(AMK_ERR_INVALID, "PhysicsParams: All components of initial_cloud_radii must be > 0.");
  if (p->cloud_radii[0] >= p->rho0 || p->cloud_radii[1] >= p->rho0)
    return fail(AMK_ERR_INVALID, "PhysicsParams: Radial radii (X and Y) must be well inside trap radius (rho0).");
  if (p->cloud_radii[2] >= p->z0)
    return fail(AMK_ERR_INVALID, "PhysicsParams: Axial radius (Z) must be well inside trap length (z0).");
  // interaction_params.cc:71-115 (energy method checked on its own value;
  // the reference re-reads the Coulomb method there, a bug not reproduced).
  auto check_method = [&](int method, const char* which) -> int {
    if (method < 0 || method > AMK_METHOD_ALLPAIRS)
      return fail(AMK_ERR_INVALID, "InteractionParams: unrecognized %s", which);
    if (method == AMK_METHOD_STANDARD && p->cutoff_radius <= 0.0)
      return fail(AMK_ERR_INVALID, "InteractionParams: cutoff_radius must be > 0 when %s is 'standard'", which);
    if (method == AMK_METHOD_BARNES_HUT && (p->barnes_hut_theta < 0.0 || p->barnes_hut_theta > 1.0))
      return fail(AMK_ERR_INVALID, "InteractionParams: barnes_hut_theta must be in [0, 1]");
    if (method == AMK_METHOD_FAST_MULTIPOLE) {
      if (p->fast_multipole_order < 1 || p->fast_multipole_order > 8)
        return fail(AMK_ERR_INVALID, "InteractionParams: fast_multipole_order must be an integer in [1, 8].");
      if (p->fast_multipole_theta < 0.0 || p->fast_multipole_theta >= 1.0)
        return fail(AMK_ERR_INVALID, "InteractionParams: fast_multipole_theta must be in [0, 1)");
    }
    return AMK_OK;
  };
  AMK_TRY(check_method(p->energy_method, "energy_method"));
  if (p->coulomb_forces_enabled) AMK_TRY(check_method(p->coulomb_method, "coulomb_method"));
  // stochastic_params.cc:35-46
  if (p->annihilation_enabled) {
    if (p->contact_radius <= 0.0)
      return fail(AMK_ERR_INVALID, "StochasticParams: contact_radius must be > 0 when annihilation_enabled is true.");
    if (p->annihilation_probability < 0.0 || p->annihilation_probability > 1.0)
      return fail(AMK_ERR_INVALID, "StochasticParams: annihilation_probability must be in [0, 1].");
  }
  return AMK_OK;
}

// ============================================================== context
extern "C" const char* amk_last_error(void) { return g_error; }

extern "C" int amk_create(const amk_params* params, int device, amk_ctx** out) {
  if (!out) return fail(AMK_ERR_INVALID, "amk_create: null output");
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return fail(AMK_ERR_CUDA, "no CUDA device visible");
  }
  if (device < 0 || device >= count) return fail(AMK_ERR_INVALID, "device %d out of range", device);
  AMK_CUDA_TRY(cudaSetDevice(device));
  amk_ctx* c = new amk_ctx();
  if (params)
    c->p = *params;
  else
    amk_params_default(&c->p);
  c->device = device;
  if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return fail(AMK_ERR_CUDA, "stream creation failed");
  }
  c->stream = c->own_stream;
  *out = c;
  return AMK_OK;
}

void fmm_destroy(amk_ctx* c);
void mlp_destroy(amk_ctx* c);

extern "C" int amk_destroy(amk_ctx* c) {
  if (!c) return AMK_OK;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  fmm_destroy(c);
  mlp_destroy(c);
  batch_destroy(c);
  destroy_events(c);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
  return AMK_OK;
}

extern "C" int amk_set_stream(amk_ctx* c, void* s) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  c->stream = s ? static_cast<cudaStream_t>(s) : c->own_stream;
  return AMK_OK;
}

extern "C" int amk_get_stream(amk_ctx* c, void** s) {
  if (!c || !s) return fail(AMK_ERR_INVALID, "null argument");
  *s = c->stream;
  return AMK_OK;
}

extern "C" int amk_synchronize(amk_ctx* c) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return AMK_OK;
}

extern "C" int amk_set_params(amk_ctx* c, const amk_params* p) {
  if (!c || !p) return fail(AMK_ERR_INVALID, "null argument");
  c->p = *p;
  return AMK_OK;
}

extern "C" int amk_get_params(const amk_ctx* c, amk_params* p) {
  if (!c || !p) return fail(AMK_ERR_INVALID, "null argument");
  *p = c->p;
  return AMK_OK;
}

static int ensure_capacity(amk_ctx* c, long n) {
  if (n <= c->capacity) return AMK_OK;
  const size_t nd = static_cast<size_t>(n) * sizeof(double);
  for (amk::DevBuf* b : {&c->x, &c->y, &c->z, &c->vx, &c->vy, &c->vz, &c->fx, &c->fy, &c->fz, &c->q, &c->m})
    AMK_TRY(b->reserve(nd));
  AMK_TRY(c->hq.reserve(static_cast<size_t>(n) * sizeof(float4)));
  AMK_TRY(c->lo.reserve(static_cast<size_t>(n) * sizeof(float4)));
  AMK_TRY(c->species.reserve(static_cast<size_t>(n)));
  AMK_TRY(c->alive.reserve(static_cast<size_t>(n)));
  AMK_TRY(c->ids.reserve(static_cast<size_t>(n) * sizeof(uint32_t)));
  c->capacity = n;
  return AMK_OK;
}

__global__ void init_particle_props_kernel(long n, const uint8_t* __restrict__ species,
                                           double* __restrict__ q, double* __restrict__ m,
                                           uint8_t* __restrict__ alive, uint32_t* __restrict__ ids,
                                           double* fx, double* fy, double* fz) {
  const long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  double mm = 0.0, qq = 0.0;
  switch (species[i]) {
    case AMK_ANTIPROTON: mm = kProtonMass; qq = -kElementaryCharge; break;
    case AMK_POSITRON: mm = kElectronMass; qq = kElementaryCharge; break;
    case AMK_ANTIHYDROGEN: mm = kProtonMass + kElectronMass; qq = 0.0; break;
    case AMK_ELECTRON: mm = kElectronMass; qq = -kElementaryCharge; break;
    case AMK_PROTON: mm = kProtonMass; qq = kElementaryCharge; break;
    case AMK_ANTIHELIUM: mm = 2 * (kProtonMass + kNeutronMass); qq = 0.0; break;
    default: break;
  }
  q[i] = qq;
  m[i] = mm;
  alive[i] = 1;
  ids[i] = static_cast<uint32_t>(i);
  fx[i] = 0.0;
  fy[i] = 0.0;
  fz[i] = 0.0;
}

__global__ void max_abs_kernel(long n, const double* __restrict__ x, const double* __restrict__ y,
                               const double* __restrict__ z, unsigned long long* out) {
  double m = 0.0;
  for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<long>(gridDim.x) * blockDim.x) {
    const double a = fmax(fabs(x[i]), fmax(fabs(y[i]), fabs(z[i])));
    if (isfinite(a)) m = fmax(m, a);
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  // non-negative doubles order like their bit patterns
  if ((threadIdx.x & 31) == 0) atomicMax(out, static_cast<unsigned long long>(__double_as_longlong(m)));
}

static int finish_load(amk_ctx* c, long n) {
  batch_destroy(c);  // instance offsets refer to the previous particle set
  c->n = n;
  c->ap_perm_n = -1;
  c->staggered = false;
  c->step = 0;
  c->energy_has_previous = false;
  if (n == 0) return AMK_OK;
  const int threads = 256;
  const unsigned blocks = static_cast<unsigned>((n + threads - 1) / threads);
  init_particle_props_kernel<<<blocks, threads, 0, c->stream>>>(
      n, c->species.as<uint8_t>(), c->q.as<double>(), c->m.as<double>(), c->alive.as<uint8_t>(),
      c->ids.as<uint32_t>(), c->fx.as<double>(), c->fy.as<double>(), c->fz.as<double>());
  AMK_TRY(check_launch(c, "init_particle_props_kernel"));
  // Power-of-two length scale from the largest |coordinate| (one readback at load time).
  int rc = AMK_OK;
  unsigned long long* mx = slot<unsigned long long>(c, kSlotStatus, 4, &rc);
  AMK_TRY(rc);
  AMK_CUDA_TRY(cudaMemsetAsync(mx, 0, sizeof(unsigned long long), c->stream));
  max_abs_kernel<<<148, 256, 0, c->stream>>>(n, c->x.as<double>(), c->y.as<double>(), c->z.as<double>(), mx);
  AMK_TRY(check_launch(c, "max_abs_kernel"));
  unsigned long long bits = 0;
  AMK_CUDA_TRY(cudaMemcpyAsync(&bits, mx, sizeof(bits), cudaMemcpyDeviceToHost, c->stream));
  AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
  double mabs;
  std::memcpy(&mabs, &bits, sizeof(mabs));
  c->length_scale = length_scale_for(mabs);
  c->stage_dirty = true;
  return AMK_OK;
}

extern "C" int amk_set_particles(amk_ctx* c, long n, const double* x, const double* y, const double* z,
                                 const double* vx, const double* vy, const double* vz,
                                 const uint8_t* species) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  if (n < 0 || n > 0x7fffffffL) return fail(AMK_ERR_LIMIT, "particle count %ld outside [0, 2^31)", n);
  if (n > 0 && (!x || !y || !z || !vx || !vy || !vz || !species))
    return fail(AMK_ERR_INVALID, "amk_set_particles: null array");
  AMK_CUDA_TRY(cudaSetDevice(c->device));
  AMK_TRY(ensure_capacity(c, n));
  const size_t nd = static_cast<size_t>(n) * sizeof(double);
  if (n > 0) {
    AMK_CUDA_TRY(cudaMemcpyAsync(c->x.ptr, x, nd, cudaMemcpyHostToDevice, c->stream));
    AMK_CUDA_TRY(cudaMemcpyAsync(c->y.ptr, y, nd, cudaMemcpyHostToDevice, c->stream));
    AMK_CUDA_TRY(cudaMemcpyAsync(c->z.ptr, z, nd, cudaMemcpyHostToDevice, c->stream));
    AMK_CUDA_TRY(cudaMemcpyAsync(c->vx.ptr, vx, nd, cudaMemcpyHostToDevice, c->stream));
    AMK_CUDA_TRY(cudaMemcpyAsync(c->vy.ptr, vy, nd, cudaMemcpyHostToDevice, c->stream));
    AMK_CUDA_TRY(cudaMemcpyAsync(c->vz.ptr, vz, nd, cudaMemcpyHostToDevice, c->stream));
    AMK_CUDA_TRY(cudaMemcpyAsync(c->species.ptr, species, static_cast<size_t>(n), cudaMemcpyHostToDevice, c->stream));
  }
  return finish_load(c, n);
}

extern "C" int amk_set_particles_device(amk_ctx* c, long n, const double* x, const double* y,
                                        const double* z, const double* vx, const double* vy,
                                        const double* vz, const uint8_t* species) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  if (n < 0 || n > 0x7fffffffL) return fail(AMK_ERR_LIMIT, "particle count %ld outside [0, 2^31)", n);
  if (n > 0 && (!x || !y || !z || !vx || !vy || !vz || !species))
    return fail(AMK_ERR_INVALID, "amk_set_particles_device: null array");
  AMK_CUDA_TRY(cudaSetDevice(c->device));
  AMK_TRY(ensure_capacity(c, n));
  const size_t nd = static_cast<size_t>(n) * sizeof(double);
  if (n > 0) {
    AMK_CUDA_TRY(cudaMemcpyAsync(c->x.ptr, x, nd, cudaMemcpyDeviceToDevice, c->stream));
    AMK_CUDA_TRY(cudaMemcpyAsync(c->y.ptr, y, nd, cudaMemcpyDeviceToDevice, c->stream));
    AMK_CUDA_TRY(cudaMemcpyAsync(c->z.ptr, z, nd, cudaMemcpyDeviceToDevice, c->stream));
    AMK_CUDA_TRY(cudaMemcpyAsync(c->vx.ptr, vx, nd, cudaMemcpyDeviceToDevice, c->stream));
    AMK_CUDA_TRY(cudaMemcpyAsync(c->vy.ptr, vy, nd, cudaMemcpyDeviceToDevice, c->stream));
    AMK_CUDA_TRY(cudaMemcpyAsync(c->vz.ptr, vz, nd, cudaMemcpyDeviceToDevice, c->stream));
    AMK_CUDA_TRY(cudaMemcpyAsync(c->species.ptr, species, static_cast<size_t>(n), cudaMemcpyDeviceToDevice, c->stream));
  }
  return finish_load(c, n);
}

extern "C" int amk_update_state(amk_ctx* c, const double* x, const double* y, const double* z,
                                const double* vx, const double* vy, const double* vz) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  const size_t nd = static_cast<size_t>(c->n) * sizeof(double);
  if (c->n == 0) return AMK_OK;
  if (!x || !y || !z || !vx || !vy || !vz) return fail(AMK_ERR_INVALID, "amk_update_state: null array");
  AMK_CUDA_TRY(cudaMemcpyAsync(c->x.ptr, x, nd, cudaMemcpyHostToDevice, c->stream));
  AMK_CUDA_TRY(cudaMemcpyAsync(c->y.ptr, y, nd, cudaMemcpyHostToDevice, c->stream));
  AMK_CUDA_TRY(cudaMemcpyAsync(c->z.ptr, z, nd, cudaMemcpyHostToDevice, c->stream));
  AMK_CUDA_TRY(cudaMemcpyAsync(c->vx.ptr, vx, nd, cudaMemcpyHostToDevice, c->stream));
  AMK_CUDA_TRY(cudaMemcpyAsync(c->vy.ptr, vy, nd, cudaMemcpyHostToDevice, c->stream));
  AMK_CUDA_TRY(cudaMemcpyAsync(c->vz.ptr, vz, nd, cudaMemcpyHostToDevice, c->stream));
  c->stage_dirty = true;
  return AMK_OK;
}

extern "C" int amk_set_charge_mass(amk_ctx* c, const double* charge, const double* mass) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  const size_t nd = static_cast<size_t>(c->n) * sizeof(double);
  if (c->n == 0) return AMK_OK;
  if (charge) AMK_CUDA_TRY(cudaMemcpyAsync(c->q.ptr, charge, nd, cudaMemcpyHostToDevice, c->stream));
  if (mass) AMK_CUDA_TRY(cudaMemcpyAsync(c->m.ptr, mass, nd, cudaMemcpyHostToDevice, c->stream));
  c->stage_dirty = true;
  return AMK_OK;
}

// Host arrays overwrite the force slots (the agents' coulomb_force_), the
// stable ids that key the random streams, or the alive flags.
extern "C" int amk_set_forces(amk_ctx* c, const double* fx, const double* fy, const double* fz) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  if (c->n == 0) return AMK_OK;
  if (!fx || !fy || !fz) return fail(AMK_ERR_INVALID, "amk_set_forces: null array");
  const size_t nd = static_cast<size_t>(c->n) * sizeof(double);
  AMK_CUDA_TRY(cudaMemcpyAsync(c->fx.ptr, fx, nd, cudaMemcpyHostToDevice, c->stream));
  AMK_CUDA_TRY(cudaMemcpyAsync(c->fy.ptr, fy, nd, cudaMemcpyHostToDevice, c->stream));
  AMK_CUDA_TRY(cudaMemcpyAsync(c->fz.ptr, fz, nd, cudaMemcpyHostToDevice, c->stream));
  return AMK_OK;
}

extern "C" int amk_set_ids(amk_ctx* c, const uint32_t* ids) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  if (c->n == 0) return AMK_OK;
  if (!ids) return fail(AMK_ERR_INVALID, "amk_set_ids: null array");
  AMK_CUDA_TRY(cudaMemcpyAsync(c->ids.ptr, ids, static_cast<size_t>(c->n) * sizeof(uint32_t), cudaMemcpyHostToDevice,
                               c->stream));
  return AMK_OK;
}

extern "C" int amk_set_alive(amk_ctx* c, const uint8_t* alive) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  if (c->n == 0) return AMK_OK;
  if (!alive) return fail(AMK_ERR_INVALID, "amk_set_alive: null array");
  AMK_CUDA_TRY(cudaMemcpyAsync(c->alive.ptr, alive, static_cast<size_t>(c->n), cudaMemcpyHostToDevice, c->stream));
  c->stage_dirty = true;
  return AMK_OK;
}

// Completed steps (the random streams' step is this + 1 on the next push)
// and whether the velocities are already staggered to t - dt/2.
extern "C" int amk_set_step_state(amk_ctx* c, long step, int staggered) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  if (step < 0) return fail(AMK_ERR_INVALID, "amk_set_step_state: step < 0");
  c->step = step;
  c->staggered = staggered != 0;
  return AMK_OK;
}

// Reference initial cloud, host side (penning_trap.cc:51-160). The streams are
// the C++ standard engines the reference uses, so the cloud is bit-identical.
extern "C" int amk_init_particles(amk_ctx* c) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  const amk_params& p = c->p;
  std::map<int, long> pops;
  std::map<int, double> temps;
  for (int k = 0; k < p.n_species; ++k) {
    if (p.species[k] < 0 || p.species[k] >= AMK_MAX_SPECIES || p.populations[k] < 0)
      return fail(AMK_ERR_INVALID, "bad population entry %d", k);
    pops[p.species[k]] = p.populations[k];
    temps[p.species[k]] = p.temperatures[k];
  }
  long total = 0;
  for (auto& kv : pops) total += kv.second;
  if (total <= 0) return fail(AMK_ERR_INVALID, "PenningTrapField: Total particles in PenningTrap should be > 0");
  std::vector<double> x(total), y(total), z(total), vx(total), vy(total), vz(total);
  std::vector<uint8_t> sp(total);
  {  // positions: penning_trap.cc:118-160
    std::default_random_engine rng(p.seed);
    std::uniform_real_distribution<double> ox(-p.cloud_radii[0], p.cloud_radii[0]);
    std::uniform_real_distribution<double> oy(-p.cloud_radii[1], p.cloud_radii[1]);
    std::uniform_real_distribution<double> oz(-p.cloud_radii[2], p.cloud_radii[2]);
    long w = 0;
    for (auto& kv : pops) {
      for (long i = 0; i < kv.second; ++i, ++w) {
        double px, py, pz;
        for (;;) {
          px = ox(rng);
          py = oy(rng);
          pz = oz(rng);
          const double a = px / p.cloud_radii[0], b = py / p.cloud_radii[1], d = pz / p.cloud_radii[2];
          if ((a * a) + (b * b) + (d * d) <= 1.0) break;
        }
        x[w] = px;
        y[w] = py;
        z[w] = pz;
        sp[w] = static_cast<uint8_t>(kv.first);
      }
    }
  }
  {  // velocities: penning_trap.cc:51-115
    long w = 0;
    for (auto& kv : pops) {
      const long count = kv.second;
      const double temp = temps[kv.first];
      if (temp == 0.0) {
        for (long i = 0; i < count; ++i, ++w) vx[w] = vy[w] = vz[w] = 0.0;
        continue;
      }
      double mass, charge;
      species_properties(kv.first, &mass, &charge);
      const double sigma = std::sqrt(kBoltzmann * temp / mass);
      std::mt19937 rng(p.seed);
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
      for (long i = 0; i < count; ++i, ++w) {
        vx[w] = raw[3 * i];
        vy[w] = raw[3 * i + 1];
        vz[w] = raw[3 * i + 2];
      }
    }
  }
  return amk_set_particles(c, total, x.data(), y.data(), z.data(), vx.data(), vy.data(), vz.data(), sp.data());
}

extern "C" int amk_get_particles(amk_ctx* c, double* x, double* y, double* z, double* vx, double* vy,
                                 double* vz, uint8_t* alive) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  const size_t nd = static_cast<size_t>(c->n) * sizeof(double);
  if (c->n > 0) {
    if (x) AMK_CUDA_TRY(cudaMemcpyAsync(x, c->x.ptr, nd, cudaMemcpyDeviceToHost, c->stream));
    if (y) AMK_CUDA_TRY(cudaMemcpyAsync(y, c->y.ptr, nd, cudaMemcpyDeviceToHost, c->stream));
    if (z) AMK_CUDA_TRY(cudaMemcpyAsync(z, c->z.ptr, nd, cudaMemcpyDeviceToHost, c->stream));
    if (vx) AMK_CUDA_TRY(cudaMemcpyAsync(vx, c->vx.ptr, nd, cudaMemcpyDeviceToHost, c->stream));
    if (vy) AMK_CUDA_TRY(cudaMemcpyAsync(vy, c->vy.ptr, nd, cudaMemcpyDeviceToHost, c->stream));
    if (vz) AMK_CUDA_TRY(cudaMemcpyAsync(vz, c->vz.ptr, nd, cudaMemcpyDeviceToHost, c->stream));
    if (alive) AMK_CUDA_TRY(cudaMemcpyAsync(alive, c->alive.ptr, static_cast<size_t>(c->n), cudaMemcpyDeviceToHost, c->stream));
  }
  AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return AMK_OK;
}

extern "C" int amk_get_particles_device(amk_ctx* c, double* x, double* y, double* z, double* vx,
                                        double* vy, double* vz, uint8_t* alive) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  const size_t nd = static_cast<size_t>(c->n) * sizeof(double);
  if (c->n > 0) {
    if (x) AMK_CUDA_TRY(cudaMemcpyAsync(x, c->x.ptr, nd, cudaMemcpyDeviceToDevice, c->stream));
    if (y) AMK_CUDA_TRY(cudaMemcpyAsync(y, c->y.ptr, nd, cudaMemcpyDeviceToDevice, c->stream));
    if (z) AMK_CUDA_TRY(cudaMemcpyAsync(z, c->z.ptr, nd, cudaMemcpyDeviceToDevice, c->stream));
    if (vx) AMK_CUDA_TRY(cudaMemcpyAsync(vx, c->vx.ptr, nd, cudaMemcpyDeviceToDevice, c->stream));
    if (vy) AMK_CUDA_TRY(cudaMemcpyAsync(vy, c->vy.ptr, nd, cudaMemcpyDeviceToDevice, c->stream));
    if (vz) AMK_CUDA_TRY(cudaMemcpyAsync(vz, c->vz.ptr, nd, cudaMemcpyDeviceToDevice, c->stream));
    if (alive) AMK_CUDA_TRY(cudaMemcpyAsync(alive, c->alive.ptr, static_cast<size_t>(c->n), cudaMemcpyDeviceToDevice, c->stream));
  }
  return AMK_OK;
}

extern "C" long amk_num_particles(const amk_ctx* c) { return c ? c->n : -1; }

__global__ void count_alive_kernel(long n, const uint8_t* __restrict__ alive, unsigned long long* out) {
  unsigned long long k = 0;
  for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<long>(gridDim.x) * blockDim.x)
    k += alive[i] ? 1 : 0;
  for (int o = 16; o > 0; o >>= 1) k += __shfl_xor_sync(0xffffffffu, k, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, k);
}

extern "C" long amk_num_alive(amk_ctx* c) {
  if (!c) return -1;
  if (c->n == 0) return 0;
  int rc = AMK_OK;
  unsigned long long* d = slot<unsigned long long>(c, kSlotStatus, 4, &rc);
  if (rc != AMK_OK) return rc;
  if (cudaMemsetAsync(d, 0, sizeof(unsigned long long), c->stream) != cudaSuccess) return fail(AMK_ERR_CUDA, "memset");
  count_alive_kernel<<<148, 256, 0, c->stream>>>(c->n, c->alive.as<uint8_t>(), d);
  if (check_launch(c, "count_alive_kernel") != AMK_OK) return AMK_ERR_CUDA;
  unsigned long long h = 0;
  if (cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess)
    return fail(AMK_ERR_CUDA, "readback failed");
  return static_cast<long>(h);
}

// ============================================================== forces
extern "C" int amk_coulomb_allpairs(amk_ctx* c) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  if (c->n == 0) return AMK_OK;
  return allpairs_forces(c, main_view(c));
}

extern "C" int amk_coulomb_standard(amk_ctx* c, double cutoff) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  if (c->n == 0) return AMK_OK;
  return cutoff_forces(c, main_view(c), cutoff, nullptr);
}

extern "C" int amk_coulomb_barnes_hut(amk_ctx* c, double theta) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  if (c->n == 0) return AMK_OK;
  return barnes_hut_forces(c, main_view(c), theta, c->bh_leaf);
}

// learned != 0 uses the p=2 far field plus the trained correction while it is
// trained and its audits pass; otherwise plain FMM at learned_fallback_order.
extern "C" int amk_coulomb_fmm(amk_ctx* c, int order, double theta, int learned) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  if (c->n == 0) return AMK_OK;
  if (learned) {
    if (c->learned_trained && !c->learned_fallback)
      return fmm_forces(c, main_view(c), 2, theta, c->fmm_leaf, true, nullptr);
    order = c->p.learned_fallback_order;
  }
  return fmm_forces(c, main_view(c), order, theta, c->fmm_leaf, false, nullptr);
}

extern "C" int amk_fmm_train_correction(amk_ctx* c, double theta, int sample_leaves, int steps, long batch, float lr,
                                        float* final_loss, long* samples) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  if (c->n == 0) return fail(AMK_ERR_STATE, "no particles");
  AMK_TRY(fmm_train_learned(c, main_view(c), theta, sample_leaves, steps, batch, lr, final_loss, samples));
  c->learned_trained = true;
  c->learned_fallback = false;
  return AMK_OK;
}

extern "C" int amk_fmm_audit(amk_ctx* c, int order, double theta, int learned, long samples, double* rms) {
  if (!c || !rms) return fail(AMK_ERR_INVALID, "null argument");
  *rms = 0.0;
  if (c->n == 0) return AMK_OK;
  if (learned && !c->learned_trained) return fail(AMK_ERR_STATE, "the learned correction is not trained");
  return fmm_audit(c, main_view(c), order, theta, learned != 0, samples, rms);
}

extern "C" int amk_fmm_learned_state(amk_ctx* c, int* trained, int* fallback, double* last_error) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  if (trained) *trained = c->learned_trained ? 1 : 0;
  if (fallback) *fallback = c->learned_fallback ? 1 : 0;
  if (last_error) *last_error = c->learned_last_error;
  return AMK_OK;
}

extern "C" int amk_set_leaf_sizes(amk_ctx* c, int fmm_leaf, int bh_leaf) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  if (fmm_leaf < 1 || fmm_leaf > 256 || bh_leaf < 1 || bh_leaf > 256)
    return fail(AMK_ERR_INVALID, "leaf capacities must be in [1, 256]");
  c->fmm_leaf = fmm_leaf;
  c->bh_leaf = bh_leaf;
  return AMK_OK;
}

extern "C" int amk_get_leaf_sizes(const amk_ctx* c, int* fmm_leaf, int* bh_leaf) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  if (fmm_leaf) *fmm_leaf = c->fmm_leaf;
  if (bh_leaf) *bh_leaf = c->bh_leaf;
  return AMK_OK;
}

extern "C" int amk_coulomb(amk_ctx* c) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  if (!c->p.coulomb_forces_enabled) return AMK_OK;
  switch (c->p.coulomb_method) {
    case AMK_METHOD_STANDARD: return amk_coulomb_standard(c, c->p.cutoff_radius);
    case AMK_METHOD_BARNES_HUT: return amk_coulomb_barnes_hut(c, c->p.barnes_hut_theta);
    case AMK_METHOD_FAST_MULTIPOLE:
      // fast_multipole_order is a real truncated to int (antimatter-kernel.cc:158)
      return amk_coulomb_fmm(c, static_cast<int>(c->p.fast_multipole_order), c->p.fast_multipole_theta,
                             c->p.fmm_learned);
    case AMK_METHOD_ALLPAIRS: return amk_coulomb_allpairs(c);
    default: return fail(AMK_ERR_INVALID, "unknown coulomb method %d", c->p.coulomb_method);
  }
}

extern "C" int amk_get_forces(amk_ctx* c, double* fx, double* fy, double* fz) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  const size_t nd = static_cast<size_t>(c->n) * sizeof(double);
  if (c->n > 0) {
    if (fx) AMK_CUDA_TRY(cudaMemcpyAsync(fx, c->fx.ptr, nd, cudaMemcpyDeviceToHost, c->stream));
    if (fy) AMK_CUDA_TRY(cudaMemcpyAsync(fy, c->fy.ptr, nd, cudaMemcpyDeviceToHost, c->stream));
    if (fz) AMK_CUDA_TRY(cudaMemcpyAsync(fz, c->fz.ptr, nd, cudaMemcpyDeviceToHost, c->stream));
  }
  AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return AMK_OK;
}

// ============================================================== stepping

// The push is the behaviour every step runs (LorentzForce is always attached,
// antimatter-kernel.cc:93), so it advances the step counter; the annihilation
// of the same step uses that counter for its random stream.
extern "C" int amk_push(amk_ctx* c) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  if (c->batch) return fail(AMK_ERR_STATE, "the context holds a batch: step it with amk_batch_step");
  if (c->n > 0) {
    AMK_TRY(push_step(c, static_cast<uint64_t>(c->step + 1)));
    c->stage_dirty = true;
  }
  c->step++;
  return AMK_OK;
}

extern "C" int amk_annihilate(amk_ctx* c, long* marked) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  if (c->batch) return fail(AMK_ERR_STATE, "the context holds a batch: step it with amk_batch_step");
  if (marked) *marked = 0;
  if (c->n == 0 || !c->p.annihilation_enabled) return AMK_OK;
  AMK_TRY(annihilate_step(c, static_cast<uint64_t>(c->step > 0 ? c->step : 1), marked));
  c->stage_dirty = true;
  return AMK_OK;
}

extern "C" int amk_step(amk_ctx* c, int nsteps) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  if (c->batch) return fail(AMK_ERR_STATE, "the context holds a batch: step it with amk_batch_step");
  if (nsteps < 0) return fail(AMK_ERR_INVALID, "nsteps < 0");
  AMK_CUDA_TRY(cudaSetDevice(c->device));
  for (int s = 0; s < nsteps; ++s) {
    // periodic direct-sum audit of the learned correction; a failure switches
    // the context to plain FMM at learned_fallback_order
    const amk_params& p = c->p;
    if (c->n > 0 && p.coulomb_forces_enabled && p.coulomb_method == AMK_METHOD_FAST_MULTIPOLE && p.fmm_learned &&
        c->learned_trained && !c->learned_fallback && p.learned_audit_interval > 0 &&
        c->step % p.learned_audit_interval == 0) {
      double err = 0.0;
      AMK_TRY(fmm_audit(c, main_view(c), 2, p.fast_multipole_theta, true, p.learned_audit_samples, &err));
      c->learned_last_error = err;
      if (!(err <= p.learned_error_budget)) c->learned_fallback = true;
    }
    if (c->n > 0) AMK_TRY(amk_coulomb(c));
    AMK_TRY(amk_push(c));
    if (c->n > 0 && c->p.annihilation_enabled) AMK_TRY(amk_annihilate(c, nullptr));
  }
  return AMK_OK;
}

extern "C" long amk_step_count(const amk_ctx* c) { return c ? c->step : -1; }

// ============================================================== profiling
extern "C" int amk_set_profiling(amk_ctx* c, int enabled) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  c->profiling = enabled != 0;
  return AMK_OK;
}

extern "C" int amk_phase_times(amk_ctx* c, double* ms, long* launches, int n) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  AMK_TRY(harvest_events(c));
  for (int k = 0; k < n && k < AMK_NUM_PHASES; ++k) {
    if (ms) ms[k] = c->clock.ms[k];
    if (launches) launches[k] = c->clock.launches[k];
  }
  return AMK_OK;
}

extern "C" int amk_reset_phase_times(amk_ctx* c) {
  if (!c) return fail(AMK_ERR_INVALID, "null context");
  AMK_TRY(harvest_events(c));
  for (int k = 0; k < AMK_NUM_PHASES; ++k) {
    c->clock.ms[k] = 0.0;
    c->clock.launches[k] = 0;
  }
  return AMK_OK;
}

extern "C" long amk_kernel_launches(const amk_ctx* c) { return c ? c->kernel_launches : -1; }
