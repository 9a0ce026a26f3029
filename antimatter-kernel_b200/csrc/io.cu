// Checkpoint/resume of a context and headless particle export, in place of
// BioDynaMo's backup/restore and its ParaView visualisation export
// (bdm.toml:6-13: ChargedAntiparticle agents every `interval` steps with the
// additional data member species_id). Host code only; the state is copied
// off the device with the context's stream.
//
// Checkpoint file (little-endian, version 1):
//   "AMKCKPT\0", u32 version, u32 sizeof(amk_params), amk_params,
//   i64 n, i64 step, u8 staggered, u8 energy_has_previous, u8 learned_trained,
//   u8 learned_fallback, i32 fmm_leaf, i32 bh_leaf, f64 prev_trap,
//   f64 prev_coulomb, f64 learned_last_error, f64 length_scale,
//   i64 n_mlp, f32[n_mlp] network parameters (0 when untrained),
//   i64 n_perm, i32 perm_age, u32[n_perm] all-pairs Morton order (0 when none),
//   f64[n] x y z vx vy vz fx fy fz q m, u8[n] species, u8[n] alive, u32[n] ids,
//   u64 FNV-1a hash of every byte before it.
// A context restored from it continues bit for bit like the saved one.
//
// Particle export: VTK XML UnstructuredGrid (.vtu) of the live particles as
// vertex cells with point data species_id (Int32), velocity (Float64 x 3)
// and id (UInt32), the simulated time as field data TimeValue; data inline
// as ASCII or appended raw binary. A .pvd collection lists a time series.
#include <cinttypes>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "amk_internal.cuh"

namespace amk {
namespace {

constexpr char kMagic[8] = {'A', 'M', 'K', 'C', 'K', 'P', 'T', '\0'};
constexpr uint32_t kVersion = 1;

struct Fnv {
  uint64_t h = 1469598103934665603ull;
  void add(const void* p, size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; ++i) {
      h ^= b[i];
      h *= 1099511628211ull;
    }
  }
};

struct Writer {
  FILE* f = nullptr;
  Fnv hash;
  bool ok = true;
  void put(const void* p, size_t n) {
    if (!ok || n == 0) return;
    hash.add(p, n);
    ok = std::fwrite(p, 1, n, f) == n;
  }
  template <typename T>
  void val(const T& v) {
    put(&v, sizeof(T));
  }
};

struct Reader {
  FILE* f = nullptr;
  Fnv hash;
  bool ok = true;
  void get(void* p, size_t n) {
    if (!ok || n == 0) return;
    ok = std::fread(p, 1, n, f) == n;
    if (ok) hash.add(p, n);
  }
  template <typename T>
  T val() {
    T v{};
    get(&v, sizeof(T));
    return v;
  }
};

struct HostState {
  long n = 0;
  std::vector<double> a[11];  // x y z vx vy vz fx fy fz q m
  std::vector<uint8_t> species, alive;
  std::vector<uint32_t> ids;
};

int copy_out(amk_ctx* c, HostState* h) {
  h->n = c->n;
  const size_t n = static_cast<size_t>(c->n);
  DevBuf* src[11] = {&c->x, &c->y, &c->z, &c->vx, &c->vy, &c->vz, &c->fx, &c->fy, &c->fz, &c->q, &c->m};
  for (int k = 0; k < 11; ++k) {
    h->a[k].resize(n);
    if (n) AMK_CUDA_TRY(cudaMemcpyAsync(h->a[k].data(), src[k]->ptr, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  }
  h->species.resize(n);
  h->alive.resize(n);
  h->ids.resize(n);
  if (n) {
    AMK_CUDA_TRY(cudaMemcpyAsync(h->species.data(), c->species.ptr, n, cudaMemcpyDeviceToHost, c->stream));
    AMK_CUDA_TRY(cudaMemcpyAsync(h->alive.data(), c->alive.ptr, n, cudaMemcpyDeviceToHost, c->stream));
    AMK_CUDA_TRY(cudaMemcpyAsync(h->ids.data(), c->ids.ptr, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
  }
  AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return AMK_OK;
}

struct Header {
  amk_params p;
  long n = 0, step = 0;
  uint8_t staggered = 0, has_prev = 0, learned_trained = 0, learned_fallback = 0;
  int32_t fmm_leaf = 32, bh_leaf = 8;
  double prev_trap = 0.0, prev_coulomb = 0.0, learned_last_error = -1.0, length_scale = 1.0;
};

// Reads the header fields (up to and excluding the network parameters).
int read_header(Reader& r, Header* h) {
  char magic[8];
  r.get(magic, sizeof(magic));
  if (!r.ok || std::memcmp(magic, kMagic, sizeof(magic)) != 0) return fail(AMK_ERR_INVALID, "not an amk checkpoint");
  const uint32_t version = r.val<uint32_t>();
  if (!r.ok || version != kVersion) return fail(AMK_ERR_INVALID, "checkpoint version %u, expected %u", version, kVersion);
  const uint32_t psize = r.val<uint32_t>();
  if (!r.ok || psize != sizeof(amk_params))
    return fail(AMK_ERR_INVALID, "checkpoint parameter block of %u bytes, this library's is %zu", psize,
                sizeof(amk_params));
  r.get(&h->p, sizeof(amk_params));
  h->n = static_cast<long>(r.val<int64_t>());
  h->step = static_cast<long>(r.val<int64_t>());
  h->staggered = r.val<uint8_t>();
  h->has_prev = r.val<uint8_t>();
  h->learned_trained = r.val<uint8_t>();
  h->learned_fallback = r.val<uint8_t>();
  h->fmm_leaf = r.val<int32_t>();
  h->bh_leaf = r.val<int32_t>();
  h->prev_trap = r.val<double>();
  h->prev_coulomb = r.val<double>();
  h->learned_last_error = r.val<double>();
  h->length_scale = r.val<double>();
  if (!r.ok) return fail(AMK_ERR_INVALID, "truncated checkpoint header");
  if (h->n < 0 || h->n > 0x7fffffffL) return fail(AMK_ERR_INVALID, "checkpoint particle count %ld", h->n);
  return AMK_OK;
}

std::string fmt_double(double v) {
  char b[40];
  std::snprintf(b, sizeof(b), "%.17g", v);
  return b;
}

}  // namespace
}  // namespace amk

using namespace amk;

extern "C" int amk_checkpoint_save(amk_ctx* c, const char* path) {
  if (!c || !path) return fail(AMK_ERR_INVALID, "null argument");
  if (c->batch) return fail(AMK_ERR_STATE, "amk_checkpoint_save: the context holds a batch (save single instances)");
  AMK_CUDA_TRY(cudaSetDevice(c->device));
  HostState h;
  AMK_TRY(copy_out(c, &h));
  std::vector<float> mlp;
  if (c->learned_trained) {
    mlp.resize(static_cast<size_t>(amk_mlp_num_params()));
    AMK_TRY(amk_mlp_get_params(c, mlp.data(), static_cast<long>(mlp.size())));
  }
  std::vector<uint32_t> perm;
  if (c->ap_perm_n == c->n && c->n > 0) {
    perm.resize(static_cast<size_t>(c->n));
    AMK_CUDA_TRY(cudaMemcpyAsync(perm.data(), c->ap_perm.ptr, perm.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                 c->stream));
    AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
  }
  const std::string tmp = std::string(path) + ".tmp";
  Writer w;
  w.f = std::fopen(tmp.c_str(), "wb");
  if (!w.f) return fail(AMK_ERR_INVALID, "cannot open '%s' for writing", tmp.c_str());
  w.put(kMagic, sizeof(kMagic));
  w.val<uint32_t>(kVersion);
  w.val<uint32_t>(static_cast<uint32_t>(sizeof(amk_params)));
  w.put(&c->p, sizeof(amk_params));
  w.val<int64_t>(c->n);
  w.val<int64_t>(c->step);
  w.val<uint8_t>(c->staggered ? 1 : 0);
  w.val<uint8_t>(c->energy_has_previous ? 1 : 0);
  w.val<uint8_t>(c->learned_trained ? 1 : 0);
  w.val<uint8_t>(c->learned_fallback ? 1 : 0);
  w.val<int32_t>(c->fmm_leaf);
  w.val<int32_t>(c->bh_leaf);
  w.val<double>(c->prev_trap);
  w.val<double>(c->prev_coulomb);
  w.val<double>(c->learned_last_error);
  w.val<double>(c->length_scale);
  w.val<int64_t>(static_cast<int64_t>(mlp.size()));
  w.put(mlp.data(), mlp.size() * sizeof(float));
  w.val<int64_t>(static_cast<int64_t>(perm.size()));
  w.val<int32_t>(c->ap_perm_age);
  w.put(perm.data(), perm.size() * sizeof(uint32_t));
  for (int k = 0; k < 11; ++k) w.put(h.a[k].data(), h.a[k].size() * sizeof(double));
  w.put(h.species.data(), h.species.size());
  w.put(h.alive.data(), h.alive.size());
  w.put(h.ids.data(), h.ids.size() * sizeof(uint32_t));
  const uint64_t digest = w.hash.h;
  w.put(&digest, sizeof(digest));
  const bool ok = w.ok && std::fclose(w.f) == 0;
  if (!ok || std::rename(tmp.c_str(), path) != 0) {
    std::remove(tmp.c_str());
    return fail(AMK_ERR_INVALID, "writing checkpoint '%s' failed", path);
  }
  return AMK_OK;
}

extern "C" int amk_checkpoint_info(const char* path, long* n, long* step, amk_params* params) {
  if (!path) return fail(AMK_ERR_INVALID, "null path");
  Reader r;
  r.f = std::fopen(path, "rb");
  if (!r.f) return fail(AMK_ERR_INVALID, "cannot open checkpoint '%s'", path);
  Header h;
  const int rc = read_header(r, &h);
  std::fclose(r.f);
  if (rc != AMK_OK) return rc;
  if (n) *n = h.n;
  if (step) *step = h.step;
  if (params) *params = h.p;
  return AMK_OK;
}

extern "C" int amk_checkpoint_load(amk_ctx* c, const char* path) {
  if (!c || !path) return fail(AMK_ERR_INVALID, "null argument");
  Reader r;
  r.f = std::fopen(path, "rb");
  if (!r.f) return fail(AMK_ERR_INVALID, "cannot open checkpoint '%s'", path);
  Header h;
  int rc = read_header(r, &h);
  std::vector<float> mlp;
  std::vector<uint32_t> perm;
  HostState s;
  int32_t perm_age = 0;
  if (rc == AMK_OK) {
    const int64_t n_mlp = r.val<int64_t>();
    if (r.ok && n_mlp != 0 && n_mlp != amk_mlp_num_params()) rc = fail(AMK_ERR_INVALID, "checkpoint network size");
    if (rc == AMK_OK) {
      mlp.resize(static_cast<size_t>(n_mlp));
      r.get(mlp.data(), mlp.size() * sizeof(float));
      const int64_t n_perm = r.val<int64_t>();
      perm_age = r.val<int32_t>();
      if (r.ok && n_perm != 0 && n_perm != h.n) rc = fail(AMK_ERR_INVALID, "checkpoint permutation size");
      if (rc == AMK_OK) {
        perm.resize(static_cast<size_t>(n_perm));
        r.get(perm.data(), perm.size() * sizeof(uint32_t));
        const size_t n = static_cast<size_t>(h.n);
        for (int k = 0; k < 11; ++k) {
          s.a[k].resize(n);
          r.get(s.a[k].data(), n * sizeof(double));
        }
        s.species.resize(n);
        s.alive.resize(n);
        s.ids.resize(n);
        r.get(s.species.data(), n);
        r.get(s.alive.data(), n);
        r.get(s.ids.data(), n * sizeof(uint32_t));
        const uint64_t expect = r.hash.h;
        uint64_t digest = 0;
        if (r.ok) r.ok = std::fread(&digest, 1, sizeof(digest), r.f) == sizeof(digest);
        if (!r.ok) rc = fail(AMK_ERR_INVALID, "truncated checkpoint '%s'", path);
        else if (digest != expect) rc = fail(AMK_ERR_INVALID, "checkpoint '%s' fails its checksum", path);
      }
    }
  }
  std::fclose(r.f);
  if (rc != AMK_OK) return rc;
  // the parameters first, then the particles (which reset the step state)
  AMK_TRY(amk_set_params(c, &h.p));
  const long n = h.n;
  const std::vector<double>* a = s.a;
  AMK_TRY(amk_set_particles(c, n, a[0].data(), a[1].data(), a[2].data(), a[3].data(), a[4].data(), a[5].data(),
                            s.species.data()));
  if (n > 0) {
    const size_t nd = static_cast<size_t>(n) * sizeof(double);
    DevBuf* dst[5] = {&c->fx, &c->fy, &c->fz, &c->q, &c->m};
    for (int k = 0; k < 5; ++k)
      AMK_CUDA_TRY(cudaMemcpyAsync(dst[k]->ptr, a[6 + k].data(), nd, cudaMemcpyHostToDevice, c->stream));
    AMK_CUDA_TRY(cudaMemcpyAsync(c->alive.ptr, s.alive.data(), static_cast<size_t>(n), cudaMemcpyHostToDevice, c->stream));
    AMK_CUDA_TRY(cudaMemcpyAsync(c->ids.ptr, s.ids.data(), static_cast<size_t>(n) * sizeof(uint32_t),
                                 cudaMemcpyHostToDevice, c->stream));
    if (!perm.empty()) {
      AMK_TRY(c->ap_perm.reserve(perm.size() * sizeof(uint32_t)));
      AMK_CUDA_TRY(cudaMemcpyAsync(c->ap_perm.ptr, perm.data(), perm.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                                   c->stream));
      c->ap_perm_n = n;
      c->ap_perm_age = perm_age;
    }
  }
  if (!mlp.empty()) AMK_TRY(amk_mlp_set_params(c, mlp.data(), static_cast<long>(mlp.size())));
  AMK_CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->step = h.step;
  c->staggered = h.staggered != 0;
  c->energy_has_previous = h.has_prev != 0;
  c->prev_trap = h.prev_trap;
  c->prev_coulomb = h.prev_coulomb;
  c->fmm_leaf = h.fmm_leaf;
  c->bh_leaf = h.bh_leaf;
  c->learned_trained = h.learned_trained != 0;
  c->learned_fallback = h.learned_fallback != 0;
  c->learned_last_error = h.learned_last_error;
  c->length_scale = h.length_scale;
  c->stage_dirty = true;
  return AMK_OK;
}

extern "C" int amk_write_vtu(const char* path, long n, const double* x, const double* y, const double* z,
                             const double* vx, const double* vy, const double* vz, const uint8_t* species,
                             const uint8_t* alive, const uint32_t* ids, double time, int binary) {
  if (!path || n < 0) return fail(AMK_ERR_INVALID, "amk_write_vtu: bad argument");
  if (n > 0 && (!x || !y || !z || !species)) return fail(AMK_ERR_INVALID, "amk_write_vtu: null array");
  std::vector<long> live;
  live.reserve(static_cast<size_t>(n));
  for (long i = 0; i < n; ++i)
    if (!alive || alive[i]) live.push_back(i);
  const long m = static_cast<long>(live.size());
  std::vector<double> pts(3 * static_cast<size_t>(m)), vel(3 * static_cast<size_t>(m), 0.0);
  std::vector<int32_t> sp(static_cast<size_t>(m));
  std::vector<uint32_t> uid(static_cast<size_t>(m));
  std::vector<int64_t> conn(static_cast<size_t>(m)), offs(static_cast<size_t>(m));
  std::vector<uint8_t> types(static_cast<size_t>(m), 1);  // VTK_VERTEX
  for (long k = 0; k < m; ++k) {
    const long i = live[k];
    pts[3 * k] = x[i];
    pts[3 * k + 1] = y[i];
    pts[3 * k + 2] = z[i];
    if (vx && vy && vz) {
      vel[3 * k] = vx[i];
      vel[3 * k + 1] = vy[i];
      vel[3 * k + 2] = vz[i];
    }
    sp[k] = species[i];
    uid[k] = ids ? ids[i] : static_cast<uint32_t>(i);
    conn[k] = k;
    offs[k] = k + 1;
  }
  struct Arr {
    const char* type;
    const char* name;
    int comps;
    const void* data;
    size_t elem, count;
    const char* section;
  };
  const Arr arrays[] = {
      {"Float64", "Points", 3, pts.data(), 8, pts.size(), "Points"},
      {"Int64", "connectivity", 1, conn.data(), 8, conn.size(), "Cells"},
      {"Int64", "offsets", 1, offs.data(), 8, offs.size(), "Cells"},
      {"UInt8", "types", 1, types.data(), 1, types.size(), "Cells"},
      {"Int32", "species_id", 1, sp.data(), 4, sp.size(), "PointData"},
      {"Float64", "velocity", 3, vel.data(), 8, vel.size(), "PointData"},
      {"UInt32", "id", 1, uid.data(), 4, uid.size(), "PointData"},
  };
  FILE* f = std::fopen(path, "wb");
  if (!f) return fail(AMK_ERR_INVALID, "cannot open '%s' for writing", path);
  std::fprintf(f, "<?xml version=\"1.0\"?>\n<VTKFile type=\"UnstructuredGrid\" version=\"1.0\" "
                  "byte_order=\"LittleEndian\" header_type=\"UInt64\">\n<UnstructuredGrid>\n");
  std::fprintf(f, "<FieldData><DataArray type=\"Float64\" Name=\"TimeValue\" NumberOfTuples=\"1\" format=\"ascii\">%s"
                  "</DataArray></FieldData>\n", fmt_double(time).c_str());
  std::fprintf(f, "<Piece NumberOfPoints=\"%ld\" NumberOfCells=\"%ld\">\n", m, m);
  uint64_t offset = 0;
  const char* open_section = nullptr;
  for (const Arr& a : arrays) {
    if (!open_section || std::strcmp(open_section, a.section) != 0) {
      if (open_section) std::fprintf(f, "</%s>\n", open_section);
      if (std::strcmp(a.section, "PointData") == 0)
        std::fprintf(f, "<PointData Scalars=\"species_id\" Vectors=\"velocity\">\n");
      else
        std::fprintf(f, "<%s>\n", a.section);
      open_section = a.section;
    }
    const char* nm = std::strcmp(a.name, "Points") == 0 ? "" : a.name;
    if (binary) {
      std::fprintf(f, "<DataArray type=\"%s\" Name=\"%s\" NumberOfComponents=\"%d\" format=\"appended\" "
                      "offset=\"%" PRIu64 "\"/>\n", a.type, nm, a.comps, offset);
      offset += sizeof(uint64_t) + a.elem * a.count;
    } else {
      std::fprintf(f, "<DataArray type=\"%s\" Name=\"%s\" NumberOfComponents=\"%d\" format=\"ascii\">\n", a.type, nm,
                   a.comps);
      for (size_t k = 0; k < a.count; ++k) {
        const char* sep = (k + 1) % 12 == 0 ? "\n" : " ";
        if (std::strcmp(a.type, "Float64") == 0)
          std::fprintf(f, "%s%s", fmt_double(static_cast<const double*>(a.data)[k]).c_str(), sep);
        else if (std::strcmp(a.type, "Int64") == 0)
          std::fprintf(f, "%" PRId64 "%s", static_cast<const int64_t*>(a.data)[k], sep);
        else if (std::strcmp(a.type, "Int32") == 0)
          std::fprintf(f, "%d%s", static_cast<const int32_t*>(a.data)[k], sep);
        else if (std::strcmp(a.type, "UInt32") == 0)
          std::fprintf(f, "%u%s", static_cast<const uint32_t*>(a.data)[k], sep);
        else
          std::fprintf(f, "%u%s", static_cast<unsigned>(static_cast<const uint8_t*>(a.data)[k]), sep);
      }
      std::fprintf(f, "\n</DataArray>\n");
    }
  }
  std::fprintf(f, "</%s>\n</Piece>\n</UnstructuredGrid>\n", open_section);
  bool ok = true;
  if (binary) {
    std::fprintf(f, "<AppendedData encoding=\"raw\">\n_");
    for (const Arr& a : arrays) {
      const uint64_t bytes = a.elem * a.count;
      ok = ok && std::fwrite(&bytes, sizeof(bytes), 1, f) == 1;
      if (bytes) ok = ok && std::fwrite(a.data, 1, bytes, f) == bytes;
    }
    std::fprintf(f, "\n</AppendedData>\n");
  }
  std::fprintf(f, "</VTKFile>\n");
  ok = std::fclose(f) == 0 && ok;
  return ok ? AMK_OK : fail(AMK_ERR_INVALID, "writing '%s' failed", path);
}

extern "C" int amk_export_vtk(amk_ctx* c, const char* path, int binary) {
  if (!c || !path) return fail(AMK_ERR_INVALID, "null argument");
  AMK_CUDA_TRY(cudaSetDevice(c->device));
  HostState h;
  AMK_TRY(copy_out(c, &h));
  const double time = static_cast<double>(c->step) * c->p.dt;
  return amk_write_vtu(path, h.n, h.a[0].data(), h.a[1].data(), h.a[2].data(), h.a[3].data(), h.a[4].data(),
                       h.a[5].data(), h.species.data(), h.alive.data(), h.ids.data(), time, binary);
}

extern "C" int amk_write_pvd(const char* path, long n, const char* const* files, const double* times) {
  if (!path || n < 0 || (n > 0 && (!files || !times))) return fail(AMK_ERR_INVALID, "amk_write_pvd: bad argument");
  FILE* f = std::fopen(path, "wb");
  if (!f) return fail(AMK_ERR_INVALID, "cannot open '%s' for writing", path);
  std::fprintf(f, "<?xml version=\"1.0\"?>\n<VTKFile type=\"Collection\" version=\"1.0\" "
                  "byte_order=\"LittleEndian\">\n<Collection>\n");
  for (long k = 0; k < n; ++k)
    std::fprintf(f, "<DataSet timestep=\"%s\" part=\"0\" file=\"%s\"/>\n", fmt_double(times[k]).c_str(), files[k]);
  std::fprintf(f, "</Collection>\n</VTKFile>\n");
  return std::fclose(f) == 0 ? AMK_OK : fail(AMK_ERR_INVALID, "writing '%s' failed", path);
}
