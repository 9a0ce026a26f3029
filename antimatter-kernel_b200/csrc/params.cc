// params.json reader with the reference's keys and quirks
// (params/physics_params.cc:42-100, interaction_params.cc:30-47,
// stochastic_params.cc:13-24). A small recursive-descent JSON parser: the
// reference's nlohmann::json comes with BioDynaMo and is not a dependency
// here.
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "amk.h"

namespace amk {
int fail(int code, const char* fmt, ...);
}

namespace {

struct JValue {
  enum Kind { kNull, kBool, kNumber, kString, kObject, kArray } kind = kNull;
  bool b = false;
  double num = 0.0;
  std::string str;
  std::vector<std::pair<std::string, std::shared_ptr<JValue>>> obj;  // insertion order
  std::vector<std::shared_ptr<JValue>> arr;
  const JValue* get(const char* key) const {
    for (auto& kv : obj)
      if (kv.first == key) return kv.second.get();
    return nullptr;
  }
};

struct Parser {
  const std::string& s;
  size_t i = 0;
  bool ok = true;
  explicit Parser(const std::string& src) : s(src) {}
  void ws() {
    while (i < s.size() && std::isspace(static_cast<unsigned char>(s[i]))) ++i;
  }
  std::shared_ptr<JValue> value() {
    ws();
    auto v = std::make_shared<JValue>();
    if (i >= s.size()) {
      ok = false;
      return v;
    }
    const char ch = s[i];
    if (ch == '{') {
      v->kind = JValue::kObject;
      ++i;
      ws();
      if (i < s.size() && s[i] == '}') {
        ++i;
        return v;
      }
      while (ok) {
        ws();
        auto k = value();
        if (k->kind != JValue::kString) {
          ok = false;
          break;
        }
        ws();
        if (i >= s.size() || s[i] != ':') {
          ok = false;
          break;
        }
        ++i;
        auto val = value();
        v->obj.emplace_back(k->str, val);
        ws();
        if (i < s.size() && s[i] == ',') {
          ++i;
          continue;
        }
        if (i < s.size() && s[i] == '}') {
          ++i;
          break;
        }
        ok = false;
      }
    } else if (ch == '[') {
      v->kind = JValue::kArray;
      ++i;
      ws();
      if (i < s.size() && s[i] == ']') {
        ++i;
        return v;
      }
      while (ok) {
        v->arr.push_back(value());
        ws();
        if (i < s.size() && s[i] == ',') {
          ++i;
          continue;
        }
        if (i < s.size() && s[i] == ']') {
          ++i;
          break;
        }
        ok = false;
      }
    } else if (ch == '"') {
      v->kind = JValue::kString;
      ++i;
      while (i < s.size() && s[i] != '"') {
        if (s[i] == '\\' && i + 1 < s.size()) ++i;
        v->str.push_back(s[i++]);
      }
      if (i >= s.size()) ok = false;
      ++i;
    } else if (s.compare(i, 4, "true") == 0) {
      v->kind = JValue::kBool;
      v->b = true;
      i += 4;
    } else if (s.compare(i, 5, "false") == 0) {
      v->kind = JValue::kBool;
      i += 5;
    } else if (s.compare(i, 4, "null") == 0) {
      i += 4;
    } else {
      char* end = nullptr;
      v->num = std::strtod(s.c_str() + i, &end);
      if (end == s.c_str() + i) {
        ok = false;
        return v;
      }
      v->kind = JValue::kNumber;
      i = static_cast<size_t>(end - s.c_str());
    }
    return v;
  }
};

int species_from_name(const std::string& n) {  // physics_params.cc:14-22
  if (n == "antiproton") return AMK_ANTIPROTON;
  if (n == "positron") return AMK_POSITRON;
  if (n == "antihydrogen") return AMK_ANTIHYDROGEN;
  if (n == "electron") return AMK_ELECTRON;
  if (n == "proton") return AMK_PROTON;
  return -1;
}

int method_from_name(const std::string& n) {  // interaction_params.cc:14-28 + README spellings
  if (n == "standard") return AMK_METHOD_STANDARD;
  if (n == "barnes-hut" || n == "barnes_hut") return AMK_METHOD_BARNES_HUT;
  if (n == "fast-multipole" || n == "fast_multipole") return AMK_METHOD_FAST_MULTIPOLE;
  if (n == "allpairs" || n == "all-pairs") return AMK_METHOD_ALLPAIRS;
  return -1;
}

bool num(const JValue* v, double* out) {
  if (!v) return false;
  if (v->kind == JValue::kNumber) {
    *out = v->num;
    return true;
  }
  if (v->kind == JValue::kBool) {
    *out = v->b ? 1.0 : 0.0;
    return true;
  }
  return false;
}

}  // namespace

extern "C" int amk_params_load_json(const char* path, amk_params* p) {
  if (!path || !p) return amk::fail(AMK_ERR_INVALID, "null argument");
  std::ifstream f(path);
  if (!f.is_open()) return amk::fail(AMK_ERR_IO, "params file '%s' not found", path);
  std::stringstream ss;
  ss << f.rdbuf();
  const std::string src = ss.str();
  Parser parser(src);
  auto root = parser.value();
  if (!parser.ok || root->kind != JValue::kObject) return amk::fail(AMK_ERR_INVALID, "'%s' is not a JSON object", path);
  const JValue& j = *root;
  double d = 0.0;
  if (num(j.get("seed"), &d)) p->seed = static_cast<int>(d);
  if (num(j.get("b0"), &d)) p->b0 = d;
  if (num(j.get("trap_voltage"), &d)) p->trap_voltage = d;
  if (num(j.get("z0"), &d)) p->z0 = d;
  if (num(j.get("rho0"), &d)) p->rho0 = d;
  if (num(j.get("bath_temperature"), &d)) p->bath_temperature = d;
  if (num(j.get("cooling_scale"), &d)) p->cooling_scale = d;
  double mass_charge_ratio = 1e-6;
  if (const JValue* pops = j.get("particle_populations")) {
    if (pops->kind != JValue::kObject) return amk::fail(AMK_ERR_INVALID, "particle_populations must be an object");
    int n = 0;
    for (auto& kv : pops->obj) {
      const int s = species_from_name(kv.first);
      if (s < 0)
        return amk::fail(AMK_ERR_INVALID, "PhysicsParams::LoadParams: unrecognized species name '%s'", kv.first.c_str());
      if (n >= AMK_MAX_SPECIES) return amk::fail(AMK_ERR_LIMIT, "too many populations");
      double cnt = 0.0;
      if (!num(kv.second.get(), &cnt)) return amk::fail(AMK_ERR_INVALID, "population of '%s' is not a number", kv.first.c_str());
      p->species[n] = s;
      p->populations[n] = static_cast<long>(cnt);
      p->temperatures[n] = 0.0;
      ++n;
      double m = 0.0, q = 0.0;
      amk_species_properties(s, &m, &q);
      mass_charge_ratio = std::fmin(mass_charge_ratio, m / std::fabs(q));
    }
    p->n_species = n;
  }
  p->dt = (mass_charge_ratio * 3.14159265358979323846) / (p->b0 * 2);  // physics_params.cc:74
  if (const JValue* temps = j.get("particle_temperatures")) {
    for (auto& kv : temps->obj) {
      const int s = species_from_name(kv.first);
      if (s < 0)
        return amk::fail(AMK_ERR_INVALID, "PhysicsParams::LoadParams: unrecognized species name '%s'", kv.first.c_str());
      double t = 0.0;
      if (!num(kv.second.get(), &t)) return amk::fail(AMK_ERR_INVALID, "temperature of '%s' is not a number", kv.first.c_str());
      t = std::trunc(t);  // read as size_t in the reference (physics_params.cc:81)
      for (int k = 0; k < p->n_species; ++k)
        if (p->species[k] == s) p->temperatures[k] = t;
    }
  }
  if (num(j.get("num_steps"), &d)) p->num_steps = static_cast<long>(d);
  if (const JValue* r = j.get("initial_cloud_radii")) {
    if (num(r->get("radius_x"), &d)) p->cloud_radii[0] = d;
    if (num(r->get("radius_y"), &d)) p->cloud_radii[1] = d;
    if (num(r->get("radius_z"), &d)) p->cloud_radii[2] = d;
  }
  if (num(j.get("coulomb_forces_enabled"), &d)) p->coulomb_forces_enabled = d != 0.0;
  if (const JValue* m = j.get("coulomb_computation_method")) {
    const int k = method_from_name(m->str);
    if (k < 0) return amk::fail(AMK_ERR_INVALID, "InteractionParams: unrecognized coulomb_method '%s'", m->str.c_str());
    p->coulomb_method = k;
  }
  if (const JValue* m = j.get("energy_computation_method")) {
    const int k = method_from_name(m->str);
    if (k < 0) return amk::fail(AMK_ERR_INVALID, "InteractionParams: unrecognized energy_method '%s'", m->str.c_str());
    p->energy_method = k;
  }
  if (num(j.get("cutoff_radius"), &d)) p->cutoff_radius = d;
  if (num(j.get("barnes_hut_theta"), &d)) p->barnes_hut_theta = d;
  if (num(j.get("fast_multipole_order"), &d)) p->fast_multipole_order = d;
  if (num(j.get("fast_multipole_theta"), &d)) p->fast_multipole_theta = d;
  if (num(j.get("fmm_learned"), &d)) p->fmm_learned = d != 0.0;
  if (num(j.get("annihilation_enabled"), &d)) p->annihilation_enabled = d != 0.0;
  if (num(j.get("contact_radius"), &d)) p->contact_radius = d;
  if (num(j.get("annihilation_probability"), &d)) p->annihilation_probability = d;
  return AMK_OK;
}
