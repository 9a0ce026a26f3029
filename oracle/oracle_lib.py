"""ctypes access to the CPU oracle (TEST INFRASTRUCTURE ONLY).

Two libraries live here:

* ``liboracle.so`` -- the repository's FP64 restatement of the reference's
  per-step arithmetic (``amk_oracle.cc``), always buildable with g++.
* ``_ref/libamkref.so`` -- the reference's own ``barnes-hut.cc``,
  ``fast-multipole.cc`` and ``penning_trap.cc`` compiled in place from the
  reference tree (only where that tree exists; the built file travels with the
  repository copy otherwise).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline legs of
``bench.py`` import this module; the CUDA library never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libamkref.so")
REFERENCE_TREE = os.environ.get("AMK_REFERENCE_TREE", "/root/reference")

_dp = C.POINTER(C.c_double)
_u8p = C.POINTER(C.c_uint8)
_u32p = C.POINTER(C.c_uint32)
_lp = C.POINTER(C.c_long)
_ip = C.POINTER(C.c_int)


def build(ref: bool = True) -> None:
    """Compile the oracle (and, when the reference tree is present, _ref)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    if ref and os.path.isdir(os.path.join(REFERENCE_TREE, "src")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={REFERENCE_TREE}"], check=True)


def _ptr(a, t=_dp):
    if a is None:
        return None
    return a.ctypes.data_as(t)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build(ref=False)
        L = C.CDLL(ORACLE_SO)
        L.orc_dt.restype = C.c_double
        L.orc_cooling_time.restype = C.c_double
        L.orc_annihilation_uniform.restype = C.c_double
        L.orc_annihilation_uniform.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64]
        L.orc_annihilation.restype = C.c_long
        L.orc_cooling.argtypes = [C.c_long, _dp, _dp, _dp, _dp, _dp, _u8p, _u32p, C.c_double,
                                  C.c_double, C.c_double, C.c_double, C.c_uint32, C.c_uint64]
        L.orc_cooling_normals.argtypes = [C.c_uint32, C.c_uint32, C.c_uint64, _dp]
        L.orc_annihilation.argtypes = [C.c_long, _dp, _dp, _dp, _u8p, _u8p, _u32p, C.c_double,
                                       C.c_double, C.c_uint32, C.c_uint64]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            build(ref=True)
        R = C.CDLL(REF_SO)
        R.amkref_bh_tree.restype = C.c_long
        _ref = R
    return _ref


# ----------------------------------------------------------------- species
SPECIES = {"antiproton": 0, "positron": 1, "antihydrogen": 2, "electron": 3,
           "proton": 4, "antihelium": 5}


def species_props(species):
    s = np.asarray(species)
    m = np.empty(s.shape, np.float64)
    q = np.empty(s.shape, np.float64)
    mm, qq = C.c_double(), C.c_double()
    table = {}
    for v in np.unique(s):
        lib().orc_species_props(int(v), C.byref(mm), C.byref(qq))
        table[int(v)] = (mm.value, qq.value)
    for v, (a, b) in table.items():
        m[s == v] = a
        q[s == v] = b
    return m, q


def dt_for(species_list, b0):
    arr = np.asarray(species_list, np.int32)
    return lib().orc_dt(len(arr), _ptr(arr, _ip), C.c_double(b0))


# ----------------------------------------------------------------- forces
def allpairs(x, y, z, q, alive=None, want_phi=False):
    x, y, z, q = map(_f64, (x, y, z, q))
    n = len(x)
    fx, fy, fz = np.zeros(n), np.zeros(n), np.zeros(n)
    phi = np.zeros(n) if want_phi else None
    al = None if alive is None else np.ascontiguousarray(alive, np.uint8)
    lib().orc_allpairs(C.c_long(n), _ptr(x), _ptr(y), _ptr(z), _ptr(q), _ptr(al, _u8p),
                       _ptr(fx), _ptr(fy), _ptr(fz), _ptr(phi))
    return (fx, fy, fz, phi) if want_phi else (fx, fy, fz)


def allpairs_subset(x, y, z, q, targets):
    x, y, z, q = map(_f64, (x, y, z, q))
    t = np.ascontiguousarray(targets, np.int64)
    k = len(t)
    fx, fy, fz = np.zeros(k), np.zeros(k), np.zeros(k)
    lib().orc_allpairs_subset(C.c_long(len(x)), _ptr(x), _ptr(y), _ptr(z), _ptr(q), C.c_long(k),
                              _ptr(t, _lp), _ptr(fx), _ptr(fy), _ptr(fz))
    return fx, fy, fz


def cutoff(x, y, z, q, rc, alive=None):
    x, y, z, q = map(_f64, (x, y, z, q))
    n = len(x)
    fx, fy, fz = np.zeros(n), np.zeros(n), np.zeros(n)
    al = None if alive is None else np.ascontiguousarray(alive, np.uint8)
    lib().orc_cutoff(C.c_long(n), _ptr(x), _ptr(y), _ptr(z), _ptr(q), _ptr(al, _u8p),
                     C.c_double(rc), _ptr(fx), _ptr(fy), _ptr(fz))
    return fx, fy, fz


# ----------------------------------------------------------------- push
def boris_push(state, fx, fy, fz, b0, voltage, z0, rho0, dt, stagger):
    """In-place Boris push of ``state`` (dict of float64 arrays)."""
    s = state
    fx, fy, fz = _f64(fx).copy(), _f64(fy).copy(), _f64(fz).copy()
    al = s.get("alive")
    lib().orc_boris_push(C.c_long(len(s["x"])), _ptr(s["x"]), _ptr(s["y"]), _ptr(s["z"]),
                         _ptr(s["vx"]), _ptr(s["vy"]), _ptr(s["vz"]), _ptr(fx), _ptr(fy),
                         _ptr(fz), _ptr(s["q"]), _ptr(s["m"]), _ptr(al, _u8p), C.c_double(b0),
                         C.c_double(voltage), C.c_double(z0), C.c_double(rho0), C.c_double(dt),
                         C.c_int(1 if stagger else 0))


def cooling(state, b0, dt, tau_scale, bath_temp, seed, step, ids=None):
    s = state
    n = len(s["x"])
    ids = np.arange(n, dtype=np.uint32) if ids is None else np.ascontiguousarray(ids, np.uint32)
    al = s.get("alive")
    lib().orc_cooling(n, _ptr(s["vx"]), _ptr(s["vy"]), _ptr(s["vz"]), _ptr(s["q"]), _ptr(s["m"]),
                      _ptr(al, _u8p), _ptr(ids, _u32p), b0, dt, tau_scale, bath_temp, seed, step)


def cooling_time(q, m, b):
    return lib().orc_cooling_time(C.c_double(q), C.c_double(m), C.c_double(b))


def annihilation(state, contact_radius, probability, seed, step, ids=None):
    s = state
    n = len(s["x"])
    ids = np.arange(n, dtype=np.uint32) if ids is None else np.ascontiguousarray(ids, np.uint32)
    return lib().orc_annihilation(n, _ptr(s["x"]), _ptr(s["y"]), _ptr(s["z"]),
                                  _ptr(s["species"], _u8p), _ptr(s["alive"], _u8p),
                                  _ptr(ids, _u32p), contact_radius, probability, seed, step)


def energy_standard(state, voltage, z0, rho0, cutoff_radius):
    s = state
    out = np.zeros(4)
    lib().orc_energy_standard(C.c_long(len(s["x"])), _ptr(s["x"]), _ptr(s["y"]), _ptr(s["z"]),
                              _ptr(s["vx"]), _ptr(s["vy"]), _ptr(s["vz"]), _ptr(s["q"]),
                              _ptr(s["m"]), _ptr(s.get("alive"), _u8p), C.c_double(voltage),
                              C.c_double(z0), C.c_double(rho0), C.c_double(cutoff_radius),
                              _ptr(out))
    return {"kinetic": out[0], "trap_potential": out[1], "coulomb_potential": out[2],
            "num_active": int(out[3])}


def philox4x32(k0, k1, ctr):
    c = np.ascontiguousarray(ctr, np.uint32)
    out = np.zeros(4, np.uint32)
    lib().orc_philox4x32(C.c_uint32(k0), C.c_uint32(k1), _ptr(c, _u32p), _ptr(out, _u32p))
    return out


# ----------------------------------------------------------------- ICs
def _species_arrays(populations):
    sp = np.array([SPECIES[k] if isinstance(k, str) else int(k) for k in populations], np.int32)
    cnt = np.array(list(populations.values()), np.int64)
    return sp, cnt


def initial_positions(populations, radii, seed, use_ref=False):
    sp, cnt = _species_arrays(populations)
    out = np.zeros((int(cnt.sum()), 3))
    r = _f64(radii)
    f = ref().amkref_initial_positions if use_ref else lib().orc_initial_positions
    f(C.c_int(len(sp)), _ptr(sp, _ip), _ptr(cnt, _lp), _ptr(r), C.c_int(seed), _ptr(out))
    return out


def initial_velocities(populations, temperatures, seed, use_ref=False):
    sp, cnt = _species_arrays(populations)
    temps = _f64([temperatures.get(k, 0.0) for k in populations])
    out = np.zeros((int(cnt.sum()), 3))
    f = ref().amkref_initial_velocities if use_ref else lib().orc_initial_velocities
    f(C.c_int(len(sp)), _ptr(sp, _ip), _ptr(cnt, _lp), _ptr(temps), C.c_int(seed), _ptr(out))
    return out


def species_column(populations):
    """Species per particle in the reference's creation order (enum order)."""
    sp, cnt = _species_arrays(populations)
    order = np.argsort(sp, kind="stable")
    return np.concatenate([np.full(cnt[k], sp[k], np.uint8) for k in order])


# ----------------------------------------------------------------- reference solvers
def ref_bh_forces(x, y, z, q, theta, leaf_capacity=8):
    x, y, z, q = map(_f64, (x, y, z, q))
    n = len(x)
    fx, fy, fz = np.zeros(n), np.zeros(n), np.zeros(n)
    ref().amkref_bh_forces(C.c_long(n), _ptr(x), _ptr(y), _ptr(z), _ptr(q), C.c_double(theta),
                           C.c_long(leaf_capacity), _ptr(fx), _ptr(fy), _ptr(fz))
    return fx, fy, fz


def ref_bh_forces_subset(x, y, z, q, theta, targets, leaf_capacity=8):
    x, y, z, q = map(_f64, (x, y, z, q))
    t = np.ascontiguousarray(targets, np.int64)
    k = len(t)
    fx, fy, fz = np.zeros(k), np.zeros(k), np.zeros(k)
    ref().amkref_bh_forces_subset(C.c_long(len(x)), _ptr(x), _ptr(y), _ptr(z), _ptr(q),
                                  C.c_double(theta), C.c_long(leaf_capacity), C.c_long(k),
                                  _ptr(t, _lp), _ptr(fx), _ptr(fy), _ptr(fz), None)
    return fx, fy, fz


def ref_bh_potentials(x, y, z, q, theta, leaf_capacity=8):
    x, y, z, q = map(_f64, (x, y, z, q))
    n = len(x)
    phi = np.zeros(n)
    ref().amkref_bh_potentials(C.c_long(n), _ptr(x), _ptr(y), _ptr(z), _ptr(q), C.c_double(theta),
                               C.c_long(leaf_capacity), _ptr(phi))
    return phi


def ref_bh_tree(x, y, z, q, leaf_capacity=8):
    x, y, z, q = map(_f64, (x, y, z, q))
    n = len(x)
    cap = 4 * n + 64
    f = np.zeros((cap, 12))
    g = np.zeros((cap, 11), np.int64)
    order = np.zeros(n, np.int64)
    nn = ref().amkref_bh_tree(C.c_long(n), _ptr(x), _ptr(y), _ptr(z), _ptr(q),
                              C.c_long(leaf_capacity), C.c_long(cap), _ptr(f), _ptr(g, _lp),
                              _ptr(order, _lp))
    assert nn >= 0
    return f[:nn], g[:nn], order


def ref_driver(method, x, y, z, q, alive, theta, order=0):
    """The reference's own drop-in drivers on ChargedAntiparticle agents:
    method "barnes-hut" (ComputeBarnesHutCoulombForces, barnes-hut.cc:271-299)
    or "fast-multipole" (ComputeFastMultipoleCoulombForces,
    fast-multipole.cc:682-709). Annihilated agents keep a zero force slot."""
    x, y, z, q = map(_f64, (x, y, z, q))
    n = len(x)
    al = np.ascontiguousarray(alive, np.uint8)
    fx, fy, fz = np.zeros(n), np.zeros(n), np.zeros(n)
    if method == "barnes-hut":
        ref().amkref_compute_barnes_hut_coulomb_forces(C.c_long(n), _ptr(x), _ptr(y), _ptr(z), _ptr(q),
                                                       _ptr(al, _u8p), C.c_double(theta), _ptr(fx), _ptr(fy),
                                                       _ptr(fz))
    else:
        ref().amkref_compute_fast_multipole_coulomb_forces(C.c_long(n), _ptr(x), _ptr(y), _ptr(z), _ptr(q),
                                                           _ptr(al, _u8p), C.c_int(order), C.c_double(theta),
                                                           _ptr(fx), _ptr(fy), _ptr(fz))
    return fx, fy, fz


def ref_fmm(x, y, z, q, order, theta, leaf_capacity=32, forces=True, energy=False):
    x, y, z, q = map(_f64, (x, y, z, q))
    n = len(x)
    fx = fy = fz = None
    if forces:
        fx, fy, fz = np.zeros(n), np.zeros(n), np.zeros(n)
    e = C.c_double(0.0)
    ref().amkref_fmm(C.c_long(n), _ptr(x), _ptr(y), _ptr(z), _ptr(q), C.c_int(order),
                     C.c_double(theta), C.c_long(leaf_capacity), _ptr(fx), _ptr(fy), _ptr(fz),
                     C.byref(e) if energy else None)
    return (fx, fy, fz), (e.value if energy else None)


# ----------------------------------------------------------------- reference behaviours
class RefWorld:
    """The reference's own per-agent code (lorentz.cc, cooling.cc,
    annihilation.cc, coulomb_interaction.cc via oracle/_ref) on stand-in
    agents: uid = index; each step runs the behaviours phase by phase over
    agents in ascending uid order, with the stand-in Random replaying the CUDA
    library's Philox draws (see ref_behaviours.cc)."""

    def __init__(self, pos, vel, species, b0, voltage, z0, rho0, dt, cooling_scale=0.0, bath_temp=0.0,
                 annihilation=False, contact_radius=0.0, probability=0.0, seed=0):
        R = ref()
        R.amkref_world_create.restype = C.c_void_p
        R.amkref_world_behaviours.restype = C.c_long
        R.amkref_world_behaviours.argtypes = [C.c_void_p, C.c_uint64, C.c_int, C.c_int, C.c_int]
        R.amkref_world_destroy.argtypes = [C.c_void_p]
        R.amkref_cooling_time.restype = C.c_double
        pos = np.ascontiguousarray(pos, np.float64)
        vel = np.ascontiguousarray(vel, np.float64)
        self.n = len(pos)
        x, y, z = (np.ascontiguousarray(pos[:, k]) for k in range(3))
        vx, vy, vz = (np.ascontiguousarray(vel[:, k]) for k in range(3))
        sp = np.ascontiguousarray(species, np.uint8)
        self._h = R.amkref_world_create(
            C.c_long(self.n), _ptr(x), _ptr(y), _ptr(z), _ptr(vx), _ptr(vy), _ptr(vz), _ptr(sp, _u8p),
            C.c_double(b0), C.c_double(voltage), C.c_double(z0), C.c_double(rho0), C.c_double(dt),
            C.c_double(cooling_scale), C.c_double(bath_temp), C.c_int(1 if annihilation else 0),
            C.c_double(contact_radius), C.c_double(probability), C.c_uint32(seed))
        self.h = C.c_void_p(self._h)

    def close(self):
        if self._h:
            ref().amkref_world_destroy(self.h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_alive(self, alive):
        a = np.ascontiguousarray(alive, np.uint8)
        ref().amkref_world_set_alive(self.h, _ptr(a, _u8p))

    def set_forces(self, fx, fy, fz):
        fx, fy, fz = map(_f64, (fx, fy, fz))
        ref().amkref_world_set_forces(self.h, _ptr(fx), _ptr(fy), _ptr(fz))

    def coulomb_standard(self, cutoff):
        ref().amkref_world_coulomb_standard(self.h, C.c_double(cutoff))

    def behaviours(self, step, lorentz=True, cooling=True, annihilation=True):
        return ref().amkref_world_behaviours(self.h, int(step), int(lorentz), int(cooling), int(annihilation))

    def state(self):
        n = self.n
        arr = {k: np.zeros(n) for k in ("x", "y", "z", "vx", "vy", "vz", "fx", "fy", "fz")}
        alive = np.zeros(n, np.uint8)
        ref().amkref_world_get(self.h, *[_ptr(arr[k]) for k in ("x", "y", "z", "vx", "vy", "vz")],
                               _ptr(alive, _u8p), *[_ptr(arr[k]) for k in ("fx", "fy", "fz")])
        arr["alive"] = alive
        return arr


def ref_cooling_time(charge, mass, b_mag):
    ref().amkref_cooling_time.restype = C.c_double
    return ref().amkref_cooling_time(C.c_double(charge), C.c_double(mass), C.c_double(b_mag))


def ref_is_antiparticle_pair(a, b):
    return bool(ref().amkref_is_antiparticle_pair(int(a), int(b)))
