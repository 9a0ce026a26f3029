"""Python host side of the B200 antimatter-kernel particle path.

A thin ctypes layer over ``libamk.so`` (the C ABI declared in
``include/amk.h``). It mirrors the reference's interfaces:

* ``Simulation``: the context (particles resident in HBM) with the driver's
  per-step order -- Coulomb solver, LorentzForce + CyclotronCooling,
  AnnihilationInteraction (src/antimatter-kernel.cc:153-162);
* ``compute_standard_coulomb_forces`` / ``compute_barnes_hut_coulomb_forces``
  / ``compute_fast_multipole_coulomb_forces``: the three drop-in solver
  functions (coulomb_interaction.h:10, barnes-hut.h:76, fast-multipole.h:73);
* ``BarnesHutTree`` and ``FastMultipoleSolver``: the solver classes
  (barnes-hut.h:28-74, fast-multipole.h:46-71);
* ``load_params``: params.json with the reference's keys.

There is no CPU path: every call runs the CUDA library, and loading fails
loudly when the library or a GPU is missing.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "libamk.so")

AMK_OK = 0
ERRORS = {-1: "invalid", -2: "cuda", -3: "nomem", -4: "state", -5: "timeout",
          -6: "unsupported", -7: "limit", -8: "io"}

METHOD = {"standard": 0, "barnes-hut": 1, "barnes_hut": 1, "fast-multipole": 2,
          "fast_multipole": 2, "allpairs": 3}
SPECIES = {"antiproton": 0, "positron": 1, "antihydrogen": 2, "electron": 3,
           "proton": 4, "antihelium": 5}

CLOUD = {"uniform": 0, "gaussian": 1}
PHASES = ["stage", "allpairs", "cutoff", "sort", "tree", "bh_walk", "fmm_up", "fmm_lists",
          "fmm_m2l", "fmm_down", "fmm_p2p", "mlp", "push", "annihilation", "energy", "fmm_m2l_products",
          "fmm_near"]


class AmkError(RuntimeError):
    pass


class Params(C.Structure):
    """Mirror of ``amk_params`` (include/amk.h)."""
    _fields_ = [
        ("seed", C.c_int), ("b0", C.c_double), ("trap_voltage", C.c_double),
        ("z0", C.c_double), ("rho0", C.c_double), ("dt", C.c_double),
        ("num_steps", C.c_long), ("bath_temperature", C.c_double),
        ("cooling_scale", C.c_double), ("cooling_enabled", C.c_int),
        ("coulomb_forces_enabled", C.c_int), ("coulomb_method", C.c_int),
        ("energy_method", C.c_int), ("cutoff_radius", C.c_double),
        ("barnes_hut_theta", C.c_double), ("fast_multipole_order", C.c_double),
        ("fast_multipole_theta", C.c_double), ("fmm_learned", C.c_int),
        ("annihilation_enabled", C.c_int), ("contact_radius", C.c_double),
        ("annihilation_probability", C.c_double), ("n_species", C.c_int),
        ("species", C.c_int * 6), ("populations", C.c_long * 6),
        ("temperatures", C.c_double * 6), ("cloud_radii", C.c_double * 3),
        ("learned_audit_interval", C.c_long), ("learned_error_budget", C.c_double),
        ("learned_fallback_order", C.c_int), ("learned_audit_samples", C.c_long),
    ]


class TuneCandidate(C.Structure):
    _fields_ = [("method", C.c_int), ("order", C.c_int), ("theta", C.c_double), ("leaf", C.c_int),
                ("ms", C.c_double), ("rms", C.c_double), ("meets", C.c_int)]


class EnergyOut(C.Structure):
    _fields_ = [("kinetic", C.c_double), ("trap_potential", C.c_double),
                ("coulomb_potential", C.c_double), ("total", C.c_double),
                ("num_active", C.c_long)]


_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_u8p = C.POINTER(C.c_uint8)
_lib = None


def build() -> None:
    """Compile libamk.so for sm_100a in-tree (needs nvcc, no GPU)."""
    subprocess.run(["make", "-s", "-j8", "-C", PKG_DIR], check=True)


def lib():
    """The loaded CUDA library (built on first use when absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    sig = {
        "amk_params_default": (C.c_int, [C.POINTER(Params)]),
        "amk_params_load_json": (C.c_int, [C.c_char_p, C.POINTER(Params)]),
        "amk_params_validate": (C.c_int, [C.POINTER(Params), C.c_int]),
        "amk_dt_for_species": (C.c_double, [C.c_int, C.POINTER(C.c_int), C.c_double]),
        "amk_species_properties": (C.c_int, [C.c_int, _dp, _dp]),
        "amk_trap_dimension": (C.c_double, [C.c_double, C.c_double]),
        "amk_cooling_time": (C.c_double, [C.c_double, C.c_double, C.c_double]),
        "amk_create": (C.c_int, [C.POINTER(Params), C.c_int, C.POINTER(vp)]),
        "amk_destroy": (C.c_int, [vp]),
        "amk_last_error": (C.c_char_p, []),
        "amk_set_stream": (C.c_int, [vp, vp]),
        "amk_get_stream": (C.c_int, [vp, C.POINTER(vp)]),
        "amk_synchronize": (C.c_int, [vp]),
        "amk_set_params": (C.c_int, [vp, C.POINTER(Params)]),
        "amk_get_params": (C.c_int, [vp, C.POINTER(Params)]),
        "amk_set_particles": (C.c_int, [vp, C.c_long, _dp, _dp, _dp, _dp, _dp, _dp, _u8p]),
        "amk_set_particles_device": (C.c_int, [vp, C.c_long, vp, vp, vp, vp, vp, vp, vp]),
        "amk_set_charge_mass": (C.c_int, [vp, _dp, _dp]),
        "amk_update_state": (C.c_int, [vp, vp, vp, vp, vp, vp, vp]),
        "amk_measure_fp32_peak": (C.c_int, [vp, _dp, _dp]),
        "amk_measure_fp64_peak": (C.c_int, [vp, _dp, _dp]),
        "amk_init_particles": (C.c_int, [vp]),
        "amk_get_particles": (C.c_int, [vp, _dp, _dp, _dp, _dp, _dp, _dp, _u8p]),
        "amk_get_particles_device": (C.c_int, [vp, vp, vp, vp, vp, vp, vp, vp]),
        "amk_num_particles": (C.c_long, [vp]),
        "amk_num_alive": (C.c_long, [vp]),
        "amk_coulomb_standard": (C.c_int, [vp, C.c_double]),
        "amk_coulomb_allpairs": (C.c_int, [vp]),
        "amk_coulomb_barnes_hut": (C.c_int, [vp, C.c_double]),
        "amk_coulomb_fmm": (C.c_int, [vp, C.c_int, C.c_double, C.c_int]),
        "amk_coulomb": (C.c_int, [vp]),
        "amk_get_forces": (C.c_int, [vp, _dp, _dp, _dp]),
        "amk_push": (C.c_int, [vp]),
        "amk_annihilate": (C.c_int, [vp, C.POINTER(C.c_long)]),
        "amk_step": (C.c_int, [vp, C.c_int]),
        "amk_step_count": (C.c_long, [vp]),
        "amk_energy": (C.c_int, [vp, C.c_int, C.POINTER(EnergyOut)]),
        "amk_solve_allpairs": (C.c_int, [vp, C.c_long, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]),
        "amk_solve_cutoff": (C.c_int, [vp, C.c_long, _dp, _dp, _dp, _dp, C.c_double, _dp, _dp, _dp]),
        "amk_solve_barnes_hut": (C.c_int, [vp, C.c_long, _dp, _dp, _dp, _dp, C.c_double, C.c_long,
                                           _dp, _dp, _dp, _dp]),
        "amk_solve_fmm": (C.c_int, [vp, C.c_long, _dp, _dp, _dp, _dp, C.c_int, C.c_double, C.c_long,
                                    _dp, _dp, _dp, _dp]),
        "amk_bh_tree_dump": (C.c_long, [vp, C.c_long, _dp, _dp, _dp, _dp, C.c_long, C.c_long, _dp,
                                        C.POINTER(C.c_long)]),
        "amk_fmm_stats": (C.c_int, [vp, C.POINTER(C.c_long), C.c_int]),
        "amk_fmm_train_correction": (C.c_int, [vp, C.c_double, C.c_int, C.c_int, C.c_long, C.c_float, _fp,
                                                C.POINTER(C.c_long)]),
        "amk_fmm_audit": (C.c_int, [vp, C.c_int, C.c_double, C.c_int, C.c_long, _dp]),
        "amk_fmm_learned_state": (C.c_int, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), _dp]),
        "amk_mlp_num_params": (C.c_int, []),
        "amk_mlp_set_params": (C.c_int, [vp, _fp, C.c_long]),
        "amk_mlp_get_params": (C.c_int, [vp, _fp, C.c_long]),
        "amk_mlp_forward": (C.c_int, [vp, _fp, C.c_long, _fp]),
        "amk_mlp_gradients": (C.c_int, [vp, _fp, _fp, C.c_long, _fp, _fp, _fp]),
        "amk_mlp_train": (C.c_int, [vp, _fp, _fp, C.c_long, C.c_int, C.c_long, C.c_float, _fp]),
        "amk_force_error": (C.c_int, [vp, C.c_long, _dp, _dp]),
        "amk_set_leaf_sizes": (C.c_int, [vp, C.c_int, C.c_int]),
        "amk_get_leaf_sizes": (C.c_int, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "amk_autotune": (C.c_int, [vp, C.c_double, C.c_long, C.c_int, C.POINTER(TuneCandidate), C.c_int,
                                   C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "amk_batch_set": (C.c_int, [vp, C.c_int, C.POINTER(Params), C.POINTER(C.c_long)]),
        "amk_batch_step": (C.c_int, [vp, C.c_int, C.c_int, C.c_int]),
        "amk_batch_coulomb": (C.c_int, [vp]),
        "amk_batch_energy": (C.c_int, [vp, C.c_int, C.POINTER(EnergyOut)]),
        "amk_batch_autotune": (C.c_int, [vp, C.c_double, C.c_long, C.POINTER(C.c_int)]),
        "amk_batch_status": (C.c_int, [vp, C.POINTER(C.c_int), C.POINTER(C.c_long)]),
        "amk_batch_info": (C.c_int, [vp, C.POINTER(C.c_long), C.POINTER(C.c_long), C.POINTER(C.c_int)]),
        "amk_set_profiling": (C.c_int, [vp, C.c_int]),
        "amk_phase_times": (C.c_int, [vp, _dp, C.POINTER(C.c_long), C.c_int]),
        "amk_reset_phase_times": (C.c_int, [vp]),
        "amk_kernel_launches": (C.c_long, [vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return _lib


def check(rc: int, what: str = "") -> None:
    if rc != AMK_OK:
        msg = lib().amk_last_error().decode(errors="replace")
        raise AmkError(f"{what}: {ERRORS.get(rc, rc)}: {msg}")


def _d(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# ------------------------------------------------------------------ params
def default_params() -> Params:
    p = Params()
    check(lib().amk_params_default(C.byref(p)), "amk_params_default")
    return p


def load_params(path: str, base: Params | None = None) -> Params:
    """params.json with the reference's keys (physics/interaction/stochastic)."""
    p = base if base is not None else default_params()
    check(lib().amk_params_load_json(path.encode(), C.byref(p)), "amk_params_load_json")
    return p


def validate_params(p: Params, strict: bool = True) -> None:
    check(lib().amk_params_validate(C.byref(p), 1 if strict else 0), "amk_params_validate")


def make_params(**kw) -> Params:
    """Params from keyword arguments; ``populations``/``temperatures`` are
    dicts by species name, ``cloud_radii`` a 3-sequence, methods by name."""
    p = default_params()
    pops = kw.pop("populations", None)
    temps = kw.pop("temperatures", {})
    radii = kw.pop("cloud_radii", None)
    for key in ("coulomb_method", "energy_method"):
        if key in kw and isinstance(kw[key], str):
            kw[key] = METHOD[kw[key]]
    dt_given = "dt" in kw
    for k, v in kw.items():
        setattr(p, k, v)
    if pops is not None:
        p.n_species = len(pops)
        for i, (name, cnt) in enumerate(pops.items()):
            sp = SPECIES[name] if isinstance(name, str) else int(name)
            p.species[i] = sp
            p.populations[i] = int(cnt)
            p.temperatures[i] = float(temps.get(name, 0.0))
        if not dt_given:
            arr = (C.c_int * p.n_species)(*[p.species[i] for i in range(p.n_species)])
            p.dt = lib().amk_dt_for_species(p.n_species, arr, p.b0)
    if radii is not None:
        for i in range(3):
            p.cloud_radii[i] = float(radii[i])
    return p


def species_properties(species: int):
    m, q = C.c_double(), C.c_double()
    check(lib().amk_species_properties(int(species), C.byref(m), C.byref(q)))
    return m.value, q.value


# ------------------------------------------------------------------ context
class Simulation:
    """A context on one GPU holding the particle state in HBM."""

    def __init__(self, params: Params | None = None, device: int = 0):
        self._h = C.c_void_p()
        p = params if params is not None else default_params()
        check(lib().amk_create(C.byref(p), int(device), C.byref(self._h)), "amk_create")

    def close(self):
        if self._h:
            lib().amk_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    # -- params
    @property
    def params(self) -> Params:
        p = Params()
        check(lib().amk_get_params(self._h, C.byref(p)))
        return p

    @params.setter
    def params(self, p: Params):
        check(lib().amk_set_params(self._h, C.byref(p)))

    # -- streams
    def set_stream(self, stream_ptr: int | None):
        check(lib().amk_set_stream(self._h, C.c_void_p(stream_ptr or 0)))

    def stream(self) -> int:
        s = C.c_void_p()
        check(lib().amk_get_stream(self._h, C.byref(s)))
        return s.value or 0

    def synchronize(self):
        check(lib().amk_synchronize(self._h), "amk_synchronize")

    # -- particles
    def set_particles(self, x, y, z, vx, vy, vz, species):
        x, y, z, vx, vy, vz = map(_f64, (x, y, z, vx, vy, vz))
        sp = np.ascontiguousarray(species, np.uint8)
        check(lib().amk_set_particles(self._h, len(x), _d(x), _d(y), _d(z), _d(vx), _d(vy), _d(vz),
                                      sp.ctypes.data_as(_u8p)), "amk_set_particles")

    def set_particles_device(self, n, x, y, z, vx, vy, vz, species):
        """Device pointers (ints), e.g. torch ``tensor.data_ptr()``."""
        check(lib().amk_set_particles_device(self._h, int(n), x, y, z, vx, vy, vz, species),
              "amk_set_particles_device")

    def update_state(self, x, y, z, vx, vy, vz):
        """Host arrays (numpy float64, or host pointers as ints) overwrite x, v."""
        keep = [a if isinstance(a, int) else _f64(a) for a in (x, y, z, vx, vy, vz)]
        ptrs = [a if isinstance(a, int) else a.ctypes.data for a in keep]
        check(lib().amk_update_state(self._h, *[C.c_void_p(p) for p in ptrs]), "amk_update_state")
        del keep

    def measure_fp32_peak(self):
        t, ms = C.c_double(), C.c_double()
        check(lib().amk_measure_fp32_peak(self._h, C.byref(t), C.byref(ms)), "amk_measure_fp32_peak")
        return t.value

    def measure_fp64_peak(self):
        """FP64 tensor-pipe throughput in TFLOP/s (probe kernel)."""
        t, ms = C.c_double(), C.c_double()
        check(lib().amk_measure_fp64_peak(self._h, C.byref(t), C.byref(ms)), "amk_measure_fp64_peak")
        return t.value

    def set_charge_mass(self, charge=None, mass=None):
        q = None if charge is None else _f64(charge)
        m = None if mass is None else _f64(mass)
        check(lib().amk_set_charge_mass(self._h, _d(q), _d(m)))

    def init_particles(self):
        check(lib().amk_init_particles(self._h), "amk_init_particles")

    def init_particles_gpu(self, distribution: str = "uniform"):
        """The context's cloud generated on the GPU ("uniform" ellipsoid or
        "gaussian"); Philox draws, not the reference's std:: streams."""
        check(lib().amk_init_particles_gpu(self._h, CLOUD[distribution]), "amk_init_particles_gpu")

    def batch_init(self, params, distribution: str = "uniform"):
        """Generates every instance's cloud on the GPU and sets the batch."""
        arr = (Params * len(params))(*params)
        check(lib().amk_batch_init_particles(self._h, len(params), arr, CLOUD[distribution]),
              "amk_batch_init_particles")
        self._batch_n = len(params)

    def num_particles(self) -> int:
        return int(lib().amk_num_particles(self._h))

    def num_alive(self) -> int:
        n = int(lib().amk_num_alive(self._h))
        if n < 0:
            check(n, "amk_num_alive")
        return n

    def get_particles(self):
        n = self.num_particles()
        arrs = [np.empty(n) for _ in range(6)]
        alive = np.empty(n, np.uint8)
        check(lib().amk_get_particles(self._h, *[_d(a) for a in arrs], alive.ctypes.data_as(_u8p)))
        return dict(zip(["x", "y", "z", "vx", "vy", "vz"], arrs), alive=alive)

    def get_particles_device(self, x, y, z, vx, vy, vz, alive):
        check(lib().amk_get_particles_device(self._h, x, y, z, vx, vy, vz, alive))

    # -- forces
    def coulomb_standard(self, cutoff):
        check(lib().amk_coulomb_standard(self._h, float(cutoff)), "amk_coulomb_standard")

    def coulomb_allpairs(self):
        check(lib().amk_coulomb_allpairs(self._h), "amk_coulomb_allpairs")

    def coulomb_barnes_hut(self, theta):
        check(lib().amk_coulomb_barnes_hut(self._h, float(theta)), "amk_coulomb_barnes_hut")

    def coulomb_fmm(self, order, theta, learned=False):
        check(lib().amk_coulomb_fmm(self._h, int(order), float(theta), 1 if learned else 0),
              "amk_coulomb_fmm")

    def coulomb(self):
        check(lib().amk_coulomb(self._h), "amk_coulomb")

    def get_forces(self):
        n = self.num_particles()
        f = [np.empty(n) for _ in range(3)]
        check(lib().amk_get_forces(self._h, *[_d(a) for a in f]))
        return tuple(f)

    # -- behaviours
    def push(self):
        check(lib().amk_push(self._h), "amk_push")

    def annihilate(self) -> int:
        m = C.c_long(0)
        check(lib().amk_annihilate(self._h, C.byref(m)), "amk_annihilate")
        return m.value

    def step(self, n: int = 1):
        check(lib().amk_step(self._h, int(n)), "amk_step")

    def step_count(self) -> int:
        return int(lib().amk_step_count(self._h))

    def energy(self, time_centre: bool = True) -> dict:
        e = EnergyOut()
        check(lib().amk_energy(self._h, 1 if time_centre else 0, C.byref(e)), "amk_energy")
        return {"kinetic": e.kinetic, "trap_potential": e.trap_potential,
                "coulomb_potential": e.coulomb_potential, "total": e.total,
                "num_active": e.num_active}

    # -- profiling
    def set_profiling(self, on: bool):
        check(lib().amk_set_profiling(self._h, 1 if on else 0))

    def phase_times(self):
        ms = (C.c_double * len(PHASES))()
        cnt = (C.c_long * len(PHASES))()
        check(lib().amk_phase_times(self._h, ms, cnt, len(PHASES)))
        return {PHASES[k]: (ms[k], cnt[k]) for k in range(len(PHASES))}

    def reset_phase_times(self):
        check(lib().amk_reset_phase_times(self._h))

    def kernel_launches(self) -> int:
        return int(lib().amk_kernel_launches(self._h))

    # -- stateless solver mirrors
    def solve_allpairs(self, x, y, z, q, want_phi=False):
        x, y, z, q = map(_f64, (x, y, z, q))
        n = len(x)
        fx, fy, fz = np.empty(n), np.empty(n), np.empty(n)
        phi = np.empty(n) if want_phi else None
        check(lib().amk_solve_allpairs(self._h, n, _d(x), _d(y), _d(z), _d(q), _d(fx), _d(fy), _d(fz),
                                       _d(phi)), "amk_solve_allpairs")
        return (fx, fy, fz, phi) if want_phi else (fx, fy, fz)

    def solve_cutoff(self, x, y, z, q, cutoff):
        x, y, z, q = map(_f64, (x, y, z, q))
        n = len(x)
        fx, fy, fz = np.empty(n), np.empty(n), np.empty(n)
        check(lib().amk_solve_cutoff(self._h, n, _d(x), _d(y), _d(z), _d(q), float(cutoff), _d(fx),
                                     _d(fy), _d(fz)), "amk_solve_cutoff")
        return fx, fy, fz

    def solve_barnes_hut(self, x, y, z, q, theta, leaf_capacity=8, want_phi=False):
        x, y, z, q = map(_f64, (x, y, z, q))
        n = len(x)
        fx, fy, fz = np.empty(n), np.empty(n), np.empty(n)
        phi = np.empty(n) if want_phi else None
        check(lib().amk_solve_barnes_hut(self._h, n, _d(x), _d(y), _d(z), _d(q), float(theta),
                                         int(leaf_capacity), _d(fx), _d(fy), _d(fz), _d(phi)),
              "amk_solve_barnes_hut")
        return (fx, fy, fz, phi) if want_phi else (fx, fy, fz)

    def fmm_stats(self):
        out = (C.c_long * 11)()
        check(lib().amk_fmm_stats(self._h, out, 11))
        keys = ("cells", "leaves", "m2l_pairs", "p2p_leaf_pairs", "p2p_particle_pairs", "depth",
                "sources", "order", "m2l_class_pairs", "m2l_classes", "m2l_chunks")
        return dict(zip(keys, list(out)))

    # -- learned FMM correction
    def fmm_train_correction(self, theta=0.5, sample_leaves=4096, steps=2000, batch=4096, lr=1e-3):
        loss = C.c_float()
        samples = C.c_long()
        check(lib().amk_fmm_train_correction(self._h, float(theta), int(sample_leaves), int(steps), int(batch),
                                             float(lr), C.byref(loss), C.byref(samples)),
              "amk_fmm_train_correction")
        return loss.value, samples.value

    def fmm_audit(self, order=2, theta=0.5, learned=False, samples=1024):
        e = C.c_double()
        check(lib().amk_fmm_audit(self._h, int(order), float(theta), 1 if learned else 0, int(samples),
                                  C.byref(e)), "amk_fmm_audit")
        return e.value

    def fmm_learned_state(self):
        t, f, e = C.c_int(), C.c_int(), C.c_double()
        check(lib().amk_fmm_learned_state(self._h, C.byref(t), C.byref(f), C.byref(e)))
        return {"trained": bool(t.value), "fallback": bool(f.value), "last_error": e.value}

    # -- audit and tuning
    def force_error(self, samples=1024):
        """(rms, max) relative error of the current forces vs the FP64 exact sum."""
        r, m = C.c_double(), C.c_double()
        check(lib().amk_force_error(self._h, int(samples), C.byref(r), C.byref(m)), "amk_force_error")
        return r.value, m.value

    def set_fmm_precision(self, mode: str = "fp64"):
        """M2L class-product arithmetic: "fp64" (the reference's) or "tensor"
        (split-BF16 tcgen05 products for orders 5-7)."""
        check(lib().amk_set_fmm_precision(self._h, {"fp64": 0, "tensor": 1}[mode]), "amk_set_fmm_precision")

    def set_leaf_sizes(self, fmm_leaf=32, bh_leaf=8):
        check(lib().amk_set_leaf_sizes(self._h, int(fmm_leaf), int(bh_leaf)), "amk_set_leaf_sizes")

    def leaf_sizes(self):
        a, b = C.c_int(), C.c_int()
        check(lib().amk_get_leaf_sizes(self._h, C.byref(a), C.byref(b)), "amk_get_leaf_sizes")
        return a.value, b.value

    def autotune(self, error_budget=1e-5, samples=1024, flags=0):
        """Runs the autotuner; returns (candidates, chosen index)."""
        cap = 256
        out = (TuneCandidate * cap)()
        n, ch = C.c_int(0), C.c_int(-1)
        rc = lib().amk_autotune(self._h, float(error_budget), int(samples), int(flags), out, cap, C.byref(n),
                                C.byref(ch))
        cands = [{"method": out[k].method, "order": out[k].order, "theta": out[k].theta, "leaf": out[k].leaf,
                  "ms": out[k].ms, "rms": out[k].rms, "meets": bool(out[k].meets)} for k in range(min(n.value, cap))]
        check(rc, "amk_autotune")
        return cands, ch.value

    # -- batched instances
    def batch_set(self, params, offsets):
        """Splits the particle set into instances: params[i] steps particles
        [offsets[i], offsets[i+1])."""
        n = len(params)
        arr = (Params * n)(*params)
        off = np.ascontiguousarray(offsets, np.int64)
        if len(off) != n + 1:
            raise ValueError("offsets needs len(params) + 1 entries")
        check(lib().amk_batch_set(self._h, n, arr, off.ctypes.data_as(C.POINTER(C.c_long))), "amk_batch_set")
        self._batch_n = n

    def batch_step(self, n: int = 1, graph_chunk: int = 0, serial: bool = False):
        check(lib().amk_batch_step(self._h, int(n), int(graph_chunk), 1 if serial else 0), "amk_batch_step")

    def batch_autotune(self, error_budget=1e-5, samples=512):
        """Per-instance method choice by measurement; returns the methods."""
        m = np.zeros(getattr(self, "_batch_n", 0), np.int32)
        check(lib().amk_batch_autotune(self._h, float(error_budget), int(samples),
                                       m.ctypes.data_as(C.POINTER(C.c_int))), "amk_batch_autotune")
        return m

    def batch_energy(self, time_centre: bool = True):
        """Per-instance energies: a list of dicts like energy()."""
        n = getattr(self, "_batch_n", 0)
        arr = (EnergyOut * max(n, 1))()
        check(lib().amk_batch_energy(self._h, 1 if time_centre else 0, arr), "amk_batch_energy")
        return [{"kinetic": e.kinetic, "trap_potential": e.trap_potential,
                 "coulomb_potential": e.coulomb_potential, "total": e.total, "num_active": e.num_active}
                for e in arr[:n]]

    def batch_coulomb(self):
        check(lib().amk_batch_coulomb(self._h), "amk_batch_coulomb")

    def batch_status(self):
        ov = C.c_int(0)
        counts = np.zeros(getattr(self, "_batch_n", 0), np.int64)
        check(lib().amk_batch_status(self._h, C.byref(ov), counts.ctypes.data_as(C.POINTER(C.c_long))),
              "amk_batch_status")
        return {"overflow": bool(ov.value), "alive": counts}

    def batch_info(self):
        n, u, g = C.c_long(), C.c_long(), C.c_int()
        check(lib().amk_batch_info(self._h, C.byref(n), C.byref(u), C.byref(g)), "amk_batch_info")
        return {"instances": n.value, "work_units": u.value, "graphable": bool(g.value)}

    # -- checkpoint / export
    def checkpoint_save(self, path: str):
        check(lib().amk_checkpoint_save(self._h, os.fsencode(path)), "amk_checkpoint_save")

    def checkpoint_load(self, path: str):
        check(lib().amk_checkpoint_load(self._h, os.fsencode(path)), "amk_checkpoint_load")

    def export_vtk(self, path: str, binary: bool = True):
        check(lib().amk_export_vtk(self._h, os.fsencode(path), 1 if binary else 0), "amk_export_vtk")

    # -- learned correction (MLP)
    def mlp_params(self):
        n = lib().amk_mlp_num_params()
        p = np.empty(n, np.float32)
        check(lib().amk_mlp_get_params(self._h, p.ctypes.data_as(_fp), n), "amk_mlp_get_params")
        return p

    def set_mlp_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        check(lib().amk_mlp_set_params(self._h, p.ctypes.data_as(_fp), len(p)), "amk_mlp_set_params")

    def mlp_forward(self, x):
        x = np.ascontiguousarray(x, np.float32)
        y = np.empty((len(x), 3), np.float32)
        check(lib().amk_mlp_forward(self._h, x.ctypes.data_as(_fp), len(x), y.ctypes.data_as(_fp)),
              "amk_mlp_forward")
        return y

    def mlp_gradients(self, x, t):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        g = np.empty(lib().amk_mlp_num_params(), np.float32)
        yh = np.empty((len(x), 3), np.float32)
        loss = C.c_float()
        check(lib().amk_mlp_gradients(self._h, x.ctypes.data_as(_fp), t.ctypes.data_as(_fp), len(x),
                                      g.ctypes.data_as(_fp), C.byref(loss), yh.ctypes.data_as(_fp)),
              "amk_mlp_gradients")
        return loss.value, g, yh

    def mlp_train(self, x, t, steps, batch, lr):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        loss = C.c_float()
        check(lib().amk_mlp_train(self._h, x.ctypes.data_as(_fp), t.ctypes.data_as(_fp), len(x), int(steps),
                                  int(batch), float(lr), C.byref(loss)), "amk_mlp_train")
        return loss.value

    def bh_tree(self, x, y, z, q, leaf_capacity=8):
        """Barnes-Hut octree nodes in the reference's order (see amk_bh_tree_dump)."""
        x, y, z, q = map(_f64, (x, y, z, q))
        cap = 4 * len(x) + 64
        f = np.zeros((cap, 12))
        g = np.zeros((cap, 11), np.int64)
        nn = lib().amk_bh_tree_dump(self._h, len(x), _d(x), _d(y), _d(z), _d(q), int(leaf_capacity), cap,
                                    _d(f), g.ctypes.data_as(C.POINTER(C.c_long)))
        if nn < 0:
            check(int(nn), "amk_bh_tree_dump")
        return f[:nn], g[:nn]

    def solve_fmm(self, x, y, z, q, order, theta, leaf_capacity=32, want_energy=False):
        x, y, z, q = map(_f64, (x, y, z, q))
        n = len(x)
        fx, fy, fz = np.empty(n), np.empty(n), np.empty(n)
        e = C.c_double(0.0)
        check(lib().amk_solve_fmm(self._h, n, _d(x), _d(y), _d(z), _d(q), int(order), float(theta),
                                  int(leaf_capacity), _d(fx), _d(fy), _d(fz),
                                  C.cast(C.byref(e), _dp) if want_energy else None),
              "amk_solve_fmm")
        return ((fx, fy, fz), e.value) if want_energy else (fx, fy, fz)


# ------------------------------------------------------------------ reference-shaped API
_default_sim = None


def _solver_sim() -> Simulation:
    global _default_sim
    if _default_sim is None:
        _default_sim = Simulation()
    return _default_sim


class BarnesHutTree:
    """BarnesHutTree(theta, leaf_capacity=8) of barnes-hut.h:28-74, on the GPU.

    ``build(positions, charges)`` stores the sources; ``compute_forces()`` and
    ``compute_potentials()`` evaluate every source against all the others
    (self excluded), as ComputeForce(pos, q, i) / ComputePotential(pos, i).
    """

    def __init__(self, theta: float, leaf_capacity: int = 8):
        self.theta = float(theta)
        self.leaf_capacity = max(1, int(leaf_capacity))
        self._src = None

    def build(self, positions, charges):
        p = np.asarray(positions, np.float64)
        self._src = (p[:, 0].copy(), p[:, 1].copy(), p[:, 2].copy(), _f64(charges))

    def compute_forces(self):
        x, y, z, q = self._src
        fx, fy, fz = _solver_sim().solve_barnes_hut(x, y, z, q, self.theta, self.leaf_capacity)
        return np.stack([fx, fy, fz], axis=1)

    def compute_potentials(self):
        x, y, z, q = self._src
        *_, phi = _solver_sim().solve_barnes_hut(x, y, z, q, self.theta, self.leaf_capacity,
                                                 want_phi=True)
        return phi


class FastMultipoleSolver:
    """FastMultipoleSolver(order, theta, leaf_capacity=32) of fast-multipole.h:46-71."""

    def __init__(self, order: int, theta: float, leaf_capacity: int = 32):
        self.order = min(max(int(order), 1), 8)
        self.theta = float(theta)
        self.leaf_capacity = max(1, int(leaf_capacity))

    def compute(self, positions, charges, forces=True, energy=True):
        p = np.asarray(positions, np.float64)
        (fx, fy, fz), e = _solver_sim().solve_fmm(p[:, 0], p[:, 1], p[:, 2], charges, self.order,
                                                  self.theta, self.leaf_capacity, want_energy=True)
        return (np.stack([fx, fy, fz], axis=1) if forces else None), (e if energy else None)

    def compute_forces(self, positions, charges):
        return self.compute(positions, charges, energy=False)[0]

    def compute_potential_energy(self, positions, charges):
        return self.compute(positions, charges, forces=False)[1]


def compute_standard_coulomb_forces(sim: Simulation, cutoff_radius: float):
    """ComputeStandardCoulombForces(rm, cutoff_radius), coulomb_interaction.h:10."""
    sim.coulomb_standard(cutoff_radius)


def compute_barnes_hut_coulomb_forces(sim: Simulation, theta: float):
    """ComputeBarnesHutCoulombForces(rm, theta), barnes-hut.h:76."""
    sim.coulomb_barnes_hut(theta)


def compute_fast_multipole_coulomb_forces(sim: Simulation, order: int, theta: float):
    """ComputeFastMultipoleCoulombForces(rm, order, theta), fast-multipole.h:73."""
    sim.coulomb_fmm(order, theta)


def checkpoint_info(path: str):
    """(particles, step, Params) of a checkpoint file; needs no GPU."""
    n, st, p = C.c_long(), C.c_long(), Params()
    check(lib().amk_checkpoint_info(os.fsencode(path), C.byref(n), C.byref(st), C.byref(p)),
          "amk_checkpoint_info")
    return n.value, st.value, p


def write_vtu(path: str, x, y, z, species, vx=None, vy=None, vz=None, alive=None, ids=None, time=0.0,
              binary=True):
    """VTK XML UnstructuredGrid of host particle arrays (amk_write_vtu); no GPU."""
    x, y, z = map(_f64, (x, y, z))
    v = [None if a is None else _f64(a) for a in (vx, vy, vz)]
    sp = np.ascontiguousarray(species, np.uint8)
    al = None if alive is None else np.ascontiguousarray(alive, np.uint8)
    ii = None if ids is None else np.ascontiguousarray(ids, np.uint32)
    check(lib().amk_write_vtu(os.fsencode(path), len(x), _d(x), _d(y), _d(z), *[_d(a) for a in v],
                              sp.ctypes.data_as(_u8p), None if al is None else al.ctypes.data_as(_u8p),
                              None if ii is None else ii.ctypes.data_as(C.POINTER(C.c_uint32)),
                              C.c_double(time), 1 if binary else 0), "amk_write_vtu")


def write_pvd(path: str, files, times):
    arr = (C.c_char_p * len(files))(*[os.fsencode(f) for f in files])
    t = _f64(times)
    check(lib().amk_write_pvd(os.fsencode(path), len(files), arr, _d(t)), "amk_write_pvd")
