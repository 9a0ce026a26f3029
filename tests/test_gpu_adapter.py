"""The BioDynaMo drop-in adapter (antimatter-kernel_b200/adapter/
amk_bdm_adapter.cc, .h): the reference's Coulomb drivers, solver classes
(BarnesHutTree, FastMultipoleSolver), behaviours (LorentzForce,
CyclotronCooling, AnnihilationInteraction, run through the per-step
standalone operation) and ComputeTotalEnergy with their own signatures,
compiled against stand-ins of BioDynaMo's types (tests/bdm_stub) and linked
to libamk. Forces on agents must match the reference's own drivers (and the
FP64 cutoff oracle), annihilated agents must be left untouched and neutral
agents get zero force under the FMM; the classes must match the reference's
classes; the adapter's step loop must match the reference's own per-agent
code run by the oracle's harness."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle_lib as O
from conftest import E, ROOT, gaussian_cloud, rel_errors

ADAPTER = os.path.join(ROOT, "antimatter-kernel_b200", "adapter", "amk_bdm_adapter.cc")
GOLD = os.path.join(ROOT, "tests", "golden")
STUB = os.path.join(ROOT, "tests", "bdm_stub")
LIBDIR = os.path.join(ROOT, "antimatter-kernel_b200")


def build_harness(out_dir):
    """Compiles the adapter and the test harness into one shared library."""
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    out = os.path.join(out_dir, "libamk_adapter_harness.so")
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", f"-I{STUB}", f"-I{os.path.join(ROOT, 'include')}",
           f"-I{os.path.dirname(ADAPTER)}", ADAPTER, os.path.join(STUB, "harness.cc"), f"-L{LIBDIR}", "-lamk", f"-Wl,-rpath,{LIBDIR}", "-o", out]
    subprocess.run(cmd, check=True, capture_output=True)
    return out


def test_adapter_compiles_and_links(tmp_path):
    import amk
    amk.lib()  # libamk.so built
    lib = C.CDLL(build_harness(str(tmp_path)))
    assert hasattr(lib, "harness_run")


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    import amk
    amk.lib()
    lib = C.CDLL(build_harness(str(tmp_path_factory.mktemp("adapter"))))
    dp = C.POINTER(C.c_double)
    lib.harness_run.argtypes = [C.c_int, C.c_long, dp, dp, dp, dp, C.POINTER(C.c_uint8), C.c_double, C.c_int,
                                dp, dp, dp]
    lib.harness_run.restype = C.c_int

    def run(method, x, y, z, q, annihilated, param, order=0):
        if method == "lib":
            return lib
        n = len(x)
        arrs = [np.ascontiguousarray(a, np.float64) for a in (x, y, z, q)]
        an = np.ascontiguousarray(annihilated, np.uint8)
        f = [np.zeros(n) for _ in range(3)]
        rc = lib.harness_run(method, n, *[a.ctypes.data_as(dp) for a in arrs], an.ctypes.data_as(C.POINTER(C.c_uint8)),
                             float(param), int(order), *[a.ctypes.data_as(dp) for a in f])
        assert rc == 0
        return f
    return run


def agents(n, seed):
    x, y, z, q = gaussian_cloud(n, seed)
    rng = np.random.default_rng(seed)
    annihilated = (rng.random(n) < 0.1).astype(np.uint8)
    q = np.where(rng.random(n) < 0.05, 0.0, q)  # some neutral agents
    return x, y, z, q, annihilated


@pytest.mark.gpu
def test_standard_driver_matches_fp64_cutoff(harness):
    x, y, z, q, ann = agents(3000, 1)
    fx, fy, fz = harness(0, x, y, z, q, ann, 3e-5)
    live = ann == 0
    assert np.all(np.isnan(fx[~live]))  # annihilated agents untouched
    gx, gy, gz = O.cutoff(x[live], y[live], z[live], q[live], 3e-5)
    scale = max(np.max(np.abs(gx)), 1e-300)
    for a, b in zip((fx[live], fy[live], fz[live]), (gx, gy, gz)):
        assert np.max(np.abs(a - b)) <= 1e-12 * scale
    fx0, _, _ = harness(0, x, y, z, q, ann, 0.0)  # cutoff <= 0: zero force on every live agent
    assert np.all(fx0[live] == 0.0) and np.all(np.isnan(fx0[~live]))


@pytest.mark.gpu
def test_barnes_hut_and_fmm_drivers_match_the_reference_drivers(harness):
    if not O.ref_available():
        pytest.skip("reference library not built")
    x, y, z, q, ann = agents(4000, 2)
    live = ann == 0
    for method, param, order, tol in ((1, 0.5, 0, 1e-10), (2, 0.5, 4, 1e-9)):
        f = harness(method, x, y, z, q, ann, param, order)
        assert np.all(np.isnan(f[0][~live]))
        name = "barnes-hut" if method == 1 else "fast-multipole"
        g = O.ref_driver(name, x, y, z, q, 1 - ann, param, order)
        charged = live & (q != 0)
        rel, _ = rel_errors([a[charged] for a in f], [b[charged] for b in g])
        assert np.max(rel) < tol, (name, np.max(rel))
        neutral = live & (q == 0)
        assert all(np.all(a[neutral] == 0.0) for a in f)


@pytest.mark.gpu
def test_solver_classes_match_the_reference_classes(harness):
    lib = harness("lib", None, None, None, None, None, None)
    dp = C.POINTER(C.c_double)
    lib.harness_bh_class.restype = C.c_long
    lib.harness_bh_class.argtypes = [C.c_long, dp, dp, dp, dp, C.c_double, C.c_long, dp, dp, C.c_double, C.c_double,
                                     C.c_double, C.c_double, dp, dp]
    lib.harness_fmm_class.argtypes = [C.c_long, dp, dp, dp, dp, C.c_int, C.c_double, dp, dp]
    x, y, z, q = gaussian_cloud(3000, 5)
    ptr = [np.ascontiguousarray(a).ctypes.data_as(dp) for a in (x, y, z, q)]
    for theta in (0.0, 0.5):
        f, phi, fe, pe = np.zeros(9000), np.zeros(3000), np.zeros(3), np.zeros(1)
        point = (1e-5, -2e-5, 3e-5)
        nn = lib.harness_bh_class(3000, *ptr, theta, 8, f.ctypes.data_as(dp), phi.ctypes.data_as(dp), *point,
                                  2 * E, fe.ctypes.data_as(dp), pe.ctypes.data_as(dp))
        assert nn > 0
        if O.ref_available():
            ref = O.ref_bh_forces(x, y, z, q, theta, 8)
            rel, _ = rel_errors(f.reshape(-1, 3).T, ref)
            assert np.max(rel) < 1e-10
            rphi = O.ref_bh_potentials(x, y, z, q, theta, 8)
            assert np.max(np.abs(phi - rphi)) <= 1e-10 * np.max(np.abs(rphi))
            assert nn == len(O.ref_bh_tree(x, y, z, q, 8)[0])
        if theta == 0.0:  # a point that is not a source: the exact sum
            d = np.stack([point[0] - x, point[1] - y, point[2] - z])
            r = np.sqrt((d ** 2).sum(0))
            exact = 8.9875517923e9 * 2 * E * (q * d / r ** 3).sum(1)
            assert np.max(np.abs(fe - exact)) <= 1e-10 * np.max(np.abs(exact))
            assert abs(pe[0] - (q / r).sum()) <= 1e-10 * abs((q / r).sum())
    f, e = np.zeros(9000), np.zeros(1)
    assert lib.harness_fmm_class(3000, *ptr, 4, 0.5, f.ctypes.data_as(dp), e.ctypes.data_as(dp)) == 0
    if O.ref_available():
        (rx, ry, rz), re = O.ref_fmm(x, y, z, q, 4, 0.5, 32, forces=True, energy=True)
        rel, _ = rel_errors(f.reshape(-1, 3).T, (rx, ry, rz))
        assert np.max(rel) < 1e-9
        assert abs(e[0] - re) <= 1e-10 * abs(re)
    lib.harness_cooling_time.restype = C.c_double
    lib.harness_cooling_time.argtypes = [C.c_double] * 3
    assert lib.harness_cooling_time(E, 9.1093837015e-31, 1.0) == O.cooling_time(E, 9.1093837015e-31, 1.0)
    assert [lib.harness_is_pair(a, b) for a, b in ((0, 4), (4, 0), (1, 3), (0, 1), (2, 2))] == [1, 1, 1, 0, 0]


def _adapter_steps(harness, pos, vel, sp, trap, dt, steps, rc, contact):
    lib = harness("lib", None, None, None, None, None, None)
    dp, u8 = C.POINTER(C.c_double), C.POINTER(C.c_uint8)
    lib.harness_steps.argtypes = ([C.c_long] + [dp] * 6 + [u8, dp, dp, u8] + [C.c_double] * 8 +
                                  [C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, dp])
    n = len(pos)
    m, q = O.species_props(sp)
    arr = [np.ascontiguousarray(pos[:, k]) for k in range(3)] + [np.ascontiguousarray(vel[:, k]) for k in range(3)]
    alive = np.ones(n, np.uint8)
    energy = np.zeros(8)
    rc_ = lib.harness_steps(n, *[a.ctypes.data_as(dp) for a in arr], sp.ctypes.data_as(u8), q.ctypes.data_as(dp),
                            m.ctypes.data_as(dp), alive.ctypes.data_as(u8), trap["b0"], trap["voltage"], trap["z0"],
                            trap["rho0"], dt, rc, 1.0, 4.0, 1, contact, 1.0, 42, steps, energy.ctypes.data_as(dp))
    assert rc_ == 0
    st = dict(zip(("x", "y", "z", "vx", "vy", "vz"), arr), alive=alive, q=q, m=m)
    return st, energy


def _dense_readme_cloud():
    g = np.load(os.path.join(GOLD, "readme_ic.npz"))
    rng = np.random.default_rng(4)
    pos = g["pos"] * 0.4 + rng.normal(0, 1e-7, (len(g["pos"]), 3))  # denser: contacts within a few steps
    return pos, g["vel"].copy(), g["species"]


@pytest.mark.gpu
def test_behaviour_steps_equal_the_library_step(harness):
    # the reference application's loop on the adapter (standard Coulomb
    # driver, the three behaviours per agent, the per-step operation, the
    # energy) equals the library's own amk_step on the same particles, after
    # every step count checked (the first difference is reported)
    import amk
    pos, vel, sp = _dense_readme_cloud()
    n = len(pos)
    trap = dict(b0=1.0, voltage=10.0, z0=0.01, rho0=0.01)
    dt, rc, contact = O.dt_for([1, 3], 1.0), 1e-5, 4e-6
    d = np.sqrt(0.01 ** 2 / 2 + 0.01 ** 2 / 4)  # the adapter hands the library z0 = sqrt(2) d, rho0 = 0
    p = amk.make_params(seed=42, b0=1.0, trap_voltage=10.0, z0=np.sqrt(2.0) * d, rho0=0.0, dt=dt,
                        populations={"positron": 100, "electron": 100}, coulomb_method="standard",
                        cutoff_radius=rc, cooling_enabled=1, cooling_scale=1.0, bath_temperature=4.0,
                        annihilation_enabled=1, contact_radius=contact, annihilation_probability=1.0)
    counts = (1, 2, 3, 5, 8, 13, 20, 30)
    lib_states = {}
    with amk.Simulation(p) as s:
        s.set_particles(pos[:, 0], pos[:, 1], pos[:, 2], vel[:, 0], vel[:, 1], vel[:, 2], sp)
        for k in range(1, counts[-1] + 1):
            s.step(1)
            if k in counts:
                lib_states[k] = s.get_particles()
    for k in counts:
        st, energy = _adapter_steps(harness, pos, vel, sp, trap, dt, k, rc, contact)
        lib = lib_states[k]
        live = (st["alive"] == 1) & (lib["alive"] == 1)
        diff = {f: float(np.max(np.abs(st[f] - lib[f])[live], initial=0.0)) for f in ("x", "y", "z", "vx", "vy", "vz")}
        n_alive = int((st["alive"] != lib["alive"]).sum())
        assert n_alive == 0 and max(diff.values()) == 0.0, (k, n_alive, diff)
        for f in ("x", "y", "z", "vx", "vy", "vz"):
            assert np.array_equal(st[f], lib[f]), (k, f)  # annihilated particles stay where they died
    assert lib["alive"].sum() < n
    # the last two energies: raw, then time-centred with the first
    e_last = O.energy_standard(st, trap["voltage"], trap["z0"], trap["rho0"], rc)
    assert abs(energy[4] - e_last["kinetic"]) <= 1e-12 * e_last["kinetic"]
    assert energy[7] == e_last["num_active"]
    assert abs(energy[5] - 0.5 * (energy[1] + e_last["trap_potential"])) <= 1e-12 * abs(e_last["trap_potential"])


@pytest.mark.gpu
def test_behaviour_steps_match_the_reference_code(harness):
    # against the reference's own coulomb_interaction.cc, lorentz.cc,
    # cooling.cc and annihilation.cc (oracle/_ref, same Philox draws) over
    # the first 10 steps of the dense cloud
    if not O.ref_available():
        pytest.skip("reference library not built")
    pos, vel, sp = _dense_readme_cloud()
    trap = dict(b0=1.0, voltage=10.0, z0=0.01, rho0=0.01)
    dt, steps, rc, contact = O.dt_for([1, 3], 1.0), 10, 1e-5, 4e-6
    st, _ = _adapter_steps(harness, pos, vel, sp, trap, dt, steps, rc, contact)
    w = O.RefWorld(pos, vel, sp, dt=dt, cooling_scale=1.0, bath_temp=4.0, annihilation=True,
                   contact_radius=contact, probability=1.0, seed=42, **trap)
    for step in range(1, steps + 1):
        w.coulomb_standard(rc)
        w.behaviours(step)
    r = w.state()
    diff = {k: float(np.max(np.abs(st[k] - r[k])) / np.max(np.abs(r[k]))) for k in ("x", "y", "z", "vx", "vy", "vz")}
    assert np.array_equal(st["alive"], r["alive"]), (int((st["alive"] != r["alive"]).sum()), diff)
    assert r["alive"].sum() < len(pos)
    assert max(diff.values()) <= 1e-9, diff
