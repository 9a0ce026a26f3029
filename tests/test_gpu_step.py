"""GPU parity of the per-step behaviours (Boris push + cyclotron cooling,
annihilation, energies) and of whole README-scale steps against the oracle."""
import os

import numpy as np
import pytest

import amk
import oracle_lib as O
from conftest import E, gaussian_cloud

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NOTEBOOK_STEP0 = {"kinetic": 4.21895e-18, "trap_potential": -3.18438e-22,
                  "coulomb_potential": 5.47464e-24}


def readme_params(**over):
    kw = dict(seed=42, b0=1.0, trap_voltage=10.0, z0=0.01, rho0=0.01, num_steps=100,
              populations={"positron": 100, "electron": 100},
              temperatures={"positron": 1e3, "electron": 1e3}, cloud_radii=(1e-4, 1e-4, 1e-4),
              bath_temperature=4.0, cooling_scale=1.0, coulomb_forces_enabled=1,
              coulomb_method="standard", energy_method="standard", cutoff_radius=1e-5,
              annihilation_enabled=1, contact_radius=5e-6, annihilation_probability=1.0)
    kw.update(over)
    return amk.make_params(**kw)


def oracle_state(pos, vel, sp):
    m, q = O.species_props(sp)
    return dict(x=pos[:, 0].copy(), y=pos[:, 1].copy(), z=pos[:, 2].copy(), vx=vel[:, 0].copy(),
                vy=vel[:, 1].copy(), vz=vel[:, 2].copy(), q=q, m=m,
                alive=np.ones(len(sp), np.uint8), species=np.asarray(sp, np.uint8))


def test_init_particles_bit_exact_and_step0_energy():
    g = np.load(os.path.join(GOLD, "readme_ic.npz"))
    with amk.Simulation(readme_params()) as s:
        s.init_particles()
        st = s.get_particles()
        assert np.array_equal(np.stack([st["x"], st["y"], st["z"]], 1), g["pos"])
        assert np.array_equal(np.stack([st["vx"], st["vy"], st["vz"]], 1), g["vel"])
        e = s.energy(time_centre=True)
        for k, v in NOTEBOOK_STEP0.items():
            assert float(f"{e[k]:.5e}") == v, (k, e[k])
        assert e["num_active"] == 200


def test_push_and_cooling_match_oracle():
    g = np.load(os.path.join(GOLD, "readme_ic.npz"))
    p = readme_params(annihilation_enabled=0)
    with amk.Simulation(p) as s:
        s.init_particles()
        ref = oracle_state(g["pos"], g["vel"], g["species"])
        for step in range(1, 6):
            s.coulomb_standard(p.cutoff_radius)
            fx, fy, fz = s.get_forces()
            gx, gy, gz = O.cutoff(ref["x"], ref["y"], ref["z"], ref["q"], p.cutoff_radius, ref["alive"])
            for a, b in zip((fx, fy, fz), (gx, gy, gz)):
                assert np.max(np.abs(a - b)) <= 1e-10 * max(np.max(np.abs(b)), 1e-300)
            s.push()
            O.boris_push(ref, gx, gy, gz, p.b0, p.trap_voltage, p.z0, p.rho0, p.dt, step == 1)
            O.cooling(ref, p.b0, p.dt, p.cooling_scale, p.bath_temperature, p.seed, step)
        st = s.get_particles()
        for k in ("x", "y", "z", "vx", "vy", "vz"):
            assert np.max(np.abs(st[k] - ref[k])) <= 1e-10 * np.max(np.abs(ref[k])), k


def test_boris_only_multistep_matches_oracle():
    x, y, z, _ = gaussian_cloud(1000, 3, sigma=(1e-4, 1e-4, 1e-4))
    rng = np.random.default_rng(3)
    vel = rng.normal(0, 1e4, (1000, 3))
    sp = np.where(rng.random(1000) < 0.5, 1, 3).astype(np.uint8)
    p = readme_params(coulomb_forces_enabled=0, annihilation_enabled=0, cooling_enabled=0)
    with amk.Simulation(p) as s:
        s.set_particles(x, y, z, vel[:, 0], vel[:, 1], vel[:, 2], sp)
        ref = oracle_state(np.stack([x, y, z], 1), vel, sp)
        zero = np.zeros(1000)
        for step in range(1, 21):
            s.step(1)
            O.boris_push(ref, zero, zero, zero, p.b0, p.trap_voltage, p.z0, p.rho0, p.dt, step == 1)
        st = s.get_particles()
        for k in ("x", "y", "z", "vx", "vy", "vz"):
            assert np.max(np.abs(st[k] - ref[k])) <= 1e-12 * np.max(np.abs(ref[k])), k


def test_cooling_with_bath_matches_oracle_one_step():
    x, y, z, _ = gaussian_cloud(2000, 8, sigma=(1e-4, 1e-4, 1e-4))
    rng = np.random.default_rng(8)
    vel = rng.normal(0, 1e5, (2000, 3))
    sp = np.where(rng.random(2000) < 0.5, 1, 3).astype(np.uint8)
    p = readme_params(coulomb_forces_enabled=0, annihilation_enabled=0, cooling_scale=1e-9,
                      bath_temperature=300.0)
    with amk.Simulation(p) as s:
        s.set_particles(x, y, z, vel[:, 0], vel[:, 1], vel[:, 2], sp)
        ref = oracle_state(np.stack([x, y, z], 1), vel, sp)
        s.step(1)
        zero = np.zeros(2000)
        O.boris_push(ref, zero, zero, zero, p.b0, p.trap_voltage, p.z0, p.rho0, p.dt, True)
        O.cooling(ref, p.b0, p.dt, p.cooling_scale, p.bath_temperature, p.seed, 1)
        st = s.get_particles()
        for k in ("vx", "vy", "vz"):
            assert np.max(np.abs(st[k] - ref[k])) <= 1e-11 * np.max(np.abs(ref[k])), k
        # strong damping (tau = 2.6e-11 s, ~10 e-folds of v_perp^2 per 60
        # steps): v_perp relaxes to the bath, sigma^2 = kT/m per component
        p2 = s.params
        p2.cooling_scale = 1e-11
        s.params = p2
        s.step(300)
        st = s.get_particles()
        m = 9.1093837015e-31
        vperp2 = np.mean(st["vx"] ** 2 + st["vy"] ** 2) / 2
        assert abs(vperp2 / (1.380649e-23 * 300.0 / m) - 1.0) < 0.1


def test_annihilation_bit_exact_vs_oracle():
    # dense two-species cloud so that many contacts compete for partners
    n = 3000
    rng = np.random.default_rng(12)
    pos = rng.uniform(-2e-5, 2e-5, (n, 3))
    sp = np.where(rng.random(n) < 0.5, 1, 3).astype(np.uint8)
    for prob, seed in ((1.0, 42), (0.5, 42), (0.5, 7), (0.0, 1)):
        p = readme_params(annihilation_probability=prob, contact_radius=1.5e-6, seed=seed,
                          coulomb_forces_enabled=0)
        with amk.Simulation(p) as s:
            s.set_particles(pos[:, 0], pos[:, 1], pos[:, 2], np.zeros(n), np.zeros(n), np.zeros(n), sp)
            ref = oracle_state(pos, np.zeros((n, 3)), sp)
            for _ in range(2):  # second call sees the survivors of the first
                marked = s.annihilate()
                mo = O.annihilation(ref, p.contact_radius, prob, seed, 1)
                assert np.array_equal(s.get_particles()["alive"], ref["alive"]), (prob, seed)
                assert marked == mo
            if prob == 0.0:
                assert ref["alive"].all()
            else:
                assert not ref["alive"].all()


def test_readme_run_energy_and_population():
    p = readme_params()
    with amk.Simulation(p) as s:
        s.init_particles()
        e0 = s.energy()
        s.step(100)
        e1 = s.energy()
        assert s.step_count() == 100
        assert 0 < e1["num_active"] <= 200 and e1["num_active"] % 2 == 0
        assert np.isfinite(e1["total"])
        # annihilation removes kinetic energy; the total cannot grow much
        assert e1["total"] < e0["total"] * 1.05


def test_readme_steps_match_the_reference_code_fixture():
    # 40 full steps (cutoff forces, Boris push, cooling at 4 K, annihilation
    # at 5e-6 m with p = 1) against the fixture the reference's own
    # coulomb_interaction.cc / lorentz.cc / cooling.cc / annihilation.cc
    # produced (tests/golden/make_golden.py): the annihilated set bit-exact
    # every step, positions and velocities to 1e-9
    ref = np.load(os.path.join(GOLD, "readme_steps_ref.npz"))
    with amk.Simulation(readme_params()) as s:
        s.init_particles()
        for step in range(ref["x"].shape[0]):
            s.step(1)
            st = s.get_particles()
            assert np.array_equal(st["alive"], ref["alive"][step]), step
            for k in ("x", "y", "z", "vx", "vy", "vz"):
                a, b = st[k], ref[k][step]
                assert np.max(np.abs(a - b)) <= 1e-9 * np.max(np.abs(b)), (step, k)
    assert ref["alive"][-1].sum() < 200


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built")
def test_push_cooling_annihilation_match_the_reference_world():
    # a denser two-species cloud stepped by the library and by the
    # reference's own per-agent code, same forces each step
    n = 2400
    rng = np.random.default_rng(21)
    pos = rng.normal(0, 3e-5, (n, 3))
    vel = rng.normal(0, 2e4, (n, 3))
    sp = np.where(rng.random(n) < 0.5, 1, 3).astype(np.uint8)
    p = readme_params(contact_radius=1.5e-6, annihilation_probability=0.5, cooling_scale=1e-8,
                      bath_temperature=20.0, seed=5, cutoff_radius=4e-6)
    w = O.RefWorld(pos, vel, sp, b0=p.b0, voltage=p.trap_voltage, z0=p.z0, rho0=p.rho0, dt=p.dt,
                   cooling_scale=p.cooling_scale, bath_temp=p.bath_temperature, annihilation=True,
                   contact_radius=p.contact_radius, probability=p.annihilation_probability, seed=p.seed)
    with amk.Simulation(p) as s:
        s.set_particles(pos[:, 0], pos[:, 1], pos[:, 2], vel[:, 0], vel[:, 1], vel[:, 2], sp)
        marked = 0
        for step in range(1, 9):
            s.coulomb_standard(p.cutoff_radius)
            w.coulomb_standard(p.cutoff_radius)
            f = s.get_forces()
            r = w.state()
            live = r["alive"].astype(bool)
            for a, b in zip(f, (r["fx"], r["fy"], r["fz"])):
                assert np.max(np.abs(a[live] - b[live])) <= 1e-10 * max(np.max(np.abs(b)), 1e-300)
            s.push()
            s.annihilate()
            marked += w.behaviours(step)
            st, r = s.get_particles(), w.state()
            assert np.array_equal(st["alive"], r["alive"]), step
            for k in ("x", "y", "z", "vx", "vy", "vz"):
                assert np.max(np.abs(st[k] - r[k])) <= 1e-10 * np.max(np.abs(r[k])), (step, k)
        assert marked > 0


@pytest.mark.parametrize("grid_min", [None, "1"])
def test_annihilation_grid_matcher_bit_exact_vs_oracle(monkeypatch, grid_min):
    # tens of thousands of contacts: the grid-wide matching rounds (and, with
    # AMK_MATCH_GRID_MIN=1, the same rounds on every contact set, followed
    # by the one-CTA finish) give the sequential greedy pass's set
    if grid_min is not None:
        monkeypatch.setenv("AMK_MATCH_GRID_MIN", grid_min)
    n = 20000
    rng = np.random.default_rng(31)
    pos = rng.uniform(-5e-5, 5e-5, (n, 3))
    sp = rng.choice(np.array([0, 1, 3, 4], np.uint8), n)
    p = readme_params(annihilation_probability=0.7, contact_radius=3e-6, seed=3, coulomb_forces_enabled=0,
                      populations={"positron": n // 2, "electron": n - n // 2})
    with amk.Simulation(p) as s:
        s.set_particles(pos[:, 0], pos[:, 1], pos[:, 2], np.zeros(n), np.zeros(n), np.zeros(n), sp)
        ref = oracle_state(pos, np.zeros((n, 3)), sp)
        for step in (1, 2):
            marked = s.annihilate()
            mo = O.annihilation(ref, p.contact_radius, p.annihilation_probability, p.seed, 1)
            assert marked == mo and (step == 2 or mo > 1000)
            assert np.array_equal(s.get_particles()["alive"], ref["alive"])
