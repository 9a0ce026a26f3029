"""The oracle's FP64 restatement of the per-agent behaviours, pinned to the
reference's own code: lorentz.cc, cooling.cc, annihilation.cc and
coulomb_interaction.cc compiled in place (oracle/_ref) against BioDynaMo
stand-ins whose Random replays the CUDA library's Philox draws and whose
neighbour search visits agents in ascending id. CPU only."""
import numpy as np
import pytest

import oracle_lib as O
from conftest import E, gaussian_cloud

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference library not built")

MASS = {1: 9.1093837015e-31, 3: 9.1093837015e-31, 0: 1.67262192369e-27, 4: 1.67262192369e-27}


def cloud(n, seed, sigma=1e-4, vscale=1e4, species=(1, 3)):
    x, y, z, _ = gaussian_cloud(n, seed, sigma=(sigma, sigma, sigma))
    rng = np.random.default_rng(seed + 1)
    vel = rng.normal(0, vscale, (n, 3))
    sp = np.asarray(species, np.uint8)[rng.integers(0, len(species), n)]
    return np.stack([x, y, z], 1), vel, sp


def oracle_state(pos, vel, sp):
    m, q = O.species_props(sp)
    return dict(x=pos[:, 0].copy(), y=pos[:, 1].copy(), z=pos[:, 2].copy(), vx=vel[:, 0].copy(),
                vy=vel[:, 1].copy(), vz=vel[:, 2].copy(), q=q, m=m, alive=np.ones(len(sp), np.uint8),
                species=sp.copy())


TRAP = dict(b0=1.5, voltage=20.0, z0=0.01, rho0=0.012, dt=6e-12)


@needs_ref
def test_boris_push_equals_reference_lorentz_force():
    pos, vel, sp = cloud(800, 1, species=(0, 1, 3, 4))
    rng = np.random.default_rng(2)
    ref = O.RefWorld(pos, vel, sp, **TRAP)
    st = oracle_state(pos, vel, sp)
    for step in range(1, 21):
        f = rng.normal(0, 1e-20, (3, 800))
        ref.set_forces(*f)
        ref.behaviours(step, lorentz=True, cooling=False, annihilation=False)
        O.boris_push(st, *f, TRAP["b0"], TRAP["voltage"], TRAP["z0"], TRAP["rho0"], TRAP["dt"], step == 1)
    r = ref.state()
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.array_equal(r[k], st[k]), k  # same FP64 operations, no contraction
    assert np.all(r["fx"] == 0.0)  # the force slot is consumed (lorentz.cc:70)


@needs_ref
def test_cooling_equals_reference_cyclotron_cooling():
    pos, vel, sp = cloud(600, 3, species=(0, 1, 3))
    for scale, bath in ((1.0, 4.0), (1e-9, 4.0), (1e-6, 0.0)):
        ref = O.RefWorld(pos, vel, sp, cooling_scale=scale, bath_temp=bath, seed=77, **TRAP)
        st = oracle_state(pos, vel, sp)
        for step in range(1, 6):
            ref.behaviours(step, lorentz=False, cooling=True, annihilation=False)
            O.cooling(st, TRAP["b0"], TRAP["dt"], scale, bath, 77, step)
        r = ref.state()
        for k in ("vx", "vy", "vz"):
            assert np.array_equal(r[k], st[k]), (scale, bath, k)
    for q, m, b in ((E, MASS[1], 1.0), (2 * E, MASS[0], 3.0), (0.0, MASS[1], 1.0)):
        assert O.ref_cooling_time(q, m, b) == O.cooling_time(q, m, b)


@needs_ref
@pytest.mark.parametrize("prob,radius", [(1.0, 8e-6), (0.5, 1.2e-5), (0.2, 2e-5)])
def test_annihilation_equals_reference_interaction(prob, radius):
    pos, vel, sp = cloud(1500, 5, species=(0, 1, 3, 4))
    ref = O.RefWorld(pos, vel, sp, annihilation=True, contact_radius=radius, probability=prob, seed=9,
                     **TRAP)
    st = oracle_state(pos, vel, sp)
    total = 0
    for step in range(1, 4):
        marked = ref.behaviours(step, lorentz=False, cooling=False, annihilation=True)
        assert marked == O.annihilation(st, radius, prob, 9, step)
        total += marked
    assert total > 0
    assert np.array_equal(ref.state()["alive"], st["alive"])  # the same annihilated set, bit for bit
    for a in range(6):
        for b in range(6):
            assert O.ref_is_antiparticle_pair(a, b) == ({a, b} in ({0, 4}, {1, 3}))


@needs_ref
def test_cutoff_forces_equal_reference_standard_coulomb():
    pos, vel, sp = cloud(2000, 7, species=(0, 1, 3))
    alive = np.ones(2000, np.uint8)
    alive[::7] = 0
    ref = O.RefWorld(pos, vel, sp, **TRAP)
    ref.set_alive(alive)
    ref.coulomb_standard(2e-5)
    r = ref.state()
    _, q = O.species_props(sp)
    f = O.cutoff(pos[:, 0], pos[:, 1], pos[:, 2], q, 2e-5, alive)
    live = alive.astype(bool)
    for a, b in zip((r["fx"], r["fy"], r["fz"]), f):
        assert np.max(np.abs(a[live] - b[live])) <= 1e-13 * np.max(np.abs(b))


def test_oracle_reproduces_the_reference_readme_steps_fixture():
    # the committed fixture was produced by the reference's own step code;
    # the oracle's restatement must reproduce it (this test needs no
    # reference library)
    import os
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "readme_ic.npz"))
    ref = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "readme_steps_ref.npz"))
    st = oracle_state(g["pos"], g["vel"], g["species"])
    dt = float(ref["dt"])
    for step in range(1, ref["x"].shape[0] + 1):
        f = O.cutoff(st["x"], st["y"], st["z"], st["q"], 1e-5, st["alive"])
        O.boris_push(st, *f, 1.0, 10.0, 0.01, 0.01, dt, step == 1)
        O.cooling(st, 1.0, dt, 1.0, 4.0, 42, step)
        O.annihilation(st, 5e-6, 1.0, 42, step)
        assert np.array_equal(st["alive"], ref["alive"][step - 1]), step
        for k in ("x", "y", "z", "vx", "vy", "vz"):
            a, b = st[k], ref[k][step - 1]
            assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b)), (step, k)
