"""GPU cloud generators (the reference's penning_trap.cc:51-160 shapes on
Philox draws): species order and counts, every position inside the
ellipsoid, the moments of the uniform-ellipsoid and Gaussian shapes, zero
mean drift per species with the reference's sqrt(n/(n-1)) rescale,
determinism, and a batch of instances equal to the instances generated one
context at a time."""
import numpy as np
import pytest

import amk

pytestmark = pytest.mark.gpu
KB = 1.380649e-23
MASS = {0: 1.67262192369e-27, 1: 9.1093837015e-31, 3: 9.1093837015e-31}


def params(n_e=60000, n_p=40000, radii=(5e-4, 5e-4, 2e-3), temp=100.0, seed=7):
    return amk.make_params(seed=seed, b0=5.0, trap_voltage=100.0, z0=0.02, rho0=0.02, cutoff_radius=2e-5,
                           populations={"positron": n_e, "antiproton": n_p},
                           temperatures={"positron": temp, "antiproton": temp}, cloud_radii=radii)


def test_uniform_ellipsoid_cloud_statistics():
    p = params()
    with amk.Simulation(p) as s:
        s.init_particles_gpu("uniform")
        st = s.get_particles()
    x, y, z = st["x"], st["y"], st["z"]
    sp = None
    a, b, c = 5e-4, 5e-4, 2e-3
    r = (x / a) ** 2 + (y / b) ** 2 + (z / c) ** 2
    assert np.all(r <= 1.0 + 1e-12)
    # uniform ball: <x^2> = a^2 / 5, <r^3> uniform in [0, 1]
    for v, rad in ((x, a), (y, b), (z, c)):
        assert abs(np.mean(v ** 2) / (rad ** 2 / 5) - 1) < 0.02
        assert abs(np.mean(v)) < 0.01 * rad
    rr = r ** 1.5
    assert abs(np.mean(rr) - 0.5) < 0.01
    # species in the reference's order: antiprotons (code 0) first
    with amk.Simulation(p) as s:
        s.init_particles_gpu("uniform")
        n = s.num_particles()
        assert n == 100000
    vel = np.stack([st["vx"], st["vy"], st["vz"]], 1)
    for lo, hi, code in ((0, 40000, 0), (40000, 100000, 1)):
        v = vel[lo:hi]
        sigma2 = KB * 100.0 / MASS[code]
        assert np.max(np.abs(v.mean(0))) <= 1e-12 * np.sqrt(sigma2)  # drift removed exactly
        assert abs(np.mean(v ** 2) / sigma2 - 1) < 0.02


def test_gaussian_cloud_and_determinism():
    p = params(radii=(1e-4, 1e-4, 3e-4))
    with amk.Simulation(p) as s:
        s.init_particles_gpu("gaussian")
        a = s.get_particles()
        s.init_particles_gpu("gaussian")
        b = s.get_particles()
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.array_equal(a[k], b[k])
    for v, sg in ((a["x"], 1e-4), (a["y"], 1e-4), (a["z"], 3e-4)):
        assert abs(np.std(v) / sg - 1) < 0.02
    q = params(radii=(1e-4, 1e-4, 3e-4), seed=8)
    with amk.Simulation(q) as s:
        s.init_particles_gpu("gaussian")
        c = s.get_particles()
    assert not np.array_equal(a["x"], c["x"])


def test_batch_init_equals_instances_generated_alone():
    ps = [params(n_e=300 + 50 * i, n_p=200 + 30 * i, radii=(1e-4 * (1 + i), 2e-4, 3e-4), temp=4.0 * (i + 1),
                 seed=100 + i) for i in range(5)]
    with amk.Simulation() as s:
        s.batch_init(ps, "uniform")
        st = s.get_particles()
        info = s.batch_info()
        assert info["instances"] == 5
        s.batch_step(3)  # the batch is set and steps
    at = 0
    for p in ps:
        with amk.Simulation(p) as s1:
            s1.init_particles_gpu("uniform")
            one = s1.get_particles()
        n = len(one["x"])
        for k in ("x", "y", "z", "vx", "vy", "vz"):
            assert np.array_equal(st[k][at:at + n], one[k])
        at += n
    assert at == len(st["x"])
