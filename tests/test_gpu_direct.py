"""GPU parity of the direct solvers against the FP64 oracle and the
reference's own outputs (golden fixtures)."""
import os

import numpy as np
import pytest

import oracle_lib as O
from conftest import E, gaussian_cloud, rel_errors

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# FP32 pair math with double-float positions and compensated accumulation:
# per-particle |dF|/|F| RMS below 1e-6 against the FP64 oracle.
DIRECT_RMS_TOL = 1e-6
DIRECT_MAX_TOL = 2e-5


def test_allpairs_vs_oracle_mixed(sim):
    x, y, z, q = gaussian_cloud(4096, 1)
    f = sim.solve_allpairs(x, y, z, q)
    g = O.allpairs(x, y, z, q)
    rel, glob = rel_errors(f, g)
    assert np.sqrt(np.mean(rel ** 2)) < DIRECT_RMS_TOL
    assert np.max(rel) < DIRECT_MAX_TOL
    assert glob < DIRECT_RMS_TOL


def test_allpairs_vs_reference_bh_theta0_fixture(sim):
    g = np.load(os.path.join(GOLD, "bh_n2000.npz"))
    fx, fy, fz, phi = sim.solve_allpairs(g["x"], g["y"], g["z"], g["q"], want_phi=True)
    ref = g["f_theta0.0"]
    rel, _ = rel_errors((fx, fy, fz), ref.T)
    assert np.sqrt(np.mean(rel ** 2)) < DIRECT_RMS_TOL
    pref = g["phi_theta0.0"]
    # phi sums +-q/r with ~100x cancellation: bound the error by the scale
    assert np.max(np.abs(phi - pref)) < 2e-6 * np.max(np.abs(pref))


def test_allpairs_ragged_sizes(sim):
    for n in (1, 2, 3, 31, 255, 257, 511, 513, 1000, 2049):
        x, y, z, q = gaussian_cloud(n, n)
        f = sim.solve_allpairs(x, y, z, q)
        if n == 1:
            assert all(np.all(a == 0.0) for a in f)
            continue
        g = O.allpairs(x, y, z, q)
        rel, _ = rel_errors(f, g)
        assert np.sqrt(np.mean(rel ** 2)) < DIRECT_RMS_TOL, n


def test_allpairs_positive_cloud_and_momentum(sim):
    x, y, z, q = gaussian_cloud(8192, 5, mixed=False)
    fx, fy, fz = sim.solve_allpairs(x, y, z, q)
    g = O.allpairs(x, y, z, q)
    rel, _ = rel_errors((fx, fy, fz), g)
    assert np.sqrt(np.mean(rel ** 2)) < DIRECT_RMS_TOL
    # Newton's third law: the net force vanishes to rounding
    tot = np.abs(np.array([fx.sum(), fy.sum(), fz.sum()]))
    assert np.all(tot < 1e-6 * np.sum(np.abs(fx) + np.abs(fy) + np.abs(fz)))


def test_allpairs_edge_cases(sim):
    # duplicated position (r = 0: skipped as in barnes-hut.cc:35), neutral
    # source (q = 0), far outlier
    x = np.array([0.0, 0.0, 1e-5, 2e-5, 5e-3])
    y = np.array([0.0, 0.0, 0.0, 1e-5, 0.0])
    z = np.zeros(5)
    q = np.array([E, -E, E, 0.0, -E])
    f = sim.solve_allpairs(x, y, z, q)
    g = O.allpairs(x, y, z, q)
    # particle 2 feels a dipole whose two terms cancel to 4e-6 of each term:
    # FP32 pair arithmetic resolves forces to ~1e-7 of the largest term
    scale = max(np.max(np.abs(b)) for b in g)
    for a, b in zip(f, g):
        assert np.all(np.isfinite(a))
        assert np.max(np.abs(a - b)) < 1e-7 * scale
    assert f[0][3] == 0.0 and f[1][3] == 0.0  # neutral target gets no force


def test_allpairs_large_sampled(sim):
    x, y, z, q = gaussian_cloud(65536, 9, sigma=(2e-4, 2e-4, 5e-4))
    f = sim.solve_allpairs(x, y, z, q)
    t = np.random.default_rng(0).choice(65536, 512, replace=False)
    g = O.allpairs_subset(x, y, z, q, t)
    rel, _ = rel_errors(tuple(a[t] for a in f), g)
    assert np.sqrt(np.mean(rel ** 2)) < DIRECT_RMS_TOL
    assert np.max(rel) < DIRECT_MAX_TOL


def test_cutoff_vs_oracle(sim):
    x, y, z, q = gaussian_cloud(3000, 2)
    for rc in (2e-5, 5e-5, 1e-4):
        f = sim.solve_cutoff(x, y, z, q, rc)
        g = O.cutoff(x, y, z, q, rc)
        for a, b in zip(f, g):
            assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b)) + 1e-300
    zero = sim.solve_cutoff(x, y, z, q, 0.0)
    assert all(np.all(a == 0.0) for a in zero)


def test_cutoff_huge_radius_equals_allpairs(sim):
    x, y, z, q = gaussian_cloud(1500, 4)
    f = sim.solve_cutoff(x, y, z, q, 1.0)
    g = O.allpairs(x, y, z, q)
    for a, b in zip(f, g):
        assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b))
