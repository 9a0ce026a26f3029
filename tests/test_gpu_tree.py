"""GPU Barnes-Hut against the reference: the octree is node-for-node the
reference's BarnesHutTree (same order, centres, sizes, ranges, children),
and forces/potentials match the reference's outputs (golden fixtures) to
FP64 summation-order rounding."""
import os

import numpy as np
import pytest

import oracle_lib as O
from conftest import E, gaussian_cloud, rel_errors

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
BH_TOL = 1e-10  # FP64 walk: only the summation order differs from the reference


def test_bh_tree_is_the_reference_tree(sim):
    g = np.load(os.path.join(GOLD, "bh_n2000.npz"))
    f, i = sim.bh_tree(g["x"], g["y"], g["z"], g["q"], 8)
    rf, ri = g["tree_f"], g["tree_i"]
    assert f.shape == rf.shape, (f.shape, rf.shape)
    assert np.array_equal(i, ri)                      # children, begin, end, is_leaf
    assert np.array_equal(f[:, :4], rf[:, :4])        # centres and half sizes, bit-exact
    assert np.allclose(f[:, 4:6], rf[:, 4:6], rtol=1e-13, atol=0)
    cen = np.abs(rf[:, 6:12]).max()
    assert np.max(np.abs(f[:, 6:12] - rf[:, 6:12])) <= 1e-12 * cen


@pytest.mark.parametrize("theta", [0.0, 0.5, 0.7])
def test_bh_forces_match_reference_fixture(sim, theta):
    g = np.load(os.path.join(GOLD, "bh_n2000.npz"))
    f = sim.solve_barnes_hut(g["x"], g["y"], g["z"], g["q"], theta)
    ref = g[f"f_theta{theta}"].T
    rel, glob = rel_errors(f, ref)
    assert np.max(rel) < BH_TOL, np.max(rel)


def test_bh_potentials_match_reference_fixture(sim):
    g = np.load(os.path.join(GOLD, "bh_n2000.npz"))
    for theta in (0.0, 0.5):
        *_, phi = sim.solve_barnes_hut(g["x"], g["y"], g["z"], g["q"], theta, want_phi=True)
        ref = g[f"phi_theta{theta}"]
        assert np.max(np.abs(phi - ref)) <= 1e-10 * np.max(np.abs(ref))


def test_bh_theta0_is_allpairs(sim):
    x, y, z, q = gaussian_cloud(3000, 21)
    f = sim.solve_barnes_hut(x, y, z, q, 0.0)
    g = O.allpairs(x, y, z, q)
    rel, _ = rel_errors(f, g)
    assert np.max(rel) < BH_TOL


def test_bh_leaf_capacities_and_neutral_sources(sim):
    x, y, z, q = gaussian_cloud(1500, 22)
    q[::7] = 0.0  # neutral particles sit in the tree but carry no charge
    for cap in (1, 3, 8, 64):
        f, i = sim.bh_tree(x, y, z, q, cap)
        if O.ref_available():
            rf, ri, _ = O.ref_bh_tree(x, y, z, q, cap)
            assert np.array_equal(i, ri) and np.array_equal(f[:, :4], rf[:, :4])
        fx = sim.solve_barnes_hut(x, y, z, q, 0.6, leaf_capacity=cap)
        if O.ref_available():
            ref = O.ref_bh_forces(x, y, z, q, 0.6, cap)
            rel, _ = rel_errors(fx, ref)
            assert np.max(rel) < BH_TOL
        assert np.all(fx[0][q == 0.0] == 0.0)


def test_bh_small_and_degenerate_sets(sim):
    for n in (1, 2, 8, 9):
        x, y, z, q = gaussian_cloud(n, 30 + n)
        f = sim.solve_barnes_hut(x, y, z, q, 0.5)
        g = O.allpairs(x, y, z, q)
        for a, b in zip(f, g):
            assert np.allclose(a, b, rtol=1e-12, atol=0)
    # all particles at one point: half clamps to 1e-30, every pair is skipped
    x = np.zeros(20)
    f = sim.solve_barnes_hut(x, x, x, np.full(20, E), 0.5)
    assert all(np.all(a == 0.0) for a in f)


def test_bh_large_cloud_against_reference_build(sim):
    if not O.ref_available():
        pytest.skip("reference build not present")
    x, y, z, q = gaussian_cloud(50000, 23, mixed=False)
    f = sim.solve_barnes_hut(x, y, z, q, 0.7)
    ref = O.ref_bh_forces(x, y, z, q, 0.7)
    rel, _ = rel_errors(f, ref)
    assert np.max(rel) < BH_TOL


def test_context_barnes_hut_skips_annihilated(sim):
    import amk
    x, y, z, q = gaussian_cloud(400, 24)
    sp = np.where(q > 0, 1, 3).astype(np.uint8)
    p = amk.make_params(populations={"positron": 200, "electron": 200}, coulomb_method="barnes-hut",
                        barnes_hut_theta=0.5, annihilation_enabled=1, contact_radius=2e-5,
                        annihilation_probability=1.0)
    with amk.Simulation(p) as s:
        s.set_particles(x, y, z, np.zeros(400), np.zeros(400), np.zeros(400), sp)
        s.annihilate()
        alive = s.get_particles()["alive"].astype(bool)
        assert 0 < alive.sum() < 400
        s.coulomb_barnes_hut(0.5)
        f = s.get_forces()
        assert np.all(f[0][~alive] == 0.0)
        ref = O.ref_bh_forces(x[alive], y[alive], z[alive], q[alive], 0.5) if O.ref_available() else None
        if ref is not None:
            rel, _ = rel_errors(tuple(a[alive] for a in f), ref)
            assert np.max(rel) < BH_TOL


def test_bh_fp32_leaf_sums_in_tensor_mode():
    # tensor precision mode: FP32 leaf sums on double-float differences,
    # FP64 opening test and monopoles; forces and potentials stay within
    # FP32 rounding of the FP64 walk (mixed charges, neutral sources)
    import amk
    x, y, z, q = gaussian_cloud(20000, 23)
    q[::11] = 0.0
    with amk.Simulation() as s:
        ref = s.solve_barnes_hut(x, y, z, q, 0.6, want_phi=True)
        s.set_fmm_precision("tensor")
        got = s.solve_barnes_hut(x, y, z, q, 0.6, want_phi=True)
        again = s.solve_barnes_hut(x, y, z, q, 0.6, want_phi=True)
    assert all(np.array_equal(a, b) for a, b in zip(got, again))  # deterministic
    rel, glob = rel_errors(got[:3], ref[:3])
    assert glob < 1e-6 and np.sqrt(np.mean(rel ** 2)) < 1e-5, (glob, np.sqrt(np.mean(rel ** 2)))
    assert np.all(got[0][q == 0.0] == 0.0)
    assert np.max(np.abs(got[3] - ref[3])) <= 1e-6 * np.max(np.abs(ref[3]))
