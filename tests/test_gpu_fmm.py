"""GPU Cartesian FMM against the reference's FastMultipoleSolver: forces and
energies from the reference's own code (golden fixtures, N = 2,000), theta = 0
equal to the exact sum, and accuracy against the exact sum no worse than the
reference's at the same order and theta."""
import json
import os

import numpy as np
import pytest

import oracle_lib as O
from conftest import E, gaussian_cloud, rel_errors

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FMM_TOL = 1e-9  # FP64 expansions; only summation order differs from the reference


@pytest.mark.parametrize("order,theta", [(2, 0.5), (4, 0.5), (6, 0.5), (4, 0.0)])
def test_fmm_matches_reference_fixture(sim, order, theta):
    g = np.load(os.path.join(GOLD, "fmm_n2000.npz"))
    f, e = sim.solve_fmm(g["x"], g["y"], g["z"], g["q"], order, theta, want_energy=True)
    ref = g[f"f_p{order}_theta{theta}"].T
    rel, glob = rel_errors(f, ref)
    assert np.max(rel) < FMM_TOL, np.max(rel)
    eref = float(g[f"e_p{order}_theta{theta}"])
    assert abs(e - eref) <= 1e-10 * abs(eref)


def test_fmm_theta0_is_allpairs(sim):
    x, y, z, q = gaussian_cloud(2500, 40)
    f = sim.solve_fmm(x, y, z, q, 3, 0.0)
    rel, _ = rel_errors(f, O.allpairs(x, y, z, q))
    assert np.max(rel) < FMM_TOL


def test_fmm_error_no_worse_than_reference():
    import amk
    err = json.load(open(os.path.join(GOLD, "fmm_n4000_err.json")))["errors"]
    with amk.Simulation() as s:
        for label, mixed in (("mixed", True), ("positive", False)):
            x, y, z, q = gaussian_cloud(4000, 11)
            if not mixed:
                q = np.full(4000, E)
            exact = O.allpairs(x, y, z, q)
            for p in (2, 4, 6):
                f = s.solve_fmm(x, y, z, q, p, 0.5)
                rel, glob = rel_errors(f, exact)
                ref = err[f"{label}_p{p}"]
                assert np.sqrt(np.mean(rel ** 2)) <= ref["rms"] * (1 + 1e-6), (label, p)
                assert glob <= ref["global"] * (1 + 1e-6), (label, p)


def test_fmm_order_clamp_and_leaf_capacity(sim):
    x, y, z, q = gaussian_cloud(1200, 41)
    a = sim.solve_fmm(x, y, z, q, 0, 0.5)
    b = sim.solve_fmm(x, y, z, q, 1, 0.5)
    assert all(np.array_equal(u, v) for u, v in zip(a, b))   # order clamped to [1, 8]
    a = sim.solve_fmm(x, y, z, q, 12, 0.5)
    b = sim.solve_fmm(x, y, z, q, 8, 0.5)
    assert all(np.array_equal(u, v) for u, v in zip(a, b))
    if O.ref_available():
        for cap in (4, 16, 100):
            f = sim.solve_fmm(x, y, z, q, 3, 0.6, leaf_capacity=cap)
            (rx, ry, rz), _ = O.ref_fmm(x, y, z, q, 3, 0.6, cap)
            rel, _ = rel_errors(f, (rx, ry, rz))
            assert np.max(rel) < FMM_TOL, cap


def test_fmm_neutral_and_annihilated_particles():
    import amk
    x, y, z, q = gaussian_cloud(600, 42)
    sp = np.where(q > 0, 1, 3).astype(np.uint8)
    sp[::10] = 2  # antihydrogen: neutral, force 0 (fast-multipole.cc:690)
    p = amk.make_params(populations={"positron": 300, "electron": 300}, annihilation_enabled=1,
                        contact_radius=2e-5, annihilation_probability=1.0)
    with amk.Simulation(p) as s:
        s.set_particles(x, y, z, np.zeros(600), np.zeros(600), np.zeros(600), sp)
        s.annihilate()
        alive = s.get_particles()["alive"].astype(bool)
        s.coulomb_fmm(4, 0.5)
        f = s.get_forces()
        charged = alive & (sp != 2)
        assert np.all(f[0][~charged] == 0.0)
        qq = np.where(sp == 1, E, -E)
        if O.ref_available():
            (rx, ry, rz), _ = O.ref_fmm(x[charged], y[charged], z[charged], qq[charged], 4, 0.5)
            rel, _ = rel_errors(tuple(a[charged] for a in f), (rx, ry, rz))
            assert np.max(rel) < FMM_TOL


def test_fmm_energy_method_in_context():
    import amk
    g = np.load(os.path.join(GOLD, "fmm_n2000.npz"))
    n = len(g["x"])
    sp = np.where(g["q"] > 0, 1, 3).astype(np.uint8)
    p = amk.make_params(populations={"positron": n // 2, "electron": n - n // 2},
                        energy_method="fast-multipole", fast_multipole_order=4.0,
                        fast_multipole_theta=0.5)
    with amk.Simulation(p) as s:
        s.set_particles(g["x"], g["y"], g["z"], np.zeros(n), np.zeros(n), np.zeros(n), sp)
        e = s.energy(time_centre=False)
        eref = float(g["e_p4_theta0.5"])
        assert abs(e["coulomb_potential"] - eref) <= 1e-10 * abs(eref)


def test_fmm_above_a_million_particles_matches_reference(sim):
    # more than 2^20 sources: the radix sorts of the tree keys and of the
    # interaction pairs take their multi-CTA histogram-scan path
    if not O.ref_available():
        pytest.skip("reference library not built")
    x, y, z, _ = gaussian_cloud(1_100_000, 77)
    q = np.full(len(x), E)
    f = sim.solve_fmm(x, y, z, q, 2, 0.5)
    (rx, ry, rz), _ = O.ref_fmm(x, y, z, q, 2, 0.5, 32)
    rel, _ = rel_errors(f, (rx, ry, rz))
    assert np.max(rel) < FMM_TOL


@pytest.mark.parametrize("reach,chunk", [(1, None), (3, None), (None, 1000), (2, 777)])
def test_fmm_per_pair_path_and_chunk_seams(sim, monkeypatch, reach, chunk):
    # M2L pairs run as per-class products; a narrowed class reach sends the
    # pairs beyond it through the per-pair recurrence path, and a small chunk
    # size splits targets' pair lists across chunks
    g = np.load(os.path.join(GOLD, "fmm_n2000.npz"))
    if reach is not None:
        monkeypatch.setenv("AMK_FMM_M2L_REACH", str(reach))
    if chunk is not None:
        monkeypatch.setenv("AMK_FMM_M2L_CHUNK_PAIRS", str(chunk))
    for order in (2, 6):
        f = sim.solve_fmm(g["x"], g["y"], g["z"], g["q"], order, 0.5)
        rel, _ = rel_errors(f, g[f"f_p{order}_theta0.5"].T)
        assert np.max(rel) < FMM_TOL, (order, np.max(rel))


@pytest.mark.parametrize("order", [7, 8])
def test_fmm_high_orders_match_reference(sim, order):
    if not O.ref_available():
        pytest.skip("reference library not built")
    x, y, z, q = gaussian_cloud(3000, 43)
    f = sim.solve_fmm(x, y, z, q, order, 0.5)
    (rx, ry, rz), _ = O.ref_fmm(x, y, z, q, order, 0.5, 32)
    rel, _ = rel_errors(f, (rx, ry, rz))
    assert np.max(rel) < FMM_TOL, np.max(rel)


def test_fmm_off_origin_cloud_at_order_8(sim):
    # a cloud centred far from the origin (1e3 sigma): the unit-cube frame
    # subtracts the box centre, and lattice classes must not accept pairs
    # whose centres are off the lattice by more than their rounding
    if not O.ref_available():
        pytest.skip("reference library not built")
    x, y, z, q = gaussian_cloud(3000, 44)
    x, y, z = x + 0.1, y - 0.1, z + 0.3
    f = sim.solve_fmm(x, y, z, q, 8, 0.5)
    (rx, ry, rz), _ = O.ref_fmm(x, y, z, q, 8, 0.5, 32)
    rel, _ = rel_errors(f, (rx, ry, rz))
    assert np.max(rel) < FMM_TOL, np.max(rel)


@pytest.mark.parametrize("order", [5, 6, 7])
def test_tensor_core_products_match_the_fp64_path(order):
    # split-BF16 tcgen05 class products (FP32 per-pair products): the forces
    # stay within 1e-6 RMS (1e-5 at worst) of the FP64 products and the error
    # against the exact sum is unchanged
    import amk
    x, y, z, q = gaussian_cloud(20000, 45, mixed=False)
    exact = O.allpairs(x, y, z, q)
    with amk.Simulation() as s:
        ref = s.solve_fmm(x, y, z, q, order, 0.5)
        s.set_fmm_precision("tensor")
        got = s.solve_fmm(x, y, z, q, order, 0.5)
        st = s.fmm_stats()
        assert st["m2l_class_pairs"] > 0
        again = s.solve_fmm(x, y, z, q, order, 0.5)
    assert all(np.array_equal(a, b) for a, b in zip(got, again))  # run-to-run deterministic
    rel, _ = rel_errors(got, ref)
    assert np.sqrt(np.mean(rel ** 2)) < 1e-6 and np.max(rel) < 1e-5, (np.sqrt(np.mean(rel ** 2)), np.max(rel))
    e_ref = np.sqrt(np.mean(rel_errors(ref, exact)[0] ** 2))
    e_tc = np.sqrt(np.mean(rel_errors(got, exact)[0] ** 2))
    assert e_tc <= 1.02 * e_ref + 1e-7, (e_tc, e_ref)


def test_tensor_core_products_with_per_pair_path_and_chunk_seams(sim, monkeypatch):
    # pairs outside the classes (narrowed reach) and chunk seams in the
    # tensor-core mode, against the reference's FMM at p=6
    import amk
    g = np.load(os.path.join(GOLD, "fmm_n2000.npz"))
    monkeypatch.setenv("AMK_FMM_M2L_REACH", "2")
    monkeypatch.setenv("AMK_FMM_M2L_CHUNK_PAIRS", "1500")
    with amk.Simulation() as s:
        s.set_fmm_precision("tensor")
        f = s.solve_fmm(g["x"], g["y"], g["z"], g["q"], 6, 0.5)
    # mixed charges: far fields partly cancel, so the bound is on the global
    # ratio ||dF|| / ||F|| (per particle on the cancelled ones it is larger)
    rel, glob = rel_errors(f, g["f_p6_theta0.5"].T)
    assert glob < 1e-6 and np.max(rel) < 1e-4, (glob, np.max(rel))


def test_traversal_overflow_retry_gives_the_same_forces(monkeypatch):
    # the traversal's lists start at 64 entries, so its first passes overflow
    # and it runs again with larger lists: the same forces, bit for bit
    import amk
    x, y, z, q = gaussian_cloud(20000, 47, mixed=False)
    with amk.Simulation() as s:
        base = s.solve_fmm(x, y, z, q, 4, 0.5)
        st0 = s.fmm_stats()
        monkeypatch.setenv("AMK_FMM_LIST_CAP", "64")
        got = s.solve_fmm(x, y, z, q, 4, 0.5)
        st1 = s.fmm_stats()
    assert all(np.array_equal(a, b) for a, b in zip(base, got))
    assert st0["m2l_pairs"] == st1["m2l_pairs"] and st0["p2p_leaf_pairs"] == st1["p2p_leaf_pairs"]


def test_tensor_mode_takes_at_least_the_fp64_class_pairs():
    # the tensor-core mode folds classes below 4 pairs by reflection, so at
    # least as many pairs are class products as in the FP64 mode, the same
    # M2L pairs in total
    import amk
    x, y, z, q = gaussian_cloud(20000, 45, mixed=False)
    with amk.Simulation() as s:
        s.solve_fmm(x, y, z, q, 6, 0.5)
        fp64 = s.fmm_stats()
        s.set_fmm_precision("tensor")
        s.solve_fmm(x, y, z, q, 6, 0.5)
        tc = s.fmm_stats()
    assert tc["m2l_pairs"] == fp64["m2l_pairs"]
    assert tc["m2l_class_pairs"] >= fp64["m2l_class_pairs"], (tc, fp64)
