"""CPU oracle pinned against the reference: golden fixtures produced by the
reference's own compiled code (tests/golden/make_golden.py), the notebook's
stored step-0 energies and the published Philox known-answer vectors."""
import json
import os

import numpy as np
import pytest

import oracle_lib as O
from conftest import E, gaussian_cloud

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
README_POPS = {"positron": 100, "electron": 100}
README_TEMPS = {"positron": 1e3, "electron": 1e3}
# simulation_analysis.ipynb:161 -- the CSV holds 6 significant digits
NOTEBOOK_STEP0 = {"kinetic": 4.21895e-18, "trap_potential": -3.18438e-22,
                  "coulomb_potential": 5.47464e-24, "num_active": 200}


def sig6(v):
    return float(f"{v:.5e}")


def readme_state():
    g = np.load(os.path.join(GOLD, "readme_ic.npz"))
    pos, vel, sp = g["pos"], g["vel"], g["species"]
    m, q = O.species_props(sp)
    return dict(x=pos[:, 0].copy(), y=pos[:, 1].copy(), z=pos[:, 2].copy(), vx=vel[:, 0].copy(),
                vy=vel[:, 1].copy(), vz=vel[:, 2].copy(), q=q, m=m,
                alive=np.ones(len(sp), np.uint8), species=sp.astype(np.uint8))


def test_philox_known_answers():
    # Random123 philox4x32-10 known-answer vectors
    assert list(O.philox4x32(0, 0, [0, 0, 0, 0])) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert list(O.philox4x32(0xffffffff, 0xffffffff, [0xffffffff] * 4)) == [
        0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert list(O.philox4x32(0xa4093822, 0x299f31d0,
                             [0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344])) == [
        0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]


def test_initial_conditions_match_reference_fixture():
    g = np.load(os.path.join(GOLD, "readme_ic.npz"))
    pos = O.initial_positions(README_POPS, [1e-4] * 3, 42)
    vel = O.initial_velocities(README_POPS, README_TEMPS, 42)
    assert np.array_equal(pos, g["pos"])
    assert np.array_equal(vel, g["vel"])
    assert list(g["species"][:3]) == [1, 1, 1] and list(g["species"][-3:]) == [3, 3, 3]
    # penning_trap.cc:77 -- a fresh mt19937(seed) per species
    assert np.array_equal(vel[:100], vel[100:])


@pytest.mark.skipif(not O.ref_available(), reason="reference build not present")
def test_initial_conditions_match_reference_build():
    pos = O.initial_positions(README_POPS, [1e-4] * 3, 42, use_ref=True)
    assert np.array_equal(pos, O.initial_positions(README_POPS, [1e-4] * 3, 42))


def test_step0_energies_match_notebook():
    e = O.energy_standard(readme_state(), 10.0, 0.01, 0.01, 1e-5)
    for k in ("kinetic", "trap_potential", "coulomb_potential"):
        assert sig6(e[k]) == NOTEBOOK_STEP0[k], (k, e[k])
    assert e["num_active"] == 200


def test_dt_and_cooling_time_known_answers():
    dt = O.dt_for([1, 3], 1.0)  # physics_params.cc:60-74
    assert abs(dt - 8.930966882e-12) / dt < 1e-9
    tau = O.cooling_time(E, 9.1093837015e-31, 1.0)  # README.md:266 "about 2.6 s"
    assert 2.5 < tau < 2.7 and abs(tau - 2.5793) < 1e-3
    period = 2 * np.pi * 9.1093837015e-31 / (E * 1.0)  # "about 36 ps"
    assert abs(period - 35.72e-12) < 0.01e-12
    assert abs(O.dt_for([1, 3], 3.0) - 2.977e-12) < 1e-15


def test_allpairs_oracle_equals_reference_bh_theta0():
    g = np.load(os.path.join(GOLD, "bh_n2000.npz"))
    f = np.stack(O.allpairs(g["x"], g["y"], g["z"], g["q"]), axis=1)
    ref = g["f_theta0.0"]
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(f - ref)) / scale < 1e-12


def test_allpairs_potential_equals_reference_bh_theta0():
    g = np.load(os.path.join(GOLD, "bh_n2000.npz"))
    *_, phi = O.allpairs(g["x"], g["y"], g["z"], g["q"], want_phi=True)
    ref = g["phi_theta0.0"]
    assert np.max(np.abs(phi - ref)) / np.max(np.abs(ref)) < 1e-12


def test_reference_fmm_theta0_is_allpairs():
    g = np.load(os.path.join(GOLD, "fmm_n2000.npz"))
    f = np.stack(O.allpairs(g["x"], g["y"], g["z"], g["q"]), axis=1)
    assert np.max(np.abs(g["f_p4_theta0.0"] - f)) / np.max(np.abs(f)) < 1e-12


def test_reference_error_table_is_ordered():
    err = json.load(open(os.path.join(GOLD, "fmm_n4000_err.json")))["errors"]
    for kind in ("mixed", "positive"):
        assert err[f"{kind}_p2"]["rms"] > err[f"{kind}_p4"]["rms"] > err[f"{kind}_p6"]["rms"]


def test_cutoff_oracle_matches_allpairs_for_huge_cutoff():
    x, y, z, q = gaussian_cloud(500, 3)
    a = O.allpairs(x, y, z, q)
    c = O.cutoff(x, y, z, q, 1.0)
    for u, v in zip(a, c):
        assert np.max(np.abs(u - v)) <= 1e-12 * np.max(np.abs(u))
    zero = O.cutoff(x, y, z, q, 0.0)
    assert all(np.all(v == 0) for v in zero)


def test_boris_conserves_speed_in_pure_b():
    rng = np.random.default_rng(0)
    n = 64
    s = dict(x=np.zeros(n), y=np.zeros(n), z=np.zeros(n), vx=rng.normal(size=n) * 1e3,
             vy=rng.normal(size=n) * 1e3, vz=rng.normal(size=n) * 1e3, q=np.full(n, -E),
             m=np.full(n, 9.1093837015e-31), alive=np.ones(n, np.uint8))
    v0 = np.sqrt(s["vx"] ** 2 + s["vy"] ** 2 + s["vz"] ** 2)
    for k in range(50):  # zero voltage: only the magnetic rotation acts
        O.boris_push(s, np.zeros(n), np.zeros(n), np.zeros(n), 1.0, 0.0, 0.01, 0.01, 1e-12, k == 0)
    v1 = np.sqrt(s["vx"] ** 2 + s["vy"] ** 2 + s["vz"] ** 2)
    assert np.max(np.abs(v1 - v0) / v0) < 1e-13


def test_cooling_noise_moments():
    vals = []
    buf = np.zeros(3)
    for i in range(20000):
        O.lib().orc_cooling_normals(7, i, 3, buf.ctypes.data_as(O._dp))
        vals.append(buf.copy())
    v = np.array(vals)
    assert np.all(np.abs(v.mean(axis=0)) < 0.03)
    assert np.all(np.abs(v.var(axis=0) - 1.0) < 0.04)


def _ann_state(pos, species):
    pos = np.asarray(pos, float)
    n = len(pos)
    return dict(x=pos[:, 0].copy(), y=pos[:, 1].copy(), z=pos[:, 2].copy(),
                species=np.asarray(species, np.uint8), alive=np.ones(n, np.uint8))


def test_annihilation_rule_greedy_in_id_order():
    # chain e+(0) - e-(1) - e+(2) - e-(3), spacing 1e-6 < contact 1.5e-6
    pos = [[0, 0, 0], [1e-6, 0, 0], [2e-6, 0, 0], [3e-6, 0, 0]]
    s = _ann_state(pos, [1, 3, 1, 3])
    marked = O.annihilation(s, 1.5e-6, 1.0, 42, 1)
    assert marked == 4 and list(s["alive"]) == [0, 0, 0, 0]
    # same species never pair; neutral never pairs
    s = _ann_state(pos, [1, 1, 2, 2])
    assert O.annihilation(s, 1.5e-6, 1.0, 42, 1) == 0
    # p = 0 never annihilates
    s = _ann_state(pos, [1, 3, 1, 3])
    assert O.annihilation(s, 1.5e-6, 0.0, 42, 1) == 0
    # e+(0) sits between two e-: it takes the lower id partner
    s = _ann_state([[0, 0, 0], [1e-6, 0, 0], [-1e-6, 0, 0]], [1, 3, 3])
    O.annihilation(s, 1.5e-6, 1.0, 42, 1)
    assert list(s["alive"]) == [0, 0, 1]
    # antiproton / proton
    s = _ann_state([[0, 0, 0], [1e-6, 0, 0]], [0, 4])
    assert O.annihilation(s, 1.5e-6, 1.0, 42, 1) == 2
