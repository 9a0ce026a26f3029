"""amk_run, the native replacement of the reference application's main loop:
the reference's params.json in, the reference's console lines and energy CSV
out (same header, same logging schedule, time-centred energies), computed on
the GPU through the C ABI."""
import csv
import json
import os
import subprocess

import numpy as np
import pytest

import amk
from conftest import ROOT

pytestmark = pytest.mark.gpu
RUN = os.path.join(ROOT, "antimatter-kernel_b200", "amk_run")
HEADER = ["step", "kinetic_energy_J", "trap_potential_energy_J", "potential_energy_J", "total_energy_J",
          "num_active_particles", "fractional_drift", "absolute_drift_J"]
# README-scale run: the parameter file the reference ships
README_PARAMS = {
    "seed": 42, "b0": 1, "trap_voltage": 10, "z0": 0.01, "rho0": 0.01, "num_steps": 1e2,
    "particle_populations": {"positron": 100, "electron": 100},
    "particle_temperatures": {"positron": 1e3, "electron": 1e3},
    "initial_cloud_radii": {"radius_x": 1e-4, "radius_y": 1e-4, "radius_z": 1e-4},
    "bath_temperature": 4, "cooling_scale": 1, "coulomb_forces_enabled": True,
    "coulomb_computation_method": "standard", "energy_computation_method": "standard", "cutoff_radius": 1e-5,
    "barnes_hut_theta": 0.7, "fast_multipole_order": 4, "fast_multipole_theta": 0.5,
    "annihilation_enabled": True, "contact_radius": 5e-6, "annihilation_probability": 1,
}


def run_driver(tmp_path, params):
    if not os.path.exists(RUN):
        subprocess.run(["make", "-s", "-C", os.path.dirname(RUN), "amk_run"], check=True)
    path = tmp_path / "params.json"
    path.write_text(json.dumps(params))
    out = tmp_path / "output"
    out.mkdir()
    res = subprocess.run([RUN, str(path), str(out)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    with open(out / "energy_analysis_data.csv") as f:
        rows = list(csv.reader(f))
    return path, res.stdout, rows


def test_readme_run_csv_and_console(tmp_path):
    path, stdout, rows = run_driver(tmp_path, README_PARAMS)
    assert rows[0] == HEADER
    body = [[float(v) for v in r] for r in rows[1:]]
    assert [int(r[0]) for r in body] == list(range(0, 101))  # num_steps / 100 = 1: every step is logged
    # step 0 equals the reference notebook's stored row (6 printed digits)
    assert body[0][1:4] == [4.21895e-18, -3.18438e-22, 5.47464e-24]
    assert body[0][5] == 200 and body[0][6] == 0.0
    assert "Simulation completed successfully!" in stdout
    assert stdout.count("final position:") == 200
    assert "step 100  KE=" in stdout
    # the same loop through the Python binding gives the same energies
    p = amk.load_params(str(path))
    with amk.Simulation(p) as s:
        s.init_particles()
        e0 = s.energy(time_centre=True)
        ref = {0: e0}
        for step in range(1, 101):
            s.step(1)
            ref[step] = s.energy(time_centre=True)
    scale = 1.602176634e-19 * 10
    for r in body:
        e = ref[int(r[0])]
        want = [e["kinetic"], e["trap_potential"], e["coulomb_potential"], e["total"], e["num_active"],
                (e["total"] - e0["total"]) / scale, e["total"] - e0["total"]]
        for got, w in zip(r[1:], want):
            assert abs(got - w) <= 1e-5 * max(abs(w), 1e-300) + 1e-30, (r[0], got, w)


def test_coulomb_disabled_zeroes_the_coulomb_column(tmp_path):
    params = dict(README_PARAMS, coulomb_forces_enabled=False, num_steps=300)
    _, _, rows = run_driver(tmp_path, params)
    body = np.array([[float(v) for v in r] for r in rows[1:]])
    assert np.all(body[:, 3] == 0.0)
    # 300 steps: logged every 3 steps
    assert list(body[:, 0].astype(int)) == [0] + list(range(3, 301, 3))
