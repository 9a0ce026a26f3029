"""C-ABI checks that need no GPU: the library loads, exports every symbol
include/amk.h declares, parses params.json with the reference's keys and
quirks, validates like the reference, and fails loudly without a device."""
import ctypes as C
import json
import os
import re
import subprocess

import numpy as np
import pytest

import amk

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "amk.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(amk_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = amk.lib()
    names = declared_symbols()
    assert len(names) > 30
    out = subprocess.run(["nm", "-D", "--defined-only", amk.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r" T (amk_\w+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    for n in names:
        getattr(lib, n)


def test_library_is_sm100a():
    out = subprocess.run(["cuobjdump", "--list-elf", amk.LIB_PATH], capture_output=True, text=True)
    if out.returncode == 0:
        assert "sm_100a" in out.stdout


def write_params(tmp_path, **over):
    base = {"seed": 42, "b0": 1, "trap_voltage": 10, "z0": 0.01, "rho0": 0.01, "num_steps": 1e2,
            "particle_populations": {"positron": 100, "electron": 100},
            "particle_temperatures": {"positron": 1e3, "electron": 1e3},
            "initial_cloud_radii": {"radius_x": 1e-4, "radius_y": 1e-4, "radius_z": 1e-4},
            "bath_temperature": 4, "cooling_scale": 1, "coulomb_forces_enabled": True,
            "coulomb_computation_method": "standard", "energy_computation_method": "standard",
            "cutoff_radius": 1e-5, "barnes_hut_theta": 0.7, "fast_multipole_order": 4,
            "fast_multipole_theta": 0.5, "annihilation_enabled": True, "contact_radius": 5e-6,
            "annihilation_probability": 1}
    base.update(over)
    path = tmp_path / "params.json"
    path.write_text(json.dumps(base))
    return str(path)


def test_params_json_readme_config(tmp_path):
    p = amk.load_params(write_params(tmp_path))
    assert p.seed == 42 and p.b0 == 1.0 and p.trap_voltage == 10.0
    assert p.num_steps == 100 and p.n_species == 2
    assert [p.species[i] for i in range(2)] == [1, 3]
    assert [p.populations[i] for i in range(2)] == [100, 100]
    assert abs(p.dt - 8.930966882e-12) / p.dt < 1e-9  # physics_params.cc:60-74
    assert p.coulomb_method == 0 and p.cutoff_radius == 1e-5
    assert p.annihilation_enabled == 1 and p.contact_radius == 5e-6
    assert p.fast_multipole_order == 4.0
    amk.validate_params(p)


def test_params_quirks(tmp_path):
    # temperatures are read as integers (physics_params.cc:81)
    p = amk.load_params(write_params(tmp_path, particle_temperatures={"positron": 4.7, "electron": 1e3}))
    assert p.temperatures[0] == 4.0
    # README spellings of the method names are accepted
    p = amk.load_params(write_params(tmp_path, coulomb_computation_method="barnes_hut"))
    assert p.coulomb_method == 1
    with pytest.raises(amk.AmkError):
        amk.load_params(write_params(tmp_path, coulomb_computation_method="tree"))
    with pytest.raises(amk.AmkError):
        amk.load_params(write_params(tmp_path, particle_populations={"muon": 3}))
    with pytest.raises(amk.AmkError):
        amk.load_params(str(tmp_path / "missing.json"))


def test_params_validation_rules(tmp_path):
    p = amk.load_params(write_params(tmp_path))
    bad = [("b0", 0.0), ("z0", -1.0), ("bath_temperature", -1.0), ("cutoff_radius", 0.0),
           ("contact_radius", 0.0), ("annihilation_probability", 1.5)]
    for key, val in bad:
        q = amk.load_params(write_params(tmp_path))
        setattr(q, key, val)
        with pytest.raises(amk.AmkError):
            amk.validate_params(q)
    q = amk.load_params(write_params(tmp_path, cooling_scale=10))
    with pytest.raises(amk.AmkError):
        amk.validate_params(q, strict=True)  # physics_params.cc:139
    amk.validate_params(q, strict=False)
    q = amk.load_params(write_params(tmp_path, coulomb_computation_method="fast-multipole",
                                     energy_computation_method="fast-multipole",
                                     fast_multipole_order=9))
    with pytest.raises(amk.AmkError):
        amk.validate_params(q)


def test_host_helpers():
    m, q = amk.species_properties(3)
    assert m == 9.1093837015e-31 and q == -1.602176634e-19
    assert amk.species_properties(2)[1] == 0.0
    d = amk.lib().amk_trap_dimension(0.01, 0.01)
    assert abs(d - np.sqrt(0.01 ** 2 / 2 + 0.01 ** 2 / 4)) < 1e-18
    tau = amk.lib().amk_cooling_time(1.602176634e-19, 9.1093837015e-31, 1.0)
    assert abs(tau - 2.5793) < 1e-3


def test_context_fails_loudly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(amk.AmkError, match="cuda"):
        amk.Simulation()
