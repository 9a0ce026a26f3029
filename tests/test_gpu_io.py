"""Checkpoint/resume and particle export on the GPU: a context restored from
a checkpoint continues bit for bit like the saved one (cutoff + cooling +
annihilation, all-pairs with its Morton order, FMM); corrupt files are
refused; the exported .vtu holds the live particles; the driver resumes a
checkpointed run with the uninterrupted run's CSV rows."""
import json
import os
import subprocess

import numpy as np
import pytest

import amk
from test_gpu_driver import README_PARAMS
from test_gpu_step import readme_params
from test_io import read_vtu

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _state(s):
    st = s.get_particles()
    st["f"] = np.stack(s.get_forces())
    return st


def _same(a, b):
    for k in ("x", "y", "z", "vx", "vy", "vz", "alive", "f"):
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("over", [
    dict(),  # README run: cutoff forces, cooling at 4 K, annihilation
    dict(coulomb_method="allpairs", annihilation_enabled=0),
    dict(coulomb_method="fast-multipole", fast_multipole_order=4, fast_multipole_theta=0.5),
])
def test_checkpoint_resume_is_bit_exact(tmp_path, over):
    path = str(tmp_path / "run.ckpt")
    p = readme_params(**over)
    with amk.Simulation(p) as s:
        s.init_particles()
        s.step(6)
        s.energy()  # a time-centring history to carry over
        s.step(1)
        s.checkpoint_save(path)
        e_after = s.energy()
        s.step(9)
        want = _state(s)
        e_want = s.energy()
    n, step, q = amk.checkpoint_info(path)
    assert (n, step) == (200, 7) and q.coulomb_method == p.coulomb_method
    with amk.Simulation() as r:  # default parameters: the file replaces them
        r.checkpoint_load(path)
        assert r.step_count() == 7 and r.params.cooling_scale == p.cooling_scale
        assert r.energy() == e_after  # the time-centring history was restored
        r.step(9)
        _same(_state(r), want)
        assert r.energy() == e_want


def test_corrupt_and_truncated_checkpoints_are_refused(tmp_path):
    path = str(tmp_path / "a.ckpt")
    with amk.Simulation(readme_params()) as s:
        s.init_particles()
        s.step(2)
        s.checkpoint_save(path)
        raw = bytearray(open(path, "rb").read())
        raw[len(raw) // 2] ^= 0x40
        open(path + ".bad", "wb").write(bytes(raw))
        open(path + ".cut", "wb").write(bytes(raw[: len(raw) - 100]))
        before = s.get_particles()
        for bad in (path + ".bad", path + ".cut"):
            with pytest.raises(amk.AmkError):
                s.checkpoint_load(bad)
            after = s.get_particles()  # a refused file leaves the context untouched
            assert np.array_equal(before["x"], after["x"])


def test_export_vtk_holds_the_live_particles(tmp_path):
    path = str(tmp_path / "p.vtu")
    with amk.Simulation(readme_params(contact_radius=2e-5)) as s:
        s.init_particles()
        s.step(3)
        st = s.get_particles()
        s.export_vtk(path)
    d = read_vtu(path)
    live = st["alive"].astype(bool)
    assert 0 < live.sum() < 200
    assert np.array_equal(d["Points"], np.stack([st["x"], st["y"], st["z"]], 1)[live])
    assert np.array_equal(d["id"], np.nonzero(live)[0].astype(np.uint32))
    assert abs(d["_time"] - 3 * readme_params().dt) <= 1e-25


def test_driver_resume_reproduces_the_uninterrupted_run(tmp_path):
    exe = os.path.join(ROOT, "antimatter-kernel_b200", "amk_run")
    params = tmp_path / "params.json"
    params.write_text(json.dumps(dict(README_PARAMS, num_steps=20)))
    env = dict(os.environ, AMK_RUN_NO_POSITIONS="1")
    full, part = tmp_path / "full", tmp_path / "part"
    full.mkdir()
    part.mkdir()
    subprocess.run([exe, str(params), str(full), "--vtk-every", "10"], check=True, env=env, capture_output=True)
    ck = str(tmp_path / "c.ckpt")
    # the interrupted run: checkpoints every 8 steps, "crashes" after step 12
    p12 = tmp_path / "params12.json"
    p12.write_text(json.dumps(dict(README_PARAMS, num_steps=12)))
    subprocess.run([exe, str(p12), str(part), "--checkpoint", ck, "--checkpoint-every", "8"], check=True, env=env,
                   capture_output=True)
    n, step, _ = amk.checkpoint_info(ck)
    assert step == 8
    # resume from step 8 with the full run's step count: rows after step 8 are appended
    lines = (part / "energy_analysis_data.csv").read_text().splitlines()
    keep = [ln for ln in lines if not ln[0].isdigit() or int(ln.split(",")[0]) <= 8]
    (part / "energy_analysis_data.csv").write_text("\n".join(keep) + "\n")
    # the run length comes from the params file given on resume
    subprocess.run([exe, str(params), str(part), "--resume", ck], check=True, env=env, capture_output=True)
    assert (part / "energy_analysis_data.csv").read_text() == (full / "energy_analysis_data.csv").read_text()
    pvd = (full / "particles.pvd").read_text()
    assert "particles_0.vtu" in pvd and "particles_20.vtu" in pvd
    assert read_vtu(str(full / "particles_20.vtu"))["_n"] <= 200
