"""Generates the golden fixtures in this directory from the reference itself.

The reference's own ``barnes-hut.cc``, ``fast-multipole.cc`` and
``penning_trap.cc`` are compiled in place (``make -C oracle ref``) and called
through ``oracle/oracle_lib.py``. Run from the repository root on a machine
that has the reference tree:

    python tests/golden/make_golden.py

Fixtures (all inputs seeded, all outputs from the reference's code):
  readme_ic.npz   README-scale initial cloud (100 e+ + 100 e-, seed 42)
  bh_n2000.npz    Barnes-Hut forces (theta 0, 0.5, 0.7), potentials and the
                  octree of a 2,000-charge Gaussian cloud
  fmm_n2000.npz   FMM forces and energies (p = 2, 4, 6 at theta 0.5; p = 4 at
                  theta 0) on the same cloud
  fmm_n4000_err.json  the reference's RMS relative force error against the
                  exact sum for p = 2, 4, 6 at theta 0.5 (N = 4,000 Gaussian)
  readme_steps_ref.npz  the README-scale run (params of the README: cutoff
                  1e-5 m, cooling at 4 K, annihilation 5e-6 m with p = 1,
                  seed 42) stepped 40 times by the reference's own per-step
                  code: ComputeStandardCoulombForces, then LorentzForce,
                  CyclotronCooling and AnnihilationInteraction on every agent
                  (coulomb_interaction.cc, lorentz.cc, cooling.cc,
                  annihilation.cc via oracle/ref_behaviours.cc, whose Random
                  stand-in replays the CUDA library's Philox draws); positions,
                  velocities and alive flags after every step

`python tests/golden/make_golden.py readme_steps` regenerates only the last.
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle_lib as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
E = 1.602176634e-19


def gaussian_cloud(n, seed, sigma=(1e-4, 1e-4, 3e-4)):
    rng = np.random.default_rng(seed)
    x = rng.normal(0.0, sigma[0], n)
    y = rng.normal(0.0, sigma[1], n)
    z = rng.normal(0.0, sigma[2], n)
    q = np.where(rng.random(n) < 0.5, E, -E)
    return x, y, z, q


def errors(f, g):
    num = np.sqrt(sum((a - b) ** 2 for a, b in zip(f, g)))
    den = np.sqrt(sum(b ** 2 for b in g))
    return {"rms": float(np.sqrt(np.mean((num / den) ** 2))),
            "global": float(np.sqrt(np.sum(num ** 2) / np.sum(den ** 2)))}


def main():
    O.build(ref=True)
    # README-scale cloud from the reference's own generators
    pops = {"positron": 100, "electron": 100}
    temps = {"positron": 1e3, "electron": 1e3}
    pos = O.initial_positions(pops, [1e-4, 1e-4, 1e-4], 42, use_ref=True)
    vel = O.initial_velocities(pops, temps, 42, use_ref=True)
    np.savez_compressed(os.path.join(OUT, "readme_ic.npz"), pos=pos, vel=vel,
                        species=O.species_column(pops))

    x, y, z, q = gaussian_cloud(2000, 7)
    bh = {"x": x, "y": y, "z": z, "q": q}
    for th in (0.0, 0.5, 0.7):
        f = O.ref_bh_forces(x, y, z, q, th, 8)
        bh[f"f_theta{th}"] = np.stack(f, axis=1)
    bh["phi_theta0.5"] = O.ref_bh_potentials(x, y, z, q, 0.5, 8)
    bh["phi_theta0.0"] = O.ref_bh_potentials(x, y, z, q, 0.0, 8)
    nf, ni, order = O.ref_bh_tree(x, y, z, q, 8)
    bh["tree_f"] = nf
    bh["tree_i"] = ni
    np.savez_compressed(os.path.join(OUT, "bh_n2000.npz"), **bh)

    fm = {"x": x, "y": y, "z": z, "q": q}
    for p, th in ((2, 0.5), (4, 0.5), (6, 0.5), (4, 0.0)):
        f, e = O.ref_fmm(x, y, z, q, p, th, 32, forces=True, energy=True)
        fm[f"f_p{p}_theta{th}"] = np.stack(f, axis=1)
        fm[f"e_p{p}_theta{th}"] = np.array(e)
    np.savez_compressed(os.path.join(OUT, "fmm_n2000.npz"), **fm)

    # Reference accuracy at N = 4,000 (Gaussian sigma 1e-4, 1e-4, 3e-4 m) for
    # a mixed +-e cloud and a positron-only cloud: per-particle RMS of
    # |dF|/|F| ("rms") and the global norm ratio ||dF|| / ||F|| ("global").
    err = {}
    for label, mixed in (("mixed", True), ("positive", False)):
        x4, y4, z4, q4 = gaussian_cloud(4000, 11)
        if not mixed:
            q4 = np.full(4000, E)
        exact = O.allpairs(x4, y4, z4, q4)
        for p in (2, 4, 6):
            f, _ = O.ref_fmm(x4, y4, z4, q4, p, 0.5, 32)
            err[f"{label}_p{p}"] = errors(f, exact)
        f = O.ref_bh_forces(x4, y4, z4, q4, 0.7, 8)
        err[f"{label}_bh0.7"] = errors(f, exact)
    with open(os.path.join(OUT, "fmm_n4000_err.json"), "w") as fh:
        json.dump({"seed": 11, "n": 4000, "sigma": [1e-4, 1e-4, 3e-4], "fmm_theta": 0.5,
                   "errors": err}, fh, indent=1)
    print(json.dumps(err))


def readme_steps(steps=40):
    O.build(ref=True)
    g = np.load(os.path.join(OUT, "readme_ic.npz"))
    sp = g["species"]
    dt = O.dt_for([1, 3], 1.0)
    w = O.RefWorld(g["pos"], g["vel"], sp, b0=1.0, voltage=10.0, z0=0.01, rho0=0.01, dt=dt,
                   cooling_scale=1.0, bath_temp=4.0, annihilation=True, contact_radius=5e-6,
                   probability=1.0, seed=42)
    out = {k: [] for k in ("x", "y", "z", "vx", "vy", "vz", "alive")}
    for step in range(1, steps + 1):
        w.coulomb_standard(1e-5)
        w.behaviours(step)
        st = w.state()
        for k in out:
            out[k].append(st[k])
    np.savez_compressed(os.path.join(OUT, "readme_steps_ref.npz"), dt=dt,
                        **{k: np.array(v) for k, v in out.items()})
    print("readme_steps: alive after", steps, "steps:", int(out["alive"][-1].sum()))


if __name__ == "__main__":
    if sys.argv[1:] == ["readme_steps"]:
        readme_steps()
    else:
        main()
        readme_steps()
