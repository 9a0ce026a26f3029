"""The long run at scale, at a size a test can afford (20,000 particles,
300 steps): learned p=2 with the direct-sum audit and its p=6 fallback
against plain p=6, cooling and annihilation on, FP64 total-energy drift
logged every 100 steps as the reference's driver does
(antimatter-kernel.cc:137-142, 180-182). The learned correction misses the
1e-5 budget, so the first audit (before step 1) switches the run to plain
p=6 and the two drift series agree exactly; with the audit disabled the
learned run's drift stays within 1e-3 of the trap depth of plain p=6's."""
import numpy as np
import pytest
import torch

import amk
import bench

pytestmark = pytest.mark.gpu


def _run(learned, audit_interval=100, steps=300):
    p = bench.long_params(learned, n_half=10000)
    p.learned_audit_interval = audit_interval
    with amk.Simulation(p) as s:
        s.init_particles_gpu("uniform")
        if learned:
            s.fmm_train_correction(0.5, sample_leaves=256, steps=300, batch=2048, lr=1e-3)
        stream = torch.cuda.ExternalStream(s.stream(), device=torch.device("cuda", 0))
        _, _, rows = bench.long_run(s, stream, steps, 100)
        state = s.fmm_learned_state() if learned else None
    return rows, state


def test_learned_with_fallback_matches_plain_p6_drift():
    plain, _ = _run(False)
    learned, st = _run(True)
    assert st["trained"] and st["fallback"] and st["last_error"] > 1e-5
    assert [r["step"] for r in learned] == [0, 100, 200, 300]
    for a, b in zip(learned, plain):
        assert a["total_J"] == b["total_J"] and a["alive"] == b["alive"]
    assert all(np.isfinite(r["fractional_drift"]) for r in plain)


def test_learned_without_audit_tracks_plain_p6_drift():
    plain, _ = _run(False)
    learned, st = _run(True, audit_interval=0)
    assert st["trained"] and not st["fallback"]
    gap = max(abs(a["fractional_drift"] - b["fractional_drift"]) for a, b in zip(learned, plain))
    assert gap < 1e-3, gap
