"""Learned p=2 FMM correction: trained on the GPU by the library's own
kernels on FP64 exact residuals, audited against the exact sum, and
replaced by plain FMM when an audit exceeds the error budget (including
after deliberately corrupted weights)."""
import numpy as np
import pytest

import amk
from conftest import E, gaussian_cloud

pytestmark = pytest.mark.gpu


def cloud_sim(n=65536, seed=50, **over):
    x, y, z, _ = gaussian_cloud(n, seed, mixed=False)
    kw = dict(populations={"positron": n}, coulomb_method="fast-multipole", fast_multipole_order=2.0,
              fast_multipole_theta=0.5, fmm_learned=1, cooling_enabled=0)
    kw.update(over)
    s = amk.Simulation(amk.make_params(**kw))
    s.set_particles(x, y, z, np.zeros(n), np.zeros(n), np.zeros(n), np.ones(n, np.uint8))
    return s


def test_training_and_measured_gain_on_a_held_out_cloud():
    # trained on one cloud (all of its particles), audited on it and on a
    # second cloud of the same shape (another seed): the correction must
    # reduce the p=2 error by at least 10 % on the cloud it was trained on and
    # by at least 5 % on the held-out one (measured: about 20 % and 11 %). The
    # gain stays far from the 1e-5 budget because the p=2 residual is
    # dominated by the source cells' dropped moments, which per-particle
    # features cannot see; a network that learned nothing fails both bounds.
    with cloud_sim() as s:
        plain = s.fmm_audit(2, 0.5, False, 2048)
        loss, samples = s.fmm_train_correction(0.5, sample_leaves=4096, steps=8000, batch=4096, lr=5e-4)
        assert samples == 65536 and np.isfinite(loss)
        learned = s.fmm_audit(2, 0.5, True, 2048)
        assert s.fmm_learned_state()["trained"]
        x, y, z, _ = gaussian_cloud(65536, 51, mixed=False)
        s.set_particles(x, y, z, np.zeros(65536), np.zeros(65536), np.zeros(65536), np.ones(65536, np.uint8))
        plain_b = s.fmm_audit(2, 0.5, False, 2048)
        learned_b = s.fmm_audit(2, 0.5, True, 2048)
        p6_b = s.fmm_audit(6, 0.5, False, 2048)
    print(f"RMS relative force error, training cloud: p=2 {plain:.3e}, p=2 + MLP {learned:.3e}; "
          f"held-out cloud: p=2 {plain_b:.3e}, p=2 + MLP {learned_b:.3e}, p=6 {p6_b:.3e}")
    assert learned < 0.9 * plain, (learned, plain)
    assert learned_b < 0.95 * plain_b, (learned_b, plain_b)
    assert p6_b < 1e-2 * plain_b


def test_failed_audit_falls_back_to_plain_fmm():
    with cloud_sim(learned_audit_interval=1, learned_error_budget=1e-5, learned_fallback_order=6) as s:
        s.fmm_train_correction(0.5, sample_leaves=256, steps=50, batch=1024, lr=1e-3)
        st = s.fmm_learned_state()
        assert st["trained"] and not st["fallback"]
        s.step(1)  # the audit before the step exceeds 1e-5 -> fallback
        st = s.fmm_learned_state()
        assert st["fallback"] and st["last_error"] > 1e-5
        s.coulomb_fmm(2, 0.5, learned=True)
        f_learned = s.get_forces()
        s.coulomb_fmm(6, 0.5)
        f_p6 = s.get_forces()
        assert all(np.array_equal(a, b) for a, b in zip(f_learned, f_p6))


def test_corrupted_weights_are_caught_by_the_audit():
    with cloud_sim(n=20000, learned_audit_interval=1, learned_error_budget=0.05) as s:
        s.fmm_train_correction(0.5, sample_leaves=256, steps=50, batch=1024, lr=1e-3)
        p = s.mlp_params()
        s.set_mlp_params(np.full_like(p, 50.0))  # garbage network
        bad = s.fmm_audit(2, 0.5, True, 1024)
        assert bad > 0.05
        s.step(1)
        assert s.fmm_learned_state()["fallback"]
