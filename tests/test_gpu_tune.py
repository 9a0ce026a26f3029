"""Force audit against the FP64 exact sum, leaf-size control and the
autotuner (measured method / order / theta / leaf choice under an error
budget)."""
import numpy as np
import pytest

import amk
import oracle_lib as O
from conftest import gaussian_cloud

pytestmark = pytest.mark.gpu


def cloud(n, seed, **over):
    x, y, z, q = gaussian_cloud(n, seed)
    sp = np.where(q > 0, 1, 3).astype(np.uint8)
    kw = dict(populations={"positron": n // 2, "electron": n - n // 2}, cooling_enabled=0, annihilation_enabled=0)
    kw.update(over)
    s = amk.Simulation(amk.make_params(**kw))
    s.set_particles(x, y, z, np.zeros(n), np.zeros(n), np.zeros(n), sp)
    return s, (x, y, z, q)


def test_force_error_equals_oracle_error_over_all_particles():
    n = 4096
    s, (x, y, z, q) = cloud(n, 3)
    with s:
        gx, gy, gz = O.allpairs(x, y, z, q)
        den = np.sqrt(gx ** 2 + gy ** 2 + gz ** 2)
        for call in (lambda: s.coulomb_allpairs(), lambda: s.coulomb_barnes_hut(0.7),
                     lambda: s.coulomb_fmm(4, 0.5)):
            call()
            fx, fy, fz = s.get_forces()
            rel = np.sqrt((fx - gx) ** 2 + (fy - gy) ** 2 + (fz - gz) ** 2) / den
            rms, mx = s.force_error(samples=n)
            assert abs(rms - np.sqrt(np.mean(rel ** 2))) <= 1e-6 * rms
            assert abs(mx - rel.max()) <= 1e-6 * mx


def test_fmm_leaf_size_changes_tree_not_accuracy():
    s, _ = cloud(20000, 4)
    with s:
        assert s.leaf_sizes() == (32, 8)
        s.coulomb_fmm(6, 0.5)
        f32 = s.get_forces()
        e32 = s.force_error(2048)[0]
        s.set_leaf_sizes(64, 8)
        s.coulomb_fmm(6, 0.5)
        f64 = s.get_forces()
        e64 = s.force_error(2048)[0]
        assert not np.array_equal(f32[0], f64[0])
        # mixed charges: particles whose forces nearly cancel dominate the
        # relative error; the leaf size must not change it much
        assert e32 < 1e-3 and e64 < 2.0 * e32
        with pytest.raises(amk.AmkError):
            s.set_leaf_sizes(0, 8)


def test_autotune_picks_fastest_candidate_within_budget():
    s, _ = cloud(20000, 5)
    with s:
        cands, chosen = s.autotune(error_budget=1e-5, samples=1024)
        assert chosen >= 0
        w = cands[chosen]
        assert w["meets"] and w["rms"] <= 1e-5
        timed = [c for c in cands if c["ms"] >= 0]
        assert all(c["ms"] >= w["ms"] for c in timed if c["meets"])
        p = s.params
        assert p.coulomb_method == w["method"]
        if w["method"] == 2:
            assert int(p.fast_multipole_order) == w["order"] and s.leaf_sizes()[0] == w["leaf"]
        # the configured solver gives the audited accuracy through amk_coulomb
        s.coulomb()
        assert s.force_error(1024)[0] <= 1e-5 * 1.01
        s.step(1)
        # a loose budget admits cheaper methods
        cands2, chosen2 = s.autotune(error_budget=1e-2, samples=512, flags=1)
        assert cands2[chosen2]["method"] != 3 and cands2[chosen2]["rms"] <= 1e-2


def test_autotune_reports_impossible_budget():
    s, _ = cloud(3000, 6)
    with s:
        with pytest.raises(amk.AmkError):
            s.autotune(error_budget=1e-13, samples=256)
