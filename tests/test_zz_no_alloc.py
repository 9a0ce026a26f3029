"""The allocation-free cutoff solver, called through the C ABI.

It serves callers that cannot let a library allocate device memory (their
device memory is owned by their own pool, or their step loop cannot take
cudaMalloc's device-wide synchronisation); its scratch is a static device
array. This checks it against the existing cutoff entry point on two calls
in a row (the second call must not see the first call's leftovers) and that
sizes beyond its maximum are refused. The file sorts last so that a run that
stops at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import amk
import oracle_lib as O
from conftest import gaussian_cloud

pytestmark = pytest.mark.gpu

TOL = 1e-12  # the cutoff solver's FP64 tolerance in test_gpu_direct.py


def _fn():
    f = amk.lib().amk_coulomb_standard_noalloc
    vp = C.c_void_p
    f.restype = C.c_int
    f.argtypes = [vp, vp, vp, vp, vp, C.c_long, C.c_double, vp, vp, vp, vp]
    return f


def _call(x, y, z, q, rc, alive=None):
    import torch
    dev = torch.device("cuda", 0)
    t = [torch.tensor(a, dtype=torch.float64, device=dev) for a in (x, y, z, q)]
    al = None if alive is None else torch.tensor(alive, dtype=torch.uint8, device=dev)
    out = [torch.full((len(x),), np.nan, dtype=torch.float64, device=dev) for _ in range(3)]
    stream = torch.cuda.current_stream(dev)
    rc_ = _fn()(*[a.data_ptr() for a in t], None if al is None else al.data_ptr(), len(x), rc,
               *[o.data_ptr() for o in out], stream.cuda_stream)
    torch.cuda.synchronize(dev)
    amk.check(rc_, "amk_coulomb_standard_noalloc")
    return tuple(o.cpu().numpy() for o in out)


def _close(a, b):
    for u, v in zip(a, b):
        assert np.all(np.isfinite(u))
        assert np.max(np.abs(u - v)) <= TOL * max(np.max(np.abs(v)), 1e-300)


def test_noalloc_matches_cutoff_entry_point_twice(sim):
    # first call: 3,000 particles; second call: a different, smaller cloud
    # with a different radius and some dead particles
    x, y, z, q = gaussian_cloud(3000, 71)
    _close(_call(x, y, z, q, 5e-5), sim.solve_cutoff(x, y, z, q, 5e-5))
    x, y, z, q = gaussian_cloud(1800, 72)
    alive = np.ones(1800, np.uint8)
    alive[::5] = 0
    got = _call(x, y, z, q, 3e-5, alive)
    live = alive.astype(bool)
    ref = sim.solve_cutoff(x[live], y[live], z[live], q[live], 3e-5)
    _close(tuple(g[live] for g in got), ref)
    assert all(np.all(g[~live] == 0.0) for g in got)


def test_noalloc_at_its_maximum_size_and_against_the_oracle(sim):
    # n = 65,536 fills every region of the static array (16 sort tiles, the
    # full digit histogram); a small case is also held to the FP64 oracle
    x, y, z, q = gaussian_cloud(65536, 73)
    _close(_call(x, y, z, q, 1e-5), sim.solve_cutoff(x, y, z, q, 1e-5))
    x, y, z, q = gaussian_cloud(700, 74)
    _close(_call(x, y, z, q, 4e-5), O.cutoff(x, y, z, q, 4e-5))


def test_noalloc_zero_radius_and_empty_input():
    x, y, z, q = gaussian_cloud(500, 75)
    got = _call(x, y, z, q, 0.0)  # cutoff_radius <= 0: every force is zero
    assert all(np.all(g == 0.0) for g in got)
    vp = C.c_void_p(1)
    assert _fn()(vp, vp, vp, vp, None, 0, 1e-5, vp, vp, vp, None) == 0  # n = 0: nothing to do


def test_noalloc_rejects_sizes_beyond_its_maximum():
    vp = C.c_void_p(1)
    rc = _fn()(vp, vp, vp, vp, None, 65537, 1e-5, vp, vp, vp, None)
    assert rc == -7  # AMK_ERR_LIMIT, before any device work
    assert "maximum" in amk.lib().amk_last_error().decode()
