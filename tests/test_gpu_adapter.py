"""The BioDynaMo drop-in adapter (antimatter-kernel_b200/adapter/
amk_bdm_adapter.cc): the reference's three Coulomb drivers with their own
signatures, compiled against stand-ins of BioDynaMo's agent and resource
manager types and linked to libamk. Its forces on agents must match the
reference's own drivers (and the FP64 cutoff oracle), annihilated agents
must be left untouched and neutral agents get zero force under the FMM."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle_lib as O
from conftest import E, ROOT, gaussian_cloud, rel_errors

ADAPTER = os.path.join(ROOT, "antimatter-kernel_b200", "adapter", "amk_bdm_adapter.cc")
STUB = os.path.join(ROOT, "tests", "bdm_stub")
LIBDIR = os.path.join(ROOT, "antimatter-kernel_b200")


def build_harness(out_dir):
    """Compiles the adapter and the test harness into one shared library."""
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    out = os.path.join(out_dir, "libamk_adapter_harness.so")
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", f"-I{STUB}", f"-I{os.path.join(ROOT, 'include')}",
           ADAPTER, os.path.join(STUB, "harness.cc"), f"-L{LIBDIR}", "-lamk", f"-Wl,-rpath,{LIBDIR}", "-o", out]
    subprocess.run(cmd, check=True, capture_output=True)
    return out


def test_adapter_compiles_and_links(tmp_path):
    import amk
    amk.lib()  # libamk.so built
    lib = C.CDLL(build_harness(str(tmp_path)))
    assert hasattr(lib, "harness_run")


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    import amk
    amk.lib()
    lib = C.CDLL(build_harness(str(tmp_path_factory.mktemp("adapter"))))
    dp = C.POINTER(C.c_double)
    lib.harness_run.argtypes = [C.c_int, C.c_long, dp, dp, dp, dp, C.POINTER(C.c_uint8), C.c_double, C.c_int,
                                dp, dp, dp]
    lib.harness_run.restype = C.c_int

    def run(method, x, y, z, q, annihilated, param, order=0):
        n = len(x)
        arrs = [np.ascontiguousarray(a, np.float64) for a in (x, y, z, q)]
        an = np.ascontiguousarray(annihilated, np.uint8)
        f = [np.zeros(n) for _ in range(3)]
        rc = lib.harness_run(method, n, *[a.ctypes.data_as(dp) for a in arrs], an.ctypes.data_as(C.POINTER(C.c_uint8)),
                             float(param), int(order), *[a.ctypes.data_as(dp) for a in f])
        assert rc == 0
        return f
    return run


def agents(n, seed):
    x, y, z, q = gaussian_cloud(n, seed)
    rng = np.random.default_rng(seed)
    annihilated = (rng.random(n) < 0.1).astype(np.uint8)
    q = np.where(rng.random(n) < 0.05, 0.0, q)  # some neutral agents
    return x, y, z, q, annihilated


@pytest.mark.gpu
def test_standard_driver_matches_fp64_cutoff(harness):
    x, y, z, q, ann = agents(3000, 1)
    fx, fy, fz = harness(0, x, y, z, q, ann, 3e-5)
    live = ann == 0
    assert np.all(np.isnan(fx[~live]))  # annihilated agents untouched
    gx, gy, gz = O.cutoff(x[live], y[live], z[live], q[live], 3e-5)
    scale = max(np.max(np.abs(gx)), 1e-300)
    for a, b in zip((fx[live], fy[live], fz[live]), (gx, gy, gz)):
        assert np.max(np.abs(a - b)) <= 1e-12 * scale
    fx0, _, _ = harness(0, x, y, z, q, ann, 0.0)  # cutoff <= 0: zero force on every live agent
    assert np.all(fx0[live] == 0.0) and np.all(np.isnan(fx0[~live]))


@pytest.mark.gpu
def test_barnes_hut_and_fmm_drivers_match_the_reference_drivers(harness):
    if not O.ref_available():
        pytest.skip("reference library not built")
    x, y, z, q, ann = agents(4000, 2)
    live = ann == 0
    for method, param, order, tol in ((1, 0.5, 0, 1e-10), (2, 0.5, 4, 1e-9)):
        f = harness(method, x, y, z, q, ann, param, order)
        assert np.all(np.isnan(f[0][~live]))
        name = "barnes-hut" if method == 1 else "fast-multipole"
        g = O.ref_driver(name, x, y, z, q, 1 - ann, param, order)
        charged = live & (q != 0)
        rel, _ = rel_errors([a[charged] for a in f], [b[charged] for b in g])
        assert np.max(rel) < tol, (name, np.max(rel))
        neutral = live & (q == 0)
        assert all(np.all(a[neutral] == 0.0) for a in f)
