"""Pin the CPU oracle and the host functions of the C ABI against the reference's known
answers: its own test KATs (tests/Seis3DBoundaryRegression.cpp:70-82,
tests/SolverRegression.cpp:67-83, docs budget table) and golden vectors produced by the
reference's own host code (tests/golden/make_cpu_golden.py)."""
import json
import os
from ctypes import POINTER, byref, c_float

import numpy as np
import pytest

import oracle
from cmakepro_cuda_seissim_v2_b200 import capi, seis3d

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")

with open(os.path.join(GOLDEN, "ref3d_host.json")) as _f:
    HOST = json.load(_f)
TABLES = dict(np.load(os.path.join(GOLDEN, "ref3d_coefficients.npz")))
GIB = 1073741824.0


def _oracle_validate(overrides):
    c = seis3d.default_context(**overrides)
    return oracle.oracle_library().oracle3d_validate(byref(c)), c


def _product_validate(overrides):
    c = seis3d.default_context(**overrides)
    try:
        seis3d.validate_context3D(c)
        return 0, c
    except seis3d.InvalidArgument:
        return 1, c


@pytest.mark.parametrize("label", sorted(HOST))
@pytest.mark.parametrize("impl", ["oracle", "product"])
def test_validation_matches_reference(label, impl, solver_lib):
    entry = HOST[label]
    status, c = (_oracle_validate if impl == "oracle" else _product_validate)(entry["input"])
    assert status == (0 if entry["status"] == 0 else 1)
    if entry["status"] == 0:
        for k, v in entry["derived"].items():
            assert getattr(c, k) == v, k
        assert int(np.float32(c.dt3D).view(np.uint32)) == entry["dt_bits"]
        assert int(np.float32(c.safeDt3D).view(np.uint32)) == entry["safe_dt_bits"]
        assert c.maxVp3D == pytest.approx(entry["maxVp3D"], rel=0, abs=0)


@pytest.mark.parametrize("label", sorted(k for k, v in HOST.items() if v["status"] == 0))
@pytest.mark.parametrize("impl", ["oracle", "product"])
def test_memory_budget_matches_reference(label, impl, solver_lib):
    entry = HOST[label]
    c = seis3d.default_context(**entry["input"])
    if impl == "oracle":
        b = capi.MemoryBudget()
        assert oracle.oracle_library().oracle3d_estimate_memory(byref(c), byref(b)) == 0
    else:
        b = seis3d.estimate_memory3D(c)
    assert [b.fieldBytes3D, b.cpmlBytes3D, b.viewBytes3D, b.totalBytes3D] == entry["budget"]


def test_published_budget_lines(solver_lib):
    # docs/development/SEIS3D_IMPLEMENTATION.md:172-179 (GiB, 3 decimals), printed by the
    # reference's BUDGET lines.
    published = {(96, 96, 96): 0.140, (160, 160, 160): 0.443, (300, 300, 300): 1.987, (300, 300, 400): 2.516}
    for (nx, ny, nz), gib in published.items():
        b = seis3d.estimate_memory3D(seis3d.default_context(nx3D=nx, ny3D=ny, nz3D=nz))
        assert round(b.totalBytes3D / GIB, 3) == gib


@pytest.mark.parametrize("name", sorted(TABLES))
def test_cpml_coefficients_bit_exact(name, solver_lib):
    label, axis = name.rsplit("_axis", 1)
    axis = int(axis)
    c = seis3d.default_context(**HOST[label]["input"])
    seis3d.validate_context3D(c)
    ref = TABLES[name].view(np.uint32)
    mine = seis3d.make_cpml_coefficients3D(c, axis).ravel().view(np.uint32)
    out = np.zeros(ref.size, dtype=np.float32)
    oracle.oracle_library().oracle3d_make_coefficients(byref(c), axis, out.ctypes.data_as(POINTER(c_float)))
    assert np.array_equal(mine, ref)
    assert np.array_equal(out.view(np.uint32), ref)


def test_cpml_refresh_equals_fresh_profile(solver_lib):
    # Seis3DWorkspaceRegression.cpp:244-250: coefficients refreshed at a new frequency are
    # bit-equal to a fresh initialisation at that frequency; a different frequency changes them.
    c = seis3d.validate_context3D(seis3d.default_context(nx3D=32, ny3D=24, nz3D=28, pml3D=8))
    c50 = c.copy()
    c50.frequency3D = 50.0
    seis3d.validate_context3D(c50)
    fresh = seis3d.validate_context3D(seis3d.default_context(nx3D=32, ny3D=24, nz3D=28, pml3D=8, frequency3D=50.0))
    for axis in range(3):
        a = seis3d.make_cpml_coefficients3D(c50, axis)
        assert np.array_equal(a.view(np.uint32), seis3d.make_cpml_coefficients3D(fresh, axis).view(np.uint32))
        assert not np.array_equal(a, seis3d.make_cpml_coefficients3D(c, axis))


def test_stencil_polynomial_moments():
    # tests/SolverRegression.cpp:67-74: sum 2 w_k (k+1/2)^d = delta_{d,1} for odd d <= 7.
    w = [1225.0 / 1024, -245.0 / 3072, 49.0 / 5120, -5.0 / 7168]
    for degree in (1, 3, 5, 7):
        moment = sum(2.0 * w[k] * (k + 0.5) ** degree for k in range(4))
        assert abs(moment - (1.0 if degree == 1 else 0.0)) < 1e-10
