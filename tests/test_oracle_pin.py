"""The CPU oracle is pinned to the reference before it is trusted.

* its rate coefficients against the reference's own golden vectors (the
  K_REF tables of each generated project's krome_check.cpp, computed by the
  reference's independent network interpreter), with the reference's
  tolerance 1e-8;
* its solves bit for bit against the reference's strict build: the
  committed fixtures (tests/golden/<net>.npz, made by make_golden.py from
  oracle/_ref), and, where oracle/_ref exists, a live comparison on
  further seeded cells;
* the large network (Semenov), whose oracle factors the Newton matrix with
  its own sparse LU (a minimum-degree order fixed at generation, where the
  reference's sparse solver orders and pivots at run time), at the noise
  level of the problem itself instead of bit for bit.
"""
import ctypes

import numpy as np
import pytest

from conftest import ALL_NETWORKS, NETWORKS, ROOT, golden, parity, parity_major
from krome_x_b200 import netinfo, workloads
from oracle import Oracle, reference_solve

_D = ctypes.POINTER(ctypes.c_double)


def _ptr(a):
    return a.ctypes.data_as(_D)


@pytest.mark.parametrize("key", ALL_NETWORKS)
def test_rates_match_reference_golden_vectors(key):
    g = golden(key)
    orc = Oracle(key)
    lib = orc.lib
    lib.oracle_rates.argtypes = [ctypes.c_double, _D, _D, _D]
    lib.oracle_rates.restype = None
    info = netinfo.load(key)
    # the probe parameters of the reference's check: 1.3e-17, Tdust 10 K
    par = np.array([10.0 if s == "Tdust" else 1.3e-17 for s in info["params"]])
    n = np.ascontiguousarray(g["k_n"], dtype=float)
    nrea = lib.oracle_nrea()
    worst = 0.0
    for t, T in enumerate(g["k_T"]):
        k = np.zeros(nrea)
        lib.oracle_rates(float(T), _ptr(n), _ptr(par), _ptr(k))
        a, b = k[g["k_idx"]], g["k_ref"][t]
        d = np.abs(a - b) / np.maximum(np.maximum(np.abs(a), np.abs(b)), 1e-300)
        worst = max(worst, d.max())
    assert worst < 1e-8, worst


@pytest.mark.parametrize("key", NETWORKS)
def test_solve_bitwise_equal_to_reference_fixture(key):
    g = golden(key)
    opts = workloads.OPTIONS[key]
    out = Oracle(key).solve(g["n"], g["T"], g["dt"], g["par"], **opts)
    assert out["ret"] == g["ret"]
    np.testing.assert_array_equal(out["flags"], g["flags"])
    np.testing.assert_array_equal(out["n"], g["n_out"])
    np.testing.assert_array_equal(out["T"], g["T_out"])


@pytest.mark.parametrize("key", NETWORKS)
def test_solve_bitwise_equal_to_reference_live(key):
    if not (ROOT / "oracle" / "_ref" / ("libkrome_%s_strict.so" % key)).exists():
        pytest.skip("oracle/_ref not built here (oracle/build_ref.py)")
    info = netinfo.load(key)
    n, T, dt, par = workloads.GENERATORS[key](192, info, seed=23)
    opts = workloads.OPTIONS[key]
    ref = reference_solve(key, n, T, dt, par, strict=True, **opts)
    out = Oracle(key).solve(n, T, dt, par, **opts)
    np.testing.assert_array_equal(out["flags"], ref["flags"])
    np.testing.assert_array_equal(out["n"], ref["n"])
    np.testing.assert_array_equal(out["T"], ref["T"])


def test_sparse_solve_matches_reference_fixture_at_noise_level():
    """16 reference-solved cells of the surface-chemistry workload: every
    abundance above 1e-12 of the cell's density within 1e-4 (the spread one
    input ulp makes), most within 10 rtol, total mass conserved"""
    key = "semenov"
    g = golden(key)
    opts = workloads.OPTIONS[key]
    out = Oracle(key).solve(g["n"], g["T"], g["dt"], g["par"], **opts)
    assert out["ret"] == g["ret"]
    m = parity_major(out["n"], out["flags"], g["n_out"], g["flags"], g["n"],
                     opts["rtol"])
    assert m["flags_equal"] == 1.0 and m["cells"] == len(g["n"]), m
    assert m["max_rel"] < 1e-4 and m["frac"] >= 0.75, m
    mass = np.asarray(netinfo.load(key)["mass_g"])
    rho = g["n_out"] @ mass
    np.testing.assert_allclose(out["n"] @ mass, rho, rtol=1e-12)
    np.testing.assert_array_equal(out["T"], g["T_out"])


def test_oracle_required_parameter_rule():
    """a REQUIRED parameter unset in one row: nothing integrated, that cell
    -105, the others 0 (reference solve_cells.hpp:133-140)"""
    key = "primordial"
    info = netinfo.load(key)
    n, T, dt, par = workloads.GENERATORS[key](8, info, seed=2)
    par[3, info["params"].index("tff")] = np.nan
    out = Oracle(key).solve(n, T, dt, par, **workloads.OPTIONS[key])
    assert out["ret"] == -105
    assert list(out["flags"]) == [0, 0, 0, -105, 0, 0, 0, 0]
    np.testing.assert_array_equal(out["n"], n)
    np.testing.assert_array_equal(out["T"], T)


def test_oracle_nonpositive_dt_skipped():
    key = "galaxy_ism"
    info = netinfo.load(key)
    n, T, dt, par = workloads.GENERATORS[key](6, info, seed=4)
    dt[[1, 4]] = [0.0, -1.0]
    out = Oracle(key).solve(n, T, dt, par, **workloads.OPTIONS[key])
    assert out["ret"] == 0
    np.testing.assert_array_equal(out["n"][[1, 4]], n[[1, 4]])
    assert (out["stats"][[1, 4]] == 0).all()
    assert (out["stats"][[0, 2, 3, 5], 0] > 0).all()


def test_oracle_lu32_form_keeps_the_fp64_error():
    """the oracle's twin of the FP32 Newton-matrix form: against the
    rtol = 1e-12 solve its error is the FP64 form's, and its FP64 refactor
    fallback is exercised (nlu64 > 0) while the FP64 form never counts one"""
    key = "galaxy_ism"
    info = netinfo.load(key)
    n, T, dt, par = workloads.GENERATORS[key](384, info, seed=41)
    o = workloads.OPTIONS[key]
    orc = Oracle(key)
    tight = orc.solve(n, T, dt, par, **dict(o, rtol=1e-12, max_steps=2000000))
    r64 = orc.solve(n, T, dt, par, **o)
    r32 = orc.solve(n, T, dt, par, lu32=1, **o)
    m64 = parity(r64["n"], r64["T"], r64["flags"], tight["n"], tight["T"],
                 tight["flags"], o["rtol"])
    m32 = parity(r32["n"], r32["T"], r32["flags"], tight["n"], tight["T"],
                 tight["flags"], o["rtol"])
    assert m32["flags_equal"] == 1.0 and m64["flags_equal"] == 1.0
    assert m32["frac"] >= m64["frac"] - 0.02, (m32, m64)
    assert r32["stats"][:, 9].sum() > 0
    assert (r64["stats"][:, 9] == 0).all()
