"""The equilibrium driver (the reference's krome_equilibrium_cells,
runtime/interfaces/C/krome.h:366-376; solve_equilibrium at
runtime/core/solve_cell.hpp:2249-2301): every cell integrated to steady
state in intervals t0 factor^k, each a full solve from the current state.

The oracle restates the driver over its own solve (oracle.Oracle.
equilibrium) and equals the reference's strict build bit for bit; the
library runs the intervals on the GPU (one solve launch per interval over
the batch, the per-cell bookkeeping in two small kernels) and matches the
oracle's flags, with the states at the benchmark's parity bar."""
import ctypes

import numpy as np
import pytest

from conftest import ROOT, parity
from krome_x_b200 import krome, netinfo, workloads
from oracle import Oracle, reference_equilibrium

KEY = "primordial"
OPTS = dict(rtol=1e-6, atol_n=1e-20, atol_T=1e-6, jac=1, linsol=1)


def _cells(ncell, seed):
    info = netinfo.load(KEY)
    n, T, dt, par = workloads.primordial(ncell, info, seed=seed)
    return n, T, par


def test_oracle_equilibrium_equals_the_reference():
    if not (ROOT / "oracle" / "_ref" / ("libkrome_%s_strict.so" % KEY)).exists():
        pytest.skip("oracle/_ref not built here (oracle/build_ref.py)")
    n, T, par = _cells(12, 81)
    ref = reference_equilibrium(KEY, n, T, par, strict=True, evolve_T=0,
                                **OPTS)
    out = Oracle(KEY).equilibrium(n, T, par, evolve_T=0, **OPTS)
    np.testing.assert_array_equal(out["flags"], ref["flags"])
    np.testing.assert_array_equal(out["n"], ref["n"])
    np.testing.assert_array_equal(out["T"], ref["T"])
    assert set(ref["flags"]) <= {0, 1} and (ref["flags"] == 0).any()
    # a short t_max: flag 1, the state at t_max returned
    yr = 31557600.0
    ref = reference_equilibrium(KEY, n[:4], T[:4], par[:4], strict=True,
                                evolve_T=0, eq_tmax=300 * yr, **OPTS)
    out = Oracle(KEY).equilibrium(n[:4], T[:4], par[:4], evolve_T=0,
                                  tmax=300 * yr, **OPTS)
    np.testing.assert_array_equal(out["flags"], ref["flags"])
    np.testing.assert_array_equal(out["n"], ref["n"])
    assert (ref["flags"] == 1).all()


def test_equilibrium_rejects_bad_arguments():
    net = krome.load(KEY)
    lib = net._lib
    f = lib.krome_equilibrium_cells
    f.restype = ctypes.c_int
    D = ctypes.POINTER(ctypes.c_double)
    f.argtypes = [ctypes.c_int, D, D, D, ctypes.c_int, ctypes.c_void_p,
                  ctypes.POINTER(ctypes.c_int), ctypes.c_void_p]
    opts = net.options(**OPTS)
    n = np.ones((2, net.nspec))
    T = np.ones(2)
    assert f(2, n.ctypes.data_as(D), None, None, 0, None, None, opts._h) == -1
    assert f(-1, n.ctypes.data_as(D), T.ctypes.data_as(D), None, 0, None,
             None, opts._h) == -1
    par = np.ones((2, 8))
    assert f(2, n.ctypes.data_as(D), T.ctypes.data_as(D),
             par.ctypes.data_as(D), 5, None, None, opts._h) == -1
    assert f(0, n.ctypes.data_as(D), T.ctypes.data_as(D), None, 0, None,
             None, opts._h) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("evolve_T", [0, 1])
def test_gpu_equilibrium_matches_the_oracle(evolve_T):
    net = krome.load(KEY)
    n, T, par = _cells(256, 82 + evolve_T)
    yr = 31557600.0
    # evolve_T: a t_max of 1e6 yr keeps the thermal runs short
    eq = dict(tmax=1e6 * yr) if evolve_T else {}
    ref = Oracle(KEY).equilibrium(n, T, par, evolve_T=evolve_T, **eq, **OPTS)
    opts = net.options(evolve_T=evolve_T, **OPTS,
                       **({"eq_tmax": eq["tmax"]} if evolve_T else {}))
    nn, TT = n.copy(), T.copy()
    fl = np.zeros(256, dtype=np.intc)
    D = ctypes.POINTER(ctypes.c_double)
    f = net._lib.krome_equilibrium_cells
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, D, D, D, ctypes.c_int, ctypes.c_void_p,
                  ctypes.POINTER(ctypes.c_int), ctypes.c_void_p]
    r = f(256, nn.ctypes.data_as(D), TT.ctypes.data_as(D),
          np.ascontiguousarray(par).ctypes.data_as(D), net.npar, None,
          fl.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), opts._h)
    nz = ref["flags"][ref["flags"] != 0]
    assert r == (nz[0] if len(nz) else 0)
    np.testing.assert_array_equal(fl, ref["flags"])
    # the intervals end where max |dn| / n falls below 1e-5: the states agree
    # at that tolerance's parity bar
    m = parity(nn, TT, fl, ref["n"], ref["T"], ref["flags"], 1e-5)
    assert m["flags_equal"] == 1.0 and m["frac"] >= 0.9, m
