"""krome_b200_solve_cells_noalloc: the solve for callers that cannot let the
library allocate device memory (a code whose memory pool owns the whole
GPU, or a time step that must not pay cudaMalloc's device-wide
synchronization). It stages its device copies in a fixed 16 MiB array
compiled into the library.

Checked through the C ABI against krome_solve_cells on two calls in a row
with different cells (the shared array keeps the previous call's contents),
within the parity tolerance of the other GPU tests (10 rtol; the two run
the same kernel, so they agree exactly), and a call larger than the array
is refused with FLAG_DEVICE_MEMORY before anything is touched. This file is
collected last."""
import ctypes

import numpy as np
import pytest

from krome_x_b200 import build, krome, netinfo, workloads

pytestmark = pytest.mark.gpu

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def _call(fn, net, n, T, dt, par, opts):
    n, T = n.copy(), T.copy()
    fl = np.full(len(T), 7, dtype=np.intc)
    args = [len(T), n.ctypes.data_as(_D), T.ctypes.data_as(_D),
            dt.ctypes.data_as(_D), par.ctypes.data_as(_D), net.npar]
    if fn == "krome_solve_cells":
        r = net._lib.krome_solve_cells(*args, None, fl.ctypes.data_as(_I),
                                       opts._h)
    else:
        r = getattr(net._lib, fn)(*args, fl.ctypes.data_as(_I), opts._h)
    return r, n, T, fl


def test_noalloc_matches_krome_solve_cells_on_two_calls():
    key = "primordial3"
    net = krome.load(key)
    lib = net._lib
    lib.krome_b200_solve_cells_noalloc.restype = ctypes.c_int
    lib.krome_b200_solve_cells_noalloc.argtypes = [
        ctypes.c_int, _D, _D, _D, _D, ctypes.c_int, _I, ctypes.c_void_p]
    assert hasattr(ctypes.CDLL(str(build.lib_path(key))),
                   "krome_b200_solve_cells_noalloc")
    info = netinfo.load(key)
    o = workloads.OPTIONS[key]
    opts = net.options(evolve_T=o["evolve_T"], jac=o["jac"], rtol=o["rtol"],
                       atol_n=o["atol_n"], atol_T=o["atol_T"],
                       kernel="persistent", layout=1)
    for seed, ncell in ((41, 3000), (42, 1111)):  # two calls in a row
        n, T, dt, par = workloads.primordial3(ncell, info, seed=seed)
        n[5] = np.nan  # one failing cell: its flag and untouched row
        r0, n0, T0, f0 = _call("krome_solve_cells", net, n, T, dt, par, opts)
        r1, n1, T1, f1 = _call("krome_b200_solve_cells_noalloc", net, n, T,
                               dt, par, opts)
        assert r1 == r0 != 0
        np.testing.assert_array_equal(f1, f0)
        ok = f0 == 0
        assert ok.sum() == ncell - 1
        np.testing.assert_allclose(n1[ok], n0[ok], rtol=10 * o["rtol"],
                                   atol=o["atol_n"])
        np.testing.assert_allclose(T1[ok], T0[ok], rtol=10 * o["rtol"])
        np.testing.assert_array_equal(n1[~ok], n[~ok])


def test_noalloc_refuses_calls_larger_than_its_array():
    key = "primordial3"
    net = krome.load(key)
    lib = net._lib
    lib.krome_b200_solve_cells_noalloc.restype = ctypes.c_int
    lib.krome_b200_solve_cells_noalloc.argtypes = [
        ctypes.c_int, _D, _D, _D, _D, ctypes.c_int, _I, ctypes.c_void_p]
    info = netinfo.load(key)
    per_cell = 8 * (net.nspec + 2 + net.npar) + 4
    ncell = (16 << 20) // per_cell + 1024
    n, T, dt, par = workloads.primordial3(ncell, info, seed=3)
    r, n1, T1, fl = _call("krome_b200_solve_cells_noalloc", net, n, T, dt,
                          par, net.options(evolve_T=1, rtol=1e-6))
    assert r == -111 and (fl == -111).all()
    np.testing.assert_array_equal(n1, n)
    np.testing.assert_array_equal(T1, T)
