"""krome_b200_solve_cells_noalloc: the solve for callers that cannot let the
library allocate device memory (a code whose memory pool owns the whole
GPU, or a time step that must not pay cudaMalloc's device-wide
synchronization). It stages its device copies in a fixed 16 MiB array
compiled into the library; a call with no cells is the warm-up that loads
the library's device code and lets the driver reserve the kernel's local
memory before the caller's pool takes the GPU.

Checked through the C ABI against krome_solve_cells: the two run the same
kernel on the same cells, so the results must be equal bit for bit, on two
calls in a row with different cells (the shared array keeps the previous
call's contents) and without a flags array; in a fresh process where the
warm-up and the no-allocation call are the process's first solves, with
the device's free memory unchanged across the call; and a call larger than
the array is refused with FLAG_DEVICE_MEMORY before anything is touched.
This file is collected last."""
import ctypes
import json
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

from conftest import ROOT
from krome_x_b200 import build, krome, netinfo, workloads

pytestmark = pytest.mark.gpu

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
KEY = "primordial3"


def _bind(net):
    fn = net._lib.krome_b200_solve_cells_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_int, _D, _D, _D, _D, ctypes.c_int, _I,
                   ctypes.c_void_p]
    return fn


def _opts(net):
    o = workloads.OPTIONS[KEY]
    return net.options(evolve_T=o["evolve_T"], jac=o["jac"], rtol=o["rtol"],
                       atol_n=o["atol_n"], atol_T=o["atol_T"],
                       kernel="persistent", layout=1)


def _call(fn, net, n, T, dt, par, opts, with_flags=True):
    n, T = n.copy(), T.copy()
    fl = np.full(len(T), 7, dtype=np.intc)
    fp = fl.ctypes.data_as(_I) if with_flags else None
    args = [len(T), n.ctypes.data_as(_D), T.ctypes.data_as(_D),
            dt.ctypes.data_as(_D), par.ctypes.data_as(_D), net.npar]
    if fn == "krome_solve_cells":
        r = net._lib.krome_solve_cells(*args, None, fp, opts._h)
    else:
        r = _bind(net)(*args, fp, opts._h)
    return r, n, T, fl


def test_noalloc_equals_krome_solve_cells_on_two_calls():
    net = krome.load(KEY)
    assert hasattr(ctypes.CDLL(str(build.lib_path(KEY))),
                   "krome_b200_solve_cells_noalloc")
    info = netinfo.load(KEY)
    opts = _opts(net)
    assert _bind(net)(0, None, None, None, None, 0, None, opts._h) == 0
    for seed, ncell in ((41, 3000), (42, 1111)):  # two calls in a row
        n, T, dt, par = workloads.primordial3(ncell, info, seed=seed)
        n[5] = np.nan  # one failing cell: its flag and untouched row
        r0, n0, T0, f0 = _call("krome_solve_cells", net, n, T, dt, par, opts)
        r1, n1, T1, f1 = _call("krome_b200_solve_cells_noalloc", net, n, T,
                               dt, par, opts)
        assert r1 == r0 != 0
        np.testing.assert_array_equal(f1, f0)
        assert (f0 == 0).sum() == ncell - 1
        np.testing.assert_array_equal(n1, n0)
        np.testing.assert_array_equal(T1, T0)
        np.testing.assert_array_equal(n1[f0 != 0], n[f0 != 0])
        # without a flags array: the same return code and results
        r2, n2, T2, _ = _call("krome_b200_solve_cells_noalloc", net, n, T,
                              dt, par, opts, with_flags=False)
        assert r2 == r0
        np.testing.assert_array_equal(n2, n0)
        np.testing.assert_array_equal(T2, T0)


def test_noalloc_takes_no_device_memory_once_warm():
    import torch
    net = krome.load(KEY)
    info = netinfo.load(KEY)
    opts = _opts(net)
    assert _bind(net)(0, None, None, None, None, 0, None, opts._h) == 0
    n, T, dt, par = workloads.primordial3(2048, info, seed=43)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    r, n1, T1, fl = _call("krome_b200_solve_cells_noalloc", net, n, T, dt,
                          par, opts)
    free1 = torch.cuda.mem_get_info()[0]
    assert r == 0 and (fl == 0).all()
    assert free1 == free0, (free0, free1)


_FRESH = textwrap.dedent("""
    import ctypes, json, sys
    import numpy as np
    sys.path.insert(0, %(root)r)
    from krome_x_b200 import krome, netinfo, workloads
    key = %(key)r
    D = ctypes.POINTER(ctypes.c_double)
    I = ctypes.POINTER(ctypes.c_int)
    net = krome.load(key)
    fn = net._lib.krome_b200_solve_cells_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_int, D, D, D, D, ctypes.c_int, I, ctypes.c_void_p]
    o = workloads.OPTIONS[key]
    opts = net.options(evolve_T=o["evolve_T"], jac=o["jac"], rtol=o["rtol"],
                       atol_n=o["atol_n"], atol_T=o["atol_T"],
                       kernel="persistent", layout=1)
    warm = fn(0, None, None, None, None, 0, None, opts._h)
    import torch
    torch.cuda.mem_get_info()
    free0 = torch.cuda.mem_get_info()[0]
    n, T, dt, par = workloads.primordial3(1500, netinfo.load(key), seed=44)
    a = [n.copy(), T.copy(), np.zeros(1500, dtype=np.intc)]
    r1 = fn(1500, a[0].ctypes.data_as(D), a[1].ctypes.data_as(D),
            dt.ctypes.data_as(D), par.ctypes.data_as(D), net.npar,
            a[2].ctypes.data_as(I), opts._h)
    free1 = torch.cuda.mem_get_info()[0]
    b = [n.copy(), T.copy(), np.zeros(1500, dtype=np.intc)]
    r0 = net._lib.krome_solve_cells(
        1500, b[0].ctypes.data_as(D), b[1].ctypes.data_as(D),
        dt.ctypes.data_as(D), par.ctypes.data_as(D), net.npar, None,
        b[2].ctypes.data_as(I), opts._h)
    print(json.dumps(dict(warm=warm, r1=r1, r0=r0, free0=free0, free1=free1,
                          n=bool((a[0] == b[0]).all()),
                          T=bool((a[1] == b[1]).all()),
                          f=bool((a[2] == b[2]).all()),
                          ok=int((a[2] == 0).sum()))))
""")


def test_noalloc_first_solve_of_a_fresh_process():
    code = _FRESH % dict(root=str(ROOT), key=KEY)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True,
                         text=True, timeout=600, env=dict(os.environ))
    assert out.returncode == 0, out.stderr[-2000:]
    res = json.loads(out.stdout.strip().splitlines()[-1])
    assert res["warm"] == 0 and res["r1"] == res["r0"] == 0, res
    assert res["n"] and res["T"] and res["f"] and res["ok"] == 1500, res
    assert res["free1"] == res["free0"], res


def test_noalloc_refuses_calls_larger_than_its_array():
    net = krome.load(KEY)
    info = netinfo.load(KEY)
    per_cell = 8 * (net.nspec + 2 + net.npar) + 4
    ncell = (16 << 20) // per_cell + 1024
    n, T, dt, par = workloads.primordial3(ncell, info, seed=3)
    r, n1, T1, fl = _call("krome_b200_solve_cells_noalloc", net, n, T, dt,
                          par, net.options(evolve_T=1, rtol=1e-6))
    assert r == -111 and (fl == -111).all()
    np.testing.assert_array_equal(n1, n)
    np.testing.assert_array_equal(T1, T)
