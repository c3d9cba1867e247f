"""Concurrent host callers (reference threading contract: solve_cells may be
called from several host threads, runtime/core/solve_kokkos.hpp:1223-1241;
one options handle, only read, serves concurrent calls,
runtime/interfaces/C/krome.cpp:407-409). Each thread's results must equal
the same solve made alone, bit for bit, and calls from several threads
overlap on the GPU: each takes its own staging buffer and stream."""
import ctypes
import threading
import time

import numpy as np
import pytest

from krome_x_b200 import krome, netinfo, workloads

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def _dp(a):
    return None if a is None else a.ctypes.data_as(_D)


def _cases(key, k, ncell):
    info = netinfo.load(key)
    return [workloads.GENERATORS[key](ncell, info, seed=700 + i)
            for i in range(k)]


def _raw_solve(net, opts, case):
    """krome_solve_cells on copies of the case (cell-major host arrays)"""
    n, T, dt, par = case
    n = np.ascontiguousarray(n, dtype=float).copy()
    T = np.ascontiguousarray(T, dtype=float).copy()
    dt = np.ascontiguousarray(dt, dtype=float)
    P, stride = net._params(par, n.shape[0])
    flags = np.zeros(n.shape[0], dtype=np.intc)
    ierr = net._lib.krome_solve_cells(n.shape[0], _dp(n), _dp(T), _dp(dt),
                                      _dp(P), stride, None,
                                      flags.ctypes.data_as(_I), opts._h)
    return ierr, flags, n, T


@pytest.mark.gpu
@pytest.mark.parametrize("key", ["primordial3", "galaxy_ism"])
def test_concurrent_callers_equal_serial_calls(key):
    net = krome.load(key)
    opts = net.options(**workloads.OPTIONS[key])  # one handle, shared
    cases = _cases(key, 6, 700)
    serial = [_raw_solve(net, opts, c) for c in cases]
    out = [None] * (2 * len(cases))
    errors = []

    def work(t):
        try:
            c = cases[t % len(cases)]
            if t < len(cases):  # the C entry point
                out[t] = _raw_solve(net, opts, c)
            else:               # the Python batch entry point
                r = net.solve_batch(*c, opts=opts, check=False)
                out[t] = (r.ierr, r.flags, r.n, r.Tgas)
        except Exception as e:  # reported on the main thread
            errors.append(e)

    threads = [threading.Thread(target=work, args=(t,)) for t in range(len(out))]
    for th in threads:
        th.start()
    for th in threads:
        th.join(timeout=300)
    assert not any(th.is_alive() for th in threads)
    assert not errors, errors
    for t, got in enumerate(out):
        want = serial[t % len(cases)]
        assert got[0] == want[0]
        np.testing.assert_array_equal(got[1], want[1])
        np.testing.assert_array_equal(got[2], want[2])
        np.testing.assert_array_equal(got[3], want[3])


@pytest.mark.gpu
def test_concurrent_callers_overlap():
    """four threads' calls (256 cells each: a batch that occupies a few SMs)
    finish in well under the time of the same four calls in a row"""
    key = "primordial3"
    net = krome.load(key)
    opts = net.options(**workloads.OPTIONS[key])
    cases = _cases(key, 4, 256)
    out = [None] * len(cases)

    def work(t):
        out[t] = _raw_solve(net, opts, cases[t])

    def concurrent():
        threads = [threading.Thread(target=work, args=(t,))
                   for t in range(len(cases))]
        t0 = time.perf_counter()
        for th in threads:
            th.start()
        for th in threads:
            th.join(timeout=300)
        assert not any(th.is_alive() for th in threads)
        return time.perf_counter() - t0

    concurrent()  # warm-up: four slots (staging buffer and stream) exist
    t0 = time.perf_counter()
    serial = [_raw_solve(net, opts, c) for c in cases]
    t_serial = time.perf_counter() - t0
    t_conc = concurrent()
    for got, want in zip(out, serial):
        np.testing.assert_array_equal(got[2], want[2])
    assert t_conc < 0.75 * t_serial, (t_conc, t_serial)


@pytest.mark.gpu
def test_pageable_and_pinned_host_arrays_solve_alike():
    """krome_solve_cells on pageable arrays (staged through the call's
    pinned buffer) and on pinned ones (copied directly): the same results"""
    import torch
    key = "primordial3"
    net = krome.load(key)
    opts = net.options(**workloads.OPTIONS[key])
    case = _cases(key, 1, 1000)[0]
    a = _raw_solve(net, opts, case)
    pin = lambda v: torch.from_numpy(np.ascontiguousarray(v, dtype=float)) \
        .pin_memory().numpy()
    n, T, dt = (pin(v) for v in case[:3])
    P, stride = net._params(case[3], n.shape[0])
    P = pin(P)
    flags = pin(np.zeros(n.shape[0])).astype(np.intc)
    ierr = net._lib.krome_solve_cells(n.shape[0], _dp(n), _dp(T), _dp(dt),
                                      _dp(P), stride, None,
                                      flags.ctypes.data_as(_I), opts._h)
    assert a[0] == ierr
    np.testing.assert_array_equal(a[1], flags)
    np.testing.assert_array_equal(a[2], n)
    np.testing.assert_array_equal(a[3], T)
