"""The C-ABI libraries load without a GPU, export every entry point that
include/krome_b200.h declares, and honour the reference's argument
conventions in everything that is decided before the device is touched
(option keys and values, bad arguments, the required-parameter rule)."""
import ctypes
import re

import numpy as np
import pytest

from conftest import ALL_NETWORKS, ROOT
from krome_x_b200 import build, krome, netinfo

HEADER = ROOT / "include" / "krome_b200.h"
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def declared_symbols():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(krome_\w+)\s*\(", text)))


def test_header_declares_the_reference_entry_points():
    syms = declared_symbols()
    for s in ("krome_solve_cells", "krome_opts_new", "krome_opts_set",
              "krome_opts_get", "krome_opts_free", "krome_params_default",
              "krome_param_required_by", "krome_flag_message",
              "krome_get_rates", "krome_b200_solve_device"):
        assert s in syms


@pytest.mark.parametrize("key", ALL_NETWORKS)
def test_library_exports_every_declared_symbol(key):
    lib = ctypes.CDLL(str(build.build(key)))
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


@pytest.mark.parametrize("key", ALL_NETWORKS)
def test_network_description_matches_metadata(key):
    net = krome.load(key)
    info = netinfo.load(key)
    assert net.species == tuple(info["species"])
    assert net.params == tuple(info["params"])
    d = net.params_default()
    for a, b in zip(d, info["defaults"]):
        assert (np.isnan(a) and np.isnan(b)) or a == b
    assert net.nspec == len(info["species"]) and net.nrea == info["nrea"]
    assert net.idx("e-") == info["species"].index("e-")


def test_options_keys_and_values():
    net = krome.load("primordial")
    o = net.options()
    assert o["rtol"] == 1e-8 and o["max_steps"] == 100000
    o["rtol"] = 1e-6
    assert o["rtol"] == 1e-6
    o["jac"] = "analytic"
    assert o["jac"] == 1.0
    for bad in (("jac", 3), ("linsol", 7), ("kernel", 2), ("layout", 5),
                ("max_restarts", -1), ("lane_minb", 9)):
        with pytest.raises(krome.KromeError):
            o[bad[0]] = bad[1]
    with pytest.raises(krome.KromeError):
        o["no_such_key"] = 1.0
    lib = net._lib
    v = ctypes.c_double()
    assert lib.krome_opts_get(o._h, b"no_such_key", ctypes.byref(v)) == -1
    assert lib.krome_opts_set(None, b"rtol", 1.0) == -1


def test_bad_arguments_return_minus_one():
    net = krome.load("galaxy_ism")
    lib = net._lib
    h = net.options()._h
    n = np.ones((2, net.nspec))
    T = np.ones(2)
    dt = np.ones(2)
    par = np.tile(net.params_default(), (2, 1))
    fl = np.zeros(2, dtype=np.intc)
    P = lambda a: a.ctypes.data_as(_D)
    # negative ncell, null arrays, a par stride that is neither 0 nor npar
    assert lib.krome_solve_cells(-1, P(n), P(T), P(dt), P(par), 0, None,
                                 fl.ctypes.data_as(_I), h) == -1
    assert lib.krome_solve_cells(2, None, P(T), P(dt), P(par), 0, None,
                                 fl.ctypes.data_as(_I), h) == -1
    assert lib.krome_solve_cells(2, P(n), P(T), P(dt), P(par), 3, None,
                                 fl.ctypes.data_as(_I), h) == -1
    assert lib.krome_solve_cells(2, P(n), P(T), P(dt), P(par), 0, None,
                                 fl.ctypes.data_as(_I), None) == -1
    assert lib.krome_solve_cells(0, P(n), P(T), P(dt), P(par), 0, None,
                                 fl.ctypes.data_as(_I), h) == 0


def test_required_parameter_rejects_the_whole_call_before_the_device():
    """reference solve_cells.hpp:133-140: an unset REQUIRED parameter in any
    row: nothing integrated, that cell -105, the others 0, return -105"""
    net = krome.load("primordial")
    n = np.full((3, net.nspec), 1.0)
    T = np.full(3, 100.0)
    dt = np.full(3, 1e10)
    par = np.tile(net.params_default(), (3, 1))
    par[:, net.params.index("tff")] = [1e12, np.nan, 1e12]
    fl = np.full(3, 7, dtype=np.intc)
    n0, T0 = n.copy(), T.copy()
    r = net._lib.krome_solve_cells(3, n.ctypes.data_as(_D), T.ctypes.data_as(_D),
                                   dt.ctypes.data_as(_D), par.ctypes.data_as(_D),
                                   net.npar, None, fl.ctypes.data_as(_I),
                                   net.options(evolve_T=1)._h)
    assert r == -105
    assert list(fl) == [0, -105, 0]
    np.testing.assert_array_equal(n, n0)
    np.testing.assert_array_equal(T, T0)


def test_python_binding_raises_before_the_call_on_missing_parameter():
    net = krome.load("primordial")
    with pytest.raises(krome.KromeError, match="tff"):
        net.solve(np.ones(net.nspec), 100.0, 1e10)


def test_unsupported_configurations_return_minus_104():
    net = krome.load("galaxy_ism")
    n = np.ones((2, net.nspec))
    for o in (dict(linsol="sparse"), dict(lu32=1, layout=0)):
        opts = net.options(**o)
        r = net.solve(n, 100.0, 1e5, opts=opts, check=False)
        assert r.ierr == -104 and (r.flags == -104).all(), o
        np.testing.assert_array_equal(r.n, n)


def test_solve_batch_requires_strict_shapes():
    net = krome.load("galaxy_ism")
    with pytest.raises(krome.KromeError):
        net.solve_batch(np.ones(net.nspec), [1.0], [1.0])
    with pytest.raises(krome.KromeError):
        net.solve_batch(np.ones((2, net.nspec)), 100.0, [1.0, 1.0])
    with pytest.raises(krome.KromeError):
        net.solve(np.ones((2, net.nspec + 1)), 100.0, 1.0)


def test_flag_messages():
    net = krome.load("primordial")
    assert "unset" in net.flag_message(-105)
    assert "FLAG_TOO_MUCH_WORK" in net.flag_message(-1)
    assert net.flag_message(0) == "success"


def test_noalloc_entry_point_refuses_before_the_device():
    """the no-allocation solve: bad arguments and the large networks'
    refusal (their sparse path needs its own workspace) are decided on the
    host, every flag written"""
    fn_t = [ctypes.c_int, _D, _D, _D, _D, ctypes.c_int, _I, ctypes.c_void_p]
    big = krome.load("semenov")
    fn = big._lib.krome_b200_solve_cells_noalloc
    fn.restype, fn.argtypes = ctypes.c_int, fn_t
    n = np.ones((3, big.nspec))
    T, dt = np.full(3, 20.0), np.full(3, 1e10)
    fl = np.zeros(3, dtype=np.intc)
    h = big.options()._h
    P = lambda a: a.ctypes.data_as(_D)
    assert fn(3, P(n), P(T), P(dt), None, 0, fl.ctypes.data_as(_I), h) == -104
    assert (fl == -104).all()
    small = krome.load("primordial3")
    fn = small._lib.krome_b200_solve_cells_noalloc
    fn.restype, fn.argtypes = ctypes.c_int, fn_t
    n = np.ones((3, small.nspec))
    assert fn(0, None, None, None, None, 0, None, None) == -1
    assert fn(3, None, P(T), P(dt), None, 0, None, small.options()._h) == -1
    par = np.tile(small.params_default(), (3, 1))
    assert fn(3, P(n), P(T), P(dt), P(par), 5, None, small.options()._h) == -1
    # an unset REQUIRED parameter (tff): -105 before the device
    fl[:] = 7
    assert fn(3, P(n), P(T), P(dt), P(par), small.npar, fl.ctypes.data_as(_I),
              small.options(evolve_T=1)._h) == -105
    assert (fl == -105).all()
