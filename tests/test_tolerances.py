"""Per-species tolerances (krome_opts_set_atol_species / rtol_species;
reference runtime/interfaces/C/krome.h:175-185, solve_cell.hpp:866-879,
2129-2139, bdf_cell.hpp:689-713): each species' atol replaces atol_n in
CVODE's weights, and a per-species rtol that differs from the scalar
switches the weights to KROME's per-slot form. The oracle equals the
reference's build with them bit for bit; the kernels match the oracle."""
import ctypes

import numpy as np
import pytest

from conftest import NETWORKS, ROOT, parity
from krome_x_b200 import krome, netinfo, workloads
from oracle import Oracle, reference_solve

_D = ctypes.POINTER(ctypes.c_double)


def _species_tols(key, seed):
    info = netinfo.load(key)
    ns = len(info["species"])
    rng = np.random.default_rng(seed)
    atol = np.where(rng.uniform(size=ns) < 0.5, -1.0,
                    10.0 ** rng.uniform(-22, -16, ns))
    rtol = np.where(rng.uniform(size=ns) < 0.5, -1.0,
                    10.0 ** rng.uniform(-7, -5, ns))
    return atol, rtol


def _set(lib, h, atol, rtol):
    for q, v in (("atol", atol), ("rtol", rtol)):
        f = getattr(lib, "krome_opts_set_%s_species" % q)
        f.argtypes = [ctypes.c_void_p, _D]
        f.restype = ctypes.c_int
        assert f(h, None if v is None else v.ctypes.data_as(_D)) == 0


@pytest.mark.parametrize("key", NETWORKS)
def test_oracle_species_tolerances_equal_the_reference(key):
    if not (ROOT / "oracle" / "_ref" / ("libkrome_%s_strict.so" % key)).exists():
        pytest.skip("oracle/_ref not built here (oracle/build_ref.py)")
    info = netinfo.load(key)
    n, T, dt, par = workloads.GENERATORS[key](48, info, seed=51)
    atol, rtol = _species_tols(key, 1)
    for a, r in ((atol, None), (atol, rtol)):
        o = dict(workloads.OPTIONS[key], atol_species=a, rtol_species=r)
        ref = reference_solve(key, n, T, dt, par, strict=True, **o)
        out = Oracle(key).solve(n, T, dt, par, **o)
        np.testing.assert_array_equal(out["flags"], ref["flags"])
        np.testing.assert_array_equal(out["n"], ref["n"])
        np.testing.assert_array_equal(out["T"], ref["T"])


def test_species_tolerance_api():
    net = krome.load("primordial3")
    lib = ctypes.CDLL(str(net.path))
    o = net.options(rtol=1e-6, atol_n=1e-20)
    get = lib.krome_opts_get_atol_species
    get.argtypes = [ctypes.c_void_p, _D]
    set_ = lib.krome_opts_set_atol_species
    set_.argtypes = [ctypes.c_void_p, _D]
    v = np.full(net.nspec, -1.0)
    v[2] = 1e-15
    assert set_(o._h, v.ctypes.data_as(_D)) == 0
    out = np.zeros(net.nspec)
    assert get(o._h, out.ctypes.data_as(_D)) == 0
    want = np.full(net.nspec, 1e-20)
    want[2] = 1e-15
    np.testing.assert_array_equal(out, want)
    bad = v.copy()
    bad[0] = np.nan
    assert set_(o._h, bad.ctypes.data_as(_D)) == -1
    bad[0] = 0.0
    assert set_(o._h, bad.ctypes.data_as(_D)) == -1
    assert set_(o._h, None) == 0
    assert get(o._h, out.ctypes.data_as(_D)) == 0
    np.testing.assert_array_equal(out, np.full(net.nspec, 1e-20))


@pytest.mark.gpu
@pytest.mark.parametrize("key", NETWORKS)
@pytest.mark.parametrize("layout", ["lane", "warp"])
def test_gpu_species_tolerances_match_the_oracle(key, layout):
    info = netinfo.load(key)
    n, T, dt, par = workloads.GENERATORS[key](512, info, seed=52)
    atol, rtol = _species_tols(key, 2)
    o = dict(workloads.OPTIONS[key])
    ref = Oracle(key).solve(n, T, dt, par, atol_species=atol,
                            rtol_species=rtol, **o)
    net = krome.load(key)
    opts = net.options(**dict(o, layout=0 if layout == "warp" else 1))
    lib = ctypes.CDLL(str(net.path))
    _set(lib, opts._h, atol, rtol)
    r = net.solve_batch(n, T, dt, par, opts=opts, check=False, stats=True)
    m = parity(r.n, r.Tgas, r.flags, ref["n"], ref["T"], ref["flags"],
               o["rtol"])
    assert m["flags_equal"] == 1.0 and m["frac"] >= 0.85, m
    # the tolerances change the integration: the step counts follow
    g, c = r.stats[:, 0].mean(), ref["stats"][:, 0].mean()
    assert abs(g - c) <= 0.03 * c + 0.5, (g, c)


@pytest.mark.gpu
def test_large_network_rejects_species_tolerances():
    net = krome.load("semenov")
    info = netinfo.load("semenov")
    n, T, dt, par = workloads.semenov(2, info, seed=6)
    opts = net.options(**workloads.OPTIONS["semenov"])
    lib = ctypes.CDLL(str(net.path))
    _set(lib, opts._h, np.full(net.nspec, 1e-20), None)
    r = net.solve_batch(n, T, dt, par, opts=opts, check=False)
    assert r.ierr == -104
