"""The large-network (sparse-LU) path: the Semenov surface-chemistry network,
655 species and 5639 reactions, fixed Tgas.

Its GPU solve runs the same CVODE as the oracle with the same static-pivot
sparse LU (a minimum-degree order fixed at generation); the bar is the
large-network parity metric (conftest.parity_major): every abundance above
1e-12 of the cell's density within 2e-4 -- one input ulp moves the oracle by
up to ~5e-5 on this workload -- most cells within 10 rtol, flags equal, and
the total mass conserved."""
import ctypes

import numpy as np
import pytest

from conftest import golden, parity_major
from krome_x_b200 import krome, netinfo, workloads
from oracle import Oracle

KEY = "semenov"


def _opts(net, **extra):
    o = workloads.OPTIONS[KEY]
    return net.options(evolve_T=o["evolve_T"], jac=o["jac"], linsol=o["linsol"],
                       rtol=o["rtol"], atol_n=o["atol_n"], atol_T=o["atol_T"],
                       max_steps=o["max_steps"], **extra)


def test_workload_is_neutral_and_sets_the_surface_parameters():
    info = netinfo.load(KEY)
    n, T, dt, par = workloads.semenov(64, info, seed=1)
    charge = np.asarray(info["charge"], dtype=float)
    np.testing.assert_allclose(n @ charge, 0.0, atol=1e-12 * n.sum(axis=1).max())
    P = info["params"]
    np.testing.assert_array_equal(par[:, P.index("Tdust")], T)
    assert (par[:, P.index("xdust")] > 0).all()
    assert (dt == 3.15e13).all() and ((T >= 10) & (T <= 300)).all()


@pytest.mark.gpu
def test_sparse_parity_with_reference_fixture():
    g = golden(KEY)
    net = krome.load(KEY)
    r = net.solve_batch(g["n"], g["T"], g["dt"], g["par"], opts=_opts(net),
                        check=False)
    m = parity_major(r.n, r.flags, g["n_out"], g["flags"], g["n"],
                     workloads.OPTIONS[KEY]["rtol"])
    assert m["flags_equal"] == 1.0 and m["cells"] == len(g["n"]), m
    assert m["max_rel"] < 2e-4 and m["frac"] >= 0.7, m
    assert r.ierr == g["ret"]
    np.testing.assert_array_equal(r.Tgas, g["T_out"])


@pytest.mark.gpu
def test_sparse_parity_with_oracle_and_conservation():
    info = netinfo.load(KEY)
    n, T, dt, par = workloads.semenov(32, info, seed=3)
    ref = Oracle(KEY).solve(n, T, dt, par, **workloads.OPTIONS[KEY])
    net = krome.load(KEY)
    r = net.solve_batch(n, T, dt, par, opts=_opts(net), check=False,
                        stats=True)
    m = parity_major(r.n, r.flags, ref["n"], ref["flags"], n,
                     workloads.OPTIONS[KEY]["rtol"])
    assert m["flags_equal"] == 1.0 and m["cells"] == 32, m
    assert m["max_rel"] < 2e-4 and m["frac"] >= 0.7, m
    mass = np.asarray(info["mass_g"])
    np.testing.assert_allclose(r.n @ mass, n @ mass, rtol=1e-10)
    # the same integrator: step counts agree to within the chaotic spread
    g, c = r.stats[:, 0].mean(), ref["stats"][:, 0].mean()
    assert abs(g - c) <= 0.05 * c, (g, c)


@pytest.mark.gpu
def test_sparse_rates_match_reference_golden_vectors():
    g = golden(KEY)
    net = krome.load(KEY)
    par = np.array([10.0 if s == "Tdust" else 1.3e-17 for s in net.params])
    for t, T in enumerate(g["k_T"]):
        k = net.rates(g["k_n"], T, par)[0]
        a, b = k[g["k_idx"]], g["k_ref"][t]
        d = np.abs(a - b) / np.maximum(np.maximum(np.abs(a), np.abs(b)), 1e-300)
        assert d.max() < 1e-8, (T, d.max())


@pytest.mark.gpu
def test_sparse_edge_cases():
    """dt <= 0 untouched with flag 0; an unset required parameter rejects
    the whole call (-105) before the device; fault injection reports -1 and
    leaves the cell untouched"""
    info = netinfo.load(KEY)
    n, T, dt, par = workloads.semenov(8, info, seed=4)
    net = krome.load(KEY)
    dt[[2, 5]] = [0.0, -1.0]
    r = net.solve_batch(n, T, dt, par, opts=_opts(net, fail_every=4),
                        check=False)
    assert list(r.flags) == [0, 0, 0, -1, 0, 0, 0, -1]
    for c in (2, 3, 5, 7):
        np.testing.assert_array_equal(r.n[c], n[c])
    assert not np.array_equal(r.n[0], n[0])


@pytest.mark.gpu
def test_sparse_unsupported_forms_return_minus_104():
    """the large path runs fixed Tgas and FP64 sparse (or auto) LU; the
    dense LU, evolve_T, the FP32 Newton matrix and the adjoint are the small
    networks' forms"""
    info = netinfo.load(KEY)
    n, T, dt, par = workloads.semenov(2, info, seed=6)
    net = krome.load(KEY)
    for extra in (dict(linsol=1), dict(linsol=2), dict(lu32=1)):
        r = net.solve_batch(n, T, dt, par, opts=_opts(net, **extra),
                            check=False)
        assert r.ierr == -104, extra
        np.testing.assert_array_equal(r.n, n)
    o = net.options(evolve_T=1, linsol=3)
    assert net.solve_batch(n, T, dt, par, opts=o, check=False).ierr == -104
    with pytest.raises(krome.KromeError):
        net.adjoint(n, T, dt, par, gn=np.ones_like(n), opts=_opts(net))
    lib = ctypes.CDLL(str(net.path))
    lib.krome_b200_rhs_throughput.restype = ctypes.c_int
    out = ctypes.c_double(0.0)
    D = ctypes.POINTER(ctypes.c_double)
    assert lib.krome_b200_rhs_throughput(
        2, n.ctypes.data_as(D), T.ctypes.data_as(D), par.ctypes.data_as(D),
        ctypes.c_int(net.npar), 1, ctypes.byref(out)) == -104
