"""The reference's own Python binding drives this library.

The reference's generated projects carry its ctypes binding
(runtime/interfaces/python/krome.py, copied into each project by its
generator: oracle/_ref/gen/<net>/krome.py, written here by
oracle/build_ref.py). Its Network class prototypes every entry point of the
reference's C interface when it loads a library, so loading
libkrome_b200_<net>.so through it checks the drop-in's symbol set. The
metadata and the host queries it exposes are compared with the reference's
own library (oracle/_ref/libkrome_<net>.so) through the same binding, in a
spawned process (each generated reference library in its own process), and
on the GPU its Network.solve is held to the solve's parity bar against the
oracle."""
import importlib.util
import multiprocessing as mp

import numpy as np
import pytest

from conftest import ALL_NETWORKS, NETWORKS, ROOT, assert_at_floor, parity
from krome_x_b200 import build, netinfo, workloads

GEN = ROOT / "oracle" / "_ref" / "gen"


def _binding(key):
    path = GEN / key / "krome.py"
    if not path.exists():
        pytest.skip("the reference's generated projects are not built here "
                    "(oracle/build_ref.py)")
    spec = importlib.util.spec_from_file_location("refkrome_" + key, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _inputs(key):
    info = netinfo.load(key)
    n, T, dt, par = workloads.GENERATORS[key](16, info, seed=51)
    return n, T, par


def _survey(key, lib_path, n, T, par):
    """everything the binding reports about a network and the host queries
    on a few cells (run in the process that owns lib_path)"""
    spec = importlib.util.spec_from_file_location(
        "refkrome_" + key, GEN / key / "krome.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    net = mod.Network(lib_path)
    out = {a: getattr(net, a) for a in (
        "name", "nspec", "nrea", "npar", "species", "params", "required",
        "elements", "reactions", "heating_terms", "cooling_terms",
        "coolants", "photo_reactions", "photo_reactants", "photo_pdiss",
        "lw_reactions")}
    out["masses"] = net.masses
    out["charges"] = net.charges
    out["composition"] = net.composition
    out["defaults"] = net.params_default()
    P = par if par.ndim == 2 else np.tile(par, (len(T), 1))
    for q in ("mu", "rho", "ntot", "hnuclei", "charge", "electrons",
              "free_fall_time", "element_totals"):
        out[q] = getattr(net, q)(n)
    out["jeans_length"] = net.jeans_length(n, T)
    out["free_fall_time_rho"] = net.free_fall_time_rho(net.rho(n))
    out["scale_Z"] = net.scale_Z(n, -1.0)
    out["gamma"] = net.gamma(n, T, par=P)
    out["fluxes"] = net.fluxes(n, T, par=P)
    th = net.thermal(n, T, par=P)
    out["thermal"] = (th.heat, th.cool, th.dTdt,
                      [th.heating[s] for s in net.heating_terms],
                      [th.cooling[s] for s in net.cooling_terms])
    out["qeff"] = net.qeff(n, T, par=P)
    out["num2col"] = net.num2col(n[:, 0], n, T, par=P)
    # the photon-field helpers
    lo, hi = net.bins_log(12, 1.0, 200.0)
    out["bins_log"] = (lo, hi)
    out["bins_lin"] = net.bins_lin(5, 2.0, 30.0)
    for name, args in (("spectrum_draine", ()),
                       ("spectrum_blackbody", (3e4,)),
                       ("spectrum_j21", (1.0, 1.0))):
        fn = getattr(net, name, None)
        if fn is not None:
            out[name] = fn(lo, hi, *args)
    return out


def _ref_worker(args):
    key, n, T, par = args
    return _survey(key, str(ROOT / "oracle" / "_ref" / ("libkrome_%s.so" % key)),
                   n, T, par)


def _same(a, b, rtol):
    if isinstance(a, (str, bytes, int, dict)) or a is None:
        return a == b
    if isinstance(a, tuple) and (not a or isinstance(a[0], (str, int))):
        return tuple(a) == tuple(b)
    try:
        A = np.asarray(a, dtype=float)
        B = np.asarray(b, dtype=float)
    except (TypeError, ValueError):
        return all(_same(x, y, rtol) for x, y in zip(a, b))
    if A.shape != B.shape:
        return False
    both_nan = np.isnan(A) & np.isnan(B)
    return bool(np.all(both_nan | (np.abs(A - B) <= rtol * np.abs(B))))


@pytest.mark.parametrize("key", ALL_NETWORKS)
def test_reference_binding_loads_this_library(key):
    """every entry point the reference's binding prototypes is exported"""
    mod = _binding(key)
    net = mod.Network(str(build.build(key)))
    info = netinfo.load(key)
    assert net.species == tuple(info["species"])
    assert len(net.reactions) == net.nrea
    o = net.options(evolve_T=key != "semenov", rtol=1e-6, jac="fd",
                    eq_tmax=1e10, c_red=1e9)
    assert o["eq_tmax"] == 1e10 and o["c_red"] == 1e9
    assert o.ndust == 0 and o.nbins == 0


@pytest.mark.parametrize("key", NETWORKS)
def test_metadata_and_queries_equal_the_reference(key):
    if not (ROOT / "oracle" / "_ref" / ("libkrome_%s.so" % key)).exists():
        pytest.skip("oracle/_ref not built here (oracle/build_ref.py)")
    _binding(key)
    n, T, par = _inputs(key)
    ours = _survey(key, str(build.build(key)), n, T, par)
    with mp.get_context("spawn").Pool(1) as pool:
        ref = pool.map(_ref_worker, [(key, n, T, par)])[0]
    assert set(ours) == set(ref)
    # the same expressions and operation order on the host: equal to
    # roundoff (the reference's production build contracts differently)
    for k in ref:
        assert _same(ours[k], ref[k], 1e-12), (k, ours[k], ref[k])


@pytest.mark.gpu
def test_reference_binding_solves_on_the_gpu():
    """Network.solve of the reference's binding, 512 primordial3 cells of
    the benchmark workload, held to the parity bar against the oracle"""
    from oracle import Oracle
    key = "primordial3"
    mod = _binding(key)
    net = mod.Network(str(build.build(key)))
    info = netinfo.load(key)
    n, T, dt, par = workloads.primordial3(512, info, seed=52)
    o = workloads.OPTIONS[key]
    opts = net.options(evolve_T=bool(o["evolve_T"]), jac="auto",
                       rtol=o["rtol"], atol_n=o["atol_n"], atol_T=o["atol_T"])
    res = net.solve(n, T, dt, par=par, opts=opts, check=False)
    ref = Oracle(key).solve(n, T, dt, par, **o)
    m = parity(res.n, res.Tgas, res.flags, ref["n"], ref["T"], ref["flags"],
               o["rtol"])
    assert_at_floor(m, "primordial3/first/512/52")
    assert res.ierr == ref["ret"]
    # inputs untouched (the binding's solve returns new arrays)
    n2, T2, _, _ = workloads.primordial3(512, info, seed=52)
    np.testing.assert_array_equal(n, n2)
    np.testing.assert_array_equal(T, T2)


def _photo_survey(key, lib_path, n, T, par):
    """the photon-bin tables and field queries through the binding"""
    spec = importlib.util.spec_from_file_location(
        "refkrome_" + key, GEN / key / "krome.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    net = mod.Network(lib_path)
    out = {"xsec": [[net._lib.krome_photo_xsec(r, E) for E in
                     (0.8, 3.0, 12.0, 14.0, 14.6, 16.0, 20.0, 40.0, 60.0, 500.0)]
                    for r in range(len(net.photo_reactions))]}
    P = par if par.ndim == 2 else np.tile(par, (len(T), 1))
    for name, (lo, hi), extra in (
            ("log", net.bins_log(24, 0.7, 300.0), {}),
            ("lin", net.bins_lin(10, 5.0, 40.0), {}),
            ("alpha0", net.bins_log(16, 0.7, 100.0), {"alpha": 0.0}),
            ("alpha2", net.bins_log(16, 0.7, 100.0), {"alpha": 2.0}),
            ("broad", net.bins_log(16, 2.0, 30.0), {"broad": (3000.0, 2e5)})):
        o = net.options()
        if "alpha" in extra:
            o.set_photo_alpha(extra["alpha"])
        if "broad" in extra:
            o.set_photo_broadening(*extra["broad"])
        o.set_photo(lo, hi)
        Phi = np.outer(np.linspace(0.5, 2.0, len(T)),
                       net.spectrum_draine(lo, hi) + net.spectrum_j21(lo, hi, 1.0, 1.0))
        out[name] = dict(nbins=o.nbins, sigma=o.photo_sigma(), lw=o.lw_weights(),
                         habing=net.habing(Phi, o) if hasattr(net, "habing") else None,
                         heat=net.photo_heating(n, T, o, par=P, Phi=Phi),
                         fluxes=net.fluxes(n, T, par=P, Phi=Phi, opts=o),
                         ratio=net.ratio_flux_draine(Phi, o))
    return out


def _ref_photo_worker(args):
    key, n, T, par = args
    return _photo_survey(key, str(ROOT / "oracle" / "_ref" / ("libkrome_%s.so" % key)),
                         n, T, par)


def test_photon_bins_equal_the_reference():
    """galaxy_ism's eight photo reactions: the bin-averaged cross sections
    (several binnings, in-bin spectra, Doppler broadening of the tabulated
    ones), the Lyman-Werner weights, the photoheating and the reaction
    fluxes of a field, against the reference's library"""
    key = "galaxy_ism"
    if not (ROOT / "oracle" / "_ref" / ("libkrome_%s.so" % key)).exists():
        pytest.skip("oracle/_ref not built here (oracle/build_ref.py)")
    _binding(key)
    n, T, par = _inputs(key)
    ours = _photo_survey(key, str(build.build(key)), n, T, par)
    with mp.get_context("spawn").Pool(1) as pool:
        ref = pool.map(_ref_photo_worker, [(key, n, T, par)])[0]
    assert set(ours) == set(ref)
    for k in ref:
        if isinstance(ref[k], dict):
            for q in ref[k]:
                if ref[k][q] is None:
                    continue
                assert _same(ours[k][q], ref[k][q], 1e-12), (k, q)
        else:
            assert _same(ours[k], ref[k], 1e-13), k
    assert np.asarray(ours["log"]["sigma"]).max() > 0
