"""Further networks through the emitter: primordialZ (the reference's
networks/primordialZ.knet, default thermal options; 27 species, 74
reactions, fixed Tgas), solved by the small-network kernels.

Its rates depend on the densities (the metal reactions switch off above
ntot = 1e14, the H2 dissociation rates depend on the H nuclei density):
the analytic Jacobian adds their dk/dn terms as the reference's does
(kromex/codegen.py:8462-8560: symbolic derivatives, difference quotients
of rates that call fitted functions, the aggregates' coupling U W^T).
With either Jacobian the oracle equals the reference's build bit for bit,
and the kernels match the oracle.

earlyUniverse (networks/earlyUniverse.knet, default thermal options, 16
species, fixed Tgas) adds the RECFAST recombination rates (csrc/
kb_physics.h) and a freeze directive: its e-, H and D species stop above
z = 2243. As the reference does (solve_cell.hpp:1631-1642), a network with
freezable species runs without the charge-invariant Newton correction; a
cell whose freeze holds has the frozen species' rows of the rhs and of the
analytic Jacobian at zero (freeze_rows_, jac_cell_: solve_cell.hpp:711-720,
1118-1131), so those species keep their input densities, and the
conservation does not move them (conserved_fixed_, 1442-1450)."""
import re

import numpy as np
import pytest

from conftest import ROOT, parity
from krome_x_b200 import krome, netinfo, workloads
from oracle import Oracle, reference_solve

KEY = "primordialZ"
SMALL = ("primordial", "primordial3", "galaxy_ism", KEY, "earlyUniverse")
FURTHER = (KEY, "earlyUniverse")


def _ndep(key):
    h = (ROOT / "krome_x_b200" / "networks" / ("net_%s.h" % key)).read_text()
    return int(re.search(r"KB_RATE_NDEP = (\d+);", h).group(1))


@pytest.mark.parametrize("key", SMALL)
def test_density_dependent_rates_match_the_reference_jacobian(key):
    gen = ROOT / "oracle" / "_ref" / "gen" / key
    if not gen.exists():
        pytest.skip("oracle/_ref not built here (oracle/build_ref.py)")
    jac = next(gen.glob("net_*_jacobian.hpp")).read_text()
    has_dk = "// dk of " in jac or "numerical dk/dn" in jac
    assert (_ndep(key) > 0) == has_dk


@pytest.mark.parametrize("key", FURTHER)
def test_oracle_equals_the_reference(key):
    if not (ROOT / "oracle" / "_ref" / ("libkrome_%s_strict.so" % key)).exists():
        pytest.skip("oracle/_ref not built here (oracle/build_ref.py)")
    info = netinfo.load(key)
    n, T, dt, par = workloads.GENERATORS[key](48, info, seed=61)
    o = workloads.OPTIONS[key]
    ref = reference_solve(key, n, T, dt, par, strict=True, **o)
    out = Oracle(key).solve(n, T, dt, par, **o)
    assert (ref["flags"] == 0).all()
    np.testing.assert_array_equal(out["flags"], ref["flags"])
    np.testing.assert_array_equal(out["n"], ref["n"])
    np.testing.assert_array_equal(out["T"], ref["T"])


# the analytic Jacobian on networks whose rates depend on the densities
# (explicit, and JAC_AUTO at fixed Tgas: solve_cell.hpp:2141-2142)
ANALYTIC = [("primordial3", {"jac": 1}), ("galaxy_ism", {"jac": 1}),
            (KEY, {"jac": 1}), (KEY, {"jac": 0}), ("earlyUniverse", {"jac": 0})]


@pytest.mark.parametrize("key,extra", ANALYTIC,
                         ids=["%s-jac%d" % (k, e["jac"]) for k, e in ANALYTIC])
def test_analytic_jacobian_with_rate_terms_equals_the_reference(key, extra):
    if not (ROOT / "oracle" / "_ref" / ("libkrome_%s_strict.so" % key)).exists():
        pytest.skip("oracle/_ref not built here (oracle/build_ref.py)")
    info = netinfo.load(key)
    n, T, dt, par = workloads.GENERATORS[key](24, info, seed=91)
    o = dict(workloads.OPTIONS[key], **extra)
    ref = reference_solve(key, n, T, dt, par, strict=True, **o)
    out = Oracle(key).solve(n, T, dt, par, **o)
    assert (ref["flags"] == 0).all()
    np.testing.assert_array_equal(out["flags"], ref["flags"])
    np.testing.assert_array_equal(out["n"], ref["n"])
    np.testing.assert_array_equal(out["T"], ref["T"])


def _frozen_case(ncell, seed):
    """earlyUniverse cells, every other one above the freeze redshift"""
    key = "earlyUniverse"
    info = netinfo.load(key)
    n, T, dt, par = workloads.GENERATORS[key](ncell, info, seed=seed)
    iz = info["params"].index("zredshift")
    hot = np.arange(ncell) % 2 == 1
    par[hot, iz] = 3000.0
    return key, info, n, T, dt, par, hot


def _frozen_rows(info, par):
    """per cell, the species a freeze directive holds (earlyUniverse: every
    H and D species and the electrons above z = 2243)"""
    sp = info["species"]
    held = [i for i, s in enumerate(sp)
            if s in ("E", "e-", "H", "H2", "H+", "H2+", "H-", "D", "D+",
                     "HD", "HD+", "H2D+", "H3+")]
    iz = info["params"].index("zredshift")
    m = np.zeros((len(par), len(sp)), dtype=bool)
    m[np.ix_(par[:, iz] > 2243.0, held)] = True
    return m


def test_oracle_equals_the_reference_with_frozen_rows():
    key, info, n, T, dt, par, hot = _frozen_case(16, 66)
    o = workloads.OPTIONS[key]
    out = Oracle(key).solve(n, T, dt, par, **o)
    assert (out["flags"] == 0).all()
    fr = _frozen_rows(info, par)
    assert fr[hot].sum(axis=1).min() >= 10
    np.testing.assert_array_equal(out["n"][fr], n[fr])
    assert (out["n"][hot] != n[hot]).any()  # the helium still evolves
    if not (ROOT / "oracle" / "_ref" / ("libkrome_%s_strict.so" % key)).exists():
        pytest.skip("oracle/_ref not built here (oracle/build_ref.py)")
    ref = reference_solve(key, n, T, dt, par, strict=True, **o)
    np.testing.assert_array_equal(out["flags"], ref["flags"])
    np.testing.assert_array_equal(out["n"], ref["n"])
    np.testing.assert_array_equal(out["T"], ref["T"])


def test_conservation_holds_frozen_species():
    """krome_conserve_cells with the cells' parameter rows: species a freeze
    directive holds do not move (the reference's conserved_fixed_)"""
    import ctypes
    key, info, n, T, dt, par, hot = _frozen_case(16, 68)
    net = krome.load(key)
    lib = ctypes.CDLL(str(net.path))
    D = ctypes.POINTER(ctypes.c_double)
    lib.krome_nelem.restype = ctypes.c_int
    ne = lib.krome_nelem()
    tot = np.zeros((16, ne))
    lib.krome_get_element_totals(16, n.ctypes.data_as(D), tot.ctypes.data_as(D))
    adv = n * np.random.default_rng(2).uniform(0.9, 1.1, n.shape)
    v = adv.copy()
    fl = np.zeros(16, dtype=np.intc)
    lib.krome_conserve_cells(16, v.ctypes.data_as(D), tot.ctypes.data_as(D),
                             ne, par.ctypes.data_as(D), net.npar,
                             fl.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    fr = _frozen_rows(info, par)
    np.testing.assert_array_equal(v[fr], adv[fr])
    assert (v[~hot] != adv[~hot]).any()


@pytest.mark.parametrize("key", FURTHER)
def test_workload_is_physical(key):
    info = netinfo.load(key)
    n, T, dt, par = workloads.GENERATORS[key](256, info, seed=63)
    assert (n > 0).all()
    q = np.asarray(info["charge"], dtype=float)
    np.testing.assert_allclose(n @ q, 0.0, atol=1e-12 * n.sum(axis=1).max())


# fixed-Tgas solves of the small networks: primordialZ's workload, and the
# benchmark networks at fixed Tgas (primordial: the analytic Jacobian;
# galaxy_ism: the difference quotients its density-dependent rates take)
FIXED_T = [(KEY, {}), ("earlyUniverse", {}), ("primordial", {"evolve_T": 0}),
           ("galaxy_ism", {"evolve_T": 0})]


@pytest.mark.gpu
@pytest.mark.parametrize("key,extra", FIXED_T, ids=[k for k, _ in FIXED_T])
@pytest.mark.parametrize("layout", ["lane", "warp"])
def test_gpu_matches_the_oracle(key, extra, layout):
    info = netinfo.load(key)
    n, T, dt, par = workloads.GENERATORS[key](512, info, seed=64)
    o = dict(workloads.OPTIONS[key], **extra)
    ref = Oracle(key).solve(n, T, dt, par, **o)
    net = krome.load(key)
    opts = net.options(**dict(o, layout=0 if layout == "warp" else 1))
    r = net.solve_batch(n, T, dt, par, opts=opts, check=False, stats=True)
    m = parity(r.n, r.Tgas, r.flags, ref["n"], ref["T"], ref["flags"], o["rtol"])
    assert m["flags_equal"] == 1.0 and m["frac"] >= 0.85, m
    g, c = r.stats[:, 0].mean(), ref["stats"][:, 0].mean()
    assert abs(g - c) <= 0.03 * c + 0.5, (g, c)


@pytest.mark.gpu
@pytest.mark.parametrize("key,extra", ANALYTIC,
                         ids=["%s-jac%d" % (k, e["jac"]) for k, e in ANALYTIC])
@pytest.mark.parametrize("layout", ["lane", "warp"])
def test_gpu_analytic_jacobian_with_rate_terms_matches_the_oracle(key, extra,
                                                                  layout):
    info = netinfo.load(key)
    n, T, dt, par = workloads.GENERATORS[key](256, info, seed=65)
    o = dict(workloads.OPTIONS[key], **extra)
    ref = Oracle(key).solve(n, T, dt, par, **o)
    net = krome.load(key)
    opts = net.options(**dict(o, layout=0 if layout == "warp" else 1))
    r = net.solve_batch(n, T, dt, par, opts=opts, check=False, stats=True)
    m = parity(r.n, r.Tgas, r.flags, ref["n"], ref["T"], ref["flags"], o["rtol"])
    assert m["flags_equal"] == 1.0 and m["frac"] >= 0.85, m
    g, c = r.stats[:, 0].mean(), ref["stats"][:, 0].mean()
    assert abs(g - c) <= 0.03 * c + 0.5, (g, c)


@pytest.mark.gpu
@pytest.mark.parametrize("layout", ["lane", "warp"])
def test_gpu_matches_the_oracle_with_frozen_rows(layout):
    key, info, n, T, dt, par, hot = _frozen_case(256, 67)
    o = workloads.OPTIONS[key]
    ref = Oracle(key).solve(n, T, dt, par, **o)
    net = krome.load(key)
    opts = net.options(**dict(o, layout=0 if layout == "warp" else 1))
    r = net.solve_batch(n, T, dt, par, opts=opts, check=False)
    m = parity(r.n, r.Tgas, r.flags, ref["n"], ref["T"], ref["flags"], o["rtol"])
    assert m["flags_equal"] == 1.0 and m["frac"] >= 0.85, m
    fr = _frozen_rows(info, par)
    np.testing.assert_array_equal(r.n[fr], n[fr])
