"""Further networks through the emitter: primordialZ (the reference's
networks/primordialZ.knet, default thermal options; 27 species, 74
reactions, fixed Tgas), solved by the small-network kernels.

Its rates depend on the densities (the metal reactions switch off above
ntot = 1e14, the H2 dissociation rates depend on the H nuclei density):
the reference's analytic Jacobian adds their dk/dn terms
(kromex/codegen.py:8462-8560), which the emitted analytic Jacobian does
not, so such networks take the difference-quotient Jacobian (the default
resolves to it; an explicit analytic one is refused with -104). With it the
oracle equals the reference's build bit for bit, and the kernels match the
oracle.

earlyUniverse (networks/earlyUniverse.knet, default thermal options, 16
species, fixed Tgas) adds the RECFAST recombination rates (csrc/
kb_physics.h) and a freeze directive: its e-, H and D species stop above
z = 2243. As the reference does (solve_cell.hpp:1631-1642), a network with
freezable species runs without the charge-invariant Newton correction; the
frozen rows themselves are not built, so a cell whose freeze holds is
refused (-104)."""
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


def test_oracle_refuses_the_analytic_jacobian_with_rate_terms():
    info = netinfo.load(KEY)
    n, T, dt, par = workloads.GENERATORS[KEY](4, info, seed=62)
    o = dict(workloads.OPTIONS[KEY], jac=1)
    out = Oracle(KEY).solve(n, T, dt, par, **o)
    assert (out["flags"] == -104).all()
    # the default resolves to the difference quotients: the same solve
    a = Oracle(KEY).solve(n, T, dt, par, **dict(o, jac=0))
    b = Oracle(KEY).solve(n, T, dt, par, **dict(o, jac=2))
    np.testing.assert_array_equal(a["n"], b["n"])


def _frozen_case(ncell, seed):
    """earlyUniverse cells, every other one above the freeze redshift"""
    key = "earlyUniverse"
    info = netinfo.load(key)
    n, T, dt, par = workloads.GENERATORS[key](ncell, info, seed=seed)
    iz = info["params"].index("zredshift")
    hot = np.arange(ncell) % 2 == 1
    par[hot, iz] = 3000.0
    return key, info, n, T, dt, par, hot


def test_oracle_refuses_cells_whose_freeze_holds():
    key, info, n, T, dt, par, hot = _frozen_case(8, 66)
    out = Oracle(key).solve(n, T, dt, par, **workloads.OPTIONS[key])
    assert (out["flags"][hot] == -104).all()
    assert (out["flags"][~hot] == 0).all()
    np.testing.assert_array_equal(out["n"][hot], n[hot])


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
def test_gpu_refuses_the_analytic_jacobian_with_rate_terms():
    info = netinfo.load(KEY)
    n, T, dt, par = workloads.GENERATORS[KEY](8, info, seed=65)
    net = krome.load(KEY)
    opts = net.options(**dict(workloads.OPTIONS[KEY], jac=1))
    r = net.solve_batch(n, T, dt, par, opts=opts, check=False)
    assert r.ierr == -104 and (r.flags == -104).all()


@pytest.mark.gpu
@pytest.mark.parametrize("layout", ["lane", "warp"])
def test_gpu_refuses_cells_whose_freeze_holds(layout):
    key, info, n, T, dt, par, hot = _frozen_case(64, 67)
    o = workloads.OPTIONS[key]
    ref = Oracle(key).solve(n, T, dt, par, **o)
    net = krome.load(key)
    opts = net.options(**dict(o, layout=0 if layout == "warp" else 1))
    r = net.solve_batch(n, T, dt, par, opts=opts, check=False)
    np.testing.assert_array_equal(r.flags, ref["flags"])
    assert (r.flags[hot] == -104).all()
    np.testing.assert_array_equal(r.n[hot], n[hot])
