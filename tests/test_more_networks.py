"""A further network through the emitter: primordialZ (the reference's
networks/primordialZ.knet, default thermal options; 27 species, 74
reactions, fixed Tgas), solved by the small-network kernels.

Its rates depend on the densities (the metal reactions switch off above
ntot = 1e14, the H2 dissociation rates depend on the H nuclei density):
the reference's analytic Jacobian adds their dk/dn terms
(kromex/codegen.py:8462-8560), which the emitted analytic Jacobian does
not, so such networks take the difference-quotient Jacobian (the default
resolves to it; an explicit analytic one is refused with -104). With it the
oracle equals the reference's build bit for bit, and the kernels match the
oracle."""
import re

import numpy as np
import pytest

from conftest import ROOT, parity
from krome_x_b200 import krome, netinfo, workloads
from oracle import Oracle, reference_solve

KEY = "primordialZ"
SMALL = ("primordial", "primordial3", "galaxy_ism", KEY)


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


def test_oracle_equals_the_reference():
    if not (ROOT / "oracle" / "_ref" / ("libkrome_%s_strict.so" % KEY)).exists():
        pytest.skip("oracle/_ref not built here (oracle/build_ref.py)")
    info = netinfo.load(KEY)
    n, T, dt, par = workloads.GENERATORS[KEY](48, info, seed=61)
    o = workloads.OPTIONS[KEY]
    ref = reference_solve(KEY, n, T, dt, par, strict=True, **o)
    out = Oracle(KEY).solve(n, T, dt, par, **o)
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


def test_workload_is_physical():
    info = netinfo.load(KEY)
    n, T, dt, par = workloads.GENERATORS[KEY](256, info, seed=63)
    assert (n > 0).all()
    q = np.asarray(info["charge"], dtype=float)
    np.testing.assert_allclose(n @ q, 0.0, atol=1e-12 * n.sum(axis=1).max())


# fixed-Tgas solves of the small networks: primordialZ's workload, and the
# benchmark networks at fixed Tgas (primordial: the analytic Jacobian;
# galaxy_ism: the difference quotients its density-dependent rates take)
FIXED_T = [(KEY, {}), ("primordial", {"evolve_T": 0}),
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
