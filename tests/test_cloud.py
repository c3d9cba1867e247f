"""A second large network on the sparse path: the reference's gas-phase
dark-cloud chemistry (networks/cloud.knet: 452 species, 4,429 reactions, no
density-dependent rates), emitted by the same generator as Semenov and
solved by the same block-per-cell kernel from its own generation-time
tables (a 292-row sparse part, a 160-row dense block). The bar is the large
networks' parity metric (conftest.parity_major), as for Semenov. Its rates
against the reference's K_REF vectors, its exports and its metadata are
checked with every network's (test_oracle_pin, test_abi)."""
import numpy as np
import pytest

from conftest import golden, parity_major
from krome_x_b200 import krome, netinfo, workloads
from oracle import Oracle

KEY = "cloud"


def test_cloud_oracle_equals_reference_fixture_bitwise():
    """16 reference-solved cells: the oracle equals the reference's strict
    build bit for bit (on this network the generation-time elimination
    order is the reference's own), flags and Tgas too"""
    g = golden(KEY)
    opts = workloads.OPTIONS[KEY]
    out = Oracle(KEY).solve(g["n"], g["T"], g["dt"], g["par"], **opts)
    assert out["ret"] == g["ret"]
    m = parity_major(out["n"], out["flags"], g["n_out"], g["flags"], g["n"],
                     opts["rtol"])
    assert m["flags_equal"] == 1.0 and m["cells"] == len(g["n"]), m
    np.testing.assert_array_equal(out["n"], g["n_out"])
    np.testing.assert_array_equal(out["flags"], g["flags"])
    np.testing.assert_array_equal(out["T"], g["T_out"])


@pytest.mark.gpu
def test_cloud_gpu_parity_with_reference_fixture_and_oracle():
    """the GPU's sparse path on this network's tables against the
    reference's fixture and the oracle: the large networks' bar, flags
    equal, the oracle's step counts within the chaotic spread, mass
    conserved"""
    g = golden(KEY)
    opts = workloads.OPTIONS[KEY]
    net = krome.load(KEY)
    r = net.solve_batch(g["n"], g["T"], g["dt"], g["par"],
                        opts=net.options(**opts), check=False, stats=True)
    m = parity_major(r.n, r.flags, g["n_out"], g["flags"], g["n"],
                     opts["rtol"])
    assert m["flags_equal"] == 1.0 and m["cells"] == len(g["n"]), m
    assert m["max_rel"] < 2e-4 and m["frac"] >= 0.7, m
    assert r.ierr == g["ret"]
    np.testing.assert_array_equal(r.Tgas, g["T_out"])
    info = netinfo.load(KEY)
    n, T, dt, par = workloads.cloud(32, info, seed=3)
    ref = Oracle(KEY).solve(n, T, dt, par, **opts)
    r = net.solve_batch(n, T, dt, par, opts=net.options(**opts), check=False,
                        stats=True)
    m = parity_major(r.n, r.flags, ref["n"], ref["flags"], n, opts["rtol"])
    assert m["flags_equal"] == 1.0 and m["cells"] == 32, m
    assert m["max_rel"] < 2e-4 and m["frac"] >= 0.7, m
    mass = np.asarray(info["mass_g"])
    np.testing.assert_allclose(r.n @ mass, n @ mass, rtol=1e-10)
    a, b = r.stats[:, 0].mean(), ref["stats"][:, 0].mean()
    assert abs(a - b) <= 0.05 * b, (a, b)


EVT = dict(evolve_T=1, jac=1)


def test_cloud_evolved_tgas_oracle_equals_reference_bitwise():
    """8 reference-solved cells with Tgas evolved and the hybrid Jacobian:
    the oracle's bordered sparse LU (B' = L^-1 cB, C' = cC U^-1, the Schur
    complement Z and the bordered solve) equals the reference's strict
    build bit for bit; Tgas (no thermal processes) comes back unchanged"""
    g = golden("cloud_evt")
    opts = dict(workloads.OPTIONS[KEY])
    opts.update(EVT)
    out = Oracle(KEY).solve(g["n"], g["T"], g["dt"], g["par"], **opts)
    np.testing.assert_array_equal(out["flags"], g["flags"])
    np.testing.assert_array_equal(out["n"], g["n_out"])
    np.testing.assert_array_equal(out["T"], g["T_out"])
    np.testing.assert_array_equal(g["T_out"], g["T"])


@pytest.mark.gpu
def test_cloud_gpu_evolved_tgas_parity():
    """the GPU's bordered solve on this network against the reference's
    evolved-Tgas fixture: the large networks' bar, flags equal, Tgas
    returned"""
    g = golden("cloud_evt")
    opts = dict(workloads.OPTIONS[KEY])
    opts.update(EVT)
    net = krome.load(KEY)
    r = net.solve_batch(g["n"], g["T"], g["dt"], g["par"],
                        opts=net.options(**opts), check=False)
    m = parity_major(r.n, r.flags, g["n_out"], g["flags"], g["n"],
                     opts["rtol"])
    assert m["flags_equal"] == 1.0 and m["cells"] == len(g["n"]), m
    assert m["max_rel"] < 2e-4 and m["frac"] >= 0.7, m
    np.testing.assert_array_equal(r.Tgas, g["T_out"])
