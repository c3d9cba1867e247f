"""Photon bins on the device (the reference's photo module, runtime/core/
photo.hpp, and the photo branch of its rate evaluation, solve_cell.hpp:
609-614): with photon bins on the handle every cell brings its field
Phi[nbins] (krome_cells' Phi), and each photo reaction's rate is
k_r = sum_b sigma_rb Phi_b with the bins' averaged cross sections.

galaxy_ism's eight photo reactions (H, He, He+, H-, H2 ionization, H2+
dissociation and ionization, H2 photodissociation) under a seeded field per
cell: the Draine interstellar field scaled by G0 in [0.1, 10] plus a J21
power law, J21 in [1e-3, 1], on 24 logarithmic bins of 0.7-300 eV. The
oracle solves the same cells bit for bit as the reference's own build; the
GPU kernels are held to the parity bar against the oracle."""
import numpy as np
import pytest

from conftest import ROOT, assert_at_floor, parity
from krome_x_b200 import krome, netinfo, workloads
from oracle import Oracle, reference_solve

KEY = "galaxy_ism"


def photo_case(ncell, seed):
    """the cells, their field, the bins and the bins' cross sections"""
    info = netinfo.load(KEY)
    n, T, dt, par = workloads.galaxy_ism(ncell, info, seed=seed)
    net = krome.load(KEY)
    lo, hi = net.bins_log(24, 0.7, 300.0)
    rng = np.random.default_rng(seed + 1)
    G0 = np.exp(rng.uniform(np.log(0.1), np.log(10.0), ncell))
    J21 = np.exp(rng.uniform(np.log(1e-3), np.log(1.0), ncell))
    Phi = (G0[:, None] * net.spectrum_draine(lo, hi)[None, :]
           + J21[:, None] * net.spectrum_j21(lo, hi, 1.0, 1.0)[None, :])
    opts = net.options(**workloads.OPTIONS[KEY]).set_photo(lo, hi)
    return net, opts, (n, T, dt, par), Phi, (lo, hi), opts.photo_sigma()


def test_oracle_photo_solve_equals_the_reference():
    if not (ROOT / "oracle" / "_ref" / ("libkrome_%s_strict.so" % KEY)).exists():
        pytest.skip("oracle/_ref not built here (oracle/build_ref.py)")
    net, opts, (n, T, dt, par), Phi, bins, sigma = photo_case(48, 61)
    o = workloads.OPTIONS[KEY]
    ref = reference_solve(KEY, n, T, dt, par, strict=True, photo_bins=bins,
                          Phi=Phi, **o)
    out = Oracle(KEY).solve(n, T, dt, par, photo_sigma=sigma, Phi=Phi, **o)
    np.testing.assert_array_equal(out["flags"], ref["flags"])
    np.testing.assert_array_equal(out["n"], ref["n"])
    np.testing.assert_array_equal(out["T"], ref["T"])
    # the field matters: the same cells without it end elsewhere
    dark = Oracle(KEY).solve(n, T, dt, par, **o)
    e = np.where(dark["n"] > 1e-14, np.abs(dark["n"] - out["n"]) / dark["n"], 0)
    assert e.max() > 1e-2


def test_solve_refuses_bins_without_a_field():
    net = krome.load(KEY)
    info = netinfo.load(KEY)
    n, T, dt, par = workloads.galaxy_ism(4, info, seed=1)
    opts = net.options(**workloads.OPTIONS[KEY]).set_photo(*net.bins_log(4, 1.0, 50.0))
    with pytest.raises(krome.KromeError, match="Phi"):
        net.solve(n, T, dt, par, opts=opts)
    import ctypes
    fl = np.zeros(4, dtype=np.intc)
    D = ctypes.POINTER(ctypes.c_double)
    r = net._lib.krome_solve_cells(4, n.ctypes.data_as(D), T.ctypes.data_as(D),
                                   dt.ctypes.data_as(D), par.ctypes.data_as(D),
                                   net.npar, None,
                                   fl.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                   opts._h)
    assert r == -103 and (fl == -103).all()


@pytest.mark.gpu
@pytest.mark.parametrize("layout,kernel", [("lane", "persistent"),
                                           ("lane", "plain"),
                                           ("warp", "persistent")])
def test_gpu_photo_solve_matches_the_oracle(layout, kernel):
    net, opts, (n, T, dt, par), Phi, bins, sigma = photo_case(512, 62)
    o = workloads.OPTIONS[KEY]
    opts.set(kernel=kernel, layout=0 if layout == "warp" else 1)
    r = net.solve_batch(n, T, dt, par, opts=opts, check=False, Phi=Phi)
    ref = Oracle(KEY).solve(n, T, dt, par, photo_sigma=sigma, Phi=Phi, **o)
    m = parity(r.n, r.Tgas, r.flags, ref["n"], ref["T"], ref["flags"], o["rtol"])
    assert_at_floor(m, "galaxy_ism/photo/512/62")


@pytest.mark.gpu
def test_gpu_photo_rates_match_the_field():
    net, opts, (n, T, dt, par), Phi, bins, sigma = photo_case(64, 63)
    k = net.rates(n, T, par, Phi=Phi, opts=opts)
    k0 = net.rates(n, T, par)
    pr = [net._lib.krome_photo_reaction(r) for r in range(net._lib.krome_nphoto())]
    expect = Phi @ sigma.T  # [ncell, nphoto]
    np.testing.assert_allclose(k[:, pr], expect, rtol=1e-12, atol=0)
    others = np.setdiff1d(np.arange(net.nrea), pr)
    np.testing.assert_array_equal(k[:, others], k0[:, others])
    assert (k0[:, pr] == 0).all()
