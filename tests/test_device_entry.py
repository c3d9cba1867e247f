"""The reference's mass-fraction and device-resident entry points
(krome_solve_cells_x, krome_solve_cells_device, krome_solve_cells_x_device;
reference runtime/interfaces/C/krome.h:296-349).

The lane-per-cell kernel reads and writes the caller's layout itself
(species-major with a leading dimension, or cell-major; densities or mass
fractions with the gas density), so their results equal krome_solve_cells'
bit for bit on the same cells; a failed cell keeps its input; the summary
counts the cells; the required-parameter rule rejects the whole call. The
device-array consistent advection (krome_conserve_cells_device, _x_device,
krome.h:351-360) equals the host entry's."""
import ctypes

import numpy as np
import pytest

from krome_x_b200 import krome, netinfo, workloads

KEY = "primordial3"
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


class Summary(ctypes.Structure):
    _fields_ = [("device", ctypes.c_long), ("host", ctypes.c_long),
                ("failed", ctypes.c_long)]


def _lib(net):
    lib = ctypes.CDLL(str(net.path))
    V = ctypes.c_void_p
    lib.krome_solve_cells.argtypes = [ctypes.c_int, _D, _D, _D, _D,
                                      ctypes.c_int, V, _I, V]
    lib.krome_solve_cells_x.argtypes = [ctypes.c_int, _D, _D, _D, _D, _D,
                                        ctypes.c_int, V, _I, V]
    lib.krome_solve_cells_device.argtypes = [
        ctypes.c_int, V, ctypes.c_int, ctypes.c_long, V, V, V, ctypes.c_int,
        V, V, ctypes.POINTER(Summary), V]
    lib.krome_solve_cells_x_device.argtypes = [
        ctypes.c_int, V, V, ctypes.c_int, ctypes.c_long, V, V, V,
        ctypes.c_int, V, V, ctypes.POINTER(Summary), V]
    for f in ("krome_solve_cells", "krome_solve_cells_x",
              "krome_solve_cells_device", "krome_solve_cells_x_device"):
        getattr(lib, f).restype = ctypes.c_int
    return lib


def _case(ncell, seed=21):
    info = netinfo.load(KEY)
    n, T, dt, par = workloads.primordial3(ncell, info, seed=seed)
    mass = np.asarray(info["mass_g"])
    rho = n @ mass
    x = n * mass / rho[:, None]
    return n, T, dt, par, x, rho, mass


def _opts(net, **extra):
    o = dict(workloads.OPTIONS[KEY])
    o.update(extra)
    return net.options(**o)


def _host(lib, net, n, T, dt, par, opts):
    n, T = n.copy(), T.copy()
    fl = np.zeros(len(T), dtype=np.intc)
    r = lib.krome_solve_cells(len(T), n.ctypes.data_as(_D), T.ctypes.data_as(_D),
                              dt.ctypes.data_as(_D), par.ctypes.data_as(_D),
                              net.npar, None, fl.ctypes.data_as(_I), opts._h)
    return r, n, T, fl


def test_bad_arguments_return_minus_one_before_the_device():
    net = krome.load(KEY)
    lib = _lib(net)
    o = _opts(net)
    buf = (ctypes.c_double * 64)()
    p = ctypes.cast(buf, ctypes.c_void_p)
    s = Summary()
    # a layout that does not exist, a leading dimension below ncell
    assert lib.krome_solve_cells_device(4, p, 2, 0, p, p, p, 0, None, None,
                                        ctypes.byref(s), o._h) == -1
    assert lib.krome_solve_cells_device(4, p, 0, 3, p, p, p, 0, None, None,
                                        ctypes.byref(s), o._h) == -1
    assert lib.krome_solve_cells_device(4, p, 1, 0, p, p, p, 5, None, None,
                                        ctypes.byref(s), o._h) == -1
    assert lib.krome_solve_cells_x_device(4, p, None, 1, 0, p, p, p, 0, None,
                                          None, ctypes.byref(s), o._h) == -1
    assert lib.krome_solve_cells_device(0, p, 1, 0, p, p, p, 0, None, None,
                                        ctypes.byref(s), o._h) == 0
    assert (s.device, s.host, s.failed) == (0, 0, 0)
    x = np.zeros((2, net.nspec))
    T = np.ones(2)
    assert lib.krome_solve_cells_x(2, x.ctypes.data_as(_D), None,
                                   T.ctypes.data_as(_D), T.ctypes.data_as(_D),
                                   None, 0, None, None, o._h) == -1


@pytest.mark.gpu
@pytest.mark.parametrize("layout,pad", [(0, 0), (0, 7), (1, 0)])
def test_device_entry_equals_the_host_entry(layout, pad):
    import torch
    net = krome.load(KEY)
    lib = _lib(net)
    ncell = 512
    n, T, dt, par, _, _, _ = _case(ncell)
    opts = _opts(net, fail_every=9)
    r0, n0, T0, f0 = _host(lib, net, n, T, dt, par, opts)
    dev = torch.device("cuda:0")
    ld = ncell + pad
    if layout == 0:
        a = np.zeros((net.nspec, ld))
        a[:, :ncell] = n.T
    else:
        a = n.copy()
    t = lambda v: torch.tensor(np.ascontiguousarray(v), device=dev)
    da, dT, ddt, dp = t(a), t(T), t(dt), t(par)
    dfl = torch.zeros(ncell, dtype=torch.int32, device=dev)
    s = Summary()
    r = lib.krome_solve_cells_device(
        ncell, da.data_ptr(), layout, ld if layout == 0 else 0, dT.data_ptr(),
        ddt.data_ptr(), dp.data_ptr(), net.npar, None, dfl.data_ptr(),
        ctypes.byref(s), opts._h)
    out = da.cpu().numpy()
    nout = out[:, :ncell].T if layout == 0 else out
    assert r == r0 == -1  # the injected failures: the lowest one's flag
    np.testing.assert_array_equal(dfl.cpu().numpy(), f0)
    np.testing.assert_array_equal(nout, n0)
    np.testing.assert_array_equal(dT.cpu().numpy(), T0)
    if layout == 0 and pad:
        assert (out[:, ncell:] == 0).all()  # the padding is not touched
    failed = int((f0 != 0).sum())
    assert (s.device, s.host, s.failed) == (ncell - failed, 0, failed)
    np.testing.assert_array_equal(nout[f0 != 0], n[f0 != 0])


@pytest.mark.gpu
@pytest.mark.parametrize("renormalize", [0, 1])
def test_mass_fraction_entries_equal_the_density_solve(renormalize):
    import torch
    net = krome.load(KEY)
    lib = _lib(net)
    ncell = 256
    n, T, dt, par, x, rho, mass = _case(ncell, seed=4)
    opts = _opts(net, renormalize_x=renormalize)
    # the host entry
    xh, Th = x.copy(), T.copy()
    fh = np.zeros(ncell, dtype=np.intc)
    rh = lib.krome_solve_cells_x(ncell, xh.ctypes.data_as(_D),
                                 rho.ctypes.data_as(_D), Th.ctypes.data_as(_D),
                                 dt.ctypes.data_as(_D), par.ctypes.data_as(_D),
                                 net.npar, None, fh.ctypes.data_as(_I), opts._h)
    # the same through the density entry, converted by hand
    nin = np.where(mass > 0, rho[:, None] * x / mass, 0.0)
    r0, n0, T0, f0 = _host(lib, net, nin, T, dt, par, opts)
    assert rh == r0
    np.testing.assert_array_equal(fh, f0)
    want = mass * n0 / rho[:, None]
    if renormalize:
        s = want.sum(axis=1)
        want = want * (x.sum(axis=1) / s)[:, None]
    ok = f0 == 0
    np.testing.assert_allclose(xh[ok], want[ok], rtol=1e-14, atol=0)
    np.testing.assert_array_equal(Th, T0)
    if renormalize:
        np.testing.assert_allclose(xh.sum(axis=1), x.sum(axis=1), rtol=1e-14)
    # the device entry, species-major: the host entry's result bit for bit
    dev = torch.device("cuda:0")
    t = lambda v: torch.tensor(np.ascontiguousarray(v), device=dev)
    dx, drho, dT, ddt, dp = t(x.T), t(rho), t(T), t(dt), t(par)
    s = Summary()
    rd = lib.krome_solve_cells_x_device(
        ncell, dx.data_ptr(), drho.data_ptr(), 0, 0, dT.data_ptr(),
        ddt.data_ptr(), dp.data_ptr(), net.npar, None, None, ctypes.byref(s),
        opts._h)
    assert rd == rh
    np.testing.assert_array_equal(dx.cpu().numpy().T, xh)
    np.testing.assert_array_equal(dT.cpu().numpy(), Th)
    assert s.device == int(ok.sum())


@pytest.mark.gpu
def test_device_entry_required_parameter_rule():
    import torch
    net = krome.load(KEY)
    lib = _lib(net)
    ncell = 16
    n, T, dt, par, _, _, _ = _case(ncell)
    par = par.copy()
    par[5, net.params.index("tff")] = np.nan
    dev = torch.device("cuda:0")
    t = lambda v: torch.tensor(np.ascontiguousarray(v), device=dev)
    dn, dT, ddt, dp = t(n), t(T), t(dt), t(par)
    dfl = torch.zeros(ncell, dtype=torch.int32, device=dev)
    s = Summary()
    r = lib.krome_solve_cells_device(ncell, dn.data_ptr(), 1, 0, dT.data_ptr(),
                                     ddt.data_ptr(), dp.data_ptr(), net.npar,
                                     None, dfl.data_ptr(), ctypes.byref(s),
                                     _opts(net)._h)
    assert r == -105
    fl = dfl.cpu().numpy()
    assert fl[5] == -105 and (np.delete(fl, 5) == 0).all()
    np.testing.assert_array_equal(dn.cpu().numpy(), n)
    assert (s.device, s.failed) == (0, 1)


@pytest.mark.gpu
def test_python_solve_x_matches_the_c_entry():
    net = krome.load(KEY)
    lib = _lib(net)
    n, T, dt, par, x, rho, _ = _case(64, seed=9)
    opts = _opts(net)
    r = net.solve_x(x, rho, T, dt, par, opts=opts, check=False)
    xh, Th = x.copy(), T.copy()
    fh = np.zeros(64, dtype=np.intc)
    lib.krome_solve_cells_x(64, xh.ctypes.data_as(_D), rho.ctypes.data_as(_D),
                            Th.ctypes.data_as(_D), dt.ctypes.data_as(_D),
                            par.ctypes.data_as(_D), net.npar, None,
                            fh.ctypes.data_as(_I), opts._h)
    np.testing.assert_array_equal(r.n, xh)
    np.testing.assert_array_equal(r.Tgas, Th)
    np.testing.assert_array_equal(r.flags, fh)
    # the caller's arrays are not modified (the reference's contract)
    np.testing.assert_array_equal(x, _case(64, seed=9)[4])


def _conserve_lib(net):
    lib = ctypes.CDLL(str(net.path))
    V = ctypes.c_void_p
    for f in ("krome_conserve_cells_device", "krome_conserve_cells_x_device"):
        fn = getattr(lib, f)
        fn.argtypes = [ctypes.c_int, V, ctypes.c_int, ctypes.c_long, V,
                       ctypes.c_int, V, ctypes.c_int, V]
        fn.restype = ctypes.c_int
    for f in ("krome_conserve_cells", "krome_conserve_cells_x",
              "krome_get_element_totals", "krome_get_element_totals_x"):
        getattr(lib, f).restype = ctypes.c_int
    return lib


def test_device_conservation_rejects_bad_arguments():
    net = krome.load(KEY)
    lib = _conserve_lib(net)
    buf = (ctypes.c_double * 64)()
    p = ctypes.cast(buf, ctypes.c_void_p)
    f = lib.krome_conserve_cells_device
    assert f(4, p, 2, 0, p, 0, None, 0, None) == -1          # layout
    assert f(4, p, 0, 3, p, 0, None, 0, None) == -1          # ld < ncell
    assert f(4, p, 1, 0, p, 3, None, 0, None) == -1          # ref_stride
    assert f(4, p, 1, 0, None, 0, None, 0, None) == -1       # no ref
    assert f(0, p, 1, 0, p, 0, None, 0, None) == 0           # nothing to do


@pytest.mark.gpu
@pytest.mark.parametrize("mass", [0, 1])
@pytest.mark.parametrize("layout,pad", [(0, 5), (1, 0)])
def test_device_conservation_equals_the_host_entry(mass, layout, pad):
    """krome_conserve_cells(_x)_device (reference krome.h:351-360) on the
    caller's layout: the host entry's cells and flags (the projection's
    arithmetic may contract differently on the device: 1e-13)"""
    import torch
    net = krome.load(KEY)
    lib = _conserve_lib(net)
    ncell = 300
    n, T, dt, par, x, rho, m = _case(ncell, seed=17)
    nelem = lib.krome_nelem()
    rng = np.random.default_rng(5)
    adv = n * rng.uniform(0.7, 1.3, n.shape)
    adv[3, 0] = -1e-30
    tot = np.zeros((ncell, nelem))
    if mass:
        v = adv * m / rho[:, None]
        lib.krome_get_element_totals_x(ncell, x.ctypes.data_as(_D),
                                       tot.ctypes.data_as(_D))
        host = lib.krome_conserve_cells_x
        dev_fn = lib.krome_conserve_cells_x_device
    else:
        v = adv
        lib.krome_get_element_totals(ncell, n.ctypes.data_as(_D),
                                     tot.ctypes.data_as(_D))
        host = lib.krome_conserve_cells
        dev_fn = lib.krome_conserve_cells_device
    vh = v.copy()
    fh = np.zeros(ncell, dtype=np.intc)
    rh = host(ncell, vh.ctypes.data_as(_D), tot.ctypes.data_as(_D), nelem,
              None, 0, fh.ctypes.data_as(_I))
    dev = torch.device("cuda:0")
    ld = ncell + pad
    if layout == 0:
        a = np.zeros((net.nspec, ld))
        a[:, :ncell] = v.T
    else:
        a = v.copy()
    t = lambda z: torch.tensor(np.ascontiguousarray(z), device=dev)
    da, dref = t(a), t(tot)
    dfl = torch.zeros(ncell, dtype=torch.int32, device=dev)
    rd = dev_fn(ncell, da.data_ptr(), layout, ld if layout == 0 else 0,
                dref.data_ptr(), nelem, None, 0, dfl.data_ptr())
    out = da.cpu().numpy()
    vd = out[:, :ncell].T if layout == 0 else out
    assert rd == rh
    np.testing.assert_array_equal(dfl.cpu().numpy(), fh)
    np.testing.assert_allclose(vd, vh, rtol=1e-13, atol=1e-300)
    if layout == 0 and pad:
        assert (out[:, ncell:] == 0).all()
    # without flags: the same return value
    da2 = t(a)
    assert dev_fn(ncell, da2.data_ptr(), layout, ld if layout == 0 else 0,
                  dref.data_ptr(), nelem, None, 0, None) == rh
