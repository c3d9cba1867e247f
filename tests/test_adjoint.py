"""The discrete adjoint (krome_b200_adjoint, the torch.autograd wrapper).

The gradient is that of the discrete solution (the forward's step sizes,
orders and Newton decisions held fixed, each accepted corrector
differentiated at its root). Checks, on the benchmark's differentiation
workload (the primordial network, x_H2 = n_H2 / n_H and Tgas as outputs,
the initial n and Tgas and the per-reaction ln-multipliers as inputs):

* the oracle's reverse sweep is the exact transpose of its tangent sweep
  over the same tape (a dot-product test to 1e-9);
* the oracle's gradient against central finite differences of
  tight-tolerance (rtol 1e-11) solves, step 1e-3 in ln k and relative 1e-4
  in the state, on 64 cells, every ln k, every species and Tgas, per cell
  as the largest difference over the gradient relative to its largest
  component: every cell whose temperature stays on one side of the
  network's piecewise rate breakpoints within 1e-4. A cell that crosses
  one (primordial's H+ + e- -> H fit jumps at 5500 K) differs by up to a
  few 1e-2: the finite differences see the jump move with the crossing
  time, which the adjoint of the smooth pieces leaves out (the same cells
  at rtol 1e-10 still differ by that much, while the others agree to
  ~1e-10);
* the GPU adjoint against the oracle's on the same seeded cells (the
  parity of the forward solves carries over to the gradients), and against
  the same finite differences;
* the autograd wrapper against the host entry point, and the failure rules
  (a full tape: -120, the cell untouched, zero gradients).
"""
import ctypes
import re

import numpy as np
import pytest

from conftest import NETWORKS, ROOT
from krome_x_b200 import krome, netinfo, workloads
from oracle import Oracle

KEY = "primordial"
TIGHT = dict(rtol=1e-11, max_steps=5000000)


def cells(ncell, seed, pick=None):
    """seeded primordial cells; pick: keep the densest `pick` of them"""
    info = netinfo.load(KEY)
    n, T, dt, par = workloads.primordial(ncell, info, seed=seed)
    if pick is not None:
        idx = np.argsort(-n[:, info["species"].index("H")])[:pick]
        n, T, dt, par = n[idx], T[idx], dt[idx], par[idx]
    return info, n, T, dt, par


def seeds(info, n, T):
    """x_H2 = n_H2 / n_H (initial H nuclei, constant weights) and Tgas / T0"""
    sp = info["species"]
    w = np.array([{"H": 1, "H+": 1, "H-": 1, "H2": 2, "H2+": 2,
                   "HD": 1}.get(s, 0) for s in sp], dtype=float)
    nH = n @ w
    gx = np.zeros_like(n)
    gx[:, sp.index("H2")] = 1.0 / nH
    return gx, np.zeros(len(T)), np.zeros_like(n), 1.0 / T


def normalised_error(g, ref):
    """per cell: max |g - ref| / max |ref|"""
    scale = np.maximum(np.abs(ref).max(axis=1), 1e-300)
    return np.abs(g - ref).max(axis=1) / scale


def fd_gradients(n, T, dt, par, objs, reactions, species, eps=1e-3):
    """central differences of tight oracle solves: d obj / d ln k_r for the
    given reactions, d obj / d ln n_j for the given species and d / d ln T0
    (objs: functions of (n_out, T_out) -> per-cell values)"""
    orc = Oracle(KEY)
    nrea = orc.lib.oracle_nrea()
    o = dict(workloads.OPTIONS[KEY], **TIGHT)
    z = np.zeros_like(n)
    zt = np.zeros(len(T))

    def run(nn, TT, lnm=None):
        r = orc.adjoint(nn, TT, dt, par, z, zt, lnm=lnm, **o)
        assert (r["flags"] == 0).all()
        return [f(r["n"], r["T"]) for f in objs]
    out = [dict(k={}, n={}, T=None) for _ in objs]
    for r in reactions:
        lp = np.zeros(nrea)
        lp[r] = eps
        a, b = run(n, T, lp), run(n, T, -lp)
        for i in range(len(objs)):
            out[i]["k"][r] = (a[i] - b[i]) / (2 * eps)
    for j in species:
        npl, nmi = n.copy(), n.copy()
        npl[:, j] *= 1 + 1e-4
        nmi[:, j] *= 1 - 1e-4
        a, b = run(npl, T), run(nmi, T)
        for i in range(len(objs)):
            out[i]["n"][j] = (a[i] - b[i]) / 2e-4
    a, b = run(n, T * (1 + 1e-4)), run(n, T * (1 - 1e-4))
    for i in range(len(objs)):
        out[i]["T"] = (a[i] - b[i]) / 2e-4
    return out


def breakpoints(key):
    """the temperatures at which the network's piecewise rate fits switch
    (the emitted groups' range tests)"""
    h = (ROOT / "krome_x_b200" / "networks" / ("net_%s.h" % key)).read_text()
    return sorted({float(v) for v in
                   re.findall(r"\bT (?:<|>=|>|<=) ([0-9][0-9.e+]*)", h)})


def crossing(T0, Tend, key=KEY):
    """per cell: whether its temperature passes a rate breakpoint between
    the initial and the final state"""
    lo, hi = np.minimum(T0, Tend), np.maximum(T0, Tend)
    bp = np.array(breakpoints(key))
    return ((lo[:, None] < bp[None, :]) & (bp[None, :] < hi[:, None])).any(1)


def check_against_fd(res_for_seed, n, T, Tend, fd, reactions, species,
                     frac=1.0):
    """res_for_seed(i) -> (dm, dn0, dT0) of objective i; the per-cell
    normalised errors: within 1e-4 on (a fraction frac of) the cells whose
    temperature stays between two rate breakpoints, those within 1e-3 all,
    and at most 0.1 on the others (a wrong sign or a missing term is an
    O(1) error)"""
    cross = crossing(T, Tend)
    assert (~cross).sum() >= len(T) // 2, cross
    for i, f in enumerate(fd):
        dm, dn0, dT0 = res_for_seed(i)
        ref = np.stack([f["k"][r] for r in reactions]
                       + [f["n"][j] for j in species] + [f["T"]], axis=1)
        got = np.stack([dm[:, r] for r in reactions]
                       + [dn0[:, j] * n[:, j] for j in species]
                       + [dT0 * T], axis=1)
        err = normalised_error(got, ref)
        assert (err[~cross] <= 1e-4).mean() >= frac, (i, err[~cross], err)
        assert (err[~cross] <= 1e-3).all(), (i, err[~cross].max(), err)
        assert (err <= 0.1).all(), (i, err)


REACTIONS = list(range(38))
SPECIES = ("D", "D+", "E", "H", "H+", "H-", "H2", "H2+", "HD", "He", "He+",
           "He++")


_FD = {}


def fd_case():
    """64 seeded cells (the densest of 192), every reaction, species and
    Tgas; computed once per process"""
    if "case" not in _FD:
        info, n, T, dt, par = cells(192, seed=5, pick=64)
        sp = info["species"]
        species = [sp.index(s if s in sp else "e-") for s in SPECIES]
        gx, gxT, gT0n, gT = seeds(info, n, T)
        objs = [lambda a, b: (a * gx).sum(1), lambda a, b: b * gT]
        fd = fd_gradients(n, T, dt, par, objs, REACTIONS, species)
        _FD["case"] = ((n, T, dt, par), species, ((gx, gxT), (gT0n, gT)), fd)
    return _FD["case"]


def test_oracle_adjoint_is_the_transpose_of_its_tangent():
    info, n, T, dt, par = cells(48, seed=5, pick=6)
    orc = Oracle(KEY)
    lib = orc.lib
    D = ctypes.POINTER(ctypes.c_double)
    lib.oracle_tangent_one.restype = ctypes.c_int
    lib.oracle_tangent_one.argtypes = [D] * 8 + [ctypes.c_void_p]
    import oracle as om
    o = workloads.OPTIONS[KEY]
    so = om._Opts(1, o["jac"], o["rtol"], o["atol_n"], o["atol_T"], 100000,
                  7, 10, 5, 1, 0)
    rng = np.random.default_rng(1)
    nrea = lib.oracle_nrea()
    p = lambda a: a.ctypes.data_as(D)
    for c in range(len(T)):
        lam = rng.normal(size=n.shape[1] + 1)
        dy0 = rng.normal(size=n.shape[1] + 1) * np.append(n[c], T[c])
        dm = rng.normal(size=nrea)
        dyf = np.zeros(n.shape[1] + 1)
        assert lib.oracle_tangent_one(p(n[c].copy()), p(T[c:c + 1].copy()),
                                      p(dt[c:c + 1].copy()), p(par[c].copy()),
                                      None, p(dy0), p(dm), p(dyf),
                                      ctypes.byref(so)) == 0
        a = orc.adjoint(n[c:c + 1], T[c:c + 1], dt[c:c + 1], par[c:c + 1],
                        lam[None, :-1], lam[-1:], **o)
        lhs = lam @ dyf
        rhs = (np.append(a["dn0"][0], a["dT0"][0]) @ dy0 + a["dm"][0] @ dm)
        assert abs(lhs - rhs) <= 1e-8 * (abs(lhs) + abs(rhs)), (c, lhs, rhs)


def test_oracle_adjoint_matches_tight_finite_differences():
    (n, T, dt, par), species, sd, fd = fd_case()
    orc = Oracle(KEY)
    o = workloads.OPTIONS[KEY]
    res = [orc.adjoint(n, T, dt, par, g, gt, **o) for g, gt in sd]
    check_against_fd(lambda i: (res[i]["dm"], res[i]["dn0"], res[i]["dT0"]),
                     n, T, res[0]["T"], fd, REACTIONS, species)


@pytest.mark.parametrize("key", NETWORKS)
def test_thermal_row_form_equals_the_thermal_term(key):
    """the adjoint's Tgas row evaluates the cooling's temperature-only parts
    once per row (thermal_pre at the accepted state y) and every column from
    them: the same value as the thermal term itself, bit for bit, at states
    that differ from y in one density"""
    D = ctypes.POINTER(ctypes.c_double)
    lib = Oracle(key).lib
    lib.oracle_thermal_forms.argtypes = [ctypes.c_double, D, D, D, D, D]
    lib.oracle_thermal_forms.restype = None
    lib.oracle_rates.argtypes = [ctypes.c_double, D, D, D]
    info = netinfo.load(key)
    n, T, dt, par = workloads.GENERATORS[key](24, info, seed=12)
    nrea = lib.oracle_nrea()
    for c in range(len(n)):
        y = np.ascontiguousarray(n[c])
        pr = np.ascontiguousarray(np.broadcast_to(par, (len(n), len(info["params"])))[c])
        k = np.zeros(nrea + 1)
        lib.oracle_rates(float(T[c]), y.ctypes.data_as(D), pr.ctypes.data_as(D),
                         k.ctypes.data_as(D))
        Tth = min(max(float(T[c]), 2.73), 1e9)
        for j in range(len(y)):
            yp = y.copy()
            yp[j] += max(1e-7 * abs(y[j]), 1e-9 * np.abs(y).sum(), 1e-30)
            out = np.zeros(2)
            lib.oracle_thermal_forms(Tth, y.ctypes.data_as(D),
                                     yp.ctypes.data_as(D), k.ctypes.data_as(D),
                                     pr.ctypes.data_as(D), out.ctypes.data_as(D))
            assert out[0] == out[1], (key, c, j, out)


def test_adjoint_bad_arguments_and_required_parameters():
    net = krome.load(KEY)
    N = 3
    n = np.ones((N, net.nspec))
    T = np.full(N, 100.0)
    dt = np.full(N, 1e8)
    par = np.ascontiguousarray(net.param_rows(N, tff=1e12))
    D = ctypes.POINTER(ctypes.c_double)
    p = lambda a: a.ctypes.data_as(D)
    g = np.zeros((N, net.nspec))
    out = [np.zeros((N, net.nspec)), np.zeros(N), np.zeros((N, net.nrea))]
    lnm = np.zeros(net.nrea)
    o = net.options()
    lib = net._lib
    assert lib.krome_b200_adjoint(N, p(n), p(T), p(dt), p(par), net.npar,
                                  p(lnm), 5, p(g), p(T), None, p(out[0]),
                                  p(out[1]), p(out[2]), 0, o._h) == -1
    assert lib.krome_b200_adjoint(N, p(n), p(T), p(dt), p(par), 7, None, 0,
                                  p(g), p(T), None, p(out[0]), p(out[1]),
                                  p(out[2]), 0, o._h) == -1
    bad = par.copy()
    bad[1, list(net.params).index("tff")] = np.nan
    flags = np.zeros(N, dtype=np.intc)
    r = lib.krome_b200_adjoint(N, p(n), p(T), p(dt), p(bad), net.npar, None,
                               0, p(g), p(T),
                               flags.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                               p(out[0]), p(out[1]), p(out[2]), 0, o._h)
    assert r == -105 and flags.tolist() == [0, -105, 0]


def gpu_opts(net):
    o = workloads.OPTIONS[KEY]
    return net.options(evolve_T=o["evolve_T"], jac=o["jac"], rtol=o["rtol"],
                       atol_n=o["atol_n"], atol_T=o["atol_T"])


@pytest.mark.gpu
def test_gpu_adjoint_matches_oracle_adjoint():
    info, n, T, dt, par = cells(512, seed=7)
    gx, _, _, gT = seeds(info, n, T)
    net = krome.load(KEY)
    lnm = np.random.default_rng(3).normal(0.0, 0.05, net.nrea)
    g = net.adjoint(n, T, dt, par, gn=gx, gT=gT, lnm=lnm, opts=gpu_opts(net),
                    check=False)
    ref = Oracle(KEY).adjoint(n, T, dt, par, gx, gT, lnm=lnm,
                              **workloads.OPTIONS[KEY])
    assert (g.flags == ref["flags"]).all()
    ok = g.flags == 0
    e_m = normalised_error(g.dm[ok], ref["dm"][ok])
    y0 = np.concatenate([n, T[:, None]], axis=1)[ok]
    e_y = normalised_error(np.concatenate([g.dn0, g.dT0[:, None]], 1)[ok] * y0,
                           np.concatenate([ref["dn0"], ref["dT0"][:, None]],
                                          1)[ok] * y0)
    # the forward solves agree at the parity bar on ~95 % of the cells; the
    # gradients of those cells agree to well within it
    assert np.median(e_m) < 1e-4 and np.median(e_y) < 1e-4, (e_m, e_y)
    assert (e_m < 1e-2).mean() >= 0.95 and (e_y < 1e-2).mean() >= 0.95


@pytest.mark.gpu
def test_gpu_adjoint_matches_tight_finite_differences():
    (n, T, dt, par), species, sd, fd = fd_case()
    net = krome.load(KEY)
    res = [net.adjoint(n, T, dt, par, gn=g, gT=gt, opts=gpu_opts(net))
           for g, gt in sd]
    # the GPU's forward differs from the oracle's in the last bits, which
    # the solve's step decisions amplify to the rtol level
    check_against_fd(lambda i: (res[i].dm, res[i].dn0, res[i].dT0),
                     n, T, res[0].Tgas, fd, REACTIONS, species, frac=0.98)


@pytest.mark.gpu
def test_autograd_wrapper_matches_host_entry_point():
    import torch
    from krome_x_b200 import autograd
    info, n, T, dt, par = cells(256, seed=11)
    net = krome.load(KEY)
    gx, _, _, gT = seeds(info, n, T)
    lnm = np.zeros(net.nrea)
    host = net.adjoint(n, T, dt, par, gn=gx, gT=gT, lnm=lnm,
                       opts=gpu_opts(net), check=False)
    dev = torch.device("cuda:0")
    t = lambda a, rg=False: torch.tensor(a, dtype=torch.float64, device=dev,
                                         requires_grad=rg)
    n0, T0, m = t(n, True), t(T, True), t(lnm, True)
    nout, Tout, flags = autograd.solve(net, n0, T0, m, t(dt), t(par),
                                       gpu_opts(net))
    loss = (nout * t(gx)).sum() + (Tout * t(gT)).sum()
    loss.backward()
    assert (flags.cpu().numpy() == host.flags).all()
    np.testing.assert_array_equal(nout.detach().cpu().numpy(), host.n)
    np.testing.assert_array_equal(n0.grad.cpu().numpy(), host.dn0)
    np.testing.assert_array_equal(T0.grad.cpu().numpy(), host.dT0)
    # a multiplier shared by every cell: the sum of the per-cell gradients
    np.testing.assert_allclose(m.grad.cpu().numpy(), host.dm.sum(0),
                               rtol=1e-12, atol=0)


@pytest.mark.gpu
def test_memory_bounded_adjoint_equals_the_full_tape():
    """max_tape_bytes below the batch's tapes: the forward keeps no tape and
    the backward recomputes chunks of cells from their initial states --
    the same results and gradients, bit for bit (per-cell multiplier and
    parameter rows, so the chunks slice every per-cell array)"""
    import torch
    from krome_x_b200 import autograd
    info, n, T, dt, par = cells(300, seed=12)
    net = krome.load(KEY)
    gx, _, _, gT = seeds(info, n, T)
    rng = np.random.default_rng(3)
    lnm = rng.normal(0.0, 0.05, (300, net.nrea))
    dev = torch.device("cuda:0")
    t = lambda a, rg=False: torch.tensor(a, dtype=torch.float64, device=dev,
                                         requires_grad=rg)
    out = []
    for budget in (None, 64 * 32768 * 8):  # all at once; chunks of 64 cells
        n0, T0, m = t(n, True), t(T, True), t(lnm, True)
        nout, Tout, flags = autograd.solve(net, n0, T0, m, t(dt), t(par),
                                           gpu_opts(net), tape_cap=32768,
                                           max_tape_bytes=budget)
        ((nout * t(gx)).sum() + (Tout * t(gT)).sum()).backward()
        out.append([x.detach().cpu().numpy() for x in
                    (nout, Tout, flags, n0.grad, T0.grad, m.grad)])
    assert (out[0][2] == 0).mean() > 0.9
    for a, b in zip(out[0], out[1]):
        np.testing.assert_array_equal(a, b)


@pytest.mark.gpu
def test_full_tape_fails_the_cell_untouched():
    info, n, T, dt, par = cells(64, seed=13)
    net = krome.load(KEY)
    gx, _, _, gT = seeds(info, n, T)
    r = net.adjoint(n, T, dt, par, gn=gx, gT=gT, opts=gpu_opts(net),
                    tape_cap=64, check=False)
    full = r.flags == -120
    assert full.any() and r.ierr != 0
    np.testing.assert_array_equal(r.n[full], n[full])
    assert (r.dm[full] == 0).all() and (r.dn0[full] == 0).all()
