"""The large-network (sparse-LU) path: the Semenov surface-chemistry network,
655 species and 5639 reactions, fixed Tgas, and evolved Tgas through the
Newton matrix's Tgas border.

Its GPU solve runs the same CVODE as the oracle with the same static-pivot
sparse LU (a minimum-degree order fixed at generation); the bar is the
large-network parity metric (conftest.parity_major): every abundance above
1e-12 of the cell's density within 2e-4 -- one input ulp moves the oracle by
up to ~5e-5 on this workload -- most cells within 10 rtol, flags equal, and
the total mass conserved."""
import ctypes
import re

import numpy as np
import pytest

from conftest import ROOT, golden, parity_major
from krome_x_b200 import krome, netinfo, workloads
from oracle import Oracle

KEY = "semenov"
TABLES = ("sp_rp", "sp_ci", "sp_di", "sp_perm", "sp_jpos", "bk_frow",
          "bk_flp", "bk_brow", "bk_blp", "bk_uoff", "bk_tgt", "bk_jt",
          "bk_l21e", "bk_sk", "bk_sp", "bk_sl", "bk_so", "bk_st", "bkl_lp",
          "bkl_lpl", "bkl_lk", "bkl_tp", "bkl_tgt", "bkl_cp", "bkl_cl",
          "bkl_cu")


@pytest.fixture(scope="module", params=("semenov", "cloud"))
def sched(request):
    """the sparse LU's generation-time tables and constants, read from the
    generated network header (each large network's)"""
    text = (ROOT / "krome_x_b200" / "networks"
            / ("net_%s.h" % request.param)).read_text()
    t = {}
    for name in TABLES:
        m = re.search(r"#define KB_T_%s ([0-9,\-]+)" % name, text)
        t[name] = np.array([int(x) for x in m.group(1).split(",")])
    for k, v in re.findall(r"constexpr int (BK_\w+|NSPEC|NNZ_LU|NNZ_J) = "
                           r"(-?\d+);", text):
        t[k] = int(v)
    return t


def _block_lu(t, A, S):
    """the kernel's factorization (bdf_big.cuh block_lu), phase by phase:
    the sparse rows level by level (each level's rows in reverse order: the
    rows of a level are independent), the dense rows' sparse columns level
    by level of the pivot steps (bkl_*: the level's multipliers, then its
    targets' contributions in order), the dense block in panels of 16.
    Returns 1 / the pivots."""
    rp, ci, di = t["sp_rp"], t["sp_ci"], t["sp_di"]
    m, D, LD, n = t["BK_M"], t["BK_D"], t["BK_LD"], t["NSPEC"]
    rpiv = np.zeros(n)

    def elim(p0, p1):
        for p in range(p0, p1):
            k = ci[p]
            l = A[p] * rpiv[k]
            A[p] = l
            q0, q1 = di[k] + 1, rp[k + 1]
            tg = t["bk_tgt"][t["bk_uoff"][p]:t["bk_uoff"][p] + q1 - q0]
            u = A[q0:q1].copy()
            a = tg >= 0
            A[tg[a]] -= l * u[a]
            S[-1 - tg[~a]] -= l * u[~a]
    flp, frow = t["bk_flp"], t["bk_frow"]
    for L in range(t["BK_NLF"]):
        for i in frow[flp[L]:flp[L + 1]][::-1]:
            elim(rp[i], di[i])
            rpiv[i] = 1.0 / A[di[i]]
    cp = t["bkl_cp"]
    for L in range(t["BK_NSL"]):  # the dense rows' columns, level by level
        e0, e1 = t["bkl_lp"][L], t["bkl_lp"][L + 1]
        pl = t["bkl_lpl"][e0:e1]
        A[pl] = A[pl] * rpiv[t["bkl_lk"][e0:e1]]
        t0, t1 = t["bkl_tp"][L], t["bkl_tp"][L + 1]
        c0, c1 = cp[t0], cp[t1]
        w = A[t["bkl_cl"][c0:c1]] * A[t["bkl_cu"][c0:c1]]
        # each contribution's target, in the targets' order (ufunc.at
        # subtracts repeated targets one after another)
        tg = np.repeat(t["bkl_tgt"][t0:t1], np.diff(cp[t0:t1 + 1]))
        a = tg >= 0
        np.subtract.at(A, tg[a], w[a])
        np.subtract.at(S, -1 - tg[~a], w[~a])
    Sm = S.reshape(D, LD)[:, :D]
    for c0 in range(0, D, 16):
        pe = min(c0 + 16, D)
        for c in range(c0, pe):
            rpiv[m + c] = 1.0 / Sm[c, c]
            Sm[c + 1:, c] *= rpiv[m + c]
            Sm[c + 1:, c + 1:pe] -= np.outer(Sm[c + 1:, c], Sm[c, c + 1:pe])
        if pe == D:
            break
        for r in range(1, pe - c0):
            Sm[c0 + r, pe:] -= Sm[c0 + r, c0:c0 + r] @ Sm[c0:c0 + r, pe:]
        Sm[pe:, pe:] -= Sm[pe:, c0:pe] @ Sm[c0:pe, pe:]
    return rpiv


def _block_solve(t, A, S, rpiv, b):
    """the kernel's solve (bdf_big.cuh block_solve)"""
    rp, ci, di, perm = t["sp_rp"], t["sp_ci"], t["sp_di"], t["sp_perm"]
    m, D, LD, n = t["BK_M"], t["BK_D"], t["BK_LD"], t["NSPEC"]
    x = np.empty(n)
    v = b[perm].copy()
    flp, frow = t["bk_flp"], t["bk_frow"]
    for L in range(1, t["BK_NLF"]):
        for i in frow[flp[L]:flp[L + 1]]:
            v[i] -= A[rp[i]:di[i]] @ v[ci[rp[i]:di[i]]]
    for i in range(m, n):
        e = t["bk_l21e"][i - m]
        v[i] -= A[rp[i]:e] @ v[ci[rp[i]:e]]
    Sm = S.reshape(D, LD)[:, :D]
    w = v[m:]
    for b0 in range(0, D, 32):
        be = min(b0 + 32, D)
        for j in range(b0, be):
            w[j + 1:be] -= Sm[j + 1:be, j] * w[j]
        w[be:] -= Sm[be:, b0:be] @ w[b0:be]
    for be in range(D, 0, -32):
        b0 = max(be - 32, 0)
        for j in range(be - 1, b0 - 1, -1):
            w[j] *= rpiv[m + j]
            w[b0:j] -= Sm[b0:j, j] * w[j]
        w[:b0] -= Sm[:b0, b0:be] @ w[b0:be]
    blp, brow = t["bk_blp"], t["bk_brow"]
    for L in range(t["BK_NLB"]):
        for i in brow[blp[L]:blp[L + 1]]:
            q0, q1 = di[i] + 1, rp[i + 1]
            v[i] = (v[i] - A[q0:q1] @ v[ci[q0:q1]]) * rpiv[i]
    x[perm] = v
    return x


def test_block_schedule_is_consistent(sched):
    """each sparse row eliminates only with rows of lower levels, its
    updates land in its own row, the Jacobian's places agree with the LU
    pattern's"""
    t = sched
    rp, ci, di = t["sp_rp"], t["sp_ci"], t["sp_di"]
    m, D, LD, n = t["BK_M"], t["BK_D"], t["BK_LD"], t["NSPEC"]
    assert m + D == n and LD >= D and D * LD * 8 <= 210 * 1024
    lev = np.full(n, -1)
    for L in range(t["BK_NLF"]):
        lev[t["bk_frow"][t["bk_flp"][L]:t["bk_flp"][L + 1]]] = L
    assert (lev[:m] >= 0).all() and sorted(t["bk_frow"]) == list(range(m))
    for i in range(m):
        ks = ci[rp[i]:di[i]]
        assert (lev[ks] < lev[i]).all()
    blev = np.full(n, -1)
    for L in range(t["BK_NLB"]):
        blev[t["bk_brow"][t["bk_blp"][L]:t["bk_blp"][L + 1]]] = L
    for i in range(m):
        js = ci[di[i] + 1:rp[i + 1]]
        js = js[js < m]
        assert (blev[js] < blev[i]).all()
    row_of = np.repeat(np.arange(n), np.diff(rp))
    for i in range(n):
        for p in range(rp[i], di[i]):
            k = ci[p]
            if k >= m:
                continue
            q0, q1 = di[k] + 1, rp[k + 1]
            tg = t["bk_tgt"][t["bk_uoff"][p]:t["bk_uoff"][p] + q1 - q0]
            for q, g in zip(range(q0, q1), tg):
                j = ci[q]
                if g >= 0:
                    assert row_of[g] == i and ci[g] == j
                else:
                    assert i >= m and j >= m and -1 - g == (i - m) * LD + (j - m)
    # the Schur steps: every dense row's sparse-column L entry once, each
    # pivot's entries after those of lower pivots, rows in order
    sl, sk, sp = t["bk_sl"], t["bk_sk"], t["bk_sp"]
    assert (np.diff(sk) > 0).all() and len(sl) == len(set(sl.tolist()))
    want = [p for i in range(m, n) for p in range(rp[i], t["bk_l21e"][i - m])]
    assert sorted(want) == sorted(sl.tolist())
    for s in range(t["BK_NSCHUR"]):
        ps = sl[sp[s]:sp[s + 1]]
        assert (ci[ps] == sk[s]).all() and (np.diff(row_of[ps]) > 0).all()
    # the Schur levels: every L entry divided once, by its pivot; a level's
    # targets distinct; what a level reads (multipliers, U values) is
    # written by no later level and by no target of its own
    lpl = t["bkl_lpl"]
    assert sorted(lpl.tolist()) == sorted(sl.tolist())
    assert (ci[lpl] == t["bkl_lk"]).all()
    lvl_of = {}
    for L in range(t["BK_NSL"]):
        for pl in lpl[t["bkl_lp"][L]:t["bkl_lp"][L + 1]]:
            lvl_of[int(pl)] = L
    last_write = {}
    for L in range(t["BK_NSL"]):
        tg = t["bkl_tgt"][t["bkl_tp"][L]:t["bkl_tp"][L + 1]]
        assert len(set(tg.tolist())) == len(tg)
        for g in tg[tg >= 0]:
            last_write[int(g)] = L
    for L in range(t["BK_NSL"]):
        t0, t1 = t["bkl_tp"][L], t["bkl_tp"][L + 1]
        c0, c1 = t["bkl_cp"][t0], t["bkl_cp"][t1]
        for pl in t["bkl_cl"][c0:c1]:
            assert lvl_of[int(pl)] <= L and last_write.get(int(pl), -1) < lvl_of[int(pl)]
        for q in t["bkl_cu"][c0:c1]:
            assert row_of[q] < m and int(q) not in last_write
    for q, g in zip(t["sp_jpos"], t["bk_jt"]):
        i, j = row_of[q], ci[q]
        if i < m or j < m:
            assert g == q
        else:
            assert -1 - g == (i - m) * LD + (j - m)


def test_block_schedule_factors_and_solves_the_newton_matrix(sched):
    """the kernel's factorization and solve, restated on the CPU from the
    generated tables, solve I - gamma J (a diagonally dominant J on the
    network's pattern) to 1e-12 of numpy's dense solve"""
    t = sched
    rp, ci, perm = t["sp_rp"], t["sp_ci"], t["sp_perm"]
    m, D, LD, n = t["BK_M"], t["BK_D"], t["BK_LD"], t["NSPEC"]
    rng = np.random.default_rng(5)
    row_of = np.repeat(np.arange(n), np.diff(rp))
    jpos = t["sp_jpos"]
    cnt = np.bincount(row_of[jpos], minlength=n)
    J = rng.uniform(-1.0, 1.0, len(jpos)) / cnt[row_of[jpos]]
    c = -0.9
    M = np.eye(n)
    A = np.zeros(t["NNZ_LU"])
    S = np.zeros(D * LD)
    for e, q in enumerate(jpos):
        M[perm[row_of[q]], perm[ci[q]]] += J[e] * c
        g = t["bk_jt"][e]
        if g >= 0:
            A[g] = J[e] * c
        else:
            S[-1 - g] = J[e] * c
    for i in range(n):
        if i < m:
            A[t["sp_di"][i]] += 1.0
        else:
            S[(i - m) * (LD + 1)] += 1.0
    rpiv = _block_lu(t, A, S)
    assert np.isfinite(rpiv).all()
    for _ in range(3):
        b = rng.standard_normal(n)
        x = _block_solve(t, A, S, rpiv, b)
        ref = np.linalg.solve(M, b)
        np.testing.assert_allclose(x, ref, rtol=0, atol=1e-12 * np.abs(ref).max())


def test_rate_forms_of_the_large_path_equal_the_direct_rates():
    """the generated rate parts (with the H-nuclei density passed in) are the
    generated rates bit for bit; the three-point form of the density-
    dependent rates the kernel evaluates at every rhs matches them to 1e-12
    over states with every ice coverage (bare, partial, saturated)"""
    info = netinfo.load(KEY)
    lib = Oracle(KEY).lib
    D = ctypes.POINTER(ctypes.c_double)
    lib.oracle_rates.argtypes = [ctypes.c_double, D, D, D]
    lib.oracle_rates.restype = None
    lib.oracle_rates_forms.argtypes = [ctypes.c_double, D, D, D, D]
    lib.oracle_rates_forms.restype = ctypes.c_int
    n, T, dt, par = workloads.semenov(12, info, seed=8)
    ice = info["species"].index("H2O_DUST")
    P = info["params"]
    sites = (4 * np.pi * par[:, P.index("xdust")] * par[:, P.index("gsize2")]
             / 9e-16)
    n[:4, ice] = 0.0
    n[4:8, ice] = sites[4:8] * np.linspace(0.1, 0.9, 4)
    n[8:, ice] = sites[8:] * 3.0
    nrea = lib.oracle_nrea()
    worst = 0.0
    for c in range(len(n)):
        row = np.ascontiguousarray(n[c])
        pr = np.ascontiguousarray(par[c])
        kd, kp, ka = np.zeros(nrea), np.zeros(nrea), np.zeros(nrea)
        lib.oracle_rates(T[c], row.ctypes.data_as(D), pr.ctypes.data_as(D),
                         kd.ctypes.data_as(D))
        aff = lib.oracle_rates_forms(T[c], row.ctypes.data_as(D),
                                     pr.ctypes.data_as(D),
                                     kp.ctypes.data_as(D), ka.ctypes.data_as(D))
        assert aff == 1
        np.testing.assert_array_equal(kp, kd)
        big = np.abs(kd) > 1e-300
        worst = max(worst, (np.abs(ka - kd)[big] / np.abs(kd[big])).max())
    assert worst < 1e-12, worst


def _opts(net, **extra):
    o = dict(workloads.OPTIONS[KEY])
    o.update(extra)
    return net.options(**o)


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


EVT = dict(evolve_T=1, jac=1)


def test_oracle_evolved_tgas_matches_reference_fixture_at_noise_level():
    """8 reference-solved cells with Tgas evolved and the hybrid Jacobian
    (the sparse LU bordered by the Tgas row and column): the oracle's
    bordered factorization and solve at the same noise level as the
    fixed-Tgas pin; Tgas (no thermal processes) comes back unchanged"""
    g = golden("semenov_evt")
    opts = dict(workloads.OPTIONS[KEY])
    opts.update(EVT)
    out = Oracle(KEY).solve(g["n"], g["T"], g["dt"], g["par"], **opts)
    assert out["ret"] == g["ret"]
    m = parity_major(out["n"], out["flags"], g["n_out"], g["flags"], g["n"],
                     opts["rtol"])
    assert m["flags_equal"] == 1.0 and m["cells"] == len(g["n"]), m
    assert m["max_rel"] < 1e-4 and m["frac"] >= 0.75, m
    np.testing.assert_array_equal(out["T"], g["T_out"])
    np.testing.assert_array_equal(g["T_out"], g["T"])
    # a different solve from the fixed-Tgas one: the norms run over the
    # Tgas component too, so the step sequence differs
    fixed = Oracle(KEY).solve(g["n"][:2], g["T"][:2], g["dt"][:2],
                              g["par"][:2], **workloads.OPTIONS[KEY])
    assert (fixed["stats"][:, 0] != out["stats"][:2, 0]).any()


def test_oracle_evolved_tgas_edge_rules():
    """evolved Tgas on the large path: Tgas <= 0 fails with -110 and the
    cell untouched; JAC_AUTO's difference quotients are refused (-104)"""
    info = netinfo.load(KEY)
    n, T, dt, par = workloads.semenov(2, info, seed=6)
    T = T.copy()
    T[1] = -5.0
    opts = dict(workloads.OPTIONS[KEY])
    opts.update(EVT)
    out = Oracle(KEY).solve(n[1:], T[1:], dt[1:], par[1:], **opts)
    assert list(out["flags"]) == [-110]
    np.testing.assert_array_equal(out["n"], n[1:])
    opts.update(jac=0)
    out = Oracle(KEY).solve(n[:1], T[:1], dt[:1], par[:1], **opts)
    assert list(out["flags"]) == [-104]


@pytest.mark.gpu
def test_sparse_evolved_tgas_parity():
    """the GPU's bordered solve against the reference fixture and the
    oracle: the large-network metric, flags equal, Tgas returned, the
    oracle's step counts within the chaotic spread, mass conserved; the
    edge rules (-110, -104) as the oracle's"""
    g = golden("semenov_evt")
    opts = dict(workloads.OPTIONS[KEY])
    opts.update(EVT)
    net = krome.load(KEY)
    r = net.solve_batch(g["n"], g["T"], g["dt"], g["par"],
                        opts=net.options(**opts), check=False, stats=True)
    m = parity_major(r.n, r.flags, g["n_out"], g["flags"], g["n"],
                     opts["rtol"])
    assert m["flags_equal"] == 1.0 and m["cells"] == len(g["n"]), m
    assert m["max_rel"] < 2e-4 and m["frac"] >= 0.7, m
    np.testing.assert_array_equal(r.Tgas, g["T_out"])
    ref = Oracle(KEY).solve(g["n"], g["T"], g["dt"], g["par"], **opts)
    m = parity_major(r.n, r.flags, ref["n"], ref["flags"], g["n"],
                     opts["rtol"])
    assert m["max_rel"] < 2e-4 and m["frac"] >= 0.7, m
    a, b = r.stats[:, 0].mean(), ref["stats"][:, 0].mean()
    assert abs(a - b) <= 0.05 * b, (a, b)
    mass = np.asarray(netinfo.load(KEY)["mass_g"])
    np.testing.assert_allclose(r.n @ mass, g["n"] @ mass, rtol=1e-10)
    info = netinfo.load(KEY)
    n, T, dt, par = workloads.semenov(2, info, seed=6)
    T = T.copy()
    T[1] = -5.0
    r = net.solve_batch(n[1:], T[1:], dt[1:], par[1:],
                        opts=net.options(**opts), check=False)
    assert list(r.flags) == [-110]
    np.testing.assert_array_equal(r.n, n[1:])
    opts.update(jac=0)
    r = net.solve_batch(n[:1], T[:1], dt[:1], par[:1],
                        opts=net.options(**opts), check=False)
    assert r.ierr == -104


@pytest.mark.gpu
def test_sparse_unsupported_forms_return_minus_104():
    """the large path runs the FP64 sparse (or auto) LU, Tgas fixed or
    evolved with the analytic Jacobian; the dense LU, the difference-
    quotient Jacobian, the FP32 Newton matrix and the adjoint are the small
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
