"""ctypes access to the CPU oracle and to the reference's own libraries.

Test infrastructure only (the checker): tests/, ``__graft_entry__.smoke()``
and bench.py's CPU-baseline leg use it; the product never does.

* ``Oracle(net)``     the restatement (oracle/_build/liboracle_<net>.so,
                      built on demand from oracle/bdf_oracle.cpp).
* ``Reference(net)``  the reference's generated ``krome_solve_cells``
                      compiled from its own sources (oracle/_ref/, made by
                      oracle/build_ref.py where the reference tree exists);
                      ``strict=True`` the bit-for-bit pin build.
"""
import ctypes
import os
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_L = ctypes.POINTER(ctypes.c_long)
NSTAT = 10
STAT_NAMES = ("nst", "nfe", "nfeDQ", "nje", "nsetups", "nni", "nnf", "netf",
              "restarts", "nlu64")


class _Opts(ctypes.Structure):
    _fields_ = [("evolve_T", ctypes.c_int), ("jac", ctypes.c_int),
                ("rtol", ctypes.c_double), ("atol_n", ctypes.c_double),
                ("atol_T", ctypes.c_double), ("max_steps", ctypes.c_long),
                ("max_err_fails", ctypes.c_int),
                ("max_conv_fails", ctypes.c_int),
                ("max_restarts", ctypes.c_int),
                ("clip_negative", ctypes.c_int), ("lu32", ctypes.c_int),
                ("conserve", ctypes.c_int),
                ("atol_sp", ctypes.POINTER(ctypes.c_double)),
                ("rtol_sp", ctypes.POINTER(ctypes.c_double)),
                ("ph_sigma", ctypes.POINTER(ctypes.c_double)),
                ("ph_phi", ctypes.POINTER(ctypes.c_double)),
                ("ph_B", ctypes.c_int)]


def _ptr(a, t=_D):
    return None if a is None else a.ctypes.data_as(t)


class Oracle:
    def __init__(self, net):
        import sys
        sys.path.insert(0, str(HERE))
        import build as _b  # oracle/build.py
        self.lib = ctypes.CDLL(str(_b.build(net)))
        self.lib.oracle_solve_cells.restype = ctypes.c_int
        self.lib.oracle_solve_cells.argtypes = [
            ctypes.c_int, _D, _D, _D, _D, ctypes.c_int, _I,
            ctypes.POINTER(_Opts), _L, ctypes.c_int]
        self.nspec = self.lib.oracle_nspec()
        self.npar = self.lib.oracle_npar()

    def solve(self, n, T, dt, par, evolve_T=1, jac=0, rtol=1e-6, atol_n=1e-20,
              atol_T=1e-6, max_steps=100000, max_err_fails=7,
              max_conv_fails=10, max_restarts=5, clip_negative=1, lu32=0,
              conserve=0, atol_species=None, rtol_species=None, threads=None,
              photo_sigma=None, Phi=None, **_):
        """photo_sigma [nphoto][nbins] (the bins' averaged cross sections)
        and Phi [ncell][nbins]: each cell's photo rates from its field"""
        n = np.array(n, dtype=float, order="C", copy=True)
        T = np.array(T, dtype=float, order="C", copy=True)
        dt = np.ascontiguousarray(dt, dtype=float)
        par = np.ascontiguousarray(par, dtype=float)
        ncell = n.shape[0]
        stride = 0 if par.ndim == 1 else self.npar
        flags = np.zeros(ncell, dtype=np.intc)
        stats = np.zeros((ncell, NSTAT), dtype=np.int64)
        o = _Opts(int(evolve_T), int(jac), rtol, atol_n, atol_T,
                  int(max_steps), max_err_fails, max_conv_fails,
                  max_restarts, int(clip_negative), int(lu32), int(conserve))
        sp = [None if v is None else np.ascontiguousarray(v, dtype=float)
              for v in (atol_species, rtol_species)]
        o.atol_sp, o.rtol_sp = _ptr(sp[0]), _ptr(sp[1])
        if Phi is not None:
            sig = np.ascontiguousarray(photo_sigma, dtype=float)
            Phi = np.ascontiguousarray(Phi, dtype=float).reshape(ncell, -1)
            o.ph_sigma, o.ph_phi, o.ph_B = _ptr(sig), _ptr(Phi), Phi.shape[1]
        nt = threads or os.cpu_count() or 1
        t0 = time.perf_counter()
        ret = self.lib.oracle_solve_cells(
            ncell, _ptr(n), _ptr(T), _ptr(dt), _ptr(par), stride,
            _ptr(flags, _I), ctypes.byref(o), _ptr(stats, _L), nt)
        self.seconds = time.perf_counter() - t0
        return dict(n=n, T=T, flags=flags, stats=stats, ret=ret)

    def equilibrium(self, n, T, par, t0=100 * 31557600.0,
                    tmax=5e8 * 31557600.0, factor=3.0, ertol=1e-5,
                    eatol=1e-12, evolve_T=0, **opts):
        """integrate every cell to steady state, restating the reference's
        solve_equilibrium (runtime/core/solve_cell.hpp:2249-2301) over this
        oracle's solve: outputs at t0 factor^k, each interval a solve from
        the current state; converged (0) when max_i |dn_i| / max(n_i,
        eatol ntot) (and |dT| / T with evolve_T) between outputs is below
        ertol, 1 at tmax, a failed interval restores the input (its flag).
        The defaults are the reference's handle keys eq_t0 (100 yr),
        eq_tmax (5e8 yr), eq_factor, eq_rtol, eq_atol."""
        n = np.array(n, dtype=float, order="C", copy=True)
        T = np.array(T, dtype=float, order="C", copy=True)
        par = np.ascontiguousarray(par, dtype=float)
        ncell = n.shape[0]
        nin, Tin = n.copy(), T.copy()
        t = np.zeros(ncell)
        dt = np.full(ncell, t0)
        done = np.zeros(ncell, dtype=bool)
        flags = np.zeros(ncell, dtype=np.intc)
        for _ in range(10000):
            act = ~done
            if not act.any():
                break
            prev, Tprev = n.copy(), T.copy()
            d = np.where(act, dt, 0.0)
            out = self.solve(n, T, d, par, evolve_T=evolve_T, **opts)
            fail = act & (out["flags"] != 0)
            n[fail], T[fail] = nin[fail], Tin[fail]
            flags[fail] = out["flags"][fail]
            done |= fail
            ok = act & ~fail
            n[ok], T[ok] = out["n"][ok], out["T"][ok]
            for c in np.nonzero(ok)[0]:  # the reference's scalar order
                t[c] += dt[c]
                tot = 0.0
                for v in n[c]:  # ntot_: the sequential sum
                    tot += v
                floor = eatol * tot
                w = abs(T[c] - Tprev[c]) / T[c] if evolve_T else 0.0
                for i in range(n.shape[1]):
                    w = max(w, abs(n[c, i] - prev[c, i]) / max(n[c, i], floor))
                if w < ertol:
                    done[c] = True
                elif t[c] >= tmax:
                    flags[c] = 1
                    done[c] = True
                else:
                    dt[c] = min((factor - 1.0) * t[c], tmax - t[c])
        return dict(n=n, T=T, flags=flags)

    def adjoint(self, n, T, dt, par, gn, gT, lnm=None, evolve_T=1, jac=0,
                rtol=1e-6, atol_n=1e-20, atol_T=1e-6, max_steps=100000,
                max_err_fails=7, max_conv_fails=10, max_restarts=5,
                clip_negative=1, lu32=0, threads=None, **_):
        """the discrete adjoint (oracle_adjoint_cells): the forward solve
        with rate multipliers exp(lnm) and the gradient of
        sum(gn * n_out) + sum(gT * T_out) w.r.t. n0, T0 and lnm"""
        lib = self.lib
        if not getattr(self, "_adj", False):
            lib.oracle_adjoint_cells.restype = ctypes.c_int
            lib.oracle_adjoint_cells.argtypes = [
                ctypes.c_int, _D, _D, _D, _D, ctypes.c_int, _D, ctypes.c_int,
                _D, _D, _I, ctypes.POINTER(_Opts), _D, _D, _D, _L,
                ctypes.c_int]
            self._adj = True
        n = np.array(n, dtype=float, order="C", copy=True)
        T = np.array(T, dtype=float, order="C", copy=True)
        dt = np.ascontiguousarray(dt, dtype=float)
        par = np.ascontiguousarray(par, dtype=float)
        gn = np.ascontiguousarray(gn, dtype=float)
        gT = np.ascontiguousarray(gT, dtype=float)
        ncell = n.shape[0]
        nrea = lib.oracle_nrea()
        stride = 0 if par.ndim == 1 else self.npar
        lstride = 0
        if lnm is not None:
            lnm = np.ascontiguousarray(lnm, dtype=float)
            lstride = 0 if lnm.ndim == 1 else nrea
        flags = np.zeros(ncell, dtype=np.intc)
        stats = np.zeros((ncell, NSTAT), dtype=np.int64)
        dn0 = np.zeros((ncell, self.nspec))
        dT0 = np.zeros(ncell)
        dm = np.zeros((ncell, nrea))
        o = _Opts(int(evolve_T), int(jac), rtol, atol_n, atol_T,
                  int(max_steps), max_err_fails, max_conv_fails,
                  max_restarts, int(clip_negative), int(lu32))
        nt = threads or os.cpu_count() or 1
        t0 = time.perf_counter()
        ret = lib.oracle_adjoint_cells(
            ncell, _ptr(n), _ptr(T), _ptr(dt), _ptr(par), stride, _ptr(lnm),
            lstride, _ptr(gn), _ptr(gT), _ptr(flags, _I), ctypes.byref(o),
            _ptr(dn0), _ptr(dT0), _ptr(dm), _ptr(stats, _L), nt)
        self.seconds = time.perf_counter() - t0
        return dict(n=n, T=T, flags=flags, stats=stats, ret=ret, dn0=dn0,
                    dT0=dT0, dm=dm)


class Reference:
    """the reference's krome_solve_cells (its generated C ABI)"""

    def __init__(self, net, strict=False):
        name = "libkrome_%s%s.so" % (net, "_strict" if strict else "")
        path = HERE / "_ref" / name
        if not path.exists():
            raise FileNotFoundError(
                "%s missing: run oracle/build_ref.py where the reference "
                "tree is available" % path)
        lib = self.lib = ctypes.CDLL(str(path))
        lib.krome_opts_new.restype = ctypes.c_void_p
        lib.krome_opts_set.argtypes = [ctypes.c_void_p, ctypes.c_char_p,
                                       ctypes.c_double]
        lib.krome_opts_set.restype = ctypes.c_int
        lib.krome_opts_free.argtypes = [ctypes.c_void_p]
        lib.krome_solve_cells.restype = ctypes.c_int
        lib.krome_solve_cells.argtypes = [ctypes.c_int, _D, _D, _D, _D,
                                          ctypes.c_int, ctypes.c_void_p, _I,
                                          ctypes.c_void_p]
        lib.krome_npar.restype = ctypes.c_int
        self.npar = lib.krome_npar()

    def solve(self, n, T, dt, par, **opts):
        n = np.array(n, dtype=float, order="C", copy=True)
        T = np.array(T, dtype=float, order="C", copy=True)
        dt = np.ascontiguousarray(dt, dtype=float)
        par = np.ascontiguousarray(par, dtype=float)
        ncell = n.shape[0]
        stride = 0 if par.ndim == 1 else self.npar
        flags = np.zeros(ncell, dtype=np.intc)
        h = self.lib.krome_opts_new()
        opts = dict(opts)
        opts.setdefault("error_report", 0)
        opts.setdefault("path", 1)
        keep = []
        for q in ("atol", "rtol"):  # per-species tolerances
            v = opts.pop(q + "_species", None)
            if v is not None:
                v = np.ascontiguousarray(v, dtype=float)
                keep.append(v)
                f = getattr(self.lib, "krome_opts_set_%s_species" % q)
                f.argtypes = [ctypes.c_void_p, _D]
                if f(h, _ptr(v)) != 0:
                    raise KeyError(q + "_species")
        # photon bins (Elo, Ehi) and each cell's field Phi[ncell][nbins]
        bins = opts.pop("photo_bins", None)
        Phi = opts.pop("Phi", None)
        cells = None
        if bins is not None:
            lo = np.ascontiguousarray(bins[0], dtype=float)
            hi = np.ascontiguousarray(bins[1], dtype=float)
            keep += [lo, hi]
            self.lib.krome_opts_set_photo.argtypes = [ctypes.c_void_p,
                                                      ctypes.c_int, _D, _D]
            if self.lib.krome_opts_set_photo(h, len(lo), _ptr(lo), _ptr(hi)) != 0:
                raise KeyError("photo_bins")
        if Phi is not None:
            Phi = np.ascontiguousarray(Phi, dtype=float).reshape(ncell, -1)
            keep.append(Phi)
            cells = (_D * 3)(_ptr(Phi), None, None)
        for k, v in opts.items():
            if k in ("threads",):
                continue
            if self.lib.krome_opts_set(h, k.encode(), float(v)) != 0:
                raise KeyError(k)
        t0 = time.perf_counter()
        ret = self.lib.krome_solve_cells(ncell, _ptr(n), _ptr(T), _ptr(dt),
                                         _ptr(par), stride,
                                         None if cells is None else ctypes.addressof(cells),
                                         _ptr(flags, _I), h)
        self.seconds = time.perf_counter() - t0
        self.lib.krome_opts_free(h)
        return dict(n=n, T=T, flags=flags, ret=ret)


    def equilibrium(self, n, T, par, **opts):
        """the reference's krome_equilibrium_cells (krome.h:366-376)"""
        n = np.array(n, dtype=float, order="C", copy=True)
        T = np.array(T, dtype=float, order="C", copy=True)
        par = np.ascontiguousarray(par, dtype=float)
        ncell = n.shape[0]
        flags = np.zeros(ncell, dtype=np.intc)
        h = self.lib.krome_opts_new()
        opts = dict(opts)
        opts.setdefault("error_report", 0)
        for k, v in opts.items():
            if self.lib.krome_opts_set(h, k.encode(), float(v)) != 0:
                raise KeyError(k)
        f = self.lib.krome_equilibrium_cells
        f.restype = ctypes.c_int
        f.argtypes = [ctypes.c_int, _D, _D, _D, ctypes.c_int, ctypes.c_void_p,
                      _I, ctypes.c_void_p]
        ret = f(ncell, _ptr(n), _ptr(T), _ptr(par),
                0 if par.ndim == 1 else self.npar, None, _ptr(flags, _I), h)
        self.lib.krome_opts_free(h)
        return dict(n=n, T=T, flags=flags, ret=ret)


def _ref_worker(args):
    net, strict, n, T, dt, par, opts = args
    out = Reference(net, strict=strict).solve(n, T, dt, par, **opts)
    return out


def _ref_eq_worker(args):
    net, strict, n, T, par, opts = args
    return Reference(net, strict=strict).equilibrium(n, T, par, **opts)


def reference_equilibrium(net, n, T, par, strict=False, **opts):
    """Reference(net).equilibrium in a spawned child process"""
    import multiprocessing as mp
    with mp.get_context("spawn").Pool(1) as pool:
        return pool.map(_ref_eq_worker, [(net, strict, n, T, par, opts)])[0]


def reference_solve(net, n, T, dt, par, strict=False, **opts):
    """Reference(net).solve in a spawned child process: the reference's
    generated tables are function-local statics, which GCC emits as
    process-wide unique symbols, so two networks' libraries must never share
    a process"""
    import multiprocessing as mp
    with mp.get_context("spawn").Pool(1) as pool:
        return pool.map(_ref_worker, [(net, strict, n, T, dt, par, opts)])[0]
