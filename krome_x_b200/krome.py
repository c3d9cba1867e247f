"""Python binding of libkrome_b200_<net>.so (ctypes), mirroring the
reference's generated binding (runtime/interfaces/python/krome.py): the
same ``Network`` / ``Options`` / ``Result`` / ``KromeError`` names, the same
``solve(n, Tgas, dt, par, opts)`` semantics (new arrays returned, inputs
never modified, a REQUIRED parameter left unset raises before the call,
``check=True`` raises on a failed cell), plus ``solve_batch`` (strict
shapes: ``n[N, nspec]``, ``Tgas[N]``, ``dt[N]``, ``par`` one row or
``[N, npar]``) and ``solve_device`` for arrays already in GPU memory
(torch CUDA tensors or raw device pointers).

    from krome_x_b200 import krome
    net = krome.load("primordial")
    opts = net.options(evolve_T=True, rtol=1e-6, jac="analytic")
    res = net.solve_batch(n, Tgas, dt, par, opts=opts)

There is no CPU fallback: the library computes on the GPU or fails.
"""
import ctypes
from pathlib import Path

import numpy as np

from . import netinfo

__all__ = ["load", "Network", "Options", "Result", "KromeError"]

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_L = ctypes.POINTER(ctypes.c_long)
_ENUMS = {"jac": ("auto", "analytic", "fd"),
          "linsol": ("auto", "dense", "lapack", "sparse"),
          "path": ("auto", "percell", "device"),
          "kernel": ("plain", "persistent")}
STAT_NAMES = ("nst", "nfe", "nfeDQ", "nje", "nsetups", "nni", "nnf", "netf",
              "restarts", "nlu64")
LIBDIR = Path(__file__).resolve().parent / "lib"


class KromeError(RuntimeError):
    """a rejected argument or option, or a failed solve."""


def load(network):
    """the Network of a generated network key (e.g. "primordial") or of a
    library path"""
    return Network(network)


def _dptr(a):
    return None if a is None else a.ctypes.data_as(_D)


class Result:
    """solve() output: new arrays n, Tgas, the per-cell flags, the returned
    flag ierr and (solve_batch with stats=True) per-cell counters"""

    def __init__(self, n, Tgas, flags, ierr, stats=None):
        self.n, self.Tgas, self.flags, self.ierr = n, Tgas, flags, ierr
        self.stats = stats

    def __repr__(self):
        return "<krome_b200 Result ierr=%d>" % self.ierr


class Options:
    """an options handle (krome_opts), set by key as in the reference"""

    def __init__(self, net, **values):
        self._net = net
        self._lib = net._lib
        self._h = ctypes.c_void_p(self._lib.krome_opts_new())
        for k, v in values.items():
            self[k] = v

    def __setitem__(self, key, value):
        if key in _ENUMS and isinstance(value, str):
            value = _ENUMS[key].index(value)
        if isinstance(value, bool):
            value = int(value)
        if self._lib.krome_opts_set(self._h, key.encode(), float(value)) != 0:
            raise KromeError("bad option %s = %r" % (key, value))

    def __getitem__(self, key):
        v = ctypes.c_double()
        if self._lib.krome_opts_get(self._h, key.encode(), ctypes.byref(v)) != 0:
            raise KromeError("unknown option %s" % key)
        return v.value

    def set(self, **values):
        for k, v in values.items():
            self[k] = v
        return self

    # -- photon bins (reference runtime/interfaces/python/krome.py:1337-1400)
    def set_photo(self, Elo, Ehi):
        """photon bins [eV edges]; a solve then needs each cell's field
        Phi[ncell, nbins] (photons cm^-2 s^-1 per bin)"""
        lo = np.ascontiguousarray(Elo, dtype=float)
        hi = np.ascontiguousarray(Ehi, dtype=float)
        if lo.shape != hi.shape or lo.ndim != 1:
            raise KromeError("Elo and Ehi must be 1-D arrays of one shape")
        if self._lib.krome_opts_set_photo(self._h, lo.size, _dptr(lo),
                                          _dptr(hi)) != 0:
            raise KromeError("invalid photon bins (need 0 < Elo < Ehi)")
        return self

    def set_photo_alpha(self, alpha):
        """the in-bin photon spectrum dN/dE ~ E^-alpha"""
        if self._lib.krome_opts_set_photo_alpha(self._h, float(alpha)) != 0:
            raise KromeError("alpha must be finite")
        return self

    def set_photo_broadening(self, Tgas, vturb=0.0):
        """Doppler broadening of the tabulated cross sections"""
        if self._lib.krome_opts_set_photo_broadening(
                self._h, float(Tgas), float(vturb)) != 0:
            raise KromeError("broadening needs Tgas >= 0 and vturb >= 0")
        return self

    @property
    def nbins(self):
        return self._lib.krome_opts_nbins(self._h)

    def photo_sigma(self):
        """the bin-averaged cross sections [nphoto, nbins] [cm^2]"""
        out = np.zeros((self._lib.krome_nphoto(), self.nbins))
        if out.size and self._lib.krome_opts_photo_sigma(self._h,
                                                          _dptr(out)) != 0:
            raise KromeError("photon bins not configured")
        return out

    def __del__(self):
        try:
            self._lib.krome_opts_free(self._h)
        except Exception:
            pass


class Network:
    """one generated network, compiled into libkrome_b200_<net>.so"""

    def __init__(self, network):
        p = Path(network)
        if p.suffix == ".so":
            path = p
            key = p.stem[len("libkrome_b200_"):]
        else:
            key = str(network)
            path = LIBDIR / ("libkrome_b200_%s.so" % key)
        if not path.exists():
            raise KromeError("library %s not found: build it with "
                             "python -m krome_x_b200.build %s" % (path, key))
        self.key = key
        self.path = path
        lib = self._lib = ctypes.CDLL(str(path))
        proto = {
            "krome_network_name": (ctypes.c_char_p, []),
            "krome_version": (ctypes.c_char_p, []),
            "krome_nspec": (ctypes.c_int, []),
            "krome_nrea": (ctypes.c_int, []),
            "krome_npar": (ctypes.c_int, []),
            "krome_species_name": (ctypes.c_char_p, [ctypes.c_int]),
            "krome_species_index": (ctypes.c_int, [ctypes.c_char_p]),
            "krome_param_name": (ctypes.c_char_p, [ctypes.c_int]),
            "krome_param_index": (ctypes.c_int, [ctypes.c_char_p]),
            "krome_param_required_by": (ctypes.c_char_p, [ctypes.c_int]),
            "krome_params_default": (None, [_D]),
            "krome_flag_message": (ctypes.c_char_p, [ctypes.c_int]),
            "krome_opts_new": (ctypes.c_void_p, []),
            "krome_opts_free": (None, [ctypes.c_void_p]),
            "krome_opts_set": (ctypes.c_int, [ctypes.c_void_p,
                                              ctypes.c_char_p,
                                              ctypes.c_double]),
            "krome_opts_get": (ctypes.c_int, [ctypes.c_void_p,
                                              ctypes.c_char_p, _D]),
            "krome_solve_cells": (ctypes.c_int, [
                ctypes.c_int, _D, _D, _D, _D, ctypes.c_int, ctypes.c_void_p,
                _I, ctypes.c_void_p]),
            "krome_solve_cells_x": (ctypes.c_int, [
                ctypes.c_int, _D, _D, _D, _D, _D, ctypes.c_int,
                ctypes.c_void_p, _I, ctypes.c_void_p]),
            "krome_b200_solve_batch": (ctypes.c_int, [
                ctypes.c_int, _D, _D, _D, _D, ctypes.c_int, _I, _L,
                ctypes.c_void_p]),
            "krome_b200_solve_device": (ctypes.c_int, [
                ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                ctypes.c_void_p, ctypes.c_void_p]),
            "krome_has_device": (ctypes.c_int, []),
            "krome_b200_nstat": (ctypes.c_int, []),
            "krome_get_rates": (ctypes.c_int, [
                ctypes.c_int, _D, _D, _D, ctypes.c_int, _D, ctypes.c_void_p,
                _D]),
            "krome_b200_hydro_step": (ctypes.c_int, [
                ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                ctypes.c_void_p]),
            "krome_b200_graph_new": (ctypes.c_void_p, [
                ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                ctypes.c_void_p]),
            "krome_b200_graph_launch": (ctypes.c_int, [ctypes.c_void_p,
                                                       ctypes.c_void_p]),
            "krome_b200_graph_free": (None, [ctypes.c_void_p]),
            "krome_b200_fp64_peak": (ctypes.c_int, [_D]),
            "krome_b200_adjoint": (ctypes.c_int, [
                ctypes.c_int, _D, _D, _D, _D, ctypes.c_int, _D, ctypes.c_int,
                _D, _D, _I, _D, _D, _D, ctypes.c_long, ctypes.c_void_p]),
            "krome_b200_adjoint_record_device": (ctypes.c_int, [
                ctypes.c_int] + [ctypes.c_void_p] * 4 + [ctypes.c_int,
                ctypes.c_void_p, ctypes.c_int] + [ctypes.c_void_p] * 4
                + [ctypes.c_long] + [ctypes.c_void_p] * 4),
            "krome_b200_adjoint_device": (ctypes.c_int, [
                ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                ctypes.c_void_p, ctypes.c_int] + [ctypes.c_void_p] * 4
                + [ctypes.c_long] + [ctypes.c_void_p] * 8),
        }
        proto.update({
            "krome_opts_set_photo": (ctypes.c_int, [ctypes.c_void_p,
                                                    ctypes.c_int, _D, _D]),
            "krome_opts_set_photo_alpha": (ctypes.c_int, [ctypes.c_void_p,
                                                          ctypes.c_double]),
            "krome_opts_set_photo_broadening": (
                ctypes.c_int, [ctypes.c_void_p, ctypes.c_double,
                               ctypes.c_double]),
            "krome_opts_nbins": (ctypes.c_int, [ctypes.c_void_p]),
            "krome_opts_photo_sigma": (ctypes.c_int, [ctypes.c_void_p, _D]),
            "krome_nphoto": (ctypes.c_int, []),
            "krome_bins_log": (ctypes.c_int, [ctypes.c_int, ctypes.c_double,
                                              ctypes.c_double, _D, _D]),
            "krome_spectrum_draine": (ctypes.c_int, [ctypes.c_int, _D, _D,
                                                     _D]),
            "krome_spectrum_j21": (ctypes.c_int, [ctypes.c_int, _D, _D,
                                                  ctypes.c_double,
                                                  ctypes.c_double, _D]),
        })
        for name, (res, args) in proto.items():
            fn = getattr(lib, name)
            fn.restype, fn.argtypes = res, args
        self.name = lib.krome_network_name().decode()
        self.version = lib.krome_version().decode()
        self.nspec = lib.krome_nspec()
        self.nrea = lib.krome_nrea()
        self.npar = lib.krome_npar()
        self.species = tuple(lib.krome_species_name(i).decode()
                             for i in range(self.nspec))
        self.params = tuple(lib.krome_param_name(i).decode()
                            for i in range(self.npar))
        self.required = {s: lib.krome_param_required_by(i).decode()
                         for i, s in enumerate(self.params)
                         if lib.krome_param_required_by(i).decode()}
        self._pidx = {s: i for i, s in enumerate(self.params)}
        self.info = netinfo.load(key) if (netinfo.NETDIR / (
            "net_%s.json" % key)).exists() else None
        self._opts = None

    def __repr__(self):
        return "<krome_b200 Network %s: %d species, %d reactions>" % (
            self.name, self.nspec, self.nrea)

    # -- description ------------------------------------------------------

    def idx(self, name):
        i = self._lib.krome_species_index(name.encode())
        if i < 0:
            raise KromeError("unknown species %r" % name)
        return i

    def params_default(self):
        row = np.zeros(self.npar)
        self._lib.krome_params_default(_dptr(row))
        return row

    def param_rows(self, ncell, **values):
        rows = np.repeat(self.params_default()[None, :], ncell, axis=0)
        for k, v in values.items():
            if k not in self._pidx:
                raise KromeError("unknown parameter %r" % k)
            rows[:, self._pidx[k]] = np.broadcast_to(np.asarray(v, float),
                                                     (ncell,))
        return rows

    def flag_message(self, flag):
        return self._lib.krome_flag_message(int(flag)).decode()

    def options(self, **values):
        return Options(self, **values)

    @property
    def has_device(self):
        return bool(self._lib.krome_has_device())

    # -- solves -------------------------------------------------------------

    def _options(self, opts):
        if opts is not None:
            return opts
        if self._opts is None:
            self._opts = Options(self)
        return self._opts

    def _params(self, par, ncell):
        stride, P = 0, None
        if isinstance(par, dict):
            P = self.param_rows(ncell, **par)
            stride = self.npar
        elif par is not None:
            P = np.ascontiguousarray(par, dtype=float)
            if P.shape == (self.npar,):
                stride = 0
            elif P.shape == (ncell, self.npar):
                stride = self.npar
            else:
                raise KromeError("par must have shape (%d,) or (%d, %d), got "
                                 "%s" % (self.npar, ncell, self.npar, P.shape))
        rows = (self.params_default()[None, :] if P is None
                else P.reshape(-1, self.npar))
        unset = [s for s in self.required
                 if np.isnan(rows[:, self._pidx[s]]).any()]
        if unset:
            raise KromeError("required parameter(s) not set: %s" % "; ".join(
                "%s (for %s)" % (s, self.required[s]) for s in unset))
        return P, stride

    def _run(self, n, T, dtv, P, stride, opts, check, stats, Phi=None):
        ncell = n.shape[0]
        flags = np.zeros(ncell, dtype=np.intc)
        st = np.zeros((ncell, len(STAT_NAMES)), dtype=np.int64) if stats else None
        if Phi is not None:  # the field rows: krome_solve_cells' extra
            if stats:
                raise KromeError("per-cell counters are not returned with a "
                                 "photon field")
            F = np.array(np.broadcast_to(np.asarray(Phi, dtype=float),
                                         (ncell, opts.nbins)), order="C",
                         copy=True)
            cells = (_D * 3)(_dptr(F), None, None)
            ierr = self._lib.krome_solve_cells(
                ncell, _dptr(n), _dptr(T), _dptr(dtv), _dptr(P), stride,
                ctypes.addressof(cells), flags.ctypes.data_as(_I), opts._h)
        else:
            ierr = self._lib.krome_b200_solve_batch(
                ncell, _dptr(n), _dptr(T), _dptr(dtv), _dptr(P), stride,
                flags.ctypes.data_as(_I),
                None if st is None else st.ctypes.data_as(_L), opts._h)
        if check and ierr != 0:
            bad = np.flatnonzero(flags)
            raise KromeError("krome_solve_cells returned %d: %s (failed cells: "
                             "%s); pass check=False to get the result anyway"
                             % (ierr, self.flag_message(ierr),
                                bad[:20].tolist() or "n/a"))
        return flags, ierr, st

    def solve(self, n, Tgas, dt, par=None, opts=None, check=True,
              stats=False, Phi=None):
        """integrate every cell over its own dt [s] (reference
        runtime/interfaces/python/krome.py:458-507): n[nspec] or
        n[ncell, nspec], Tgas and dt scalars or per cell, par None / a dict
        / one row / rows; Phi the photon field per bin (one row for every
        cell or [ncell, nbins]) with photon bins on opts. Returns a Result
        with new arrays."""
        n = np.array(n, dtype=float, order="C", copy=True)
        if n.ndim == 0 or n.ndim > 2 or n.shape[-1] != self.nspec:
            raise KromeError("n must have shape (%d,) or (ncell, %d), got %s"
                             % (self.nspec, self.nspec, n.shape))
        single = n.ndim == 1
        n = n.reshape(-1, self.nspec)
        ncell = n.shape[0]
        T = np.array(np.broadcast_to(np.asarray(Tgas, dtype=float), (ncell,)),
                     order="C", copy=True)
        dtv = np.array(np.broadcast_to(np.asarray(dt, dtype=float), (ncell,)),
                       order="C", copy=True)
        opts = self._options(opts)
        P, stride = self._params(par, ncell)
        if opts.nbins > 0 and Phi is None:
            raise KromeError("photon bins are configured (set_photo): Phi "
                             "is required")
        flags, ierr, st = self._run(n, T, dtv, P, stride, opts, check, stats,
                                    Phi if opts.nbins > 0 else None)
        if single:
            return Result(n[0], T[0], flags[0], ierr,
                          None if st is None else st[0])
        return Result(n, T, flags, ierr, st)

    def solve_x(self, x, rho, Tgas, dt, par=None, opts=None, check=True):
        """solve() with mass fractions (reference runtime/interfaces/python/
        krome.py:509-542): x[nspec] or x[ncell, nspec] and the gas density
        rho [g cm^-3], scalar or per cell; n = rho x / m on the way in,
        x = m n / rho on the way out (renormalize_x rescales to the input
        sum) for the cells that succeed. Returns a Result whose n holds the
        new mass fractions."""
        x = np.array(x, dtype=float, order="C", copy=True)
        if x.ndim == 0 or x.ndim > 2 or x.shape[-1] != self.nspec:
            raise KromeError("x must have shape (%d,) or (ncell, %d), got %s"
                             % (self.nspec, self.nspec, x.shape))
        single = x.ndim == 1
        x = x.reshape(-1, self.nspec)
        ncell = x.shape[0]
        cell = lambda v: np.array(np.broadcast_to(np.asarray(v, dtype=float),
                                                  (ncell,)), order="C", copy=True)
        rh, T, dtv = cell(rho), cell(Tgas), cell(dt)
        opts = self._options(opts)
        P, stride = self._params(par, ncell)
        flags = np.zeros(ncell, dtype=np.intc)
        ierr = self._lib.krome_solve_cells_x(
            ncell, _dptr(x), _dptr(rh), _dptr(T), _dptr(dtv), _dptr(P), stride,
            None, flags.ctypes.data_as(_I), opts._h)
        if check and ierr != 0:
            bad = np.flatnonzero(flags)
            raise KromeError("krome_solve_cells_x returned %d: %s (failed "
                             "cells: %s); pass check=False to get the result "
                             "anyway" % (ierr, self.flag_message(ierr),
                                         bad[:20].tolist() or "n/a"))
        if single:
            return Result(x[0], T[0], flags[0], ierr)
        return Result(x, T, flags, ierr)

    def solve_batch(self, n, Tgas, dt, par=None, opts=None, check=True,
                    stats=False, Phi=None):
        """the batched entry point: n[N, nspec], Tgas[N], dt[N] exactly
        (no scalar broadcast), par None / dict / one row / [N, npar]"""
        n = np.asarray(n, dtype=float)
        if n.ndim != 2 or n.shape[1] != self.nspec:
            raise KromeError("solve_batch: n must be (N, %d), got %s"
                             % (self.nspec, n.shape))
        N = n.shape[0]
        for name, v in (("Tgas", Tgas), ("dt", dt)):
            if np.shape(v) != (N,):
                raise KromeError("solve_batch: %s must be (%d,), got %s"
                                 % (name, N, np.shape(v)))
        return self.solve(n, Tgas, dt, par=par, opts=opts, check=check,
                          stats=stats, Phi=Phi)

    def adjoint(self, n, Tgas, dt, par=None, gn=None, gT=None, lnm=None,
                opts=None, tape_cap=0, check=True):
        """the discrete adjoint of the batched solve (krome_b200_adjoint):
        the solve of n[N, nspec], Tgas[N], dt[N] with every rate
        coefficient multiplied by exp(lnm) (lnm None, one row [nrea] or
        [N, nrea]), and the gradient of sum(gn * n_out) + sum(gT * T_out)
        with respect to the initial n (dn0), Tgas (dT0) and lnm (dm, per
        cell). tape_cap: doubles of tape per cell (0: the default 32768).
        Returns a Result with dn0, dT0, dm attached."""
        n = np.array(n, dtype=float, order="C", copy=True)
        if n.ndim != 2 or n.shape[1] != self.nspec:
            raise KromeError("adjoint: n must be (N, %d), got %s"
                             % (self.nspec, n.shape))
        N = n.shape[0]
        T = np.array(Tgas, dtype=float, order="C", copy=True).reshape(N)
        dtv = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, float), (N,)))
        opts = self._options(opts)
        P, stride = self._params(par, N)
        gn = np.ascontiguousarray(np.zeros_like(n) if gn is None else gn,
                                  dtype=float).reshape(N, self.nspec)
        gT = np.ascontiguousarray(np.zeros(N) if gT is None else gT,
                                  dtype=float).reshape(N)
        lstride = 0
        if lnm is not None:
            lnm = np.ascontiguousarray(lnm, dtype=float)
            lstride = 0 if lnm.ndim == 1 else self.nrea
        flags = np.zeros(N, dtype=np.intc)
        dn0 = np.zeros((N, self.nspec))
        dT0 = np.zeros(N)
        dm = np.zeros((N, self.nrea))
        ierr = self._lib.krome_b200_adjoint(
            N, _dptr(n), _dptr(T), _dptr(dtv), _dptr(P), stride,
            None if lnm is None else _dptr(lnm), lstride, _dptr(gn),
            _dptr(gT), flags.ctypes.data_as(_I), _dptr(dn0), _dptr(dT0),
            _dptr(dm), int(tape_cap), opts._h)
        if check and ierr != 0:
            raise KromeError("krome_b200_adjoint returned %d: %s"
                             % (ierr, self.flag_message(ierr)))
        r = Result(n, T, flags, ierr)
        r.dn0, r.dT0, r.dm = dn0, dT0, dm
        return r

    def _check_stats(self, stats, N):
        """a device stats array must hold N rows of the library's counters:
        the kernels write nstat of them per cell"""
        if stats is None or isinstance(stats, int):
            return
        nst = self._lib.krome_b200_nstat()
        if tuple(stats.shape) != (N, nst) or stats.dtype.itemsize != 8:
            raise KromeError("stats must be int64 [%d, %d], got %s %s"
                             % (N, nst, tuple(stats.shape), stats.dtype))

    def solve_device(self, n, Tgas, dt, par, flags, opts=None, stats=None,
                     cursor=None, stream=0):
        """device-resident solve: every argument a CUDA array (torch tensor
        or an int device pointer): n[N, nspec] and Tgas[N] updated in place,
        dt[N], par one row or [N, npar], flags[N] int32; cursor one uint32
        (the work queue of the persistent kernel); asynchronous on stream"""
        def ptr(x):
            if x is None:
                return None
            return x if isinstance(x, int) else x.data_ptr()
        N = int(n.shape[0])
        npar_el = int(par.numel()) if hasattr(par, "numel") else self.npar
        stride = 0 if npar_el == self.npar else self.npar
        self._check_stats(stats, N)
        opts = self._options(opts)
        r = self._lib.krome_b200_solve_device(
            N, ptr(n), ptr(Tgas), ptr(dt), ptr(par), stride, ptr(flags),
            ptr(stats), ptr(cursor), opts._h, ctypes.c_void_p(stream))
        if r != 0:
            raise KromeError("krome_b200_solve_device returned %d: %s"
                             % (r, self.flag_message(r)))
        return r

    def rates(self, n, Tgas, par=None, Phi=None, opts=None):
        """the rate coefficients k[ncell, nrea] at each cell's rate
        temperature (krome_get_rates, computed on the GPU), with the photo
        rates of the field Phi on opts' photon bins"""
        n = np.ascontiguousarray(np.atleast_2d(n), dtype=float)
        ncell = n.shape[0]
        T = np.ascontiguousarray(np.broadcast_to(np.asarray(Tgas, float),
                                                 (ncell,)))
        P, stride = self._params(par, ncell)
        k = np.zeros((ncell, self.nrea))
        F = None
        if Phi is not None:
            F = np.array(np.broadcast_to(np.asarray(Phi, dtype=float),
                                         (ncell, opts.nbins)), order="C")
        r = self._lib.krome_get_rates(ncell, _dptr(n), _dptr(T), _dptr(P),
                                      stride, _dptr(F),
                                      None if opts is None else opts._h,
                                      _dptr(k))
        if r != 0:
            raise KromeError("krome_get_rates returned %d" % r)
        return k

    def bins_log(self, nbins, lower, upper):
        """(Elo, Ehi) of nbins logarithmic bins in [lower, upper] eV"""
        lo, hi = np.zeros(nbins), np.zeros(nbins)
        if self._lib.krome_bins_log(nbins, lower, upper, _dptr(lo), _dptr(hi)) != 0:
            raise KromeError("invalid binning")
        return lo, hi

    def spectrum_draine(self, Elo, Ehi):
        """the Draine (1978) interstellar field per bin [photons cm^-2 s^-1]"""
        lo, hi = np.ascontiguousarray(Elo, float), np.ascontiguousarray(Ehi, float)
        out = np.zeros(lo.size)
        if self._lib.krome_spectrum_draine(lo.size, _dptr(lo), _dptr(hi), _dptr(out)) != 0:
            raise KromeError("invalid bins")
        return out

    def spectrum_j21(self, Elo, Ehi, J21=1.0, alpha=1.0):
        """a J21 power-law field per bin [photons cm^-2 s^-1]"""
        lo, hi = np.ascontiguousarray(Elo, float), np.ascontiguousarray(Ehi, float)
        out = np.zeros(lo.size)
        if self._lib.krome_spectrum_j21(lo.size, _dptr(lo), _dptr(hi), J21,
                                        alpha, _dptr(out)) != 0:
            raise KromeError("invalid bins")
        return out

    def fp64_peak(self):
        """the measured FP64 peak of the GPU [TFLOP/s]"""
        v = ctypes.c_double()
        if self._lib.krome_b200_fp64_peak(ctypes.byref(v)) != 0:
            raise KromeError("no GPU for the FP64 peak measurement")
        return v.value

    def hydro_graph(self, n, Tgas, dt, par, flags, opts, stats=None,
                    cursor=None, factor=1.01, dtfrac=0.01, stream=None):
        """a HydroGraph: one collapse-driver step (tff, densities x factor,
        dt = dtfrac tff, then the solve) captured as a CUDA graph on the
        device arrays (torch CUDA tensors), replayed by .launch()"""
        return HydroGraph(self, n, Tgas, dt, par, flags, opts, stats, cursor,
                          factor, dtfrac, stream)


class HydroGraph:
    """the captured hydro step (krome_b200_graph_new / _launch / _free)"""

    def __init__(self, net, n, Tgas, dt, par, flags, opts, stats, cursor,
                 factor, dtfrac, stream):
        import torch
        self.net = net
        self.stream = stream or torch.cuda.Stream()
        self.cursor = cursor if cursor is not None else torch.zeros(
            1, dtype=torch.int32, device=n.device)
        net._check_stats(stats, int(n.shape[0]))
        self._keep = (n, Tgas, dt, par, flags, stats, opts)
        ptr = lambda x: None if x is None else x.data_ptr()
        self._h = net._lib.krome_b200_graph_new(
            int(n.shape[0]), ptr(n), ptr(Tgas), ptr(dt), ptr(par),
            net.npar, net.params.index("tff"), factor, dtfrac, ptr(flags),
            ptr(stats), ptr(self.cursor), opts._h,
            ctypes.c_void_p(self.stream.cuda_stream))
        if not self._h:
            raise KromeError("CUDA graph capture of the hydro step failed")

    def launch(self):
        r = self.net._lib.krome_b200_graph_launch(
            ctypes.c_void_p(self._h), ctypes.c_void_p(self.stream.cuda_stream))
        if r != 0:
            raise KromeError("graph launch failed (%d)" % r)

    def free(self):
        if self._h:
            self.net._lib.krome_b200_graph_free(ctypes.c_void_p(self._h))
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
