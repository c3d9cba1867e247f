"""Seeded synthetic batches of the benchmark workloads.

No dataset is involved: every batch is drawn with ``numpy.random.
default_rng(seed)`` from the distributions the benchmark names, laid out as
``krome_solve_cells`` takes them (``n[ncell, nspec]`` cell-major, species in
the network's code-point order, ``Tgas[ncell]``, ``dt[ncell]``,
``par[ncell, npar]``).

* ``primordial``   (configs 0 and 2) n_H log-uniform in [1, 1e6] cm^-3,
  Tgas log-uniform in [10, 1e4] K, H : H+ : e- : He = 1e4 : 1 : 1 : 775 with
  H = n_H, every other species 1e-20 n_H; dt = 3.15e10 s; tff the free-fall
  time of the cell (reference runtime/core/query.hpp:176-182).
* ``primordial3``  (config 1) n_H log-uniform in [1, 1e14], Tgas in
  [50, 5000] K, x_H2 in [1e-6, 0.5], x_e = x_H+ in [1e-8, 1e-2] (all
  log-uniform), He/H = 0.0775, H = n_H - 2 n_H2 - n_H+; trace species
  1e-20 n_H. The hydro loop: per call tff = t_ff(n), every density x 1.01,
  dt = 0.01 tff (the reference's collapse driver,
  examples/tests/collapse/test.cpp:47-63).
* ``semenov``      (config 3) n_H log-uniform in [1e2, 1e7], Tgas in
  [10, 300] K (fixed); the initial abundances of the reference's
  cloudSurface test (Semenov 2010: He 0.09, H2 0.5, C+ 1.2e-4, N 7.6e-5,
  O 2.56e-4, S+ 8e-8, Si+ 8e-9, Fe+ 3e-9, Na+ 2e-9, Mg+ 7e-9, P+ 2e-10,
  Cl+ 1e-9, times n_H) each x log-uniform [0.5, 2], every other species
  1e-20 n_H, electrons for neutrality; that test's parameters (Av 10,
  crflux 1.3e-17, grains of 0.1 micron: gsize 1e-5, gsize2 1e-10, xdust =
  0.01 rho / (4/3 pi 3 a^3 1.43) grains per cm^3, also GRAIN0's density,
  Tdust = Tgas); dt = 3.15e13 s (examples/tests/cloudSurface/test.cpp).
* ``cloud``        the reference's gas-phase dark-cloud network (452
  species), a second network on the sparse path: Semenov's n_H, Tgas and
  initial abundances (the species both networks have), every other species
  1e-20 n_H, electrons for neutrality, grains GRAIN0 = 1.3e-12 n_H; Av 10,
  crate 1.3e-17, gas_dust_ratio 1; dt = 3.15e13 s.
* ``galaxy_ism``   (config 4) n_H log-uniform in [1e-2, 1e4], Tgas in
  [10, 1e6] K, crate in [1e-17, 1e-16], G0 in [0.3, 3], d2g in
  [0.003, 0.03] (log-uniform, one decade around the typical values);
  H2 1e-6 n_H, H+ = e- = 1e-4 n_H, He 0.0775 n_H; dt = 3.15e11 s.
* ``primordialZ``  (a further network, default thermal options, fixed
  Tgas) n_H log-uniform in [1, 1e6], Tgas in [30, 3000] K, x_H2 in
  [1e-6, 0.5], x_H+ in [1e-6, 1e-3], metallicity Z in [1e-3, 1] (all
  log-uniform): C+ 1.4e-4 Z n_H, O 3.2e-4 Z n_H, He 0.0775 n_H, H = n_H -
  2 n_H2 - n_H+ (floored at the trace level), electrons for neutrality,
  trace species 1e-20 n_H; dt = 3.15e11 s; the difference-quotient
  Jacobian (its rates depend on the densities).
* ``earlyUniverse`` (a further network, default thermal options, fixed
  Tgas) the reference's early-universe driver's cosmology
  (examples/tests/earlyUniverse/test.cpp: h = 0.704, Omega0 = 1,
  Omega_b = 0.0456, Tcmb0 = 2.73 K) at redshift z log-uniform in
  [20, 2000]: n = 0.0456 x 9.19e-6 (1+z)^3 cm^-3, Tgas = Trad = 2.73 (1+z),
  ionized fraction x log-uniform in [1e-4, 1] for H and D (D/H = 4.3e-5 /
  0.924), He neutral (He+ 1e-6 of He), electrons for neutrality, trace
  species 1e-40 n; dt = a 1 % step in 1+z; the difference-quotient
  Jacobian (its rates depend on the densities).
"""
import numpy as np

GRAVITY = 6.6743e-08
PI = 3.141592653589793


def loguniform(rng, lo, hi, size):
    return np.exp(rng.uniform(np.log(lo), np.log(hi), size))


def free_fall_time(n, mass_g):
    """sqrt(3 pi / (32 G rho)) per cell (rho = sum n_i m_i, sequential)"""
    rho = np.zeros(n.shape[0])
    for i in range(n.shape[1]):
        rho = rho + n[:, i] * mass_g[i]
    return np.sqrt(3.0 * PI / (32.0 * GRAVITY * np.maximum(rho, 1e-40)))


def _index(species):
    return {s: i for i, s in enumerate(species)}


def primordial(ncell, info, seed=0):
    species, mass_g, param_names = info["species"], info["mass_g"], info["params"]
    rng = np.random.default_rng(seed)
    ix = _index(species)
    nH = loguniform(rng, 1.0, 1e6, ncell)
    T = loguniform(rng, 10.0, 1e4, ncell)
    n = np.repeat((1e-20 * nH)[:, None], len(species), axis=1)
    n[:, ix["H"]] = nH
    n[:, ix["H+"]] = nH * 1e-4
    n[:, ix["e-"]] = nH * 1e-4
    n[:, ix["He"]] = nH * 0.0775
    dt = np.full(ncell, 3.15e10)
    par = _default_rows(ncell, info)
    par[:, param_names.index("tff")] = free_fall_time(n, mass_g)
    return n, T, dt, par


def primordial3(ncell, info, seed=0):
    species, mass_g, param_names = info["species"], info["mass_g"], info["params"]
    rng = np.random.default_rng(seed)
    ix = _index(species)
    nH = loguniform(rng, 1.0, 1e14, ncell)
    T = loguniform(rng, 50.0, 5000.0, ncell)
    xH2 = loguniform(rng, 1e-6, 0.5, ncell)
    xe = loguniform(rng, 1e-8, 1e-2, ncell)
    n = np.repeat((1e-20 * nH)[:, None], len(species), axis=1)
    n[:, ix["H2"]] = xH2 * nH
    n[:, ix["H+"]] = xe * nH
    n[:, ix["e-"]] = xe * nH
    n[:, ix["He"]] = 0.0775 * nH
    # H = n_H - 2 n_H2 - n_H+, floored at the trace level: with x_H2 near
    # 0.5 and a large ionisation fraction the difference is negative, an
    # unphysical input whose clipping would break the nuclei balance
    n[:, ix["H"]] = np.maximum(nH - 2.0 * n[:, ix["H2"]] - n[:, ix["H+"]],
                               1e-20 * nH)
    par = _default_rows(ncell, info)
    tff = free_fall_time(n, mass_g)
    par[:, param_names.index("tff")] = tff
    dt = 0.01 * tff
    return n, T, dt, par


def hydro_step(n, par, mass_g, param_names):
    """one call of the collapse loop, in place: tff of the current state,
    densities x 1.01, dt = 0.01 tff (returned)"""
    tff = free_fall_time(n, mass_g)
    par[:, param_names.index("tff")] = tff
    n *= 1.01
    return 0.01 * tff


def galaxy_ism(ncell, info, seed=0):
    species, mass_g, param_names = info["species"], info["mass_g"], info["params"]
    rng = np.random.default_rng(seed)
    ix = _index(species)
    nH = loguniform(rng, 1e-2, 1e4, ncell)
    T = loguniform(rng, 10.0, 1e6, ncell)
    n = np.repeat((1e-20 * nH)[:, None], len(species), axis=1)
    n[:, ix["H"]] = nH
    n[:, ix["H2"]] = 1e-6 * nH
    n[:, ix["H+"]] = 1e-4 * nH
    n[:, ix["e-"]] = 1e-4 * nH
    n[:, ix["He"]] = 0.0775 * nH
    par = _default_rows(ncell, info)
    par[:, param_names.index("crate")] = loguniform(rng, 1e-17, 1e-16, ncell)
    par[:, param_names.index("G0")] = loguniform(rng, 0.3, 3.0, ncell)
    par[:, param_names.index("d2g")] = loguniform(rng, 0.003, 0.03, ncell)
    dt = np.full(ncell, 3.15e11)
    return n, T, dt, par


def primordialZ(ncell, info, seed=0):
    species = info["species"]
    rng = np.random.default_rng(seed)
    ix = _index(species)
    nH = loguniform(rng, 1.0, 1e6, ncell)
    T = loguniform(rng, 30.0, 3000.0, ncell)
    xH2 = loguniform(rng, 1e-6, 0.5, ncell)
    xHp = loguniform(rng, 1e-6, 1e-3, ncell)
    Z = loguniform(rng, 1e-3, 1.0, ncell)
    n = np.repeat((1e-20 * nH)[:, None], len(species), axis=1)
    n[:, ix["H2"]] = xH2 * nH
    n[:, ix["H+"]] = xHp * nH
    n[:, ix["H"]] = np.maximum(nH - 2.0 * n[:, ix["H2"]] - n[:, ix["H+"]],
                               1e-20 * nH)
    n[:, ix["He"]] = 0.0775 * nH
    n[:, ix["C+"]] = 1.4e-4 * Z * nH
    n[:, ix["O"]] = 3.2e-4 * Z * nH
    q = np.asarray(info["charge"], dtype=float)
    e = ix["e-"]
    n[:, e] = 0.0
    n[:, e] = n @ q
    par = _default_rows(ncell, info)
    dt = np.full(ncell, 3.15e11)
    return n, T, dt, par


def earlyUniverse(ncell, info, seed=0):
    species, param_names = info["species"], info["params"]
    rng = np.random.default_rng(seed)
    ix = _index(species)
    hubble0 = 1e2 * 0.704 * 1e5 / 3.0856775814913673e24  # s^-1
    z = loguniform(rng, 20.0, 2000.0, ncell)
    a = 1.0 + z
    dd = 0.0456 * 9.19e-6 * a ** 3
    x = loguniform(rng, 1e-4, 1.0, ncell)
    n = np.repeat((1e-40 * dd)[:, None], len(species), axis=1)
    n[:, ix["H+"]] = 0.924 * dd * x
    n[:, ix["H"]] = 0.924 * dd * (1.0 - x) + 1e-40 * dd
    n[:, ix["D+"]] = 4.3e-5 * dd * x
    n[:, ix["D"]] = 4.3e-5 * dd * (1.0 - x) + 1e-40 * dd
    n[:, ix["He"]] = 0.076 * dd
    n[:, ix["He+"]] = 0.076e-6 * dd
    q = np.asarray(info["charge"], dtype=float)
    e = ix["e-"]
    n[:, e] = 0.0
    n[:, e] = n @ q
    T = 2.73 * a
    par = _default_rows(ncell, info)
    par[:, param_names.index("zredshift")] = z
    par[:, param_names.index("Trad")] = T
    par[:, param_names.index("Tcmb")] = 2.73
    par[:, param_names.index("hubble0")] = hubble0
    par[:, param_names.index("omega0")] = 1.0
    dt = 0.01 * a / (hubble0 * a * a * np.sqrt(z + 1.0))
    return n, T, dt, par


SEMENOV_INITIAL = (("He", 9e-2), ("H2", 0.5), ("C+", 1.2e-4), ("N", 7.6e-5),
                   ("O", 2.56e-4), ("S+", 8e-8), ("Si+", 8e-9), ("Fe+", 3e-9),
                   ("Na+", 2e-9), ("Mg+", 7e-9), ("P+", 2e-10), ("Cl+", 1e-9))


def semenov(ncell, info, seed=0):
    species, mass_g, param_names = info["species"], info["mass_g"], info["params"]
    rng = np.random.default_rng(seed)
    ix = _index(species)
    nH = loguniform(rng, 1e2, 1e7, ncell)
    T = loguniform(rng, 10.0, 300.0, ncell)
    n = np.repeat((1e-20 * nH)[:, None], len(species), axis=1)
    for s, x in SEMENOV_INITIAL:
        n[:, ix[s]] = x * nH * loguniform(rng, 0.5, 2.0, ncell)
    charge = np.asarray(info["charge"], dtype=float)
    ions = [i for i, s in enumerate(species) if s != "e-"]
    n[:, ix["e-"]] = np.maximum((n[:, ions] * charge[ions]).sum(axis=1), 0.0)
    rho = np.zeros(ncell)
    for i in range(len(species)):
        rho = rho + n[:, i] * mass_g[i]
    a = 1e-5
    xdust = 0.01 * rho / (4.0 / 3.0 * PI * 3.0 * a ** 3 * 1.43)
    n[:, ix["GRAIN0"]] = xdust
    par = _default_rows(ncell, info)
    for name, v in (("Av", 10.0), ("crflux", 1.3e-17), ("gsize", a),
                    ("gsize2", a * a)):
        par[:, param_names.index(name)] = v
    par[:, param_names.index("xdust")] = xdust
    par[:, param_names.index("Tdust")] = T
    dt = np.full(ncell, 3.15e13)
    return n, T, dt, par


def cloud(ncell, info, seed=0):
    species, param_names = info["species"], info["params"]
    rng = np.random.default_rng(seed)
    ix = _index(species)
    nH = loguniform(rng, 1e2, 1e7, ncell)
    T = loguniform(rng, 10.0, 300.0, ncell)
    n = np.repeat((1e-20 * nH)[:, None], len(species), axis=1)
    for s, x in SEMENOV_INITIAL:
        n[:, ix[s]] = x * nH * loguniform(rng, 0.5, 2.0, ncell)
    n[:, ix["GRAIN0"]] = 1.3e-12 * nH
    charge = np.asarray(info["charge"], dtype=float)
    ions = [i for i, s in enumerate(species) if s != "e-"]
    n[:, ix["e-"]] = np.maximum((n[:, ions] * charge[ions]).sum(axis=1), 0.0)
    par = _default_rows(ncell, info)
    for name, v in (("Av", 10.0), ("crate", 1.3e-17), ("gas_dust_ratio", 1.0)):
        par[:, param_names.index(name)] = v
    dt = np.full(ncell, 3.15e13)
    return n, T, dt, par


def _default_rows(ncell, info):
    """every cell's parameter row at the network defaults (NaN: required)"""
    return np.repeat(np.asarray(info["defaults"], dtype=float)[None, :],
                     ncell, axis=0)


def hydro_step_info(n, par, info):
    return hydro_step(n, par, info["mass_g"], info["params"])


GENERATORS = {"primordial": primordial, "primordial3": primordial3,
              "galaxy_ism": galaxy_ism, "semenov": semenov, "cloud": cloud,
              "primordialZ": primordialZ, "earlyUniverse": earlyUniverse}

# the solve options of each workload (krome_opts keys)
OPTIONS = {
    "primordial": dict(evolve_T=1, jac=1, linsol=1, rtol=1e-6, atol_n=1e-20,
                       atol_T=1e-6),
    "primordial3": dict(evolve_T=1, jac=0, linsol=0, rtol=1e-6,
                        atol_n=1e-20, atol_T=1e-6),
    "galaxy_ism": dict(evolve_T=1, jac=0, linsol=0, rtol=1e-6,
                       atol_n=1e-20, atol_T=1e-6),
    "primordialZ": dict(evolve_T=0, jac=2, linsol=0, rtol=1e-6,
                        atol_n=1e-20, atol_T=1e-6),
    "earlyUniverse": dict(evolve_T=0, jac=2, linsol=0, rtol=1e-6,
                          atol_n=1e-20, atol_T=1e-6),
    "semenov": dict(evolve_T=0, jac=0, linsol=3, rtol=1e-6, atol_n=1e-20,
                    atol_T=1e-6, max_steps=1000000),
    "cloud": dict(evolve_T=0, jac=0, linsol=3, rtol=1e-6, atol_n=1e-20,
                  atol_T=1e-6, max_steps=1000000),
}
