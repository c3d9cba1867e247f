"""The oracle's own noise floor on the parity tests' workloads.

CVODE's step and order decisions amplify last-bit differences of the
inputs chaotically, so a solve's sensitivity to its last bits bounds how
closely two correct implementations (the GPU's CUDA math and FMA
contraction against the host's) can agree. This script measures it with the
oracle alone: each case is solved once as given and five more times with
every input (densities, Tgas, dt, parameters) moved by one ulp in a random
direction, and the benchmark's parity metric (conftest.parity) is taken
between the unperturbed and each perturbed solve. Recorded per case: the
smallest fraction of passing cells and the worst cell's largest relative
error (abundances above atol/rtol; Tgas) over the five draws.

Cases (each matching a parity test or smoke()): the first call of each
small network's workload (512 cells, seed 3; 1024 cells, seed 11; the
FP32-LU tests' 1024 cells, seed 31, solved by the oracle's FP32-LU twin; smoke()'s 64 primordial3 cells, seed
7; the reference binding's 512 primordial3 cells, seed 52; 512
galaxy_ism cells under a photon field, seed 62), the full
4,096-cell config-0 batch (primordial, analytic Jacobian, seed 0), and the
primordial3 hydro loop (4,096 cells, seed 1000, 10 calls; each call's
inputs are the unperturbed loop's state, so the floor is that of one call).

    python tests/golden/noise_floor.py       # writes tests/golden/noise_floor.json
"""
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT / "tests"))

from conftest import parity  # noqa: E402
from krome_x_b200 import netinfo, workloads  # noqa: E402
from oracle import Oracle  # noqa: E402

DRAWS = 5


def ulp_move(a, rng):
    a = np.asarray(a, dtype=float)
    up = rng.integers(0, 2, size=a.shape).astype(bool)
    out = np.where(up, np.nextafter(a, np.inf), np.nextafter(a, -np.inf))
    return np.where(np.isfinite(a) & (a != 0.0), out, a)


def floor_of(orc, key, n, T, dt, par, opts, rng):
    base = orc.solve(n, T, dt, par, **opts)
    fracs, worst, worstT = [], 0.0, 0.0
    for _ in range(DRAWS):
        pert = orc.solve(ulp_move(n, rng), ulp_move(T, rng), ulp_move(dt, rng),
                         ulp_move(par, rng), **opts)
        m = parity(pert["n"], pert["T"], pert["flags"], base["n"], base["T"],
                   base["flags"], opts["rtol"])
        fracs.append(m["frac"])
        worst = max(worst, m["max_rel"])
        worstT = max(worstT, m["max_relT"])
    return base, dict(frac=min(fracs), max_rel=worst, max_relT=worstT)


def first_call(key, ncell, seed, rng, **over):
    info = netinfo.load(key)
    n, T, dt, par = workloads.GENERATORS[key](ncell, info, seed=seed)
    opts = dict(workloads.OPTIONS[key], **over)
    _, f = floor_of(Oracle(key), key, n, T, dt, par, opts, rng)
    return f


def photo_floor(ncell, seed, rng):
    """galaxy_ism under its seeded photon field (tests/test_photo.py); the
    field rows are held, the cells' other inputs moved"""
    from test_photo import photo_case
    net, opts, (n, T, dt, par), Phi, bins, sigma = photo_case(ncell, seed)
    key = "galaxy_ism"
    o = dict(workloads.OPTIONS[key], photo_sigma=sigma, Phi=Phi)
    _, f = floor_of(Oracle(key), key, n, T, dt, par, o, rng)
    return f


def hydro_loop(ncell, seed, calls, rng):
    key = "primordial3"
    info = netinfo.load(key)
    n, T, dt, par = workloads.primordial3(ncell, info, seed=seed)
    par = np.array(par, copy=True)
    opts = workloads.OPTIONS[key]
    orc = Oracle(key)
    per_call = []
    for c in range(calls):
        if c > 0:
            dt = workloads.hydro_step_info(n, par, info)
        base, f = floor_of(orc, key, n, T, dt, par, opts, rng)
        per_call.append(f)
        ok = base["flags"] == 0
        n = np.where(ok[:, None], base["n"], n)
        T = np.where(ok, base["T"], T)
    return dict(frac=min(f["frac"] for f in per_call),
                max_rel=max(f["max_rel"] for f in per_call),
                max_relT=max(f["max_relT"] for f in per_call),
                calls=per_call)


def main():
    rng = np.random.default_rng(2024)
    out = {}
    for key in ("primordial", "primordial3", "galaxy_ism"):
        out["%s/first/512/3" % key] = first_call(key, 512, 3, rng)
        out["%s/first/1024/11" % key] = first_call(key, 1024, 11, rng)
    for key in ("primordial3", "galaxy_ism"):  # the FP32-LU tests: the twin
        out["%s/first/1024/31" % key] = first_call(key, 1024, 31, rng, lu32=1)
    out["primordial3/first/64/7"] = first_call("primordial3", 64, 7, rng)
    out["primordial3/first/512/52"] = first_call("primordial3", 512, 52, rng)
    out["primordial/config0/4096/0"] = first_call("primordial", 4096, 0, rng)
    out["galaxy_ism/photo/512/62"] = photo_floor(512, 62, rng)
    out["primordial3/hydro/4096/1000"] = hydro_loop(4096, 1000, 10, rng)
    (HERE / "noise_floor.json").write_text(json.dumps(out, indent=1) + "\n")
    for k, v in out.items():
        print("%-32s frac %.4f  worst %.3g  worstT %.3g"
              % (k, v["frac"], v["max_rel"], v["max_relT"]))


if __name__ == "__main__":
    main()
