"""Generate the golden fixtures of the parity tests from the reference.

Run where the reference tree and oracle/_ref (oracle/build_ref.py) exist:
``python tests/golden/make_golden.py``. For each benchmark network it writes
``tests/golden/<net>.npz`` with

* ``k_T, k_n, k_idx, k_ref``: the reference's own golden rate vectors -- the
  K_REF table the reference generator writes into each project's
  krome_check.cpp (rate coefficients at three temperatures, computed by its
  independent network interpreter, kromex/netcheck.py), with the probe
  parameters of that check (every parameter 1.3e-17, Tdust 10 K);
* ``n, T, dt, par`` / ``n_out, T_out, flags``: 64 seeded cells (16 for
  the large networks, Semenov and cloud) of the
  benchmark workload solved by the reference's strict build
  (oracle/_ref/libkrome_<net>_strict.so, krome_solve_cells) with the
  workload's options, each network in its own process (the generated
  libraries must not share one).

and ``tests/golden/semenov_evt.npz`` / ``cloud_evt.npz``: 8 seeded cells of
each large network solved by the reference's strict build with Tgas evolved
and the analytic (hybrid) Jacobian (``evolve_T=1, jac=1``): the sparse LU
with its Tgas border (``python tests/golden/make_golden.py semenov_evt
cloud_evt``).
"""
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

from krome_x_b200 import netinfo, workloads  # noqa: E402
from oracle import reference_solve  # noqa: E402

NCELL = 64


def _array(text, name):
    m = re.search(r"%s\[[^\]]*\](?:\[[^\]]*\])?\s*=\s*(\{.*?\});" % name, text,
                  re.S)
    body = m.group(1).replace("{", "[").replace("}", "]")
    return np.array(eval(body), dtype=float)


# fixtures of other solve options: name -> (network, cells, options added)
VARIANTS = {"semenov_evt": ("semenov", 8, dict(evolve_T=1, jac=1)),
            "cloud_evt": ("cloud", 8, dict(evolve_T=1, jac=1))}


def variant(name):
    key, ncell, extra = VARIANTS[name]
    info = netinfo.load(key)
    n, T, dt, par = workloads.GENERATORS[key](ncell, info, seed=11)
    opts = dict(workloads.OPTIONS[key])
    opts.update(extra)
    out = reference_solve(key, n, T, dt, par, strict=True, **opts)
    np.savez_compressed(HERE / ("%s.npz" % name), n=n, T=T, dt=dt, par=par,
                        n_out=out["n"], T_out=out["T"], flags=out["flags"],
                        ret=out["ret"])
    print(name, "flags", np.unique(out["flags"]), "->", HERE / ("%s.npz" % name))


def main(keys=None):
    for name in [k for k in keys or () if k in VARIANTS]:
        variant(name)
    keys = [k for k in keys or () if k not in VARIANTS] if keys else None
    if keys == []:
        return
    for key in keys or ("primordial", "primordial3", "galaxy_ism", "semenov"):
        info = netinfo.load(key)
        chk = (ROOT / "oracle" / "_ref" / "gen" / key / "krome_check.cpp").read_text()
        k_T = _array(chk, "T_REF")
        k_n = _array(chk, "N_REF")
        k_idx = _array(chk, "I_REF").astype(np.int32)
        k_ref = _array(chk, "K_REF")
        # the large networks' cells take ~1 s each in the reference
        ncell = 16 if key in ("semenov", "cloud") else NCELL
        n, T, dt, par = workloads.GENERATORS[key](ncell, info, seed=11)
        opts = dict(workloads.OPTIONS[key])
        out = reference_solve(key, n, T, dt, par, strict=True, **opts)
        np.savez_compressed(HERE / ("%s.npz" % key), k_T=k_T, k_n=k_n,
                            k_idx=k_idx, k_ref=k_ref, n=n, T=T, dt=dt, par=par,
                            n_out=out["n"], T_out=out["T"], flags=out["flags"],
                            ret=out["ret"])
        print(key, "flags", np.unique(out["flags"]), "->", HERE / ("%s.npz" % key))


if __name__ == "__main__":
    main(sys.argv[1:])
