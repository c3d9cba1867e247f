"""Shared fixtures of the test suite.

Markers: ``gpu`` for tests that need a CUDA device (run on the B200 host with
``pytest -m gpu``); everything else runs on the CPU (``-m "not gpu"``).
"""
import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

NETWORKS = ("primordial", "primordial3", "galaxy_ism")
# networks past the dense kernels' size, solved by the sparse path
LARGE = ("semenov", "cloud")
ALL_NETWORKS = NETWORKS + LARGE


# the oracle's one-ulp noise floor of each parity case (tests/golden/
# noise_floor.py): the smallest fraction of passing cells and the worst
# cell's relative error over five draws of one-ulp input moves
NOISE_FLOOR = json.loads((ROOT / "tests" / "golden" / "noise_floor.json").read_text())
# the bars against the floor: the fraction may fall 0.03 below it (a batch
# of 512 cells has a sampling spread of about that size); the worst cell may
# reach three times the floor's (the GPU's CUDA math and contraction move
# many last bits at once: one more draw of the same chaotic amplification,
# and the maximum of five draws itself moves by up to 1.5x between sets of
# draws)
FRAC_MARGIN = 0.03
WORST_FACTOR = 3.0


def assert_at_floor(m, case):
    """the parity metric m of a GPU solve against the oracle's floor of
    `case`: flags equal, the fraction of passing cells and the worst cell
    (abundances and Tgas) at the floor"""
    f = NOISE_FLOOR[case]
    assert m["flags_equal"] == 1.0, (case, m)
    assert m["frac"] >= f["frac"] - FRAC_MARGIN, (case, m, f)
    assert m["max_rel"] <= WORST_FACTOR * f["max_rel"], (case, m, f)
    assert m["max_relT"] <= max(WORST_FACTOR * f["max_relT"], 1e-12), (case, m, f)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def golden(key):
    return np.load(ROOT / "tests" / "golden" / ("%s.npz" % key))


def parity(a_n, a_T, a_flags, b_n, b_T, b_flags, rtol, atol=1e-20):
    """the parity metric of the benchmark: over the cells where both
    solves succeed, the relative error of every abundance above atol/rtol
    (the rtol-dominated ones) and of Tgas must be <= 10 rtol; returns the
    fraction of such cells that pass, the CVODE-weighted error
    |a - b| / (rtol |b| + atol) of the others (max), and the flag
    agreement"""
    ok = (a_flags == 0) & (b_flags == 0)
    na, nb = a_n[ok], b_n[ok]
    big = np.abs(nb) > atol / rtol
    with np.errstate(all="ignore"):
        rel = np.where(big, np.abs(na - nb) / np.abs(nb), 0.0)
        wgt = np.where(big, 0.0, np.abs(na - nb) / (rtol * np.abs(nb) + atol))
    relT = np.abs(a_T[ok] - b_T[ok]) / np.abs(b_T[ok])
    cell_ok = (rel.max(axis=1) <= 10 * rtol) & (relT <= 10 * rtol)
    return dict(cells=int(ok.sum()),
                frac=float(cell_ok.mean()) if ok.any() else 1.0,
                max_rel=float(rel.max()) if ok.any() else 0.0,
                max_relT=float(relT.max()) if ok.any() else 0.0,
                max_weighted_trace=float(wgt.max()) if ok.any() else 0.0,
                flags_equal=float(np.mean(a_flags == b_flags)))


def parity_major(a_n, a_flags, b_n, b_flags, n0, rtol, xmin=1e-12):
    """the parity metric of the large networks: per cell, the largest
    relative error of the abundances above xmin of the cell's total initial
    density (the species a surface-chemistry run is read for), over the
    cells where both solves succeed; the fraction within 10 rtol, the worst
    cell, and the flag agreement. Hundreds of species over 1e13 s make these
    solves more sensitive than the small networks': one ulp on the inputs
    moves the worst cell by up to ~5e-5 (rtol 1e-6)."""
    ok = (a_flags == 0) & (b_flags == 0)
    nH = n0[ok].sum(axis=1)
    na, nb = a_n[ok], b_n[ok]
    big = np.abs(nb) > xmin * nH[:, None]
    with np.errstate(all="ignore"):
        rel = np.where(big, np.abs(na - nb) / np.abs(nb), 0.0).max(axis=1)
    return dict(cells=int(ok.sum()),
                frac=float((rel <= 10 * rtol).mean()) if ok.any() else 1.0,
                max_rel=float(rel.max()) if ok.any() else 0.0,
                flags_equal=float(np.mean(a_flags == b_flags)))


@pytest.fixture(scope="session")
def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
