"""Metadata of the generated networks (species, masses, charges, parameter
names and defaults), read from the JSON the emitter writes beside each
header; NaN marks a REQUIRED parameter."""
import json
from pathlib import Path

import numpy as np

NETDIR = Path(__file__).resolve().parent / "networks"


def available():
    return sorted(p.stem[len("net_"):] for p in NETDIR.glob("net_*.json"))


def load(key):
    meta = json.loads((NETDIR / ("net_%s.json" % key)).read_text())
    meta["defaults"] = [np.nan if d is None else float(d)
                        for d in meta["defaults"]]
    meta["mass_g"] = np.asarray(meta["mass_g"], dtype=float)
    return meta
