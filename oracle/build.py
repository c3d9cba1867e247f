"""Build the CPU oracle (test infrastructure only: the checker).

Compiles ``oracle/bdf_oracle.cpp`` once per generated network header into
``oracle/_build/liboracle_<net>.so`` with strict IEEE flags (``-O2
-ffp-contract=off``: no contraction, so the oracle rounds as the reference's
strict build does) and OpenMP over cells.

Usage: ``python oracle/build.py [net ...]`` (default: every header in
krome_x_b200/networks).
"""
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
OUT = HERE / "_build"
FLAGS = ["-O2", "-std=c++17", "-ffp-contract=off", "-fopenmp", "-fPIC",
         "-shared", "-fvisibility=hidden"]


def networks():
    return sorted(p.stem[len("net_"):]
                  for p in (ROOT / "krome_x_b200" / "networks").glob("net_*.h"))


def build(key, force=False):
    OUT.mkdir(parents=True, exist_ok=True)
    src = HERE / "bdf_oracle.cpp"
    hdr = ROOT / "krome_x_b200" / "networks" / ("net_%s.h" % key)
    lib = OUT / ("liboracle_%s.so" % key)
    deps = [src, hdr] + list((ROOT / "krome_x_b200" / "csrc").glob("kb_*.h"))
    if (not force and lib.exists()
            and lib.stat().st_mtime > max(d.stat().st_mtime for d in deps)):
        return lib
    cmd = (["g++"] + FLAGS + ["-I" + str(ROOT),
           '-DKB_NET_HEADER="krome_x_b200/networks/net_%s.h"' % key,
           "-DKB_ORACLE_EXPORT", str(src), "-o", str(lib)])
    subprocess.run(cmd, check=True)
    return lib


def main(argv):
    for k in (argv or networks()):
        print("built", build(k, force=True))


if __name__ == "__main__":
    main(sys.argv[1:])
