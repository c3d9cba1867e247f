"""Build the reference solver libraries used as the pinned CPU baseline.

Test infrastructure only (the checker, never the product): this recipe runs
the reference's own project generator (kromex, imported from the reference
tree) for the four benchmark networks and compiles each generated project
with g++ directly -- not the reference's Makefile -- into
``oracle/_ref/libkrome_<net>.so``. Everything is written under
``oracle/_ref/`` (git-ignored; it still travels to the GPU host with the
working tree, where ``/root/reference`` does not exist).

Network configurations (reference ``kromex.Preprocessor`` options):

* ``primordial``   networks/primordial.knet, cooling [ATOMIC, H2], heating
  [CHEM, COMPRESS]                                   (benchmark configs 0, 2)
* ``primordial3``  networks/primordial3.knet, cooling [H2, CONT, CHEM],
  heating [COMPRESS, CHEM], h2_opacity RIPAMONTI, gamma EXACT   (config 1)
* ``semenov``      examples/tests/cloudSurface/options.toml (the surface
  options are mandatory for Semenov.knet)                       (config 3)
* ``galaxy_ism``   networks/galaxy_ism.knet, default flags      (config 4)
* ``primordialZ``  networks/primordialZ.knet, default flags
* ``earlyUniverse``  networks/earlyUniverse.knet, default flags

Two libraries per network: ``libkrome_<net>.so`` with the generated
projects' production flags (``-O3 -std=c++17 -ffp-contract=fast
-fopenmp-simd``) plus ``-fopenmp``, so that ``krome_solve_cells`` runs its
OpenMP loop over cells on every host core (the timed CPU baseline; the
reference's default Python build is single-threaded), and
``libkrome_<net>_strict.so`` (``-O2 -ffp-contract=off``, single-threaded),
the build the CPU restatement is checked against bit for bit.

Usage: ``python oracle/build_ref.py [net ...]`` (default: all four).
"""
import os
import subprocess
import sys
import time
from pathlib import Path

# the reference tree: KROME_REFERENCE, else its mount point in the build
# container (this recipe is the one place that names it)
REF = Path(os.environ.get("KROME_REFERENCE", "/root/reference"))
HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
CXXFLAGS = ["-O3", "-std=c++17", "-ffp-contract=fast", "-fopenmp-simd",
            "-fopenmp", "-fPIC"]
# the strict build the checker is pinned to bit for bit: no contraction, no
# OpenMP (the reference's `#pragma omp simd` reductions stay sequential)
STRICT_FLAGS = ["-O2", "-std=c++17", "-ffp-contract=off", "-fPIC"]


def _configure(key):
    from kromex import Preprocessor
    if key == "primordial":
        kp = Preprocessor(network="primordial")
        kp.thermal.cooling = ["ATOMIC", "H2"]
        kp.thermal.heating = ["CHEM", "COMPRESS"]
    elif key == "primordial3":
        kp = Preprocessor(network="primordial3")
        kp.thermal.cooling = ["H2", "CONT", "CHEM"]
        kp.thermal.heating = ["COMPRESS", "CHEM"]
        kp.thermal.h2_opacity = "RIPAMONTI"
        kp.thermal.gamma = "EXACT"
    elif key in ("galaxy_ism", "primordialZ", "earlyUniverse", "cloud"):
        kp = Preprocessor(network=key)
    elif key == "semenov":
        kp = Preprocessor.from_file(
            str(REF / "examples/tests/cloudSurface/options.toml"))
        kp.project.network = str(REF / "networks/Semenov.knet")
    else:
        raise ValueError("unknown network key %r" % key)
    kp.project.bindings = ["python"]
    return kp


def build(key):
    gen = OUT / "gen" / key
    lib = OUT / ("libkrome_%s.so" % key)
    kp = _configure(key)
    t0 = time.time()
    kp.run(str(gen))
    netname = next(gen.glob("net_*_data.cpp")).name[len("net_"):-len("_data.cpp")]
    cmd = (["g++"] + CXXFLAGS + ["-shared", "-I" + str(gen),
           str(gen / "krome.cpp"), str(gen / ("net_%s_data.cpp" % netname)),
           "-o", str(lib)])
    subprocess.run(cmd, check=True)
    strict = OUT / ("libkrome_%s_strict.so" % key)
    cmd = (["g++"] + STRICT_FLAGS + ["-shared", "-I" + str(gen),
           str(gen / "krome.cpp"), str(gen / ("net_%s_data.cpp" % netname)),
           "-o", str(strict)])
    subprocess.run(cmd, check=True)
    print("built %s and %s (%s) in %.1f s" % (lib, strict, netname,
                                              time.time() - t0))
    return lib


def main(argv):
    sys.path.insert(0, str(REF))
    sys.path.insert(0, str(REF / "kromex"))
    OUT.mkdir(parents=True, exist_ok=True)
    keys = argv or ["primordial", "primordial3", "galaxy_ism", "primordialZ",
                    "earlyUniverse", "semenov", "cloud"]
    for k in keys:
        build(k)


if __name__ == "__main__":
    main(sys.argv[1:])
