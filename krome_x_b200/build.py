"""Build the C-ABI libraries: ``krome_x_b200/lib/libkrome_b200_<net>.so``,
one per generated network (as the reference compiles its krome.cpp once
per generated project), for sm_100a with nvcc, in-tree.

The CUDA runtime is linked statically so the library needs only the driver.
``python -m krome_x_b200.build [net ...]`` (default: every network header).
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
LIBDIR = PKG / "lib"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-shared",
         "-Xcompiler", "-fPIC,-fvisibility=hidden", "-cudart", "static"]


def networks():
    return sorted(p.stem[len("net_"):]
                  for p in (PKG / "networks").glob("net_*.h"))


def lib_path(key):
    return LIBDIR / ("libkrome_b200_%s.so" % key)


def _sources(key):
    return ([PKG / "csrc" / "krome_b200.cu", PKG / "networks" / ("net_%s.h" % key)]
            + list((PKG / "csrc").glob("*.cuh")) + list((PKG / "csrc").glob("*.h")))


def stale(key):
    lib = lib_path(key)
    if not lib.exists():
        return True
    t = lib.stat().st_mtime
    return any(s.stat().st_mtime > t for s in _sources(key))


def build(key, force=False, verbose=False):
    lib = lib_path(key)
    if not force and not stale(key):
        return lib
    LIBDIR.mkdir(parents=True, exist_ok=True)
    tmp = lib.with_suffix(".so.tmp")
    cmd = ([NVCC] + ARCH + FLAGS + ["-I" + str(ROOT),
           '-DKB_NET_HEADER="krome_x_b200/networks/net_%s.h"' % key,
           str(PKG / "csrc" / "krome_b200.cu"), "-o", str(tmp)])
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s" % (key, r.stderr[-4000:]))
    os.replace(tmp, lib)
    if verbose:
        print(r.stderr)
    return lib


def build_all(keys=None, force=False):
    keys = keys or networks()
    with ThreadPoolExecutor(max_workers=min(len(keys), os.cpu_count() or 1)) as ex:
        return list(ex.map(lambda k: build(k, force), keys))


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("-")]
    for p in build_all(args or None, force="--force" in sys.argv):
        print("built", p)
