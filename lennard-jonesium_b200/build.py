"""Build the engine's shared library (lib/liblj_gpu.so) for sm_100a.

    python lennard-jonesium_b200/build.py [--force] [--verbose]

Compiles every csrc/*.cu and csrc/*.cpp translation unit with nvcc
(-gencode arch=compute_100a,code=sm_100a) and links them into one shared
object that exports the C ABI of include/lj_gpu.h.  Objects are rebuilt when
a source or header is newer than the library.
"""

import argparse
import pathlib
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = HERE / "csrc"
OUT = HERE / "lib"
OBJ = HERE / "lib" / "obj"
LIB = OUT / "liblj_gpu.so"

NVCC = "nvcc"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++20", "-Xcompiler", "-fPIC", "-I", str(ROOT / "include"),
          "-I", str(CSRC)]


def _sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def _deps():
    return _sources() + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + \
        sorted((ROOT / "include").glob("*.h"))


def build(force=False, verbose=False, ptxas_info=False):
    OBJ.mkdir(parents=True, exist_ok=True)
    newest = max(p.stat().st_mtime for p in _deps())
    if LIB.exists() and not force and LIB.stat().st_mtime >= newest and not ptxas_info:
        return LIB
    objs = []
    for src in _sources():
        obj = OBJ / (src.stem + ".o")
        cmd = [NVCC, *ARCH, *COMMON, "-c", str(src), "-o", str(obj)]
        if ptxas_info:
            cmd.insert(1, "-Xptxas=-v")
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    cmd = [NVCC, *ARCH, "-shared", "-o", str(LIB), *objs, "-lcudart"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose, a.ptxas_info))
    sys.exit(0)
