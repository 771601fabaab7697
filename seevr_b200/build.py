"""Build libseevr_cuda.so in-tree (sm_100a) and the test oracle.

    python seevr_b200/build.py [--force] [--ptxas]

CUDA sources are compiled with nvcc for sm_100a only, -fmad=false so that
every float product and sum rounds on its own (the results match the FP32
oracle bit for bit), and host C++ with the system g++ without FP
contraction.  Objects go to seevr_b200/_build/, the library to
seevr_b200/libseevr_cuda.so.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libseevr_cuda.so"
INCLUDE = ROOT / "include"

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
CXX = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "-fmad=false", "--expt-relaxed-constexpr",
    "-ccbin", CXX,
    "-Xcompiler", "-fPIC,-O3,-ffp-contract=off,-fno-fast-math",
    "-I", str(INCLUDE),
]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-fopenmp",
             "-march=x86-64-v3", "-Wall", "-I", str(INCLUDE)]

CU_SOURCES = sorted(CSRC.glob("*.cu"))
CPP_SOURCES = sorted(CSRC.glob("*.cpp"))
HEADERS = sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted(INCLUDE.glob("*.h"))


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def _compile(src: Path, force: bool) -> Path:
    obj = BUILD / (src.name + ".o")
    if not force and not _stale(obj, [src, *HEADERS, Path(__file__)]):
        return obj
    if src.suffix == ".cu":
        _run([NVCC, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)])
    else:
        _run([CXX, *CXX_FLAGS, "-c", str(src), "-o", str(obj)])
    return obj


def build(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = CU_SOURCES + CPP_SOURCES
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), srcs))
    if force or _stale(LIB, objs):
        tmp = LIB.with_suffix(".so.tmp")
        _run([NVCC, *ARCH, "-shared", "-ccbin", CXX, "-o", str(tmp), *map(str, objs),
              "-Xcompiler", "-fopenmp", "-lgomp", "-lcudart"])
        os.replace(tmp, LIB)
    if verbose:
        print(f"built {LIB}")
    return LIB


def build_oracle(force: bool = False) -> Path:
    """Compile the CPU oracle (test infrastructure) with its Makefile."""
    out = ROOT / "oracle" / "liboracle.so"
    if force and out.exists():
        out.unlink()
    _run(["make", "-s", "-C", str(ROOT / "oracle")])
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print -Xptxas -v register/smem usage")
    a = ap.parse_args(argv)
    if a.ptxas:
        for src in CU_SOURCES:
            print(_run([NVCC, *NVCC_FLAGS, "-Xptxas", "-v", "-c", str(src), "-o", os.devnull]))
        return 0
    build(force=a.force, verbose=True)
    build_oracle(force=a.force)
    return 0


if __name__ == "__main__":
    sys.exit(main())
