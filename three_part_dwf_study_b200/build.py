"""Build recipe for the sm_100a shared library (``_lib/libdwfb200.so``).

Compiles every ``csrc/*.cu`` and ``csrc/*.cpp`` with nvcc for
``-gencode arch=compute_100a,code=sm_100a`` and links them into one shared
library exporting the C ABI of ``include/dwf_b200.h``. Objects are rebuilt
only when a source or header is newer than the library.

    python -m three_part_dwf_study_b200.build [--force] [-v]
"""
import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
REPO = PKG.parent
CSRC = PKG / "csrc"
OUT_DIR = PKG / "_lib"
LIB = OUT_DIR / "libdwfb200.so"
OBJ_DIR = PKG / "_build"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
HOST_CXX = "/usr/bin/g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                   "-ccbin", HOST_CXX, "-I", str(REPO / "include")]
CPP_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-I", str(REPO / "include"),
             "-I", "/usr/local/cuda/include"]


def _sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def _headers():
    return (sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.hpp"))
            + sorted((REPO / "include").glob("*.h")))


def _stale(target, deps):
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(src, verbose):
    obj = OBJ_DIR / (src.name + ".o")
    if src.suffix == ".cu":
        cmd = [NVCC] + CU_FLAGS + ["-c", str(src), "-o", str(obj)]
    else:
        cmd = [HOST_CXX] + CPP_FLAGS + ["-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {src.name}\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr.strip():
        print(r.stderr)
    return obj


def build(force=False, verbose=False):
    """Compile and link the library if any source changed. Returns its path."""
    srcs = _sources()
    deps = srcs + _headers()
    if not force and not _stale(LIB, deps):
        return LIB
    if not Path(NVCC).exists():
        raise RuntimeError(f"nvcc not found at {NVCC}")
    OBJ_DIR.mkdir(exist_ok=True)
    OUT_DIR.mkdir(exist_ok=True)
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [NVCC] + ARCH + ["-shared", "-ccbin", HOST_CXX, "-o", str(tmp)] + [str(o) for o in objs]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=a.verbose))


if __name__ == "__main__":
    sys.exit(main())
