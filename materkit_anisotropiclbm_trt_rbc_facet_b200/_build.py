"""In-tree build of the CUDA library ``libmkb200.so`` for sm_100a.

Compiles every translation unit under ``csrc/`` with nvcc (in parallel, only
when a source or header is newer than its object) and links them into the
package directory, so the shared object travels with the source tree.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmkb200.so")
INCLUDE = os.path.normpath(os.path.join(HERE, "..", "include"))

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "--expt-relaxed-constexpr",
                  "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
                  "-I", INCLUDE]
SOURCES = ["mk_kernels.cu", "mk_multiphase.cu", "mk_ensemble.cu", "mk_adjoint.cu", "mk_noalloc.cu", "mk_interface.cu", "mk_api.cpp", "mk_slab.cpp", "mk_case.cpp", "mk_xml.cpp"]


def _nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _headers() -> list[str]:
    out = [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    out += [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh", ".h"))]
    return out


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, verbose: bool) -> tuple[str, bool]:
    obj = os.path.join(OBJ, os.path.splitext(src)[0] + ".o")
    path = os.path.join(CSRC, src)
    deps = [path] + _headers()
    if not _stale(obj, deps):
        return obj, False
    # the object is stamped with its newest input's time as read before the
    # compile starts, so a source edited while nvcc runs is seen as newer
    stamp = max(os.path.getmtime(d) for d in deps)
    cmd = [_nvcc()] + NVFLAGS + ["-c", path, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [_nvcc(), "-x", "cu"] + NVFLAGS + ["-c", path, "-o", obj]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    os.utime(obj, (stamp, stamp))
    return obj, True


def build(verbose: bool = False) -> str:
    """Build libmkb200.so if needed and return its path."""
    os.makedirs(OBJ, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        done = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    objs = [o for o, _ in done]
    if any(rebuilt for _, rebuilt in done) or _stale(LIB, objs):
        cmd = [_nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose=True))
