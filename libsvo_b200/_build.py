"""Builds ``libsvo_b200/_lib/libsvo_b200.so`` in-tree.

C++ host sources go through g++, CUDA sources through nvcc for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``) with FMA contraction off
(``-fmad=false``; the kernels also use explicit round-to-nearest intrinsics),
and the shared object links the CUDA runtime statically.  The build needs no
GPU: nvcc cross-compiles.

``build_sanitized()`` (``--sanitize``) builds a second library,
``_lib/libsvo_b200_asan.so``, whose host code is compiled with
AddressSanitizer and UndefinedBehaviorSanitizer (the CUDA objects are the
regular ones); load it with the sanitizer runtimes preloaded
(``SANITIZER_PRELOAD``) and ``LIBSVO_B200_LIB`` pointing at it.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
OBJ_DIR = PKG / "_build"
LIB_DIR = PKG / "_lib"
LIB = LIB_DIR / "libsvo_b200.so"

CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC",
                     "-Xptxas", "-warn-spills"]
CXX_FLAGS = ["-std=c++17", "-O2", "-fPIC", "-pthread", "-Wall", "-Wextra", "-Wno-unused-parameter",
             f"-I{CUDA_HOME / 'include'}"]


def sources():
    return sorted(CSRC.glob("*.cpp")) + sorted(CSRC.glob("*.cu"))


def _headers():
    return list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))


def _stale(obj: Path, src: Path, newest_header: float) -> bool:
    if not obj.is_file():
        return True
    t = obj.stat().st_mtime
    return t < src.stat().st_mtime or t < newest_header or t < Path(__file__).stat().st_mtime


def _compile(src: Path, obj: Path, verbose: bool):
    if src.suffix == ".cu":
        cmd = [NVCC, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
    else:
        cmd = ["g++", *CXX_FLAGS, "-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {src.name}\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip() and verbose:
        print(r.stderr, file=sys.stderr)


def build(force: bool = False, verbose: bool = False) -> Path:
    OBJ_DIR.mkdir(parents=True, exist_ok=True)
    LIB_DIR.mkdir(parents=True, exist_ok=True)
    newest = max((h.stat().st_mtime for h in _headers()), default=0.0)
    jobs = []
    objs = []
    for src in sources():
        obj = OBJ_DIR / (src.name + ".o")
        objs.append(obj)
        if force or _stale(obj, src, newest):
            jobs.append((src, obj))
    if jobs:
        with ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            list(ex.map(lambda j: _compile(j[0], j[1], verbose), jobs))
    if jobs or not LIB.is_file() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", str(LIB), *map(str, objs),
               "-Xcompiler", "-pthread", "-lrt", "-ldl"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed\n{r.stdout}\n{r.stderr}")
    return LIB


SAN_DIR = OBJ_DIR / "asan"
SAN_LIB = LIB_DIR / "libsvo_b200_asan.so"
SAN_FLAGS = ["-fsanitize=address,undefined", "-fno-omit-frame-pointer", "-fno-sanitize-recover=undefined"]


def sanitizer_preload() -> str:
    """The sanitizer runtimes a host process must preload to load SAN_LIB."""
    libs = []
    for name in ("libasan.so", "libubsan.so"):
        r = subprocess.run(["g++", f"-print-file-name={name}"], capture_output=True, text=True, check=True)
        libs.append(r.stdout.strip())
    return " ".join(libs)


def build_sanitized(verbose: bool = False) -> Path:
    """The library with AddressSanitizer/UBSan-instrumented host code."""
    build(verbose=verbose)  # the CUDA objects
    SAN_DIR.mkdir(parents=True, exist_ok=True)
    newest = max((h.stat().st_mtime for h in _headers()), default=0.0)
    jobs, objs = [], []
    for src in sorted(CSRC.glob("*.cpp")):
        obj = SAN_DIR / (src.name + ".o")
        objs.append(obj)
        if _stale(obj, src, newest):
            jobs.append((src, obj))

    def compile_one(job):
        src, obj = job
        cmd = ["g++", *CXX_FLAGS, "-O1", "-g", *SAN_FLAGS, "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"compile failed: {src.name}\n{r.stdout}\n{r.stderr}")

    if jobs:
        with ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            list(ex.map(compile_one, jobs))
    cu_objs = [OBJ_DIR / (src.name + ".o") for src in sorted(CSRC.glob("*.cu"))]
    inputs = objs + cu_objs
    if jobs or not SAN_LIB.is_file() or any(o.stat().st_mtime > SAN_LIB.stat().st_mtime for o in inputs):
        cmd = ["g++", "-shared", *SAN_FLAGS, "-o", str(SAN_LIB), *map(str, inputs),
               f"-L{CUDA_HOME / 'lib64'}", "-lcudart_static", "-lrt", "-ldl", "-pthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed\n{r.stdout}\n{r.stderr}")
    return SAN_LIB


if __name__ == "__main__":
    if "--sanitize" in sys.argv:
        print(build_sanitized(verbose="-v" in sys.argv))
    else:
        print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
