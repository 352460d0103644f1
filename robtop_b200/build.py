"""Build the sm_100a solver library ``robtop_b200/librtb200.so`` in place.

nvcc cross-compiles every ``csrc/*.cu`` for ``arch=compute_100a,code=sm_100a``
(no GPU needed) and links them into one shared library whose exported
``extern "C"`` symbols are declared in ``include/rtb200.h``.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(ROOT, "_build", "rtb200")
LIB = os.path.join(HERE, "librtb200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "--expt-relaxed-constexpr", "-Xptxas", "-O3"]


def _nvcc():
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _host_cxx():
    # the image's default CC wrapper lacks some spec files; prefer the system compiler
    for c in ("/usr/bin/g++", shutil.which("g++")):
        if c and os.path.exists(c):
            return c
    return None


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers_mtime():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(ROOT, "include", "rtb200.h"))
    return max(os.path.getmtime(h) for h in hs if os.path.exists(h))


def _compile(src, verbose=False, extra=()):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), _headers_mtime()) and not extra:
        return obj
    cmd = [_nvcc(), *ARCH, *FLAGS, *extra, "-c", src, "-o", obj]
    cxx = _host_cxx()
    if cxx:
        cmd[1:1] = ["-ccbin", cxx]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        print(r.stderr, file=sys.stderr)
    return obj


def build(verbose=False, ptxas_info=False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    extra = ("-Xptxas", "-v") if ptxas_info else ()
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose or ptxas_info, extra), srcs))
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(o) for o in objs) and not extra:
        return LIB
    cmd = [_nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
    cxx = _host_cxx()
    if cxx:
        cmd[1:1] = ["-ccbin", cxx]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


COMPAT_SRC = os.path.join(ROOT, "tests", "cpp", "compat_main.cpp")
COMPAT_BIN = os.path.join(ROOT, "tests", "cpp", "compat_test")


def build_compat_driver() -> str:
    """C++ driver of the reference-signature layer (tests/cpp/compat_main.cpp)."""
    lib = build()
    if os.path.exists(COMPAT_BIN) and os.path.getmtime(COMPAT_BIN) >= max(os.path.getmtime(COMPAT_SRC),
                                                                           os.path.getmtime(lib)):
        return COMPAT_BIN
    cxx = _host_cxx() or "g++"
    cmd = [cxx, "-O2", "-std=c++17", COMPAT_SRC, "-o", COMPAT_BIN, "-I/usr/local/cuda/include", f"-L{HERE}",
           "-lrtb200", f"-Wl,-rpath,{HERE}", "-Wl,-rpath,$ORIGIN/../../robtop_b200"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compat driver build failed:\n{r.stdout}\n{r.stderr}")
    return COMPAT_BIN


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv))
    print(build_compat_driver())
