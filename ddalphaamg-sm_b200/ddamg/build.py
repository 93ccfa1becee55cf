"""Builds libddamg.so (the CUDA library behind include/ddamg.h) in-tree for sm_100a.

    python -m ddamg.build            (from ddalphaamg-sm_b200/)
    python ddalphaamg-sm_b200/ddamg/build.py

Objects go to ddalphaamg-sm_b200/_build/, the library to ddalphaamg-sm_b200/ddamg/libddamg.so and the
command-line driver (driver/ddamg_main.cpp, the reference's main against the C ABI) to ddamg/ddamg_main.
Sources are recompiled when they (or a header) are newer than their object.
"""
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)                # ddalphaamg-sm_b200/
REPO = os.path.dirname(ROOT)
CSRC = os.path.join(ROOT, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "libddamg.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "-I" + os.path.join(REPO, "include"), "-I" + CSRC, "--expt-relaxed-constexpr"]


def _headers_mtime():
    hs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
    hs.append(os.path.join(REPO, "include", "ddamg.h"))
    return max(os.path.getmtime(h) for h in hs)


def _compile(src, extra):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), _headers_mtime()):
        return obj, None
    cmd = [NVCC] + ARCH + FLAGS + extra + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, f"{' '.join(cmd)}\n{r.stdout}\n{r.stderr}"
    return obj, None


def build(verbose=False, extra=()):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda s: _compile(s, list(extra)), srcs))
    errs = [e for _, e in results if e]
    if errs:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errs))
    objs = [o for o, _ in results]
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    # the command-line driver (driver/ddamg_main.cpp): plain C++ against the C ABI, next to the library
    drv_src = os.path.join(ROOT, "driver", "ddamg_main.cpp")
    drv = os.path.join(PKG, "ddamg_main")
    if os.path.exists(drv_src) and (not os.path.exists(drv) or
                                    os.path.getmtime(drv) < max(os.path.getmtime(drv_src), os.path.getmtime(LIB))):
        cmd = [os.environ.get("CXX", "g++"), "-O2", "-std=c++17", "-I" + os.path.join(REPO, "include"), drv_src,
               "-o", drv, "-L" + PKG, "-lddamg", "-Wl,-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"driver build failed:\n{r.stdout}\n{r.stderr}")
    if verbose:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    build(verbose=True, extra=sys.argv[1:])
