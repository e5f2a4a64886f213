"""Build recipe for libvortexlab_b200.so (in-tree, sm_100a only).

Compiles the host C++ with g++ and the CUDA translation units with nvcc for
``-gencode arch=compute_100a,code=sm_100a``. The step kernels of every storage format are compiled
with ``-fmad=false`` and the host code with ``-ffp-contract=off``: the compiler fuses no
multiply-add, which keeps the FP64 path bit-identical to the reference solver and makes every
narrow-format kernel round exactly as written (their collision spells its fused multiply-adds out
with intrinsics), so that no two kernels round the same expression differently. Run
``python vortexlab_b200/_build.py``.
"""
from __future__ import annotations

import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# When run as a script, drop this package directory from the import path so that the package's
# own module names (signal.py) cannot shadow the standard library.
sys.path[:] = [p for p in sys.path if os.path.abspath(p or ".") != HERE]

import concurrent.futures as cf  # noqa: E402
import shutil  # noqa: E402
import subprocess  # noqa: E402

CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libvortexlab_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    cand = os.environ.get("NVCC") or os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    if not os.path.exists(cand):
        cand = shutil.which("nvcc") or cand
    return cand


def _cxx():
    return os.environ.get("CXX") or shutil.which("g++") or "g++"


def _sources(defines=()):
    cxx, nvcc = _cxx(), _nvcc()
    inc = ["-I", CSRC, "-I", os.path.join(os.path.dirname(HERE), "include")]
    host_flags = ["-O3", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-Wall"]
    cu_flags = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
                       "--expt-relaxed-constexpr", "-Xptxas", "-v"] + [f"-D{d}" for d in defines]
    jobs = [
        ("vl_host.o", [cxx] + host_flags + inc + ["-c", os.path.join(CSRC, "vl_host.cpp")]),
        ("vl_api.o", [nvcc] + cu_flags + ["-fmad=false"] + inc + ["-c", os.path.join(CSRC, "vl_api.cu")]),
        ("vl_step_f64.o", [nvcc] + cu_flags + ["-fmad=false"] + inc + ["-c", os.path.join(CSRC, "vl_step_f64.cu")]),
        ("vl_step_lp.o", [nvcc] + cu_flags + ["-fmad=false"] + inc + ["-c", os.path.join(CSRC, "vl_step_lp.cu")]),
        ("vl_batch.o", [nvcc] + cu_flags + ["-fmad=false"] + inc + ["-c", os.path.join(CSRC, "vl_batch.cu")]),
        ("vl_nn.o", [nvcc] + cu_flags + inc + ["-c", os.path.join(CSRC, "vl_nn.cu")]),
        ("vl_noalloc.o", [nvcc] + cu_flags + ["-fmad=false"] + inc + ["-c", os.path.join(CSRC, "vl_noalloc.cu")]),
    ]
    return jobs


def _stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def _deps():
    out = []
    for d in (CSRC, os.path.join(os.path.dirname(HERE), "include")):
        for f in os.listdir(d):
            if f.endswith((".cu", ".cuh", ".cpp", ".hpp", ".h")):
                out.append(os.path.join(d, f))
    return out + [os.path.abspath(__file__)]


def build(verbose: bool = False, force: bool = False, out: str = LIB, defines=(), build_dir: str = BUILD) -> str:
    """Compiles every translation unit that is out of date and links the shared library.

    ``defines`` (NAME=VALUE strings) and ``out`` / ``build_dir`` build a variant of the library
    elsewhere, for example with other launch bounds, without touching the default build."""
    global BUILD, LIB
    BUILD, LIB = build_dir, out
    os.makedirs(BUILD, exist_ok=True)
    deps = _deps()
    jobs = _sources(defines)
    todo = [(o, cmd) for o, cmd in jobs if force or _stale(os.path.join(BUILD, o), deps)]

    def run(item):
        obj, cmd = item
        cmd = cmd + ["-o", os.path.join(BUILD, obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        with open(os.path.join(BUILD, obj + ".log"), "w") as f:
            f.write(r.stdout + r.stderr)
        return obj

    if todo:
        with cf.ThreadPoolExecutor(max_workers=len(todo)) as ex:
            for obj in ex.map(run, todo):
                if verbose:
                    print("built", obj)
    if todo or not os.path.exists(LIB):
        objs = [os.path.join(BUILD, o) for o, _ in jobs]
        cmd = [_nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-cudart", "static", "-lpthread", "-ldl", "-lrt"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose:
            print("linked", LIB)
    return LIB


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--out", default=LIB)
    ap.add_argument("--build-dir", default=BUILD)
    ap.add_argument("-D", dest="defines", action="append", default=[])
    a = ap.parse_args()
    build(verbose=True, force=a.force, out=a.out, defines=a.defines, build_dir=a.build_dir)
