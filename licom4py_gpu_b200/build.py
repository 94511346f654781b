"""Build the package's native libraries in-tree.

Two shared libraries are produced under ``licom4py_gpu_b200/lib/``:

* ``libduogrid.so`` -- host C++ duogrid geometry generator (``csrc/duogrid_gen.cpp``),
  compiled with ``-ffp-contract=off`` so its IEEE double arithmetic follows the
  Fortran expression order term by term.
* ``libbt.so`` -- the sm_100a CUDA barotropic solver and its C-ABI
  (``csrc/bt_*.cu``), compiled with ``nvcc -gencode arch=compute_100a,code=sm_100a``.

Run ``python -m licom4py_gpu_b200.build`` (or call :func:`build_all`).  The
build only needs nvcc and g++; no GPU is required.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
INCLUDE = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("CXX", shutil.which("g++") or "g++")

# (source, extra nvcc flags): the float64 kernels and the C-ABI are built
# without FMA contraction so float64 results round like the reference's
# arithmetic; the float32 precision form keeps FMA.
CUDA_SOURCES = [("bt_kernels_f64.cu", ["-fmad=false"]), ("bt_kernels_f32.cu", ["-fmad=true"]),
                ("bt_capi.cu", ["-fmad=false"]), ("bt_reduce.cu", ["-fmad=false"]),
                ("bt_noalloc.cu", ["-fmad=false"]), ("bt_batch_f64.cu", ["-fmad=false"]),
                ("bt_batch_f32.cu", ["-fmad=true"]), ("bt_batch_capi.cu", ["-fmad=false"]),
                ("bt_resident_f64.cu", ["-fmad=false"]), ("bt_resident_f32.cu", ["-fmad=true"])]
CUDA_HEADERS = ["bt_common.cuh", "bt_stencil.cuh", "bt_launch.cuh", "bt_kernels.cuh", "bt_plan.cuh",
                "bt_batch.cuh", "bt_batch_kernels.cuh", "bt_resident.cuh"]
ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _newer(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.exists(s) and os.path.getmtime(s) > t for s in sources)


def _run(cmd: list[str]) -> None:
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(
            "build command failed:\n  " + " ".join(cmd) + "\n" + res.stdout + res.stderr
        )


def build_duogrid(force: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    out = os.path.join(LIBDIR, "libduogrid.so")
    src = os.path.join(CSRC, "duogrid_gen.cpp")
    hdr = os.path.join(INCLUDE, "licom_duogrid.h")
    if force or _newer(out, [src, hdr, __file__]):
        _run([CXX, "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off",
              "-fno-fast-math", "-I", INCLUDE, src, "-o", out + ".tmp"])
        os.replace(out + ".tmp", out)
    return out


def build_bt(force: bool = False, verbose_ptxas: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    out = os.path.join(LIBDIR, "libbt.so")
    srcs = [os.path.join(CSRC, s) for s, _ in CUDA_SOURCES]
    deps = srcs + [os.path.join(CSRC, h) for h in CUDA_HEADERS] + [
        os.path.join(INCLUDE, "licom_bt.h"), __file__]
    if force or _newer(out, deps):
        objdir = os.path.join(HERE, "_build")
        os.makedirs(objdir, exist_ok=True)
        objs = []
        from concurrent.futures import ThreadPoolExecutor

        def compile_one(item):
            src, flags = item
            obj = os.path.join(objdir, os.path.basename(src) + ".o")
            cmd = [NVCC, *ARCH_FLAGS, "-lineinfo", "-O3", "-std=c++17", *flags,
                   "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC, "-c", os.path.join(CSRC, src),
                   "-o", obj]
            if verbose_ptxas:
                cmd.insert(3, "-Xptxas=-v")
            _run(cmd)
            return obj

        with ThreadPoolExecutor(max_workers=len(CUDA_SOURCES)) as ex:
            objs = list(ex.map(compile_one, CUDA_SOURCES))
        _run([NVCC, *ARCH_FLAGS, "--shared", "-Xcompiler", "-fPIC", *objs, "-lcudart", "-o", out + ".tmp"])
        os.replace(out + ".tmp", out)
    return out


def build_all(force: bool = False) -> list[str]:
    return [build_duogrid(force), build_bt(force)]


if __name__ == "__main__":
    for p in build_all(force="--force" in sys.argv):
        print(p)
