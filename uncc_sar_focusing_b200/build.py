"""Build the engine's native libraries in-tree for sm_100a.

    python -m uncc_sar_focusing_b200.build          # incremental
    python -m uncc_sar_focusing_b200.build --force

Outputs (git-ignored, shipped with the tree):
    uncc_sar_focusing_b200/lib/libsarbp.so          C ABI of include/sarbp.h
    uncc_sar_focusing_b200/lib/libsarbp_probes.so   pipe-throughput probes (bench roofline)
    uncc_sar_focusing_b200/lib/libsarbp_compat.so   the reference's C++ symbols
                                                    cuda_focus_SAR_image<float,float>
                                                    and <double,double> (built only
                                                    when SARBP_REFERENCE names the
                                                    reference checkout whose headers
                                                    it compiles against)
Register / shared-memory usage of every kernel goes to _build/ptxas.log.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libsarbp.so")
COMPAT_LIB = os.path.join(LIBDIR, "libsarbp_compat.so")
PROBE_LIB = os.path.join(LIBDIR, "libsarbp_probes.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
# the reference checkout (its headers define the shim's exported signatures);
# the shim is built only when the environment names one
REFERENCE = os.environ.get("SARBP_REFERENCE", "")
REFERENCE_INCLUDE = os.path.join(REFERENCE, "include") if REFERENCE else ""

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden",
                  "-Xptxas", "-v", "--expt-relaxed-constexpr", "-ccbin", "g++"]
SOURCES = ["api.cu", "batch.cu", "range_compress.cu", "bp_mixed.cu", "bp_fp64.cu", "bp_adjoint.cu", "noalloc.cu", "mf.cu",
           "entropy.cu"]
HEADERS = ["bp_common.cuh", "bp_tile.cuh", "sarbp_internal.h", "host_common.h"]


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, log=None):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if log is not None:
        log.append(r.stderr)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} ... {cmd[-1]}")
    return r


def build_lib(force: bool = False, jobs: int = 8) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "sarbp.h")]
    objs, todo = [], []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _newer(o, [s] + hdrs + [__file__]):
            todo.append((s, o))
    logs = []
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        futs = [ex.submit(_run, [NVCC] + CUFLAGS + ["-c", s, "-o", o], logs) for s, o in todo]
        for f in futs:
            f.result()
    if todo:
        with open(os.path.join(BUILD, "ptxas.log"), "a") as fh:
            fh.write("\n".join(logs))
    if force or _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs +
             ["-cudart", "static", "-lcufft", "-Xlinker", f"-rpath,{CUDA_HOME}/lib64"])
    return LIB


def build_probes(force: bool = False) -> str:
    src = os.path.join(CSRC, "probes.cu")
    if force or _newer(PROBE_LIB, [src, __file__]):
        _run([NVCC] + CUFLAGS + ["-shared", "-o", PROBE_LIB, src, "-cudart", "static"])
    return PROBE_LIB


def build_compat(force: bool = False) -> str | None:
    """The reference-facing C++ shim needs the reference's headers (its
    SAR_Aperture / SAR_ImageFormationParameters / CArray types define the
    symbol's signature).  Skipped when they are not present."""
    src = os.path.join(CSRC, "compat", "cuda_focus_sar_image.cpp")
    if not os.path.exists(src) or not REFERENCE_INCLUDE:
        return None
    if not os.path.isdir(REFERENCE_INCLUDE):
        raise RuntimeError(f"SARBP_REFERENCE={REFERENCE} has no include/ directory")
    if force or _newer(COMPAT_LIB, [src, LIB, os.path.join(ROOT, "include", "sarbp.h")]):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-w", "-DCUDAFUNCTION=",
              f"-I{REFERENCE_INCLUDE}", f"-I{REFERENCE_INCLUDE}/third_party", f"-I{ROOT}/include",
              "-o", COMPAT_LIB, src, f"-L{LIBDIR}", "-lsarbp", "-Wl,-rpath,$ORIGIN"])
    return COMPAT_LIB


def build(force: bool = False) -> None:
    if not os.path.exists(NVCC):
        raise RuntimeError(f"nvcc not found at {NVCC}")
    build_lib(force)
    build_probes(force)
    build_compat(force)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--clean", action="store_true")
    args = ap.parse_args()
    if args.clean:
        shutil.rmtree(BUILD, ignore_errors=True)
        shutil.rmtree(LIBDIR, ignore_errors=True)
    build(args.force)
    print(LIB)


if __name__ == "__main__":
    main()
