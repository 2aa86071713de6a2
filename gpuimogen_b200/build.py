"""In-tree build of the CUDA library for sm_100a.

Produces, next to this file:
  libimogen_b200.so         the product library (nvcc default: multiply-adds contracted)
  libimogen_b200_strict.so  the same sources with -fmad=false -DIB_STRICT_ARITH: every expression
                            is the reference kernels' own, one IEEE operation at a time, so the
                            test suite can compare it bit for bit with the CPU oracle.  The
                            product build instead contracts multiply-adds and replaces a few
                            divisions by reciprocals or comparisons (same mathematics, last-bit
                            differences), checked against the oracle within a tolerance.
  imogen_run                the standalone driver (driver/imogen_run.cpp), host code linked
                            against the product library through its C ABI only.

Usage: python -m gpuimogen_b200.build [--force] [--only product|strict]
"""
import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

SOURCES = [
    "ib_capi.cu",
    "ib_tma.cu",
    "ib_ensemble.cu",
    "ib_mlp.cu",
    "ib_drag_learned.cu",
    "ib_sweep_hllc64.cu",
    "ib_sweep_hllc32.cu",
    "ib_sweep_hll64.cu",
    "ib_xinjin.cu",
    "ib_reduce.cu",
    "ib_boundary.cu",
    "ib_drag.cu",
    "ib_tags.cu",
    "ib_time.cu",
    "ib_sweep_cyl.cu",
    "ib_cylsrc.cu",
]
HEADERS = ["ib_common.cuh", "ib_internal.cuh", "ib_sweep.cuh", "ib_sweep_launch.cuh", "ib_tma.cuh", "ib_bc.cuh",
           "ib_cfl.cuh", "ib_drag.cuh", "ib_tcgen05.cuh", "ib_cyl.cuh"]

BASE_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "-I" + os.path.join(ROOT, "include"),
]

VARIANTS = {
    "product": ("libimogen_b200.so", []),
    "strict": ("libimogen_b200_strict.so", ["-fmad=false", "-DIB_STRICT_ARITH"]),
}


def _newest_input():
    paths = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    paths.append(os.path.join(ROOT, "include", "imogen_b200.h"))
    paths.append(os.path.abspath(__file__))
    return max(os.path.getmtime(p) for p in paths)


# Files whose single-precision arithmetic is only the FP32-flux form: FP32 division and square
# root there use the hardware approximations (FP64 arithmetic is unaffected by these flags).
FP32_FAST = ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"]
PER_FILE = {"ib_sweep_hllc32.cu": FP32_FAST, "ib_ensemble.cu": FP32_FAST}


def _compile(src, obj, extra):
    cmd = [NVCC] + BASE_FLAGS + extra + PER_FILE.get(src, []) + ["-c", os.path.join(CSRC, src), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd), r.stderr))
    return obj


def build_variant(name, force=False, jobs=None):
    libname, extra = VARIANTS[name]
    out = os.path.join(HERE, libname)
    if not force and os.path.exists(out) and os.path.getmtime(out) >= _newest_input():
        return out
    objdir = os.path.join(ROOT, "_build", name)
    os.makedirs(objdir, exist_ok=True)
    objs = [os.path.join(objdir, s.replace(".cu", ".o")) for s in SOURCES]
    jobs = jobs or max(1, min(len(SOURCES), os.cpu_count() or 4))
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        futs = [ex.submit(_compile, s, o, extra) for s, o in zip(SOURCES, objs)]
        for f in futs:
            f.result()
    tmp = out + ".tmp"
    cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", tmp] + objs + ["-lcudart_static"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
    os.replace(tmp, out)
    return out


DRIVER_SRC = os.path.join(HERE, "driver", "imogen_run.cpp")


def build_driver(force=False):
    """The standalone driver: host C++ against the product library (runtime path $ORIGIN)."""
    lib = build_variant("product")
    out = os.path.join(HERE, "imogen_run")
    newest = max(os.path.getmtime(DRIVER_SRC), os.path.getmtime(lib),
                 os.path.getmtime(os.path.join(ROOT, "include", "imogen_b200.h")))
    if not force and os.path.exists(out) and os.path.getmtime(out) >= newest:
        return out
    tmp = out + ".tmp"
    cmd = [NVCC, "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"), DRIVER_SRC, "-o", tmp,
           "-L" + HERE, "-limogen_b200", "-Xlinker", "-rpath", "-Xlinker", "$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("driver build failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
    os.replace(tmp, out)
    return out


def build(force=False, only=None):
    names = [only] if only else list(VARIANTS)
    out = [build_variant(n, force=force) for n in names]
    if only in (None, "product"):
        out.append(build_driver(force=force))
    return out


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--only", choices=list(VARIANTS))
    a = ap.parse_args()
    for p in build(force=a.force, only=a.only):
        print(p)
    sys.exit(0)
