"""Build ``libfeatomic_b200.so`` in-tree with nvcc for sm_100a.

    python -m rascaline_b200.build [--force]

Host C++ and CUDA sources in ``csrc/`` are compiled to objects under
``_build/`` and linked into ``rascaline_b200/libfeatomic_b200.so`` (static
CUDA runtime, so the library loads without a CUDA toolkit on the library
path).  Host code is compiled without FMA contraction so that the cell-list
arithmetic keeps featomic's evaluation order.
"""
import argparse
import concurrent.futures
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBRARY = os.path.join(HERE, "libfeatomic_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# The FP64 drop-in kernels evaluate featomic's expressions in featomic's order
# without contracting a*b+c into FMAs (rustc never contracts), so that sums
# that cancel keep the reference's rounding.
DEVICE = ["-fmad=false"]
# The FP32 forms (dense adjoint, batched molecules, learned surrogate) are not
# held to featomic's rounding: their kernels contract into FMAs.
FMA_SOURCES = ("dense.cu", "dense_mma.cu", "surrogate.cu", "surrogate_mma.cu", "batched_kernels_")
COMMON = [
    "-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-Xcompiler", "-fopenmp",
    f"-I{os.path.join(ROOT, 'include')}", f"-I{CSRC}", "--expt-relaxed-constexpr", "-Wno-deprecated-gpu-targets",
]


def nvcc():
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found")
    return path


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.hpp")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
                  glob.glob(os.path.join(ROOT, "include", "*.h")))


def up_to_date():
    if not os.path.exists(LIBRARY):
        return False
    t = os.path.getmtime(LIBRARY)
    return all(os.path.getmtime(f) <= t for f in sources() + headers() + [__file__])


def _object_current(src, obj):
    """An object is reused when it is newer than its source, every header and
    this script (a header change rebuilds every object)."""
    if not os.path.exists(obj):
        return False
    t = os.path.getmtime(obj)
    return all(os.path.getmtime(f) <= t for f in [src, __file__] + headers())


def _compile(src, verbose, force=True):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if not force and not verbose and _object_current(src, obj):
        return obj, ""
    device = ["-fmad=true"] if os.path.basename(src).startswith(FMA_SOURCES) else DEVICE
    cmd = [nvcc()] + ARCH + device + COMMON + ["-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [nvcc(), "-x", "c++"] + COMMON + ["-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError(f"compilation of {src} failed:\n{' '.join(cmd)}\n{out.stdout}\n{out.stderr}")
    return obj, out.stderr


def build(force=False, verbose=False, jobs=None):
    os.makedirs(BUILD, exist_ok=True)
    # one build at a time: a concurrent build could leave objects compiled
    # against older headers that look up to date
    import fcntl
    with open(os.path.join(BUILD, ".lock"), "w") as lock:
        fcntl.flock(lock, fcntl.LOCK_EX)
        return _build_locked(force, verbose, jobs)


def _build_locked(force, verbose, jobs):
    if not force and up_to_date():
        return LIBRARY
    jobs = jobs or min(8, os.cpu_count() or 1)
    with concurrent.futures.ThreadPoolExecutor(jobs) as pool:
        results = list(pool.map(lambda s: _compile(s, verbose, force), sources()))
    if verbose:
        for _, log in results:
            if log:
                sys.stderr.write(log)
    objects = [r[0] for r in results]
    tmp = LIBRARY + ".tmp"
    cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", tmp] + objects + ["-lgomp"]
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{out.stdout}\n{out.stderr}")
    os.replace(tmp, LIBRARY)
    return LIBRARY


def main():
    parser = argparse.ArgumentParser()
    parser.add_argument("--force", action="store_true")
    parser.add_argument("--verbose", action="store_true", help="print -Xptxas -v resource usage")
    args = parser.parse_args()
    print(build(force=args.force, verbose=args.verbose))


if __name__ == "__main__":
    main()
