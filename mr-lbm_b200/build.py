"""Build libmrlbm.so (the C-ABI library, include/mrlbm.h) for sm_100a, and
its bounds-check build libmrlbm_check.so (-DMRLBM_BOUNDS_CHECK: the step
kernels check every shared-memory and global access and NaN-poison their
exchange buffers; for tests only).

    python mr-lbm_b200/build.py [--force] [-j N] [--no-check]

Every translation unit under csrc/ is compiled by nvcc for
`-gencode arch=compute_100a,code=sm_100a` in parallel into _build/ (and
_build_check/), then linked.  Objects are rebuilt when any source or header
under csrc/ (or include/) is newer than the object.
"""
import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
VARIANTS = {"": (os.path.join(HERE, "_build"), os.path.join(HERE, "libmrlbm.so"), []),
            "check": (os.path.join(HERE, "_build_check"), os.path.join(HERE, "libmrlbm_check.so"),
                      ["-DMRLBM_BOUNDS_CHECK"])}
BUILD, LIB, _ = VARIANTS[""]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
         "-ccbin", "/usr/bin/g++", "-I", os.path.join(ROOT, "include")]


def _newest(paths):
    return max(os.path.getmtime(p) for p in paths) if paths else 0.0


def build(force=False, jobs=None, verbose=False, extra_flags=(), check=True):
    """Both builds (check=False: the product library only); returns its path."""
    lib = build_variant("", force, jobs, verbose, extra_flags)
    if check:
        build_variant("check", force, jobs, verbose, extra_flags)
    return lib


def build_variant(name, force=False, jobs=None, verbose=False, extra_flags=()):
    BUILD, LIB, vflags = VARIANTS[name]
    extra_flags = list(vflags) + list(extra_flags)
    os.makedirs(BUILD, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    hdr_time = _newest(headers)
    todo = []
    objs = []
    for src in sources:
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src), hdr_time):
            todo.append((src, obj))

    def compile_one(item):
        src, obj = item
        cmd = [NVCC] + ARCH + FLAGS + list(extra_flags) + ["-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, r.stdout, r.stderr))
        return src, r.stderr

    if todo:
        n = jobs or min(len(todo), os.cpu_count() or 4)
        with cf.ThreadPoolExecutor(max_workers=n) as ex:
            for src, err in ex.map(compile_one, todo):
                if verbose:
                    print("compiled", os.path.basename(src), file=sys.stderr)
                    if err.strip():
                        print(err, file=sys.stderr)
    if todo or not os.path.exists(LIB) or os.path.getmtime(LIB) < _newest(objs):
        cmd = [NVCC] + ARCH + ["-shared", "-ccbin", "/usr/bin/g++", "-o", LIB] + objs + ["-lcudart", "-ldl"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (r.stdout, r.stderr))
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("-v", action="store_true")
    ap.add_argument("--no-check", action="store_true", help="skip the bounds-check build")
    args = ap.parse_args()
    print(build(force=args.force, jobs=args.j, verbose=args.v, check=not args.no_check))
