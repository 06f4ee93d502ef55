"""Build recipe of the CUDA library libow3d.so (sm_100a), in-tree.

    python oceanwave3d-fortran90_b200/build.py [--force] [--jobs N]

Compiles every csrc/*.cu and csrc/*.cpp with nvcc for
``-gencode arch=compute_100a,code=sm_100a`` and links one shared library
next to this file, so that it travels with the source tree.
"""
import argparse
import concurrent.futures as cf
import os
import pathlib
import shutil
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT = HERE / "libow3d.so"
BUILD = HERE / "_build"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xcompiler", "-Wall", "-Xcompiler", "-Wno-unused-function"]


def nvcc():
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found")
    return p


def sources():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def headers():
    return sorted(list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list((HERE.parent / "include").glob("*.h")))


def _needs(obj, src, deps):
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or any(d.stat().st_mtime > t for d in deps)


def compile_one(src, extra=()):
    obj = BUILD / (src.name + ".o")
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stderr}")
    return obj, r.stderr


def build(force=False, jobs=None, verbose=False, extra=()):
    BUILD.mkdir(exist_ok=True)
    srcs = sources()
    deps = headers()
    todo = [s for s in srcs if force or _needs(BUILD / (s.name + ".o"), s, deps)]
    jobs = jobs or min(len(todo) or 1, os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        for obj, err in ex.map(lambda s: compile_one(s, extra), todo):
            if verbose and err.strip():
                print(err, file=sys.stderr)
    objs = [BUILD / (s.name + ".o") for s in srcs]
    if force or not OUT.exists() or any(o.stat().st_mtime > OUT.stat().st_mtime for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(OUT), *map(str, objs), "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true", help="print register/spill usage")
    a = ap.parse_args()
    extra = ["-Xptxas", "-v"] if a.ptxas_v else []
    print(build(force=a.force or a.ptxas_v, jobs=a.jobs, verbose=a.verbose or a.ptxas_v, extra=extra))
