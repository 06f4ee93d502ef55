"""Build recipe of the CUDA library libow3d.so (sm_100a), in-tree.

    python oceanwave3d-fortran90_b200/build.py [--force] [--jobs N]

Compiles every csrc/*.cu and csrc/*.cpp with nvcc for
``-gencode arch=compute_100a,code=sm_100a`` and links the objects twice, next
to this file so that both travel with the source tree:
* libow3d.so, the product: it exports exactly the functions that
  include/ow3d.h declares (a linker version script built from the header);
* libow3d_dev.so, the testing build: the same objects with every ow3d_*
  symbol exported, the probes of include/ow3d_test.h included.
"""
import argparse
import re
import concurrent.futures as cf
import os
import pathlib
import shutil
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT = HERE / "libow3d.so"
OUT_DEV = HERE / "libow3d_dev.so"
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
    api = HERE.parent / "include" / "ow3d.h"
    for out, script in ((OUT_DEV, None), (OUT, api)):
        stamp = [o.stat().st_mtime for o in objs] + ([api.stat().st_mtime] if script else [])
        if force or not out.exists() or any(t > out.stat().st_mtime for t in stamp):
            link(out, objs, export_list(script) if script else None)
    return OUT


def api_functions(header):
    """Names of the functions a C header declares (comments removed)."""
    text = re.sub(r"/\*.*?\*/", " ", header.read_text(), flags=re.S)
    text = re.sub(r"//[^\n]*", " ", text)
    return sorted(set(re.findall(r"\b(ow3d_[A-Za-z0-9_]+)\s*\(", text)))


def export_list(header):
    names = api_functions(header)
    if not names:
        raise RuntimeError(f"no functions found in {header}")
    script = BUILD / "ow3d_exports.map"
    script.write_text("{\n  global:\n" + "".join(f"    {n};\n" for n in names) + "  local: *;\n};\n")
    return script


def link(out, objs, version_script=None):
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(out), *map(str, objs), "-lcudart"]
    if version_script:
        cmd += ["-Xlinker", f"--version-script={version_script}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true", help="print register/spill usage")
    a = ap.parse_args()
    extra = ["-Xptxas", "-v"] if a.ptxas_v else []
    print(build(force=a.force or a.ptxas_v, jobs=a.jobs, verbose=a.verbose or a.ptxas_v, extra=extra))
