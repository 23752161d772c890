"""Build the in-tree CUDA library ``libaccint_b200.so`` for sm_100a.

    python build.py            # incremental: recompiles changed sources only
    python build.py --force    # rebuild everything

Each ``csrc/*.cu`` is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` (no fast-math: the FP64
path must stay IEEE) into ``_build/`` and linked into ``libaccint_b200.so`` next
to this file, so the library travels with the source tree.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "libaccint_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
         "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "-I", os.path.join(HERE, "..", "include")]


def _deps(src):
    deps = [src]
    for f in os.listdir(SRC):
        if f.endswith((".h", ".cuh", ".inc")):
            deps.append(os.path.join(SRC, f))
    deps.append(os.path.join(HERE, "..", "include", "libaccint_b200.h"))
    return deps


def _compile(src, force):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if not force and os.path.exists(obj):
        t = os.path.getmtime(obj)
        if all(os.path.getmtime(d) <= t for d in _deps(src)):
            return obj, None
    cmd = [NVCC, *FLAGS, "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, r.stdout + r.stderr
    return obj, None


def build(force=False, verbose=True):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(os.path.join(SRC, f) for f in os.listdir(SRC) if f.endswith(".cu"))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda s: _compile(s, force), srcs))
    errs = [e for _, e in results if e]
    if errs:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errs))
    objs = [o for o, _ in results]
    if force or not os.path.exists(OUT) or any(os.path.getmtime(o) > os.path.getmtime(OUT) for o in objs):
        cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", OUT, *objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    if verbose:
        print("built", OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv)
