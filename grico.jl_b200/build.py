"""Build libgrico_b200.so in-tree for sm_100a (nvcc, no JIT cache)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "grico_b200", "libgrico_b200.so")
SOURCES = ["host_space.cpp", "grico_plan.cu", "grico_solve.cu", "grico_mg.cu", "grico_cnn.cu", "grico_multi.cu", "grico_shard.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
         "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "-shared", "-lcudart"]


def needs_build() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    for name in os.listdir(CSRC):
        if os.path.getmtime(os.path.join(CSRC, name)) > t:
            return True
    hdr = os.path.join(HERE, "..", "include", "grico_b200.h")
    return os.path.getmtime(hdr) > t


BUILD_DIR = os.path.join(HERE, "_build")


def _headers_mtime() -> float:
    paths = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    paths.append(os.path.join(HERE, "..", "include", "grico_b200.h"))
    return max(os.path.getmtime(p) for p in paths)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles the sources whose object is older than the source or any header (one nvcc per
    source, in parallel; objects kept in grico.jl_b200/_build), then links."""
    if not force and not needs_build():
        return OUT
    from concurrent.futures import ThreadPoolExecutor

    os.makedirs(BUILD_DIR, exist_ok=True)
    compile_flags = [f for f in FLAGS if f not in ("-shared", "-lcudart")]
    hdr = _headers_mtime()
    objs = [os.path.join(BUILD_DIR, os.path.splitext(s)[0] + ".o") for s in SOURCES]
    cmds = []
    for src, obj in zip(SOURCES, objs):
        path = os.path.join(CSRC, src)
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(path), hdr):
            cmds.append([NVCC, *compile_flags, "-c", path, "-o", obj + ".tmp"])
    if verbose:
        for c in cmds:
            print(" ".join(c), file=sys.stderr)
    if cmds:
        with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
            results = list(ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds))
        for c, r in zip(cmds, results):
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise subprocess.CalledProcessError(r.returncode, c)
        for c in cmds:
            os.replace(c[-1], c[-1][:-len(".tmp")])
    link = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", OUT + ".tmp", *objs, "-lcudart"]
    if verbose:
        print(" ".join(link), file=sys.stderr)
    subprocess.run(link, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
