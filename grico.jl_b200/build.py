"""Build libgrico_b200.so in-tree for sm_100a (nvcc, no JIT cache)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "grico_b200", "libgrico_b200.so")
SOURCES = ["host_space.cpp", "grico_plan.cu", "grico_solve.cu", "grico_mg.cu", "grico_cnn.cu", "grico_multi.cu"]
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


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles every source to an object in parallel (one nvcc per source), then links."""
    if not force and not needs_build():
        return OUT
    import tempfile
    from concurrent.futures import ThreadPoolExecutor

    compile_flags = [f for f in FLAGS if f not in ("-shared", "-lcudart")]
    with tempfile.TemporaryDirectory(prefix="grico_build_") as tmp:
        objs = [os.path.join(tmp, os.path.splitext(s)[0] + ".o") for s in SOURCES]
        cmds = [[NVCC, *compile_flags, "-c", os.path.join(CSRC, s), "-o", o] for s, o in zip(SOURCES, objs)]
        if verbose:
            for c in cmds:
                print(" ".join(c), file=sys.stderr)
        with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
            results = list(ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds))
        for c, r in zip(cmds, results):
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise subprocess.CalledProcessError(r.returncode, c)
        link = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", OUT + ".tmp", *objs, "-lcudart"]
        if verbose:
            print(" ".join(link), file=sys.stderr)
        subprocess.run(link, check=True)
        os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
