"""Build ``libsdot_cuda.so`` in-tree for sm_100a (B200).

    python -m semidiscreteot_b200.build [--force]

nvcc compiles every ``csrc/*.cu`` to an object file (in parallel, under
``csrc/_build/``) and links them into one shared library with CUDA linked
statically, so the library loads on machines without a GPU (it only needs one
to create a context).
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libsdot_cuda.so")
NVCC_FLAGS = [
    "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
    "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr",
]
OBJ_DIR = os.path.join(CSRC, "_build")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def needs_build() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
    deps.append(os.path.join(HERE, "..", "include", "sdot.h"))
    return any(os.path.getmtime(p) > t for p in deps if os.path.exists(p))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return OUT
    from concurrent.futures import ThreadPoolExecutor
    nvcc = os.environ.get("NVCC", "nvcc")
    os.makedirs(OBJ_DIR, exist_ok=True)
    objs = [os.path.join(OBJ_DIR, os.path.basename(src)[:-3] + ".o") for src in sources()]
    cmds = [[nvcc, *NVCC_FLAGS, "-c", "-o", o, src] for src, o in zip(sources(), objs)]
    if verbose:
        for c in cmds:
            print(" ".join(c), file=sys.stderr)
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        rcs = list(ex.map(lambda c: subprocess.run(c).returncode, cmds))
    if any(rcs):
        raise RuntimeError(f"nvcc failed for {[s for s, rc in zip(sources(), rcs) if rc]}")
    link = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC",
            "-o", OUT + ".tmp", *objs]
    if verbose:
        print(" ".join(link), file=sys.stderr)
    subprocess.run(link, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
