"""Build libmdgpu.so in-tree for sm_100a with nvcc (no JIT cache: the .so travels with the tree)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmdgpu.so")
SOURCES = ["api.cu", "binning.cu", "pairs.cu", "pairs_brick.cu", "integrate.cu", "peaks.cu", "noalloc.cu", "adjoint.cu",
           "traj.cu", "coupling.cu",
           "batch.cu", "phase_space.cu", "rigid.cu"]
HEADERS = ["md_internal.h", "reduce.cuh", "pair_common.cuh", "brick.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xptxas", "-warn-spills",
]
LINK_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-cudart", "static"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "mdgpu.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, out: str = LIB, defines=()) -> str:
    """Compile libmdgpu.so when a source is newer than it (or force): one nvcc per source file in
    parallel, then one link. `out` and `defines` (-D values) serve tuning builds elsewhere.
    Returns the library path."""
    if not force and out == LIB and not defines and not _stale():
        return out
    objdir = os.path.join(os.path.dirname(out), "_build")
    os.makedirs(objdir, exist_ok=True)
    base = [nvcc()] + NVCC_FLAGS + ["-I", os.path.join(ROOT, "include"), "-I", CSRC] + [f"-D{d}" for d in defines]
    if verbose:
        base.insert(1, "-Xptxas=-v")

    def compile_one(f):
        obj = os.path.join(objdir, f.replace(".cu", ".o"))
        cmd = base + ["-c", os.path.join(CSRC, f), "-o", obj]
        res = subprocess.run(cmd, capture_output=True, text=True)
        return f, obj, res

    from concurrent.futures import ThreadPoolExecutor

    with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 4)) as ex:
        results = list(ex.map(compile_one, SOURCES))
    failed = False
    for f, _, res in results:
        if res.returncode != 0 or verbose:
            sys.stderr.write(res.stdout + res.stderr)
        failed |= res.returncode != 0
    if failed:
        raise RuntimeError("nvcc failed to build libmdgpu.so")
    cmd = [nvcc()] + LINK_FLAGS + ["-o", out + ".tmp"] + [obj for _, obj, _ in results]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed to link libmdgpu.so")
    os.replace(out + ".tmp", out)
    return out


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
