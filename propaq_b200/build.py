"""Builds libpropaq_cuda.so in-tree for sm_100a (B200) with nvcc.

The library holds every CUDA kernel of the engine and the C ABI declared in
include/propaq_cuda.h.  FMA contraction is disabled on both the device
(-fmad=false) and the host (-ffp-contract=off): the engine must round each
multiply and add separately, exactly as the reference's Rust code does, for
its coefficients to match bit for bit.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB_DIR = PKG / "lib"
LIB = LIB_DIR / "libpropaq_cuda.so"
# The 4-, 8-, 16-, 32- and 64-word kernels are separate translation units
# (they include pq_kernels.cu; the 32- and 64-word ones split again by
# algebra) so that they compile in parallel with the rest; the longest
# compiles come first.
WIDTH_UNITS = ["pq_kernels_w64.cu", "pq_kernels_w64_majorana.cu", "pq_kernels_w32.cu", "pq_kernels_w32_majorana.cu",
               "pq_kernels_w16.cu", "pq_kernels_w4.cu", "pq_kernels_w8.cu"]
SOURCES = WIDTH_UNITS[:4] + ["pq_kernels.cu"] + WIDTH_UNITS[4:] + ["pq_host.cu", "pq_noalloc.cu", "pq_sort.cu"]
HEADERS = ["pq_device.cuh", "pq_kernels.cuh", "pq_tableau.h", "pq_class.cuh", "pq_sort.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-fmad=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
    "-Xptxas", "-v",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build propaq_b200")


def _stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = [CSRC / s for s in SOURCES + HEADERS] + [PKG.parent / "include" / "propaq_cuda.h"]
    return any(d.stat().st_mtime > t for d in deps)


OBJ_DIR = PKG / "_build"  # objects, kept for incremental builds (not shipped with the library)


def _obj(src: str) -> Path:
    return OBJ_DIR / (Path(src).stem + ".o")


# What each translation unit includes (besides itself).
_KERNEL_DEPS = ["pq_device.cuh", "pq_kernels.cuh", "pq_class.cuh"]
DEPS = {
    "pq_kernels.cu": _KERNEL_DEPS,
    **{u: _KERNEL_DEPS + ["pq_kernels.cu"] for u in WIDTH_UNITS},
    "pq_host.cu": ["pq_device.cuh", "pq_kernels.cuh", "pq_sort.cuh", "pq_tableau.h", "../../include/propaq_cuda.h"],
    "pq_noalloc.cu": ["pq_device.cuh", "../../include/propaq_cuda.h"],
    "pq_sort.cu": ["pq_device.cuh", "pq_sort.cuh"],
}


def _obj_stale(src: str) -> bool:
    """An object is rebuilt when it is missing or older than its source or a
    file it includes."""
    obj = _obj(src)
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    deps = [CSRC / src] + [CSRC / h for h in DEPS[src]]
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compiles the engine if any source is newer than the library; only the
    translation units whose inputs changed are recompiled (objects are kept
    beside the library)."""
    if not force and not _stale():
        return LIB
    LIB_DIR.mkdir(exist_ok=True)
    OBJ_DIR.mkdir(exist_ok=True)

    def compile_one(src):
        obj = _obj(src)
        cmd = [nvcc(), *NVCC_FLAGS, "-c", str(CSRC / src), "-o", str(obj)]
        return src, str(obj), subprocess.run(cmd, capture_output=True, text=True)

    todo = [s for s in SOURCES if force or _obj_stale(s)]
    with ThreadPoolExecutor(max_workers=max(1, min(len(todo) or 1, os.cpu_count() or 1))) as pool:
        results = list(pool.map(compile_one, todo))
    for src, obj, r in results:
        if r.returncode != 0:
            Path(obj).unlink(missing_ok=True)
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed on {src}")
        if verbose:
            sys.stderr.write(r.stderr)
    objs = [str(_obj(s)) for s in SOURCES]
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", str(tmp), "-ldl"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc link failed")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
