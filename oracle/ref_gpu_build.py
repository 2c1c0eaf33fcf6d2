"""Build recipe for the reference's own GPU transport kernel (test and
baseline infrastructure).

The reference keeps its CUDA kernel ``cuVMC`` as a source string inside
``pymopt/voxel_gpu/_cukernel.py:10-229``; CuPy's ``RawKernel`` compiles it at
run time.  CuPy is not installed in this image.  This recipe instead:

1. reads that string from the reference tree, unchanged;
2. writes it to ``oracle/_ref/cuvmc_reference.cu``;
3. compiles it with nvcc for sm_100a, together with ``oracle/ref_gpu_launch.cu``
   (a launcher written for this project), into ``oracle/_ref/libcuvmc_ref.so``.

``oracle/_ref`` is git-ignored: no reference source enters the history.  The
built library travels with the working tree to machines without the
reference.  The nvcc options keep NVRTC's defaults, which CuPy uses: IEEE
divide and square root, FMA contraction on, no fast math.

Only ``tests/`` and the reference legs of ``bench.py`` load the result.  The
product path never does.
"""
from __future__ import annotations

import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT_DIR, "libcuvmc_ref.so")
KERNEL_CU = os.path.join(OUT_DIR, "cuvmc_reference.cu")
LAUNCHER = os.path.join(HERE, "ref_gpu_launch.cu")
KERNEL_PY = os.path.join("pymopt", "voxel_gpu", "_cukernel.py")


def default_reference_root() -> str | None:
    """A pyMonteOpt checkout named by ``PMO_REFERENCE_ROOT``, else a checkout
    called ``reference`` beside this repository, else None (nothing to build;
    a library built earlier is kept)."""
    repo = os.path.dirname(HERE)
    for cand in (os.environ.get("PMO_REFERENCE_ROOT"),
                 os.path.join(os.path.dirname(repo), "reference")):
        if cand and os.path.exists(os.path.join(cand, KERNEL_PY)):
            return cand
    return None


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def extract(reference_root: str) -> str:
    """The CUDA source string of ``cp.RawKernel(r\"\"\"...\"\"\", "cuVMC")``."""
    with open(os.path.join(reference_root, KERNEL_PY), encoding="utf-8") as f:
        text = f.read()
    m = re.search(r'RawKernel\(\s*r"""(.*?)"""\s*,\s*"cuVMC"\s*\)', text, re.S)
    if not m:
        raise RuntimeError(f"cuVMC source string not found in {KERNEL_PY}")
    return m.group(1)


def available() -> bool:
    return os.path.exists(LIB)


def build(force: bool = False, reference_root: str | None = None) -> str | None:
    """Build ``libcuvmc_ref.so``; None when no reference checkout is given or
    found and no library was built before."""
    reference_root = reference_root or default_reference_root()
    if reference_root is None:
        return LIB if available() else None
    src = os.path.join(reference_root, KERNEL_PY)
    if not os.path.exists(src):
        return LIB if available() else None
    stale = (force or not available() or
             any(os.path.getmtime(p) > os.path.getmtime(LIB)
                 for p in (src, LAUNCHER, os.path.abspath(__file__))))
    if not stale:
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    with open(KERNEL_CU, "w", encoding="utf-8") as f:
        f.write(extract(reference_root))
    cmd = [_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo",
           "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-cudart", "static",
           "-I", OUT_DIR, LAUNCHER, "-o", LIB + ".tmp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for the reference kernel:\n{r.stdout}\n{r.stderr}")
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    print(build(force="--force" in sys.argv, reference_root=args[0] if args else None))
