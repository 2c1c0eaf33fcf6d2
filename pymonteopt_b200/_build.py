"""Build the CUDA shared library ``pymonteopt_b200/_lib/libpmo_b200.so``.

Every ``.cu`` file under ``csrc/`` is compiled with nvcc for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``), then linked into one shared
library exporting the C ABI of ``include/pmo_b200.h``.  The CUDA runtime is
linked statically so the library does not depend on which libcudart the
hosting process (PyTorch) loaded.  nvcc cross-compiles, so this runs on a
machine without a GPU.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(REPO, "include")
OUT_DIR = os.path.join(PKG, "_lib")
OBJ_DIR = os.path.join(PKG, "_build")
LIB_NAME = "libpmo_b200.so"
LIB = os.path.join(OUT_DIR, LIB_NAME)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-I", INCLUDE, "-I", CSRC]
# Per-file floating-point flags.  The FP32 product uses the hardware
# approximations for single-precision divide and sqrt; the FP64 oracle build
# keeps every product and sum separately rounded, like the CPU restatement.
PER_FILE = {
    "vmc_plain_f32.cu": ["-ftz=true", "-prec-div=false", "-prec-sqrt=false"],
    "vmc_plain_f64.cu": ["-fmad=false"],
    # the optical bench rounds every product and sum on its own, like NumPy
    "obd.cu": ["-fmad=false"],
}
DEFAULT_FP = ["-ftz=true", "-prec-div=false", "-prec-sqrt=false"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build pymonteopt_b200")


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def _deps():
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    files.append(os.path.join(INCLUDE, "pmo_b200.h"))
    files.append(os.path.abspath(__file__))
    return files


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in _deps())


def _compile(src: str, verbose_ptxas: bool) -> str:
    obj = os.path.join(OBJ_DIR, src[:-3] + ".o")
    cmd = [nvcc(), *ARCH, *COMMON, *PER_FILE.get(src, DEFAULT_FP), "-c",
           os.path.join(CSRC, src), "-o", obj]
    if verbose_ptxas:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose_ptxas:
        sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, verbose_ptxas: bool = False) -> str:
    if not force and not stale():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    srcs = sources()
    with ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose_ptxas), srcs))
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv))
