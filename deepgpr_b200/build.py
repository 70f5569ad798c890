"""Build recipe of libdeepgpr_b200.so (sm_100a) -- ``python -m deepgpr_b200.build``.

The library is compiled in-tree into ``deepgpr_b200/lib`` with strict IEEE
single precision (``-fmad=false``): the kernels evaluate the reference's
expressions in the reference's order, and FMA contraction would change the
rounding of every update.

The device code is compiled as one unit (no ``-split-compile``): split
compilation optimises groups of device functions separately, and which
kernels share a group changes with any edit of the translation unit, host
code included -- measured here, the same 3D adjoint kernel source ran 80 ms
in one split build and 107 ms in another per gradient sample.  One unit
takes about three minutes on eight cores and gives the same code for the
same kernel source.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OUT = PKG / "lib" / "libdeepgpr_b200.so"
SOURCES = ("fdtd_api.cu",)

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "-fmad=false",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "-shared",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).is_file():
            return cand
    raise FileNotFoundError("nvcc not found")


def stale() -> bool:
    if not OUT.is_file():
        return True
    t = OUT.stat().st_mtime
    deps = [CSRC / f for f in SOURCES] + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h"))
    return any(f.stat().st_mtime > t for f in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile the library if a source is newer than the built file."""
    if not force and not stale():
        return OUT
    OUT.parent.mkdir(parents=True, exist_ok=True)
    tmp = OUT.with_suffix(".so.tmp")
    cmd = [nvcc(), *NVCC_FLAGS, "-o", str(tmp), *(str(CSRC / s) for s in SOURCES)]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed ({res.returncode}):\n{res.stderr[-4000:]}")
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
