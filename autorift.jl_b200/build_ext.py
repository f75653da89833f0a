"""Build libautorift_gpu.so in-tree with nvcc for sm_100a.

The library is plain C ABI (include/autorift_gpu.h) with the CUDA runtime linked statically,
so it loads into Julia (ccall), Python (ctypes) or any other host without torch.
"""

from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
LIB = PKG / "libautorift_gpu.so"

SOURCES = ["ar_track.cu", "ar_corr_tc.cu", "ar_prepare.cu", "ar_multichip.cu", "ar_serve.cu", "ar_capi.cu"]
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = [CSRC / s for s in SOURCES] + list(CSRC.glob("*.cuh")) + [INCLUDE / "autorift_gpu.h"]
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile the CUDA library if any source is newer than it (or `force`)."""
    if not force and not _stale():
        return LIB
    cmd = [nvcc(), *GENCODE, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-O3", "--shared", "-cudart", "static", f"-I{INCLUDE}", f"-I{CSRC}",
           "-o", str(LIB) + ".tmp", *[str(CSRC / s) for s in SOURCES]]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, cwd=str(CSRC), capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + res.stdout + res.stderr)
    os.replace(str(LIB) + ".tmp", LIB)
    if verbose:
        print(res.stdout + res.stderr)
    return LIB


if __name__ == "__main__":
    import sys
    build(force="--force" in sys.argv, verbose=True)
