"""Build recipe for libbugdef.so (sm_100a) -- compiled in-tree with nvcc.

    python -m bug_defense_b200.build          # builds bug_defense_b200/_native/libbugdef.so

The library is plain CUDA C++ behind the C ABI in include/bugdef.h; no torch headers.
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT_DIR = PKG / "_native"
LIB = OUT_DIR / "libbugdef.so"
SOURCES = ["abi.cu", "tmap.cu", "mc.cu", "stencil.cu", "plume.cu", "phase.cu", "engine.cu", "record.cu", "conv3d.cu", "unet.cu",
           "selftest.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libbugdef.so")
    return exe


def _digest(extra_flags) -> str:
    h = hashlib.sha256()
    for name in sorted(os.listdir(CSRC)):
        h.update(name.encode())
        h.update((CSRC / name).read_bytes())
    h.update((ROOT / "include" / "bugdef.h").read_bytes())
    h.update(" ".join(extra_flags).encode())
    return h.hexdigest()[:16]


def build(force: bool = False, verbose: bool = False, extra_flags=(), out: Path | None = None) -> Path:
    """Compile every .cu source for sm_100a and link libbugdef.so (skipped when up to date)."""
    lib = Path(out) if out is not None else LIB
    lib.parent.mkdir(parents=True, exist_ok=True)
    stamp = lib.with_suffix(".stamp")
    dig = _digest(list(extra_flags))
    if not force and lib.exists() and stamp.exists() and stamp.read_text() == dig:
        return lib
    srcs = [str(CSRC / s) for s in SOURCES if (CSRC / s).exists()]
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-fvisibility=hidden", "-I", str(ROOT / "include"), "-I", str(CSRC),
           "--expt-relaxed-constexpr", *extra_flags, "-o", str(lib) + ".tmp", *srcs]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed ({res.returncode}):\n{res.stderr}")
    if verbose and res.stderr:
        print(res.stderr, file=sys.stderr)
    os.replace(str(lib) + ".tmp", lib)
    stamp.write_text(dig)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
