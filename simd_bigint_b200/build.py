"""Build recipe for the native library: nvcc straight to an in-tree shared
object, sm_100a only.

    python -m simd_bigint_b200.build            # -> simd_bigint_b200/_lib/libsimd_bigint_b200.so

The library is plain C ABI (include/simd_bigint_b200.h); the CUDA runtime is
linked statically so the .so carries no dependency on torch.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIBDIR = PKG / "_lib"
LIBNAME = "libsimd_bigint_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (cand == "nvcc" or Path(cand).exists()):
            return cand
    return "nvcc"


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def lib_path() -> Path:
    """The in-tree library, or the file named by SBG_LIBRARY (a build made
    elsewhere, e.g. with other -D settings)."""
    env = os.environ.get("SBG_LIBRARY")
    return Path(env) if env else LIBDIR / LIBNAME


def needs_build() -> bool:
    lib = lib_path()
    if not lib.exists():
        return True
    t = lib.stat().st_mtime
    deps = list(CSRC.glob("*")) + list((ROOT / "include").glob("*.h"))
    return any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, extra: list[str] | None = None) -> Path:
    LIBDIR.mkdir(exist_ok=True)
    out = lib_path()
    cmd = [
        nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "--shared",
        "-Xcompiler", "-fPIC,-O3", "-I", str(ROOT / "include"), "-I", str(CSRC),
        "-o", str(out), *[str(s) for s in sources()],
    ]
    if extra:
        cmd[1:1] = extra
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return out


if __name__ == "__main__":
    extra = sys.argv[1:]
    build(verbose=True, extra=extra or None)
