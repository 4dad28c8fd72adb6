"""Build recipe for libnsph.so (the product's CUDA library).

Compiles every ``csrc/*.cu`` for sm_100a with nvcc into ``libnsph.so`` next to
this file (in-tree, so it travels with the source tree). The CUDA runtime is
linked statically; torch's and this library's runtimes share the device's
primary context, so torch device pointers and streams are valid here.
"""

from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
REPO_DIR = PKG_DIR.parent
CSRC = PKG_DIR / "csrc"
LIB_PATH = PKG_DIR / "libnsph.so"

NVCC_FLAGS = [
    "-gencode",
    "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-O3",
    "-std=c++17",
    "-Xcompiler",
    "-fPIC",
    "-Xcompiler",
    "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
]


def nvcc_path() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libnsph.so")
    return cand


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted((REPO_DIR / "include").glob("*.h"))


def needs_rebuild() -> bool:
    if not LIB_PATH.exists():
        return True
    t = LIB_PATH.stat().st_mtime
    return any(p.stat().st_mtime > t for p in sources() + headers() + [Path(__file__)])


BOUNDS_LIB_PATH = PKG_DIR / "libnsph_bounds.so"


def build(force: bool = False, verbose: bool = False, bounds_check: bool = False) -> Path:
    """Compile libnsph.so if any source is newer than the library.

    bounds_check: compile the bounds-checked build (-DNSPH_BOUNDS_CHECK) into
    libnsph_bounds.so instead; load it by setting NSPH_LIBRARY to its path."""
    out = BOUNDS_LIB_PATH if bounds_check else LIB_PATH
    if not force and not bounds_check and not needs_rebuild():
        return out
    tmp = out.with_suffix(".so.tmp")
    cmd = [nvcc_path(), *NVCC_FLAGS, f"-I{REPO_DIR / 'include'}", "-shared", "-o", str(tmp)]
    if bounds_check:
        cmd.append("-DNSPH_BOUNDS_CHECK")
    cmd += [str(s) for s in sources()]
    if verbose:
        print(" ".join(cmd))
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed ({res.returncode}):\n{res.stdout}\n{res.stderr}")
    os.replace(tmp, out)
    return out


if __name__ == "__main__":
    import sys

    print(build(force=True, verbose=True, bounds_check="--bounds-check" in sys.argv[1:]))
