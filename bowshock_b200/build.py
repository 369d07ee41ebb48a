"""Builds lib/libbowshock_b200.so from csrc/ with nvcc for sm_100a only.

Run `python -m bowshock_b200.build` (or __graft_entry__.build()). The library
is built in-tree so that it ships with the source tree; nothing is installed.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB_DIR = PKG / "lib"
LIB = LIB_DIR / "libbowshock_b200.so"
OBJ_DIR = PKG / "_build"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC",
    "-Xcompiler", "-fvisibility=hidden",
]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-Wall"]


def nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    path = Path(cuda) / "bin" / "nvcc"
    return str(path) if path.exists() else (shutil.which("nvcc") or "nvcc")


def cxx() -> str:
    return os.environ.get("CXX") or shutil.which("g++") or "g++"


def sources() -> tuple[list[Path], list[Path]]:
    cu = sorted(CSRC.glob("*.cu"))
    cpp = sorted(CSRC.glob("*.cpp")) + sorted((CSRC / "host").glob("*.cpp"))
    return cu, cpp


def _newer(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return False
    t = target.stat().st_mtime
    return all(d.stat().st_mtime <= t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False) -> Path:
    """Compile every source for sm_100a and link the shared library. Skips the
    work when the library is newer than every source and header."""
    cu, cpp = sources()
    headers = list(CSRC.rglob("*.hpp")) + list(CSRC.rglob("*.cuh")) + list((ROOT / "include").glob("*.h"))
    deps = cu + cpp + headers + [Path(__file__)]
    if _newer(LIB, deps) and not ptxas_info:
        return LIB
    OBJ_DIR.mkdir(exist_ok=True)
    LIB_DIR.mkdir(exist_ok=True)
    inc = ["-I", str(ROOT / "include"), "-I", str(CSRC)]
    objs = []
    for src in cu:
        obj = OBJ_DIR / (src.stem + ".cu.o")
        cmd = [nvcc(), *NVCC_FLAGS, *inc, "-c", str(src), "-o", str(obj)]
        if ptxas_info:
            cmd += ["-Xptxas", "-v"]
        _run(cmd, verbose)
        objs.append(obj)
    for src in cpp:
        obj = OBJ_DIR / (src.parent.name + "_" + src.stem + ".o")
        cmd = [cxx(), *CXX_FLAGS,
               "-I", str(Path(os.environ.get("CUDA_HOME", "/usr/local/cuda")) / "include"),
               *inc, "-c", str(src), "-o", str(obj)]
        _run(cmd, verbose)
        objs.append(obj)
    tmp = LIB.with_suffix(".so.tmp")
    _run([nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lpthread"], verbose)
    tmp.replace(LIB)
    return LIB


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed ({r.returncode}): {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout, r.stderr, file=sys.stderr)


if __name__ == "__main__":
    info = "--ptxas" in sys.argv
    print(build(verbose=True, ptxas_info=info))
