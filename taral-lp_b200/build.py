"""Build the engine in-tree: lib/libtaral_pdhg.so (CUDA kernels for sm_100a + host code + C ABI), bin/pdhg (the
CLI) and bin/gather_floor (probe/gather_floor.cu: the random-gather floor the benchmark measures beside the SpMV
phases; a measurement tool, not part of the library).

nvcc cross-compiles without a GPU. Objects are rebuilt only when a source or header is newer.
Usage: python taral-lp_b200/build.py [--force]
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "lib" / "libtaral_pdhg.so"
CLI = PKG / "bin" / "pdhg"
PROBE = PKG / "bin" / "gather_floor"
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "-I", str(ROOT / "include")]
SOURCES = ["engine.cu", "batch.cu", "noalloc.cu", "mlp.cu", "mlp_tc.cu", "verify.cu", "scaling.cpp", "mps.cpp", "solve.cpp"]


def _headers():
    return list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "taral_pdhg.h"]


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _compile(src: str, force: bool) -> Path:
    s = CSRC / src
    o = OBJ / (s.stem + ".o")
    if force or _stale(o, [s] + _headers()):
        lang = [] if s.suffix == ".cu" else ["-x", "c++"]
        cmd = [NVCC, *ARCH, *FLAGS, *lang, "-c", str(s), "-o", str(o)]
        subprocess.run(cmd, check=True)
    return o


def build(force: bool = False) -> Path:
    OBJ.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    CLI.parent.mkdir(exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=4) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), SOURCES))
    if force or _stale(LIB, objs):
        subprocess.run([NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart_static"], check=True)
    cli_o = _compile("cli.cpp", force)
    if force or _stale(CLI, [cli_o, LIB]):
        subprocess.run([NVCC, *ARCH, "-o", str(CLI), str(cli_o), "-L", str(LIB.parent), "-ltaral_pdhg",
                        "-Xlinker", "-rpath,$ORIGIN/../lib"], check=True)
    probe_src = PKG / "probe" / "gather_floor.cu"
    if force or _stale(PROBE, [probe_src]):
        subprocess.run([NVCC, *ARCH, "-O3", "-std=c++17", "-o", str(PROBE), str(probe_src)], check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
    print(LIB)
