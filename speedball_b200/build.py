"""Build recipe for libspeedball_cuda.so (sm_100a) — in-tree, no JIT cache.

Each .cu under csrc/ is compiled with nvcc for sm_100a and linked into one
shared library next to this file (static CUDA runtime), so the built .so
travels with the source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "libspeedball_cuda.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
         "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


# Per-source flags. The receiver gathers compare at 1e-3 relative against the FP64
# restatement and are instruction-bound: their divisions and square roots use the
# approximate forms (a few ulp) instead of the IEEE-rounded subroutines.
FILE_FLAGS = {"sb_gather.cu": ["-prec-div=false", "-prec-sqrt=false"]}

VARIANT_SOURCES = ("sb_trace.cu", "sb_refit.cu", "sb_adjoint.cu")  # the sources that read the build macros
WATERTIGHT_LIB = HERE / "libspeedball_cuda_watertight.so"


def sources():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, force: bool = False, defines=(), out: Path | None = None) -> Path:
    """Compile and link. `defines` (e.g. ["SB_PRIMARY_MIN_BLOCKS=3"]) and `out`
    build a variant library elsewhere without touching the default one."""
    build_dir = BUILD if not defines else BUILD / ("v_" + "_".join(d.replace("=", "") for d in defines))
    build_dir.mkdir(parents=True, exist_ok=True)
    lib = out or LIB
    headers = list(CSRC.glob("*.cuh")) + list((HERE.parent / "include").glob("*.h")) + [Path(__file__)]
    objs = []
    dflags = [f"-D{d}" for d in defines]
    for src in sources():
        obj = build_dir / (src.stem + ".o")
        if defines and src.name not in VARIANT_SOURCES:
            obj = BUILD / (src.stem + ".o")  # unaffected by the variant macros: reuse
            if force or _stale(obj, [src] + headers):
                subprocess.run([NVCC, *ARCH, *FLAGS, *FILE_FLAGS.get(src.name, []), "-c", str(src), "-o", str(obj)],
                               check=True)
            objs.append(obj)
            continue
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            cmd = [NVCC, *ARCH, *FLAGS, *FILE_FLAGS.get(src.name, []), *dflags, "-c", str(src), "-o", str(obj)]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _stale(lib, objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", str(lib), *map(str, objs), "-cudart", "static"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return lib


def build_all(verbose: bool = False, force: bool = False) -> list:
    """The default library and the watertight-triangle-test variant."""
    return [build(verbose, force), build(verbose, force, defines=["SB_WATERTIGHT=1"], out=WATERTIGHT_LIB)]


if __name__ == "__main__":
    for lib in build_all(verbose="-v" in sys.argv, force="--force" in sys.argv):
        print(lib)
