"""Build the in-tree shared libraries.

* ``ablate_b200/lib/libablate_fv.so`` -- the product: sm_100a CUDA kernels behind the C ABI of
  ``include/ablate_fv.h`` (nvcc, ``-gencode arch=compute_100a,code=sm_100a``).
* ``oracle/liborc.so`` -- the CPU oracle used by the tests and the CPU baseline (g++ -O3, OpenMP).

Both are plain ``nvcc``/``g++`` invocations; nothing is JIT-compiled at import time, so the built
files travel with the source tree to the machine that runs them.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "ablate_b200"
CSRC = PKG / "csrc"
LIBDIR = PKG / "lib"
LIB = LIBDIR / "libablate_fv.so"
ORACLE_DIR = ROOT / "oracle"
ORACLE_LIB = ORACLE_DIR / "liborc.so"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "--expt-relaxed-constexpr",
    "-Xptxas", "-warn-spills",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _newer(target: Path, sources: list[Path]) -> bool:
    if not target.exists():
        return False
    t = target.stat().st_mtime
    return all(s.stat().st_mtime <= t for s in sources)


def build_product(force: bool = False, verbose: bool = False) -> Path:
    sources = sorted(CSRC.glob("*.cu"))
    deps = sources + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.hpp")) + [ROOT / "include" / "ablate_fv.h"]
    if not force and _newer(LIB, deps):
        return LIB
    LIBDIR.mkdir(parents=True, exist_ok=True)
    objdir = LIBDIR / "obj"
    objdir.mkdir(exist_ok=True)
    objs = [str(objdir / (src.stem + ".o")) for src in sources]
    cmds = [[_nvcc(), *NVCC_FLAGS, "-I", str(ROOT / "include"), "-c", str(src), "-o", obj] for src, obj in zip(sources, objs)]
    if verbose:
        for cmd in cmds:
            print(" ".join(cmd), flush=True)
    # one nvcc per translation unit, in parallel
    procs = [subprocess.Popen(cmd) for cmd in cmds]
    codes = [p.wait() for p in procs]
    if any(codes):
        raise subprocess.CalledProcessError(max(codes), cmds[codes.index(max(codes))])
    cmd = [_nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", str(LIB), "-lcudart"]
    subprocess.run(cmd, check=True)
    return LIB


def build_oracle(force: bool = False, verbose: bool = False) -> Path:
    sources = [ORACLE_DIR / "oracle.cpp"]
    deps = sources + [ORACLE_DIR / "oracle.h", ROOT / "include" / "ablate_fv.h"]
    if not force and _newer(ORACLE_LIB, deps):
        return ORACLE_LIB
    cmd = ["g++", "-O3", "-march=native", "-fopenmp", "-std=c++17", "-shared", "-fPIC",
           *map(str, sources), "-o", str(ORACLE_LIB)]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return ORACLE_LIB


def build_reference_flux(ref: str | Path | None = None, verbose: bool = False) -> Path | None:
    """Compile the reference's own flux-calculator sources (oracle/Makefile `ref` target) from the
    reference checkout `ref` (default: the ABLATE_REFERENCE environment variable) when one is given and
    present; the result is a checker for the oracle, never a product path."""
    ref = ref or os.environ.get("ABLATE_REFERENCE")
    if not ref:
        return None
    ref = Path(ref)
    if not (ref / "src" / "finiteVolume" / "fluxCalculator" / "ausm.cpp").exists():
        return None
    subprocess.run(["make", "-s", "-C", str(ORACLE_DIR), "ref", f"REF={ref}"], check=True)
    return ORACLE_DIR / "_ref" / "libablate_ref_flux.so"


def main(argv: list[str]) -> int:
    force = "--force" in argv
    verbose = "-v" in argv
    build_oracle(force, verbose)
    build_reference_flux(verbose=verbose)
    build_product(force, verbose)
    print(f"built {LIB} and {ORACLE_LIB}")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
