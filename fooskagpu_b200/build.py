"""Build recipe for the native libraries (nvcc / g++ invoked directly, outputs in-tree).

* ``fooskagpu_b200/libfooskagpu.so`` — the product: CUDA kernels for sm_100a + host C++ and
  the C ABI declared in ``include/fooskagpu.h``.
* ``oracle/liboracle.so`` — the CPU FP64 restatement used by tests and the CPU baseline.

Each target is rebuilt only when one of its sources is newer than the output.
"""
from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "fooskagpu_b200"
CSRC = PKG / "csrc"
LIB = PKG / "libfooskagpu.so"
ORACLE_DIR = ROOT / "oracle"
ORACLE_LIB = ORACLE_DIR / "liboracle.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale(out: Path, srcs) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(Path(s).stat().st_mtime > t for s in srcs)


def _run(cmd, cwd=None):
    r = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(map(str, cmd)) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build_product(force: bool = False, verbose: bool = False, out: Path = None, defines=()) -> Path:
    cu = [CSRC / "fg_kernels.cu", CSRC / "fg_relax.cu", CSRC / "fg_solver.cu", CSRC / "fg_noalloc.cu",
          CSRC / "fg_surrogate.cu", CSRC / "fg_mesh_gpu.cu"]
    cpp = [CSRC / "fg_mesh.cpp", CSRC / "fg_partition.cpp"]
    hdr = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [ROOT / "include" / "fooskagpu.h"]
    lib_out = out or LIB
    if not force and not _stale(lib_out, cu + cpp + hdr):
        return lib_out
    objdir = ROOT / "_build" / (lib_out.stem if out else "")
    objdir.mkdir(parents=True, exist_ok=True)
    nvcc = _nvcc()
    objs = []
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-I", str(ROOT / "include")]
    common += [f"-D{d}" for d in defines]
    for s in cu:
        o = objdir / (s.stem + ".o")
        cmd = [nvcc, *ARCH, "-lineinfo", *common, "-c", str(s), "-o", str(o)]
        if s.name == "fg_mesh_gpu.cu":
            # the mesh geometry must round exactly as the host path (no contracted multiply-adds)
            cmd.insert(1, "--fmad=false")
        if s.name == "fg_kernels.cu":
            # the stage kernels' FP32 face math uses fast division / square root / FTZ (the FP32
            # path's tolerance allows ~2 ulp); FP64 code is unaffected by these flags
            cmd.insert(1, "--use_fast_math")
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        out = _run(cmd)
        if verbose and out:
            print(out)
        objs.append(o)
    for s in cpp:
        o = objdir / (s.stem + ".o")
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-I", str(ROOT / "include"), "-c", str(s), "-o", str(o)])
        objs.append(o)
    tmp = lib_out.with_suffix(".so.tmp")
    _run([nvcc, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart"])
    os.replace(tmp, lib_out)
    return lib_out


def build_oracle(force: bool = False) -> Path:
    src = [ORACLE_DIR / "oracle.cpp", ORACLE_DIR / "oracle.h", ROOT / "include" / "fooskagpu.h"]
    if not force and not _stale(ORACLE_LIB, src):
        return ORACLE_LIB
    tmp = ORACLE_LIB.with_suffix(".so.tmp")
    _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
          "-I", str(ROOT / "include"), str(ORACLE_DIR / "oracle.cpp"), "-o", str(tmp)])
    os.replace(tmp, ORACLE_LIB)
    return ORACLE_LIB


def build_all(force: bool = False, verbose: bool = False) -> None:
    build_product(force=force, verbose=verbose)
    build_oracle(force=force)


if __name__ == "__main__":
    import sys
    build_all(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print("built", LIB, ORACLE_LIB)
