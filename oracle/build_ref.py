"""TEST INFRASTRUCTURE ONLY — recipe that compiles the reference FooskaGPU double-precision
solver from its own sources (read in place under the reference tree) into oracle/_ref/:

* ``libref_host.so``: the reference physics headers and its kernel-only files
  (thermRlx.cu, chemRlx.cu, computeViscousStresses.cu) compiled by g++ for the host with the
  stubs in refshim/, wrapped by ref_kat.cpp — used for bit-exact known-answer checks of the
  oracle and to generate tests/golden fixtures.
* ``fooska_ref_dp``: the reference CUDA solver (nvcc, sm_100a, -rdc) driven by ref_driver.cu —
  runs only on a GPU; used for stage-level fixtures and to time the reference on the B200.

Nothing from the reference is copied into the repository: sources are compiled where they
lie and the outputs stay in oracle/_ref/ (git-ignored).  Usage:
    python oracle/build_ref.py --ref <reference tree>      (or set FOOSKA_REFERENCE)
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
SHIM = HERE / "refshim"
# the reference tree: --ref, or the FOOSKA_REFERENCE environment variable (no default)
DEFAULT_REF = Path(os.environ["FOOSKA_REFERENCE"]) if os.environ.get("FOOSKA_REFERENCE") else None
DP_SUB = "mulitphase Solver/doublePrecision"

# reference translation units linked into the GPU binary (the driver replaces the others)
GPU_TUS = ["allocateHost", "buildLocalMesh", "chemRlx", "communicate", "computeFaceValues", "computeGrad",
           "computePrimVec", "computeRHS", "computeTimeStep", "computeViscousStresses", "consCalc", "decompose",
           "mainStart", "meshConnectivity", "meshProperties", "partitionConnectivity", "relaxation",
           "startDevice", "thermRlx", "translator", "update"]
HOST_TUS = ["thermRlx", "chemRlx", "computeViscousStresses"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("reference build failed:\n" + " ".join(map(str, cmd)) + "\n" + r.stdout[-4000:] + r.stderr[-4000:])


def dp_dir(ref: Path) -> Path:
    return ref / DP_SUB


def available(ref: Path = DEFAULT_REF) -> bool:
    return ref is not None and (dp_dir(Path(ref)) / "eqos.h").exists()


def build_host(ref: Path = DEFAULT_REF, force: bool = False) -> Path:
    dp = dp_dir(ref)
    OUT.mkdir(exist_ok=True)
    lib = OUT / "libref_host.so"
    srcs = [HERE / "ref_kat.cpp", SHIM / "refhost.h"] + [dp / f"{t}.cu" for t in HOST_TUS]
    if lib.exists() and not force and all(lib.stat().st_mtime > s.stat().st_mtime for s in srcs):
        return lib
    objs = []
    flags = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-include", str(SHIM / "refhost.h"),
             "-I", str(SHIM), "-I", str(dp), "-I", "/usr/local/cuda/include", "-I", str(HERE.parent / "include")]
    for t in HOST_TUS:
        o = OUT / f"host_{t}.o"
        _run(["g++", *flags, "-x", "c++", "-c", str(dp / f"{t}.cu"), "-o", str(o)])
        objs.append(o)
    o = OUT / "host_ref_kat.o"
    _run(["g++", *flags, "-c", str(HERE / "ref_kat.cpp"), "-o", str(o)])
    objs.append(o)
    _run(["g++", "-shared", "-o", str(lib), *map(str, objs)])
    return lib


def build_gpu(ref: Path = DEFAULT_REF, force: bool = False) -> Path:
    dp = dp_dir(ref)
    OUT.mkdir(exist_ok=True)
    exe = OUT / "fooska_ref_dp"
    srcs = [HERE / "ref_driver.cu"] + [dp / f"{t}.cu" for t in GPU_TUS]
    if exe.exists() and not force and all(exe.stat().st_mtime > s.stat().st_mtime for s in srcs):
        return exe
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    objdir = OUT / "gpu_obj"
    objdir.mkdir(exist_ok=True)
    # the reference launches 512-thread blocks; its flux kernel needs ~166 registers, which
    # exceeds the 64K-register file per block on sm_100a ("too many resources requested for
    # launch"), so registers are capped at 128 (= 65536 / 512) as a build flag
    flags = ["-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-rdc=true", "--expt-relaxed-constexpr", "-maxrregcount=128",
             "-Xcompiler", "-fopenmp", "-I", str(SHIM), "-I", str(dp)]
    objs = []
    for t in GPU_TUS:
        o = objdir / f"{t}.o"
        _run([nvcc, *flags, "-c", str(dp / f"{t}.cu"), "-o", str(o)])
        objs.append(o)
    o = objdir / "ref_driver.o"
    _run([nvcc, *flags, "-c", str(HERE / "ref_driver.cu"), "-o", str(o)])
    objs.append(o)
    _run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-rdc=true", "-Xcompiler", "-fopenmp",
          "-o", str(exe), *map(str, objs), "-lgomp"])
    return exe


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=str(DEFAULT_REF) if DEFAULT_REF else None,
                    help="reference tree (default: the FOOSKA_REFERENCE environment variable)")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--host-only", action="store_true")
    a = ap.parse_args()
    if not a.ref or not available(Path(a.ref)):
        print("reference tree not found (give --ref or set FOOSKA_REFERENCE); nothing to build")
        return
    ref = Path(a.ref)
    print(build_host(ref, a.force))
    if not a.host_only:
        print(build_gpu(ref, a.force))


if __name__ == "__main__":
    main()
