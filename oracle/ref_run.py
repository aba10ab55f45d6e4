"""TEST INFRASTRUCTURE ONLY — runs the reference FooskaGPU double-precision CUDA solver built by
oracle/build_ref.py (oracle/_ref/fooska_ref_dp) on a case of ours: writes the case file with
the INPUT field names, the initial conserved state in .neu element order, and parses the
driver's CUDA-event timing.  Used by the stage fixture generator (tests/golden/make_golden.py)
and by the reference arm of bench.py, which times the reference GPU build next to the CPU one.
"""
from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
EXE = HERE / "_ref" / "fooska_ref_dp"

# case fields of ours that the reference's INPUT struct does not have
EXTENSION_KEYS = ("relaxFlag", "hllcEnergyFix", "hllcTieTol", "heatFlux", "limiter", "inletVelFlag", "reserved",
                  "inletVel", "inletStateFlag", "inletP", "inletT", "pressureDatum")


def available() -> bool:
    return EXE.exists() and os.access(EXE, os.X_OK)


def write_case_file(path, c) -> None:
    """key = value lines with the INPUT field names (arrays as name[i])."""
    with open(path, "w") as f:
        for k, _t in type(c)._fields_:
            if k in EXTENSION_KEYS:
                continue
            v = getattr(c, k)
            if hasattr(v, "__len__"):
                for i in range(len(v)):
                    f.write(f"{k}[{i}] = {v[i]!r}\n")
            else:
                f.write(f"{k} = {v!r}\n")


def run(workdir, neu_path, case, U, steps: int, warmup: int = 0, dump: bool = False, timeout: float = 300.0) -> dict:
    """Run `steps` explicitLoop iterations (after `warmup` untimed ones) of the reference solver
    on mesh `neu_path` from state U (nElem x 10, .neu element order).  Returns the report of
    oracle/ref_driver.cu: cells, steps, ms (CUDA events over the timed steps), physical time, dt, status."""
    wd = Path(workdir).resolve()
    wd.mkdir(parents=True, exist_ok=True)
    sh = wd / "sh.neu"
    if Path(neu_path).resolve() != sh:
        if sh.exists() or sh.is_symlink():
            sh.unlink()
        try:
            sh.symlink_to(Path(neu_path).resolve())
        except OSError:
            shutil.copyfile(neu_path, sh)
    np.ascontiguousarray(U, dtype=np.float64).tofile(wd / "ic.bin")
    write_case_file(wd / "case.txt", case)
    cmd = [str(EXE), str(wd), str(wd / "case.txt"), str(wd / "ic.bin"), str(int(steps)), str(int(warmup))]
    if dump:
        cmd.append("--dump")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    (wd / "log.txt").write_text(r.stdout[-20000:] + r.stderr[-20000:])
    if r.returncode != 0 or not (wd / "ref_time.txt").exists():
        raise RuntimeError(f"reference solver exited {r.returncode}: {(r.stdout + r.stderr).strip()[-400:]}")
    t = (wd / "ref_time.txt").read_text().split()
    return {"cells": int(t[0]), "steps": int(t[1]), "ms": float(t[2]), "time": float(t[3]), "dt": float(t[4]),
            "status": " ".join(t[5:])}
