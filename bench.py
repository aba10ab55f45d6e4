#!/usr/bin/env python3
"""Benchmark of the per-RK-stage explicit residual path on B200.

Workload (default): Taylor-Green vortex LES with WALE on a periodic 2*pi cube of 128^3 hexes
(2,097,152 cells) stored as a Gambit .neu with elements randomly permuted (seeded) and then
renumbered by the loader; SSP-RK3; synthetic initial state (standard TGV at Ma 0.1, Re 1600).
A step is one explicitLoop iteration (3 RK stages + relaxation; dt every 100 steps).

metric  : cell-updates/s = cells x RK stages / s, mixed precision (FP32 reconstruction / HLLC /
          WALE / viscous flux, FP64 state, RK, dt, Newton) — `value`; the FP64 path on the same
          GPU is reported as `fp64_value`.
e2e     : the same metric through the public C ABI with host buffers: every step uploads U from
          pinned host memory (fg_set_state), runs fg_step and downloads U (fg_get_state).
roofline: dominant stage (face flux + owner-side gather + RK), algorithmic bytes per stage / CUDA-event time.

usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import signal
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "cell-updates/s (cells×RK stages/s) at 1 B200, mixed+surrogate vs FP64 plain; %HBM peak"
UNIT = "cell-updates/s"
NCELL_SIDE = int(os.environ.get("FG_BENCH_N", "128"))
MESH_DIR = Path(os.environ.get("FG_BENCH_MESH_DIR", tempfile.gettempdir())) / "fooskagpu_bench"


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def algorithmic_bytes(nf: float, fp64: bool):
    """Compulsory HBM bytes per cell-stage of the two-pass dataflow (tets nf=4, hexes nf=6):
    pass G reads U and writes the limited-gradient record S_G; pass F reads U, U0 (2 of 3 stages),
    S_G and the per-cell face geometry and writes U.
      S_U = 80 B, S_G = 40 values, S_geom = (1 + 7 nf) values (neighbour id, n*A, face offset per
      face + volume); values are 4 B in the mixed path and 8 B in the FP64 path."""
    w = 8 if fp64 else 4
    S_U, S_G, S_geom = 80.0, 40 * w, (1 + 7 * nf) * w
    pass_g = S_U + S_G
    pass_f = S_U + (2.0 / 3.0) * S_U + S_G + S_geom + S_U
    return pass_g, pass_f


# ------------------------------------------------------------------ workload
def mesh_setup_times(path: str, per) -> dict:
    """Seconds to load the workload mesh (parse + connectivity + geometry + ordering) with the
    host pre-processor and with the GPU one (identical arrays)."""
    from fooskagpu_b200.api import Mesh
    out = {}
    for key, gpu in (("host_s", False), ("gpu_s", True)):
        t0 = time.perf_counter()
        m = Mesh.load_neu(path, scale=1.0, periodic=per, gpu=gpu)
        out[key] = time.perf_counter() - t0
        m.close()
    return out


def tgv_mesh(rank: int, world: int, dist):
    from fooskagpu_b200 import meshgen
    L = 2 * math.pi
    MESH_DIR.mkdir(parents=True, exist_ok=True)
    path = MESH_DIR / f"tgv{NCELL_SIDE}_periodic_shuffled.neu"
    if rank == 0 and not path.exists():
        meshgen.write_neu(str(path), meshgen.box_hexes(NCELL_SIDE, NCELL_SIDE, NCELL_SIDE, L=(L, L, L), side_bc={},
                                                       shuffle=True, seed=20261203))
    if dist is not None:
        dist.barrier()
    return str(path), (L, L, L)


class Clocks:
    """nvidia-smi sampler for the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.f = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.send_signal(signal.SIGTERM)
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for k, nm in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(nm)
            except Exception:
                pass
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def rank_max(x: float, dist, device) -> float:
    """Max of a per-rank time over all ranks (replicas: each rank times its own copy of the
    workload; the slowest rank sets the whole job's time)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(world: int, cells: int, stages: int, steps: int, ms_max: float) -> float:
    """Whole-job cell-updates/s of `world` replicas that each ran `steps` steps of `cells` cells
    with `stages` RK stages, the slowest taking ms_max."""
    return world * cells * stages * steps / (ms_max / 1e3)


def time_steps(solver, steps: int, torch, stream):
    """Device time of `steps` fg_step calls on `stream` (CUDA events)."""
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        solver.step(stream=stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def run_ours(args, rank, world, local_rank, dist):
    import torch
    from fooskagpu_b200 import cases
    from fooskagpu_b200.api import Mesh, Solver

    torch.cuda.set_device(local_rank)
    dev = local_rank
    path, per = tgv_mesh(rank, world, dist)
    mesh = Mesh.load_neu(path, scale=1.0, periodic=per, gpu=True, device=dev)
    nE = mesh.n_elem
    info = mesh.info
    case = cases.tgv_case()
    a = mesh.arrays()
    U0 = cases.tgv_ic(case, a["cellCenter"])
    del a
    stream = torch.cuda.Stream(device=dev)
    rk = case.rkSteps
    out = {}

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        return rank_max(x, dist, f"cuda:{dev}")

    # ---------------- mixed path: headline value
    s = Solver(mesh, case, precision="mixed", device=dev)
    s.set_state(U0)
    for _ in range(args.warmup):
        s.step(stream=stream.cuda_stream)
    torch.cuda.synchronize()
    clocks = Clocks(dev)
    n0 = s.launch_count()
    barrier()
    clocks.start()
    ms = time_steps(s, args.steps, torch, stream)
    cl = clocks.stop()
    barrier()
    launches = s.launch_count() - n0
    ms = max_over_ranks(ms)
    value = job_value(world, nE, rk, args.steps, ms)
    # per-kernel CUDA-event times over a second timed region of the same length
    s.profile(True)
    time_steps(s, args.steps, torch, stream)
    prof = s.profile_read()
    s.profile(False)
    mem = s.memory_bytes()
    # end to end through the C ABI with pinned host buffers
    Uh = torch.empty((nE, 10), dtype=torch.float64, pin_memory=True)
    Uh.numpy()[:] = U0
    e2e_steps = max(3, min(args.steps, 20))
    s.set_state(Uh.numpy(), stream=stream.cuda_stream)
    s.step(stream=stream.cuda_stream)
    s.get_state(Uh.numpy(), stream=stream.cuda_stream)
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        s.set_state(Uh.numpy(), stream=stream.cuda_stream)
        s.step(stream=stream.cuda_stream)
        s.get_state(Uh.numpy(), stream=stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1))
    e2e_val = job_value(world, nE, rk, e2e_steps, e2e_ms)
    s.close()

    # ---------------- FP64 path on the same workload
    s64 = Solver(mesh, case, precision="fp64", device=dev)
    s64.set_state(U0)
    for _ in range(max(3, args.warmup // 2)):
        s64.step(stream=stream.cuda_stream)
    k64 = max(3, args.steps // 2)
    barrier()
    ms64 = max_over_ranks(time_steps(s64, k64, torch, stream))
    fp64_value = job_value(world, nE, rk, k64, ms64)
    s64.profile(True)
    time_steps(s64, k64, torch, stream)
    prof64 = s64.profile_read()
    s64.close()

    # ---------------- roofline of the dominant stage (face flux + gather + RK)
    peak, peak_kind = _peaks()
    nf = float(info["maxFaces"])
    bg, bf = algorithmic_bytes(nf, fp64=False)
    bg64, bf64 = algorithmic_bytes(nf, fp64=True)
    # the flux stage is two launches per RK stage: k_face then k_gather (+ RK combination)
    fl, ga = prof["flux"], prof["gather"]
    flux_ms = (fl["ms"] + ga["ms"]) / fl["launches"]
    achieved = bf * nE / (flux_ms / 1e3) / 1e9
    traffic = None
    tr_path = ROOT / "profiles" / "flux_traffic.json"
    if tr_path.exists():
        try:
            t = json.loads(tr_path.read_text())
            traffic = t.get("mixed_bytes_per_cell", None)
            if traffic is not None:
                traffic = traffic * nE
        except Exception:
            traffic = None
    # whole path: per-GPU cell-stages/s x algorithmic bytes per cell-stage (both passes)
    whole_frac = (value / world) * (bg + bf) / 1e9 / peak
    out = dict(
        metric=METRIC, value=value, unit=UNIT, n_gpus=world, steps=args.steps, warmup=args.warmup,
        ms_per_step=ms / args.steps, higher_is_better=True, scaling="weak", vs_baseline=None,
        dtype="fp32 face math + fp64 state/RK (mixed)", data="synthetic",
        config={"workload": f"tgv_les_wale_{NCELL_SIDE}^3_hex_periodic", "cells": nE, "faces": info["nFcs"],
                "rk_stages": rk, "mesh_format": "gambit .neu, elements shuffled (seed 20261203), Morton renumbered",
                "parallelism": "replicas" if world > 1 else "single-gpu",
                "l2": f"inputs larger than L2 (device working set {mem / 1e9:.2f} GB)",
                "dt": "adaptive every 100 steps (CFL 0.5)"},
        fp64_value=fp64_value, mixed_over_fp64=value / fp64_value,
        e2e={"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": nE * 80, "d2h_bytes_per_step": nE * 80,
             "steps": e2e_steps},
        gpu_launches=launches,
        roofline={"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                  "traffic": traffic, "kernel": "k_face<float> + k_gather<float> (face flux, owner-side gather + RK)",
                  "algorithmic_bytes_per_launch": bf * nE, "avg_launch_ms": flux_ms,
                  "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback",
                  "whole_path_frac": whole_frac},
        kernels={k: {"ms_per_launch": v["ms"] / v["launches"], "launches": v["launches"]} for k, v in prof.items()},
        kernels_fp64={k: {"ms_per_launch": v["ms"] / v["launches"], "launches": v["launches"]} for k, v in prof64.items()},
        clocks=cl,
    )
    # ---------------- mesh pre-processing, host vs GPU (rank 0)
    if rank == 0 and not args.no_mesh_timing:
        out["mesh_preprocess"] = mesh_setup_times(path, per)
    # ---------------- two-phase workload with the Gibbs relaxation and the learned surrogate
    if not args.no_two_phase:
        out["two_phase"] = two_phase(args, torch, stream, dev)
    # ---------------- CPU baseline (rank 0, N = 1 only): oracle FP64 on the host cores
    if rank == 0 and world == 1 and not args.no_cpu:
        out["cpu_baseline"] = cpu_baseline(mesh, case, U0, max_stages=args.cpu_stages)
    return out


def two_phase(args, torch, stream, dev):
    """Two-phase workload with the chemical (Gibbs) relaxation active: the reference's own fluid
    constants (DP/buildInput.cu) on a cube of NTP^3 hexes with slip walls and a smoothly
    perturbed liquid/vapour state (about half of the cells need the Gibbs solve each step).
    FP64 Newton-only vs mixed precision with and without the learned surrogate; the surrogate is
    trained inside this run on samples logged from the FP64 run's first steps."""
    from fooskagpu_b200 import cases, meshgen
    from fooskagpu_b200.api import Mesh, Solver, Surrogate
    ntp = int(os.environ.get("FG_BENCH_TP_N", "96"))
    MESH_DIR.mkdir(parents=True, exist_ok=True)
    path = MESH_DIR / f"two_phase_box{ntp}.neu"
    if not path.exists():
        meshgen.write_neu(str(path), meshgen.box_hexes(ntp, ntp, ntp, L=(0.02, 0.02, 0.02)))
    mesh = Mesh.load_neu(str(path), scale=1.0)
    case = cases.reference_case()
    case.rkSteps = 3
    case.hllcTieTol = 1e-4
    U0 = cases.perturbed_two_phase_ic(case, mesh.arrays()["cellCenter"], seed=5, vel=25.0)
    nE = mesh.n_elem
    steps, warm = max(5, min(args.steps, 20)), 3
    res = {"workload": f"two_phase_reference_fluid_{ntp}^3_hex_slip", "cells": nE, "steps": steps, "warmup": warm}

    def run(prec, sg=None, log=0):
        s = Solver(mesh, case, precision=prec, device=dev)
        s.set_state(U0)
        if log:
            s.relax_log(log)
        if sg is not None:
            s.set_surrogate(sg, 1e-6, 3)
        for _ in range(warm):
            s.step(stream=stream.cuda_stream)
        data = s.relax_log_read(log) if log else None
        if log:
            s.relax_log(0)
        ms = time_steps(s, steps, torch, stream)
        st = s.relax_stats()                           # the last timed step's relaxation
        U = s.get_state()
        s.profile(True)
        time_steps(s, 2, torch, stream)
        prof = s.profile_read()
        s.profile(False)
        s.close()
        return ms, prof, st, U, data

    ms64, p64, st64, U64, (X, Y) = run("fp64", log=4_000_000)
    res["fp64_value"] = nE * 3 * steps / (ms64 / 1e3)
    res["fp64_relax_ms"] = p64["relax"]["ms"] / p64["relax"]["launches"]
    g = Surrogate(device=dev, seed=1)
    t0 = time.perf_counter()
    take = min(len(X), 1_000_000)
    g.set_data(X[:take], Y[:take])
    loss = g.train(15, batch=2048, lr=2e-3, seed=2)
    res["surrogate_training"] = {"samples": take, "epochs": 15, "final_loss": loss,
                                 "seconds": time.perf_counter() - t0}
    msm, pm, stm, Um, _ = run("mixed")
    mss, ps, sts, Us, _ = run("mixed", sg=g)
    res["mixed_value"] = nE * 3 * steps / (msm / 1e3)
    res["mixed_relax_ms"] = pm["relax"]["ms"] / pm["relax"]["launches"]
    res["value"] = nE * 3 * steps / (mss / 1e3)
    res["relax_ms"] = ps["relax"]["ms"] / ps["relax"]["launches"]
    res["mixed_surrogate_over_fp64"] = res["value"] / res["fp64_value"]
    res["chem_cells"] = sts["nChem"]
    res["fallback_rate"] = sts["nFallback"] / max(1, sts["nChem"])
    res["newton_iters_per_cell"] = {"fp64_newton": st64["nIter"] / max(1, st64["nChem"] + st64["nTherm"]),
                                    "mixed_newton": stm["nIter"] / max(1, stm["nChem"] + stm["nTherm"]),
                                    "mixed_surrogate": sts["nIter"] / max(1, sts["nChem"] + sts["nTherm"])}
    rho = lambda U: U[:, 1] + U[:, 2]
    res["rho_rel_l2_vs_fp64"] = float(np.linalg.norm(rho(Us) - rho(U64)) / np.linalg.norm(rho(U64)))

    def p_liq(U):
        al = np.clip(U[:, 0], case.avfMin / 100, 1 - case.avfMin / 100)
        r = U[:, 1] / al
        gm = case.gamma[0]
        return (gm - 1) * r * (U[:, 6] / U[:, 1]) - gm * case.pInf[0] - (gm - 1) * case.eta[0] * r

    res["p_rel_l2_vs_fp64"] = float(np.linalg.norm(p_liq(Us) - p_liq(U64)) / np.linalg.norm(p_liq(U64)))
    g.close()
    mesh.close()
    return res


def cpu_baseline(mesh, case, U, max_stages=3):
    """FP64 CPU restatement (oracle) on all host threads: full RK stages on the same mesh."""
    from oracle import oracle_py as O
    th = os.cpu_count() or 1
    O.set_threads(th)
    o = O.Oracle(mesh.view(), case)
    Uc = U.copy()
    o.residual(Uc)  # warm-up (builds the per-cell face lists)
    t0 = time.perf_counter()
    stages = 0
    o.init_rk(Uc)
    while stages < max_stages:
        o.residual(Uc)
        o.update(stages % 3, 1e-4, Uc)
        stages += 1
        if time.perf_counter() - t0 > 60:
            break
    dt = time.perf_counter() - t0
    o.close()
    return {"value": mesh.n_elem * stages / dt, "unit": UNIT, "cores": th, "kind": "port",
            "sample": f"{stages} RK3 stages (residual + update, FP64) on the full {mesh.n_elem}-cell mesh"}


def reference_gpu(args):
    """The reference's own double-precision CUDA build (oracle/_ref/fooska_ref_dp, compiled from
    the reference sources by oracle/build_ref.py) on the nearest workload it can express: the
    same 128^3 hex cube, TGV state and case, with slip walls in place of the periodic faces
    (the reference has no periodic boundary), elements in the same shuffled order (the reference
    does not renumber).  Timed by CUDA events that oracle/ref_driver.cu records around its step
    loop."""
    from oracle import ref_run
    if not ref_run.available():
        return {"unavailable": "reference GPU build oracle/_ref/fooska_ref_dp not present (built from the reference sources)"}
    try:
        import torch
        if not torch.cuda.is_available():
            return {"unavailable": "no GPU visible"}
    except Exception as e:  # pragma: no cover
        return {"unavailable": f"torch: {e}"}
    from fooskagpu_b200 import cases, meshgen
    from fooskagpu_b200.api import Mesh
    L = 2 * math.pi
    MESH_DIR.mkdir(parents=True, exist_ok=True)
    path = MESH_DIR / f"tgv{NCELL_SIDE}_slip_shuffled.neu"
    if not path.exists():
        meshgen.write_neu(str(path), meshgen.box_hexes(NCELL_SIDE, NCELL_SIDE, NCELL_SIDE, L=(L, L, L), shuffle=True,
                                                       seed=20261203))
    mesh = Mesh.load_neu(str(path), scale=1.0)
    case = cases.tgv_case()
    U = cases.tgv_ic(case, mesh.arrays()["cellCenter"])
    nE = mesh.n_elem
    mesh.close()
    steps, warm = max(1, min(args.steps, 20)), 3
    try:
        rep = ref_run.run(MESH_DIR / "ref_workdir", path, case, U, steps, warm, timeout=600)
    except Exception as e:
        return {"unavailable": f"reference GPU run failed: {str(e)[:300]}"}
    ms = rep["ms"]
    return {"value": nE * case.rkSteps * steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps, "steps": steps,
            "warmup": warm, "cells": nE, "status": rep["status"], "dtype": "f64",
            "workload": f"tgv_les_wale_{NCELL_SIDE}^3_hex, slip walls (no periodic BC in the reference), "
                        "shuffled element order (no renumbering in the reference)",
            "build": "reference DP sources, nvcc 12.9 -gencode sm_100a -rdc, -maxrregcount=128, single-rank MPI/METIS stubs"}


def run_reference(args):
    """Reference arm: the reference's path has no CPU implementation of its own, so this times
    the FP64 CPU restatement of it (oracle) with all host threads on the same workload."""
    from fooskagpu_b200 import cases
    from fooskagpu_b200.api import Mesh
    path, per = tgv_mesh(0, 1, None)
    mesh = Mesh.load_neu(path, scale=1.0, periodic=per)
    case = cases.tgv_case()
    U = cases.tgv_ic(case, mesh.arrays()["cellCenter"])
    from oracle import oracle_py as O
    th = os.cpu_count() or 1
    O.set_threads(th)
    o = O.Oracle(mesh.view(), case)
    Uc = U.copy()
    tw = time.perf_counter()
    o.init_rk(Uc)
    for w in range(args.warmup):   # warm-up stages on a copy of the state
        o.residual(Uc)
        o.update(w % 3, 1e-4, Uc)
        if time.perf_counter() - tw > 60:
            break
    Uc = U.copy()
    steps = 0
    cap = max(1, min(args.steps, args.cpu_stages))
    t0 = time.perf_counter()
    o.init_rk(Uc)
    while steps < cap:
        o.residual(Uc)
        o.update(steps % 3, 1e-4, Uc)
        steps += 1
        if time.perf_counter() - t0 > 90:
            break
    dt = time.perf_counter() - t0
    val = mesh.n_elem * steps / dt
    sample = f"{steps} RK3 stages (one stage per step) on the full {mesh.n_elem}-cell mesh"
    return dict(
        impl="reference", metric=METRIC, value=val, unit=UNIT, n_gpus=1, steps=steps, warmup=args.warmup,
        ms_per_step=dt * 1e3 / steps, higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f64",
        data="synthetic",
        config={"workload": f"tgv_les_wale_{NCELL_SIDE}^3_hex_periodic", "cells": mesh.n_elem, "rk_stages": 3},
        cpu_baseline={"kind": "port", "cores": th, "sample": sample, "value": val, "unit": UNIT},
        e2e={"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        note="the reference implements this path only in CUDA; its CPU arm is the FP64 C++ restatement (oracle)",
        reference_gpu=reference_gpu(args) if not args.no_ref_gpu else None,
    )


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-stages", type=int, default=6)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true", help="reference arm: skip timing the reference GPU build")
    ap.add_argument("--no-two-phase", action="store_true", help="skip the two-phase (surrogate) workload")
    ap.add_argument("--no-mesh-timing", action="store_true", help="skip timing the host vs GPU mesh pre-processor")
    ap.add_argument("--n", type=int, default=None, help="cells per side of the TGV cube (default 128)")
    args = ap.parse_args()
    if args.n:
        global NCELL_SIDE
        NCELL_SIDE = args.n
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as D
        torch.cuda.set_device(local_rank)
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        D.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device(f"cuda:{local_rank}"))
        dist = D
    try:
        out = run_ours(args, rank, world, local_rank, dist)
        if rank == 0:
            print(json.dumps(out), flush=True)
    finally:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
