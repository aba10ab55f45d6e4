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


# the time step (with its signal-speed residual) and the conservation integral every 20 steps
# (the reference's default is 100): a timed window of 20 steps holds exactly one such step, so
# their cost is inside the number in its natural proportion
TGV_DT_EVERY = 20


def bench_tgv_case(base=None):
    from fooskagpu_b200 import cases
    c = cases.tgv_case(base=base)
    c.adaptDtItr = TGV_DT_EVERY
    return c


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
    case = bench_tgv_case()
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
    # end to end through the C ABI with pinned host buffers: every step uploads the state
    # (fg_set_state_async: copy on the solver's copy stream, device check, scatter), steps, and
    # reads the state back (fg_get_state_async: gather, copy on the solver's download stream); the
    # host waits once at the end after fg_state_join, so the upload of step k+1 (copy stream), the
    # download of step k (download stream) and the kernels overlap
    Uin = torch.empty((nE, 10), dtype=torch.float64, pin_memory=True)
    Uin.numpy()[:] = U0
    Uout = torch.empty((nE, 10), dtype=torch.float64, pin_memory=True)
    e2e_steps = max(3, min(args.steps, 20))
    s.set_state_async(Uin.numpy(), stream=stream.cuda_stream)
    s.step(stream=stream.cuda_stream)
    s.get_state(Uout.numpy(), stream=stream.cuda_stream)
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        s.set_state_async(Uin.numpy(), stream=stream.cuda_stream)
        s.step(stream=stream.cuda_stream)
        s.get_state_async(Uout.numpy(), stream=stream.cuda_stream)
    s.state_join(stream=stream.cuda_stream)   # the last download inside the timed region
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1))
    e2e_val = job_value(world, nE, rk, e2e_steps, e2e_ms)
    s.check_state()
    # the copies alone: upload (+ check + scatter) and download (+ gather) bandwidths
    def copy_gbs(fn, reps=5, ways=1):
        fn()
        s.state_join(stream=stream.cuda_stream)
        torch.cuda.synchronize()
        c0 = torch.cuda.Event(enable_timing=True)
        c1 = torch.cuda.Event(enable_timing=True)
        c0.record(stream)
        for _ in range(reps):
            fn()
        s.state_join(stream=stream.cuda_stream)
        c1.record(stream)
        torch.cuda.synchronize()
        return ways * nE * 80 * reps / (c0.elapsed_time(c1) / 1e3) / 1e9

    def both():
        s.set_state_async(Uin.numpy(), stream=stream.cuda_stream)
        s.get_state_async(Uout.numpy(), stream=stream.cuda_stream)
    h2d_gbs = copy_gbs(lambda: s.set_state_async(Uin.numpy(), stream=stream.cuda_stream))
    d2h_gbs = copy_gbs(lambda: s.get_state(Uout.numpy(), stream=stream.cuda_stream))
    # uploads and downloads back to back without steps: the two directions at once, as the e2e
    # loop needs them (the box's PCIe path may not carry both at full rate)
    duplex_gbs = copy_gbs(both, reps=10, ways=2)
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
    dram = None
    tr_path = ROOT / "profiles" / "flux_traffic.json"
    if tr_path.exists():
        try:
            t = json.loads(tr_path.read_text())
            traffic = t.get("mixed_bytes_per_cell", None)
            if traffic is not None:
                traffic = traffic * nE
            # the DRAM bytes each kernel moves (committed ncu capture, per cell) over its CUDA-event
            # time here: the measured-traffic reading of the flux / gather bar
            dram = {}
            for key, kind in (("k_face<float>", "face"), ("k_gather<float>", "gather"), ("k_grad<float>", "grad")):
                bpc = t.get(f"{kind}_bytes_per_cell")
                src = prof["flux" if kind == "face" else kind]
                if bpc is None or not src["launches"]:
                    continue
                gbs = bpc * nE / (src["ms"] / src["launches"] / 1e3) / 1e9
                dram[key] = {"bytes_per_cell": bpc, "gbs": gbs, "frac": gbs / peak}
        except Exception:
            traffic, dram = None, None
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
                "dt": f"adaptive every {TGV_DT_EVERY} steps (CFL 0.5): the timed steps include the dt and "
                      "conservation steps in proportion"},
        fp64_value=fp64_value, mixed_over_fp64=value / fp64_value,
        e2e={"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": nE * 80, "d2h_bytes_per_step": nE * 80,
             "steps": e2e_steps, "h2d_gbs": h2d_gbs, "d2h_gbs": d2h_gbs, "duplex_gbs": duplex_gbs,
             "api": "fg_set_state_async + fg_step + fg_get_state_async per step, fg_state_join, pinned host buffers"},
        gpu_launches=launches,
        roofline={"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                  "traffic": traffic, "kernel": "k_face<float> + k_gather<float> (face flux, owner-side gather + RK)",
                  "algorithmic_bytes_per_launch": bf * nE, "avg_launch_ms": flux_ms,
                  "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback",
                  "whole_path_frac": whole_frac,
                  "traffic_frac": (traffic / (flux_ms / 1e3) / 1e9 / peak) if traffic else None,
                  "dram_measured": dram},
        kernels={k: {"ms_per_launch": v["ms"] / v["launches"], "launches": v["launches"]} for k, v in prof.items()},
        kernels_fp64={k: {"ms_per_launch": v["ms"] / v["launches"], "launches": v["launches"]} for k, v in prof64.items()},
        clocks=cl,
    )
    # ---------------- mesh pre-processing, host vs GPU (rank 0)
    if rank == 0 and not args.no_mesh_timing:
        out["mesh_preprocess"] = mesh_setup_times(path, per)
    # ---------------- two-phase bubble collapse with the Gibbs relaxation and the learned surrogate
    sg = None
    if not args.no_two_phase:
        out["two_phase"], sg = bubble(args, torch, stream, dev)
    # ---------------- large liquid jet (about 40 M cells)
    if not args.no_jet:
        out["jet"] = jet(args, torch, stream, dev, surrogate=sg)
    if sg is not None:
        sg.close()
    # ---------------- CPU baseline (rank 0, N = 1 only): oracle FP64 on the host cores; its final
    # state is the reference of the accuracy check of both GPU paths
    if rank == 0 and world == 1 and not args.no_cpu:
        out["cpu_baseline"], Uref = cpu_baseline(mesh.view(), case, U0, steps=args.cpu_steps)
        out["accuracy"] = accuracy(mesh, case, U0, Uref, args.cpu_steps, dev, torch, stream)
    return out


def bubble(args, torch, stream, dev):
    """Two-phase water / vapour Rayleigh bubble collapse (the bubble-collapse configurations):
    a ball of radius 10 R0 = 10 mm, about 4 M tets graded toward the centre (meshgen.ball_tets,
    built in memory with the GPU pre-processor), a vapour bubble of R0 = 1 mm at 2340 Pa in water at
    10 MPa (Rayleigh-Plesset pressure field, 298.15 K), stiffened-gas water / vapour constants
    (cases.water_vapour_constants), Gibbs-equilibrium Newton relaxation, HLLC + MUSCL with the
    reference's limiter (below), SSP-RK3.  Three runs of the same `steps` steps from the same state:
      - FP64 with the reference Newton, logging the converged chemical solves (training data);
      - mixed precision with the Newton;
      - mixed precision with the learned surrogate, trained here on the logged states.
    Every step is timed by CUDA events; between steps (outside the timed regions) fg_probe gives
    the vapour volume and the pressure extrema.  The collapse time is the time of the vapour
    volume's minimum; the peak pressure is the largest mixture pressure within 20 steps of it.  The
    FP64 run stops 10 steps after the rebound (the vapour volume, below half its initial value, back
    30 % above its minimum) or after FG_BENCH_BALL_STEPS steps; the two mixed runs take exactly as
    many steps.  Their density and pressure fields are compared with the FP64 run's at steps 100,
    500 and 1000, and so are those of a fourth run, FP64 from the initial state perturbed by a seeded
    relative 1e-10: the collapse is chaotic once the first interface cells cavitate (about step 200
    at this resolution, the maximum pressure jumping from 9e6 to 2e8 Pa), after which FP64 itself
    moves by 10-30 % in pressure L2 under that perturbation, so the tolerance applies at step 100
    and the later steps are reported beside the perturbed FP64 run's divergence.
    The limiter is the reference's (limiter = 0): with the van Albada-type extension the vapour
    partial density of interface cells turns negative within about 60 steps at 0.1 mm spacing,
    in the oracle as on the GPU, at any CFL number tried (0.5, 0.25); the parity tests cover that
    limiter on a reduced ball."""
    from fooskagpu_b200 import cases, meshgen
    from fooskagpu_b200.api import Mesh, Solver, Surrogate
    n = int(os.environ.get("FG_BENCH_BALL_N", "91"))
    steps = int(os.environ.get("FG_BENCH_BALL_STEPS", "1600"))
    t0 = time.perf_counter()
    nm = meshgen.ball_tets(n)
    gen_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    mesh = Mesh.build(nm.nodes, nm.elems, nm.bcs, gpu=True, device=dev)
    pre_s = time.perf_counter() - t0
    del nm
    case = cases.water_vapour_case(limiter=0, adapt_itr=1)
    U0 = cases.bubble_ic(case, mesh.arrays()["cellCenter"], width=1.5 * meshgen.ball_spacing(n, 1e-3))
    nE = mesh.n_elem
    res = {"workload": f"bubble_collapse_water_vapour_ball_{nE}_tets", "cells": nE, "faces": mesh.n_fcs,
           "steps": steps, "mesh": {"generator": f"meshgen.ball_tets({n})", "generate_s": gen_s,
                                    "gpu_preprocess_s": pre_s}}
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)

    compare = (100, 500, 1000)

    def run(prec, nsteps, sg=None, log=0, stop_after_rebound=False, U_init=None):
        s = Solver(mesh, case, precision=prec, device=dev)
        s.set_state(U0 if U_init is None else U_init)
        if log:
            s.relax_log(log)
        if sg is not None:
            s.set_surrogate(sg, 1e-6, 3)
        v0 = s.probe()["vapourVolume"]
        hist, ms, failed, snaps = [], 0.0, None, {}
        chem = fall = iters = relaxed = acc_sg = polish = 0
        vmin, after = v0, -1
        for k in range(nsteps):
            e0.record(stream)
            try:
                s.step(stream=stream.cuda_stream)
            except Exception as e:            # noqa: BLE001 - a flagged state ends the run
                failed = f"step {k}: {e}"
                break
            e1.record(stream)
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
            pr = s.probe(stream=stream.cuda_stream)
            st = s.relax_stats()
            chem += st["nChem"]
            fall += st["nFallback"]
            acc_sg += st["nSurrogate"]
            polish += st["nPolish"]
            iters += st["nIter"]
            relaxed += st["nChem"] + st["nTherm"]
            hist.append((s.time()[1], pr["vapourVolume"], pr["maxPressure"]))
            if k + 1 in compare:
                snaps[k + 1] = s.get_state()
            vmin = min(vmin, pr["vapourVolume"])
            if stop_after_rebound:
                # the first collapse is over once the vapour volume, below half its initial
                # value, has risen 30 % above its minimum; 10 more steps, then stop
                if after < 0 and vmin < 0.5 * v0 and pr["vapourVolume"] > 1.3 * vmin:
                    after = 0
                elif after >= 0:
                    after += 1
                    if after >= 10:
                        break
        try:
            s.check_state()
        except Exception as e:                # noqa: BLE001
            failed = failed or str(e)
        U = s.get_state()
        data = s.relax_log_read(log) if log else None
        s.close()
        done = len(hist)
        # collapse: the vapour volume's minimum (time of the step), and the largest mixture pressure
        # within 20 steps of it
        tc = pk = None
        if done:
            kmin = min(range(done), key=lambda q: hist[q][1])
            if hist[kmin][1] < 0.5 * v0:
                tc = hist[kmin][0]
                pk = max(h[2] for h in hist[max(0, kmin - 20):kmin + 21])
        return dict(ms=ms, steps=done, U=U, snaps=snaps, hist=hist, tc=tc, peak=pk, failed=failed, chem=chem,
                    fall=fall, iters_per_cell=iters / max(1, relaxed), data=data, v0=v0, accepted=acc_sg,
                    polish_per_accepted=polish / acc_sg if acc_sg else None,
                    vmin_ratio=min((h[1] for h in hist), default=v0) / v0)

    def summary(r):
        out = {"value": nE * case.rkSteps * r["steps"] / (r["ms"] / 1e3), "steps_run": r["steps"],
               "collapse_time_s": r["tc"], "peak_pressure_pa": r["peak"],
               "min_vapour_volume_over_initial": r["vmin_ratio"],
               "chem_cells_per_step": r["chem"] / max(1, r["steps"]),
               "newton_iters_per_relaxed_cell": r["iters_per_cell"]}
        if r["failed"]:
            out["stopped"] = r["failed"][:200]
        return out

    r64 = run("fp64", steps, log=12_000_000, stop_after_rebound=True)
    steps = r64["steps"]
    res["steps"] = steps
    X, Y = r64.pop("data")
    res["fp64"] = summary(r64)
    g = Surrogate(device=dev, seed=1)
    t0 = time.perf_counter()
    take = min(len(X), 10_000_000)
    g.set_data(X[:take], Y[:take])
    epochs = 8
    loss = g.train(epochs, batch=4096, lr=2e-3, seed=2)
    res["surrogate_training"] = {"samples": take, "logged": int(len(X)), "epochs": epochs, "final_loss": loss,
                                 "seconds": time.perf_counter() - t0}
    del X, Y
    rm = run("mixed", steps)
    res["mixed"] = summary(rm)
    rs = run("mixed", steps, sg=g)
    res["mixed_surrogate"] = summary(rs)
    # the sensitivity of the FP64 run itself: a seeded relative 1e-10 perturbation of the state
    rng = np.random.default_rng(20261204)
    Up = U0 * (1.0 + 1e-10 * rng.standard_normal(U0.shape))
    Up[:, 0] = np.clip(Up[:, 0], 0.0, 1.0)
    rp = run("fp64", min(steps, max(compare)), U_init=Up)
    res["value"] = res["mixed_surrogate"]["value"]
    res["fp64_value"] = res["fp64"]["value"]
    res["mixed_surrogate_over_fp64"] = res["value"] / res["fp64_value"]
    res["mixed_over_fp64"] = res["mixed"]["value"] / res["fp64_value"]
    res["fallback_rate"] = rs["fall"] / max(1, rs["chem"])
    res["surrogate_accepted_cells"] = rs["accepted"]
    res["polish_steps_per_accepted_cell"] = rs["polish_per_accepted"]
    res["history_fp64"] = {"every": 50, "t_s": [h[0] for h in r64["hist"][::50]],
                           "vapour_volume": [h[1] for h in r64["hist"][::50]],
                           "max_pressure": [h[2] for h in r64["hist"][::50]], "initial_vapour_volume": r64["v0"]}
    # accuracy of the fast paths against the FP64 Newton run: the density / pressure fields at the
    # same steps, the collapse time and the peak pressure; beside them the divergence of the
    # perturbed FP64 run (the problem's own sensitivity)
    steps_cmp = [k for k in compare if k in r64["snaps"]]
    acc = {"compared_at_steps": steps_cmp}
    for key, r in (("mixed", rm), ("mixed_surrogate", rs), ("fp64_perturbed_1e-10", rp)):
        e = {}
        for k in steps_cmp:
            if k in r["snaps"]:
                fe = field_errors(case, r["snaps"][k], r64["snaps"][k])
                e[f"step_{k}"] = {f: fe[f] for f in ("rho", "p") if f in fe}
        if key != "fp64_perturbed_1e-10":
            if r["tc"] is not None and r64["tc"] is not None:
                e["collapse_time_rel_err"] = abs(r["tc"] - r64["tc"]) / r64["tc"]
            if r["peak"] is not None and r64["peak"]:
                e["peak_pressure_rel_err"] = abs(r["peak"] - r64["peak"]) / r64["peak"]
        acc[key] = e
    tol_step = steps_cmp[0] if steps_cmp else None
    acc["tolerance"] = {"rel_l2": 1e-4, "step": tol_step,
                        "note": "rho / p relative L2 against the FP64 Newton run, before the first cavitation; later "
                                "steps are chaotic and reported beside the 1e-10-perturbed FP64 run"}
    if tol_step is not None:
        acc["pass"] = {key: all(acc[key].get(f"step_{tol_step}", {}).get(f, {}).get("rel_l2", 1.0) <= 1e-4
                                for f in ("rho", "p")) for key in ("mixed", "mixed_surrogate")}
    res["accuracy_vs_fp64"] = acc
    mesh.close()
    return res, g


def jet(args, torch, stream, dev, surrogate=None):
    """Large multiphase liquid jet into pressurised gas: a cylinder of 40 D x 100 D (D = 0.2 mm)
    meshed by meshgen.jet_cylinder (prisms in the upstream half, prisms split into tets
    downstream; about 40 M cells at the default n = 228, 100 + 100 layers), a 200 m/s water jet
    through a D-wide inlet into gas at 5 MPa, WALE LES, SSP-RK3 (cases.jet_case).  FP64 and mixed
    precision, and mixed with the learned surrogate attached (the bubble run's, the same fluid);
    each path runs the same `steps` steps after 2 warm-up steps.  Reports the device memory of
    each solver, per-kernel times and achieved GB/s, and the mesh generation and pre-processing
    times (the host pre-processor too with --jet-host-mesh)."""
    from fooskagpu_b200 import cases, meshgen
    from fooskagpu_b200.api import Mesh, Solver
    n = int(os.environ.get("FG_BENCH_JET_N", "228"))
    nzp = int(os.environ.get("FG_BENCH_JET_NZ", "100"))
    steps = args.jet_steps
    t0 = time.perf_counter()
    nm = meshgen.jet_cylinder(n=n, nz_prism=nzp, nz_tet=nzp)
    gen_s = time.perf_counter() - t0
    res = {"workload": "liquid_jet_cylinder_40Dx100D_tet_prism", "steps": steps, "warmup": 2,
           "mesh": {"generator": f"meshgen.jet_cylinder(n={n}, nz_prism={nzp}, nz_tet={nzp})", "generate_s": gen_s}}
    t0 = time.perf_counter()
    mesh = Mesh.build(nm.nodes, nm.elems, nm.bcs, gpu=True, device=dev)
    res["mesh"]["gpu_preprocess_s"] = time.perf_counter() - t0
    if args.jet_host_mesh:
        t0 = time.perf_counter()
        mh = Mesh.build(nm.nodes, nm.elems, nm.bcs, gpu=False)
        res["mesh"]["host_preprocess_s"] = time.perf_counter() - t0
        mh.close()
    del nm
    info = mesh.info
    nE = mesh.n_elem
    res.update(cells=nE, faces=info["nFcs"], tets=info["nTet"], prisms=info["nPrism"])
    case = cases.jet_case()
    U0 = cases.jet_ic(case, mesh.arrays()["cellCenter"])
    nf = (4.0 * info["nTet"] + 5.0 * info["nPrism"]) / nE
    peak, _ = _peaks()
    for key, prec, sg in (("fp64", "fp64", None), ("mixed", "mixed", None), ("mixed_surrogate", "mixed", surrogate)):
        if key == "mixed_surrogate" and sg is None:
            continue
        t0 = time.perf_counter()
        s = Solver(mesh, case, precision=prec, device=dev)
        create_s = time.perf_counter() - t0
        s.set_state(U0)
        if sg is not None:
            s.set_surrogate(sg, 1e-6, 3)
        for _ in range(2):
            s.step(stream=stream.cuda_stream)
        ms = time_steps(s, steps, torch, stream)
        s.profile(True)
        time_steps(s, min(steps, 5), torch, stream)
        prof = s.profile_read()
        s.profile(False)
        st = s.relax_stats()
        s.check_state()
        bg, bf = algorithmic_bytes(nf, fp64=(prec == "fp64"))
        k = {kk: v["ms"] / v["launches"] for kk, v in prof.items()}
        gbs = {}
        if "grad" in k:
            gbs["grad"] = bg * nE / (k["grad"] / 1e3) / 1e9
        if "flux" in k and "gather" in k:
            gbs["face+gather"] = bf * nE / ((k["flux"] + k["gather"]) / 1e3) / 1e9
        res[key] = {"value": nE * case.rkSteps * steps / (ms / 1e3), "ms_per_step": ms / steps,
                    "device_memory_gb": s.memory_bytes() / 1e9, "solver_create_s": create_s,
                    "kernels_ms": k, "achieved_gbs": gbs,
                    "hbm_frac": {kk: v / peak for kk, v in gbs.items()},
                    "relaxation": {"chem_cells": st["nChem"], "fallback": st["nFallback"],
                                   "newton_iters_per_relaxed_cell": st["nIter"] / max(1, st["nChem"] + st["nTherm"]),
                                   "of": "the last step"}}
        s.close()
    res["value"] = res.get("mixed_surrogate", res["mixed"])["value"]
    res["mixed_over_fp64"] = res["mixed"]["value"] / res["fp64"]["value"]
    res["value_over_fp64"] = res["value"] / res["fp64"]["value"]
    res["bytes_model"] = f"per cell-stage: pass G {algorithmic_bytes(nf, False)[0]:.0f} B, pass F " \
                         f"{algorithmic_bytes(nf, False)[1]:.0f} B (mixed; faces per cell {nf:.2f})"
    mesh.close()
    return res


def cpu_baseline(view, case, U, steps=2):
    """FP64 CPU restatement (oracle) on all host threads: `steps` full explicitLoop steps (dt,
    3 RK stages, relaxation, conservation) on the full mesh.  Returns the baseline record and the
    final state (the accuracy check compares the GPU paths with it)."""
    from oracle import oracle_py as O
    th = os.cpu_count() or 1
    O.set_threads(th)
    o = O.Oracle(view, case)
    Uc = U.copy()
    t0 = time.perf_counter()
    for _ in range(steps):
        o.step(Uc)
    dt = time.perf_counter() - t0
    o.close()
    rec = {"value": view.nElem * case.rkSteps * steps / dt, "unit": UNIT, "cores": th, "kind": "port",
           "sample": f"{steps} explicitLoop steps ({case.rkSteps} RK stages + relaxation each, FP64) on the full "
                     f"{view.nElem}-cell mesh, {dt:.1f} s"}
    return rec, Uc


FIELDS = ["alpha", "alpha_rhoL", "alphaG_rhoG", "rho_u", "rho_v", "rho_w", "alpha_rhoL_eL", "alphaG_rhoG_eG",
          "rho_E", "vapour_mass"]


def field_errors(case, U, Uref) -> dict:
    """Relative L2 and Linf error per field of U against Uref (reference order): the ten conserved
    variables (momentum components normalised by the whole momentum field), the mixture density
    and the mixture pressure.  Fields that are zero everywhere in Uref are left out."""
    from fooskagpu_b200 import cases
    out = {}
    mom_l2, mom_inf = np.linalg.norm(Uref[:, 3:6]), np.abs(Uref[:, 3:6]).max()
    cols = [(FIELDS[v], U[:, v], Uref[:, v], v) for v in range(10)]
    cols.append(("rho", U[:, 1] + U[:, 2], Uref[:, 1] + Uref[:, 2], -1))
    cols.append(("p", cases.mixture_pressure(case, U), cases.mixture_pressure(case, Uref), -1))
    for name, a, b, v in cols:
        l2n, infn = (mom_l2, mom_inf) if 3 <= v <= 5 else (np.linalg.norm(b), np.abs(b).max())
        if infn == 0:
            continue
        d = a - b
        out[name] = {"rel_l2": float(np.linalg.norm(d) / l2n), "rel_linf": float(np.abs(d).max() / infn)}
    return out


# tolerances of the accuracy checks (relative L2 / Linf per field against the FP64 oracle): the
# FP64 path differs from the oracle by summation order and FMA contraction, amplified where the
# thermal Newton's absolute stopping tolerance (1e-2 Pa / 1e-2 K) changes a cell's iteration
# count; the mixed path by its FP32 face math (~1e-7 relative per stage)
ACC_TOL = {"fp64": {"rel_l2": 1e-8, "rel_linf": 1e-6}, "mixed": {"rel_l2": 1e-5, "rel_linf": 1e-4}}


def accuracy(mesh, case, U0, Uref, steps, dev, torch, stream) -> dict:
    """Both GPU paths run the oracle's `steps` explicitLoop steps from the same state; per-field
    errors against the oracle's state and the stated tolerance."""
    from fooskagpu_b200.api import Solver
    res = {"steps": steps, "against": "FP64 oracle (CPU restatement of the reference solver), same mesh, same state",
           "tolerance": ACC_TOL}
    for prec in ("fp64", "mixed"):
        s = Solver(mesh, case, precision=prec, device=dev)
        s.set_state(U0)
        for _ in range(steps):
            s.step(stream=stream.cuda_stream)
        U = s.get_state(stream=stream.cuda_stream)
        s.close()
        e = field_errors(case, U, Uref)
        tol = ACC_TOL[prec]
        res[prec] = {"fields": e, "pass": all(x["rel_l2"] <= tol["rel_l2"] and x["rel_linf"] <= tol["rel_linf"]
                                              for x in e.values())}
    return res


def reference_gpu(args):
    """The reference's own double-precision CUDA build (oracle/_ref/fooska_ref_dp, compiled from
    the reference sources by oracle/build_ref.py) on the nearest workload it can express: the
    same 128^3 hex cube, TGV state and case, with slip walls in place of the periodic faces
    (the reference has no periodic boundary), elements in the same shuffled order (the reference
    does not renumber).  Timed by CUDA events that oracle/ref_driver.cu records around its step
    loop (the end event after a device-wide synchronisation).  Nothing of this repository's
    product runs here: the mesh centres for the initial state come from the oracle's mesh
    restatement."""
    from oracle import ref_run
    if not ref_run.available():
        return {"unavailable": "reference GPU build oracle/_ref/fooska_ref_dp not present (built from the reference sources)"}
    from fooskagpu_b200 import cases, meshgen
    from oracle import oracle_mesh
    from oracle.ref_case import reference_defaults
    L = 2 * math.pi
    MESH_DIR.mkdir(parents=True, exist_ok=True)
    path = MESH_DIR / f"tgv{NCELL_SIDE}_slip_shuffled.neu"
    nm = meshgen.box_hexes(NCELL_SIDE, NCELL_SIDE, NCELL_SIDE, L=(L, L, L), shuffle=True, seed=20261203)
    if not path.exists():
        meshgen.write_neu(str(path), nm)
    case = bench_tgv_case(base=reference_defaults())
    U = cases.tgv_ic(case, oracle_mesh.build(nm.nodes, nm.elems, nm.bcs).cellCenter)
    nE = len(U)
    steps, warm = max(1, args.steps), args.warmup
    try:
        rep = ref_run.run(MESH_DIR / "ref_workdir", path, case, U, steps, warm, timeout=900)
    except Exception as e:
        return {"unavailable": f"reference GPU run failed: {str(e)[:300]}"}
    ms = rep["ms"]
    return {"value": nE * case.rkSteps * steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps, "steps": steps,
            "warmup": warm, "cells": nE, "status": rep["status"], "dtype": "f64",
            "workload": f"tgv_les_wale_{NCELL_SIDE}^3_hex, slip walls (no periodic BC in the reference), "
                        "shuffled element order (no renumbering in the reference)",
            "build": "reference DP sources, nvcc 12.9 -gencode sm_100a -rdc, -maxrregcount=128, single-rank MPI/METIS stubs"}


def run_partitioned(args, rank, world, local_rank, dist):
    """--partition: the TGV mesh split into `world` parts (space-filling-curve ranges of the
    device order, fg_mesh_partition), one part per GPU, the halo records of every RK stage moved
    by fooskagpu_b200.halo.TorchHalo over NCCL (device buffers, point to point), dt and the
    conservation integral combined with all-reduce.  The whole job's work is fixed (strong
    scaling); value = all cells x RK stages x steps / the slowest rank's time."""
    import torch
    from fooskagpu_b200 import cases
    from fooskagpu_b200.api import Mesh, Solver
    from fooskagpu_b200.halo import TorchHalo
    torch.cuda.set_device(local_rank)
    dev = local_rank
    path, per = tgv_mesh(rank, world, dist)
    mesh = Mesh.load_neu(path, scale=1.0, periodic=per, gpu=True, device=dev)
    nE = mesh.n_elem
    case = bench_tgv_case()
    U0 = cases.tgv_ic(case, mesh.arrays()["cellCenter"])
    part = mesh.partition(world, rank)
    cg = part.partition_maps()["cell_global"][:part.n_owned]
    stream = torch.cuda.Stream(device=dev)
    s = Solver(part, case, precision="mixed", device=dev)
    halo = TorchHalo(s, part, device=f"cuda:{dev}")
    Up = np.ascontiguousarray(U0[cg])
    s.set_state(Up)
    for _ in range(args.warmup):
        s.step(stream=stream.cuda_stream)
    torch.cuda.synchronize()
    dist.barrier()
    clocks = Clocks(dev)
    clocks.start()
    n0 = s.launch_count()
    ms = rank_max(time_steps(s, args.steps, torch, stream), dist, f"cuda:{dev}")
    cl = clocks.stop()
    launches = s.launch_count() - n0
    value = nE * case.rkSteps * args.steps / (ms / 1e3)
    # end to end: each rank uploads its part, steps and reads it back
    Uin = torch.empty(Up.shape, dtype=torch.float64, pin_memory=True)
    Uin.numpy()[:] = Up
    Uout = torch.empty(Up.shape, dtype=torch.float64, pin_memory=True)
    e2e_steps = max(3, min(args.steps, 20))
    dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        s.set_state_async(Uin.numpy(), stream=stream.cuda_stream)
        s.step(stream=stream.cuda_stream)
        s.get_state_async(Uout.numpy(), stream=stream.cuda_stream)
    s.state_join(stream=stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = rank_max(e0.elapsed_time(e1), dist, f"cuda:{dev}")
    info = part.part_info
    halo_cells = torch.tensor([info["nGhost"]], dtype=torch.float64, device=f"cuda:{dev}")
    dist.all_reduce(halo_cells)
    s.close()
    return dict(
        metric=METRIC, value=value, unit=UNIT, n_gpus=world, steps=args.steps, warmup=args.warmup,
        ms_per_step=ms / args.steps, higher_is_better=True, scaling="strong", vs_baseline=None,
        dtype="fp32 face math + fp64 state/RK (mixed)", data="synthetic",
        config={"workload": f"tgv_les_wale_{NCELL_SIDE}^3_hex_periodic", "cells": nE, "rk_stages": case.rkSteps,
                "parallelism": f"partitioned mesh, {world} parts (space-filling-curve ranges), NCCL halo per stage",
                "ghost_cells_total": int(halo_cells.item()), "halo_exchanges_per_step": case.rkSteps},
        e2e={"value": nE * case.rkSteps * e2e_steps / (e2e_ms / 1e3), "unit": UNIT,
             "h2d_bytes_per_step": nE * 80, "d2h_bytes_per_step": nE * 80, "steps": e2e_steps},
        gpu_launches=launches, clocks=cl)


def run_reference(args):
    """Reference arm.  The reference implements this path only in CUDA, so its CPU arm is the FP64
    C++ restatement of it (oracle), on all host threads, on the same workload: the same mesh
    (built by the oracle's own numpy restatement of the reference's pre-processing), the same
    case and initial state, the same warm-up and timed step counts (full explicitLoop steps).
    Nothing of this repository's product library is loaded.  The line also carries the
    reference's own CUDA build run on the same GPU (reference_gpu)."""
    from fooskagpu_b200 import cases, meshgen
    from oracle import oracle_mesh, oracle_py as O
    from oracle.ref_case import reference_defaults
    L = 2 * math.pi
    nm = meshgen.box_hexes(NCELL_SIDE, NCELL_SIDE, NCELL_SIDE, L=(L, L, L), side_bc={}, shuffle=True, seed=20261203)
    om = oracle_mesh.build(nm.nodes, nm.elems, nm.bcs, periodic=(L, L, L))
    del nm
    case = bench_tgv_case(base=reference_defaults())
    U = cases.tgv_ic(case, om.cellCenter)
    th = os.cpu_count() or 1
    O.set_threads(th)
    o = O.Oracle(om.view(), case)
    Uc = U.copy()
    for _ in range(args.warmup):
        o.step(Uc)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o.step(Uc)
    dt = time.perf_counter() - t0
    o.close()
    val = om.nElem * case.rkSteps * args.steps / dt
    sample = (f"{args.steps} explicitLoop steps ({case.rkSteps} RK stages + relaxation each) after {args.warmup} "
              f"warm-up steps on the full {om.nElem}-cell mesh")
    return dict(
        impl="reference", metric=METRIC, value=val, unit=UNIT, n_gpus=1, steps=args.steps, warmup=args.warmup,
        ms_per_step=dt * 1e3 / args.steps, higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f64",
        data="synthetic",
        config={"workload": f"tgv_les_wale_{NCELL_SIDE}^3_hex_periodic", "cells": om.nElem, "faces": om.nFcs,
                "rk_stages": case.rkSteps,
                "dt": f"adaptive every {TGV_DT_EVERY} steps (CFL 0.5)"},
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
    ap.add_argument("--cpu-steps", type=int, default=2, help="oracle steps of the CPU baseline / accuracy check")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true", help="reference arm: skip timing the reference GPU build")
    ap.add_argument("--no-two-phase", action="store_true", help="skip the two-phase (surrogate) workload")
    ap.add_argument("--no-mesh-timing", action="store_true", help="skip timing the host vs GPU mesh pre-processor")
    ap.add_argument("--no-jet", action="store_true", help="skip the 40 M-cell liquid jet")
    ap.add_argument("--partition", action="store_true",
                    help="one partitioned mesh over the N GPUs (NCCL halo) instead of N replicas (launched "
                         "through torch.distributed.run, N = 1 included)")
    ap.add_argument("--jet-steps", type=int, default=20, help="timed steps per path of the jet (the configuration: 200)")
    ap.add_argument("--jet-host-mesh", action="store_true", help="also time the host pre-processor on the jet mesh")
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
    # --partition needs the process group even on one GPU (one part, no neighbours: the partitioned
    # code path with nothing to exchange)
    if world > 1 or args.partition:
        import datetime
        import torch
        import torch.distributed as D
        torch.cuda.set_device(local_rank)
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        D.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device(f"cuda:{local_rank}"))
        dist = D
    try:
        if args.partition and dist is not None:
            out = run_partitioned(args, rank, world, local_rank, dist)
        else:
            out = run_ours(args, rank, world, local_rank, dist)
        if rank == 0:
            print(json.dumps(out), flush=True)
    finally:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
