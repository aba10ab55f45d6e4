"""Generate the known-answer fixtures in tests/golden/ from the reference itself.

* ``kat_physics.npz`` — seeded random inputs and the outputs of the reference's own device
  functions (eqos, cons2prim, prim2cons, waveSpeeds, bcValues, starRegion, flux, fluxSource,
  computeViscousStresses on one face, thermalRlx and chemRlx on one cell), obtained by running
  oracle/_ref/libref_host.so (the reference sources compiled for the host by
  oracle/build_ref.py).  Needs the reference tree; run here, commit the .npz.

* ``stage_*.npz`` — stage-level fixtures produced by the reference CUDA binary
  (oracle/_ref/fooska_ref_dp) on a B200, see ``run_stage_fixtures`` (run on a machine with the
  GPU into <outdir>, then packed here by ``collect``).

* ``long_tgv16_slip.npz`` — the reference CUDA binary's state after 10, 30 and 60 full steps of a
  16^3 slip-wall Taylor-Green vortex (``long_spec``), for the long-run comparison of the oracle and
  the device path.

usage: python tests/golden/make_golden.py kat
       python tests/golden/make_golden.py stage <outdir>     (GPU box)
       python tests/golden/make_golden.py collect <outdir>   (pack the GPU run into stage_*.npz)
       python tests/golden/make_golden.py long <outdir>      (GPU box)
       python tests/golden/make_golden.py collect_long <outdir>
"""
from __future__ import annotations

import ctypes as C
import json
import os
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from fooskagpu_b200 import cases, meshgen  # noqa: E402

HERE = Path(__file__).resolve().parent
PD = C.POINTER(C.c_double)
SEED = 20261203


def _p(a):
    return a.ctypes.data_as(PD)


def _cases():
    """Parameter sets covered by the fixtures: the reference's own constants, and the
    single-phase ideal gas used for the Sod / TGV configurations."""
    ref = cases.reference_case()
    ref_nowood = cases.reference_case()
    ref_nowood.woodsFlag = 0
    ig = cases.ideal_gas_case(mu=6.25e-4)
    return {"reference": ref, "reference_nowood": ref_nowood, "ideal_gas": ig}


def case_to_dict(c) -> dict:
    out = {}
    for k, t in type(c)._fields_:
        v = getattr(c, k)
        out[k] = list(v) if hasattr(v, "__len__") else v
    return out


def _unit(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def _frame(n):
    a = np.where(np.abs(n[:, :1]) < 0.9, np.array([[1.0, 0, 0]]), np.array([[0, 1.0, 0]]))
    t1 = np.cross(n, a)
    t1 /= np.linalg.norm(t1, axis=1, keepdims=True)
    t2 = np.cross(n, t1)
    return t1, t2


def _states(case, rng, n, vel):
    centres = rng.uniform(-1, 1, size=(n, 3))
    U = cases.perturbed_two_phase_ic(case, centres, seed=int(rng.integers(1 << 30)), vel=vel)
    return U


def make_kat(n=400):
    R = C.CDLL(str(ROOT / "oracle" / "_ref" / "libref_host.so"))
    out = {}
    meta = {}
    for cname, case in _cases().items():
        rng = np.random.default_rng(SEED + len(cname))
        vel = 30.0 if cname.startswith("reference") else 0.3
        if cname == "ideal_gas":
            cen = rng.uniform(0, 6.28, size=(n, 3))
            UL = cases.tgv_ic(case, cen)
            UR = cases.tgv_ic(case, cen + rng.normal(scale=0.3, size=(n, 3)))
        else:
            UL = _states(case, rng, n, vel)
            UR = _states(case, rng, n, vel)
        nrm = _unit(rng, n)
        t1, t2 = _frame(nrm)
        sL = np.zeros((n, 10)); sR = np.zeros((n, 10))
        for i in range(n):
            R.refkat_cons2prim(C.byref(case), _p(UL[i].copy()), _p(sL[i]))
            R.refkat_cons2prim(C.byref(case), _p(UR[i].copy()), _p(sR[i]))
        p2c = np.zeros((n, 10))
        for i in range(n):
            R.refkat_prim2cons(C.byref(case), _p(sL[i].copy()), _p(p2c[i]))
        ws = np.zeros((n, 9))
        for i in range(n):
            cc = np.zeros(3); ul = np.zeros(3); ur = np.zeros(3)
            R.refkat_wave_speeds(C.byref(case), _p(nrm[i].copy()), _p(t1[i].copy()), _p(t2[i].copy()),
                                 _p(sL[i].copy()), _p(sR[i].copy()), _p(cc), _p(ul), _p(ur))
            ws[i] = np.concatenate([cc, ul, ur])
        bcv = np.zeros((n, 5, 10))
        for i in range(n):
            for b in range(1, 6):
                s = sL[i].copy()
                R.refkat_bc_values(C.byref(case), _p(nrm[i].copy()), _p(t1[i].copy()), _p(t2[i].copy()), _p(s), b)
                bcv[i, b - 1] = s
        # star region of the left state with the computed wave speeds
        star = np.zeros((n, 23))
        for i in range(n):
            SK, SS = ws[i, 0], ws[i, 1]
            R.refkat_star_region(C.byref(case), _p(sL[i].copy()), _p(ws[i, 3:6].copy()), C.c_double(SK), C.c_double(SS),
                                 _p(nrm[i].copy()), _p(t1[i].copy()), _p(t2[i].copy()), _p(p2c[i].copy()), _p(star[i]))
        unc = rng.normal(scale=vel, size=(n, 3))
        are = rng.uniform(1e4, 1e6, size=(n, 2))
        fl = np.zeros((n, 10))
        for i in range(n):
            R.refkat_flux(C.byref(case), _p(sL[i].copy()), _p(nrm[i].copy()), _p(unc[i].copy()), C.c_double(are[i, 0]),
                          C.c_double(are[i, 1]), _p(fl[i]))
        fs = np.zeros((n, 6))
        for i in range(n):
            R.refkat_flux_source(C.byref(case), _p(unc[i].copy()), _p(UL[i].copy()), _p(UR[i].copy()), _p(nrm[i].copy()), _p(fs[i]))
        # viscous face: random gradients, volumes, areas; interior and boundary
        gO = rng.normal(scale=vel * 50, size=(n, 30))
        gN = rng.normal(scale=vel * 50, size=(n, 30))
        vol = rng.uniform(1e-9, 1e-6, size=(n, 2))
        area = rng.uniform(1e-6, 1e-4, size=n)
        bcs = rng.integers(0, 6, size=n)
        pf = np.concatenate([sL, sR], axis=1)
        vis = np.zeros((n, 20))
        vcase = C.pointer(type(case).from_buffer_copy(case))
        vcase.contents.viscFlag = 1
        vcase.contents.turbulence = 1
        for i in range(n):
            R.refkat_viscous_face(vcase, _p(pf[i].copy()), _p(gO[i].copy()), _p(gN[i].copy()), _p(nrm[i].copy()),
                                  C.c_double(area[i]), _p(vol[i].copy()), int(bcs[i]), _p(vis[i]))
        th = UL.copy()
        ch = UL.copy()
        for i in range(n):
            R.refkat_therm_cell(C.byref(case), _p(th[i]))
            R.refkat_chem_cell(C.byref(case), _p(ch[i]))
        out.update({f"{cname}/{k}": v for k, v in dict(
            UL=UL, UR=UR, n=nrm, t1=t1, t2=t2, solL=sL, solR=sR, prim2cons=p2c, wave=ws, bc=bcv, star=star,
            unc=unc, are=are, flux=fl, fsrc=fs, gO=gO, gN=gN, vol=vol, area=area, bcs=bcs, visc=vis,
            therm=th, chem=ch).items()})
        meta[cname] = case_to_dict(case)
    np.savez_compressed(HERE / "kat_physics.npz", **out)
    (HERE / "kat_cases.json").write_text(json.dumps(meta, indent=1))
    print("wrote", HERE / "kat_physics.npz")


# ------------------------------------------------------------------ stage fixtures (reference CUDA binary)
def stage_specs():
    """Small meshes and cases for the stage-level fixtures: every element type, every
    boundary code, inviscid and WALE-viscous, Euler and RK3, the reference's own constants
    (two-phase, chemical relaxation on) and the single-phase ideal gas."""
    specs = []
    sides_all = {"x0": "inlet", "x1": "outlet", "y0": "wall", "y1": "slip", "z0": "symmetry", "z1": "slip"}
    specs.append(dict(name="tet_ref", mesh=("tets", 6, 3, 3, (0.006, 0.003, 0.003), (-0.003, 0, 0)),
                      sides=sides_all, case="reference", ic="perturbed", rk=1, steps=3))
    specs.append(dict(name="mixed_ref_rk3", mesh=("mixed", 4, 4, 3, (0.004, 0.004, 0.003), (0, 0, 0)),
                      sides={s: "slip" for s in ("x0", "x1", "y0", "y1", "z0", "z1")}, case="reference",
                      ic="perturbed", rk=3, steps=2))
    specs.append(dict(name="hex_ig_visc", mesh=("hexes", 5, 4, 4, (1.0, 0.8, 0.8), (0, 0, 0)),
                      sides={s: "wall" for s in ("x0", "x1", "y0", "y1", "z0", "z1")}, case="ideal_visc",
                      ic="tgv", rk=3, steps=3))
    specs.append(dict(name="tet_sod", mesh=("tets", 20, 2, 2, (1.0, 0.1, 0.1), (-0.5, 0, 0)),
                      sides={s: "slip" for s in ("x0", "x1", "y0", "y1", "z0", "z1")}, case="sod",
                      ic="sod", rk=3, steps=5))
    return specs


def build_spec(spec):
    kind, nx, ny, nz, L, org = spec["mesh"]
    if kind == "tets":
        m = meshgen.box_tets(nx, ny, nz, L=L, origin=org, jitter=0.1, seed=SEED, side_bc=spec["sides"])
    elif kind == "hexes":
        m = meshgen.box_hexes(nx, ny, nz, L=L, origin=org, jitter=0.1, seed=SEED, side_bc=spec["sides"])
    else:
        m = meshgen.box_mixed(nx, ny, nz, L=L, jitter=0.0, seed=SEED, side_bc=spec["sides"])
        m.nodes = m.nodes + np.asarray(org)
    if spec["case"] == "reference":
        c = cases.reference_case()
    elif spec["case"] == "ideal_visc":
        c = cases.ideal_gas_case(mu=2e-2)
        c.adaptDtItr = 2
    else:
        c = cases.sod_case()
        c.adaptDtItr = 2
    c.rkSteps = spec["rk"]
    c.maxDt = min(c.maxDt, 1e30)
    return m, c


def ic_for(spec, c, centres):
    if spec["ic"] == "perturbed":
        return cases.perturbed_two_phase_ic(c, centres, seed=5, vel=25.0)
    if spec["ic"] == "tgv":
        return cases.tgv_ic(c, centres * (2 * np.pi))
    return cases.sod_ic(c, centres, x0=0.0)


def centres_of(mesh: meshgen.NeuMesh):
    cs = []
    for blk in mesh.elems:
        cs.append(mesh.nodes[blk].mean(axis=1))
    return np.concatenate(cs)


def run_stage_fixtures(outdir):
    from oracle import ref_run
    outdir = Path(outdir).resolve()
    for spec in stage_specs():
        wd = outdir / spec["name"]
        wd.mkdir(parents=True, exist_ok=True)
        m, c = build_spec(spec)
        meshgen.write_neu(str(wd / "sh.neu"), m)
        U = ic_for(spec, c, centres_of(m))
        try:
            rep = ref_run.run(wd, wd / "sh.neu", c, U, spec["steps"], dump=True)
            print(spec["name"], rep)
        except Exception as e:  # keep going: one failing case should not hide the others
            print(spec["name"], "failed:", e)


def collect_stage_fixtures(outdir):
    outdir = Path(outdir)
    for spec in stage_specs():
        wd = outdir / spec["name"]
        if not (wd / "ref_U.bin").exists():
            print("missing", wd)
            continue
        m, c = build_spec(spec)
        nE = m.n_elem
        rd = lambda f, dt=np.float64: np.fromfile(wd / f, dtype=dt)
        nF = len(rd("ref_mesh_area.bin"))
        d = dict(
            ic=rd("ic.bin").reshape(nE, 10), U=rd("ref_U.bin").reshape(nE, 10),
            fc2el=rd("ref_mesh_fc2el.bin", np.int32).reshape(nF, 2), bc=rd("ref_mesh_bc.bin", np.int32),
            n=rd("ref_mesh_n.bin").reshape(nF, 3), nt1=rd("ref_mesh_nt1.bin").reshape(nF, 3),
            nt2=rd("ref_mesh_nt2.bin").reshape(nF, 3), area=rd("ref_mesh_area.bin"), vol=rd("ref_mesh_vol.bin"),
            cc=rd("ref_mesh_cc.bin").reshape(nE, 3), fc=rd("ref_mesh_fc.bin").reshape(nF, 3),
            primF0=rd("ref_primF0.bin").reshape(nF, 2, 10), primF=rd("ref_primF.bin").reshape(nF, 2, 10),
            grad=rd("ref_grad.bin").reshape(nE, 10, 3), theta=rd("ref_theta.bin").reshape(nE, 10),
            wmin=rd("ref_wmin.bin").reshape(nE, 10), wmax=rd("ref_wmax.bin").reshape(nE, 10),
            rhs=rd("ref_rhs.bin").reshape(nE, 10), steps=np.array(spec["steps"]),
        )
        if (wd / "ref_dt.txt").exists():
            d["dt"] = np.array(float((wd / "ref_dt.txt").read_text().split()[0]))
        t = (wd / "ref_time.txt").read_text().split()
        d["time"] = np.array(float(t[3]))
        d["dt_final"] = np.array(float(t[4]))
        np.savez_compressed(HERE / f"stage_{spec['name']}.npz", **d)
        print("wrote", HERE / f"stage_{spec['name']}.npz")


# ------------------------------------------------------------------ long-run fixture (reference CUDA binary)
LONG_STEPS = (10, 30, 60)


def long_spec():
    """16^3 Taylor-Green vortex in a 2 pi cube with slip walls (the reference has no periodic
    boundary; u . n vanishes on the cube faces), the single-phase ideal gas at Mach 0.1,
    Re 1600, WALE, SSP-RK3, the reference's dt every 100 steps and relaxation every step."""
    L = 2 * np.pi
    m = meshgen.box_hexes(16, 16, 16, L=(L, L, L), seed=SEED)
    c = cases.tgv_case(pr=0.0)
    return m, c


def run_long_fixture(outdir):
    from oracle import ref_run
    outdir = Path(outdir).resolve()
    m, c = long_spec()
    U = cases.tgv_ic(c, centres_of(m))
    for k in LONG_STEPS:
        wd = outdir / f"long{k}"
        wd.mkdir(parents=True, exist_ok=True)
        meshgen.write_neu(str(wd / "sh.neu"), m)
        print(k, ref_run.run(wd, wd / "sh.neu", c, U, k))


def collect_long_fixture(outdir):
    outdir = Path(outdir)
    m, c = long_spec()
    U = cases.tgv_ic(c, centres_of(m))
    d = {"ic": U, "steps": np.array(LONG_STEPS)}
    for k in LONG_STEPS:
        wd = outdir / f"long{k}"
        d[f"U{k}"] = np.fromfile(wd / "ref_U.bin", dtype=np.float64).reshape(m.n_elem, 10)
        d[f"time{k}"] = np.array(float((wd / "ref_time.txt").read_text().split()[3]))
    np.savez_compressed(HERE / "long_tgv16_slip.npz", **d)
    print("wrote", HERE / "long_tgv16_slip.npz")


if __name__ == "__main__":
    cmd = sys.argv[1] if len(sys.argv) > 1 else "kat"
    if cmd == "kat":
        make_kat()
    elif cmd == "stage":
        run_stage_fixtures(sys.argv[2])
    elif cmd == "collect":
        collect_stage_fixtures(sys.argv[2])
    elif cmd == "long":
        run_long_fixture(sys.argv[2])
    elif cmd == "collect_long":
        collect_long_fixture(sys.argv[2])
