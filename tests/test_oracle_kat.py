"""Known-answer tests of the oracle against the reference's own device functions.

The fixtures in tests/golden/kat_physics.npz were produced by the reference sources compiled
for the host (tests/golden/make_golden.py kat).  The oracle must reproduce them bit for bit:
same formulas, same evaluation order, same libm.  When the reference tree is present the
live host build is checked on fresh random inputs as well."""
import ctypes as C
import json
from pathlib import Path

import numpy as np
import pytest

from fooskagpu_b200._lib import FgCase
from oracle import oracle_py as O

GOLD = Path(__file__).resolve().parent / "golden"
PD = C.POINTER(C.c_double)


def _p(a):
    return a.ctypes.data_as(PD)


def _case_from(d):
    c = FgCase()
    for k, v in d.items():
        if k == "reserved" or not hasattr(c, k):   # extension padding / fields of other versions
            continue
        if isinstance(v, list):
            arr = getattr(c, k)
            for i, x in enumerate(v):
                arr[i] = x
        else:
            setattr(c, k, v)
    return c


def _load():
    z = np.load(GOLD / "kat_physics.npz")
    meta = json.loads((GOLD / "kat_cases.json").read_text())
    return z, meta


CASES = ["reference", "reference_nowood", "ideal_gas"]


@pytest.mark.parametrize("cname", CASES)
def test_cons_prim(cname):
    z, meta = _load()
    c = _case_from(meta[cname])
    L = O.lib()
    UL = z[f"{cname}/UL"]
    for i in range(len(UL)):
        s = np.zeros(10)
        L.orc_cons2prim(C.byref(c), _p(UL[i].copy()), _p(s))
        assert np.array_equal(s, z[f"{cname}/solL"][i]), i
        u = np.zeros(10)
        L.orc_prim2cons(C.byref(c), _p(s.copy()), _p(u))
        assert np.array_equal(u, z[f"{cname}/prim2cons"][i]), i


@pytest.mark.parametrize("cname", CASES)
def test_wave_speeds_and_bc(cname):
    z, meta = _load()
    c = _case_from(meta[cname])
    L = O.lib()
    n, t1, t2 = z[f"{cname}/n"], z[f"{cname}/t1"], z[f"{cname}/t2"]
    sL, sR = z[f"{cname}/solL"], z[f"{cname}/solR"]
    for i in range(len(n)):
        cc, ul, ur = np.zeros(3), np.zeros(3), np.zeros(3)
        L.orc_wave_speeds(C.byref(c), _p(n[i].copy()), _p(t1[i].copy()), _p(t2[i].copy()), _p(sL[i].copy()),
                          _p(sR[i].copy()), _p(cc), _p(ul), _p(ur))
        assert np.array_equal(np.concatenate([cc, ul, ur]), z[f"{cname}/wave"][i]), i
        for b in range(1, 6):
            s = sL[i].copy()
            L.orc_bc_values(C.byref(c), _p(n[i].copy()), _p(t1[i].copy()), _p(t2[i].copy()), _p(s), b)
            assert np.array_equal(s, z[f"{cname}/bc"][i, b - 1]), (i, b)


@pytest.mark.parametrize("cname", CASES)
def test_star_flux_source(cname):
    z, meta = _load()
    c = _case_from(meta[cname])
    L = O.lib()
    n, t1, t2 = z[f"{cname}/n"], z[f"{cname}/t1"], z[f"{cname}/t2"]
    sL, ws, p2c = z[f"{cname}/solL"], z[f"{cname}/wave"], z[f"{cname}/prim2cons"]
    unc, are = z[f"{cname}/unc"], z[f"{cname}/are"]
    UL, UR = z[f"{cname}/UL"], z[f"{cname}/UR"]
    for i in range(len(n)):
        out = np.zeros(23)
        L.orc_star_region(C.byref(c), _p(sL[i].copy()), _p(ws[i, 3:6].copy()), ws[i, 0], ws[i, 1], _p(n[i].copy()),
                          _p(t1[i].copy()), _p(t2[i].copy()), _p(p2c[i].copy()), _p(out))
        assert np.array_equal(out, z[f"{cname}/star"][i]), ("star", i)
        f = np.zeros(10)
        L.orc_adv_flux(C.byref(c), _p(sL[i].copy()), _p(n[i].copy()), _p(unc[i].copy()), are[i, 0], are[i, 1], _p(f))
        assert np.array_equal(f, z[f"{cname}/flux"][i]), ("flux", i)
        fs = np.zeros(6)
        L.orc_flux_source(C.byref(c), _p(unc[i].copy()), _p(UL[i].copy()), _p(UR[i].copy()), _p(n[i].copy()), _p(fs))
        assert np.array_equal(fs, z[f"{cname}/fsrc"][i]), ("fsrc", i)


@pytest.mark.parametrize("cname", CASES)
def test_relaxation_cells(cname):
    z, meta = _load()
    c = _case_from(meta[cname])
    L = O.lib()
    UL = z[f"{cname}/UL"]
    nabort = 0
    for i in range(len(UL)):
        u = UL[i].copy()
        L.orc_therm_relax_cell(C.byref(c), _p(u), None)
        assert np.array_equal(u, z[f"{cname}/therm"][i]), ("therm", i)
        u = UL[i].copy()
        it = C.c_int()
        nabort += L.orc_chem_relax_cell(C.byref(c), _p(u), C.byref(it))
        assert np.array_equal(u, z[f"{cname}/chem"][i]), ("chem", i)


@pytest.mark.parametrize("cname", CASES)
def test_viscous_face(cname):
    """Oracle viscous face flux vs the reference kernel run on one face (interior and all
    boundary codes)."""
    z, meta = _load()
    c = _case_from(meta[cname])
    c.viscFlag = 1
    c.turbulence = 1
    L = O.lib()
    # restated through the oracle's full-mesh path is covered by stage tests; here the
    # per-face function is reached through a two-cell mesh view
    from fooskagpu_b200._lib import FgMeshView
    PI = C.POINTER(C.c_int32)
    for i in range(len(z[f"{cname}/area"])):
        bc = int(z[f"{cname}/bcs"][i])
        fc2el = np.array([0, 1 if bc == 0 else -1], dtype=np.int32)
        bcs = np.array([bc], dtype=np.int32)
        nrm = z[f"{cname}/n"][i].copy()
        area = np.array([z[f"{cname}/area"][i]])
        vol = z[f"{cname}/vol"][i].copy()
        zero3 = np.zeros(3)
        v = FgMeshView()
        v.nElem, v.nFcs = 2, 1
        v.fc2el = fc2el.ctypes.data_as(PI)
        v.boundCond = bcs.ctypes.data_as(PI)
        cc = np.zeros(6)
        v.cellCenter = _p(cc); v.fcCenter = _p(zero3); v.n = _p(nrm)
        v.nt1 = _p(z[f"{cname}/t1"][i].copy()); v.nt2 = _p(z[f"{cname}/t2"][i].copy())
        v.area = _p(area); v.volume = _p(vol); v.nbShift = _p(zero3)
        w = L.orc_work_new(2, 1)
        pf = np.ctypeslib.as_array(w.contents.primF, shape=(20,))
        pf[:10] = z[f"{cname}/solL"][i]
        pf[10:] = z[f"{cname}/solR"][i]
        gr = np.ctypeslib.as_array(w.contents.grad, shape=(60,))
        gr[:30] = z[f"{cname}/gO"][i]
        gr[30:] = z[f"{cname}/gN"][i]
        # only the viscous contribution: zero the convective part by an all-zero state trick is
        # not possible, so compare through the difference viscFlag=1 minus viscFlag=0
        U = np.tile(z[f"{cname}/UL"][i], (2, 1)).copy()
        c0 = FgCase.from_buffer_copy(c)
        c0.viscFlag = 0
        L.orc_rhs(C.byref(c0), C.byref(v), _p(U), w)
        r0 = np.ctypeslib.as_array(w.contents.RHS, shape=(20,)).copy()
        L.orc_rhs(C.byref(c), C.byref(v), _p(U), w)
        r1 = np.ctypeslib.as_array(w.contents.RHS, shape=(20,)).copy()
        L.orc_work_free(w)
        ref = z[f"{cname}/visc"][i]
        # the oracle adds viscous terms after convective ones (as the reference kernels run);
        # (r0 + v) - r0 is not exactly v, so compare with a relative ULP-scale tolerance
        got = r1 - r0
        scale = np.abs(r1).max() + 1e-300
        assert np.all(np.abs(got - ref) <= 1e-12 * scale), (i, bc)


def test_live_reference_if_present():
    """Fresh random inputs against the live host build of the reference (skipped when the
    reference tree / oracle/_ref is absent, e.g. on the GPU box)."""
    lib = Path(O.HERE) / "_ref" / "libref_host.so"
    if not lib.exists():
        pytest.skip("oracle/_ref/libref_host.so not built")
    from fooskagpu_b200 import cases
    R = C.CDLL(str(lib))
    L = O.lib()
    c = cases.reference_case()
    rng = np.random.default_rng(99)
    for it in range(300):
        U = cases.perturbed_two_phase_ic(c, rng.uniform(-1, 1, size=(1, 3)), seed=it, vel=40.0)[0]
        for fo, fr in (("orc_therm_relax_cell", "refkat_therm_cell"), ("orc_chem_relax_cell", "refkat_chem_cell")):
            a, b = U.copy(), U.copy()
            getattr(L, fo)(C.byref(c), _p(a), None)
            getattr(R, fr)(C.byref(c), _p(b))
            assert np.array_equal(a, b), (fo, it)
