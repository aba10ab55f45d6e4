"""TEST INFRASTRUCTURE ONLY — ctypes binding of oracle/liboracle.so, the CPU FP64 restatement
of the reference solver's residual path.  Imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg; never by the product package.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"

PD = C.POINTER(C.c_double)
VP = C.c_void_p

_lib = None


class OrcWork(C.Structure):
    _fields_ = [(k, PD) for k in ("U0", "primF", "grad", "wMin", "wMax", "ext", "theta", "RHS", "signal")]


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            from fooskagpu_b200 import build
            build.build_oracle()
        from fooskagpu_b200._lib import FgCase, FgMeshView, FgRelaxStats
        L = C.CDLL(str(LIB_PATH))
        CP = C.POINTER(FgCase)
        MP = C.POINTER(FgMeshView)
        WP = C.POINTER(OrcWork)
        sig = {
            "orc_work_new": (WP, [C.c_int, C.c_int]),
            "orc_work_free": (None, [WP]),
            "orc_set_threads": (C.c_int, [C.c_int]),
            "orc_eqos": (C.c_double, [CP, C.c_int, C.c_int, C.c_double, C.c_double]),
            "orc_cons2prim": (None, [CP, PD, PD]),
            "orc_prim2cons": (None, [CP, PD, PD]),
            "orc_wave_speeds": (None, [CP, PD, PD, PD, PD, PD, PD, PD, PD]),
            "orc_bc_values": (None, [CP, PD, PD, PD, PD, C.c_int]),
            "orc_face_flux": (None, [CP, PD, PD, PD, C.c_double, C.c_int, PD, PD, PD, PD, PD]),
            "orc_eddy_visc": (C.c_double, [PD, C.c_double]),
            "orc_star_region": (None, [CP, PD, PD, C.c_double, C.c_double, PD, PD, PD, PD, PD]),
            "orc_adv_flux": (None, [CP, PD, PD, PD, C.c_double, C.c_double, PD]),
            "orc_flux_source": (None, [CP, PD, PD, PD, PD, PD]),
            "orc_saturation_temp": (C.c_double, [CP, C.c_double, C.c_double, C.c_double]),
            "orc_therm_relax_cell": (C.c_int, [CP, PD, C.POINTER(C.c_int)]),
            "orc_chem_relax_cell": (C.c_int, [CP, PD, C.POINTER(C.c_int)]),
            "orc_prim": (None, [CP, MP, PD, WP]),
            "orc_grad": (None, [CP, MP, WP]),
            "orc_limiter": (None, [CP, MP, WP]),
            "orc_rhs": (None, [CP, MP, PD, WP]),
            "orc_residual": (None, [CP, MP, PD, WP]),
            "orc_timestep_min": (C.c_double, [CP, MP, WP]),
            "orc_update": (None, [CP, MP, C.c_int, C.c_double, PD, WP]),
            "orc_init_rk": (None, [MP, PD, WP]),
            "orc_relaxation": (None, [CP, MP, PD, C.POINTER(FgRelaxStats)]),
            "orc_cons_calc": (C.c_double, [MP, C.c_int, PD]),
            "orc_step": (None, [CP, MP, PD, WP, PD, PD, C.POINTER(C.c_int), PD, C.POINTER(FgRelaxStats)]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(PD)


def set_threads(n: int) -> int:
    return lib().orc_set_threads(int(n))


class Oracle:
    """Oracle bound to one mesh view (reference layout) and one case."""

    def __init__(self, view, case):
        self.view = view
        self.case = case
        self.nE, self.nF = view.nElem, view.nFcs
        self.w = lib().orc_work_new(self.nE, self.nF)
        self.dt = C.c_double(case.dt)
        self.time = C.c_double(0.0)
        self.istep = C.c_int(0)
        self.cons_last = C.c_double(float("nan"))

    def _arr(self, name, shape):
        ptr = getattr(self.w.contents, name)
        return np.ctypeslib.as_array(ptr, shape=shape)

    @property
    def rhs(self):
        return self._arr("RHS", (self.nE, 10))

    @property
    def grad(self):
        return self._arr("grad", (self.nE, 10, 3))

    @property
    def theta(self):
        return self._arr("theta", (self.nE, 10))

    @property
    def primF(self):
        return self._arr("primF", (self.nF, 2, 10))

    @property
    def signal(self):
        return self._arr("signal", (self.nE,))

    def residual(self, U: np.ndarray) -> np.ndarray:
        U = np.ascontiguousarray(U, dtype=np.float64)
        lib().orc_residual(C.byref(self.case), C.byref(self.view), _p(U), self.w)
        return self.rhs.copy()

    def timestep_min(self) -> float:
        return lib().orc_timestep_min(C.byref(self.case), C.byref(self.view), self.w)

    def relaxation(self, U: np.ndarray) -> dict:
        from fooskagpu_b200._lib import FgRelaxStats
        st = FgRelaxStats()
        lib().orc_relaxation(C.byref(self.case), C.byref(self.view), _p(U), C.byref(st))
        return {"nTherm": st.nTherm, "nChem": st.nChem, "nAbort": st.nAbort, "nIter": st.nIter}

    def cons_calc(self, ivar: int, U: np.ndarray) -> float:
        return lib().orc_cons_calc(C.byref(self.view), ivar, _p(np.ascontiguousarray(U)))

    def init_rk(self, U):
        lib().orc_init_rk(C.byref(self.view), _p(U), self.w)

    def update(self, irk: int, dt: float, U: np.ndarray):
        lib().orc_update(C.byref(self.case), C.byref(self.view), irk, dt, _p(U), self.w)

    def step(self, U: np.ndarray) -> None:
        from fooskagpu_b200._lib import FgRelaxStats
        st = FgRelaxStats()
        lib().orc_step(C.byref(self.case), C.byref(self.view), _p(U), self.w, C.byref(self.dt), C.byref(self.time),
                       C.byref(self.istep), C.byref(self.cons_last), C.byref(st))
        self.last_relax = {"nTherm": st.nTherm, "nChem": st.nChem, "nAbort": st.nAbort}

    def close(self):
        if self.w:
            lib().orc_work_free(self.w)
            self.w = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
