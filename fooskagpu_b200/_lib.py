"""ctypes binding of ``libfooskagpu.so`` (declarations mirror ``include/fooskagpu.h``).

The shared library is built in-tree by ``fooskagpu_b200.build``; loading fails loudly when it
is missing — there is no CPU fallback for the device path.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libfooskagpu.so"

i32 = C.c_int32
f64 = C.c_double
PD = C.POINTER(C.c_double)
PI = C.POINTER(C.c_int32)
VP = C.c_void_p
PF = C.POINTER(C.c_float)
i64 = C.c_int64
u64 = C.c_uint64
SG_NPARAM = 8836
SG_NNORM = 30

FG_OK, FG_ERR_ARG, FG_ERR_IO, FG_ERR_MESH, FG_ERR_CUDA, FG_ERR_NAN, FG_ERR_UNSUPPORTED, FG_ERR_NOMEM = range(8)
FG_PREC_FP64, FG_PREC_MIXED = 0, 1
FG_RENUMBER_NONE, FG_RENUMBER_MORTON, FG_RENUMBER_RCM = 0, 1, 2


class FgCase(C.Structure):
    """Mirror of ``fg_case`` (= the reference's ``struct INPUT`` plus extensions)."""

    _fields_ = [
        ("dt", f64), ("cfl", f64), ("adaptDt", i32), ("adaptDtItr", i32), ("maxDt", f64), ("avfMin", f64),
        ("rkSteps", i32), ("finalTime", f64), ("exportTime", f64), ("restartStep", i32), ("restartFlag", i32),
        ("neglectX", i32), ("neglectY", i32), ("neglectZ", i32), ("nMaterials", i32), ("NEQ", i32), ("scale", f64),
        ("viscFlag", i32), ("turbulence", i32), ("woodsFlag", i32),
        ("thermFntRlxFlag", i32), ("thermRlxRate", f64), ("thermUrf", f64), ("thermItrMax", i32),
        ("chemFlag", i32), ("chemFntRlxFlag", i32), ("chemRlxRate", f64), ("chemUrf", f64), ("chemItrMax", i32),
        ("chemCondesation", i32), ("chemLimit", f64),
        ("consCalcFlag", i32), ("consCalcIvar", i32),
        ("satTempUrf", f64),
        ("pInf", f64 * 2), ("gamma", f64 * 2), ("Cp", f64 * 2), ("eta", f64 * 2), ("satConst", f64 * 2),
        ("dynVisc", f64 * 2), ("heatCoef", f64 * 2), ("Pr", f64 * 2),
        ("relaxFlag", i32), ("hllcEnergyFix", i32), ("hllcTieTol", f64), ("heatFlux", i32),
        ("limiter", i32), ("inletVelFlag", i32), ("inletStateFlag", i32), ("reserved", i32 * 2),
        ("inletVel", f64 * 3), ("inletP", f64), ("inletT", f64), ("pressureDatum", f64),
    ]


class FgMeshOpts(C.Structure):
    _fields_ = [("scale", f64), ("periodic", f64 * 3), ("renumber", i32), ("gpu", i32), ("device", i32),
                ("reserved", i32 * 1)]


class FgProbe(C.Structure):
    _fields_ = [("vapourVolume", f64), ("maxPressure", f64), ("minPressure", f64), ("maxSpeed", f64)]


class FgMeshInfo(C.Structure):
    _fields_ = [(k, i32) for k in ("nElem", "nNodes", "nFcs", "nBoundary", "nPeriodic", "maxFaces",
                                   "nTet", "nPyr", "nPrism", "nHex")]


class FgMeshView(C.Structure):
    _fields_ = [("nElem", i32), ("nFcs", i32), ("fc2el", PI), ("boundCond", PI), ("cellCenter", PD),
                ("fcCenter", PD), ("n", PD), ("nt1", PD), ("nt2", PD), ("area", PD), ("volume", PD),
                ("nbShift", PD)]


class FgKernelTimes(C.Structure):
    _fields_ = [("ms", f64 * 8), ("launches", C.c_int64 * 8)]


KERNEL_KINDS = ["grad", "flux", "update", "relax", "dt", "cons", "other", "gather"]


class FgRelaxStats(C.Structure):
    _fields_ = [("nTherm", i32), ("nChem", i32), ("nAbort", i32), ("nIter", i32), ("nSurrogate", i32),
                ("nFallback", i32), ("nPolish", i32)]


class FgPartitionInfo(C.Structure):
    _fields_ = [("nParts", i32), ("part", i32), ("nOwned", i32), ("nGhost", i32), ("nSend", i32), ("nRecv", i32),
                ("nGhost1", i32)]


FG_HALO_W, FG_HALO_G = 0, 1
FG_REDUCE_MIN, FG_REDUCE_SUM = 0, 1
HALO_EXCHANGE_FN = C.CFUNCTYPE(C.c_int, VP, i32, i64, VP)
HALO_ALLREDUCE_FN = C.CFUNCTYPE(C.c_int, VP, i32, PD)


class FgHaloOps(C.Structure):
    _fields_ = [("ctx", VP), ("exchange", HALO_EXCHANGE_FN), ("allreduce", HALO_ALLREDUCE_FN)]


# name -> (restype, argtypes); every symbol here is declared in include/fooskagpu.h
SIGNATURES = {
    "fg_last_error": (C.c_char_p, []),
    "fg_case_default": (None, [C.POINTER(FgCase)]),
    "fg_mesh_load_neu": (C.c_int, [C.c_char_p, C.POINTER(FgMeshOpts), C.POINTER(VP)]),
    "fg_mesh_build": (C.c_int, [i32, PD, i32, PI, PI, PI, C.POINTER(FgMeshOpts), C.POINTER(VP)]),
    "fg_mesh_info_get": (C.c_int, [VP, C.POINTER(FgMeshInfo)]),
    "fg_mesh_view_get": (C.c_int, [VP, C.POINTER(FgMeshView)]),
    "fg_mesh_permutation": (C.c_int, [VP, PI, i32]),
    "fg_mesh_free": (None, [VP]),
    "fg_mesh_partition": (C.c_int, [VP, i32, i32, C.POINTER(VP)]),
    "fg_mesh_partition_info": (C.c_int, [VP, C.POINTER(FgPartitionInfo)]),
    "fg_mesh_partition_maps": (C.c_int, [VP, PI, PI, PI, PI, PI]),
    "fg_halo_buffer_bytes": (C.c_int, [VP, C.POINTER(i64), C.POINTER(i64)]),
    "fg_solver_set_halo": (C.c_int, [VP, C.POINTER(FgHaloOps), VP, VP]),
    "fg_solver_create": (C.c_int, [VP, C.POINTER(FgCase), i32, i32, C.POINTER(VP)]),
    "fg_solver_destroy": (C.c_int, [VP]),
    "fg_solver_memory": (C.c_int, [VP, C.POINTER(C.c_uint64)]),
    "fg_probe": (C.c_int, [VP, C.POINTER(FgProbe), VP]),
    "fg_set_state": (C.c_int, [VP, PD, VP]),
    "fg_set_state_async": (C.c_int, [VP, PD, VP]),
    "fg_get_state": (C.c_int, [VP, PD, VP]),
    "fg_get_state_async": (C.c_int, [VP, PD, VP]),
    "fg_state_join": (C.c_int, [VP, VP]),
    "fg_compute_rhs": (C.c_int, [VP, i32, VP]),
    "fg_compute_time_step": (C.c_int, [VP, PD, VP]),
    "fg_init_rk": (C.c_int, [VP, VP]),
    "fg_update": (C.c_int, [VP, i32, VP]),
    "fg_stage": (C.c_int, [VP, i32, VP]),
    "fg_relaxation": (C.c_int, [VP, C.POINTER(FgRelaxStats), VP]),
    "fg_cons_calc": (C.c_int, [VP, i32, PD, VP]),
    "fg_cons_integral_noalloc": (C.c_int, [VP, VP, i32, i32, VP, VP]),
    "fg_surrogate_create": (C.c_int, [i32, u64, C.POINTER(VP)]),
    "fg_surrogate_destroy": (C.c_int, [VP]),
    "fg_surrogate_set_data": (C.c_int, [VP, PF, PF, i64]),
    "fg_surrogate_train": (C.c_int, [VP, i32, i32, C.c_float, u64, PF]),
    "fg_surrogate_loss_grad": (C.c_int, [VP, PF, PF, i32, PF, PF]),
    "fg_surrogate_get_params": (C.c_int, [VP, PF]),
    "fg_surrogate_set_params": (C.c_int, [VP, PF]),
    "fg_surrogate_get_norm": (C.c_int, [VP, PF]),
    "fg_surrogate_set_norm": (C.c_int, [VP, PF]),
    "fg_surrogate_predict": (C.c_int, [VP, PF, i32, PF, PI]),
    "fg_solver_set_surrogate": (C.c_int, [VP, VP, f64, i32]),
    "fg_solver_set_surrogate_pass": (C.c_int, [VP, i32]),
    "fg_relax_log": (C.c_int, [VP, i64]),
    "fg_check_state": (C.c_int, [VP, PI]),
    "fg_checkpoint_write": (C.c_int, [VP, C.c_char_p]),
    "fg_checkpoint_read": (C.c_int, [VP, C.c_char_p]),
    "fg_field_dump": (C.c_int, [VP, C.c_char_p]),
    "fg_relax_stats_read": (C.c_int, [VP, C.POINTER(FgRelaxStats)]),
    "fg_relax_log_read": (C.c_int, [VP, PF, PF, i64, C.POINTER(i64)]),
    "fg_get_time": (C.c_int, [VP, PD, PD, PI]),
    "fg_set_dt": (C.c_int, [VP, f64]),
    "fg_step": (C.c_int, [VP, VP]),
    "fg_profile": (C.c_int, [VP, i32]),
    "fg_profile_read": (C.c_int, [VP, C.POINTER(FgKernelTimes)]),
    "fg_launch_count": (C.c_int, [VP, C.POINTER(C.c_uint64)]),
    "fg_get_rhs": (C.c_int, [VP, PD]),
    "fg_get_limited": (C.c_int, [VP, PD, PD]),
    "fg_get_signal": (C.c_int, [VP, PD]),
}

_lib = None


class FgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"fooskagpu error {code}: {msg}")
        self.code = code


def lib() -> C.CDLL:
    """Load ``libfooskagpu.so`` (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m fooskagpu_b200.build` "
                               "(the device path has no CPU fallback)")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != FG_OK:
        raise FgError(rc, lib().fg_last_error().decode())
