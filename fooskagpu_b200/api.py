"""Python host API over the C ABI (mirrors the reference's stage functions).

    mesh = Mesh.load_neu("sh.neu", scale=1e-3)
    case = default_case(); case.rkSteps = 3
    s = Solver(mesh, case, precision="mixed")
    s.set_state(U)          # initialize / readField
    s.step()                # one explicitLoop iteration
    U = s.get_state()
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib as L
from ._lib import FgCase, FgMeshInfo, FgMeshOpts, FgMeshView, FgRelaxStats, check, lib

_PREC = {"fp64": L.FG_PREC_FP64, "mixed": L.FG_PREC_MIXED}
_RENUM = {"none": L.FG_RENUMBER_NONE, "morton": L.FG_RENUMBER_MORTON, "rcm": L.FG_RENUMBER_RCM}


def default_case() -> FgCase:
    """The parameters the reference hard-codes in DP/buildInput.cu:10-69."""
    c = FgCase()
    lib().fg_case_default(C.byref(c))
    return c


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(L.PD)


class Mesh:
    """Pre-processed mesh (reference face order + device renumbering)."""

    def __init__(self, handle):
        self._h = handle
        info = FgMeshInfo()
        check(lib().fg_mesh_info_get(self._h, C.byref(info)))
        self.info = {k: getattr(info, k) for k, _ in FgMeshInfo._fields_}
        self.n_elem = info.nElem
        self.n_fcs = info.nFcs
        pi = L.FgPartitionInfo()
        check(lib().fg_mesh_partition_info(self._h, C.byref(pi)))
        self.part_info = {k: getattr(pi, k) for k, _ in L.FgPartitionInfo._fields_}
        self.n_owned = pi.nOwned   # cells with a state (all of them unless the mesh is a part)

    @classmethod
    def load_neu(cls, path: str, scale: float = 1.0, periodic=(0.0, 0.0, 0.0), renumber: str = "morton",
                 gpu: bool = False, device: int = 0) -> "Mesh":
        """gpu=True: face matching, face order, geometry and Morton order on the GPU (same arrays)."""
        o = FgMeshOpts()
        o.scale = scale
        for d in range(3):
            o.periodic[d] = periodic[d]
        o.renumber = _RENUM[renumber]
        o.gpu = 1 if gpu else 0
        o.device = device
        h = C.c_void_p()
        check(lib().fg_mesh_load_neu(path.encode(), C.byref(o), C.byref(h)))
        return cls(h)

    @classmethod
    def build(cls, nodes: np.ndarray, elems, bcs: dict, scale: float = 1.0, periodic=(0.0, 0.0, 0.0),
              renumber: str = "morton", gpu: bool = False, device: int = 0) -> "Mesh":
        """The same pre-processing for element lists held in memory (fg_mesh_build): nodes
        (nNodes, 3); elems, a list of (nE_k, nn_k) 0-based node-id blocks in element order; bcs,
        {name: (gambit code, element ids, local faces)} as meshgen.NeuMesh holds them."""
        code_map = {45: 1, 26: 2, 13: 3, 42: 4, 51: 5}
        n_elem = sum(len(b) for b in elems)
        el_nn = np.empty(n_elem, dtype=np.int32)
        el_nodes = np.zeros((n_elem, 8), dtype=np.int32)
        off = 0
        for b in elems:
            el_nn[off:off + len(b)] = b.shape[1]
            el_nodes[off:off + len(b), :b.shape[1]] = b
            off += len(b)
        el_bc = np.zeros((n_elem, 6), dtype=np.int32)
        for _, (code, el, fc) in bcs.items():
            if code in code_map:
                el_bc[np.asarray(el), np.asarray(fc)] = code_map[code]
        nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        o = FgMeshOpts()
        o.scale = scale
        for d in range(3):
            o.periodic[d] = periodic[d]
        o.renumber = _RENUM[renumber]
        o.gpu = 1 if gpu else 0
        o.device = device
        h = C.c_void_p()
        check(lib().fg_mesh_build(len(nodes), _dptr(nodes), n_elem, el_nn.ctypes.data_as(L.PI),
                                  el_nodes.ctypes.data_as(L.PI), el_bc.ctypes.data_as(L.PI), C.byref(o), C.byref(h)))
        return cls(h)

    def view(self) -> FgMeshView:
        v = FgMeshView()
        check(lib().fg_mesh_view_get(self._h, C.byref(v)))
        return v

    def arrays(self) -> dict:
        """Copies of the reference-layout mesh arrays (numpy)."""
        v = self.view()
        nE, nF = v.nElem, v.nFcs
        g = lambda p, k, dt=np.float64: np.ctypeslib.as_array(p, shape=(k,)).astype(dt).copy()
        return {
            "fc2el": g(v.fc2el, 2 * nF, np.int32).reshape(nF, 2),
            "boundCond": g(v.boundCond, nF, np.int32),
            "cellCenter": g(v.cellCenter, 3 * nE).reshape(nE, 3),
            "fcCenter": g(v.fcCenter, 3 * nF).reshape(nF, 3),
            "n": g(v.n, 3 * nF).reshape(nF, 3),
            "nt1": g(v.nt1, 3 * nF).reshape(nF, 3),
            "nt2": g(v.nt2, 3 * nF).reshape(nF, 3),
            "area": g(v.area, nF),
            "volume": g(v.volume, nE),
            "nbShift": g(v.nbShift, 3 * nF).reshape(nF, 3),
        }

    def partition(self, n_parts: int, part: int) -> "Mesh":
        """Part `part` of `n_parts` (contiguous ranges of the Morton device order): own cells first,
        then two layers of ghost cells (the other parts' face neighbours, then theirs); the returned
        mesh is independent of this one."""
        h = C.c_void_p()
        check(lib().fg_mesh_partition(self._h, int(n_parts), int(part), C.byref(h)))
        return Mesh(h)

    def partition_maps(self) -> dict:
        """cell_global (.neu index in the whole mesh of each cell), send/recv lists per part."""
        pi = self.part_info
        P = pi["nParts"]
        out = {"cell_global": np.empty(self.n_elem, np.int32), "send_start": np.empty(P + 1, np.int32),
               "send_cells": np.empty(max(pi["nSend"], 1), np.int32), "recv_start": np.empty(P + 1, np.int32),
               "recv_cells": np.empty(max(pi["nRecv"], 1), np.int32)}
        check(lib().fg_mesh_partition_maps(self._h, *(out[k].ctypes.data_as(L.PI) for k in
                                                      ("cell_global", "send_start", "send_cells", "recv_start",
                                                       "recv_cells"))))
        out["send_cells"] = out["send_cells"][:pi["nSend"]]
        out["recv_cells"] = out["recv_cells"][:pi["nRecv"]]
        return out

    def permutation(self) -> np.ndarray:
        p = np.empty(self.n_elem, dtype=np.int32)
        check(lib().fg_mesh_permutation(self._h, p.ctypes.data_as(L.PI), self.n_elem))
        return p

    def close(self):
        if self._h:
            lib().fg_mesh_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Solver:
    """Device solver for one mesh and case; all state lives in HBM."""

    def __init__(self, mesh: Mesh, case: FgCase, precision: str = "mixed", device: int = 0):
        self.mesh = mesh
        self.case = case
        self.precision = precision
        h = C.c_void_p()
        check(lib().fg_solver_create(mesh._h, C.byref(case), _PREC[precision], device, C.byref(h)))
        self._h = h
        self.n = mesh.n_owned     # state rows: the own cells of a part mesh
        self._halo = None

    # -- state
    def set_state(self, U: np.ndarray, stream: Optional[int] = None) -> None:
        U = np.ascontiguousarray(U, dtype=np.float64).reshape(self.n, 10)
        check(lib().fg_set_state(self._h, _dptr(U), stream))

    def set_state_async(self, U: np.ndarray, stream: Optional[int] = None) -> None:
        """Queue the upload without synchronising (fg_set_state_async); U must stay unchanged
        until the stream has passed the copy when it is pinned memory."""
        if not (U.dtype == np.float64 and U.flags["C_CONTIGUOUS"] and U.shape == (self.n, 10)):
            raise ValueError("set_state_async needs a C-contiguous float64 array of shape (n, 10)")
        check(lib().fg_set_state_async(self._h, _dptr(U), stream))

    def get_state_async(self, out: np.ndarray, stream: Optional[int] = None) -> None:
        """Queue the download into `out` (fg_get_state_async): the copy runs on the solver's
        download stream; `out` is complete once a stream joined by state_join has passed that
        point (or after a device synchronisation)."""
        if not (out.dtype == np.float64 and out.flags["C_CONTIGUOUS"] and out.shape == (self.n, 10)):
            raise ValueError("get_state_async needs a C-contiguous float64 array of shape (n, 10)")
        check(lib().fg_get_state_async(self._h, _dptr(out), stream))

    def state_join(self, stream: Optional[int] = None) -> None:
        """Make `stream` wait on the device for every get_state_async issued so far (fg_state_join)."""
        check(lib().fg_state_join(self._h, stream))

    def get_state(self, out: Optional[np.ndarray] = None, stream: Optional[int] = None) -> np.ndarray:
        if out is None:
            out = np.empty((self.n, 10), dtype=np.float64)
        check(lib().fg_get_state(self._h, _dptr(out), stream))
        return out

    def halo_buffer_bytes(self):
        sb, rb = L.i64(), L.i64()
        check(lib().fg_halo_buffer_bytes(self._h, C.byref(sb), C.byref(rb)))
        return sb.value, rb.value

    def set_halo(self, exchange, allreduce, send_ptr: int, recv_ptr: int) -> None:
        """Transport of a partitioned run: exchange(field, record_bytes, stream) moves the send
        buffer's records to the other parts and fills the receive buffer; allreduce(op, value)
        returns the combined value.  Both return normally on success (an exception is reported
        to the solver as a failed exchange)."""
        def _ex(ctx, field, rb, stream):
            try:
                exchange(int(field), int(rb), stream)
                return 0
            except Exception:
                import traceback
                traceback.print_exc()
                return 1

        def _ar(ctx, op, value):
            try:
                value[0] = float(allreduce(int(op), float(value[0])))
                return 0
            except Exception:
                import traceback
                traceback.print_exc()
                return 1

        ops = L.FgHaloOps(None, L.HALO_EXCHANGE_FN(_ex), L.HALO_ALLREDUCE_FN(_ar))
        check(lib().fg_solver_set_halo(self._h, C.byref(ops), send_ptr, recv_ptr))
        self._halo = ops   # the callbacks must outlive the solver's use of them

    # -- stage functions
    def compute_rhs(self, want_signal: bool = False, stream=None) -> None:
        check(lib().fg_compute_rhs(self._h, 1 if want_signal else 0, stream))

    def compute_time_step(self, stream=None) -> float:
        dt = C.c_double()
        check(lib().fg_compute_time_step(self._h, C.byref(dt), stream))
        return dt.value

    def init_rk(self, stream=None) -> None:
        check(lib().fg_init_rk(self._h, stream))

    def update(self, irk: int, stream=None) -> None:
        check(lib().fg_update(self._h, irk, stream))

    def stage(self, irk: int, stream=None) -> None:
        check(lib().fg_stage(self._h, irk, stream))

    def relaxation(self, stream=None) -> dict:
        st = FgRelaxStats()
        check(lib().fg_relaxation(self._h, C.byref(st), stream))
        return {"nTherm": st.nTherm, "nChem": st.nChem, "nAbort": st.nAbort, "nIter": st.nIter,
                "nSurrogate": st.nSurrogate, "nFallback": st.nFallback, "nPolish": st.nPolish}

    def check_state(self) -> int:
        """-1 if the state is healthy; raises FgError (FG_ERR_NAN) naming the step otherwise."""
        k = C.c_int32()
        check(lib().fg_check_state(self._h, C.byref(k)))
        return k.value

    # -- checkpoint / restart and field output
    def checkpoint_write(self, path: str) -> None:
        check(lib().fg_checkpoint_write(self._h, str(path).encode()))

    def checkpoint_read(self, path: str) -> None:
        check(lib().fg_checkpoint_read(self._h, str(path).encode()))

    def field_dump(self, path: str) -> None:
        check(lib().fg_field_dump(self._h, str(path).encode()))

    def relax_stats(self) -> dict:
        """Counts of the most recent relaxation (also the one inside step())."""
        st = FgRelaxStats()
        check(lib().fg_relax_stats_read(self._h, C.byref(st)))
        return {"nTherm": st.nTherm, "nChem": st.nChem, "nAbort": st.nAbort, "nIter": st.nIter,
                "nSurrogate": st.nSurrogate, "nFallback": st.nFallback, "nPolish": st.nPolish}

    # -- learned equilibrium surrogate
    def set_surrogate(self, sg: Optional["Surrogate"], rel_tol: float = 1e-6, polish_iters: int = 3) -> None:
        """Attach (or detach with None) the surrogate used by relaxation()/step()."""
        self._sg = sg
        check(lib().fg_solver_set_surrogate(self._h, sg._h if sg is not None else None, rel_tol, polish_iters))

    def set_surrogate_pass(self, mode: str = "auto") -> None:
        """Where the surrogate's polish runs: "fused" (inside the relaxation kernel), "separate" (a
        pass of its own before it) or "auto" (chosen per relaxation from the chemical cells of an
        earlier one).  The relaxed states are bitwise the same for all three."""
        modes = {"auto": 0, "fused": 1, "separate": 2}
        if mode not in modes:
            raise ValueError(f"surrogate pass mode {mode!r}: one of {sorted(modes)}")
        check(lib().fg_solver_set_surrogate_pass(self._h, modes[mode]))

    def relax_log(self, capacity: int) -> None:
        """Log chemical Newton solves as surrogate training samples (0 turns the log off)."""
        check(lib().fg_relax_log(self._h, int(capacity)))

    def relax_log_read(self, cap: int):
        X = np.empty((max(cap, 1), 3), dtype=np.float32)
        Y = np.empty((max(cap, 1), 4), dtype=np.float32)
        k = C.c_int64()
        check(lib().fg_relax_log_read(self._h, _fptr(X), _fptr(Y), int(cap), C.byref(k)))
        return X[:k.value].copy(), Y[:k.value].copy()

    def probe(self, stream=None) -> dict:
        """Vapour volume, max / min mixture pressure and max speed of the current state."""
        pr = L.FgProbe()
        check(lib().fg_probe(self._h, C.byref(pr), stream))
        return {k: getattr(pr, k) for k, _ in L.FgProbe._fields_}

    def cons_calc(self, ivar: int, stream=None) -> float:
        v = C.c_double()
        check(lib().fg_cons_calc(self._h, ivar, C.byref(v), stream))
        return v.value

    def step(self, stream=None) -> None:
        check(lib().fg_step(self._h, stream))

    def time(self):
        dt, t, it = C.c_double(), C.c_double(), C.c_int32()
        check(lib().fg_get_time(self._h, C.byref(dt), C.byref(t), C.byref(it)))
        return dt.value, t.value, it.value

    def set_dt(self, dt: float) -> None:
        check(lib().fg_set_dt(self._h, float(dt)))

    def memory_bytes(self) -> int:
        b = C.c_uint64()
        check(lib().fg_solver_memory(self._h, C.byref(b)))
        return b.value

    # -- instrumentation
    def profile(self, enable: bool = True) -> None:
        check(lib().fg_profile(self._h, 1 if enable else 0))

    def profile_read(self) -> dict:
        t = L.FgKernelTimes()
        check(lib().fg_profile_read(self._h, C.byref(t)))
        return {k: {"ms": t.ms[i], "launches": int(t.launches[i])} for i, k in enumerate(L.KERNEL_KINDS)
                if t.launches[i] > 0}

    def launch_count(self) -> int:
        v = C.c_uint64()
        check(lib().fg_launch_count(self._h, C.byref(v)))
        return int(v.value)

    # -- parity hooks
    def get_rhs(self) -> np.ndarray:
        out = np.empty((self.n, 10))
        check(lib().fg_get_rhs(self._h, _dptr(out)))
        return out

    def get_limited(self):
        g = np.empty((self.n, 10, 3))
        th = np.empty((self.n, 10))
        check(lib().fg_get_limited(self._h, _dptr(g), _dptr(th)))
        return g, th

    def get_signal(self) -> np.ndarray:
        out = np.empty(self.n)
        check(lib().fg_get_signal(self._h, _dptr(out)))
        return out

    def close(self):
        if getattr(self, "_h", None):
            lib().fg_solver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class Surrogate:
    """Learned equilibrium surrogate (MLP 3 -> 64 -> 64 -> 64 -> 4): (rho, e, Y) -> (p, T, alpha, Y_eq)."""

    NPARAM = L.SG_NPARAM
    NNORM = L.SG_NNORM

    def __init__(self, device: int = 0, seed: int = 20261203):
        h = C.c_void_p()
        check(lib().fg_surrogate_create(device, seed, C.byref(h)))
        self._h = h

    def set_data(self, X: np.ndarray, Y: np.ndarray) -> None:
        X = np.ascontiguousarray(X, dtype=np.float32).reshape(-1, 3)
        Y = np.ascontiguousarray(Y, dtype=np.float32).reshape(-1, 4)
        check(lib().fg_surrogate_set_data(self._h, _fptr(X), _fptr(Y), len(X)))

    def train(self, epochs: int, batch: int = 4096, lr: float = 2e-3, seed: int = 1) -> float:
        loss = C.c_float()
        check(lib().fg_surrogate_train(self._h, epochs, batch, lr, seed, C.byref(loss)))
        return loss.value

    def loss_grad(self, Xs: np.ndarray, Ys: np.ndarray):
        """Loss and gradient on standardised samples (no parameter update)."""
        Xs = np.ascontiguousarray(Xs, dtype=np.float32).reshape(-1, 3)
        Ys = np.ascontiguousarray(Ys, dtype=np.float32).reshape(-1, 4)
        g = np.empty(self.NPARAM, dtype=np.float32)
        loss = C.c_float()
        check(lib().fg_surrogate_loss_grad(self._h, _fptr(Xs), _fptr(Ys), len(Xs), C.byref(loss), _fptr(g)))
        return loss.value, g

    def params(self) -> np.ndarray:
        p = np.empty(self.NPARAM, dtype=np.float32)
        check(lib().fg_surrogate_get_params(self._h, _fptr(p)))
        return p

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        check(lib().fg_surrogate_set_params(self._h, _fptr(p)))

    def norm(self) -> np.ndarray:
        v = np.empty(self.NNORM, dtype=np.float32)
        check(lib().fg_surrogate_get_norm(self._h, _fptr(v)))
        return v

    def set_norm(self, v: np.ndarray) -> None:
        v = np.ascontiguousarray(v, dtype=np.float32)
        check(lib().fg_surrogate_set_norm(self._h, _fptr(v)))

    def save(self, path: str) -> None:
        """The trained network (FP32 parameters and the input / output normalisation) as .npz."""
        np.savez(path, params=self.params(), norm=self.norm(), layout=np.array([self.NPARAM, self.NNORM]))

    @classmethod
    def load(cls, path: str, device: int = 0) -> "Surrogate":
        """A surrogate with the parameters and normalisation saved by `save` (ready to predict
        and to attach to a solver; set_data is needed only to train further)."""
        d = np.load(path)
        if list(d["layout"]) != [cls.NPARAM, cls.NNORM]:
            raise ValueError(f"{path}: network layout {list(d['layout'])} differs from {[cls.NPARAM, cls.NNORM]}")
        g = cls(device=device)
        g.set_params(d["params"])
        g.set_norm(d["norm"])
        return g

    def predict(self, X: np.ndarray):
        """Tensor-core forward of raw inputs: (outputs [n][4], in-hull flags [n])."""
        X = np.ascontiguousarray(X, dtype=np.float32).reshape(-1, 3)
        Y = np.empty((len(X), 4), dtype=np.float32)
        hull = np.empty(len(X), dtype=np.int32)
        check(lib().fg_surrogate_predict(self._h, _fptr(X), len(X), _fptr(Y), hull.ctypes.data_as(L.PI)))
        return Y, hull.astype(bool)

    def close(self) -> None:
        if self._h:
            lib().fg_surrogate_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


FIELD_VARS = ["x", "y", "z", "avfL", "avfG", "rho", "U", "V", "W", "pressure", "temperature", "vaporMass", "gradRho"]


def read_field_dump(path: str) -> dict:
    """Read a field dump written by Solver.field_dump: {"time", "iStep", "data" [nElem][13], "names"}."""
    raw = open(path, "rb").read()
    if raw[:8] != b"FGFIELD1":
        raise ValueError(f"{path}: not a field dump")
    n, nv, istep, _ = np.frombuffer(raw, dtype=np.int32, count=4, offset=8)
    t = float(np.frombuffer(raw, dtype=np.float64, count=1, offset=24)[0])
    data = np.frombuffer(raw, dtype=np.float64, count=int(n) * int(nv), offset=32).reshape(int(n), int(nv))
    return {"time": t, "iStep": int(istep), "data": data.copy(), "names": FIELD_VARS[: int(nv)]}
