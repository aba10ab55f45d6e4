"""TEST INFRASTRUCTURE ONLY — numpy restatement of the reference's mesh pre-processing, so that
the oracle (and bench.py's reference arm) can build its mesh without the product library.

Follows, for element lists in .neu element order:
  - cell centres (plain node average) and per-element face centres in the reference's node
    order: DP/translator.cu:122-282;
  - face matching of conforming element faces (the reference compares face centres among
    elements sharing a node, DP/meshConnectivity.cu:97-128; on a conforming mesh that pairs the
    same faces as equal sorted node sets, which is what is matched here);
  - periodic pairing of open untagged faces whose centres differ by a box length (an option the
    reference lacks; the product's rule: centres equal within 1e-7 of the mesh span, modulo the
    box length);
  - face order and ownership: element faces visited in element / local-face order, a face is
    created by its first visitor (DP/buildLocalMesh.cu:263-313 with one partition);
  - normals from the first three geometry nodes, nt1 along edge 0 -> 1, nt2 = n x nt1, areas as
    triangle fans, volumes by tetra split from node 0: DP/meshProperties.cu:51-137.
Every floating-point expression is evaluated in the reference's operation order (no fused
multiply-adds in numpy), so the arrays are bitwise those of the product's own pre-processor.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

# per element type (by node count): face node lists for the centre average (DP/translator.cu)
# and for the normal / area (DP/operations.h), and the tetra split of the volume
_CENTRE = {
    4: [(1, 0, 2), (0, 1, 3), (1, 2, 3), (2, 0, 3)],
    5: [(0, 2, 3, 1), (0, 1, 4), (1, 3, 4), (3, 2, 4), (2, 0, 4)],
    6: [(0, 1, 4, 3), (1, 2, 5, 4), (2, 0, 3, 5), (0, 2, 1), (3, 4, 5)],
    8: [(0, 1, 5, 4), (1, 3, 7, 5), (3, 2, 6, 7), (2, 0, 4, 6), (1, 0, 2, 3), (4, 5, 7, 6)],
}
_GEOM = {
    4: [(1, 0, 2), (0, 1, 3), (1, 2, 3), (2, 0, 3)],
    5: [(0, 2, 3, 1), (0, 1, 4), (1, 3, 4), (3, 2, 4), (2, 0, 4)],
    6: [(0, 1, 4, 3), (2, 5, 4, 1), (0, 3, 5, 2), (0, 2, 1), (3, 4, 5)],
    8: [(0, 1, 5, 4), (3, 7, 5, 1), (2, 6, 7, 3), (2, 0, 4, 6), (2, 3, 1, 0), (6, 4, 5, 7)],
}
_VOLTETS = {4: [(1, 2, 3)], 5: [(1, 3, 4), (3, 2, 4)], 6: [(1, 2, 5), (1, 5, 4), (4, 5, 3)],
            8: [(1, 3, 5), (5, 3, 7), (5, 7, 4), (3, 2, 7), (7, 2, 6), (7, 6, 4)]}
_BC_CODE = {45: 1, 26: 2, 13: 3, 42: 4, 51: 5}


class OracleMesh:
    """Reference-layout mesh arrays (the MESH struct of DP/strdata.h:100-115) and a
    fg_mesh_view over them for the oracle."""

    def __init__(self, **arrays):
        self.__dict__.update(arrays)
        self.nElem = len(self.volume)
        self.nFcs = len(self.area)
        self._view = None

    def view(self):
        from fooskagpu_b200._lib import FgMeshView   # the struct layout only; no library is loaded
        if self._view is None:
            PD = C.POINTER(C.c_double)
            PI = C.POINTER(C.c_int32)
            v = FgMeshView()
            v.nElem, v.nFcs = self.nElem, self.nFcs
            v.fc2el = self.fc2el.ctypes.data_as(PI)
            v.boundCond = self.boundCond.ctypes.data_as(PI)
            for k in ("cellCenter", "fcCenter", "n", "nt1", "nt2", "area", "volume", "nbShift"):
                setattr(v, k, getattr(self, k).ctypes.data_as(PD))
            self._view = v
        return self._view


def build(nodes: np.ndarray, elems, bcs: dict, scale: float = 1.0, periodic=(0.0, 0.0, 0.0)) -> OracleMesh:
    """nodes (nNodes, 3); elems: list of (nE_k, nn_k) 0-based node-id blocks in element order;
    bcs: {name: (gambit code, element ids, local faces)}; periodic: box length per axis (0: none)."""
    nodes = np.asarray(nodes, dtype=np.float64) * scale
    nn = np.concatenate([np.full(len(b), b.shape[1], dtype=np.int64) for b in elems])
    nE = len(nn)
    el = np.zeros((nE, 8), dtype=np.int64)
    off = 0
    for b in elems:
        el[off:off + len(b), :b.shape[1]] = b
        off += len(b)
    elbc = np.zeros((nE, 6), dtype=np.int32)
    for _, (code, e, f) in bcs.items():
        if code in _BC_CODE:
            elbc[np.asarray(e), np.asarray(f)] = _BC_CODE[code]
    types = sorted(set(nn.tolist()))
    # ---- cell centres and element face centres (node order of the reference)
    cc = np.zeros((nE, 3))
    efc = np.zeros((nE, 6, 3))
    nfaces = np.zeros(nE, dtype=np.int64)
    for t in types:
        sel = np.nonzero(nn == t)[0]
        p = nodes[el[sel, :t]]                      # (k, t, 3)
        s = p[:, 0].copy()
        for k in range(1, t):
            s = s + p[:, k]
        cc[sel] = s / t
        nfaces[sel] = len(_CENTRE[t])
        for f, lst in enumerate(_CENTRE[t]):
            q = p[:, lst[0]].copy()
            for k in lst[1:]:
                q = q + p[:, k]
            efc[sel, f] = q / len(lst)
    # ---- conforming matching on sorted node sets of untagged element faces
    keys, slot = [], []
    for t in types:
        sel = np.nonzero(nn == t)[0]
        for f, lst in enumerate(_GEOM[t]):
            open_ = sel[elbc[sel, f] == 0]
            k = np.full((len(open_), 4), -1, dtype=np.int64)
            k[:, :len(lst)] = np.sort(el[open_][:, list(lst)], axis=1)
            keys.append(k)
            slot.append(open_ * 6 + f)
    keys = np.concatenate(keys)
    slot = np.concatenate(slot)
    order = np.lexsort(keys.T[::-1])
    ks, ss = keys[order], slot[order]
    same = np.all(ks[1:] == ks[:-1], axis=1)
    neig = np.full(nE * 6, -1, dtype=np.int64)
    neigfc = np.zeros(nE * 6, dtype=np.int64)
    a, b = ss[:-1][same], ss[1:][same]
    neig[a], neigfc[a] = b // 6, b % 6
    neig[b], neigfc[b] = a // 6, a % 6
    matched = np.zeros(len(ss), dtype=bool)
    matched[:-1] |= same
    matched[1:] |= same
    unmatched = np.sort(ss[~matched])
    shift = np.zeros((nE * 6, 3))
    n_periodic = 0
    L = np.asarray(periodic, dtype=np.float64) * scale
    if len(unmatched) and np.any(L > 0):
        lo, hi = nodes.min(axis=0), nodes.max(axis=0)
        span = float((hi - lo).max())
        tol = 1e-7 * (span if span > 0 else 1.0)
        c = efc.reshape(-1, 3)[unmatched]
        w = c.copy()
        for d in range(3):
            if L[d] > 0:
                v = c[:, d] - lo[d]
                v = v - L[d] * np.floor(v / L[d] + 0.5 * tol / L[d])
                v = np.where(v > L[d] - tol, v - L[d], v)
                w[:, d] = v
        q = np.round(w / (4 * tol)).astype(np.int64)
        o2 = np.lexsort(q.T[::-1])
        qs = q[o2]
        pair = np.all(qs[1:] == qs[:-1], axis=1)
        i1, i2 = o2[:-1][pair], o2[1:][pair]
        a, b = unmatched[i1], unmatched[i2]
        neig[a], neigfc[a] = b // 6, b % 6
        neig[b], neigfc[b] = a // 6, a % 6
        sh = efc.reshape(-1, 3)[b] - efc.reshape(-1, 3)[a]
        qd = np.where(L > 0, L * np.round(sh / np.where(L > 0, L, 1.0)), 0.0)
        shift[a] = qd
        shift[b] = -qd
        n_periodic = len(a)
        done = np.zeros(len(unmatched), dtype=bool)
        done[i1] = done[i2] = True
        unmatched = unmatched[~done]
    if len(unmatched):
        raise ValueError(f"open boundary face without a boundary condition: element {unmatched[0] // 6 + 1}")
    # ---- reference face order: element faces in (element, local face) order, first visitor owns
    ef = np.arange(nE * 6)
    e_of, f_of = ef // 6, ef % 6
    valid = f_of < nfaces[e_of]
    create = valid & ((neig == -1) | (neig > e_of))
    src = ef[create]
    fc2el = np.stack([src // 6, neig[src]], axis=1).astype(np.int32)
    fc2elfc = np.stack([src % 6, np.where(neig[src] == -1, 0, neigfc[src])], axis=1)
    bound = elbc.reshape(-1)[src].astype(np.int32)
    nF = len(src)
    # ---- face geometry from the owner's local face (DP/meshProperties.cu:51-101)
    fcc = efc.reshape(-1, 3)[src].copy()
    n = np.zeros((nF, 3))
    t1 = np.zeros((nF, 3))
    t2 = np.zeros((nF, 3))
    area = np.zeros(nF)
    e0, lf = src // 6, src % 6
    for t in types:
        for f, lst in enumerate(_GEOM[t]):
            sel = np.nonzero((nn[e0] == t) & (lf == f))[0]
            if not len(sel):
                continue
            P = nodes[el[e0[sel]][:, list(lst)]]          # (k, cnt, 3)
            x, y, z = P[:, :, 0], P[:, :, 1], P[:, :, 2]
            A = (y[:, 1] - y[:, 0]) * (z[:, 2] - z[:, 0]) - (y[:, 2] - y[:, 0]) * (z[:, 1] - z[:, 0])
            B = (x[:, 1] - x[:, 0]) * (z[:, 2] - z[:, 0]) - (x[:, 2] - x[:, 0]) * (z[:, 1] - z[:, 0])
            Cc = (x[:, 1] - x[:, 0]) * (y[:, 2] - y[:, 0]) - (x[:, 2] - x[:, 0]) * (y[:, 1] - y[:, 0])
            nrm = np.sqrt(A * A + B * B + Cc * Cc)
            nv = np.stack([A / nrm, -B / nrm, Cc / nrm], axis=1)
            n[sel] = nv
            d0, d1, d2 = x[:, 1] - x[:, 0], y[:, 1] - y[:, 0], z[:, 1] - z[:, 0]
            nrm1 = np.sqrt(d0 * d0 + d1 * d1 + d2 * d2)
            tv = np.stack([d0 / nrm1, d1 / nrm1, d2 / nrm1], axis=1)
            t1[sel] = tv
            a2 = nv[:, 1] * tv[:, 2] - tv[:, 1] * nv[:, 2]
            b2 = nv[:, 0] * tv[:, 2] - tv[:, 0] * nv[:, 2]
            c2 = nv[:, 0] * tv[:, 1] - tv[:, 0] * nv[:, 1]
            nrm2 = np.sqrt(a2 * a2 + b2 * b2 + c2 * c2)
            t2[sel] = np.stack([a2 / nrm2, -b2 / nrm2, c2 / nrm2], axis=1)
            ar = np.zeros(len(sel))
            for it in range(len(lst) - 2):
                dx1, dx2 = x[:, 1 + it] - x[:, 0], x[:, 2 + it] - x[:, 0]
                dy1, dy2 = y[:, 1 + it] - y[:, 0], y[:, 2 + it] - y[:, 0]
                dz1, dz2 = z[:, 1 + it] - z[:, 0], z[:, 2 + it] - z[:, 0]
                u = dy1 * dz2 - dz1 * dy2
                v = dz1 * dx2 - dx1 * dz2
                ww = dx1 * dy2 - dy1 * dx2
                ar = ar + np.abs(0.5 * np.sqrt(u * u + v * v + ww * ww))
            area[sel] = ar
    nbshift = shift[src]
    # ---- volumes by tetra split from node 0 (DP/meshProperties.cu:102-137)
    vol = np.zeros(nE)
    for t in types:
        sel = np.nonzero(nn == t)[0]
        p = nodes[el[sel, :t]]
        p0 = p[:, 0]
        acc = np.zeros(len(sel))
        for tet in _VOLTETS[t]:
            dx = [p[:, i, 0] - p0[:, 0] for i in tet]
            dy = [p[:, i, 1] - p0[:, 1] for i in tet]
            dz = [p[:, i, 2] - p0[:, 2] for i in tet]
            c0 = dy[0] * dz[1] - dz[0] * dy[1]
            c1 = dz[0] * dx[1] - dx[0] * dz[1]
            c2 = dx[0] * dy[1] - dy[0] * dx[1]
            acc = acc + (c0 * dx[2] + c1 * dy[2] + c2 * dz[2]) / 6.0
        vol[sel] = acc
    if not np.all(vol > 0):
        raise ValueError("element with non-positive volume")
    return OracleMesh(fc2el=np.ascontiguousarray(fc2el), fc2elFc=fc2elfc.astype(np.int32),
                      boundCond=np.ascontiguousarray(bound), cellCenter=np.ascontiguousarray(cc),
                      fcCenter=np.ascontiguousarray(fcc), n=n, nt1=t1, nt2=t2, area=area, volume=vol,
                      nbShift=np.ascontiguousarray(nbshift), nPeriodic=n_periodic)
