"""Seeded synthetic meshes written as Gambit neutral (.neu) files.

The files follow the grammar the reference reader accepts (DP/translator.cu:24-349): the four
section headers at column 0 with the 20-character prefixes it compares, the six counts after
five header lines, node and element lists, and boundary-condition sets whose IBCCODE maps to
the reference's codes (45 symmetry, 26 outlet, 13 inlet, 42 slip, 51 wall).

Element node order is Gambit's (tensor order for hexes, base-then-apex for pyramids, two
triangles for prisms) with positive volume, so the reference's face normals point outwards.
"""
from __future__ import annotations

import itertools
import os
from dataclasses import dataclass, field

import numpy as np

BC_CODES = {"symmetry": 45, "outlet": 26, "inlet": 13, "slip": 42, "wall": 51}

# local face node sets per element type (0-based, as the reference's face tables)
FACES = {
    4: [(1, 0, 2), (0, 1, 3), (1, 2, 3), (2, 0, 3)],
    5: [(0, 2, 3, 1), (0, 1, 4), (1, 3, 4), (3, 2, 4), (2, 0, 4)],
    6: [(0, 1, 4, 3), (1, 2, 5, 4), (2, 0, 3, 5), (0, 2, 1), (3, 4, 5)],
    8: [(0, 1, 5, 4), (1, 3, 7, 5), (3, 2, 6, 7), (2, 0, 4, 6), (1, 0, 2, 3), (4, 5, 7, 6)],
}
GAMBIT_TYPE = {4: 6, 5: 7, 6: 5, 8: 4}


@dataclass
class NeuMesh:
    nodes: np.ndarray                      # (nNodes, 3) float64
    elems: list                            # list of int arrays (nE_k, nn_k), 0-based node ids
    bcs: dict = field(default_factory=dict)  # name -> (code, el_ids 0-based, faces 0-based)

    @property
    def n_elem(self) -> int:
        return sum(len(e) for e in self.elems)


def write_neu(path: str, mesh: NeuMesh, title: str = "fooskagpu synthetic mesh") -> None:
    nodes = mesh.nodes
    n_nodes = len(nodes)
    n_elem = mesh.n_elem
    bcs = [(name, code, el, fc) for name, (code, el, fc) in mesh.bcs.items() if len(el) > 0]
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        f.write("CONTROL INFO".ljust(21) + "2.4.6\n")
        f.write("** GAMBIT NEUTRAL FILE\n")
        f.write(title + "\n")
        f.write("PROGRAM:                fooskagpu     VERSION:  2.4.6\n")
        f.write("Jan 1 2026\n")
        f.write("     NUMNP     NELEM     NGRPS    NBSETS     NDFCD     NDFVL\n")
        f.write("%10d%10d%10d%10d%10d%10d\n" % (n_nodes, n_elem, 1, len(bcs), 3, 3))
        f.write("ENDOFSECTION\n")
        f.write("NODAL COORDINATES".ljust(21) + "2.4.6\n")
        ids = np.arange(1, n_nodes + 1)
        np.savetxt(f, np.column_stack([ids, nodes]), fmt=["%10d", "%.17g", "%.17g", "%.17g"])
        f.write("ENDOFSECTION\n")
        f.write("ELEMENTS/CELLS".ljust(21) + "2.4.6\n")
        eid = 1
        for blk in mesh.elems:
            nn = blk.shape[1]
            k = len(blk)
            cols = np.column_stack([np.arange(eid, eid + k), np.full(k, GAMBIT_TYPE[nn]), np.full(k, nn), blk + 1])
            np.savetxt(f, cols, fmt="%d")
            eid += k
        f.write("ENDOFSECTION\n")
        f.write("ELEMENT GROUP".ljust(21) + "2.4.6\n")
        f.write("GROUP:          1 ELEMENTS:%11d MATERIAL:          2 NFLAGS:          1\n" % n_elem)
        f.write("                           fluid\n       0\n")
        np.savetxt(f, np.arange(1, n_elem + 1).reshape(-1, 1), fmt="%d")
        f.write("ENDOFSECTION\n")
        for name, code, el, fc in bcs:
            f.write("BOUNDARY CONDITIONS".ljust(20) + "2.4.6\n")
            f.write("%32s%8d%8d%8d%8d\n" % (name, 1, len(el), 0, code))
            types = _elem_types_of(mesh, el)
            np.savetxt(f, np.column_stack([el + 1, types, fc + 1]), fmt="%d")
            f.write("ENDOFSECTION\n")
    os.replace(tmp, path)


def _elem_types_of(mesh: NeuMesh, el: np.ndarray) -> np.ndarray:
    bounds = np.cumsum([0] + [len(b) for b in mesh.elems])
    out = np.zeros(len(el), dtype=np.int64)
    for k, blk in enumerate(mesh.elems):
        sel = (el >= bounds[k]) & (el < bounds[k + 1])
        out[sel] = GAMBIT_TYPE[blk.shape[1]]
    return out


def _lattice(nx, ny, nz, L, jitter, seed, periodic=(False, False, False)):
    i, j, k = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    idx = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1)
    h = np.array([L[0] / nx, L[1] / ny, L[2] / nz])
    pts = idx * h
    if jitter > 0:
        rng = np.random.default_rng(seed)
        interior = np.all((idx > 0) & (idx < np.array([nx, ny, nz])), axis=1)
        d = rng.uniform(-jitter, jitter, size=pts.shape) * h
        pts = pts + d * interior[:, None]
    nid = lambda a, b, c: (a * (ny + 1) + b) * (nz + 1) + c
    return pts, idx, nid


def _hex_nodes(nx, ny, nz, nid):
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    # Gambit hex order: tensor (x fastest): 0=(0,0,0) 1=(1,0,0) 2=(0,1,0) 3=(1,1,0) 4..7 at z+1
    corners = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (1, 1, 0), (0, 0, 1), (1, 0, 1), (0, 1, 1), (1, 1, 1)]
    return np.stack([nid(i + a, j + b, k + c) for (a, b, c) in corners], axis=1), (i, j, k)


def _tag_box_faces(elnodes, nn, idx, dims, side_bc):
    """Return {name: (code, el, face)} for element faces lying on the box sides.
    side_bc maps side ('x0','x1','y0','y1','z0','z1') -> bc name (or None = untagged)."""
    out = {}
    faces = FACES[nn]
    for fi, fnodes in enumerate(faces):
        fidx = idx[elnodes[:, list(fnodes)]]  # (nE, k, 3)
        for ax, lo_hi in itertools.product(range(3), (0, 1)):
            side = "xyz"[ax] + str(lo_hi)
            name = side_bc.get(side)
            if name is None:
                continue
            target = 0 if lo_hi == 0 else dims[ax]
            on = np.all(fidx[:, :, ax] == target, axis=1)
            if not np.any(on):
                continue
            el = np.nonzero(on)[0]
            code = BC_CODES[name]
            key = name
            if key in out:
                out[key] = (code, np.concatenate([out[key][1], el]), np.concatenate([out[key][2], np.full(len(el), fi)]))
            else:
                out[key] = (code, el, np.full(len(el), fi))
    return out


def box_tets(nx, ny, nz, L=(1.0, 0.1, 0.1), origin=(0.0, 0.0, 0.0), jitter=0.1, seed=20261203,
             side_bc=None, shuffle=False) -> NeuMesh:
    """Box of nx*ny*nz hexes, each split into 6 positively oriented tetrahedra along the main
    diagonal (conforming), interior nodes jittered by U(-jitter, jitter)*h (seeded)."""
    if side_bc is None:
        side_bc = {s: "slip" for s in ("x0", "x1", "y0", "y1", "z0", "z1")}
    pts, idx, nid = _lattice(nx, ny, nz, L, jitter, seed)
    pts = pts + np.asarray(origin, dtype=np.float64)
    hx, _ = _hex_nodes(nx, ny, nz, nid)
    # corner index of the hex node (a,b,c) in tensor order = a + 2b + 4c
    tets = []
    for perm in itertools.permutations(range(3)):
        path = [0]
        cur = [0, 0, 0]
        for ax in perm:
            cur[ax] = 1
            path.append(cur[0] + 2 * cur[1] + 4 * cur[2])
        t = hx[:, path]
        # orientation: sign of the permutation; swap two nodes for odd ones
        inv = sum(1 for a in range(3) for b in range(a + 1, 3) if perm[a] > perm[b])
        if inv % 2 == 1:
            t = t[:, [0, 2, 1, 3]]
        tets.append(t)
    el = np.stack(tets, axis=1).reshape(-1, 4)
    # fix any orientation (jitter keeps signs, but be safe)
    p = pts[el]
    vol = np.einsum("ij,ij->i", np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), p[:, 3] - p[:, 0])
    neg = vol < 0
    el[neg] = el[neg][:, [0, 2, 1, 3]]
    if shuffle:
        el = el[np.random.default_rng(seed + 1).permutation(len(el))]
    bcs = _tag_box_faces(el, 4, idx, (nx, ny, nz), side_bc)
    return NeuMesh(pts, [el], bcs)


def box_hexes(nx, ny, nz, L=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0), jitter=0.0, seed=20261203,
              side_bc=None, shuffle=False) -> NeuMesh:
    """Structured box of hexahedra (Gambit order).  side_bc entries of None leave the faces
    untagged (used with periodic matching)."""
    if side_bc is None:
        side_bc = {s: "slip" for s in ("x0", "x1", "y0", "y1", "z0", "z1")}
    pts, idx, nid = _lattice(nx, ny, nz, L, jitter, seed)
    pts = pts + np.asarray(origin, dtype=np.float64)
    el, _ = _hex_nodes(nx, ny, nz, nid)
    if shuffle:
        el = el[np.random.default_rng(seed + 1).permutation(len(el))]
    bcs = _tag_box_faces(el, 8, idx, (nx, ny, nz), side_bc)
    return NeuMesh(pts, [el], bcs)


def box_mixed(nx, ny, nz, L=(1.0, 1.0, 1.0), jitter=0.0, seed=20261203, side_bc=None) -> NeuMesh:
    """Box mixing all four element types: hex columns, columns of hexes split into two prisms
    (z-faces triangulated consistently) and hexes split into six pyramids around a centre node.
    Every shared face is conforming.  Used to exercise the tet/pyramid/prism/hex paths."""
    if side_bc is None:
        side_bc = {s: "slip" for s in ("x0", "x1", "y0", "y1", "z0", "z1")}
    pts, idx, nid = _lattice(nx, ny, nz, L, jitter, seed)
    hx, (i, j, k) = _hex_nodes(nx, ny, nz, nid)
    hexes, prisms, pyrs = [], [], []
    extra_pts = []
    idx_extra = []
    nbase = len(pts)
    # prisms occupy whole z-columns so their triangulated z-faces meet only prisms
    col_prism = ((i + j) % 3 == 1)
    pyr_cell = (~col_prism) & ((i + j + k) % 4 == 0)
    for c in range(len(hx)):
        h = hx[c]
        if col_prism[c]:
            # split the hex along its (0,0)-(1,1) diagonal in xy: two wedges
            prisms.append([h[0], h[1], h[3], h[4], h[5], h[7]])
            prisms.append([h[0], h[3], h[2], h[4], h[7], h[6]])
        elif pyr_cell[c]:
            ctr = pts[h].mean(axis=0)
            cid = nbase + len(extra_pts)
            extra_pts.append(ctr)
            idx_extra.append([-1, -1, -1])
            # six pyramids: base = hex face with normal pointing away from the centre
            for f in FACES[8]:
                b = [h[q] for q in f]
                # Gambit pyramid base order is tensor-like: 0,1,2,3 with 0-1 and 2-3 parallel;
                # face f lists a cycle (a,b,c,d) -> tensor order (a,b,d,c), apex last
                pyrs.append([b[0], b[1], b[3], b[2], cid])
        else:
            hexes.append(list(h))
    allp = np.concatenate([pts, np.asarray(extra_pts).reshape(-1, 3)]) if extra_pts else pts
    alli = np.concatenate([idx, np.asarray(idx_extra, dtype=idx.dtype).reshape(-1, 3)]) if idx_extra else idx
    blocks = []
    for arr, nn in ((hexes, 8), (prisms, 6), (pyrs, 5)):
        if not arr:
            continue
        a = np.asarray(arr, dtype=np.int64)
        # orient positively using the reference's volume split
        blocks.append(_orient(allp, a, nn))
    mesh = NeuMesh(allp, blocks, {})
    # boundary tags per block (global element ids)
    off = 0
    bcs = {}
    for blk in blocks:
        nn = blk.shape[1]
        t = _tag_box_faces(blk, nn, alli, (nx, ny, nz), side_bc)
        for name, (code, el, fc) in t.items():
            if name in bcs:
                bcs[name] = (code, np.concatenate([bcs[name][1], el + off]), np.concatenate([bcs[name][2], fc]))
            else:
                bcs[name] = (code, el + off, fc)
        off += len(blk)
    mesh.bcs = bcs
    return mesh


_VOLTETS = {4: [(1, 2, 3)], 5: [(1, 3, 4), (3, 2, 4)], 6: [(1, 2, 5), (1, 5, 4), (4, 5, 3)],
            8: [(1, 3, 5), (5, 3, 7), (5, 7, 4), (3, 2, 7), (7, 2, 6), (7, 6, 4)]}
_MIRROR = {5: [1, 0, 3, 2, 4], 6: [3, 4, 5, 0, 1, 2], 8: [4, 5, 6, 7, 0, 1, 2, 3]}


def _orient(pts, el, nn):
    p = pts[el]
    vol = np.zeros(len(el))
    for a, b, c in _VOLTETS[nn]:
        vol += np.einsum("ij,ij->i", np.cross(p[:, a] - p[:, 0], p[:, b] - p[:, 0]), p[:, c] - p[:, 0])
    neg = vol < 0
    if np.any(neg):
        el = el.copy()
        el[neg] = el[neg][:, _MIRROR[nn]]
    return el


def cached_neu(path_dir: str, name: str, make) -> str:
    """Write the mesh produced by make() to path_dir/name once and reuse it afterwards."""
    os.makedirs(path_dir, exist_ok=True)
    path = os.path.join(path_dir, name)
    if not os.path.exists(path):
        write_neu(path, make())
    return path
