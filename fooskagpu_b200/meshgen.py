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


class _TextOut:
    """Text writes into a binary file (the numeric sections are written as bytes)."""

    def __init__(self, fb):
        self.fb = fb

    def write(self, s: str) -> None:
        self.fb.write(s.encode())


def write_neu(path: str, mesh: NeuMesh, title: str = "fooskagpu synthetic mesh") -> None:
    nodes = mesh.nodes
    n_nodes = len(nodes)
    n_elem = mesh.n_elem
    bcs = [(name, code, el, fc) for name, (code, el, fc) in mesh.bcs.items() if len(el) > 0]
    tmp = path + ".tmp"
    with open(tmp, "wb") as fb:
        f = _TextOut(fb)
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
        np.savetxt(fb, np.column_stack([ids, nodes]), fmt=["%10d", "%.17g", "%.17g", "%.17g"])
        f.write("ENDOFSECTION\n")
        f.write("ELEMENTS/CELLS".ljust(21) + "2.4.6\n")
        eid = 1
        for blk in mesh.elems:
            nn = blk.shape[1]
            k = len(blk)
            cols = np.column_stack([np.arange(eid, eid + k), np.full(k, GAMBIT_TYPE[nn]), np.full(k, nn), blk + 1])
            _write_int_rows(fb, cols)
            eid += k
        f.write("ENDOFSECTION\n")
        f.write("ELEMENT GROUP".ljust(21) + "2.4.6\n")
        f.write("GROUP:          1 ELEMENTS:%11d MATERIAL:          2 NFLAGS:          1\n" % n_elem)
        f.write("                           fluid\n       0\n")
        _write_int_rows(fb, np.arange(1, n_elem + 1))
        f.write("ENDOFSECTION\n")
        for name, code, el, fc in bcs:
            f.write("BOUNDARY CONDITIONS".ljust(20) + "2.4.6\n")
            f.write("%32s%8d%8d%8d%8d\n" % (name, 1, len(el), 0, code))
            types = _elem_types_of(mesh, el)
            _write_int_rows(fb, np.column_stack([el + 1, types, fc + 1]))
            f.write("ENDOFSECTION\n")
    os.replace(tmp, path)


def _write_int_rows(f, arr: np.ndarray, chunk: int = 1 << 18) -> None:
    """Write a 2-D array of non-negative integers as text rows "%d %d ... %d\n" (the format of
    np.savetxt(fmt="%d")), formatted with array operations in chunks: the element lists of
    multi-million-cell meshes take seconds, not the minutes of a per-value formatter."""
    arr = np.asarray(arr, dtype=np.int64)
    if arr.ndim == 1:
        arr = arr[:, None]
    if len(arr) == 0:
        return
    if arr.min() < 0:
        raise ValueError("negative integers are not written by this formatter")
    width = [max(1, len(str(int(arr[:, c].max())))) for c in range(arr.shape[1])]
    for lo in range(0, len(arr), chunk):
        a = arr[lo:lo + chunk]
        chars, keep = [], []
        for c, w in enumerate(width):
            v = a[:, c:c + 1]
            p10 = 10 ** np.arange(w - 1, -1, -1, dtype=np.int64)
            chars.append(np.full((len(a), 1), 32, dtype=np.uint8))        # separator
            keep.append(np.full((len(a), 1), c > 0))
            chars.append(((v // p10) % 10 + 48).astype(np.uint8))
            keep.append((v >= p10) | (p10 == 1))                          # drop leading zeros
        chars.append(np.full((len(a), 1), 10, dtype=np.uint8))
        keep.append(np.ones((len(a), 1), dtype=bool))
        ch = np.concatenate(chars, axis=1).ravel()
        f.write(ch[np.concatenate(keep, axis=1).ravel()].tobytes())


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
    el = _split_hexes(pts, hx)
    if shuffle:
        el = el[np.random.default_rng(seed + 1).permutation(len(el))]
    bcs = _tag_box_faces(el, 4, idx, (nx, ny, nz), side_bc)
    return NeuMesh(pts, [el], bcs)


def _split_hexes(pts, hx):
    """Each hex (Gambit tensor order) into 6 tetrahedra around its main diagonal (node 0 to node
    7), one per order in which the three axes are crossed; every lattice face is cut along the
    same diagonal from both sides, so the split is conforming.  Tets are oriented positively."""
    tets = []
    for perm in itertools.permutations(range(3)):
        path = [0]
        cur = [0, 0, 0]
        for ax in perm:
            cur[ax] = 1
            path.append(cur[0] + 2 * cur[1] + 4 * cur[2])   # tensor index a + 2b + 4c
        t = hx[:, path]
        # orientation: sign of the permutation; swap two nodes for odd ones
        inv = sum(1 for a in range(3) for b in range(a + 1, 3) if perm[a] > perm[b])
        if inv % 2 == 1:
            t = t[:, [0, 2, 1, 3]]
        tets.append(t)
    el = np.stack(tets, axis=1).reshape(-1, 4)
    # fix any orientation (jitter and mapping keep signs, but be safe)
    p = pts[el]
    vol = np.einsum("ij,ij->i", np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), p[:, 3] - p[:, 0])
    neg = vol < 0
    el[neg] = el[neg][:, [0, 2, 1, 3]]
    return el


def ball_spacing(n: int, r: float, radius: float = 10e-3, beta: float = 3.0) -> float:
    """Lattice spacing of ball_tets(n, radius, beta) along an axis at distance r from the centre."""
    xi = np.arcsinh(r / radius * np.sinh(beta)) / beta
    return float(radius * beta * np.cosh(beta * xi) / np.sinh(beta) * 2.0 / n)


def _boundary_faces(el, nn):
    """(element, local face) pairs of the faces of the elements `el` (one type, nn nodes) that no
    other element shares: the surface of the element set."""
    keys, which = [], []
    for fi, fn in enumerate(FACES[nn]):
        f = np.sort(el[:, list(fn)], axis=1).astype(np.int64)
        k = np.zeros(len(el), dtype=np.int64)
        for c in range(f.shape[1]):
            k = k * (1 << 21) + f[:, c]
        keys.append(k)
        which.append(np.stack([np.arange(len(el)), np.full(len(el), fi)], axis=1))
    keys = np.concatenate(keys)
    which = np.concatenate(which)
    _, inv, cnt = np.unique(keys, return_inverse=True, return_counts=True)
    once = cnt[inv] == 1
    return which[once, 0], which[once, 1]


def ball_tets(n: int, radius: float = 10e-3, beta: float = 3.0, jitter: float = 0.1, seed: int = 20261203,
              bc: str = "outlet", shuffle: bool = False) -> NeuMesh:
    """Ball of radius `radius` meshed with tetrahedra, graded toward the centre.

    Structured-then-split stand-in for a jittered Delaunay ball (no mesher is available): an
    n^3 lattice of [-1, 1]^3 stretched per axis, x = radius * sinh(beta xi) / sinh(beta) (spacing
    radius * beta / sinh(beta) * 2 / n at the centre, beta coth(beta) times that at the
    surface), interior lattice points jittered by U(-jitter, jitter) lattice spacings per axis
    (seeded); the hexes whose centre lies inside the ball are kept (a stepped surface, tagged
    with the boundary condition `bc`) and split into 6 tets each (_split_hexes): about
    (pi / 6) 6 n^3 cells.  The hexes stay close to boxes, so the tets have no slivers (a lattice
    mapped onto the sphere instead flattens the cells at the images of the cube's corners)."""
    L = (2.0, 2.0, 2.0)
    pts, idx, nid = _lattice(n, n, n, L, jitter, seed)
    x = radius * np.sinh(beta * (pts - 1.0)) / np.sinh(beta)
    hx, _ = _hex_nodes(n, n, n, nid)
    centre = x[hx].mean(axis=1)
    hx = hx[np.linalg.norm(centre, axis=1) < radius]
    used = np.unique(hx)
    remap = np.full(len(x), -1, dtype=np.int64)
    remap[used] = np.arange(len(used))
    nodes = x[used]
    el = _split_hexes(nodes, remap[hx])
    if shuffle:
        el = el[np.random.default_rng(seed + 1).permutation(len(el))]
    be, bf = _boundary_faces(el, 4)
    return NeuMesh(nodes, [el], {bc: (BC_CODES[bc], be, bf)})


# vertex orders that bring prism vertex i (0-based; 0-2 bottom, 3-5 top, 3 above 0) to position 0
_PRISM_ROT = np.array([[0, 1, 2, 3, 4, 5], [1, 2, 0, 4, 5, 3], [2, 0, 1, 5, 3, 4],
                       [3, 5, 4, 0, 2, 1], [4, 3, 5, 1, 0, 2], [5, 4, 3, 2, 1, 0]])


def _split_prisms(pts, pr):
    """Prisms (rows of 6 node ids, bottom triangle then the nodes above it) into 3 tetrahedra each
    by the global-index rule of Dompierre et al. (1999, "How to subdivide pyramids, prisms and
    hexahedra into tetrahedra"): every quadrilateral face is cut along the diagonal through its
    lowest node id, the same choice from both sides, so the split is conforming with neighbouring
    split prisms, and the two triangles stay faces (conforming with unsplit prisms above/below).
    Tets are oriented positively."""
    r = _PRISM_ROT[np.argmin(pr, axis=1)]
    v = np.take_along_axis(pr, r, axis=1)
    a = np.minimum(v[:, 1], v[:, 5]) < np.minimum(v[:, 2], v[:, 4])
    t = np.empty((len(pr), 3, 4), dtype=pr.dtype)
    t[a] = np.stack([v[a][:, [0, 1, 2, 5]], v[a][:, [0, 1, 5, 4]], v[a][:, [0, 4, 5, 3]]], axis=1)
    b = ~a
    t[b] = np.stack([v[b][:, [0, 1, 2, 4]], v[b][:, [0, 4, 2, 5]], v[b][:, [0, 4, 5, 3]]], axis=1)
    el = t.reshape(-1, 4)
    p = pts[el]
    vol = np.einsum("ij,ij->i", np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), p[:, 3] - p[:, 0])
    neg = vol < 0
    el[neg] = el[neg][:, [0, 2, 1, 3]]
    return el


def jet_cylinder(n: int = 228, nz_prism: int = 100, nz_tet: int = 100, diameter: float = 0.2e-3,
                 radius_d: float = 20.0, length_d: float = 100.0, beta: float = 3.0, jitter: float = 0.1,
                 seed: int = 20261203) -> NeuMesh:
    """Cylinder of radius radius_d * D and length length_d * D along z, meshed by extrusion: a
    disk of triangles (an n x n lattice of [-1, 1]^2 stretched per axis toward the axis,
    x = R sinh(beta xi) / sinh(beta), interior points jittered by U(-jitter, jitter) lattice
    spacings (seeded); the lattice squares whose centre lies inside radius R are kept, a stepped
    rim, and split into 2 triangles each), extruded through nz_prism + nz_tet layers of equal
    thickness (interior layer heights jittered the same way).  The first nz_prism layers are
    prisms, the rest prisms split into 3 tets each (_split_prisms).  Boundaries: the z = 0 disk is
    an inlet inside radius D / 2 and a wall outside it; z = length is an outlet; the side is a
    slip wall.  (A lattice mapped onto the round disk would flatten the cells at the images of the
    square's corners.)"""
    R = radius_d * diameter
    Lz = length_d * diameter
    rng = np.random.default_rng(seed)
    i, j = np.meshgrid(np.arange(n + 1), np.arange(n + 1), indexing="ij")
    i, j = i.ravel(), j.ravel()
    xi = np.stack([i, j], axis=1) * (2.0 / n) - 1.0
    edge = (i == 0) | (i == n) | (j == 0) | (j == n)
    xi = xi + rng.uniform(-jitter, jitter, size=xi.shape) * (2.0 / n) * (~edge)[:, None]
    xy_all = R * np.sinh(beta * xi) / np.sinh(beta)
    nid2 = lambda a, b: a * (n + 1) + b
    a0, b0 = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    a0, b0 = a0.ravel(), b0.ravel()
    q00, q10, q01, q11 = nid2(a0, b0), nid2(a0 + 1, b0), nid2(a0, b0 + 1), nid2(a0 + 1, b0 + 1)
    keep = np.linalg.norm(0.25 * (xy_all[q00] + xy_all[q10] + xy_all[q01] + xy_all[q11]), axis=1) < R
    q00, q10, q01, q11 = q00[keep], q10[keep], q01[keep], q11[keep]
    tri = np.concatenate([np.stack([q00, q10, q11], axis=1), np.stack([q00, q11, q01], axis=1)])
    used = np.unique(tri)
    remap = np.full(len(xy_all), -1, dtype=np.int64)
    remap[used] = np.arange(len(used))
    tri = remap[tri]
    xy = xy_all[used]
    # counter-clockwise in (x, y), so a prism extruded along +z has positive volume
    e1, e2 = xy[tri[:, 1]] - xy[tri[:, 0]], xy[tri[:, 2]] - xy[tri[:, 0]]
    cw = e1[:, 0] * e2[:, 1] - e1[:, 1] * e2[:, 0] < 0
    tri[cw] = tri[cw][:, [0, 2, 1]]
    # rim: the edges that belong to one triangle only
    ed = np.sort(np.concatenate([tri[:, [0, 1]], tri[:, [1, 2]], tri[:, [2, 0]]]), axis=1)
    ek = ed[:, 0] * len(xy) + ed[:, 1]
    uk, cnt = np.unique(ek, return_counts=True)
    rim_keys = uk[cnt == 1]
    rim = np.zeros(len(xy), dtype=bool)
    rim[rim_keys // len(xy)] = True
    rim[rim_keys % len(xy)] = True
    nz = nz_prism + nz_tet
    z = np.linspace(0.0, Lz, nz + 1)
    z[1:-1] += rng.uniform(-jitter, jitter, size=nz - 1) * (Lz / nz)
    n2 = len(xy)
    nodes = np.empty((n2 * (nz + 1), 3))
    for k in range(nz + 1):
        nodes[k * n2:(k + 1) * n2, :2] = xy
        nodes[k * n2:(k + 1) * n2, 2] = z[k]
    ntri = len(tri)
    lay = np.arange(nz)
    pr = (tri[None, :, :] + (lay * n2)[:, None, None])                    # (nz, ntri, 3) bottom
    pr = np.concatenate([pr, pr + n2], axis=2).reshape(-1, 6)             # layer-major prisms
    prisms = pr[:nz_prism * ntri]
    tets = _split_prisms(nodes, pr[nz_prism * ntri:])
    blocks = [prisms, tets]
    # boundary faces, searched only among the elements that can have one: the first and last
    # layer and the columns over disk triangles with a rim edge
    kz = np.repeat(np.arange(nz + 1), n2)
    rim_tri = np.nonzero(rim[tri].sum(axis=1) >= 2)[0]
    lay_t = np.arange(nz_tet)
    cand = [np.unique(np.concatenate([np.arange(ntri), (np.arange(nz_prism)[:, None] * ntri + rim_tri).ravel()]))
            if nz_prism else np.zeros(0, dtype=np.int64),
            np.unique(np.concatenate([(((nz_tet - 1) * ntri + np.arange(ntri))[:, None] * 3 + np.arange(3)).ravel(),
                                      ((lay_t[:, None] * ntri + rim_tri)[:, :, None] * 3 + np.arange(3)).ravel()]))
            if nz_tet else np.zeros(0, dtype=np.int64)]
    bcs = {}
    off = 0
    for blk, cnd in zip(blocks, cand):
        nn = blk.shape[1]
        for fi, fnodes in enumerate(FACES[nn]):
            fn = blk[cnd][:, list(fnodes)]
            bottom = np.all(kz[fn] == 0, axis=1)
            top = np.all(kz[fn] == nz, axis=1)
            # a side face spans one rim edge: its nodes project onto the two ends of a rim edge
            f2 = fn % n2
            lo2, hi2 = f2.min(axis=1), f2.max(axis=1)
            two = np.all((f2 == lo2[:, None]) | (f2 == hi2[:, None]), axis=1) & (lo2 != hi2)
            side = two & np.isin(lo2 * n2 + hi2, rim_keys)
            rc = np.linalg.norm(xy[f2].mean(axis=1), axis=1)
            for name, sel in (("inlet", bottom & (rc < 0.5 * diameter)), ("wall", bottom & (rc >= 0.5 * diameter)),
                              ("outlet", top), ("slip", side & ~bottom & ~top)):
                el = cnd[np.nonzero(sel)[0]]
                if not len(el):
                    continue
                code = BC_CODES[name]
                if name in bcs:
                    bcs[name] = (code, np.concatenate([bcs[name][1], el + off]),
                                 np.concatenate([bcs[name][2], np.full(len(el), fi)]))
                else:
                    bcs[name] = (code, el + off, np.full(len(el), fi))
        off += len(blk)
    return NeuMesh(nodes, blocks, bcs)


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
