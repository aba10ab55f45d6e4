"""Space-filling-curve partition of a mesh (host C++ through the C ABI; no GPU needed): the parts'
own cells cover the mesh once; each part's first ghost layer is exactly the other parts' face
neighbours of its own cells and its second layer their further neighbours; the part keeps every
face of its own and first-layer cells with the whole mesh's orientation and geometry; and the
send list of part p to q (p's cells within two face hops of q's) matches the receive list of q
from p record for record."""
import math

import numpy as np
import pytest

from fooskagpu_b200 import meshgen
from fooskagpu_b200._lib import FgError
from fooskagpu_b200.api import Mesh

ALL_BC = {"x0": "inlet", "x1": "outlet", "y0": "wall", "y1": "slip", "z0": "symmetry", "z1": "slip"}


def _mesh(kind, tmp_path):
    p = str(tmp_path / f"{kind}.neu")
    per = (0.0, 0.0, 0.0)
    if kind == "tets":
        meshgen.write_neu(p, meshgen.box_tets(7, 4, 3, L=(0.7, 0.4, 0.3), jitter=0.1, side_bc=ALL_BC, shuffle=True))
    elif kind == "hex_periodic":
        L = 2 * math.pi
        meshgen.write_neu(p, meshgen.box_hexes(6, 5, 4, L=(L, L, L), side_bc={}, shuffle=True))
        per = (L, L, L)
    else:
        meshgen.write_neu(p, meshgen.box_mixed(4, 4, 3, L=(1.0, 1.0, 0.6), side_bc=ALL_BC))
    return Mesh.load_neu(p, scale=1.0, periodic=per)


def _faces_key(a, cg):
    """(owner, neighbour-or-minus-bc) of each face in whole-mesh .neu numbering."""
    fc = a["fc2el"]
    inner = a["boundCond"] == 0
    own = cg[fc[:, 0]]
    nb = np.where(inner, cg[np.where(inner, fc[:, 1], 0)], -a["boundCond"])
    return own, nb


@pytest.mark.parametrize("P", [1, 2, 3, 5])
@pytest.mark.parametrize("kind", ["tets", "hex_periodic", "mixed"])
def test_partition_maps(kind, P, tmp_path):
    g = _mesh(kind, tmp_path)
    ga = g.arrays()
    n = g.n_elem
    new2old = g.permutation()
    gown, gnb = _faces_key(ga, np.arange(n))
    inner = ga["boundCond"] == 0
    parts = [g.partition(P, p) for p in range(P)]
    maps = [m.partition_maps() for m in parts]
    covered = np.concatenate([mp["cell_global"][:m.n_owned] for m, mp in zip(parts, maps)])
    assert np.array_equal(covered, new2old)   # contiguous device-order ranges, in part order
    owner_part = np.empty(n, np.int64)
    for p, (m, mp) in enumerate(zip(parts, maps)):
        owner_part[mp["cell_global"][:m.n_owned]] = p
    for p, (m, mp) in enumerate(zip(parts, maps)):
        info = m.part_info
        assert (info["nParts"], info["part"], info["nOwned"]) == (P, p, m.n_owned)
        assert info["nGhost"] == m.n_elem - m.n_owned
        cg = mp["cell_global"]
        a = m.arrays()
        # per-cell data is the whole mesh's
        assert np.array_equal(a["volume"], ga["volume"][cg])
        assert np.array_equal(a["cellCenter"], ga["cellCenter"][cg])
        n1 = info["nGhost1"]
        # ghost layers: the other parts' face neighbours of own cells, then their neighbours outside
        # both, each sorted by device order
        nbr = [set() for _ in range(n)]
        for f in np.flatnonzero(inner):
            nbr[gown[f]].add(int(gnb[f]))
            nbr[gnb[f]].add(int(gown[f]))
        own_set = set(cg[:m.n_owned].tolist())
        layer1 = set()
        for x in own_set:
            layer1 |= {y for y in nbr[x] if owner_part[y] != p}
        layer2 = set()
        for x in layer1:
            layer2 |= {y for y in nbr[x] if y not in own_set and y not in layer1}
        g1, g2 = cg[m.n_owned:m.n_owned + n1], cg[m.n_owned + n1:]
        assert set(g1.tolist()) == layer1 and len(g1) == len(layer1)
        assert set(g2.tolist()) == layer2 and len(g2) == len(layer2)
        old2new = np.argsort(new2old)
        assert np.all(np.diff(old2new[g1]) > 0) and np.all(np.diff(old2new[g2]) > 0)
        # faces: exactly those touching an own or first-layer cell, in whole-mesh order, same
        # orientation / geometry
        inner_cells = own_set | layer1
        mine = np.array([int(gown[f]) in inner_cells or (bool(inner[f]) and int(gnb[f]) in inner_cells)
                         for f in range(len(gown))])
        sel = np.flatnonzero(mine)
        own, nb = _faces_key(a, cg)
        assert np.array_equal(own, gown[sel]) and np.array_equal(nb, gnb[sel])
        for k in ("n", "area", "fcCenter", "nbShift", "boundCond"):
            assert np.array_equal(a[k], ga[k][sel]), k
        # received: every ghost once, grouped by owning part, in device order
        rc = mp["recv_cells"]
        assert np.array_equal(np.sort(rc), np.arange(m.n_owned, m.n_elem))
        assert np.all(np.diff(old2new[cg[rc]]) > 0)
        assert mp["recv_start"][p] == mp["recv_start"][p + 1] and mp["send_start"][p] == mp["send_start"][p + 1]
    # what p sends to q is what q receives from p, in the same order
    for p in range(P):
        for q in range(P):
            sp, sq = maps[p], maps[q]
            sent = sp["cell_global"][sp["send_cells"][sp["send_start"][q]:sp["send_start"][q + 1]]]
            got = sq["cell_global"][sq["recv_cells"][sq["recv_start"][p]:sq["recv_start"][p + 1]]]
            assert np.array_equal(sent, got), (p, q)
            assert np.all(owner_part[got] == p)


def test_single_part_is_the_mesh(tmp_path):
    g = _mesh("tets", tmp_path)
    m = g.partition(1, 0)
    assert m.n_owned == m.n_elem == g.n_elem and m.part_info["nGhost"] == 0
    assert m.n_fcs == g.n_fcs


def test_whole_mesh_reports_one_part(tmp_path):
    g = _mesh("tets", tmp_path)
    assert g.part_info == {"nParts": 1, "part": 0, "nOwned": g.n_elem, "nGhost": 0, "nSend": 0, "nRecv": 0,
                           "nGhost1": 0}
    mp = g.partition_maps()
    assert np.array_equal(mp["cell_global"], np.arange(g.n_elem))


def test_partition_errors(tmp_path):
    g = _mesh("tets", tmp_path)
    with pytest.raises(FgError, match="nParts"):
        g.partition(0, 0)
    with pytest.raises(FgError, match="nParts"):
        g.partition(2, 2)
    with pytest.raises(FgError, match="nParts"):
        g.partition(g.n_elem + 1, 0)
    with pytest.raises(FgError, match="already a part"):
        g.partition(2, 0).partition(2, 0)
