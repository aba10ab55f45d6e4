"""Mesh pre-processing (host C++ through the C ABI; no GPU needed)."""
import math
import os

import numpy as np
import pytest

from fooskagpu_b200 import meshgen
from fooskagpu_b200._lib import FgError
from fooskagpu_b200.api import Mesh

SLIP = {s: "slip" for s in ("x0", "x1", "y0", "y1", "z0", "z1")}


def _closure(a, nE):
    clo = np.zeros((nE, 3))
    nA = a["n"] * a["area"][:, None]
    np.add.at(clo, a["fc2el"][:, 0], nA)
    inner = a["boundCond"] == 0
    np.add.at(clo, a["fc2el"][inner, 1], -nA[inner])
    return np.abs(clo).max() / np.sqrt(a["area"].max())


@pytest.mark.parametrize("kind", ["tets", "hexes", "mixed"])
def test_geometry_closed_and_positive(kind, tmp_path):
    if kind == "tets":
        mm = meshgen.box_tets(5, 3, 2, L=(1.0, 0.6, 0.4), jitter=0.1, side_bc=SLIP)
    elif kind == "hexes":
        mm = meshgen.box_hexes(5, 3, 2, L=(1.0, 0.6, 0.4), jitter=0.0, side_bc=SLIP)  # planar faces: the reference geometry is exact only then
    else:
        mm = meshgen.box_mixed(4, 4, 3, L=(1.0, 1.0, 0.6), side_bc=SLIP)
    p = str(tmp_path / "m.neu")
    meshgen.write_neu(p, mm)
    m = Mesh.load_neu(p)
    a = m.arrays()
    nE = m.n_elem
    assert nE == mm.n_elem
    assert np.all(a["volume"] > 0)
    box = {"tets": 1.0 * 0.6 * 0.4, "hexes": 1.0 * 0.6 * 0.4, "mixed": 0.6}[kind]
    assert abs(a["volume"].sum() - box) < 1e-12 * box
    assert _closure(a, nE) < 1e-12
    # unit normals, orthonormal frames
    for k in ("n", "nt1", "nt2"):
        assert np.allclose(np.linalg.norm(a[k], axis=1), 1.0, atol=1e-14)
    assert np.abs(np.einsum("ij,ij->i", a["n"], a["nt1"])).max() < 1e-12
    # every boundary face sits on the box and points outwards
    bnd = a["boundCond"] != 0
    fc = a["fcCenter"][bnd]
    lo, hi = np.zeros(3), np.array({"tets": (1.0, 0.6, 0.4), "hexes": (1.0, 0.6, 0.4), "mixed": (1.0, 1.0, 0.6)}[kind])
    on = np.isclose(fc, lo, atol=1e-12) | np.isclose(fc, hi, atol=1e-12)
    assert np.all(on.any(axis=1))
    out = (a["fcCenter"][bnd] - a["cellCenter"][a["fc2el"][bnd, 0]])
    assert np.all(np.einsum("ij,ij->i", out, a["n"][bnd]) > 0)
    # owner is the lower element index (reference face order)
    inner = ~bnd
    assert np.all(a["fc2el"][inner, 0] < a["fc2el"][inner, 1])
    assert m.info["nTet"] + m.info["nPyr"] + m.info["nPrism"] + m.info["nHex"] == nE
    if kind == "mixed":
        assert m.info["nPyr"] > 0 and m.info["nPrism"] > 0 and m.info["nHex"] > 0


def test_periodic_matching(tmp_path):
    L = 2 * math.pi
    p = str(tmp_path / "p.neu")
    meshgen.write_neu(p, meshgen.box_hexes(6, 5, 4, L=(L, L, L), side_bc={}, shuffle=True))
    m = Mesh.load_neu(p, periodic=(L, L, L))
    a = m.arrays()
    assert m.info["nBoundary"] == 0
    assert m.info["nPeriodic"] == 2 * (5 * 4 + 6 * 4 + 6 * 5) // 2
    sh = a["nbShift"]
    per = np.abs(sh).max(axis=1) > 0
    assert per.sum() == m.info["nPeriodic"]
    # shifted face centre coincides with the neighbour's own face: distance to neighbour centre
    d_nb = (a["fcCenter"] + sh - a["cellCenter"][a["fc2el"][:, 1]])
    assert np.abs(d_nb).max() < 0.6 * L / 4
    assert _closure(a, m.n_elem) < 1e-12


def test_untagged_boundary_is_an_error(tmp_path):
    p = str(tmp_path / "u.neu")
    meshgen.write_neu(p, meshgen.box_hexes(3, 3, 3, side_bc={"x0": "slip"}))
    with pytest.raises(FgError) as e:
        Mesh.load_neu(p)
    assert "open boundary face" in str(e.value)


@pytest.mark.parametrize("bad", ["missing", "truncated", "badnode", "inverted"])
def test_corrupt_mesh_errors(bad, tmp_path):
    p = str(tmp_path / "c.neu")
    mm = meshgen.box_tets(3, 2, 2, side_bc=SLIP)
    if bad == "inverted":
        mm.elems[0][0] = mm.elems[0][0][[0, 2, 1, 3]]
    meshgen.write_neu(p, mm)
    txt = open(p).read()
    if bad == "missing":
        p = str(tmp_path / "nope.neu")
    elif bad == "truncated":
        open(p, "w").write(txt[: len(txt) // 2])
    elif bad == "badnode":
        open(p, "w").write(txt.replace("ELEMENTS/CELLS       2.4.6\n1 6 4 ", "ELEMENTS/CELLS       2.4.6\n1 6 4 99999 ", 1))
    with pytest.raises(FgError) as e:
        Mesh.load_neu(p)
    assert e.value.code in (2, 3)


def test_renumbering_is_a_permutation(tmp_path):
    p = str(tmp_path / "r.neu")
    meshgen.write_neu(p, meshgen.box_tets(6, 4, 3, side_bc=SLIP, shuffle=True))
    for r in ("none", "morton", "rcm"):
        m = Mesh.load_neu(p, renumber=r)
        perm = m.permutation()
        assert np.array_equal(np.sort(perm), np.arange(m.n_elem))
        if r == "none":
            assert np.array_equal(perm, np.arange(m.n_elem))


def test_smallest_meshes(tmp_path):
    """Edge sizes: a file with no elements is rejected; one cell (six boundary faces) loads and
    partitions only into one part."""
    p = str(tmp_path / "one.neu")
    meshgen.write_neu(p, meshgen.box_hexes(1, 1, 1, side_bc=SLIP))
    m = Mesh.load_neu(p)
    assert m.n_elem == 1 and m.n_fcs == 6 and m.info["nBoundary"] == 6
    assert m.partition(1, 0).n_elem == 1
    with pytest.raises(FgError, match="nParts"):
        m.partition(2, 0)
    lines = open(p).read().split("\n")
    i = next(k for k, l in enumerate(lines) if l.strip().startswith("NUMNP"))
    hdr = lines[i + 1].split()
    hdr[1] = "0"
    lines[i + 1] = " ".join(hdr)
    txt = "\n".join(lines)
    a = txt.index("ELEMENTS/CELLS")
    b = txt.index("ENDOFSECTION", a)
    q = str(tmp_path / "zero.neu")
    open(q, "w").write(txt[:a] + txt[a:].split("\n", 1)[0] + "\n" + txt[b:])
    with pytest.raises(FgError) as e:
        Mesh.load_neu(q)
    assert e.value.code == 3
