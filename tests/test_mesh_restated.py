"""The mesh pre-processing three ways, no GPU needed: the .neu reader, the in-memory element lists
(fg_mesh_build) and the oracle's independent numpy restatement of the reference's pre-processing
(oracle/oracle_mesh.py) give bitwise the same reference-layout arrays; the oracle's library-free
case defaults equal fg_case_default; and the reference arm of the bench loads no product code."""
import math
import os
import subprocess
import sys

import numpy as np
import pytest

from fooskagpu_b200 import meshgen
from fooskagpu_b200._lib import FgCase, FgError
from fooskagpu_b200.api import Mesh, default_case
from oracle import oracle_mesh
from oracle.ref_case import reference_defaults

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
L = 2 * math.pi
MESHES = {
    "tets_shuffled": (lambda: meshgen.box_tets(5, 3, 3, shuffle=True), (0.0, 0.0, 0.0)),
    "mixed_elements": (lambda: meshgen.box_mixed(4, 4, 3), (0.0, 0.0, 0.0)),
    "periodic_hexes": (lambda: meshgen.box_hexes(6, 5, 4, L=(L, L, L), side_bc={}, shuffle=True), (L, L, L)),
    "graded_ball": (lambda: meshgen.ball_tets(6), (0.0, 0.0, 0.0)),
}


@pytest.mark.parametrize("name", list(MESHES))
def test_three_preprocessors_agree(name, tmp_path):
    make, per = MESHES[name]
    nm = make()
    p = str(tmp_path / "m.neu")
    meshgen.write_neu(p, nm)
    a = Mesh.load_neu(p, periodic=per)
    b = Mesh.build(nm.nodes, nm.elems, nm.bcs, periodic=per)
    o = oracle_mesh.build(nm.nodes, nm.elems, nm.bcs, periodic=per)
    A, B = a.arrays(), b.arrays()
    assert a.info == b.info
    assert np.array_equal(a.permutation(), b.permutation())
    for k in A:
        assert np.array_equal(A[k], B[k]), k
        assert np.array_equal(A[k], getattr(o, k)), k
    assert o.nPeriodic == a.info["nPeriodic"]


def test_build_rejects_bad_arrays():
    nm = meshgen.box_tets(2, 2, 2)
    bad = [nm.elems[0].copy()]
    bad[0][0, 0] = len(nm.nodes) + 5          # node id out of range
    with pytest.raises(FgError) as e:
        Mesh.build(nm.nodes, bad, nm.bcs)
    assert e.value.code == 3


def test_ball_is_a_graded_ball():
    nm = meshgen.ball_tets(16, radius=1e-2)
    o = oracle_mesh.build(nm.nodes, nm.elems, nm.bcs)
    rc = np.linalg.norm(o.cellCenter, axis=1)
    assert rc.max() < 1.1e-2 and np.all(o.volume > 0)                          # hexes with the centre inside
    assert abs(o.volume.sum() / (4 / 3 * math.pi * 1e-6) - 1) < 0.05            # stepped ball
    assert o.volume[rc < 2e-3].mean() < 0.1 * o.volume[rc > 8e-3].mean()        # finer at the centre
    assert set(np.unique(o.boundCond)) == {0, 2}                                # outlet surface
    # no slivers: volume against the cube of the rms edge (1 for a regular tet)
    p = nm.nodes[nm.elems[0]]
    edges = [np.linalg.norm(p[:, a] - p[:, b], axis=1) for a, b in ((0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3))]
    lrms = np.sqrt(sum(e * e for e in edges) / 6)
    v = np.einsum("ij,ij->i", np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), p[:, 3] - p[:, 0]) / 6
    assert (6 * math.sqrt(2) * v / lrms ** 3).min() > 0.01
    assert abs(meshgen.ball_spacing(16, 0.0) - 1e-2 * 3 / math.sinh(3) * 2 / 16) < 1e-15


def test_jet_cylinder_mixed_and_conforming():
    nm = meshgen.jet_cylinder(n=24, nz_prism=2, nz_tet=3)
    o = oracle_mesh.build(nm.nodes, nm.elems, nm.bcs)       # raises on an open (non-conforming) face
    assert [b.shape[1] for b in nm.elems] == [6, 4]
    ntri = len(nm.elems[0]) // 2
    assert len(nm.elems[1]) == 3 * 3 * ntri and o.nElem == ntri * (2 + 3 * 3)
    R, Lz = 20 * 0.2e-3, 100 * 0.2e-3
    assert abs(o.volume.sum() / (math.pi * R * R * Lz) - 1) < 0.05                # stepped rim
    codes = {k: v[0] for k, v in nm.bcs.items()}
    assert codes == {"inlet": 13, "wall": 51, "outlet": 26, "slip": 42}


def test_reference_defaults_equal_fg_case_default():
    a, b = reference_defaults(), default_case()
    for k, _ in FgCase._fields_:
        x, y = getattr(a, k), getattr(b, k)
        if hasattr(x, "__len__"):
            x, y = list(x), list(y)
        assert x == y, k


def test_reference_arm_loads_no_product_code():
    code = ("import sys; sys.argv=['bench.py','--impl','reference','--steps','1','--warmup','1','--n','8',"
            "'--no-ref-gpu']; sys.path.insert(0,'.'); import bench; bench.main(); "
            "print('PRODUCT' if 'libfooskagpu' in open('/proc/self/maps').read() else 'CLEAN')")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip().splitlines()[-1] == "CLEAN"
    assert '"impl": "reference"' in r.stdout
