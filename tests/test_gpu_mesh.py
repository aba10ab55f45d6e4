"""The GPU mesh pre-processor produces the host path's arrays exactly: face order and owners,
boundary codes, face and cell geometry, periodic image offsets and the Morton device order."""
import math
import os

import numpy as np
import pytest

from gpu_cases import make
from fooskagpu_b200 import meshgen
from fooskagpu_b200.api import Mesh

pytestmark = pytest.mark.gpu

KEYS = ["fc2el", "boundCond", "cellCenter", "fcCenter", "n", "nt1", "nt2", "area", "volume", "nbShift"]


def _same(path, periodic=(0.0, 0.0, 0.0)):
    a = Mesh.load_neu(path, scale=1.0, periodic=periodic)
    b = Mesh.load_neu(path, scale=1.0, periodic=periodic, gpu=True)
    assert a.info == b.info
    A, B = a.arrays(), b.arrays()
    for k in KEYS:
        assert np.array_equal(A[k], B[k]), k
    assert np.array_equal(a.permutation(), b.permutation())
    a.close()
    b.close()


@pytest.mark.parametrize("name", ["tet_ref", "mixed_ref_rk3", "tet_sod"])
def test_gpu_preprocessor_matches_host(name, meshdir):
    make(name, meshdir)   # writes the mesh file
    _same(str(meshdir / (name + ".neu")))


def test_gpu_preprocessor_periodic_shuffled(meshdir):
    L = 2 * math.pi
    path = str(meshdir / "pre_hex24.neu")
    if not os.path.exists(path):
        meshgen.write_neu(path, meshgen.box_hexes(24, 20, 16, L=(L, L, L), side_bc={}, shuffle=True))
    _same(path, periodic=(L, L, L))


def test_gpu_preprocessor_rejects_open_faces(meshdir):
    path = str(meshdir / "open.neu")
    meshgen.write_neu(path, meshgen.box_hexes(4, 4, 4, side_bc={"x0": "slip", "x1": "slip"}))
    with pytest.raises(Exception, match="open boundary face"):
        Mesh.load_neu(path, scale=1.0, gpu=True)
