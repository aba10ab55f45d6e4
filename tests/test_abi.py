"""The C-ABI libraries load and export every symbol their headers declare (no GPU calls)."""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _declared(header: Path):
    txt = header.read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b((?:fg|orc)_[a-z0-9_]+)\s*\(", txt)))


def test_product_exports_header_symbols():
    from fooskagpu_b200 import _lib
    lib = C.CDLL(str(_lib.LIB_PATH))
    names = _declared(ROOT / "include" / "fooskagpu.h")
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding covers the whole header
    assert set(names) <= set(_lib.SIGNATURES), set(names) - set(_lib.SIGNATURES)


def test_oracle_exports_header_symbols():
    from oracle import oracle_py
    lib = C.CDLL(str(oracle_py.LIB_PATH))
    names = _declared(ROOT / "oracle" / "oracle.h")
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_case_default_matches_reference_constants():
    from fooskagpu_b200.api import default_case
    c = default_case()
    # DP/buildInput.cu:10-69
    assert c.adaptDtItr == 100 and c.rkSteps == 1 and c.chemItrMax == 40 and c.thermItrMax == 25
    assert c.gamma[0] == 2.17290 and c.pInf[0] == 114907765 and c.Cp[1] == 965.98
    assert c.chemLimit == 20e-4 and c.satTempUrf == 0.8 and c.consCalcIvar == 9


def test_no_device_means_loud_error():
    """Creating a solver without a CUDA device fails with FG_ERR_CUDA instead of falling back."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    from fooskagpu_b200 import meshgen
    from fooskagpu_b200._lib import FgError
    from fooskagpu_b200.api import Mesh, Solver, default_case
    import tempfile, os
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "m.neu")
        meshgen.write_neu(p, meshgen.box_tets(2, 2, 2, side_bc={s: "slip" for s in ("x0", "x1", "y0", "y1", "z0", "z1")}))
        m = Mesh.load_neu(p)
        with pytest.raises(FgError) as e:
            Solver(m, default_case())
        assert e.value.code == 4
