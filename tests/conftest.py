import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests of the device path")


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session", autouse=True)
def _built():
    from fooskagpu_b200 import build
    build.build_all()
    yield


@pytest.fixture(scope="session")
def meshdir(tmp_path_factory):
    return tmp_path_factory.mktemp("meshes")


def rel_err(a, b, axis=0, floor=None):
    """Per-variable max error normalised by the variable's max magnitude.  `floor` (scalar or
    per-variable) bounds the normaliser from below, for quantities that are identically zero
    up to round-off in a case (e.g. the residual of a uniform volume fraction)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.abs(b).max(axis=axis)
    if floor is not None:
        scale = np.maximum(scale, floor)
    scale = np.maximum(scale, 1e-300)
    return np.abs(a - b).max(axis=axis) / scale


MOMENTUM = (3, 4, 5)


def _group_scale(b):
    """Per-variable scale of a (cells, 10) array; momentum components share the vector scale."""
    sc = np.abs(b).max(axis=0).astype(np.float64)
    if b.shape[1] >= 6:
        sc[list(MOMENTUM)] = sc[list(MOMENTUM)].max()
    return sc


def state_err(a, b):
    """Max |a - b| per variable over the state's own magnitude (momentum as a vector)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.abs(a - b).max(axis=0) / np.maximum(_group_scale(b), 1e-300)


def rate_err(a, b, U, floor=1e-10):
    """Max |a - b| per variable for rate-like arrays (residuals, increments), normalised by the
    variable's own range and, from below, by `floor` times the case's largest relative rate
    times the variable's state magnitude — variables that are constant in a case (alpha in the
    single-phase ones) have round-off-only rates on both sides."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    Us = _group_scale(np.asarray(U, dtype=np.float64))
    bs = _group_scale(b)
    rate = np.max([bs[v] / Us[v] for v in (1, 2, 8) if Us[v] > 0])
    scale = np.maximum(bs, floor * rate * Us)
    return np.abs(a - b).max(axis=0) / np.maximum(scale, 1e-300)
