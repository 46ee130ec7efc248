import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import __graft_entry__  # noqa: E402

tp = __graft_entry__.load_package()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except ImportError:
        return False


def pytest_collection_modifyitems(config, items):
    if has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(ROOT, "tests", "golden", "golden_cases.json")) as f:
        return json.load(f)


def unhex(rows):
    return np.array([[float.fromhex(v) for v in row] for row in rows], dtype=np.float64)


def col_rel_err(a, ref):
    """max over columns of max|a - ref| / max|ref| (per-coordinate relative error)."""
    scale = np.abs(ref).max(axis=0)
    scale = np.where(scale > 0, scale, 1.0)
    return float((np.abs(a - ref).max(axis=0) / scale).max())


def golden_lattice(case):
    """The Lattice of a golden case: its element records and misalignment rows."""
    rows = [{k: [float.fromhex(v) for v in row[k]] for k in ("t1", "t2", "r1", "r2")}
            for row in case.get("misalign", [])]
    return tp.Lattice.from_records(case["elements"], misalign=rows)
