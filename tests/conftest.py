"""Shared fixtures: seeded meshes for the golden cases, the golden data, and
the GPU marker.  GPU tests are marked ``@pytest.mark.gpu``; everything else
runs on CPU."""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "cuda-fabipb_b200"))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")


@pytest.fixture(scope="session")
def golden_meta():
    with open(os.path.join(GOLDEN, "cases.json")) as fp:
        return json.load(fp)


@pytest.fixture(scope="session")
def solve_meta():
    """Solve-only goldens of the larger cases and the reference's -r=2 direct solves."""
    with open(os.path.join(GOLDEN, "solve_cases.json")) as fp:
        return json.load(fp)


@pytest.fixture(scope="session")
def case_dir(tmp_path_factory):
    """All golden meshes, generated once per session from their seeds."""
    import make_golden
    d = tmp_path_factory.mktemp("cases")
    for name in make_golden.CASES:
        make_golden.generate_mesh(name, str(d))
    return str(d)


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def case_params(opts):
    return dict(order=opts["p"], depth=opts["t"], sep_ratio=opts["S"], eps1=opts["eps1"], eps2=opts["eps2"])


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))
