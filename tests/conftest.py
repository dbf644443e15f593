"""Shared test setup.

GPU tests are marked ``gpu`` and run on a B200 (``pytest -m gpu``); everything
else runs on the CPU (``pytest -m "not gpu"``).  The oracle under ``oracle/``
is the checker; the product is ``gpu-to_b200/`` (CUDA library + host binding).
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "gpu-to_b200"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU")


def load_golden(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def gputo():
    import build  # gpu-to_b200/build.py
    build.build()
    import gputo as G
    return G


@pytest.fixture(autouse=True)
def _scratch_cwd(tmp_path, monkeypatch):
    # the reference and the MEX gateway write mgcg1.log into the working directory
    monkeypatch.chdir(tmp_path)
