"""Shared pytest setup: the `gpu` marker, the package under test and the oracle."""
import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def load_package():
    """The product package (its directory name is not an identifier)."""
    return importlib.import_module("cfgable-matmul_b200")


def load_workloads():
    return importlib.import_module("cfgable-matmul_b200.workloads")


@pytest.fixture(scope="session")
def cm():
    return load_package()


@pytest.fixture(scope="session")
def wl():
    return load_workloads()


@pytest.fixture(scope="session")
def oracle():
    import oracle as o
    o.build()
    return o


def normwise(x, ref):
    """max |x - ref| / max |ref| (the error measure of every parity test)."""
    import numpy as np
    x = np.asarray(x)
    ref = np.asarray(ref)
    den = np.abs(ref).max()
    return float(np.abs(x - ref).max() / (den if den > 0 else 1.0))


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_golden(name):
    import numpy as np
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def check_gemm_summary(c, g, tol):
    """Sampled entries normwise; row / column sums (which cancel heavily for
    the sin/cos inputs) against max|C| times the number of summed entries."""
    import numpy as np
    assert normwise(c[g["sample_i"], g["sample_j"]], g["sample"]) < tol
    m, n = c.shape
    scale = float(g["absmax"])
    assert np.abs(c.sum(axis=1) - g["row_sums"]).max() < tol * scale * n
    assert np.abs(c.sum(axis=0) - g["col_sums"]).max() < tol * scale * m


def has_cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
