"""Shared fixtures. GPU tests carry the `gpu` marker; everything else runs on CPU."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the sm_100a library")


@pytest.fixture(scope="session")
def orc():
    """The CPU oracle (test infrastructure)."""
    from oracle import oracle
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def ws():
    """One workspace (CUDA stream) for the GPU tests."""
    from csharp_linearalgebra_b200 import Workspace
    w = Workspace(0)
    yield w
    w.dispose()


def net_matrix(orc, rows, cols, seed, kind="half"):
    """Matrices the reference's tests build from System.Random(seed).

    kind="half": NextDouble() - 0.5 (TestMatrix.Random, Support/TestMatrix.cs:48-56)
    kind="unit": NextDouble()*2 - 1 (MatrixExponentialTests.RandomWithOneNorm)
    Column-major fill order, as both helpers loop j outer, i inner.
    """
    r = orc.NetRandom(seed)
    a = np.zeros((rows, cols), order="F")
    for j in range(cols):
        for i in range(rows):
            d = r.next_double()
            a[i, j] = d - 0.5 if kind == "half" else d * 2.0 - 1.0
    return a


def random_with_one_norm(orc, n, target, seed):
    """MatrixExponentialTests.RandomWithOneNorm (tests/Tensile.Tests/MatrixExponentialTests.cs)."""
    a = net_matrix(orc, n, n, seed, kind="unit")
    return a * (target / orc.norm1(a))


def rel1(x, y):
    """Normwise relative difference in the 1-norm, max(||y||,1) as the scale
    (MatrixExponentialTests.RelativeDifference)."""
    x, y = np.asarray(x), np.asarray(y)
    d = np.abs(x - y).sum(axis=0).max() if x.size else 0.0
    r = np.abs(y).sum(axis=0).max() if y.size else 0.0
    return d / max(r, 1.0)


def relfro(x, y):
    x, y = np.asarray(x), np.asarray(y)
    ny = np.linalg.norm(y)
    return np.linalg.norm(x - y) / (ny if ny > 0 else 1.0)
