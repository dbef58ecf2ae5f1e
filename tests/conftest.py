"""Shared test set-up: the `gpu` marker, the package (imported by path - its
directory name is not an identifier), the oracle, and the conversions
between the oracle's per-point state (39 doubles) and the device layout."""
from __future__ import annotations

import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_package():
    return importlib.import_module("springback-precomp_b200")


@pytest.fixture(scope="session")
def pkg():
    return load_package()


@pytest.fixture(scope="session")
def orc():
    import oracle

    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("a gpu-marked test ran without a CUDA device")
    return torch.device("cuda:0")


def oracle_to_device(st: np.ndarray, nterms: int) -> np.ndarray:
    """(ne, nq, 39) oracle states -> (nfields, ne, nq) device layout."""
    ne, nq, _ = st.shape
    nf = 14 + 6 * nterms
    out = np.zeros((nf, ne, nq))
    out[0:12] = np.moveaxis(st[..., 0:12], -1, 0)
    for t in range(nterms):
        out[12 + 6 * t:18 + 6 * t] = np.moveaxis(st[..., 12 + 6 * t:18 + 6 * t], -1, 0)
    out[12 + 6 * nterms] = st[..., 36]
    out[13 + 6 * nterms] = st[..., 38]
    return out


def device_to_oracle(st: np.ndarray, nterms: int) -> np.ndarray:
    nf, ne, nq = st.shape
    out = np.zeros((ne, nq, 39))
    out[..., 0:12] = np.moveaxis(st[0:12], 0, -1)
    for t in range(nterms):
        out[..., 12 + 6 * t:18 + 6 * t] = np.moveaxis(st[12 + 6 * t:18 + 6 * t], 0, -1)
    out[..., 36] = st[12 + 6 * nterms]
    out[..., 38] = st[13 + 6 * nterms]
    return out


def dense_from_blocks(kb: np.ndarray) -> np.ndarray:
    """(ne, 64, 3, 3) node blocks -> (ne, 24, 24)."""
    return kb.reshape(-1, 8, 8, 3, 3).transpose(0, 1, 3, 2, 4).reshape(-1, 24, 24)


def rel_frobenius(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Per-element relative Frobenius error |a - b| / |b| over the trailing axes."""
    ax = tuple(range(1, a.ndim))
    den = np.sqrt((b ** 2).sum(axis=ax))
    return np.sqrt(((a - b) ** 2).sum(axis=ax)) / np.where(den > 0, den, 1.0)


X_DISTORTED = np.array([[0.05, 0.00, 0.00], [1.10, 0.10, -0.05], [1.20, 1.15, 0.10], [-0.05, 0.90, 0.05],
                        [0.10, 0.05, 0.90], [0.95, -0.05, 1.05], [1.05, 1.05, 1.20], [0.00, 1.10, 1.00]])


def deformation(x: np.ndarray, scale: float) -> np.ndarray:
    """The reference tests' displacement pattern (stretch, shear, bending,
    twist; tests/test_incompatible_modes.cpp:382-392)."""
    ue = np.zeros(24)
    for a in range(8):
        p = x[a]
        ue[3 * a:3 * a + 3] = scale * np.array([0.8 * p[0] + 0.6 * p[0] * p[2] + 0.2 * p[1],
                                                -0.3 * p[1] + 0.5 * p[1] * p[2] - 0.4 * p[0] * p[1],
                                                -0.4 * p[2] - 0.5 * p[0] ** 2 + 0.3 * p[0] * p[1] * p[2]])
    return ue
