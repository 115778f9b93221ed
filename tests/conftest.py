"""Shared pytest configuration.

Markers:
  gpu  -- needs a CUDA device (B200, sm_100a); the parity tests proper.
Everything unmarked runs on a CPU-only machine in a few minutes.
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

# Tests run the grid path's default launch choices unless a test tunes them:
# no tuning cache file is read or written.
os.environ.setdefault("BF_TUNE_CACHE", "off")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (sm_100a)")


@pytest.fixture(scope="session")
def orc():
    from oracle import loader
    return loader


@pytest.fixture(scope="session")
def ref(orc):
    if not orc.reference_available():
        pytest.skip("reference CPU core (oracle/_ref) not built")
    return orc


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from beamform_project_b200 import native
    native.lib()  # fail loudly if the product library is missing
    return torch


def rng(seed: int = 0) -> np.random.Generator:
    return np.random.default_rng(seed)


def random_voltage(T: int, F: int, A: int, seed: int = 0) -> np.ndarray:
    """Uniform random packed bytes: every nibble pattern appears."""
    return rng(seed).integers(0, 256, size=(T, F, A), dtype=np.uint8)


def grid_weights(A: int, F: int, B: int, seed: int = 1) -> np.ndarray:
    """Unit-modulus complex64 weights [B][F][A][2] with random phases."""
    ph = rng(seed).uniform(-np.pi, np.pi, size=(B, F, A))
    return np.stack([np.cos(ph), np.sin(ph)], axis=-1).astype(np.float32)


def tile_weights(w: np.ndarray) -> np.ndarray:
    """Canonical [B][F][A][2] -> tiled [F][ceil(B/32)][A][32][2] (zero padded),
    the layout of include/beamformer/indexing.hpp:54-61."""
    B, F, A, _ = w.shape
    bt = -(-B // 32)
    out = np.zeros((F, bt, A, 32, 2), np.float32)
    for b in range(B):
        out[:, b // 32, :, b % 32, :] = w[b]
    return out
