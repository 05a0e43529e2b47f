"""Shared test set-up: import paths, the ``gpu`` marker and golden-fixture loaders."""

from __future__ import annotations

import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "optical-flow-filter_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)
if os.path.join(ROOT, "oracle") not in sys.path:
    sys.path.append(os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def golden_case(name: str):
    """(meta, arrays) of a reference parity case packed by oracle/make_reference_fixtures.py."""
    z = np.load(os.path.join(GOLDEN, f"ref_case_{name}.npz"))
    meta = json.loads(bytes(z["meta"]).decode())
    return meta, {k: z[k] for k in z.files if k != "meta"}


def golden_stages():
    z = np.load(os.path.join(GOLDEN, "ref_stages.npz"))
    return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch
