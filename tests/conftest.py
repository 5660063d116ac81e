"""Shared test setup.

Markers: ``gpu`` tests need a CUDA device (run on a B200 with ``-m gpu``);
everything else runs on CPU.  The oracle restatement (oracle/_port) is built
on demand; the compiled reference (oracle/_ref) only exists where the
reference checkout was present at build time, and tests needing it skip
otherwise.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "sdf-contact-module_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _ensure_port():
    from oracle import port

    if not port.available():
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "port"], check=True)


@pytest.fixture(scope="session")
def port():
    _ensure_port()
    from oracle import port as p

    return p


@pytest.fixture(scope="session")
def ref():
    from oracle import ref as r

    if not r.available():
        pytest.skip("reference oracle (oracle/_ref) not built here")
    return r


def golden(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sdfo import _native as N

    N.load()
    N.check(N.load().sdfo_device_check(torch.cuda.current_device()))
    return torch.device("cuda")


def rel_err(a, b, floor):
    """max |a-b| / max(|b|, floor) elementwise."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor))) if a.size else 0.0
