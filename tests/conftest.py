"""Shared fixtures.  `-m gpu` tests need a CUDA device and libhadamag_b200.so; the
others run on the CPU (oracle, host-side logic, ABI surface)."""
import importlib
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libhadamag_b200.so")


@pytest.fixture(scope="session")
def hm():
    return importlib.import_module("hadamag_b200")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def ctx(hm):
    return hm._native.default_context(0)


def rand_state(dim, seed):
    g = np.random.default_rng(seed)
    v = g.normal(size=dim) + 1j * g.normal(size=dim)
    return v / np.linalg.norm(v)


def t_state(n):
    t = np.array([1, np.exp(1j * np.pi / 4)]) / np.sqrt(2)
    v = np.array([1.0 + 0j])
    for _ in range(n):
        v = np.kron(v, t)
    return v


def ghz(n):
    v = np.zeros(1 << n, dtype=complex)
    v[0] = v[-1] = 1 / np.sqrt(2)
    return v
