"""Shared test fixtures.  `-m gpu` tests need a CUDA device and libnbody_b200.so; the rest
run on the CPU (oracle pins, host logic, ABI export checks)."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")


@pytest.fixture(scope="session")
def dwarf_small():
    """A seeded 3,000-body two-component dwarf on the sample workunit's orbit."""
    from milkywayathome_client_b200 import models
    return models.plummer_plummer_dwarf(3000, seed=11)


def make_ctx(n, theta=0.5, criterion="TreeCode", useQuad=True, potential="mw", precision="fp64",
             **over):
    from milkywayathome_client_b200 import models, nbody
    cfg = models.dwarf_config(n, theta=theta, criterion=criterion, useQuad=useQuad)
    cfg.update(over)
    pot = nbody.milky_way_potential() if potential == "mw" else potential
    return nbody.NBodyCtx(potential=pot, precision=precision, **cfg)


def bits_equal(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))
