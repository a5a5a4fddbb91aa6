"""Shared test set-up: the `gpu` marker, the golden fixtures, and the checkers under oracle/."""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the sm_100a library)")


@pytest.fixture(scope="session")
def fixtures():
    return dict(np.load(os.path.join(GOLDEN, "fixtures.npz")))


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(GOLDEN, "golden.json")) as fh:
        return json.load(fh)


def host_program(fx, name):
    """The reference's compiled row program of a fixture case, as a host Program."""
    from qed_spin_b200.operators import Program
    g = lambda k: fx[f"{name}/prog/{k}"]
    return Program(g("group_flip"), g("group_setbits"), g("group_vbegin"), g("vsub_val"), g("vsub_tbegin"),
                   g("term_sign"), g("term_coeff").view(np.complex128))
