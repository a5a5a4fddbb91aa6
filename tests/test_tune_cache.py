"""The launch-shape tuner's host side through the C-ABI, without a GPU: its modes, a forced shape, and its
cache file (the choices read back as written; a missing file and a bad mode are errors)."""
import os
import tempfile

import pytest


@pytest.fixture()
def D():
    from qed_spin_b200 import build
    build.build()
    from qed_spin_b200 import device
    device.tune_clear()
    prev = device.tune_mode(-1)
    yield device
    device.tune_clear()
    device.tune_mode(prev)


def test_modes(D):
    D.tune_mode(2)
    assert D.tune_mode(0) == 2
    assert D.tune_mode(-1) == 0
    with pytest.raises(ValueError):
        D.tune_mode(3)
    with pytest.raises(ValueError):
        D.tune_mode(-2)


def test_cache_file_round_trip(D):
    lines = ["walk|N32.G128.gk1.slc1.lk4.ng33.d23.nv1.st32.11.same|sm100x148\t0\t3.39\t5.59",
             "walk_team|N24.G24.gk1.slc1.lk4.ng25.d17.nv8.st64.11.same|sm100x148\t3\t0.155\t0.214\t0.331\t0.136"]
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "in.txt")
        open(src, "w").write("\n".join(lines) + "\n")
        D.tune_load(src)
        got = D.tune_entries()
        assert got[lines[0].split("\t")[0]][0] == 0
        assert got[lines[1].split("\t")[0]][0] == 3
        out = os.path.join(d, "out.txt")
        D.tune_save(out)
        D.tune_clear()
        assert D.tune_entries() == {}
        D.tune_load(out)
        assert {k: v[0] for k, v in D.tune_entries().items()} == {k: v[0] for k, v in got.items()}
        with pytest.raises(ValueError):
            D.tune_load(os.path.join(d, "missing.txt"))


def test_force_and_clear(D):
    D.tune_force("walk", 2)
    D.tune_force("walk", -1)
    D.tune_force("walk_team", 1)
    D.tune_clear()
    assert D.tune_entries() == {}
