"""The lanes' staged Gaussian start (no GPU): qb_staged_start equals the reference engine's own staged_seed draw
(oracle/_ref: mt19937_64 and std::normal_distribution, src/engine/block_solve.cpp:263-277) bit for bit, below the
size where the draw goes parallel and well past it (three million entries, a dozen chunks of the parallel draw)."""
import numpy as np
import pytest

from oracle import ref as R


@pytest.mark.parametrize("seed,n", [(0x51ED0B70, 1000), (0x51ED900D, 3_000_000), (7, (1 << 20) + 1)])
def test_staged_start_equals_the_reference_draw(seed, n):
    if not R.available():
        pytest.fail("the reference engine library is not built (oracle/Makefile, run by __graft_entry__.build())")
    from qed_spin_b200 import device as D
    mine = D.staged_start(seed, n)
    ref = R.staged_seed(seed, n)
    assert np.array_equal(mine.view(np.uint64), ref.view(np.uint64))
