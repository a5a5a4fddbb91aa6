"""The replica plumbing of multi-GPU runs, driven on CPU by two gloo ranks: each rank times its own replica
(the oracle's host matvec standing in for the device step, rank 1 made slower), the barrier brackets the timed
region, every rank gets the max over ranks, and the whole-job rate is both ranks' units over the slowest time."""
import multiprocessing as mp
import os
import socket
import time

import numpy as np


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, port: int, q) -> None:
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    from oracle import oracle as O
    from qed_spin_b200 import lattice as lat
    from qed_spin_b200 import operators as ops
    from qed_spin_b200 import replicas
    size, r, _ = replicas.init("gloo", timeout_s=60)
    spec = lat.chain_sector(12, 6, r)   # each replica its own sector: no exchange on the path
    S = O.Sector(spec)
    P = O.Program(ops.row_program(ops.from_products(12, ops.heisenberg_products(lat.chain_bonds(12)))))
    x = np.ones(S.dim, np.complex128)
    steps = 5
    replicas.barrier(size)
    t0 = time.perf_counter()
    for _ in range(steps):
        x = S.gather(P, x)
        x /= np.linalg.norm(x)
    if r == 1:
        time.sleep(0.2)
    replicas.barrier(size)
    t = time.perf_counter() - t0
    t_max = replicas.max_over_ranks(t, size)
    q.put((r, t, t_max, replicas.whole_job_rate(steps, size, t_max)))
    replicas.finish(size)


def test_two_gloo_replicas():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, t0, m0, rate0), (r1, t1, m1, rate1) = out
    assert (r0, r1) == (0, 1)
    assert m0 == m1 == max(t0, t1) and t1 >= 0.2
    assert rate0 == rate1 == 2 * 5 / m0
