"""The request server: every result is the same alone and in a concurrent mix, requests wait for slots and
memory, and admitted requests run at the same time.

Exactness, written per test: a request's levels and spectrum served in a mix equal the same request served
alone bit for bit (the solves are deterministic: fixed reduction trees, the same lanes), and equal a direct call
of the lane on the same reduced CSRs bit for bit (the server attaches each sector's CSR). At depth 120 these
small sectors are past the loss of orthogonality, where the continued fraction amplifies any difference in the
rounding of H v, so the comparison is lane for lane.
"""
import numpy as np
import pytest

from qed_spin_b200 import lattice as lat
from qed_spin_b200 import operators as ops

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.fail("a GPU test ran without a CUDA device")
    from qed_spin_b200 import build
    build.build()


def _requests():
    rng = np.random.default_rng(3)
    omega = np.linspace(-0.5, 6.0, 200)
    out = []
    for i in range(10):
        N = int(rng.choice([12, 14, 16, 18]))
        J, K = float(rng.uniform(0.5, 1.5)), float(rng.uniform(0.0, 0.3))
        prods = ops.heisenberg_products(lat.chain_bonds(N), J) + ops.chiral_products(
            [(a, (a + 1) % N, (a + 2) % N) for a in range(N)], K)
        h = ops.row_program(ops.from_products(N, prods))
        if i % 2 == 0:
            out.append({"kind": "eigs", "spec": lat.chain_sector(N, N // 2, int(rng.integers(0, N))), "h": h,
                        "k": 1 + i % 4})
        else:
            m = int(rng.integers(1, N))
            src, tgt = lat.chain_sector(N, N // 2, 0), lat.chain_sector(N, N // 2, m)
            op = ops.cross_row_program(ops.from_products(N, ops.sz_q_products(N, 2 * np.pi * m / N)), tgt, src)
            out.append({"kind": "dynamics", "src": src, "tgt": tgt, "h": h, "op": op, "omega": omega})
    return out


def _submit(srv, r):
    if r["kind"] == "eigs":
        return srv.submit_eigs(r["spec"], r["h"], r["k"])
    return srv.submit_dynamics(r["src"], r["tgt"], r["h"], r["op"], 120, r["omega"], 0.05)


def _bits(a):
    return np.ascontiguousarray(a, np.float64).view(np.uint64)


def test_alone_equals_mix_and_direct():
    from qed_spin_b200 import device as D
    reqs = _requests()
    # alone: one server slot, each request submitted after the previous one finished
    srv = D.Server(max_active=1)
    alone = [srv.wait(_submit(srv, r)) for r in reqs]
    srv.close()
    # in a mix: all submitted at once to 4 slots under a budget that admits only some at a time
    fp = sorted(a["footprint"] for a in alone)
    budget = int(fp[-1] + fp[-2] + fp[-3])
    srv = D.Server(max_active=4, hbm_budget=budget)
    tickets = [_submit(srv, r) for r in reqs]
    mix = [srv.wait(t) for t in tickets]
    srv.close()
    for r, a, b in zip(reqs, alone, mix):
        assert a["converged"] and b["converged"]
        assert np.array_equal(_bits(a["values"]), _bits(b["values"])), r["kind"]
        if r["kind"] == "dynamics":
            assert np.array_equal(_bits(a["S"]), _bits(b["S"]))
    # the mix overlapped: some admitted requests ran at the same time, and some waited for room
    spans = [(b["t_admit"], b["t_done"]) for b in mix]
    overlap = any(s1[0] < s2[1] and s2[0] < s1[1] for i, s1 in enumerate(spans) for s2 in spans[i + 1:])
    assert overlap
    assert any(b["t_admit"] - b["t_submit"] > 1e-4 for b in mix)
    # each result against a direct call of its lane on the same reduced CSRs
    for r, a in zip(reqs, alone):
        if r["kind"] == "eigs":
            S, P = D.Sector(r["spec"]), D.Program(r["h"])
            A = D.Csr(S, S, P)
            A.attach(P)
            direct = D.eigs(S, P, r["k"])["values"]
            assert np.array_equal(_bits(a["values"]), _bits(direct))
        else:
            src, tgt = D.Sector(r["src"]), D.Sector(r["tgt"])
            hs, ht = D.Program(r["h"]), D.Program(r["h"])
            As, At = D.Csr(src, src, hs), D.Csr(tgt, tgt, ht)
            As.attach(hs)
            At.attach(ht)
            d = D.dynamics_t0(src, hs, tgt, ht, D.Program(r["op"]), 120, r["omega"], 0.05)
            assert np.array_equal(_bits(a["S"]), _bits(d["S"]))
            assert a["e0"] == d["e0"]


def test_bad_request_fails_alone():
    """A failing request reports its error; the server keeps serving the others."""
    from qed_spin_b200 import device as D
    reqs = _requests()[:2]
    srv = D.Server(max_active=2)
    bad = lat.chain_sector(12, 6, 0)
    h = ops.row_program(ops.from_products(12, ops.heisenberg_products(lat.chain_bonds(12))))
    bad_prog = ops.Program(h.group_flip[::-1].copy(), h.group_setbits, h.group_vbegin, h.vsub_val, h.vsub_tbegin,
                           h.term_sign, h.term_coeff)
    t_bad = srv.submit_eigs(bad, bad_prog, 1)
    tickets = [_submit(srv, r) for r in reqs]
    with pytest.raises(ValueError, match="group"):
        srv.wait(t_bad)
    for t in tickets:
        assert srv.wait(t)["converged"]
    srv.close()


def test_thermal_requests_served():
    """Thermal requests (one block of the thermal driver's sampled path each) served in a mix with eigs requests:
    each block's lnZ, E, V equal a direct qb_ftlm call on the same reduced-CSR lane bit for bit, and the oracle's
    FTLM of the block within 1e-8 relative."""
    from oracle import oracle as O
    from qed_spin_b200 import device as D
    N, seed = 12, 4242
    betas = 1.0 / np.linspace(0.2, 3.0, 15)
    prods = ops.xxz_products(lat.chain_bonds(N), 1.0, 0.5) + ops.zeeman_z_products(N, 0.1)
    h = ops.row_program(ops.from_products(N, prods))
    blocks = [lat.chain_sector(N, 6, 0), lat.chain_sector(N, 5, 3), lat.chain_sector(N, 4, 7)]
    srv = D.Server(max_active=4)
    tickets = [srv.submit_thermal(b, h, 8, 30, seed, betas) for b in blocks]
    tickets.append(srv.submit_eigs(blocks[0], h, 2))
    got = [srv.wait(t) for t in tickets]
    srv.close()
    Po = O.Program(h)
    for spec, g in zip(blocks, got[:3]):
        S, P = D.Sector(spec), D.Program(h)
        A = D.Csr(S, S, P)
        A.attach(P)
        one = D.ftlm(S, P, 8, 30, seed, betas)
        A.close()
        for key in ("lnZ", "E", "V"):
            assert np.array_equal(_bits(g[key]), _bits(one[key])), key
        ref = O.Sector(spec).ftlm(Po, 8, 30, seed, betas)
        for key in ("lnZ", "E", "V"):
            r = np.asarray(ref[key])
            np.testing.assert_allclose(g[key], r, rtol=1e-8, atol=1e-8 * max(np.abs(r).max(), 1e-3), err_msg=key)
    assert got[3]["converged"] and len(got[3]["values"]) == 2
