"""Sharded solves through the C ABI: QSAT with a fixed prefix of outer inputs
(the per-rank sub-problem) against the oracle, and the rank combination over
virtual ranks on one GPU (no kernels wait on one another: each rank's solve
is an ordinary launch sequence)."""
import pytest

from naivesat_b200 import shard
from naivesat_b200 import workloads as W
from oracle import oracle as O
from test_shard import oracle_sub

pytestmark = pytest.mark.gpu

KEYS = ("reversed", "solution_bits", "solution")


@pytest.mark.parametrize("t", range(6))
def test_prefix_subproblems_match_oracle(ctx, t):
    rng = W.SplitMix64(5000 + t)
    n = 16 + rng.below(6)
    c = W.random_dag(900 + t, n, 150 + 50 * (t % 3), output="live")
    q = W.alternating_quants(950 + t, n, max_block=1 + rng.below(5))
    h = ctx.circuit(c)
    full = O.qsat(O.Circuit(c.n, c.gates, c.outputs), q, mode=1)
    for s in (1, 2, 3):
        subs = []
        for p in range(1 << s):
            got = h.qsat(q, prefix_bits=s, prefix=p)
            exp = oracle_sub(c, q, s, p)
            assert {k: got[k] for k in KEYS} == exp, (q, s, p, got, exp)
            subs.append(got)
        comb = shard.combine_qsat(q, subs)
        assert {k: comb[k] for k in KEYS} == full


def test_sharded_sat_virtual_ranks(ctx):
    c = W.random_dag(77, 24, 500, output="live")
    h = ctx.circuit(c)
    cnt, low = O.sat_range(O.Circuit(c.n, c.gates, c.outputs))
    for world in (2, 4, 8):
        parts = []
        for r in range(world):
            b, e = shard.shard_range(1 << c.n, world, r)
            parts.append(h.sat(begin=b, end=e))
        got = shard.combine_sat(parts)
        assert (got["count"], got["witness"]) == (cnt, low)


def test_sharded_qsat_adder_known_answer(ctx):
    """Config 2b split over 4 virtual ranks: still FALSE with counterexample 0."""
    b = W.config("c2b")
    h = ctx.circuit(b)
    subs = [h.qsat(b.quants, prefix_bits=2, prefix=p) for p in range(4)]
    comb = shard.combine_qsat(b.quants, subs)
    assert comb["value"] is False and comb["solution"] == 0 and comb["solution_bits"] == 16


def _solve_shared(ctx0, ctx1, circ, chunk_bits):
    """One find-mode search split over two contexts on the same GPU, each
    on its own host thread, through one nsat_sat_share queue."""
    import threading
    from naivesat_b200 import api
    share = api.SatShare()
    hs = [ctx0.circuit(circ), ctx1.circuit(circ)]
    out = [None, None]

    def run(i):
        out[i] = hs[i].sat(find_all=False, chunk_bits=chunk_bits, share=share)
    th = [threading.Thread(target=run, args=(i,)) for i in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    lows = [r["witness"] for r in out if r["witness"] is not None]
    return (min(lows) if lows else None), out


def test_shared_queue_two_contexts_stop_together(ctx):
    """Two contexts claim launches from one shared queue: with an early
    witness both stop within a few launches of it (not after half the index
    space each); the lowest witness equals the single-context solve's; with
    no solution the two together scan every chunk exactly once."""
    from naivesat_b200 import api
    with api.Context(0) as other:
        early = W.Circuit(30, [(W.AND, 0, 2)], [(30, 0)], name="x0 and x2")
        low, out = _solve_shared(ctx, other, early, 20)
        assert low == 5
        # each context has at most a ring of launches in flight when the stop lands
        assert all(r["scanned"] <= 16 << 20 for r in out), [r["scanned"] for r in out]
        for seed in range(4):
            c = W.random_dag(1200 + seed, 26, 400, output="live")
            one = ctx.circuit(c).sat(find_all=False, chunk_bits=18)
            low, out = _solve_shared(ctx, other, c, 18)
            assert low == one["witness"], (seed, low, one["witness"])
        unsat = W.Circuit(24, [(W.NIMPL, 3, 3)], [(24, 0)], name="contradiction")
        low, out = _solve_shared(ctx, other, unsat, 18)
        assert low is None and sum(r["scanned"] for r in out) == 1 << 24
