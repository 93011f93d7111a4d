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
