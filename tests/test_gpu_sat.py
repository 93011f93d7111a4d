"""SAT kernel (naivesat path) against the CPU oracle, through the C ABI."""
import numpy as np
import pytest

from naivesat_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def oc(c):
    return O.Circuit(c.n, c.gates, c.outputs)


@pytest.mark.parametrize("seed,n,g", [(10, 15, 60), (11, 18, 150), (12, 20, 300), (13, 22, 500),
                                      (14, 24, 800), (15, 26, 400), (16, 12, 50), (17, 9, 30)])
def test_sat_random_dag_matches_oracle(ctx, seed, n, g):
    c = W.random_dag(seed, n, g, output="live")
    cnt, low = O.sat_range(oc(c))
    h = ctx.circuit(c)
    r = h.sat(find_all=True)
    assert r["count"] == cnt
    assert r["witness"] == low
    assert r["satisfiable"] == (cnt > 0)
    # find mode: same lowest witness
    r2 = h.sat(find_all=False, chunk_bits=15)
    assert r2["witness"] == low


def test_sat_config0_full(ctx):
    """Config 0: 24 inputs, 500 gates, seed 0 -- exact count and lowest witness."""
    c = W.config("c0")
    cnt, low = O.sat_range(oc(c))
    r = ctx.circuit(c).sat(find_all=True)
    assert (r["count"], r["witness"]) == (cnt, low)


def test_sat_config1_subrange_and_plant(ctx):
    """Config 1 (36 inputs, 3018 gates): a 2^30 range checked exactly, and the
    planted constant K appears in the lowest witness."""
    c = W.config("c1")
    h = ctx.circuit(c)
    begin, end = 3 << 30, 4 << 30
    cnt, low = O.sat_range(oc(c), begin, end)
    r = h.sat(find_all=True, begin=begin, end=end)
    assert (r["count"], r["witness"]) == (cnt, low)
    f = h.sat(find_all=False, chunk_bits=30)
    assert f["satisfiable"] and (f["witness"] & ((1 << 18) - 1)) == c.plant_k
    assert c.eval_bits([(f["witness"] >> i) & 1 for i in range(36)])[0] == 1
    ocnt, olow = O.sat_range(oc(c), 0, 1 << 30)
    assert f["witness"] == olow


def test_sat_edge_circuits(ctx):
    n = 16
    # output = input k: lowest witness 2^k, count 2^(n-1)
    for k in [0, 4, 5, 9, 10, 15]:
        c = W.Circuit(n, np.zeros((0, 3)), [(k, 0)])
        r = ctx.circuit(c).sat()
        assert r["count"] == 1 << (n - 1) and r["witness"] == 1 << k
        cneg = W.Circuit(n, np.zeros((0, 3)), [(k, 1)])
        r = ctx.circuit(cneg).sat()
        assert r["count"] == 1 << (n - 1) and r["witness"] == 0
    # contradiction: x AND NOT x -> unsatisfiable
    c = W.Circuit(n, [(W.NIMPL, 3, 3)], [(n, 0)])
    r = ctx.circuit(c).sat()
    assert not r["satisfiable"] and r["count"] == 0 and r["witness"] is None
    # tautology: NOT (x AND NOT x)
    c = W.Circuit(n, [(W.NIMPL, 3, 3)], [(n, 1)])
    r = ctx.circuit(c).sat()
    assert r["count"] == 1 << n and r["witness"] == 0
    # only the last assignment satisfies: AND of all inputs
    rb = W.RawBuilder(n)
    acc = rb.gate(W.AND, 0, 1)
    for i in range(2, n):
        acc = rb.gate(W.AND, acc, i)
    rb.output(acc)
    r = ctx.circuit(rb.fold()).sat()
    assert r["count"] == 1 and r["witness"] == (1 << n) - 1


def test_sat_ranges_partition(ctx):
    """Counts over a partition of the index space add up (sharded use)."""
    c = W.random_dag(21, 24, 400, output="live")
    h = ctx.circuit(c)
    full = h.sat()
    parts = [h.sat(begin=k << 21, end=(k + 1) << 21) for k in range(8)]
    assert sum(p["count"] for p in parts) == full["count"]
    lows = [p["witness"] for p in parts if p["witness"] is not None]
    assert (min(lows) if lows else None) == full["witness"]


def test_sat_no_optimize_matches(ctx):
    from naivesat_b200 import api
    c = W.random_dag(31, 22, 600, output="live")
    with api.Context(0, no_optimize=True) as raw:
        a = raw.circuit(c).sat()
    b = ctx.circuit(c).sat()
    assert (a["count"], a["witness"]) == (b["count"], b["witness"])


def test_sat_deterministic(ctx):
    c = W.random_dag(41, 26, 700, output="live")
    h = ctx.circuit(c)
    r1, r2 = h.sat(), h.sat()
    assert (r1["count"], r1["witness"]) == (r2["count"], r2["witness"])
