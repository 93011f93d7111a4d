"""QSAT kernel (naiveqsat path) against the oracle and the reference's own
known answers, through the C ABI."""
import json
import os

import pytest

from naivesat_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    with open(os.path.join(GOLD, name)) as f:
        return json.load(f)["cases"]


def strip(r):
    return {"reversed": r["reversed"], "solution_bits": r["solution_bits"], "solution": r["solution"]}


def test_reduce_words_aggr_tree_kats(ctx):
    """The reference's identity-circuit aggregator vectors, run through the
    QSAT reduction kernel (data mode): tree value over the item bits."""
    for c in load("aggr_tree_cpu.json"):
        r = ctx.qsat_reduce_words(c["quants"], c["words"])
        assert r["value"] == c["result"], c
    for c in load("aggr_tree_opencl.json"):
        r = ctx.qsat_reduce_words(c["quants"][-5:], c["words"])
        assert r["value"] == c["result"], c


def test_reduce_words_quant_reducer_kats(ctx):
    """qsat.rs test_quant_reducer cases with >= 32 items: final result."""
    n = 0
    for c in load("quant_reducer.json"):
        nq = len(c["quants"])
        if nq < 5:
            continue
        words = [0] * ((1 << nq) // 32)
        for k, it in enumerate(c["items"]):
            if it:
                words[k >> 5] |= 1 << (k & 31)
        assert strip(ctx.qsat_reduce_words(c["quants"], words)) == c["result"], c
        n += 1
    assert n >= 10


@pytest.mark.parametrize("t", range(16))
def test_qsat_random_matches_oracle(ctx, t):
    rng = W.SplitMix64(1000 + t)
    n = [12, 15, 16, 18, 20, 22, 24, 25][t % 8]
    c = W.random_dag(300 + t, n, 80 + 40 * (t % 5), output="live")
    # block structures: long first block, short first block, alternating
    shape = t % 4
    if shape == 0:
        q = "".join("A" if rng.below(2) else "E" for _ in range(n))
    elif shape == 1:
        f = n - 1 - rng.below(4)
        q0 = "A" if rng.below(2) else "E"
        q = q0 * f + ("E" if q0 == "A" else "A") * (n - f)
    elif shape == 2:
        q = W.alternating_quants(t, n, max_block=4)
    else:
        q0 = "A" if rng.below(2) else "E"
        q = q0 + ("E" if q0 == "A" else "A") * (n - 1)
    exp = O.qsat(O.Circuit(c.n, c.gates, c.outputs), q, mode=1)
    got = ctx.circuit(c).qsat(q)
    assert strip(got) == exp, (q, got, exp)
    # small launches: the host QuantReducer joins per-launch results
    got2 = ctx.circuit(c).qsat(q, chunk_bits=15)
    assert strip(got2) == exp


def test_qsat_all_same_quantifier(ctx):
    c = W.random_dag(7, 20, 200, output="live")
    o = O.Circuit(c.n, c.gates, c.outputs)
    for q in ["E" * 20, "A" * 20]:
        assert strip(ctx.circuit(c).qsat(q)) == O.qsat(o, q)


def test_qsat_adder_known_answers(ctx):
    """Config 2a (verdict TRUE) and 2b (FALSE, counterexample a = 0)."""
    a = W.config("c2a")
    r = ctx.circuit(a).qsat(a.quants)
    assert r["value"] is True and r["reversed"] and r["solution"] is None and r["solution_bits"] == 16
    b = W.config("c2b")
    r = ctx.circuit(b).qsat(b.quants)
    assert r["value"] is False and r["reversed"] and r["solution"] == 0 and r["solution_bits"] == 16


def test_qsat_config2c_matches_oracle(ctx):
    c = W.config("c2c")
    exp = O.qsat(O.Circuit(c.n, c.gates, c.outputs), c.quants, mode=1)
    got = ctx.circuit(c).qsat(c.quants)
    assert strip(got) == exp
