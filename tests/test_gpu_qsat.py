"""QSAT kernel (naiveqsat path) against the oracle and the reference's own
known answers, through the C ABI."""
import json
import os
import random

import numpy as np
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


def _block_data(rng, n, q):
    """Words whose innermost quantifier block (the last run of equal letters,
    item bit 0 = last quantifier) gets node values about half true: per node,
    one set bit (Exists) or one cleared bit (All) with probability 1/2."""
    L = 1
    while L < n and q[n - 1 - L] == q[-1]:
        L += 1
    words = np.full((1 << n) // 32, 0xFFFFFFFF if q[-1] == "A" else 0, dtype=np.uint32)
    for node in range(1 << (n - L)):
        if rng.random() < 0.5:
            k = (node << L) + rng.randrange(1 << L)
            words[k >> 5] ^= np.uint32(1 << (k & 31))
    return words


# (n, quantifiers): long innermost blocks fold words over iterations (the
# launch has n - 25 iteration bits): fold of every iteration level, of some
# with the rest reduced per node, units right at the fold level, a fold of
# zero levels (only levels 0..9 alike), units two nodes above the fold,
# and one of each innermost letter.
FOLD_CASES = [(26, "A" + "E" * 25), (26, "E" + "A" * 25), (26, "EEAAA" + "E" * 21),
              (27, "E" * 15 + "A" + "E" * 11), (27, "A" * 16 + "E" * 11),
              (27, "AE" * 6 + "E" + "A" * 14), (27, "E" * 16 + "A" * 11), (26, "EAE" + "A" * 13 + "E" * 10),
              (25, "A" * 5 + "E" * 20), (24, "EA" * 7 + "A" * 10), (28, "E" * 16 + "A" + "E" * 11)]


@pytest.mark.parametrize("case", range(len(FOLD_CASES)))
def test_reduce_words_folded_blocks(ctx, case):
    n, q = FOLD_CASES[case]
    rng = random.Random(4200 + case)
    for _ in range(3):
        w = _block_data(rng, n, q)
        qr = O.QuantReducer(q)
        qr.push_words(w)
        assert strip(ctx.qsat_reduce_words(q, w)) == qr.final_result(), (n, q)


@pytest.mark.parametrize("q", ["A" + "E" * 27, "E" * 2 + "A" * 12 + "E" * 14, "E" * 5 + "A" * 11 + "E" * 12,
                               "A" * 3 + "E" * 14 + "A" * 11, "E" * 16 + "A" + "E" * 11])
def test_qsat_folded_blocks_match_oracle(ctx, q):
    c = W.random_dag(41, 28, 300, output="live")
    exp = O.qsat(O.Circuit(c.n, c.gates, c.outputs), q, mode=1)
    assert strip(ctx.circuit(c).qsat(q)) == exp, q


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


def test_one_handle_many_kernels(ctx):
    """A circuit handle keeps the kernels it has loaded.  Solves of other
    kinds, ranges, launch sizes, quantifier strings and prefixes on the same
    handle, repeated, equal the oracle's answers (prefix solves: a fresh
    handle's)."""
    c = W.random_dag(77, 22, 400, output="live")
    oc = O.Circuit(c.n, c.gates, c.outputs)
    h = ctx.circuit(c)
    full = O.sat_range(oc)
    part = O.sat_range(oc, 1 << 20, 3 << 20)
    qs = ["A" + "E" * 21, "E" * 3 + "A" * 19, W.alternating_quants(5, 22, max_block=3)]
    exp = {q: O.qsat(oc, q, mode=1) for q in qs}
    for _ in range(2):
        r = h.sat()
        assert (r["count"], r["witness"]) == full
        r = h.sat(begin=1 << 20, end=3 << 20)
        assert (r["count"], r["witness"]) == part
        for q in qs:
            assert strip(h.qsat(q)) == exp[q], q
            assert strip(h.qsat(q, chunk_bits=16)) == exp[q], q
            for p in range(4):
                assert strip(h.qsat(q, prefix_bits=2, prefix=p)) == strip(ctx.circuit(c).qsat(q, prefix_bits=2, prefix=p))
