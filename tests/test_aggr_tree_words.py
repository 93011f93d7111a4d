"""The reference's test_aggr_output_cpu_code_2 vectors (qsat.rs:2837-3292,
23 vectors) reduced by the oracle's QuantReducer and by the GPU tree.

Each vector runs the reference's CPU aggregator on an identity circuit
whose input is the data itself: 2^elem_bits items (item k = bit k%32 of
data[k/32]) in 64-bit machine words, under the last elem_bits quantifiers.
It expects the call's value and, when the formula's first quantifier block
reaches into the call, `found`: the index of the machine word at which the
first decisive unit of that block is known (the unit's only word when the
block reaches the lanes, its last word when the unit spans several words).
Here the same items are reduced under the same quantifiers; the value must
equal `result`, and the lowest decisive unit of the FinalResult (its
solution, bit k = input k of the block) must select the same word.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
LANE_BITS = 6          # 64-bit machine words


def load():
    with open(os.path.join(HERE, "golden", "aggr_tree_cpu_words.json")) as f:
        return json.load(f)["cases"]


def rev(v, bits):
    return int(format(v, "0%db" % bits)[::-1], 2) if bits else 0


def check(c, reduce):
    Q, eb = c["quants"], c["elem_bits"]
    wfb = len(Q) - eb
    q = Q[wfb:]
    got = reduce(q, np.asarray(c["data"], dtype=np.uint32))
    value = (got["solution"] is not None) ^ got["reversed"]
    assert value == c["result"], (c, got)
    first = Q[0]
    reaches = all(x == first for x in Q[:wfb + 1])          # the first block reaches into the call
    decided = reaches and value == (first == "E")
    assert (c["found"] is not None) == decided, (c, got)
    if not decided:
        return
    sb = got["solution_bits"]
    unit = rev(got["solution"], sb)                          # first input most significant
    word_bits = eb - LANE_BITS
    if sb >= word_bits:
        assert unit >> (sb - word_bits) == c["found"], (c, got)
    else:
        assert c["found"] >> (word_bits - sb) == unit, (c, got)
        assert c["found"] & ((1 << (word_bits - sb)) - 1) == (1 << (word_bits - sb)) - 1, c   # the unit's last word
    assert c["mword"] == c["data"][2 * c["found"]:2 * c["found"] + 2]


def oracle_reduce(q, words):
    qr = O.QuantReducer(q)
    qr.push_words(words)
    return qr.final_result()


def test_vectors_are_present():
    cs = load()
    assert len(cs) == 23 and sum(c["found"] is not None for c in cs) == 11


def test_oracle_reproduces_every_vector():
    for c in load():
        check(c, oracle_reduce)


@pytest.mark.gpu
def test_gpu_tree_reproduces_every_vector(ctx):
    for c in load():
        check(c, lambda q, words: ctx.qsat_reduce_words(q, words))
