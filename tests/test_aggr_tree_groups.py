"""The reference's test_aggr_output_opencl_code_2 vectors (qsat.rs:3522-3857,
43 vectors, 50 groups) reduced by the oracle's QuantReducer and by the GPU
tree.

Each vector runs the reference's OpenCL aggregator on an identity circuit
whose input is the data: reduce_len groups, each of group_len 32-lane words
(item k of a group = bit k%32 of its word k/32), under the last
log2(group_len) + 5 quantifiers.  Per group it expects the value and, when
the formula's first quantifier block reaches into the group and the value
decides it, the local index of the first decisive unit: the unit's first
word when the unit spans several words, the word itself when the block
reaches the lanes; 0x7fff when there is none.  Here each group's items are
reduced under the same quantifiers; the value must match, and the lowest
decisive unit of the FinalResult must give the same local index.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from test_aggr_tree_words import oracle_reduce, rev

HERE = os.path.dirname(os.path.abspath(__file__))


def load():
    with open(os.path.join(HERE, "golden", "aggr_tree_opencl_groups.json")) as f:
        return json.load(f)["cases"]


def check(c, reduce):
    Q, gl = c["quants"], c["group_len"]
    gb = gl.bit_length() - 1
    q = Q[len(Q) - (gb + 5):]
    gstart = len(Q) - (gb + 5)
    first = Q[0]
    reaches = all(x == first for x in Q[:gstart + 1])
    for g, (result, lidx) in enumerate(c["results"]):
        words = np.asarray(c["data"][g * gl:(g + 1) * gl], dtype=np.uint32)
        got = reduce(q, words)
        value = (got["solution"] is not None) ^ got["reversed"]
        assert value == result, (c, g, got)
        if lidx is None:
            continue
        decided = reaches and value == (first == "E")
        if not decided:
            assert lidx == 0x7FFF, (c, g, got)
            continue
        sb = got["solution_bits"]
        unit = rev(got["solution"], sb)
        word = unit >> (sb - gb) if sb >= gb else unit << (gb - sb)
        assert word == lidx, (c, g, got, word)


def test_vectors_are_present():
    cs = load()
    assert len(cs) == 43 and sum(len(c["results"]) for c in cs) == 50


def test_oracle_reproduces_every_vector():
    for c in load():
        check(c, oracle_reduce)


@pytest.mark.gpu
def test_gpu_tree_reproduces_every_vector(ctx):
    for c in load():
        check(c, lambda q, words: ctx.qsat_reduce_words(q, words))
