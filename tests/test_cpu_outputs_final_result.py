"""The reference's test_get_final_results_from_cpu_outputs vectors
(qsat.rs:3859-4036, 12 cases) as item patterns for the forall/exists
reduction.

get_final_results_from_cpu_outputs (qsat.rs:871-927) decodes the output of
one CPU call over the last elem_bits = 18 inputs: words 0..7 the 256 lane
values (the last 8 inputs) of the deciding vector word, word 8 the call's
value, word 9 a solution flag and words 10..11 the index of the deciding
word among the call's 1024 (the 10 inputs above the lanes).  It returns the
FinalResult of the call's part of the formula: the first quantifier block's
bits inside the call, from the word index and, when the block reaches the
lanes, from a reducer over the lane values.  Here that call becomes 2^18
items under the same quantifiers: words below the deciding unit of the first
block carry the value that does not decide it, the deciding word carries the
given lane values when the block reaches the lanes (otherwise the deciding
value), and the words above carry the deciding value; with no solution flag
every item carries the call's value.  The items are reduced by the oracle
and by the GPU tree and compared with the expected (FinalResult, value).
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from test_opencl_quant_reducer import pack

HERE = os.path.dirname(os.path.abspath(__file__))


def load():
    with open(os.path.join(HERE, "golden", "cpu_outputs_final_result.json")) as f:
        return json.load(f)["cases"]


def items_of(c):
    Q, eb, tl = c["quants"], c["elem_bits"], c["type_len"]
    tb = tl.bit_length() - 1                         # lane bits (8)
    wb = eb - tb                                     # word-index bits (10)
    wfb = len(Q) - eb                                # first input of the call
    out = c["outputs"]
    base = tl >> 5
    value = 1 if out[base] else 0
    fqb = len(Q) - len(Q.lstrip(Q[0]))
    if out[base + 1] != 1:
        return Q[wfb:], np.full(1 << eb, value, dtype=np.uint8)
    dv = 1 if Q[0] == "E" else 0
    fw = min(fqb - wfb, wb)
    w_star = out[base + 2] | (out[base + 3] << 32)   # deciding word, first input most significant
    u_star = w_star >> (wb - fw)
    lanes = np.array([(out[i >> 5] >> (i & 31)) & 1 for i in range(tl)], dtype=np.uint8)
    items = np.empty((1 << wb, tl), dtype=np.uint8)
    for w in range(1 << wb):
        u = w >> (wb - fw)
        if u < u_star:
            items[w] = 1 - dv
        elif w == w_star and fw == wb and fqb > len(Q) - tb:
            items[w] = lanes
        else:
            items[w] = dv
    return Q[wfb:], items.reshape(-1)


def check(c, reduce):
    q, items = items_of(c)
    got = reduce(q, pack(items))
    value = (got["solution"] is not None) ^ got["reversed"]
    assert value == c["value"], (c, got)
    if c["expected"] is not None:
        assert {k: got[k] for k in ("reversed", "solution_bits", "solution")} == c["expected"], (c, got)


def oracle_reduce(q, words):
    qr = O.QuantReducer(q)
    qr.push_words(words)
    return qr.final_result()


def test_vectors_are_present():
    cs = load()
    assert len(cs) == 12 and sum(c["expected"] is not None and c["expected"]["solution"] is not None
                                 for c in cs) == 7


def test_oracle_reproduces_every_vector():
    for c in load():
        check(c, oracle_reduce)


@pytest.mark.gpu
def test_gpu_tree_reproduces_every_vector(ctx):
    for c in load():
        check(c, lambda q, words: ctx.qsat_reduce_words(q, words))
