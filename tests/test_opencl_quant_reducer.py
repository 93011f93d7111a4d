"""The reference's test_opencl_quant_reducer vectors (qsat.rs:4038-6008: 52
cases, 143 vectors) as item patterns for the forall/exists reduction.

Each vector hands the reference's multi-level reducer one u16 per group of
the bits reduce_end_bit .. reduce_end_bit + init_group_len_bits (bit 15 the
group's value, bits 0..14 the group-local index of the first decisive unit,
0x7fff none), for every assignment of the bits reduce_start_bit ..
reduce_end_bit in index order, and expects the FinalResult of the formula
from reduce_start_bit on (qsat.rs:1095-1264) and its value.  Here every group
becomes leaf items under the same quantifiers: all leaves carry the group's
value, except that when the first quantifier block reaches into the group
and the group's value decides it, the units of that block below the local
index get the other value.  A unit's leaves are constant, so one item per
unit carries the same information; the items are reduced by the oracle's
QuantReducer and by the GPU tree (nsat_qsat_reduce_words) and compared with
the reference's expected (FinalResult, value).  The reference returns no
FinalResult when the first block of the whole formula does not reach
reduce_start_bit (qsat.rs:1164-1167); only the value is compared there.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))


def load():
    with open(os.path.join(HERE, "golden", "opencl_quant_reducer.json")) as f:
        return json.load(f)["cases"]


def expand(rle):
    out = []
    for v, n in rle:
        out.extend([v] * n)
    return out


def items_of(c):
    """(quantifiers, items in index order, first block reaches the reducer?)"""
    s, e, b, Q = c["reduce_start_bit"], c["reduce_end_bit"], c["init_group_len_bits"], c["quants"]
    first = Q[0]
    dv = 1 if first == "E" else 0                    # the value that decides the first block
    run = 0
    while s + run < len(Q) and Q[s + run] == first:
        run += 1
    have_first = all(q == first for q in Q[1:s + 1])
    groups = expand(c["inputs_rle"])
    assert len(groups) == 1 << (e - s)
    fp = min(run - (e - s), b) if (have_first and run > e - s) else 0
    items = []
    for g in groups:
        v, li = (g >> 15) & 1, g & 0x7FFF
        if fp and v == dv:
            assert li != 0x7FFF
            u_star = li >> (b - fp)                  # the local index's bits of the first block
            items.extend(dv if u >= u_star else 1 - dv for u in range(1 << fp))
        else:
            items.extend([v] * (1 << fp))
    return Q[s:e + fp], items, have_first


def padded(q, items):
    """At least 5 bits (32 items): extra innermost quantifiers, the opposite
    of the last one, repeat every item (no effect on value or witness)."""
    pad = max(0, 5 - len(q))
    if pad:
        q = q + ("E" if q[-1] == "A" else "A") * pad
        items = [x for x in items for _ in range(1 << pad)]
    return q, items


def pack(items):
    a = np.asarray(items, dtype=np.uint8).reshape(-1, 32)
    return (a.astype(np.uint64) << np.arange(32, dtype=np.uint64)).sum(axis=1).astype(np.uint32)


def check(c, reduce):
    q, items, have_first = items_of(c)
    if not q:
        assert items[0] == c["value"] and c["expected"] is None
        return
    q, items = padded(q, items)
    got = reduce(q, items)
    value = (got["solution"] is not None) ^ got["reversed"]
    assert value == c["value"], (c["case"], got, c["value"])
    if c["expected"] is None:
        assert not have_first or value != (q[0] == "E"), c["case"]
    else:
        assert {k: got[k] for k in ("reversed", "solution_bits", "solution")} == c["expected"], \
            (c["case"], got, c["expected"])


def oracle_reduce(q, items):
    qr = O.QuantReducer(q)
    qr.push_words(pack(items))
    return qr.final_result()


def test_vectors_are_present():
    cases = load()
    assert len(cases) == 143 and len({c["case"] for c in cases}) == 52


def test_oracle_reproduces_every_vector():
    for c in load():
        check(c, oracle_reduce)


@pytest.mark.gpu
def test_gpu_tree_reproduces_every_vector(ctx):
    for c in load():
        check(c, lambda q, items: ctx.qsat_reduce_words(q, pack(items)))
