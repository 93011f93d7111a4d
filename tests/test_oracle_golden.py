"""The CPU oracle against the reference's own known-answer vectors.

Fixtures in tests/golden/ were extracted from the reference's unit tests by
tests/golden/gen_golden.py; this file pins the oracle to them before the
oracle is trusted as the checker of the CUDA path.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    with open(os.path.join(GOLD, name)) as f:
        return json.load(f)["cases"]


def tree_value(quants, items):
    qr = O.QuantReducer(quants)
    for k, it in enumerate(items):
        qr.push(k, it)
    fr = qr.final_result()
    return (fr["solution"] is not None) ^ fr["reversed"]


@pytest.mark.parametrize("i", range(len(load("quant_reducer.json"))))
def test_quant_reducer_kat(i):
    """qsat.rs test_quant_reducer: pushes in the given order, checks the final
    result from `push_index` on."""
    c = load("quant_reducer.json")[i]
    qr = O.QuantReducer(c["quants"])
    for j, idx in enumerate(c["ordering"]):
        qr.push(idx, c["items"][idx])
        if c["push_index"] is not None and j >= c["push_index"]:
            assert qr.final_result() == c["result"], (i, j)
    assert qr.final_result() == c["result"]


def test_quant_reducer_push_words_kat():
    """The packed-word push (items in index order) gives the reference's
    final results on the test_quant_reducer cases of >= 32 items."""
    n = 0
    for c in load("quant_reducer.json"):
        nq = len(c["quants"])
        if nq < 5:
            continue
        words = [0] * ((1 << nq) // 32)
        for k, it in enumerate(c["items"]):
            if it:
                words[k >> 5] |= 1 << (k & 31)
        qr = O.QuantReducer(c["quants"])
        qr.push_words(words)
        assert qr.final_result() == c["result"], c
        n += 1
    assert n >= 10


def test_aggr_tree_cpu_kat():
    """qsat.rs test_aggr_output_cpu_code: quantifier tree over word bits."""
    for c in load("aggr_tree_cpu.json"):
        items = [(c["words"][k >> 5] >> (k & 31)) & 1 for k in range(1 << len(c["quants"]))]
        assert tree_value(c["quants"], items) == c["result"], c


def test_aggr_tree_opencl_kat():
    """qsat.rs test_aggr_output_opencl_code: tree over one 32-lane word with
    the last five quantifiers."""
    for c in load("aggr_tree_opencl.json"):
        q = c["quants"][-5:]
        items = [(c["words"][0] >> k) & 1 for k in range(32)]
        assert tree_value(q, items) == c["result"], c


def test_greedy_find_solution_kat():
    """greedysatostop.rs test_mem_image_find_solution (10 cases)."""
    for c in load("greedy_find_solution.json"):
        sl = c["state_len"]
        data = np.zeros((c["len"] * (sl + 1)) >> 6, dtype=np.uint64)
        O.memimage_set(data, sl, c["pos_sol"], (1 << sl) | (c["next"] & ((1 << sl) - 1)))
        got = O.memimage_find_solution(data, sl, c["start"], c["len"], c["unknowns"])
        assert got == c["expected"], c


def test_greedy_mem_image_kat():
    """greedysatostop.rs test_mem_image: packed (state_len+1)-bit entries."""
    M = (1 << 64) - 1
    for c in load("greedy_mem_image.json"):
        sl, ln = c["state_len"], c["len"]
        data = np.array([((i * 5884491582115956921) + 5560939029013487713) & M
                         for i in range((ln * (sl + 1)) >> 6)], dtype=np.uint64)
        assert len(data) == (sl + 1) * (ln >> 6)
        mask = (1 << (sl + 1)) - 1
        for i in range(ln):
            O.memimage_set(data, sl, i, ((i * c["mult"]) + c["add"]) & M)
        bits = np.unpackbits(data.view(np.uint8), bitorder="little")
        for i in range(0, ln, max(1, ln // 200)):
            exp = (((i * c["mult"]) + c["add"]) & M) & mask
            raw = 0
            for b in range(sl + 1):
                raw |= int(bits[i * (sl + 1) + b]) << b
            assert raw == exp and O.memimage_get(data, sl, i) == exp, (c, i)


def test_quant_reducer_matches_scalar_qsat():
    """Chunked (mode 1) and single-reducer (mode 0) oracle QSAT agree with a
    pure scalar evaluation on small random circuits."""
    from naivesat_b200 import workloads as W
    rng = W.SplitMix64(77)
    for t in range(12):
        n = 11 + rng.below(6)
        c = W.random_dag(100 + t, n, 40 + rng.below(80), output="live")
        q = "".join("A" if rng.below(2) else "E" for _ in range(n))
        oc = O.Circuit(c.n, c.gates, c.outputs)
        r0 = O.qsat(oc, q, mode=0)
        r1 = O.qsat(oc, q, mode=1)
        qr = O.QuantReducer(q)
        for v in range(1 << n):
            bits = [(v >> (n - 1 - i)) & 1 for i in range(n)]
            qr.push(v, c.eval_bits(bits)[0])
        r2 = qr.final_result()
        assert r0 == r1 == r2, (t, q, r0, r1, r2)


def test_sat_oracle_matches_scalar():
    from naivesat_b200 import workloads as W
    for t in range(6):
        c = W.random_dag(200 + t, 12 + t, 60, output="live")
        oc = O.Circuit(c.n, c.gates, c.outputs)
        cnt, low = O.sat_range(oc)
        sols = [v for v in range(1 << c.n) if c.eval_bits([(v >> i) & 1 for i in range(c.n)])[0]]
        assert cnt == len(sols)
        assert low == (sols[0] if sols else None)


def test_file_image_partitions_kat():
    """greedysatostop.rs test_file_image (1271): chunks saved in order form
    the image, partition p holds entries [p L, (p+1) L), and a saved
    partition replaces exactly those entries.  Same generator (i * mult +
    add, then (i + changer) * mult + add), at state_len 14 instead of 26 to
    keep the CPU suite short."""
    c = load("greedy_file_image.json")[0]
    sl, mult, add, parts, changer = 14, c["mult"], c["add"], 16, c["changer"]
    m64 = (1 << 64) - 1
    mask = (1 << (sl + 1)) - 1
    n = 1 << sl
    img = np.zeros((n * (sl + 1)) // 64, dtype=np.uint64)
    for i in range(n):                         # save_chunk x 2 * parts, in order
        O.memimage_set(img, sl, i, (i * mult + add) & m64)
    plen = n // parts
    pwords = plen * (sl + 1) // 64
    for p in reversed(range(parts)):           # load_partition
        part = img[p * pwords:(p + 1) * pwords]
        for ci in range(0, plen, 37):
            i = plen * p + ci
            assert O.memimage_get(part, sl, ci) == ((i * mult + add) & m64) & mask
    for p in reversed(range(parts)):           # save_partition
        part = np.zeros(pwords, dtype=np.uint64)
        for ci in range(plen):
            O.memimage_set(part, sl, ci, ((plen * p + ci + changer) * mult + add) & m64)
        img[p * pwords:(p + 1) * pwords] = part
    for i in range(0, n, 29):
        assert O.memimage_get(img, sl, i) == ((i + changer) * mult + add) & m64 & mask
