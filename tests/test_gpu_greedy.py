"""Partitioned greedysatostop (nsat_greedy_solve, greedysatostop -p/-x):
the packed image has the reference's MemImage/FileImage layout, and the
partition-by-partition joins give the oracle's answer (the reference's
schedule), from pinned host memory and from an image file alike."""
import numpy as np
import pytest

from naivesat_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def circuits():
    yield "counter14", W.counter_stop(14)
    for seed, n, g in [(1, 12, 40), (3, 14, 42), (5, 16, 48), (7, 16, 60), (2, 13, 40), (9, 18, 54)]:
        yield "lfsr%d_%d" % (seed, n), W.lfsr_stop(seed, n, g)


def packed(table, n):
    img = np.zeros(((1 << n) * (n + 1) + 63) // 64, dtype=np.uint64)
    for s in range(1 << n):
        O.memimage_set(img, n, s, int(table[s]))
    return img


def test_image_layout_is_the_reference_memimage(ctx, tmp_path):
    c = W.lfsr_stop(3, 14, 42)
    oc = O.Circuit(c.n, c.gates, c.outputs)
    exp = packed(O.stop_table(oc), c.n)
    h = ctx.circuit(c)
    assert (h.greedy_image(4) == exp).all()
    assert (h.greedy_image(8, file_prefix=str(tmp_path) + "/") == exp).all()
    assert list(tmp_path.iterdir()) == []        # the temp image file is removed


@pytest.mark.parametrize("name,circ", list(circuits()))
@pytest.mark.parametrize("partitions", [2, 4, 8])
def test_partitioned_matches_oracle(ctx, name, circ, partitions):
    """Device-resident image for the even partition counts' first unknowns
    setting, host-spilled image (device budget of 1 byte) for the rest."""
    n = circ.n
    oc = O.Circuit(circ.n, circ.gates, circ.outputs)
    table = O.stop_table(oc)
    h = ctx.circuit(circ)
    for k, u in enumerate(sorted({n // 2, n - 2, n})):
        exp = O.greedy_partitioned(n, u, table, partitions)
        spill = (k + partitions) % 2 == 1
        got = h.greedy_partitioned(u, partitions, device_bytes=1 if spill else 0)
        assert got["storage"] == (1 if spill else 0)
        if exp is None:
            assert not got["found"], (name, u)
            continue
        assert got["found"], (name, u)
        assert (got["start"], got["end"], got["stage"], got["partition"]) == \
            (exp["start"], exp["end"], exp["stage"], exp["partition"]), (name, u, got, exp)
        assert O.stop_replay(oc, got["start"], 1 << (n + 1))[0] == got["end"]


def test_device_host_and_file_images_agree(ctx, tmp_path):
    c = W.lfsr_stop(5, 16, 48)
    h = ctx.circuit(c)
    a = h.greedy_partitioned(8, 4)
    b = h.greedy_partitioned(8, 4, device_bytes=1)
    f = h.greedy_partitioned(8, 4, file_prefix=str(tmp_path) + "/")
    assert (a["storage"], b["storage"], f["storage"]) == (0, 1, 2)
    keys = ("found", "start", "end", "stage", "partition", "joins")
    assert {k: a[k] for k in keys} == {k: b[k] for k in keys} == {k: f[k] for k in keys}
    assert a["h2d_bytes"] == 0 and b["h2d_bytes"] == f["h2d_bytes"] > 0
    assert list(tmp_path.iterdir()) == []


def test_partitioned_at_n20_against_oracle(ctx):
    c = W.lfsr_stop(11, 20, 80)
    oc = O.Circuit(c.n, c.gates, c.outputs)
    table = O.stop_table(oc)
    exp = O.greedy_partitioned(20, 12, table, 4)
    for budget in (0, 1):
        got = ctx.circuit(c).greedy_partitioned(12, 4, device_bytes=budget)
        if exp is None:
            assert not got["found"]
        else:
            assert (got["start"], got["end"], got["stage"], got["partition"]) == \
                (exp["start"], exp["end"], exp["stage"], exp["partition"])
