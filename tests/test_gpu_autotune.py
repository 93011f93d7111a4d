"""nsat_autotune: the tuned launch shape changes no answer, is one of the
timed candidates, and is reused from the kernel cache directory."""
import os

import pytest

from naivesat_b200 import api
from naivesat_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_sat_tuning_keeps_answers(ctx, tmp_path, monkeypatch):
    monkeypatch.setenv("NSAT_JIT_CACHE", str(tmp_path))
    c = W.random_dag(21, 30, 800, output="live")
    h = ctx.circuit(c)
    before = h.sat(find_all=True)
    t = h.autotune("sat", persist=True, sample_ms=20)
    assert t["candidates"] >= 8 and not t["from_cache"]
    assert t["block_threads"] in (128, 256, 512) and t["min_blocks"] >= 1
    assert t["best_rate"] >= 0.97 * t["default_rate"]
    after = h.sat(find_all=True)
    assert (after["count"], after["witness"]) == (before["count"], before["witness"])
    assert any(f.startswith("tune_") for f in os.listdir(tmp_path))
    h2 = ctx.circuit(c)
    again = h2.autotune("sat", persist=True)
    assert again["from_cache"] and again["candidates"] == 0
    assert (again["block_threads"], again["min_blocks"], again["cta_bits_max"]) == \
        (t["block_threads"], t["min_blocks"], t["cta_bits_max"])
    r = h2.sat(find_all=True)
    assert (r["count"], r["witness"]) == (before["count"], before["witness"])
    h2.autotune_reset()
    assert h2.sat(find_all=True)["count"] == before["count"]


def test_qsat_tuning_keeps_answers(ctx, tmp_path, monkeypatch):
    monkeypatch.setenv("NSAT_JIT_CACHE", str(tmp_path))
    c = W.config("c2c")
    h = ctx.circuit(c)
    before = h.qsat(c.quants)
    t = h.autotune("qsat", quants=c.quants, sample_ms=20)
    after = h.qsat(c.quants)
    for k in ("reversed", "solution_bits", "solution", "value"):
        assert after[k] == before[k]
    assert t["best_rate"] >= 0.97 * t["default_rate"]
