"""Batched serving (nsat_server_*): every job's answer in a mixed batch
equals the oracle's and equals the same job served alone."""
import pytest

from naivesat_b200 import api
from naivesat_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def small_mix(count, seed):
    return W.serving_requests(count, seed=seed, rate_hz=1e9, n_range=(12, 22), g_range=(40, 600),
                              stop_n_range=(8, 14))


def expected(req):
    c = req["circ"]
    oc = O.Circuit(c.n, c.gates, c.outputs)
    if req["kind"] == "sat":
        cnt, low = O.sat_range(oc)
        return {"satisfiable": low is not None, "witness": low}
    if req["kind"] == "qsat":
        r = O.qsat(oc, req["quants"], mode=1)
        return {"reversed": r["reversed"], "solution_bits": r["solution_bits"], "solution": r["solution"]}
    r = O.stop_solve(c.n, req["unknowns"], O.stop_table(oc), mode=1)
    if r is None:
        return {"found": False}
    return {"found": True, "start": r["start"], "end": r["end"], "steps": r["steps"]}


def project(res, exp):
    return {k: res[k] for k in exp}


def submit_all(srv, reqs):
    ids = {}
    for i, r in enumerate(reqs):
        ids[srv.submit(r["kind"], r["circ"], quants=r["quants"], unknowns=r["unknowns"], tag=i)] = i
    return ids


def test_mixed_batch_matches_oracle_and_alone(ctx):
    reqs = small_mix(48, 11)
    srv = api.Server(ctx)
    submit_all(srv, reqs)
    res = {r["tag"]: r for r in srv.run_all()}
    assert len(res) == len(reqs)
    for i, r in enumerate(reqs):
        exp = expected(r)
        assert project(res[i], exp) == exp, (i, r["kind"], res[i], exp)
    # the same jobs, each alone
    for i in range(0, len(reqs), 3):
        alone = api.Server(ctx)
        alone.submit(reqs[i]["kind"], reqs[i]["circ"], quants=reqs[i]["quants"], unknowns=reqs[i]["unknowns"])
        got = alone.run_all()[0]
        exp = expected(reqs[i])
        assert project(got, exp) == project(res[i], exp)
        alone.close()


def test_find_all_counts_every_solution(ctx):
    reqs = [r for r in small_mix(40, 31) if r["kind"] == "sat"][:12]
    srv = api.Server(ctx)
    for i, r in enumerate(reqs):
        srv.submit("sat", r["circ"], tag=i, find_all=True)
    res = {r["tag"]: r for r in srv.run_all()}
    for i, r in enumerate(reqs):
        c = r["circ"]
        cnt, low = O.sat_range(O.Circuit(c.n, c.gates, c.outputs))
        assert (res[i]["count"], res[i]["satisfiable"], res[i]["witness"]) == (cnt, low is not None, low), i


def test_large_jobs_match_one_shot_solvers(ctx):
    """n = 26..30 jobs against the compiled one-shot solvers (the oracle would
    be slow here); slices span many epochs."""
    reqs = W.serving_requests(6, seed=5, rate_hz=1e9, n_range=(26, 30), g_range=(200, 1200), mix=(0.5, 0.5, 0.0))
    srv = api.Server(ctx)
    submit_all(srv, reqs)
    sat0 = next(i for i, r in enumerate(reqs) if r["kind"] == "sat")
    srv.submit("sat", reqs[sat0]["circ"], tag=100, find_all=True)
    res = {r["tag"]: r for r in srv.run_all()}
    full = ctx.circuit(reqs[sat0]["circ"]).sat(find_all=True)
    assert (res[100]["count"], res[100]["witness"]) == (full["count"], full["witness"])
    for i, r in enumerate(reqs):
        h = ctx.circuit(r["circ"])
        if r["kind"] == "sat":
            one = h.sat(find_all=False)
            assert (res[i]["satisfiable"], res[i]["witness"]) == (one["satisfiable"], one["witness"])
        else:
            one = h.qsat(r["quants"])
            assert (res[i]["reversed"], res[i]["solution_bits"], res[i]["solution"]) == \
                (one["reversed"], one["solution_bits"], one["solution"])


def test_admission_by_memory_and_queue_limit(ctx):
    reqs = [r for r in small_mix(40, 23) if r["kind"] == "stop"][:4]
    assert reqs
    # room for about one table at a time: the rest wait in the queue
    srv = api.Server(ctx, arena_bytes=2 * 8 * (1 << 14) + 65536, max_queue=3)
    submitted = 0
    with pytest.raises(api.NsatError, match="EBUSY"):
        for r in reqs + reqs:
            srv.submit(r["kind"], r["circ"], unknowns=r["unknowns"], tag=submitted)
            submitted += 1
    assert submitted == 3
    res = srv.run_all()
    assert len(res) == 3
    for r in res:
        exp = expected(reqs[r["tag"] % len(reqs)])
        assert project(r, exp) == exp


def test_job_larger_than_arena_is_answered_with_enomem(ctx):
    """Programs are built off the caller's thread; a job that can never fit
    the arena comes back with NSAT_ENOMEM and the others are served."""
    reqs = [r for r in small_mix(30, 41) if r["kind"] == "sat"][:6]
    big = W.random_dag(3, 20, 3000, output="live")
    srv = api.Server(ctx, arena_bytes=20000, build_threads=2)
    for i, r in enumerate(reqs):
        srv.submit("sat", r["circ"], tag=i)
    srv.submit("sat", big, tag=99)
    res = {r["tag"]: r for r in srv.run_all()}
    assert res[99]["status"] == -2
    for i, r in enumerate(reqs):
        exp = expected(r)
        assert res[i]["status"] == 0
        assert project(res[i], exp) == exp


@pytest.mark.parametrize("wait", [True, False])
def test_qsat_tiering_matches_one_shot(ctx, wait):
    """QSAT jobs racing a compiled kernel (tier_min_ms=1 makes every large
    one a candidate): with tier_wait every block runs compiled, without it
    the interpreter and the compiled blocks share the job; the answers equal
    the one-shot solver's (decisive units inside blocks, blocks inside units,
    and formulas decided by the reducer alike)."""
    reqs = []
    for seed in range(8):
        n = 28 + seed % 3
        c = W.random_dag(500 + seed, n, 900, output="live")
        reqs.append((c, W.alternating_quants(seed, n, 1 + seed % 5)))
    # first blocks that reach below the tile: units smaller than a tile, no reducer
    c = W.random_dag(600, 28, 900, output="live")
    reqs.append((c, "E" * 25 + "AEA"))
    reqs.append((c, "A" * 26 + "EA"))
    srv = api.Server(ctx, tier_min_ms=1, tier_wait=wait)
    for i, (c, q) in enumerate(reqs):
        srv.submit("qsat", c, quants=q, tag=i)
    res = {r["tag"]: r for r in srv.run_all()}
    srv.close()
    compiled = 0
    for i, (c, q) in enumerate(reqs):
        one = ctx.circuit(c).qsat(q)
        got = res[i]
        assert got["status"] == 0
        assert (got["reversed"], got["solution_bits"], got["solution"]) == \
            (one["reversed"], one["solution_bits"], one["solution"]), (i, got, one)
        compiled += got["compiled_blocks"]
    if wait:
        assert compiled > 0


def test_continuous_batching_jobs_arrive_while_others_run(ctx):
    """Continuous batching: long jobs are put in flight first, then new SAT /
    QSAT / SATOSTOP jobs are submitted between server steps -- four SATOSTOP
    jobs at once while the arena has room for two of their tables, so the
    others wait for memory -- and every result equals the oracle (the
    one-shot solvers for the long jobs) and the same job served alone.  The
    epoch ranges that poll returns show that the late jobs ran in the same
    epochs as the long ones, and that the memory waiters were admitted only
    after an earlier table was released."""
    import time
    # about 1200 LUTs over 2^32 assignments each: over 100 ms of interpreter
    # time in slices that double per epoch, so they run through the whole test
    longs = [{"kind": "sat", "circ": W.random_dag(820 + s, 32, 3000, output="live"), "quants": None,
              "unknowns": 0, "find_all": True} for s in range(2)]
    qc = W.random_dag(810, 29, 400, output="live")
    longs.append({"kind": "qsat", "circ": qc, "quants": "A" * 13 + "E" * 16, "unknowns": 0})
    late = [r for r in small_mix(40, 75) if r["kind"] != "stop"][:14]
    waiters = [{"kind": "stop", "circ": W.lfsr_stop(90 + s, 14, 120), "quants": None, "unknowns": 7}
               for s in range(4)]
    table_pair = 2 * 8 * (1 << 14)
    srv = api.Server(ctx, arena_bytes=2 * table_pair + 192 * 1024, tier_min_ms=0xFFFFFFFF)
    reqs, res = [], {}

    def submit(r):
        reqs.append(r)
        srv.submit(r["kind"], r["circ"], quants=r["quants"], unknowns=r["unknowns"], tag=len(reqs) - 1,
                   find_all=r.get("find_all", False))

    trace = []        # per step: active, queued, epochs processed, kernels launched

    def step():
        a, q = srv.step()
        for x in srv.poll():
            res[x["tag"]] = x
        st = srv.stats()
        trace.append((a, q, st["epochs"], st["launches"]))
        return a, q

    for r in longs:
        submit(r)
    time.sleep(0.05)                 # programs are built on the server's builder threads
    for _ in range(3):
        step()
    assert not any(i in res for i in range(len(longs))), "long jobs must still be running"
    late_tags, wait_tags = [], []
    for k, r in enumerate(late):
        submit(r)
        late_tags.append(len(reqs) - 1)
        if k == 4:
            for w in waiters:
                submit(w)
                wait_tags.append(len(reqs) - 1)
        time.sleep(0.01)
        a, q = step()
        if k == 4:
            time.sleep(0.05)
            a, q = step()
    for x in srv.run_all():
        res[x["tag"]] = x
    srv.close()
    assert sorted(res) == list(range(len(reqs)))
    assert all(res[i]["status"] == 0 for i in res)

    # every answer: the oracle (small jobs) or the one-shot solvers (long jobs)
    for i, r in enumerate(reqs):
        if i < len(longs):
            h = ctx.circuit(r["circ"])
            if r["kind"] == "sat":
                one = h.sat(find_all=True)
                assert (res[i]["count"], res[i]["witness"]) == (one["count"], one["witness"]), i
            else:
                one = h.qsat(r["quants"])
                assert (res[i]["reversed"], res[i]["solution_bits"], res[i]["solution"]) == \
                    (one["reversed"], one["solution_bits"], one["solution"]), i
        else:
            exp = expected(r)
            assert project(res[i], exp) == exp, (i, r["kind"], res[i], exp)
    # ... and the same job served alone
    for i, r in enumerate(reqs):
        alone = api.Server(ctx, tier_min_ms=0xFFFFFFFF)
        alone.submit(r["kind"], r["circ"], quants=r["quants"], unknowns=r["unknowns"],
                     find_all=r.get("find_all", False))
        got = alone.run_all()[0]
        alone.close()
        # a find-mode SAT job's count covers the slices processed before its
        # first solution was seen, which depends on the epochs it shared, so
        # counts are compared for full-count jobs only
        sat_keys = ("count", "satisfiable", "witness") if r.get("find_all") else ("satisfiable", "witness")
        keys = sat_keys if r["kind"] == "sat" else \
            ("reversed", "solution_bits", "solution") if r["kind"] == "qsat" else ("found", "start", "end", "steps")
        assert {k: got[k] for k in keys} == {k: res[i][k] for k in keys}, (i, got, res[i])

    # the late jobs shared epochs with the long ones
    def overlaps(a, b):
        return res[a]["first_epoch"] <= res[b]["last_epoch"] and res[b]["first_epoch"] <= res[a]["last_epoch"]
    shared = [t for t in late_tags if any(overlaps(t, L) for L in range(len(longs)))]
    assert len(shared) >= len(late_tags) // 2, ([(t, res[t]["first_epoch"], res[t]["last_epoch"]) for t in late_tags],
                                                trace)
    assert all(res[L]["epochs"] > 3 for L in range(2))
    # the memory waiters: admitted after an earlier SATOSTOP job had finished and released its tables
    done_before = sorted(res[t]["done_ms"] for t in wait_tags)
    admitted_late = [t for t in wait_tags if res[t]["admit_ms"] >= done_before[0]]
    assert len(admitted_late) >= 2, ([(res[t]["admit_ms"], res[t]["done_ms"]) for t in wait_tags], trace)
    # and every waiter still ran while the long jobs were active
    assert any(overlaps(t, L) for t in wait_tags for L in range(len(longs)))


@pytest.mark.parametrize("shape", range(1, api.SERVE_SHAPES + 1))
def test_every_interpreter_shape_matches_oracle(ctx, shape):
    """The same mixed batch under each interpreter shape (words per lane,
    group size, mux tree or jump on the truth table): every answer equals
    the oracle's."""
    reqs = small_mix(24, 61)
    srv = api.Server(ctx, shape=shape, tier_min_ms=0xFFFFFFFF)
    assert srv.stats()["shape"] == shape
    submit_all(srv, reqs)
    res = {r["tag"]: r for r in srv.run_all()}
    srv.close()
    for i, r in enumerate(reqs):
        exp = expected(r)
        assert project(res[i], exp) == exp, (shape, i, r["kind"], res[i], exp)


def test_server_tune_persists_and_is_used(ctx, tmp_path, monkeypatch):
    """nsat_server_tune times every shape and four epoch budgets, persists
    its choice for this GPU, and a server created with the defaults uses it."""
    monkeypatch.setenv("NSAT_JIT_CACHE", str(tmp_path))
    t = api.server_tune(ctx, jobs=8, persist=True)
    assert 1 <= t["shape"] <= api.SERVE_SHAPES and not t["from_cache"]
    assert all(x > 0 for x in t["lut_words_per_s"])
    assert t["epoch_budget"] in (6000000, 12000000, 24000000, 48000000)
    again = api.server_tune(ctx, persist=True)
    assert again["from_cache"] and again["shape"] == t["shape"] and again["epoch_budget"] == t["epoch_budget"]
    srv = api.Server(ctx)
    assert srv.stats()["shape"] == t["shape"]
    srv.close()


def test_rollover_matches_oracle(ctx):
    """With roll-over on, warps that run out of planned work claim the next
    quarter slice of undecided SAT and SATOSTOP jobs from the device cursors;
    every answer still equals the oracle's (counts included for count-mode
    jobs, so no tile is evaluated twice or skipped)."""
    reqs = small_mix(36, 67)
    srv = api.Server(ctx, rollover=True, tier_min_ms=0xFFFFFFFF)
    for i, r in enumerate(reqs):
        srv.submit(r["kind"], r["circ"], quants=r["quants"], unknowns=r["unknowns"], tag=i,
                   find_all=(r["kind"] == "sat" and i % 2 == 0))
    res = {r["tag"]: r for r in srv.run_all()}
    srv.close()
    for i, r in enumerate(reqs):
        exp = expected(r)
        assert project(res[i], exp) == exp, (i, r["kind"], res[i], exp)
        if r["kind"] == "sat" and i % 2 == 0:
            c = r["circ"]
            assert res[i]["count"] == O.sat_range(O.Circuit(c.n, c.gates, c.outputs))[0], i
