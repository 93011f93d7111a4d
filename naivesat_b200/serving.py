"""Request-trace driver for the batched serving engine.

Replays a trace of requests (workloads.serving_requests: SAT / QSAT /
SATOSTOP circuits with Poisson arrival times) in real time against

* a Server (nsat_server_*: continuous batching; requests that arrive while
  others run are admitted as slots and arena memory free up), or
* the plain one-launch-per-instance form: one request at a time, in arrival
  order, through the one-shot solvers (a kernel compiled for that circuit
  and its own launches), which is what one naivesat / naiveqsat /
  naivesatostop process per circuit does on a GPU,

and reports solves/s and latency percentiles.  Latency runs from a
request's scheduled arrival to the moment the driver holds its result, so
host-side queueing counts.
"""
import os
import tempfile
import time

from . import api

VERDICT_KEYS = {
    "sat": ("satisfiable", "witness"),
    "qsat": ("reversed", "solution_bits", "solution"),
    "stop": ("found", "start", "end", "steps"),
}


def verdict(kind, res):
    """The part of a result that must be bit-exact between forms."""
    return tuple(res.get(k) for k in VERDICT_KEYS[kind])


def percentile(xs, p):
    if not xs:
        return None
    s = sorted(xs)
    k = min(len(s) - 1, max(0, int(round(p / 100.0 * (len(s) - 1)))))
    return s[k]


def summarize(lat_s, makespan_s, count):
    return {"requests": count, "solves_per_s": count / makespan_s if makespan_s > 0 else None,
            "makespan_s": makespan_s,
            "p50_ms": percentile(lat_s, 50) * 1e3 if lat_s else None,
            "p99_ms": percentile(lat_s, 99) * 1e3 if lat_s else None,
            "mean_ms": sum(lat_s) / len(lat_s) * 1e3 if lat_s else None}


def replay_server(srv, reqs, realtime=True, time_limit_s=None, burst=128):
    """Submits each request at its arrival time (all at time 0 when realtime
    is False), at most `burst` per step so the device starts while a backlog
    is still being submitted, steps the server, and collects results.
    Returns (results by index, latencies in s, makespan in s)."""
    t0 = time.perf_counter()
    arrival = [r["arrival_s"] if realtime else 0.0 for r in reqs]
    results, lat = {}, {}
    i = 0
    active = queued = 0
    while len(results) < len(reqs):
        now = time.perf_counter() - t0
        if time_limit_s is not None and now > time_limit_s:
            break
        b = 0
        while i < len(reqs) and arrival[i] <= now and b < burst:
            b += 1
            r = reqs[i]
            srv.submit(r["kind"], r["circ"], quants=r["quants"], unknowns=r["unknowns"], tag=i,
                       find_all=r.get("find_all", False))
            i += 1
        if active or queued or i > len(results):
            active, queued = srv.step()
        else:
            # idle: wait for the next arrival
            time.sleep(max(0.0, min(arrival[i] - now, 0.002)))
        t = time.perf_counter() - t0
        for res in srv.poll():
            k = res["tag"]
            results[k] = res
            lat[k] = t - arrival[k]
    makespan = (time.perf_counter() - t0) - (arrival[0] if reqs else 0.0)
    return results, [lat[k] for k in sorted(lat)], makespan


def solve_one(ctx, req):
    """One request through the one-shot solvers (per-circuit kernel)."""
    h = ctx.circuit(req["circ"])
    kind = req["kind"]
    if kind == "sat":
        r = h.sat(find_all=req.get("find_all", False))
        out = {"satisfiable": r["satisfiable"], "witness": r["witness"], "count": r["count"]}
    elif kind == "qsat":
        r = h.qsat(req["quants"])
        out = {"reversed": r["reversed"], "solution_bits": r["solution_bits"], "solution": r["solution"]}
    else:
        t = h.stop_table(want_steps=True)
        r = t.solve(req["unknowns"], mode=1)
        t.close()
        out = {"found": r["found"], "start": r.get("start"), "end": r.get("end"), "steps": r.get("steps")}
    h.close()
    return out


def replay_plain(ctx, reqs, realtime=True, time_limit_s=None, fresh_jit_cache=True):
    """The plain form: requests one at a time in arrival order.  With
    fresh_jit_cache every circuit is compiled as a new process would (an
    empty on-disk kernel cache).  Stops after time_limit_s.  Returns
    (results by index, latencies in s, busy time in s)."""
    old = os.environ.get("NSAT_JIT_CACHE")
    tmp = tempfile.TemporaryDirectory(prefix="nsat_plain_") if fresh_jit_cache else None
    if tmp is not None:
        os.environ["NSAT_JIT_CACHE"] = tmp.name
    try:
        t0 = time.perf_counter()
        results, lat = {}, {}
        busy = 0.0
        for i, req in enumerate(reqs):
            arr = req["arrival_s"] if realtime else 0.0
            now = time.perf_counter() - t0
            if time_limit_s is not None and now > time_limit_s:
                break
            if arr > now:
                time.sleep(arr - now)
            s = time.perf_counter()
            results[i] = solve_one(ctx, req)
            e = time.perf_counter()
            busy += e - s
            lat[i] = (e - t0) - arr
        return results, [lat[k] for k in sorted(lat)], busy
    finally:
        if tmp is not None:
            if old is None:
                os.environ.pop("NSAT_JIT_CACHE", None)
            else:
                os.environ["NSAT_JIT_CACHE"] = old
            tmp.cleanup()


def fifo_latencies(arrivals, service):
    """Latencies of a single FIFO server with the given service times (the
    plain form handles one request at a time, so its queueing follows from
    its measured service times)."""
    end = 0.0
    lat = []
    for a, sv in zip(arrivals, service):
        start = max(a, end)
        end = start + sv
        lat.append(end - a)
    return lat


def plain_service_times(ctx, reqs, time_limit_s, fresh_jit_cache=True, cache_dir=None):
    """Solves requests one at a time (back to back) until time_limit_s;
    returns (results by index, service time of each in s).  With
    fresh_jit_cache the kernels compile into an empty on-disk cache, as in a
    new process; cache_dir instead names the on-disk cache to use (a second
    pass over the same requests with the same directory finds every kernel
    compiled: the warm-cache plain form).  NVRTC also keeps what it compiles
    in the CUDA compute cache (CUDA_CACHE_PATH), which is read once per
    process: a caller timing cold compiles points it at an empty directory
    before the process first uses CUDA, as bench.py does."""
    old = os.environ.get("NSAT_JIT_CACHE")
    tmp = tempfile.TemporaryDirectory(prefix="nsat_plain_") if (fresh_jit_cache and cache_dir is None) else None
    if tmp is not None:
        os.environ["NSAT_JIT_CACHE"] = tmp.name
    elif cache_dir is not None:
        os.environ["NSAT_JIT_CACHE"] = cache_dir
    try:
        t0 = time.perf_counter()
        results, service = {}, []
        for i, req in enumerate(reqs):
            if time.perf_counter() - t0 > time_limit_s:
                break
            s = time.perf_counter()
            results[i] = solve_one(ctx, req)
            service.append(time.perf_counter() - s)
        return results, service
    finally:
        if tmp is not None or cache_dir is not None:
            if old is None:
                os.environ.pop("NSAT_JIT_CACHE", None)
            else:
                os.environ["NSAT_JIT_CACHE"] = old
        if tmp is not None:
            tmp.cleanup()


def interpreter_alone_service_times(srv, reqs):
    """The precompiled interpreter without batching: one request at a time
    through a server that holds no other job (submit, step until answered,
    next).  Returns (results by index, service time of each in s)."""
    results, service = {}, []
    for i, r in enumerate(reqs):
        s = time.perf_counter()
        srv.submit(r["kind"], r["circ"], quants=r["quants"], unknowns=r["unknowns"], tag=i,
                   find_all=r.get("find_all", False))
        got = srv.run_all()
        service.append(time.perf_counter() - s)
        assert len(got) == 1 and got[0]["tag"] == i
        results[i] = got[0]
    return results, service
