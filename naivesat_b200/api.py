"""ctypes binding of libnsat.so (the C ABI in include/nsat.h).

This is the Python face of the same entry points the command-line tools use.
There is no fallback: if libnsat.so is missing or no CUDA device is present,
the calls raise.
"""
import ctypes as C
import os
import weakref

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnsat.so")

NSAT_OK = 0
ERRORS = {-1: "EINVAL", -2: "ENOMEM", -3: "ECOMPILE", -4: "ECUDA", -5: "ETIMEOUT", -6: "ENODEV",
          -7: "EUNSUPPORTED", -8: "EPARSE", -9: "EBUSY"}

U8P = C.POINTER(C.c_uint8)
U32P = C.POINTER(C.c_uint32)
U64P = C.POINTER(C.c_uint64)


class CircuitDesc(C.Structure):
    _fields_ = [("input_len", C.c_uint32), ("gate_num", C.c_uint32), ("gates", U32P),
                ("output_num", C.c_uint32), ("outputs", U32P)]


class Opts(C.Structure):
    _fields_ = [("block_threads", C.c_uint32), ("no_optimize", C.c_uint32),
                ("verbose", C.c_uint32), ("min_blocks", C.c_uint32)]


class SatShare(C.Structure):
    """nsat_sat_share: the chunk queue of one SAT search split over several
    contexts (zero-initialised; pass the same object to every solve)."""
    _fields_ = [("next", C.c_uint64), ("stop_plus1", C.c_uint64), ("reserved", C.c_uint64 * 6)]


class SatOpts(C.Structure):
    _fields_ = [("find_all", C.c_uint32), ("chunk_bits", C.c_uint32),
                ("begin_lo", C.c_uint64), ("begin_hi", C.c_uint64),
                ("end_lo", C.c_uint64), ("end_hi", C.c_uint64), ("share", C.POINTER(SatShare))]


class SatResult(C.Structure):
    _fields_ = [("satisfiable", C.c_int32), ("launches", C.c_uint32),
                ("count_lo", C.c_uint64), ("count_hi", C.c_uint64),
                ("witness_lo", C.c_uint64), ("witness_hi", C.c_uint64),
                ("scanned_lo", C.c_uint64), ("scanned_hi", C.c_uint64),
                ("device_ms", C.c_double), ("wall_ms", C.c_double)]


class QsatOpts(C.Structure):
    _fields_ = [("chunk_bits", C.c_uint32), ("prefix_bits", C.c_uint32), ("prefix", C.c_uint64)]


class QsatResult(C.Structure):
    _fields_ = [("reversed", C.c_int32), ("solution_bits", C.c_uint32),
                ("has_solution", C.c_int32), ("value", C.c_int32),
                ("solution_lo", C.c_uint64), ("solution_hi", C.c_uint64),
                ("launches", C.c_uint32), ("chunk_bits", C.c_uint32), ("scanned", C.c_uint64),
                ("device_ms", C.c_double), ("wall_ms", C.c_double)]


class JitInfo(C.Structure):
    _fields_ = [("regs", C.c_int32), ("spill_bytes", C.c_int32), ("lop3_ops", C.c_uint32),
                ("live_gates", C.c_uint32), ("compile_ms", C.c_double)]


class TableOpts(C.Structure):
    _fields_ = [("want_steps", C.c_uint32), ("reserved", C.c_uint32)]


class StopOpts(C.Structure):
    _fields_ = [("unknowns", C.c_uint32), ("mode", C.c_uint32)]


class StopResult(C.Structure):
    _fields_ = [("found", C.c_int32), ("rounds", C.c_uint32), ("start", C.c_uint64),
                ("end", C.c_uint64), ("steps", C.c_uint64), ("build_ms", C.c_double),
                ("join_ms", C.c_double)]


class GreedyOpts(C.Structure):
    _fields_ = [("unknowns", C.c_uint32), ("partitions", C.c_uint32), ("file_prefix", C.c_char_p),
                ("device_bytes", C.c_uint64)]


class GreedyResult(C.Structure):
    _fields_ = [("found", C.c_int32), ("stage", C.c_uint32), ("partition", C.c_uint32),
                ("load_bits", C.c_uint32), ("storage", C.c_uint32), ("reserved", C.c_uint32),
                ("start", C.c_uint64), ("end", C.c_uint64),
                ("joins", C.c_uint64), ("build_ms", C.c_double), ("join_ms", C.c_double),
                ("wall_ms", C.c_double), ("h2d_bytes", C.c_uint64), ("d2h_bytes", C.c_uint64)]


class TuneOpts(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("persist", C.c_uint32), ("quants", U8P), ("sample_ms", C.c_double),
                ("threads", C.c_uint32), ("reserved", C.c_uint32)]


class TuneResult(C.Structure):
    _fields_ = [("block_threads", C.c_uint32), ("min_blocks", C.c_uint32), ("cta_bits_max", C.c_uint32),
                ("candidates", C.c_uint32), ("from_cache", C.c_uint32), ("sync_every", C.c_uint32),
                ("best_rate", C.c_double), ("default_rate", C.c_double), ("tune_ms", C.c_double)]


class ServerOpts(C.Structure):
    _fields_ = [("arena_bytes", C.c_uint64), ("max_active", C.c_uint32), ("max_queue", C.c_uint32),
                ("max_slice_tiles", C.c_uint32), ("first_slice_tiles", C.c_uint32),
                ("epoch_budget", C.c_uint64), ("build_threads", C.c_uint32), ("tier_threads", C.c_uint32),
                ("tier_min_ms", C.c_uint32), ("tier_wait", C.c_uint32), ("shape", C.c_uint32),
                ("rollover", C.c_uint32)]


class ServeTuneOpts(C.Structure):
    _fields_ = [("jobs", C.c_uint32), ("persist", C.c_uint32), ("retune", C.c_uint32), ("reserved", C.c_uint32),
                ("seed", C.c_uint64)]


class ServeTuneResult(C.Structure):
    _fields_ = [("shape", C.c_uint32), ("from_cache", C.c_uint32), ("epoch_budget", C.c_uint64),
                ("lut_words_per_s", C.c_double * 6), ("budget_solves_per_s", C.c_double * 4),
                ("budget_epoch_ms", C.c_double * 4), ("tune_ms", C.c_double)]


class JobDesc(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("unknowns", C.c_uint32), ("quants", U8P),
                ("circuit", CircuitDesc), ("tag", C.c_uint64), ("flags", C.c_uint32),
                ("reserved", C.c_uint32)]


class JobResult(C.Structure):
    _fields_ = [("id", C.c_uint64), ("tag", C.c_uint64), ("status", C.c_int32), ("kind", C.c_uint32),
                ("satisfiable", C.c_int32), ("value", C.c_int32), ("witness_lo", C.c_uint64),
                ("witness_hi", C.c_uint64), ("count", C.c_uint64), ("reversed", C.c_int32),
                ("solution_bits", C.c_uint32), ("has_solution", C.c_int32), ("found", C.c_int32),
                ("solution", C.c_uint64), ("start", C.c_uint64), ("end", C.c_uint64), ("steps", C.c_uint64),
                ("tiles", C.c_uint64), ("submit_ms", C.c_double), ("admit_ms", C.c_double),
                ("done_ms", C.c_double), ("compiled_blocks", C.c_uint32), ("epochs", C.c_uint32),
                ("first_epoch", C.c_uint64), ("last_epoch", C.c_uint64)]


class ServerStats(C.Structure):
    _fields_ = [("epochs", C.c_uint64), ("device_ms", C.c_double), ("active", C.c_uint32),
                ("queued", C.c_uint32), ("arena_used", C.c_uint64), ("arena_bytes", C.c_uint64),
                ("graph_slots", C.c_uint32), ("grid", C.c_uint32), ("launches", C.c_uint64),
                ("h2d_bytes", C.c_uint64), ("d2h_bytes", C.c_uint64), ("shape", C.c_uint32),
                ("reserved", C.c_uint32)]


EXPORTS = [
    "nsat_create", "nsat_destroy", "nsat_strerror", "nsat_last_error", "nsat_device_count",
    "nsat_circuit_new", "nsat_circuit_free", "nsat_circuit_stats", "nsat_parse",
    "nsat_parsed_get", "nsat_parsed_free", "nsat_format", "nsat_sat_solve", "nsat_qsat_solve",
    "nsat_qsat_reduce_words", "nsat_stop_table_build", "nsat_table_free", "nsat_table_read",
    "nsat_table_bytes", "nsat_stop_solve", "nsat_probe_lop3_peak", "nsat_jit_check",
    "nsat_qsat_solve_noalloc", "nsat_server_create", "nsat_server_destroy", "nsat_server_submit",
    "nsat_server_step", "nsat_server_poll", "nsat_server_stats", "nsat_gen_random_dag",
    "nsat_gen_lfsr_stop", "nsat_server_program_check", "nsat_greedy_solve", "nsat_greedy_image",
    "nsat_autotune", "nsat_autotune_reset", "nsat_probe_gather_peak", "nsat_server_tune",
]

_lib = None


def lib():
    """Loads libnsat.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libnsat.so is not built: run `make -C naivesat_b200/csrc` "
                               "(or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        L.nsat_create.argtypes = [C.c_int, C.POINTER(Opts), C.POINTER(C.c_void_p)]
        L.nsat_destroy.argtypes = [C.c_void_p]
        L.nsat_destroy.restype = None
        L.nsat_strerror.argtypes = [C.c_int]
        L.nsat_strerror.restype = C.c_char_p
        L.nsat_last_error.argtypes = [C.c_void_p]
        L.nsat_last_error.restype = C.c_char_p
        L.nsat_device_count.argtypes = []
        L.nsat_circuit_new.argtypes = [C.c_void_p, C.POINTER(CircuitDesc), C.POINTER(C.c_void_p)]
        L.nsat_circuit_free.argtypes = [C.c_void_p]
        L.nsat_circuit_free.restype = None
        L.nsat_circuit_stats.argtypes = [C.c_void_p, C.c_void_p, C.c_int, U32P, U32P]
        L.nsat_parse.argtypes = [C.c_char_p, C.c_size_t, C.POINTER(C.c_void_p)]
        L.nsat_parsed_get.argtypes = [C.c_void_p, C.POINTER(CircuitDesc), C.POINTER(U8P)]
        L.nsat_parsed_free.argtypes = [C.c_void_p]
        L.nsat_parsed_free.restype = None
        L.nsat_format.argtypes = [C.POINTER(CircuitDesc), U8P, C.c_char_p, C.c_size_t,
                                  C.POINTER(C.c_size_t)]
        L.nsat_sat_solve.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(SatOpts), C.POINTER(SatResult)]
        L.nsat_qsat_solve.argtypes = [C.c_void_p, C.c_void_p, U8P, C.POINTER(QsatOpts),
                                      C.POINTER(QsatResult)]
        L.nsat_qsat_solve_noalloc.argtypes = [C.c_void_p, C.c_void_p, U8P, C.POINTER(QsatOpts),
                                              C.POINTER(QsatResult)]
        L.nsat_qsat_reduce_words.argtypes = [C.c_void_p, U8P, C.c_uint32, U32P, C.POINTER(QsatResult)]
        L.nsat_stop_table_build.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(TableOpts),
                                            C.POINTER(C.c_void_p)]
        L.nsat_table_free.argtypes = [C.c_void_p]
        L.nsat_table_free.restype = None
        L.nsat_table_read.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, U64P]
        L.nsat_table_bytes.argtypes = [C.c_void_p]
        L.nsat_table_bytes.restype = C.c_uint64
        L.nsat_stop_solve.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(StopOpts), C.POINTER(StopResult)]
        L.nsat_probe_lop3_peak.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.nsat_probe_gather_peak.argtypes = [C.c_void_p, C.c_uint32, C.POINTER(C.c_double)]
        L.nsat_autotune.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(TuneOpts), C.POINTER(TuneResult)]
        L.nsat_autotune_reset.argtypes = [C.c_void_p]
        L.nsat_greedy_solve.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(GreedyOpts), C.POINTER(GreedyResult)]
        L.nsat_greedy_image.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_char_p, U64P, C.c_uint64]
        L.nsat_server_create.argtypes = [C.c_void_p, C.POINTER(ServerOpts), C.POINTER(C.c_void_p)]
        L.nsat_server_tune.argtypes = [C.c_void_p, C.POINTER(ServeTuneOpts), C.POINTER(ServeTuneResult)]
        L.nsat_server_destroy.argtypes = [C.c_void_p]
        L.nsat_server_destroy.restype = None
        L.nsat_server_submit.argtypes = [C.c_void_p, C.POINTER(JobDesc), C.POINTER(C.c_uint64)]
        L.nsat_server_step.argtypes = [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        L.nsat_server_poll.argtypes = [C.c_void_p, C.POINTER(JobResult), C.c_uint32, C.POINTER(C.c_uint32)]
        L.nsat_server_stats.argtypes = [C.c_void_p, C.POINTER(ServerStats)]
        L.nsat_server_program_check.argtypes = [C.POINTER(CircuitDesc), C.c_uint32, C.c_uint32, C.c_uint64, U32P,
                                                U32P, U32P]
        L.nsat_gen_random_dag.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, U32P,
                                          C.c_uint32, U32P, C.c_uint32, U32P, U32P]
        L.nsat_gen_lfsr_stop.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, U32P, C.c_uint32, U32P,
                                         C.c_uint32, U32P, U32P, U64P]
        L.nsat_jit_check.argtypes = [C.POINTER(CircuitDesc), U8P, C.c_int, C.POINTER(Opts),
                                     C.POINTER(JitInfo), C.c_char_p, C.c_size_t]
        _lib = L
    return _lib


class NsatError(RuntimeError):
    pass


def _quants_array(quants, n):
    if isinstance(quants, str):
        q = np.array([1 if ch in "Aa" else 0 for ch in quants], dtype=np.uint8)
    else:
        q = np.ascontiguousarray(np.asarray(quants, dtype=np.uint8))
    if len(q) != n:
        raise ValueError("need one quantifier per input")
    return q


def desc_of(n, gates, outputs):
    g = np.ascontiguousarray(np.asarray(gates, dtype=np.uint32).reshape(-1))
    o = np.ascontiguousarray(np.asarray(outputs, dtype=np.uint32).reshape(-1))
    d = CircuitDesc(int(n), len(g) // 3, g.ctypes.data_as(U32P), len(o) // 2, o.ctypes.data_as(U32P))
    d._keep = (g, o)
    return d


class Context:
    """One device + stream; not for concurrent use from several threads."""

    def __init__(self, device=0, block_threads=0, no_optimize=False, verbose=False, min_blocks=0):
        L = lib()
        h = C.c_void_p()
        o = Opts(block_threads, 1 if no_optimize else 0, 1 if verbose else 0, min_blocks)
        rc = L.nsat_create(device, C.byref(o), C.byref(h))
        if rc != NSAT_OK:
            raise NsatError("nsat_create(%d): %s" % (device, L.nsat_strerror(rc).decode()))
        self.h = h
        # objects whose C handles refer to this context; closed before it
        self._children = weakref.WeakSet()

    def _check(self, rc, what):
        if rc != NSAT_OK:
            msg = lib().nsat_last_error(self.h).decode(errors="replace")
            raise NsatError("%s: %s (%s) %s" % (what, ERRORS.get(rc, rc), lib().nsat_strerror(rc).decode(), msg))

    def close(self):
        if getattr(self, "h", None):
            for child in list(self._children):
                child.close()
            lib().nsat_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def circuit(self, circ):
        """Loads a workloads.Circuit (or anything with n, gates, outputs)."""
        return CircuitHandle(self, circ.n, circ.gates, circ.outputs)

    def gather_peak(self, log2_entries):
        """Random 8-byte gathers per second from a table of 2^log2_entries u64."""
        g = C.c_double()
        self._check(lib().nsat_probe_gather_peak(self.h, log2_entries, C.byref(g)), "probe_gather_peak")
        return g.value

    def lop3_peak(self):
        r, mhz = C.c_double(), C.c_double()
        self._check(lib().nsat_probe_lop3_peak(self.h, C.byref(r), C.byref(mhz)), "probe")
        return r.value, mhz.value

    def qsat_reduce_words(self, quants, words):
        q = _quants_array(quants, len(quants))
        w = np.ascontiguousarray(np.asarray(words, dtype=np.uint32))
        assert len(w) * 32 == 1 << len(q)
        r = QsatResult()
        self._check(lib().nsat_qsat_reduce_words(self.h, q.ctypes.data_as(U8P), len(q),
                                                 w.ctypes.data_as(U32P), C.byref(r)), "reduce_words")
        return _qsat_dict(r)


def _qsat_dict(r):
    return {"reversed": bool(r.reversed), "solution_bits": r.solution_bits,
            "solution": (r.solution_lo | (r.solution_hi << 64)) if r.has_solution else None,
            "value": bool(r.value), "launches": r.launches, "chunk_bits": r.chunk_bits,
            "scanned": r.scanned, "device_ms": r.device_ms, "wall_ms": r.wall_ms}


class CircuitHandle:
    def __init__(self, ctx, n, gates, outputs):
        self.ctx = ctx
        self.n = int(n)
        d = desc_of(n, gates, outputs)
        h = C.c_void_p()
        ctx._check(lib().nsat_circuit_new(ctx.h, C.byref(d), C.byref(h)), "circuit_new")
        self.h = h
        ctx._children.add(self)

    def close(self):
        if getattr(self, "h", None):
            lib().nsat_circuit_free(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def stats(self, output=0):
        live, ops = C.c_uint32(), C.c_uint32()
        self.ctx._check(lib().nsat_circuit_stats(self.ctx.h, self.h, output, C.byref(live),
                                                 C.byref(ops)), "stats")
        return live.value, ops.value

    def sat(self, find_all=True, chunk_bits=0, begin=0, end=0, share=None):
        """SAT solve over [begin, end) (end 0 = 2^n).  share: a SatShare
        given to every context that takes part in one find-mode search (each
        in its own thread); the result then covers this context's chunks."""
        o = SatOpts(1 if find_all else 0, chunk_bits, begin & 0xFFFFFFFFFFFFFFFF, begin >> 64,
                    end & 0xFFFFFFFFFFFFFFFF, end >> 64, C.pointer(share) if share is not None else None)
        r = SatResult()
        self.ctx._check(lib().nsat_sat_solve(self.ctx.h, self.h, C.byref(o), C.byref(r)), "sat_solve")
        return {"satisfiable": bool(r.satisfiable), "count": r.count_lo | (r.count_hi << 64),
                "witness": (r.witness_lo | (r.witness_hi << 64)) if r.satisfiable else None,
                "scanned": r.scanned_lo | (r.scanned_hi << 64), "launches": r.launches,
                "device_ms": r.device_ms, "wall_ms": r.wall_ms}

    def qsat(self, quants, chunk_bits=0, prefix_bits=0, prefix=0):
        """QSAT solve; with prefix_bits > 0 the outermost prefix_bits inputs
        are fixed to `prefix` (input 0 most significant) and the result is
        that of the sub-formula below them."""
        q = _quants_array(quants, self.n)
        o = QsatOpts(chunk_bits, prefix_bits, prefix)
        r = QsatResult()
        self.ctx._check(lib().nsat_qsat_solve(self.ctx.h, self.h, q.ctypes.data_as(U8P), C.byref(o),
                                              C.byref(r)), "qsat_solve")
        return _qsat_dict(r)

    def qsat_noalloc(self, quants, chunk_bits=0):
        """nsat_qsat_solve_noalloc: the same solve with no device allocation
        (scratch from the library's static device array)."""
        q = _quants_array(quants, self.n)
        o = QsatOpts(chunk_bits, 0, 0)
        r = QsatResult()
        self.ctx._check(lib().nsat_qsat_solve_noalloc(self.ctx.h, self.h, q.ctypes.data_as(U8P), C.byref(o),
                                                      C.byref(r)), "qsat_solve_noalloc")
        return _qsat_dict(r)

    def stop_table(self, want_steps=False):
        return Table(self, want_steps)

    def autotune(self, kind="sat", quants=None, persist=False, sample_ms=0.0, threads=0):
        """nsat_autotune: times candidate launch shapes on a sample of this
        circuit's index space and keeps the fastest for later solves."""
        q = _quants_array(quants, self.n) if quants is not None else None
        o = TuneOpts(0 if kind == "sat" else 1, 1 if persist else 0,
                     q.ctypes.data_as(U8P) if q is not None else None, sample_ms, threads, 0)
        r = TuneResult()
        self.ctx._check(lib().nsat_autotune(self.ctx.h, self.h, C.byref(o), C.byref(r)), "autotune")
        return {f: getattr(r, f) for f, _ in TuneResult._fields_}

    def autotune_reset(self):
        lib().nsat_autotune_reset(self.h)

    def greedy_partitioned(self, unknowns, partitions, file_prefix=None, device_bytes=0):
        """greedysatostop -p: the table as a packed image (device memory when
        it fits in device_bytes, 0 = free memory; else pinned host memory; or
        a temp file under file_prefix), joined partition by partition in the
        reference's order.  result["storage"]: 0 device, 1 host, 2 file."""
        o = GreedyOpts(unknowns, partitions, file_prefix.encode() if file_prefix is not None else None,
                       device_bytes)
        r = GreedyResult()
        self.ctx._check(lib().nsat_greedy_solve(self.ctx.h, self.h, C.byref(o), C.byref(r)), "greedy_solve")
        d = {f: getattr(r, f) for f, _ in GreedyResult._fields_}
        d["found"] = bool(r.found)
        if not r.found:
            d["start"] = d["end"] = None
        return d

    def greedy_image(self, partitions, file_prefix=None):
        """The packed (n+1)-bit table image after the first pass."""
        words = ((1 << self.n) * (self.n + 1) + 63) // 64
        out = np.zeros(words, dtype=np.uint64)
        self.ctx._check(lib().nsat_greedy_image(self.ctx.h, self.h, partitions,
                                                file_prefix.encode() if file_prefix is not None else None,
                                                out.ctypes.data_as(U64P), words), "greedy_image")
        return out


KINDS = {"sat": 0, "qsat": 1, "stop": 2}
SERVE_SHAPES = 6     # NSAT_SERVE_SHAPES


def server_tune(ctx, jobs=0, persist=False, retune=False, seed=0):
    """nsat_server_tune: times every interpreter shape and four epoch
    budgets on a seeded calibration set; returns the choice and the rates."""
    o = ServeTuneOpts(jobs, 1 if persist else 0, 1 if retune else 0, 0, seed)
    r = ServeTuneResult()
    ctx._check(lib().nsat_server_tune(ctx.h, C.byref(o), C.byref(r)), "server_tune")
    return {"shape": r.shape, "from_cache": bool(r.from_cache), "epoch_budget": r.epoch_budget,
            "lut_words_per_s": list(r.lut_words_per_s), "budget_solves_per_s": list(r.budget_solves_per_s),
            "budget_epoch_ms": list(r.budget_epoch_ms), "tune_ms": r.tune_ms}


class Server:
    """Batched serving of many SAT / QSAT / SATOSTOP jobs on one context."""

    def __init__(self, ctx, arena_bytes=0, max_active=0, max_queue=0, max_slice_tiles=0,
                 first_slice_tiles=0, epoch_budget=0, build_threads=0, tier_threads=0, tier_min_ms=0,
                 tier_wait=False, shape=0, rollover=False):
        """shape: interpreter shape 1..SERVE_SHAPES (include/nsat.h), 0 = the
        one tuned for this GPU (nsat_server_tune) or the default."""
        self.ctx = ctx
        o = ServerOpts(arena_bytes, max_active, max_queue, max_slice_tiles, first_slice_tiles, epoch_budget,
                       build_threads, tier_threads, tier_min_ms, 1 if tier_wait else 0, shape,
                       1 if rollover else 0)
        h = C.c_void_p()
        ctx._check(lib().nsat_server_create(ctx.h, C.byref(o), C.byref(h)), "server_create")
        self.h = h
        self._buf = (JobResult * 256)()
        ctx._children.add(self)

    def close(self):
        if getattr(self, "h", None):
            lib().nsat_server_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def submit(self, kind, circ, quants=None, unknowns=0, tag=0, find_all=False):
        """kind: 'sat' | 'qsat' | 'stop'.  Returns the job id (raises NsatError
        with EBUSY when the queue is full).  find_all: a SAT job enumerates
        every assignment and reports the exact count (otherwise it ends at
        the lowest witness and the count covers the tiles evaluated)."""
        d = desc_of(circ.n, circ.gates, circ.outputs)
        q = _quants_array(quants, circ.n) if quants is not None else None
        jd = JobDesc(KINDS[kind], unknowns, q.ctypes.data_as(U8P) if q is not None else None, d, tag,
                     1 if find_all else 0, 0)
        jid = C.c_uint64()
        self.ctx._check(lib().nsat_server_submit(self.h, C.byref(jd), C.byref(jid)), "server_submit")
        return jid.value

    def step(self):
        a, q = C.c_uint32(), C.c_uint32()
        self.ctx._check(lib().nsat_server_step(self.h, C.byref(a), C.byref(q)), "server_step")
        return a.value, q.value

    def poll(self):
        out = []
        while True:
            n = C.c_uint32()
            self.ctx._check(lib().nsat_server_poll(self.h, self._buf, len(self._buf), C.byref(n)), "server_poll")
            for i in range(n.value):
                r = self._buf[i]
                d = {"id": r.id, "tag": r.tag, "status": r.status, "kind": ["sat", "qsat", "stop"][r.kind],
                     "tiles": r.tiles, "compiled_blocks": r.compiled_blocks, "epochs": r.epochs,
                     "first_epoch": r.first_epoch, "last_epoch": r.last_epoch,
                     "submit_ms": r.submit_ms, "admit_ms": r.admit_ms, "done_ms": r.done_ms}
                if r.kind == 0:
                    d.update(satisfiable=bool(r.satisfiable), count=r.count,
                             witness=(r.witness_lo | (r.witness_hi << 64)) if r.satisfiable else None)
                elif r.kind == 1:
                    d.update(reversed=bool(r.reversed), solution_bits=r.solution_bits, value=bool(r.value),
                             solution=r.solution if r.has_solution else None)
                else:
                    d.update(found=bool(r.found), start=r.start if r.found else None,
                             end=r.end if r.found else None, steps=r.steps if r.found else None)
                out.append(d)
            if n.value < len(self._buf):
                return out

    def stats(self):
        st = ServerStats()
        self.ctx._check(lib().nsat_server_stats(self.h, C.byref(st)), "server_stats")
        return {f: getattr(st, f) for f, _ in ServerStats._fields_}

    def run_all(self, max_steps=10_000_000):
        """Steps until every submitted job finished; returns the results."""
        res = []
        for _ in range(max_steps):
            a, q = self.step()
            res += self.poll()
            if a == 0 and q == 0:
                return res
        raise NsatError("server did not drain in %d steps" % max_steps)


class Table:
    def __init__(self, circ, want_steps=False):
        self.ctx = circ.ctx
        self.n = circ.n
        h = C.c_void_p()
        o = TableOpts(1 if want_steps else 0, 0)
        self.ctx._check(lib().nsat_stop_table_build(self.ctx.h, circ.h, C.byref(o), C.byref(h)),
                        "stop_table_build")
        self.h = h
        self.ctx._children.add(self)

    def close(self):
        if getattr(self, "h", None):
            lib().nsat_table_free(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def read(self, first=0, count=None):
        if count is None:
            count = (1 << self.n) - first
        out = np.zeros(count, dtype=np.uint64)
        self.ctx._check(lib().nsat_table_read(self.h, first, count, out.ctypes.data_as(U64P)), "table_read")
        return out

    def nbytes(self):
        return lib().nsat_table_bytes(self.h)

    def solve(self, unknowns, mode=0):
        o = StopOpts(unknowns, mode)
        r = StopResult()
        self.ctx._check(lib().nsat_stop_solve(self.ctx.h, self.h, C.byref(o), C.byref(r)), "stop_solve")
        if not r.found:
            return {"found": False, "rounds": r.rounds, "build_ms": r.build_ms, "join_ms": r.join_ms}
        return {"found": True, "start": r.start, "end": r.end, "steps": r.steps, "rounds": r.rounds,
                "build_ms": r.build_ms, "join_ms": r.join_ms}


def parse(text):
    """gatesim text -> (n, gates (g,3), outputs (o,2), quants string or None)."""
    L = lib()
    b = text.encode()
    h = C.c_void_p()
    rc = L.nsat_parse(b, len(b), C.byref(h))
    if rc != NSAT_OK:
        raise NsatError("parse: %s" % ERRORS.get(rc, rc))
    try:
        d = CircuitDesc()
        q = U8P()
        L.nsat_parsed_get(h, C.byref(d), C.byref(q))
        gates = np.ctypeslib.as_array(d.gates, (d.gate_num * 3,)).reshape(-1, 3).copy() if d.gate_num else \
            np.zeros((0, 3), dtype=np.uint32)
        outs = np.ctypeslib.as_array(d.outputs, (d.output_num * 2,)).reshape(-1, 2).copy()
        quants = None
        if q:
            quants = "".join("A" if q[i] else "E" for i in range(d.input_len))
        return d.input_len, gates, outs, quants
    finally:
        L.nsat_parsed_free(h)


def format_circuit(n, gates, outputs, quants=None):
    L = lib()
    d = desc_of(n, gates, outputs)
    qa = _quants_array(quants, n) if quants is not None else None
    need = C.c_size_t()
    qp = qa.ctypes.data_as(U8P) if qa is not None else None
    rc = L.nsat_format(C.byref(d), qp, None, 0, C.byref(need))
    if rc != NSAT_OK:
        raise NsatError("format: %s" % ERRORS.get(rc, rc))
    buf = C.create_string_buffer(need.value + 1)
    rc = L.nsat_format(C.byref(d), qp, buf, need.value + 1, C.byref(need))
    if rc != NSAT_OK:
        raise NsatError("format: %s" % ERRORS.get(rc, rc))
    return buf.value.decode()


KIND = {"sat": 0, "qsat": 1, "table": 2}


def server_program_check(circ, kind="sat", seed=1, shape=0):
    """Host-only check of a job's interpreter program (include/nsat.h
    nsat_server_program_check) for a server of `shape` (0 = the default);
    returns (slots, luts, nops), raises on a mismatch."""
    d = desc_of(circ.n, circ.gates, circ.outputs)
    sl, lu, no = C.c_uint32(), C.c_uint32(), C.c_uint32()
    rc = lib().nsat_server_program_check(C.byref(d), KINDS[kind], shape, seed, C.byref(sl), C.byref(lu),
                                         C.byref(no))
    if rc != 0:
        raise NsatError("server_program_check: %s" % lib().nsat_strerror(rc).decode(), rc)
    return sl.value, lu.value, no.value


def jit_check(circ, kind="sat", quants=None, block_threads=0, no_optimize=False):
    """NVRTC-compiles (no device needed) the kernel a solve would use; returns
    ptxas resource usage and LUT statistics."""
    L = lib()
    d = desc_of(circ.n, circ.gates, circ.outputs)
    q = _quants_array(quants, circ.n) if quants is not None else None
    o = Opts(block_threads, 1 if no_optimize else 0, 0, 0)
    info = JitInfo()
    buf = C.create_string_buffer(1 << 16)
    rc = L.nsat_jit_check(C.byref(d), q.ctypes.data_as(U8P) if q is not None else None, KIND[kind],
                          C.byref(o), C.byref(info), buf, len(buf))
    if rc != NSAT_OK:
        raise NsatError("jit_check: %s\n%s" % (ERRORS.get(rc, rc), buf.value.decode(errors="replace")))
    return {"regs": info.regs, "spill_bytes": info.spill_bytes, "lop3_ops": info.lop3_ops,
            "live_gates": info.live_gates, "compile_ms": info.compile_ms,
            "log": buf.value.decode(errors="replace")}


def gen_random_dag(seed, n, gates, window=64, live_output=False):
    """nsat_gen_random_dag -> (gates (g,3), outputs (1,2))."""
    g = np.zeros(3 * gates, dtype=np.uint32)
    o = np.zeros(2, dtype=np.uint32)
    gn, on = C.c_uint32(), C.c_uint32()
    rc = lib().nsat_gen_random_dag(seed, n, gates, window, 1 if live_output else 0, g.ctypes.data_as(U32P),
                                   gates, o.ctypes.data_as(U32P), 1, C.byref(gn), C.byref(on))
    if rc != NSAT_OK:
        raise NsatError("gen_random_dag: %s" % ERRORS.get(rc, rc))
    return g.reshape(-1, 3), o.reshape(-1, 2)


def gen_lfsr_stop(seed, n, mixer_gates):
    """nsat_gen_lfsr_stop -> (gates, outputs, pattern)."""
    cap = mixer_gates + 2 * n + 8
    g = np.zeros(3 * cap, dtype=np.uint32)
    o = np.zeros(2 * (n + 1), dtype=np.uint32)
    gn, on, pat = C.c_uint32(), C.c_uint32(), C.c_uint64()
    rc = lib().nsat_gen_lfsr_stop(seed, n, mixer_gates, g.ctypes.data_as(U32P), cap, o.ctypes.data_as(U32P),
                                  n + 1, C.byref(gn), C.byref(on), C.byref(pat))
    if rc != NSAT_OK:
        raise NsatError("gen_lfsr_stop: %s" % ERRORS.get(rc, rc))
    return g[:3 * gn.value].reshape(-1, 3), o.reshape(-1, 2), pat.value


def device_count():
    return lib().nsat_device_count()
