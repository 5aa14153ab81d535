"""A request loop over a resident database (the C++ server of the library).

The server (``cbp_server_*`` in ``include/cother_b200.h``, host C++ in
``csrc/server.cpp``) keeps one database chunk resident on a GPU and searches
queries as they arrive: `slots` search contexts share the chunk, each with
its own stream, working memory and worker thread, so that the batches in
flight overlap on the device. When a slot is free, the oldest waiting query
and the ones behind it (up to `max_batch`) are searched together in one pass
over the database -- their rows stacked into one score matrix per slab.
Batches are admitted in arrival order by their memory footprint: a batch is
charged what one slab of its stacked rows takes (``cother_b200.slab_bytes``),
the slab cut so that one batch takes at most `max_share` of the budget, and a
slot is charged the largest footprint it has held (its buffers only grow);
a batch starts only while the sum over the slots stays within the budget.

This module binds that server with ctypes: :class:`SearchServer` returns a
Future per query, resolved with its hits, records and times.

The reference has no request loop (it is a batch program); this is the
serving form of the same search path.
"""
from __future__ import annotations

import ctypes
from concurrent.futures import Future, ThreadPoolExecutor

import numpy as np


def slab_cost(query_len: int, options=None):
    """(bytes per slab position, bytes per slab) charged for `query_len`
    stacked query rows."""
    import cother_b200 as cb
    fixed = cb.slab_bytes(query_len, 0, options)
    return cb.slab_bytes(query_len, 1, options) - fixed, fixed


def footprint(query_len: int, slab_positions: int, options=None) -> int:
    per_pos, fixed = slab_cost(query_len, options)
    return fixed + per_pos * int(slab_positions)


def ledger_choose(held, busy, budget: int, need: int, min_grant: int = 1):
    """The server's admission rule (cbp_ledger_choose): (slot, granted
    bytes) for a batch of footprint `need` given each slot's charge `held`
    and `busy` flags, or (None, 0) to wait."""
    import cother_b200 as cb
    L = cb.load_library()
    n = len(held)
    h = (ctypes.c_size_t * n)(*[int(x) for x in held])
    b = (ctypes.c_char * n)(*[bytes([1 if x else 0]) for x in busy])
    g = ctypes.c_size_t()
    i = L.cbp_ledger_choose(h, b, n, int(budget), int(need), int(min_grant), ctypes.byref(g))
    return (None, 0) if i < 0 else (i, g.value)


class ServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("slots", ctypes.c_int), ("max_batch", ctypes.c_int),
                ("budget_bytes", ctypes.c_size_t), ("max_share", ctypes.c_double),
                ("db_len", ctypes.c_uint64), ("n_seqs", ctypes.c_size_t)]


class ServerResult(ctypes.Structure):
    _fields_ = [("arrival_s", ctypes.c_double), ("start_s", ctypes.c_double), ("finish_s", ctypes.c_double),
                ("slot", ctypes.c_int), ("batch", ctypes.c_int), ("slab_positions", ctypes.c_size_t),
                ("nrecords", ctypes.c_size_t), ("nhits", ctypes.c_size_t),
                ("alignment_length", ctypes.c_size_t)]


class ServerError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class SearchServer:
    """Serve search requests against one resident database.

    submit(query) returns a Future resolved with a dict: the hit list
    (``cother_b200.sharding.Hit``, in the finalizer's order), the records,
    the request's arrival, start and finish times (seconds of a steady
    clock), its slot, the size of its batch and the slab it ran with."""

    def __init__(self, db, ss_table, options=None, slots: int = 3, max_batch: int = 4,
                 budget: int | None = None, max_share: float = 0.5, device: int = 0,
                 db_len: int | None = None, n_seqs: int | None = None):
        import cother_b200 as cb
        L = cb.load_library()
        self._L = L
        self.db = db
        self.options = options or cb.Options.defaults()
        cfg = ServerConfig()
        L.cbp_server_default_config(ctypes.byref(cfg))
        cfg.device = int(device)
        cfg.slots = int(slots)
        cfg.max_batch = int(max_batch)
        cfg.budget_bytes = int(budget or 0)
        cfg.max_share = float(max_share)
        cfg.db_len = int(db_len or 0)
        cfg.n_seqs = int(n_seqs or 0)
        self._ss = np.ascontiguousarray(ss_table, np.float32)
        beg, end = db.field_tables()
        h = ctypes.c_void_p()
        self._check(L.cbp_server_create(ctypes.byref(cfg), ctypes.byref(self.options), self._ss.ctypes.data,
                                        beg, end, ctypes.byref(h)))
        self._h = h
        b = ctypes.c_size_t()
        self._check(L.cbp_server_budget(self._h, ctypes.byref(b)))
        self.budget = b.value
        self._pool = ThreadPoolExecutor(max_workers=256)

    def _check(self, rc: int) -> None:
        if rc != 0:
            msg = self._L.cbp_server_last_error()
            raise ServerError(rc, msg.decode() if msg else "")

    # -- public -------------------------------------------------------------
    def submit(self, query) -> Future:
        beg, end = query.field_tables()
        t = ctypes.c_uint64()
        self._check(self._L.cbp_server_submit(self._h, int(query.npositions), beg, end, ctypes.byref(t)))
        return self._pool.submit(self._collect, t.value, int(query.npositions))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._L.cbp_server_destroy(self._h)     # finishes the queued requests
            self._h = None
            self._pool.shutdown(wait=True)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- internals ------------------------------------------------------------
    def _collect(self, ticket: int, query_len: int) -> dict:
        import cother_b200 as cb
        from .sharding import Hit
        L = self._L
        info = ServerResult()
        self._check(L.cbp_server_wait(self._h, ticket, -1, ctypes.byref(info)))
        recs = np.zeros((info.nrecords, cb.REC_FLOATS), np.float32)
        order = np.zeros(info.nhits, np.int32)
        n = int(info.alignment_length)
        rows = np.zeros((5, max(n, 1)), np.uint8)
        self._check(L.cbp_server_get(self._h, ticket, recs.ctypes.data, info.nrecords, order.ctypes.data,
                                     info.nhits, rows.ctypes.data, rows.shape[1]))
        L.cbp_server_release(self._h, ticket)
        alns = cb.alignments_from(recs, rows[:, :n], query_len, self.db.lens)
        tab = cb.records_table(recs)
        hits = [Hit(profile=int(tab["org_pro_no"][i]), log_evalue=float(recs[i, 8]), record=recs[i].copy(),
                    alignment=alns[i]) for i in order]
        return {"hits": hits, "records": recs, "arrival": info.arrival_s, "start": info.start_s,
                "finish": info.finish_s, "slot": info.slot, "batch": info.batch, "slab": info.slab_positions}


def latency_summary(results) -> dict:
    """queries/s and latency percentiles (ms) of completed requests."""
    lat = np.array([(x["finish"] - x["arrival"]) * 1e3 for x in results])
    svc = np.array([(x["finish"] - x["start"]) * 1e3 for x in results])
    t0 = min(x["arrival"] for x in results)
    t1 = max(x["finish"] for x in results)
    return {"queries": len(results), "queries_per_s": len(results) / (t1 - t0),
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "service_p50_ms": float(np.percentile(svc, 50)),
            "mean_batch": float(np.mean([x.get("batch", 1) for x in results]))}
