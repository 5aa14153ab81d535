"""A request loop over a resident database.

Several search contexts (slots) share one device copy of the database
(``BatchProcessing.share_database``); each has its own CUDA stream, working
memory and host thread, so the searches of the requests in flight overlap on
the device. Requests are admitted in arrival order as a slot and enough
working memory free up: a request's footprint is what its score matrices,
DP buffers and alignment rows take for one slab of the database (the slab
planner's charge, ``cother_b200.slab_bytes``), with the slab cut so that a
request never needs more than ``max_share`` of the budget. A slot keeps its buffers between requests (they
only grow), so the ledger charges each slot the largest footprint it has
held, and admits a request only if the sum over slots stays within the
budget.

The reference has no request loop (it is a batch program); this is the
serving form of the same search path.
"""
from __future__ import annotations

import collections
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np

def slab_cost(query_len: int, options=None):
    """(bytes per slab position, bytes per slab) charged for a query."""
    import cother_b200 as cb
    fixed = cb.slab_bytes(query_len, 0, options)
    return cb.slab_bytes(query_len, 1, options) - fixed, fixed


def footprint(query_len: int, slab_positions: int, options=None) -> int:
    per_pos, fixed = slab_cost(query_len, options)
    return fixed + per_pos * int(slab_positions)


def slab_positions_for(query_len: int, db_positions: int, budget: int, max_share: float,
                       options=None) -> int:
    """Largest slab (positions) whose footprint fits max_share of the budget."""
    per_pos, fixed = slab_cost(query_len, options)
    cap = max(0, int(budget * max_share) - fixed) // per_pos
    return max(1, min(int(db_positions), cap))


@dataclass
class Request:
    query: object
    arrival: float
    future: Future = field(default_factory=Future)
    slab: int = 0
    need: int = 0


class Ledger:
    """Admission by memory footprint (pure host logic).

    A slot's buffers only grow, so each slot is charged the largest
    footprint it has held. A request gets its full footprint on a free slot
    when the charge stays within the budget; if it does not fit now but
    would fit on a busy slot once that finishes, it waits; otherwise (no
    slot will ever have room for all of it) it gets what the roomiest free
    slot can hold, at least `min_grant`, and runs with a smaller slab."""

    def __init__(self, nslots: int, budget: int):
        self.held = [0] * nslots
        self.busy = [False] * nslots
        self.budget = int(budget)

    def choose(self, need: int, min_grant: int = 1):
        """(slot, granted bytes) for a request of footprint `need`, or
        (None, 0) to wait."""
        total = sum(self.held)
        best, best_growth = None, None
        for i, b in enumerate(self.busy):
            if b:
                continue
            growth = max(0, need - self.held[i])
            if total + growth <= self.budget and (best is None or growth < best_growth):
                best, best_growth = i, growth
        if best is not None:
            return best, need
        if any(b and total + max(0, need - self.held[i]) <= self.budget
               for i, b in enumerate(self.busy)):
            return None, 0
        room = [(self.budget - (total - self.held[i]), i) for i, b in enumerate(self.busy) if not b]
        if not room:
            return None, 0
        avail, i = max(room)
        return (i, avail) if avail >= min_grant else (None, 0)

    def take(self, i: int, grant: int) -> None:
        self.busy[i] = True
        self.held[i] = max(self.held[i], grant)
        assert sum(self.held) <= self.budget

    def give_back(self, i: int) -> None:
        self.busy[i] = False


class SearchServer:
    """Serve search requests against one resident database.

    `run_search(slot, request)` does the search of one request on one slot;
    the default runs the CUDA path through the slot's BatchProcessing
    context. Results are delivered through the Future returned by submit():
    a dict with the hit list (``cother_b200.sharding.Hit``), the records,
    and the request's arrival, start and finish times."""

    def __init__(self, db, ss_table, options=None, slots: int = 3, budget: int | None = None,
                 max_share: float = 0.5, device: int = 0, db_len: int | None = None,
                 n_seqs: int | None = None, run_search=None):
        self.db = db
        self.options = options
        self._longest = int(np.max(db.lens))   # a slab holds whole profiles
        self.nslots = int(slots)
        self.max_share = float(max_share)
        self._cv = threading.Condition()
        self._queue = collections.deque()
        self._stop = False
        self._done = False
        self._contexts = []
        self._run = run_search or self._run_cuda
        if run_search is None:
            import cother_b200 as cb
            owner = cb.BatchProcessing(ss_table, options, device=device, dev_mem_bytes=1 << 20)
            owner.transfer_cpm_data(db)
            if budget is None:
                # what is free once the database is resident
                budget = int(cb.device_memory(device)[0] * 0.7)
            for _ in range(self.nslots):
                bp = cb.BatchProcessing(ss_table, options, device=device, dev_mem_bytes=budget)
                bp.share_database(owner)
                bp.set_db_details(db_len or db.npositions, n_seqs or db.nprofiles)
                self._contexts.append(bp)
            self._owner = owner
        self.ledger = Ledger(self.nslots, budget if budget is not None else 1 << 62)
        self._threads = [threading.Thread(target=self._worker, args=(i,), daemon=True)
                         for i in range(self.nslots)]
        self._dispatcher = threading.Thread(target=self._dispatch, daemon=True)
        self._assigned = [None] * self.nslots
        for t in self._threads:
            t.start()
        self._dispatcher.start()

    # -- public -------------------------------------------------------------
    def submit(self, query) -> Future:
        r = Request(query=query, arrival=time.perf_counter())
        r.slab = slab_positions_for(query.npositions, self.db.npositions, self.ledger.budget,
                                    self.max_share, self.options)
        if r.slab < min(self._longest, self.db.npositions):
            raise ValueError("the memory budget cannot hold one slab of the longest profile "
                             "for this query length")
        r.need = footprint(query.npositions, r.slab, self.options)
        with self._cv:
            self._queue.append(r)
            self._cv.notify_all()
        return r.future

    def close(self) -> None:
        with self._cv:
            self._stop = True
            self._cv.notify_all()
        self._dispatcher.join()
        for t in self._threads:
            t.join()
        for bp in self._contexts:
            bp.close()
        if self._contexts:
            self._owner.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- internals ------------------------------------------------------------
    def _dispatch(self) -> None:
        with self._cv:
            while True:
                while not self._stop and not self._queue:
                    self._cv.wait()
                if not self._queue:            # stopped and drained
                    self._done = True
                    self._cv.notify_all()
                    return
                head = self._queue[0]          # first come, first served
                per_pos, fixed = slab_cost(head.query.npositions, self.options)
                i, grant = self.ledger.choose(head.need, fixed + per_pos * self._longest)
                if i is None:
                    self._cv.wait()
                    continue
                self._queue.popleft()
                if grant < head.need:
                    head.slab = (grant - fixed) // per_pos
                    head.need = footprint(head.query.npositions, head.slab, self.options)
                self.ledger.take(i, head.need)
                self._assigned[i] = head
                self._cv.notify_all()

    def _worker(self, i: int) -> None:
        while True:
            with self._cv:
                while self._assigned[i] is None and not self._done:
                    self._cv.wait()
                r = self._assigned[i]
                if r is None:
                    return
            start = time.perf_counter()
            try:
                result = self._run(i, r)
                result.update(arrival=r.arrival, start=start, finish=time.perf_counter(), slot=i)
                r.future.set_result(result)
            except Exception as e:  # noqa: BLE001 - handed to the caller
                r.future.set_exception(e)
            with self._cv:
                self._assigned[i] = None
                self.ledger.give_back(i)
                self._cv.notify_all()

    def _run_cuda(self, i: int, r: Request) -> dict:
        from cother_b200.sharding import local_hits
        bp = self._contexts[i]
        bp.set_max_slab_positions(r.slab)
        bp.process_score_matrix(r.query)
        return {"hits": local_hits(bp, 0, r.query.npositions), "records": bp.hit_records()}


def latency_summary(results) -> dict:
    """queries/s and latency percentiles (ms) of completed requests."""
    lat = np.array([(x["finish"] - x["arrival"]) * 1e3 for x in results])
    svc = np.array([(x["finish"] - x["start"]) * 1e3 for x in results])
    t0 = min(x["arrival"] for x in results)
    t1 = max(x["finish"] for x in results)
    return {"queries": len(results), "queries_per_s": len(results) / (t1 - t0),
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "service_p50_ms": float(np.percentile(svc, 50))}
