"""The request loop's host logic on CPU: admission by memory footprint, first
come first served, overlapping requests, and the budget never exceeded. The
searches are stand-ins that sleep; tests/test_serving_gpu.py runs the CUDA
path."""
import threading
import time
from types import SimpleNamespace

import numpy as np

from cother_b200.serving import Ledger, SearchServer, footprint, latency_summary


def test_ledger_fits_waits_and_grants_less():
    L = Ledger(3, 100)
    assert L.choose(40) == (0, 40)
    L.take(0, 40)
    i, g = L.choose(50)
    assert g == 50 and i in (1, 2)
    L.take(i, 50)
    # 40 + 50 held; 30 more does not fit on the last free slot, but fits on
    # slot 0 once it is free: wait
    assert L.choose(30) == (None, 0)
    L.give_back(0)
    assert L.choose(30) == (0, 30)
    # every slot idle, held (40, 50, 0), no room for 80 anywhere: the
    # roomiest free slot (the one holding 50: 100 - 40 available) gets 60
    L.give_back(i)
    assert L.choose(80, min_grant=10) == (i, 60)
    assert L.choose(80, min_grant=70) == (None, 0)
    L.take(i, 60)
    assert sum(L.held) <= L.budget


def test_server_admits_in_order_overlaps_and_stays_in_budget():
    rng = np.random.default_rng(0)
    db = SimpleNamespace(npositions=10_000, lens=np.array([300] * 33 + [100]))
    budget = footprint(200, 10_000) * 2            # two mid-size requests at a time
    running, peak, order = [0], [0], []
    lock = threading.Lock()
    ledger_ok = [True]

    def fake(slot, r):
        with lock:
            running[0] += 1
            peak[0] = max(peak[0], running[0])
            order.append(r.arrival)
            if sum(server.ledger.held) > server.ledger.budget:
                ledger_ok[0] = False
        time.sleep(0.002 * r.query.npositions / 10)
        with lock:
            running[0] -= 1
        return {"hits": [], "records": np.zeros((0, 18), np.float32), "slab": r.slab}

    server = SearchServer(db, None, slots=3, budget=budget, max_share=0.5, run_search=fake)
    lens = rng.integers(40, 1200, 20)
    futs = []
    for L in lens:
        futs.append(server.submit(SimpleNamespace(npositions=int(L))))
        time.sleep(0.001)
    res = [f.result(timeout=60) for f in futs]
    server.close()
    assert len(res) == 20 and ledger_ok[0]
    assert order == sorted(order)                   # started in arrival order
    assert peak[0] >= 2                             # requests overlapped
    for L, r in zip(lens, res):                     # every slab holds whole profiles
        assert r["slab"] >= 300 and footprint(int(L), r["slab"]) <= budget
    s = latency_summary(res)
    assert s["queries"] == 20 and s["p99_ms"] >= s["p50_ms"] > 0
