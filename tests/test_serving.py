"""The request loop's host logic on CPU: the server's admission rule
(cbp_ledger_choose: a batch fits, waits, or gets less than its footprint and
runs with a smaller slab; the budget is never exceeded), the footprint
charge and the latency summary. tests/test_serving_gpu.py runs the server
itself on the GPU."""
import numpy as np

from cother_b200.serving import footprint, latency_summary, ledger_choose


def test_ledger_fits_waits_and_grants_less():
    held, busy, budget = [0, 0, 0], [False, False, False], 100
    assert ledger_choose(held, busy, budget, 40) == (0, 40)
    held[0], busy[0] = 40, True
    i, g = ledger_choose(held, busy, budget, 50)
    assert g == 50 and i in (1, 2)
    held[i], busy[i] = 50, True
    # 40 + 50 held; 30 more does not fit on the last free slot, but fits on
    # slot 0 once it is free: wait
    assert ledger_choose(held, busy, budget, 30) == (None, 0)
    busy[0] = False
    assert ledger_choose(held, busy, budget, 30) == (0, 30)
    # every slot idle, held (40, 50, 0), no room for 80 anywhere: the
    # roomiest free slot (the one holding 50: 100 - 40 available) gets 60
    busy[i] = False
    assert ledger_choose(held, busy, budget, 80, min_grant=10) == (i, 60)
    assert ledger_choose(held, busy, budget, 80, min_grant=70) == (None, 0)


def test_ledger_never_exceeds_the_budget():
    rng = np.random.default_rng(3)
    budget = 1000
    held, busy = [0] * 4, [False] * 4
    for _ in range(400):
        need = int(rng.integers(1, 600))
        i, g = ledger_choose(held, busy, budget, need, min_grant=need // 2)
        if i is not None:
            assert not busy[i] and g >= need // 2
            held[i] = max(held[i], g)
            busy[i] = True
            assert sum(held) <= budget
        # finish a random busy slot
        b = [k for k in range(4) if busy[k]]
        if b and rng.random() < 0.6:
            busy[int(rng.choice(b))] = False


def test_footprint_grows_with_rows_and_slab():
    assert footprint(200, 10_000) < footprint(400, 10_000) < footprint(400, 20_000)


def test_latency_summary():
    res = [{"arrival": 0.0, "start": 0.1 * k, "finish": 0.1 * k + 0.5, "batch": 1 + k % 2} for k in range(10)]
    s = latency_summary(res)
    assert s["queries"] == 10 and s["p99_ms"] >= s["p50_ms"] > 0 and 1.0 <= s["mean_batch"] <= 2.0
