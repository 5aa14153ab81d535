"""The allocation-free phase-1 DP entry point (cbp_dp1_noalloc).

Callers that cannot allocate device memory while they search -- their
device memory is owned by their own pool, or a cudaMalloc would stall work
they have enqueued -- pass their own device buffers and get the phase-1 DP
with the band scratch taken from a fixed array inside the library. This test
calls it through the C ABI twice in a row (the scratch keeps the previous
call's contents) and checks both results against the regular entry point
(cbp_process): backtrack codes, maxima and their cells bit for bit.

This file sorts last so that a run stopping at the first failure has run
every other test before it.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _regular_path(q, db, ss, thld):
    import cother_b200 as cb
    o = cb.Options.defaults()
    o.all_codes = 1     # backtrack codes of every profile, whatever passes
    bp = cb.BatchProcessing(ss, o)
    bp.set_score_threshold(thld)
    bp.transfer_cpm_data(db)
    bp.process_score_matrix(q)
    sc, _, first = bp.read_score_matrix(q.npositions, db.npositions)
    assert first == 0
    btck = bp.read_btck(q.npositions, sc.shape[1])
    rec, _ = bp.read_phase1()
    bp.close()
    return sc, btck, rec


def test_dp1_noalloc_matches_regular_entry_point(ss_table):
    import torch
    import cother_b200 as cb
    from cother_b200 import synth

    q = synth.make_profiles([120], 301, True)
    db = synth.make_profiles([40, 3, 150, 96, 1, 64, 250, 33], 302, False)
    # none passes: the records carry the raw maxima
    sc, btck_ref, rec_hi = _regular_path(q, db, ss_table, 3.0e38)
    # all pass: the records carry the maxima's cells as end coordinates
    _, _, rec_lo = _regular_path(q, db, ss_table, -1.0)

    dev = torch.device("cuda:0")
    Lq, ld = sc.shape
    t_sc = torch.from_numpy(np.ascontiguousarray(sc)).to(dev)
    t_qtrn = torch.from_numpy(np.ascontiguousarray(q.trn)).to(dev)
    t_dtrn = torch.from_numpy(np.ascontiguousarray(db.trn)).to(dev)
    t_len = torch.from_numpy(np.ascontiguousarray(db.lens, np.int32)).to(dev)
    t_start = torch.from_numpy(np.ascontiguousarray(db.starts, np.int64)).to(dev)
    P = db.nprofiles
    L = cb.load_library()
    stream = torch.cuda.current_stream(dev)
    for call in range(2):
        t_bt = torch.full((Lq, ld), 255, dtype=torch.uint8, device=dev)
        t_max = torch.full((P,), -1.0, dtype=torch.float32, device=dev)
        t_xy = torch.zeros((P,), dtype=torch.int32, device=dev)
        rc = L.cbp_dp1_noalloc(t_sc.data_ptr(), ld, Lq, t_qtrn.data_ptr(), db.npositions, P,
                               t_dtrn.data_ptr(), t_len.data_ptr(), t_start.data_ptr(), 0, P, 0,
                               t_bt.data_ptr(), t_max.data_ptr(), t_xy.data_ptr(),
                               ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, L.cbp_last_error()
        torch.cuda.synchronize(dev)
        assert np.array_equal(t_bt.cpu().numpy(), btck_ref), call
        assert np.array_equal(t_max.cpu().numpy(), rec_hi["score"]), call
        assert np.array_equal(t_xy.cpu().numpy().view(np.uint32), rec_lo["end"]), call


def test_dp1_noalloc_rejects_wide_slabs():
    import cother_b200 as cb
    L = cb.load_library()
    dummy = ctypes.c_void_p(16)   # never dereferenced: the size check comes first
    rc = L.cbp_dp1_noalloc(dummy, 65537, 10, dummy, 100, 1, dummy, dummy, dummy, 0, 1, 0,
                           dummy, dummy, dummy, None)
    assert rc == 5
    assert b"65536" in L.cbp_last_error()


def test_dp1_noalloc_skips_profiles_outside_the_slab(ss_table):
    """A profile whose columns do not lie inside [0, ld) of the slab -- one
    starting before the slab, one running past its last column -- is skipped
    by the kernel and flagged (NaN maximum, coordinates 0xffffffff): nothing
    of it is written, so the shared scratch array cannot be overrun. The
    other profiles keep their results."""
    import torch
    import cother_b200 as cb
    from cother_b200 import synth

    q = synth.make_profiles([70], 311, True)
    db = synth.make_profiles([40, 90, 33, 64, 20], 312, False)
    sc, btck_ref, rec_hi = _regular_path(q, db, ss_table, 3.0e38)
    dev = torch.device("cuda:0")
    Lq, ld = sc.shape
    P = db.nprofiles
    starts = np.ascontiguousarray(db.starts, np.int64).copy()
    starts[0] = -5                       # begins before the slab
    starts[4] = ld - 7                   # 20 positions, ends 13 columns past it
    t_sc = torch.from_numpy(np.ascontiguousarray(sc)).to(dev)
    t_qtrn = torch.from_numpy(np.ascontiguousarray(q.trn)).to(dev)
    t_dtrn = torch.from_numpy(np.ascontiguousarray(db.trn)).to(dev)
    t_len = torch.from_numpy(np.ascontiguousarray(db.lens, np.int32)).to(dev)
    t_start = torch.from_numpy(starts).to(dev)
    t_bt = torch.full((Lq, ld), 255, dtype=torch.uint8, device=dev)
    t_max = torch.full((P,), -1.0, dtype=torch.float32, device=dev)
    t_xy = torch.zeros((P,), dtype=torch.int32, device=dev)
    L = cb.load_library()
    stream = torch.cuda.current_stream(dev)
    rc = L.cbp_dp1_noalloc(t_sc.data_ptr(), ld, Lq, t_qtrn.data_ptr(), db.npositions, P,
                           t_dtrn.data_ptr(), t_len.data_ptr(), t_start.data_ptr(), 0, P, 0,
                           t_bt.data_ptr(), t_max.data_ptr(), t_xy.data_ptr(),
                           ctypes.c_void_p(stream.cuda_stream))
    assert rc == 0, L.cbp_last_error()
    torch.cuda.synchronize(dev)
    mx = t_max.cpu().numpy()
    xy = t_xy.cpu().numpy().view(np.uint32)
    bt = t_bt.cpu().numpy()
    for p in (0, 4):
        assert np.isnan(mx[p]) and xy[p] == 0xffffffff, p
        s0, Ld = int(db.starts[p]), int(db.lens[p])
        assert (bt[:, s0:s0 + Ld] == 255).all(), p     # its own columns untouched
    for p in (1, 2, 3):
        s0, Ld = int(db.starts[p]), int(db.lens[p])
        assert mx[p] == rec_hi["score"][p], p
        assert np.array_equal(bt[:, s0:s0 + Ld], btck_ref[:, s0:s0 + Ld]), p
