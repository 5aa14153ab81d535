"""CPU tests of the oracle: pinned against the reference's own CPU code and
golden vectors (no GPU)."""
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN, ROOT


def test_logf_accuracy(oracle_lib):
    rng = np.random.default_rng(5)
    xs = np.exp(rng.uniform(-87, 88, 20000)).astype(np.float32)
    xs = np.concatenate([xs, np.float32([1e-40, 1e-45, 1.0, 2.0, 0.5, 3.4e38, 1.4142135, 0.70710677])])
    got = np.array([oracle_lib.logf(float(x)) for x in xs], np.float64)
    ref = np.log(xs.astype(np.float64))
    ulp = np.abs(got - ref) / np.spacing(np.abs(ref).astype(np.float32)).astype(np.float64)
    ulp[ref == 0] = np.abs(got[ref == 0]) / np.spacing(np.float32(1))
    assert ulp.max() < 2.0


def test_dms_pair_scores(oracle_lib):
    L = oracle_lib.lib()
    # table values of the two-level interpolation: s(d1,d2) = 0.35 + 0.02*min - 0.0375*max
    for d1 in range(0, 25):
        for d2 in range(0, 25):
            a, b = min(max(d1, d2), 20), min(min(d1, d2), 20)
            want = 0.35 + 0.02 * b - 0.0375 * a
            assert abs(L.orc_dms_pair_score(d1, d2) - want) < 1e-6
    assert L.orc_dms_pair_score(255, 3) == -1.0
    assert L.orc_dms_pair_score(7, 255) == -1.0


def test_ddms_matches_reference_cpu_code(oracle_lib):
    """The oracle's DDMS segment DP equals the reference's own CPU
    restatement (cother-scores-optimizer/ddms.cxx) on committed vectors, with
    that restatement's pair-score rounding (each operation rounded)."""
    z = np.load(os.path.join(GOLDEN, "ddms_ref.npz"))
    n = 0
    for q, d, r in zip(z["qlists"], z["dlists"], z["ref"]):
        s, raw, comp = oracle_lib.ddms_cell(q, d, fused=False)
        if r == -777.0:
            continue
        assert comp == 1
        assert np.float32(np.rint(np.float32(raw) * np.float32(16.0))) == r
        n += 1
    assert n > 300


def test_ddms_matches_reference_live(oracle_lib):
    """Same check against the reference library built here, when present."""
    R = oracle_lib.ref_lib()
    if R is None:
        pytest.skip("reference tree not available")
    from cother_b200 import synth
    q = synth.make_profiles([70], 1234, True)
    d = synth.make_profiles([90, 30], 1235, False)
    ql, dl = q.dd_lists(), d.dd_lists()
    for i in range(0, 70, 3):
        for j in range(0, 120, 7):
            s, raw, comp = oracle_lib.ddms_cell(ql[i], dl[j], fused=False)
            x = np.full(110, 255, np.int32); x[:ql[i][0] + 1] = ql[i][:ql[i][0] + 1]
            y = np.full(110, 255, np.int32); y[:dl[j][0] + 1] = dl[j][:dl[j][0] + 1]
            r = R.ref_ddms_scaled_sum(x.ctypes.data, y.ctypes.data)
            if r == -777.0:
                continue
            assert np.float32(np.rint(np.float32(raw) * np.float32(16.0))) == r


def test_ddms_short_lists(oracle_lib):
    q = np.full(100, 255, np.uint8); q[0] = 5; q[1:6] = [5, 6, 7, 8, 9]
    d = np.full(100, 255, np.uint8); d[0] = 40; d[1:41] = 8
    s, raw, comp = oracle_lib.ddms_cell(q, d, dstsegm=6)
    assert comp == 0 and s == 0.0
    q[0] = 6; q[6] = 10
    s, raw, comp = oracle_lib.ddms_cell(q, d, dstsegm=6)
    assert comp == 1


def test_score_matrix_oracle_shapes(oracle_lib, ss_table):
    from cother_b200 import synth
    q = synth.make_profiles([23], 3, True)
    db = synth.make_profiles([17, 40, 5], 4, False)
    sc, ms = oracle_lib.score_matrix(q, db, ss_table)
    assert sc.shape == (23, 62) and ms.shape == (23, 62)
    assert np.isfinite(sc).all() and np.isfinite(ms).all()
    sc2, ms2 = oracle_lib.score_matrix(q, db, ss_table, col0=17, ncols=40, nthreads=3)
    assert np.array_equal(sc2, sc[:, 17:57]) and np.array_equal(ms2, ms[:, 17:57])


def test_library_nn_weights_equal_fixture():
    """The significance-network weights compiled into the CUDA library
    (kNNWeightsTable in cother_b200/csrc/api.cu) are the reference's table
    (src/libmycu/cupro/CuDeviceMemory.cu:43-80, fixture nn_weights.npy)."""
    import re
    src = open(os.path.join(ROOT, "cother_b200", "csrc", "api.cu")).read()
    i = src.index("kNNWeightsTable[kNNWeights] = {")
    body = src[i:src.index("};", i)].split("{", 1)[1]
    vals = np.array([np.float32(v.rstrip("f")) for v in
                     re.findall(r"[-+]?[0-9]*\.?[0-9]+(?:[eE][-+]?[0-9]+)?f?", body)], np.float32)
    ref = np.load(os.path.join(GOLDEN, "nn_weights.npy"))
    assert vals.shape == ref.shape
    assert np.array_equal(vals, ref)


def test_cvs_map_smoothing_and_fixture():
    """The CVS map reader's smoothing (CVS2Scores::SmoothScores): 5-point
    running means, the first entries taking the first full window and the
    trailing ones (and '+' entries) the last; and the committed map."""
    sys.path.insert(0, GOLDEN)
    import make_fixtures as mf
    f = np.float32
    k = [f(x) for x in (-1.0, -0.5, 0.0, 0.5, 1.0, 1.5, 2.0)]
    keys, sc, shift = mf.smooth_cvs_scores(k, [f(x) for x in (1, 2, 3, 4, 5, 6, 7)])
    assert shift == 2 and np.array_equal(sc, np.array([3, 3, 3, 4, 5, 5, 5], np.float32))
    _, sc, _ = mf.smooth_cvs_scores(k, [f(x) for x in (1, 2, 3, 4, 5, 6)] + [mf.CVS_PLUS])
    assert np.array_equal(sc, np.array([3, 3, 3, 4, 4, 4, 4], np.float32))
    z = np.load(os.path.join(GOLDEN, "cvs2s.npz"))
    keys, scores, shift = z["keys"], z["scores"], int(z["shift"])
    assert len(keys) == len(scores) == 93 and shift == 5
    assert np.array_equal(keys, (np.arange(93, dtype=np.float32) - 5) * np.float32(0.5))
    assert np.all(np.isfinite(scores)) and scores[0] < 0 < scores[-1]


def test_cvs_constants(oracle_lib):
    """1/kappa0, -(nu0+2)/2 and the constant term of the CVS log-odds."""
    lk, pw, ct = oracle_lib.cvs_constants()
    assert lk == np.float32(10.0) and pw == np.float32(-10.5)
    import math
    exact = (9.5 - 10.5) * (math.log(0.1) - math.log(2.1)) + sum(
        math.log(20 - i) - math.log(2) for i in range(1, 20))
    assert abs(ct - exact) < 1e-4


def test_fast_expf_vectorized(oracle_lib):
    """The vectorized Schraudolph exponential equals the oracle's C one bit
    for bit (including its cut-off at -16)."""
    import ctypes
    L = oracle_lib.lib()
    L.orc_fast_expf.restype = ctypes.c_float
    L.orc_fast_expf.argtypes = [ctypes.c_float]
    rng = np.random.default_rng(11)
    a = np.concatenate([rng.uniform(-20.0, 4.0, 3000), rng.uniform(-1.0, 1.0, 1000),
                        np.array([-16.0, -15.999999, 0.0, -0.0], np.float64)]).astype(np.float32)
    got = oracle_lib.fast_expf(a)
    ref = np.array([L.orc_fast_expf(float(x)) for x in a], np.float32)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_map_posteriors_fp64_restatement(oracle_lib, ss_table):
    """The FP64 forward-backward of the MAP stage: posteriors are
    probabilities, the top-scoring cells of a planted homolog approach 1, and
    the FP32 stage's posteriors (Schraudolph exp/log) lie within 0.25 of
    them (the error the GPU test reports per form)."""
    from cother_b200 import synth
    O = oracle_lib
    q = synth.make_profiles([90], 1201, True)
    db = synth.make_profiles([120, 80], 1202, False)
    synth.plant_homologs(q, db, 1.0, seed=1203)
    sc, ms = O.score_matrix(q, db, ss_table, nthreads=4)
    for p in range(db.nprofiles):
        s0, Ld = int(db.starts[p]), int(db.lens[p])
        S, M = sc[:, s0:s0 + Ld], ms[:, s0:s0 + Ld]
        mo = O.map_pair(q, db, p, S, M, -30.0)
        P64, lz = O.map_posteriors64(q, db, p, S, M, -30.0)
        assert np.all(P64 >= 0.0) and np.all(P64 <= 1.0 + 1e-9)
        assert P64.max() > 0.9 and np.isfinite(lz)
        P32 = O.fast_expf(mo["fb"] - np.float32(mo["logz"])).astype(np.float64)
        assert np.max(np.abs(P32 - P64)) < 0.25
