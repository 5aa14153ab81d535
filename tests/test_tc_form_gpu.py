"""The tensor-core forms of the profile-profile term (BF16x3 and TF32x3 on
the tcgen05 tensor cores) against the plain FP32 form and an FP64
restatement.

With the SS and DDMS terms off, a cell's score is log(sum) - shift, where
sum = sum_a q_a d_a / (0.5 (qbg_a + dbg_a)); the test computes the sums in
FP64 and bounds each form's error (the plain form is the reference's FP32
operation order). With every term on, the forms must report the same top
hits in the same order, scores within 1e-4 and log E-values within 1e-3
relative of the plain form."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _scores(q, db, ss, **opt):
    import cother_b200 as cb
    o = cb.Options.defaults()
    for k, v in opt.items():
        setattr(o, k, v)
    with cb.BatchProcessing(ss, o) as bp:
        bp.set_score_threshold(3.0e38)
        bp.transfer_cpm_data(db)
        bp.process_score_matrix(q)
        sc, _, _ = bp.read_score_matrix(q.npositions, db.npositions)
    return sc.astype(np.float64)


def test_forms_against_fp64(ss_table):
    import cother_b200 as cb
    from cother_b200 import synth
    q = synth.make_profiles([130], 951, True)
    db = synth.make_profiles(synth.lognormal_lengths(30, 150, 30, 400, seed=952), 953, False)
    qtf = q.tf.astype(np.float64)                       # [20][Lq]
    qbg = q.bkg[:, 0].astype(np.float64)
    dtf = db.tf.astype(np.float64)                      # [20][N]
    dbg = db.bkg.astype(np.float64)[:, db.addrpro]      # [20][N]
    w = dtf / (0.5 * (qbg[:, None] + dbg))
    ref = np.log(qtf.T @ w) - 0.002                     # MAPALN=1 shift
    errs = {}
    for name, form in (("plain", cb.TC_PLAIN), ("bf16x3", cb.TC_BF16X3), ("tf32x3", cb.TC_TF32X3)):
        sc = _scores(q, db, ss_table, ssswgt=0.0, ddmswgt=0.0, tc_form=form)
        errs[name] = float(np.max(np.abs(sc - ref)))
    # a few float32 ulps of the log; the split forms keep about FP32 accuracy
    assert errs["plain"] < 2e-6, errs
    assert errs["bf16x3"] < 2e-5, errs
    assert errs["tf32x3"] < 2e-5, errs


def test_forms_report_the_same_top_hits(ss_table):
    import cother_b200 as cb
    from cother_b200 import synth
    q = synth.make_profiles([180], 961, True)
    db = synth.make_profiles(synth.lognormal_lengths(400, 180, 30, 600, seed=962), 963, False)
    synth.plant_homologs(q, db, 0.05, seed=964)
    res = {}
    for form in (cb.TC_PLAIN, cb.TC_BF16X3, cb.TC_TF32X3):
        o = cb.Options.defaults()
        o.tc_form = form
        with cb.BatchProcessing(ss_table, o) as bp:
            bp.set_db_details(db.npositions, db.nprofiles)
            bp.transfer_cpm_data(db)
            bp.process_score_matrix(q)
            recs = cb.records_table(bp.hit_records())
            order = bp.hit_list()
            res[form] = (recs, order)
    def top(form, n=50):
        recs, order = res[form]
        sel = order[:n]
        return recs["org_pro_no"][sel], recs["score"][sel], recs["log_evalue"][sel]

    p0, s0, e0 = top(cb.TC_PLAIN)
    assert len(p0) >= 10
    for form in (cb.TC_BF16X3, cb.TC_TF32X3):
        p1, s1, e1 = top(form)
        assert np.array_equal(p1, p0), form
        assert np.all(np.abs(s1 - s0) <= 1e-4 * np.abs(s0) + 1e-6), form
        assert np.all(np.abs(e1 - e0) <= 1e-3 * np.abs(e0) + 1e-6), form


def test_forms_dp_optima_and_evalues_against_fp64(ss_table):
    """Phase-1 optima and log E-values of each form against the same stages
    run by the oracle on FP64 cell scores (the profile-profile term alone,
    rounded once to FP32): the DP and the statistics stay FP32 in every
    form, so this isolates the error the contraction brings into them."""
    import cother_b200 as cb
    from cother_b200 import synth
    from oracle import oracle as O
    q = synth.make_profiles([150], 971, True)
    db = synth.make_profiles(synth.lognormal_lengths(40, 150, 30, 400, seed=972), 973, False)
    synth.plant_homologs(q, db, 0.2, seed=974)
    qtf = q.tf.astype(np.float64)
    qbg = q.bkg[:, 0].astype(np.float64)
    dbg = db.bkg.astype(np.float64)[:, db.addrpro]
    ref = (np.log(qtf.T @ (db.tf.astype(np.float64) / (0.5 * (qbg[:, None] + dbg)))) - 0.002)
    ref32 = ref.astype(np.float32)
    thld = -1.0e30
    rec64, _ = O.dp1(q, db, ref32, 0, 0, db.nprofiles, thld)
    sspace = float(db.npositions) * q.npositions

    def logE(S, rec):
        out = []
        for p in range(db.nprofiles):
            s0, Ld = int(db.starts[p]), int(db.lens[p])
            st, _ = O.pair_statistics(S[:, s0:s0 + Ld], q.aa, db.aa[s0:s0 + Ld], rec["score"][p],
                                      rec["psts"][p], q.npositions, Ld, q.eno[0], db.eno[p], sspace)
            out.append(st[2])
        return np.array(out, np.float64)

    e64 = logE(ref32, rec64)
    report = {}
    for name, form in (("plain", cb.TC_PLAIN), ("bf16x3", cb.TC_BF16X3), ("tf32x3", cb.TC_TF32X3)):
        sc = _scores(q, db, ss_table, ssswgt=0.0, ddmswgt=0.0, tc_form=form).astype(np.float32)
        rec, _ = O.dp1(q, db, sc, 0, 0, db.nprofiles, thld)
        e = logE(sc, rec)
        d_cell = float(np.max(np.abs(sc.astype(np.float64) - ref)))
        d_opt = float(np.max(np.abs(rec["maxsc"].astype(np.float64) - rec64["maxsc"]) /
                             np.maximum(np.abs(rec64["maxsc"].astype(np.float64)), 1.0)))
        d_sc = float(np.max(np.abs(rec["score"].astype(np.float64) - rec64["score"]) /
                            np.maximum(np.abs(rec64["score"].astype(np.float64)), 1.0)))
        d_e = float(np.max(np.abs(e - e64) / np.maximum(np.abs(e64), 1.0)))
        report[name] = (d_cell, d_opt, d_sc, d_e)
        assert d_opt < 1e-4 and d_sc < 1e-4 and d_e < 1e-3, (name, report[name])
    print("\nform    cell max-abs  DP optimum rel  phase-1 score rel  log E rel   (vs FP64 cells)")
    for name, (a, b, c, d) in report.items():
        print(f"{name:7s} {a:12.3e}  {b:14.3e}  {c:17.3e}  {d:10.3e}")


def test_fp64_parameter_fit(oracle_lib, ss_table):
    """The precision forms fit lambda, K and H of every passed pair in FP64
    on the GPU and compute its E-value from them (the rest stays FP32).
    Checked against the oracle's FP64 restatement of the fit on the same
    histogram (relative 1e-9), the FP32 fit of the same run against the
    oracle's FP32 fit (bit for bit), and each pair's log E-value against the
    oracle's FP32 E-value computation fed the oracle's FP64 parameters. The
    FP32 fit's relative error against FP64 is reported."""
    import cother_b200 as cb
    from cother_b200 import synth
    O = oracle_lib
    q = synth.make_profiles([160], 981, True)
    db = synth.make_profiles(synth.lognormal_lengths(60, 160, 30, 400, seed=982), 983, False)
    synth.plant_homologs(q, db, 0.2, seed=984)
    o = cb.Options.defaults()
    o.tc_form = cb.TC_BF16X3
    with cb.BatchProcessing(ss_table, o) as bp:
        bp.set_score_threshold(-1.0)            # every pair passes
        bp.set_db_details(db.npositions * 100, db.nprofiles * 100)
        bp.transfer_cpm_data(db)
        bp.process_score_matrix(q)
        sc, _, _ = bp.read_score_matrix(q.npositions, db.npositions)
        recs = cb.records_table(bp.read_statistics())
        fits = bp.read_fits()
        sspace, _ = bp.search_space()
    n = len(recs["score"])
    assert n == db.nprofiles and fits.shape == (n, 8)
    errs = {"lambda": 0.0, "K": 0.0, "H": 0.0}
    nfit = 0
    for k in range(n):
        p = int(recs["org_pro_no"][k])
        s0, Ld = int(db.starts[p]), int(db.lens[p])
        st, cnt = O.pair_statistics(sc[:, s0:s0 + Ld], q.aa, db.aa[s0:s0 + Ld], recs["score"][k],
                                    recs["psts"][k], q.npositions, Ld, q.eno[0], db.eno[p], sspace)
        f64 = O.stat_params64(cnt)
        # FP64 fit: the oracle's FP64 restatement
        assert np.allclose(fits[k, :4], f64, rtol=1e-9, atol=1e-12), (p, fits[k, :4], f64)
        # FP32 fit of the same run: the oracle's FP32 fit, bit for bit
        assert np.array_equal(fits[k, 4:].astype(np.float32),
                              np.array([st[8], st[9], st[7], st[6]], np.float32)), (p, fits[k, 4:], st)
        # the E-value from the FP64 parameters
        sig = O.significance(q.npositions, Ld, q.eno[0], db.eno[p], recs["score"][k], recs["psts"][k],
                             np.float32(f64[0]), np.float32(f64[1]), sspace)
        assert recs["log_evalue"][k] == sig[2], (p, recs["log_evalue"][k], sig[2])
        assert recs["lambda"][k] == np.float32(f64[0]) and recs["K"][k] == np.float32(f64[1])
        if f64[0] > 0 and f64[1] > 0:
            nfit += 1
            for name, i in (("lambda", 0), ("K", 1), ("H", 2)):
                errs[name] = max(errs[name], abs(fits[k, 4 + i] - fits[k, i]) / abs(fits[k, i]))
    assert nfit >= 10, nfit
    assert errs["lambda"] < 1e-4 and errs["K"] < 1e-3 and errs["H"] < 1e-4, errs
    print("\nFP32 parameter fit vs FP64 (%d pairs): max relative error lambda %.2e, K %.2e, H %.2e"
          % (nfit, errs["lambda"], errs["K"], errs["H"]))


def test_map_posteriors_against_fp64(oracle_lib, ss_table):
    """MAP posteriors of every form against FP64. For each pair the MAP
    stage realigns (all terms on, planted homologs), the GPU's forward +
    backward values equal the oracle's FP32 restatement of the stage bit for
    bit, given the form's own cell scores. The posteriors the MAP DP reads,
    exp(fb - log Z) with the stage's Schraudolph exponential, are compared
    with the same model evaluated in FP64 with exact exp/log on the same
    cells: the difference is the FP32 stage's, dominated by the fast
    exp/log approximations that the reference uses and this build
    reproduces. Also reported: each tensor-core form's posteriors against
    the plain form's."""
    import cother_b200 as cb
    from cother_b200 import synth
    O = oracle_lib
    q = synth.make_profiles([150], 991, True)
    db = synth.make_profiles(synth.lognormal_lengths(40, 150, 30, 400, seed=992), 993, False)
    synth.plant_homologs(q, db, 0.2, seed=994)
    Lq = q.npositions
    report, post = {}, {}
    for name, form in (("plain", cb.TC_PLAIN), ("bf16x3", cb.TC_BF16X3), ("tf32x3", cb.TC_TF32X3)):
        o = cb.Options.defaults()
        o.tc_form = form
        with cb.BatchProcessing(ss_table, o) as bp:
            bp.set_db_details(180 * 1000, 1000)
            bp.transfer_cpm_data(db)
            bp.process_score_matrix(q)
            sc, ms, _ = bp.read_score_matrix(Lq, db.npositions)
            recs = cb.records_table(bp.hit_records())
            alns = bp.alignments(Lq)
            st = cb.records_table(bp.read_statistics())
            errs, n = [], 0
            for k in range(len(recs["org_pro_no"])):
                if alns[k] is None:
                    continue
                p = int(recs["org_pro_no"][k])
                s0, Ld = int(db.starts[p]), int(db.lens[p])
                S, M = sc[:, s0:s0 + Ld], ms[:, s0:s0 + Ld]
                epa = float(st["log_evalue_pair"][k])
                mo = O.map_pair(q, db, p, S, M, epa)
                fb = bp.map_fb(k, Lq)
                assert np.array_equal(fb.view(np.uint32), mo["fb"].view(np.uint32)), (name, p)
                P32 = O.fast_expf(fb - np.float32(mo["logz"])).astype(np.float64)
                P64, _ = O.map_posteriors64(q, db, p, S, M, epa)
                big = P64 >= 0.01
                errs.append((float(np.max(np.abs(P32 - P64))),
                             float(np.max(np.abs(P32 - P64)[big] / P64[big])) if big.any() else 0.0))
                post[(name, p)] = P32
                n += 1
        assert n >= 5, (name, n)
        report[name] = (n, max(e[0] for e in errs), max(e[1] for e in errs))
        assert report[name][1] < 0.25, (name, report[name])
    vs_plain = {}
    for name in ("bf16x3", "tf32x3"):
        d = [float(np.max(np.abs(post[(name, p)] - post[("plain", p)])))
             for (f, p) in post if f == "plain" and (name, p) in post]
        vs_plain[name] = max(d) if d else float("nan")
    print("\nform    pairs  posterior max-abs vs FP64  max rel (P64 >= 0.01)  max-abs vs plain")
    for name, (n, a, r) in report.items():
        print(f"{name:7s} {n:5d}  {a:24.3e}  {r:22.3e}  {vs_plain.get(name, 0.0):16.3e}")
