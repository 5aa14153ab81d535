"""ctypes loader for the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module, and only as the checker. The product path
(``cother_b200``) never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libddmsref.so")
REFERENCE_TREE = "/root/reference"

_lib = None
_ref = None


def build(force: bool = False) -> None:
    """Compile the oracle and, when the reference tree is present, the
    reference's DDMS restatement, its CUDA kernels and its description
    formatters (oracle/_ref/)."""
    args = ["make", "-s", "-C", HERE, "all"]
    if force:
        subprocess.run(["make", "-s", "-C", HERE, "clean"], check=True)
    subprocess.run(args, check=True)
    if os.path.isdir(os.path.join(REFERENCE_TREE, "cother-scores-optimizer")):
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)
    if os.path.isdir(os.path.join(REFERENCE_TREE, "src", "libmycu")):
        subprocess.run(["make", "-s", "-C", HERE, "refgpu"], check=True)
    if os.path.isfile(os.path.join(REFERENCE_TREE, "src", "liblib", "fmtdescription.h")):
        subprocess.run(["make", "-s", "-C", HERE, "fmtref"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        L.orc_logf.restype = ctypes.c_float
        L.orc_logf.argtypes = [ctypes.c_float]
        L.orc_dms_pair_score.restype = ctypes.c_float
        L.orc_dms_pair_score.argtypes = [ctypes.c_int, ctypes.c_int]
        L.orc_ddms_cell.restype = ctypes.c_float
        L.orc_ddms_cell.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_float,
                                    ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_int)]
        L.orc_ddms_cell_ex.restype = ctypes.c_float
        L.orc_ddms_cell_ex.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                       ctypes.c_float, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_float),
                                       ctypes.POINTER(ctypes.c_int)]
        sm_args = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_longlong, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_longlong, ctypes.c_longlong,
                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_longlong]
        L.orc_score_matrix.restype = None
        L.orc_score_matrix.argtypes = sm_args
        L.orc_score_matrix_mt.restype = None
        L.orc_cvs_constants.restype = None
        L.orc_score_matrix_mt.argtypes = [ctypes.c_int] + sm_args
        L.orc_dp1_profile.restype = ctypes.c_float
        L.orc_dp1_profile.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_longlong,
                                      ctypes.c_void_p, ctypes.c_longlong, ctypes.c_void_p,
                                      ctypes.c_longlong, ctypes.c_void_p,
                                      ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        L.orc_dp1_finalize.restype = ctypes.c_int
        L.orc_dp1_finalize.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_longlong,
                                       ctypes.c_void_p, ctypes.c_float, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_float, ctypes.POINTER(ctypes.c_float),
                                       ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_uint32),
                                       ctypes.POINTER(ctypes.c_uint32)]
        L.orc_score_threshold.restype = None
        L.orc_score_threshold.argtypes = [ctypes.c_size_t, ctypes.c_size_t, ctypes.c_float,
                                          ctypes.c_float, ctypes.c_float,
                                          ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]
        _lib = L
    return _lib


def ref_lib():
    """The reference's own DDMS restatement, or None when not built here."""
    global _ref
    if _ref is None and os.path.exists(REF_LIB):
        R = ctypes.CDLL(REF_LIB)
        R.ref_ddms_scaled_sum.restype = ctypes.c_float
        R.ref_ddms_scaled_sum.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        _ref = R
    return _ref


class ScoreParams(ctypes.Structure):
    _fields_ = [("ssswgt", ctypes.c_float), ("ddmswgt", ctypes.c_float),
                ("dstsegm", ctypes.c_int), ("initshift", ctypes.c_float),
                ("cvswgt", ctypes.c_float),
                ("q_cv", ctypes.c_void_p), ("q_cvprior", ctypes.c_void_p),
                ("q_cvnorm2", ctypes.c_void_p),
                ("d_cv", ctypes.c_void_p), ("d_cvprior", ctypes.c_void_p),
                ("d_cvnorm2", ctypes.c_void_p),
                ("cvs_scores", ctypes.c_void_p), ("cvs_card", ctypes.c_int),
                ("cvs_shift", ctypes.c_int), ("cvs_key_first", ctypes.c_float),
                ("cvs_key_last", ctypes.c_float), ("cvs_ambiguous", ctypes.c_void_p),
                ("cvs_int_priors", ctypes.c_int)]


def load_cvs_map(path=None):
    """The committed CVS map: dict(keys, scores, shift)."""
    path = path or os.path.join(os.path.dirname(HERE), "tests", "golden", "cvs2s.npz")
    z = np.load(path)
    return {"keys": np.ascontiguousarray(z["keys"], np.float32),
            "scores": np.ascontiguousarray(z["scores"], np.float32),
            "shift": int(z["shift"])}


def cvs_constants():
    """(1/kappa0, -(nu0+2)/2, constant term) of the CVS score."""
    a, b, c = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
    lib().orc_cvs_constants(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
    return a.value, b.value, c.value


def logf(x: float) -> float:
    return lib().orc_logf(x)


def ddms_cell(qlist: np.ndarray, dlist: np.ndarray, dstsegm: int = 6, ddmswgt: float = 0.2,
              fused: bool = True):
    """DDMS of one cell: (score, top-3 sum, computed). `fused` selects the
    pair-score rounding of the reference's CUDA kernel (True) or of its CPU
    restatement in cother-scores-optimizer (False)."""
    q = np.ascontiguousarray(qlist, dtype=np.uint8)
    d = np.ascontiguousarray(dlist, dtype=np.uint8)
    raw = ctypes.c_float()
    comp = ctypes.c_int()
    s = lib().orc_ddms_cell_ex(q.ctypes.data, d.ctypes.data, dstsegm, ddmswgt, int(fused),
                               ctypes.byref(raw), ctypes.byref(comp))
    return s, raw.value, comp.value


def score_matrix(query, db, ss_table, ssswgt=0.12, ddmswgt=0.2, dstsegm=6, initshift=0.002,
                 col0=0, ncols=None, nthreads=1, cvswgt=0.0, cvs_map=None, ambiguous=False,
                 mapaln=True):
    """(scores, modscores) [Lq][ncols] for query vs db columns [col0, col0+ncols).

    With cvswgt > 0 the context-vector term is added (both profile sets
    must carry context vectors; the map defaults to the committed one);
    with ambiguous=True a third array [Lq][ncols] (uint8) marks the cells
    whose map lookup the reference's fast logarithm may move to a
    neighbouring entry. mapaln=False is the MAPALN=0 configuration (the
    caller passes initshift=0.0003; the CVS log priors are truncated)."""
    Lq = query.npositions
    N, P = db.npositions, db.nprofiles
    if ncols is None:
        ncols = N - col0
    q_tf = np.ascontiguousarray(query.tf, np.float32)
    q_bkg = np.ascontiguousarray(query.bkg[:, 0], np.float32)
    q_ss = np.ascontiguousarray(query.ss, np.float32)
    q_dd = query.dd_lists()
    d_tf = np.ascontiguousarray(db.tf, np.float32)
    d_bkg = np.ascontiguousarray(db.bkg, np.float32)
    d_pro = np.ascontiguousarray(db.addrpro, np.int32)
    d_ss = np.ascontiguousarray(db.ss, np.float32)
    d_dd = db.dd_lists()
    T = np.ascontiguousarray(ss_table, np.float32)
    sc = np.zeros((Lq, ncols), np.float32)
    ms = np.zeros((Lq, ncols), np.float32)
    prm = ScoreParams(ssswgt, ddmswgt, dstsegm, initshift)
    keep = []
    amb = np.zeros((Lq, ncols), np.uint8) if ambiguous else None
    if cvswgt > 0.0:
        if query.cv is None or db.cv is None:
            raise ValueError("CVSWGT > 0 needs context vectors on both profile sets")
        m = cvs_map or load_cvs_map()
        arrs = [np.ascontiguousarray(x, np.float32) for x in
                (query.cv, query.cvprior, query.cvnorm2, db.cv, db.cvprior, db.cvnorm2, m["scores"])]
        keep += arrs
        prm.cvswgt = float(cvswgt)
        (prm.q_cv, prm.q_cvprior, prm.q_cvnorm2, prm.d_cv, prm.d_cvprior, prm.d_cvnorm2,
         prm.cvs_scores) = [a.ctypes.data for a in arrs]
        prm.cvs_card = len(m["scores"])
        prm.cvs_shift = int(m["shift"])
        prm.cvs_key_first = float(m["keys"][0])
        prm.cvs_key_last = float(m["keys"][-1])
        prm.cvs_int_priors = 0 if mapaln else 1
        if amb is not None:
            prm.cvs_ambiguous = amb.ctypes.data
    lib().orc_score_matrix_mt(int(nthreads), Lq, q_tf.ctypes.data, q_bkg.ctypes.data,
                              q_ss.ctypes.data, q_dd.ctypes.data, N, P, d_tf.ctypes.data,
                              d_bkg.ctypes.data, d_pro.ctypes.data, d_ss.ctypes.data,
                              d_dd.ctypes.data, T.ctypes.data, ctypes.byref(prm),
                              int(col0), int(ncols), sc.ctypes.data, ms.ctypes.data, int(ncols))
    del keep
    return (sc, ms, amb) if ambiguous else (sc, ms)


def dp1(query, db, scores, col0, p0, nprof, thld):
    """Phase-1 DP + finalization for profiles p0..p0+nprof-1 of db whose
    score columns start at chunk position col0 in `scores` ([Lq][ncols]).

    Returns (records, btck) with records a dict of arrays (score, psts, beg,
    end, passed, maxsc, maxr, maxc) and btck [Lq][ncols] uint8."""
    L = lib()
    Lq = query.npositions
    sc = np.ascontiguousarray(scores, np.float32)
    ncols = sc.shape[1]
    btck = np.zeros((Lq, ncols), np.uint8)
    qtrn = np.ascontiguousarray(query.trn, np.float32)
    dtrn = np.ascontiguousarray(db.trn, np.float32)
    NT = dtrn.shape[1]
    out = {k: [] for k in ("score", "psts", "beg", "end", "passed", "maxsc", "maxr", "maxc")}
    starts = db.starts
    for k in range(nprof):
        p = p0 + k
        Ld = int(db.lens[p])
        c0 = int(starts[p]) - col0
        sub = np.ascontiguousarray(sc[:, c0:c0 + Ld])
        bt = np.zeros((Lq, Ld), np.uint8)
        mr, mc = ctypes.c_int(), ctypes.c_int()
        tb = int(starts[p]) + p
        dptr = dtrn.ctypes.data + 4 * tb
        m = L.orc_dp1_profile(Lq, Ld, sub.ctypes.data, Ld, qtrn.ctypes.data, qtrn.shape[1], dptr, NT,
                              bt.ctypes.data, ctypes.byref(mr), ctypes.byref(mc))
        s_, ps = ctypes.c_float(), ctypes.c_float()
        b, e = ctypes.c_uint32(), ctypes.c_uint32()
        pas = L.orc_dp1_finalize(Lq, Ld, sub.ctypes.data, Ld, bt.ctypes.data, m, mr.value, mc.value,
                                 float(thld), ctypes.byref(s_), ctypes.byref(ps), ctypes.byref(b),
                                 ctypes.byref(e))
        btck[:, c0:c0 + Ld] = bt
        for key, v in (("score", s_.value), ("psts", ps.value), ("beg", b.value), ("end", e.value),
                       ("passed", pas), ("maxsc", m), ("maxr", mr.value), ("maxc", mc.value)):
            out[key].append(v)
    rec = {k: np.array(v) for k, v in out.items()}
    rec["score"] = rec["score"].astype(np.float32)
    rec["psts"] = rec["psts"].astype(np.float32)
    rec["maxsc"] = rec["maxsc"].astype(np.float32)
    return rec, btck


def score_threshold(qlen, dbsize, evalue=10.0, lam=0.561132, K=0.001488):
    a, b = ctypes.c_float(), ctypes.c_float()
    lib().orc_score_threshold(int(qlen), int(dbsize), float(evalue), float(lam), float(K),
                              ctypes.byref(a), ctypes.byref(b))
    return a.value, b.value


# ---------------------------------------------------------------------------
# statistics
_GOLDEN = os.path.join(os.path.dirname(HERE), "tests", "golden")


class SigParams(ctypes.Structure):
    _fields_ = [("ssemodel", ctypes.c_int), ("searchspace", ctypes.c_float),
                ("ref_lambda", ctypes.c_float), ("ref_K", ctypes.c_float),
                ("exp_gapped_lambda", ctypes.c_float), ("exp_gapped_K", ctypes.c_float),
                ("nnweights", ctypes.c_void_p)]


def _stats_lib():
    L = lib()
    if not getattr(L, "_stats_bound", False):
        L.orc_expf.restype = ctypes.c_float
        L.orc_expf.argtypes = [ctypes.c_float]
        L.orc_lgammaf.restype = ctypes.c_float
        L.orc_lgammaf.argtypes = [ctypes.c_float]
        L.orc_lbetaincf.restype = ctypes.c_float
        L.orc_lbetaincf.argtypes = [ctypes.c_float] * 3
        L.orc_lgammainc_Qf.restype = ctypes.c_float
        L.orc_lgammainc_Qf.argtypes = [ctypes.c_float] * 2
        L.orc_score_histogram.restype = None
        L.orc_score_histogram.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_longlong,
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L.orc_stat_params.restype = None
        L.orc_stat_params.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.orc_stat_params64.restype = None
        L.orc_stat_params64.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.orc_significance.restype = None
        L.orc_significance.argtypes = [ctypes.POINTER(SigParams), ctypes.c_int, ctypes.c_int,
                                       ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                       ctypes.c_float, ctypes.c_float, ctypes.c_void_p]
        L.orc_length_adjustment.restype = None
        L.orc_length_adjustment.argtypes = [ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                            ctypes.c_float, ctypes.c_size_t, ctypes.c_ulonglong,
                                            ctypes.c_size_t, ctypes.POINTER(ctypes.c_ulonglong),
                                            ctypes.POINTER(ctypes.c_size_t)]
        L._stats_bound = True
    return L


def cother_par():
    import json
    return json.load(open(os.path.join(_GOLDEN, "cother_par.json")))


def nn_weights():
    return np.load(os.path.join(_GOLDEN, "nn_weights.npy")).astype(np.float32)


def length_adjustment(m, n, N):
    par = cother_par()["GAPPED_A_1"]
    ss, dl = ctypes.c_ulonglong(), ctypes.c_size_t()
    _stats_lib().orc_length_adjustment(par["Lambda"], par["K"], par["Alpha"], par["Beta"], int(m),
                                       int(n), int(N), ctypes.byref(ss), ctypes.byref(dl))
    return ss.value, dl.value


def stat_params64(counts):
    """The parameter fit in FP64 from a pair's score histogram (641 counts):
    (lambda, K, H, expected score), lambda and the expected score per
    unscaled score unit."""
    c = np.ascontiguousarray(counts, np.int32)
    out = np.zeros(4, np.float64)
    _stats_lib().orc_stat_params64(c.ctypes.data, out.ctypes.data)
    return out


def significance(Lq, Ld, qeno, deno, score, psts, lam, K, searchspace, ssemodel=2):
    """(lambda_est, K_est, logE, logEpA) of a pair from given lambda and K
    (the FP32 E-value computation)."""
    L = _stats_lib()
    par = cother_par()
    w = nn_weights()
    sp = SigParams(int(ssemodel), float(searchspace), par["UNGAPPED"]["Lambda"], par["UNGAPPED"]["K"],
                   par["GAPPED_A_1"]["Lambda"], par["GAPPED_A_1"]["K"], w.ctypes.data)
    o4 = np.zeros(4, np.float32)
    L.orc_significance(ctypes.byref(sp), int(Lq), int(Ld), float(qeno), float(deno), float(score),
                       float(psts), float(lam), float(K), o4.ctypes.data)
    return o4


def pair_statistics(S, qaa, daa, score, psts, Lq, Ld, qeno, deno, searchspace, ssemodel=2,
                    xuninf=1):
    """(lambda_est, K_est, logE, logEpA, min, max, E, H, lambda, K) for one
    passed pair; S is its [Lq][Ld] score sub-matrix."""
    L = _stats_lib()
    S = np.ascontiguousarray(S, np.float32)
    qa = np.ascontiguousarray(qaa, np.int8)
    da = np.ascontiguousarray(daa, np.int8)
    counts = np.zeros(641, np.int32)
    L.orc_score_histogram(Lq, Ld, S.ctypes.data, S.shape[1], qa.ctypes.data, da.ctypes.data,
                          int(xuninf), counts.ctypes.data)
    prm = np.zeros(6, np.float32)
    up = np.zeros(21, np.float32)
    L.orc_stat_params(counts.ctypes.data, prm.ctypes.data, up.ctypes.data)
    par = cother_par()
    w = nn_weights()
    sp = SigParams(int(ssemodel), float(searchspace), par["UNGAPPED"]["Lambda"], par["UNGAPPED"]["K"],
                   par["GAPPED_A_1"]["Lambda"], par["GAPPED_A_1"]["K"], w.ctypes.data)
    o4 = np.zeros(4, np.float32)
    L.orc_significance(ctypes.byref(sp), int(Lq), int(Ld), float(qeno), float(deno), float(score),
                       float(psts), float(prm[4]), float(prm[5]), o4.ctypes.data)
    return np.concatenate([o4, prm]), counts


# ---------------------------------------------------------------------------
# phase-2 MAP realignment
class MapIn(ctypes.Structure):
    _fields_ = [("Lq", ctypes.c_int), ("Ld", ctypes.c_int), ("S", ctypes.c_void_p),
                ("M", ctypes.c_void_p), ("lds", ctypes.c_longlong), ("qtrn", ctypes.c_void_p),
                ("qts", ctypes.c_longlong), ("dtrn", ctypes.c_void_p), ("dts", ctypes.c_longlong),
                ("epa", ctypes.c_float), ("minpp", ctypes.c_float), ("modscores", ctypes.c_int),
                ("qaa", ctypes.c_void_p), ("daa", ctypes.c_void_p), ("qss", ctypes.c_void_p),
                ("dss", ctypes.c_void_p), ("printsss", ctypes.c_int), ("qsssinuse", ctypes.c_int),
                ("dsssinuse", ctypes.c_int)]


class MapOut(ctypes.Structure):
    _fields_ = [("fb", ctypes.c_void_p), ("btck", ctypes.c_void_p), ("aln", ctypes.c_void_p * 5),
                ("maxlogprob", ctypes.c_float), ("logz", ctypes.c_float), ("mapmax", ctypes.c_float),
                ("alnlen", ctypes.c_int), ("idts", ctypes.c_int), ("psts", ctypes.c_int),
                ("gaps", ctypes.c_int), ("beg", ctypes.c_uint32), ("end", ctypes.c_uint32)]


def map_pair(query, db, p, S, M, epa, minpp=0.28, modscores=True, printsss=True):
    """MAP realignment of query vs profile p; S, M: the pair's [Lq][Ld]
    scores and modular scores. Returns a dict (fb, btck, alignment rows,
    counts, coordinates, logz, maxlogprob, mapmax)."""
    L = lib()
    if not getattr(L, "_map_bound", False):
        L.orc_map_pair.restype = ctypes.c_int
        L.orc_map_pair.argtypes = [ctypes.POINTER(MapIn), ctypes.POINTER(MapOut)]
        L._map_bound = True
    p = int(p)
    Lq = query.npositions
    Ld = int(db.lens[p])
    s0 = int(db.starts[p])
    S = np.ascontiguousarray(S, np.float32)
    M = np.ascontiguousarray(M, np.float32)
    qtrn = np.ascontiguousarray(query.trn, np.float32)
    dtrn = np.ascontiguousarray(db.trn, np.float32)
    qaa = np.ascontiguousarray(query.aa, np.int8)
    daa = np.ascontiguousarray(db.aa[s0:s0 + Ld], np.int8)
    qss = np.ascontiguousarray(query.ssstate, np.int8)
    dss = np.ascontiguousarray(db.ssstate[s0:s0 + Ld], np.int8)
    fb = np.zeros((Lq, Ld), np.float32)
    bt = np.zeros((Lq, Ld), np.uint8)
    bufs = [ctypes.create_string_buffer(Lq + Ld + 2) for _ in range(5)]
    mi = MapIn(Lq, Ld, S.ctypes.data, M.ctypes.data, S.shape[1], qtrn.ctypes.data, qtrn.shape[1],
               dtrn.ctypes.data + 4 * (s0 + p), dtrn.shape[1], float(epa), float(minpp),
               int(modscores), qaa.ctypes.data, daa.ctypes.data, qss.ctypes.data, dss.ctypes.data,
               int(printsss), 1, 1)
    mo = MapOut()
    mo.fb = fb.ctypes.data
    mo.btck = bt.ctypes.data
    for i in range(5):
        mo.aln[i] = ctypes.cast(bufs[i], ctypes.c_void_p)
    L.orc_map_pair(ctypes.byref(mi), ctypes.byref(mo))
    return {"fb": fb, "btck": bt, "aln": [b.value.decode() for b in bufs], "alnlen": mo.alnlen,
            "idts": mo.idts, "psts": mo.psts, "gaps": mo.gaps, "beg": mo.beg, "end": mo.end,
            "logz": mo.logz, "maxlogprob": mo.maxlogprob, "mapmax": mo.mapmax}


def map_posteriors64(query, db, p, S, M, epa, modscores=True):
    """The MAP forward-backward of query vs profile p in FP64 with exact
    exp/log (orc_map_posteriors64): the match-state posterior of every cell
    [Lq][Ld] (float64) and log Z. S, M as for map_pair."""
    L = lib()
    if not getattr(L, "_post64_bound", False):
        L.orc_map_posteriors64.restype = ctypes.c_int
        L.orc_map_posteriors64.argtypes = [ctypes.POINTER(MapIn), ctypes.c_void_p,
                                           ctypes.POINTER(ctypes.c_double)]
        L._post64_bound = True
    p = int(p)
    Lq = query.npositions
    Ld = int(db.lens[p])
    s0 = int(db.starts[p])
    S = np.ascontiguousarray(S, np.float32)
    M = np.ascontiguousarray(M, np.float32)
    qtrn = np.ascontiguousarray(query.trn, np.float32)
    dtrn = np.ascontiguousarray(db.trn, np.float32)
    qaa = np.ascontiguousarray(query.aa, np.int8)
    daa = np.ascontiguousarray(db.aa[s0:s0 + Ld], np.int8)
    mi = MapIn(Lq, Ld, S.ctypes.data, M.ctypes.data, S.shape[1], qtrn.ctypes.data, qtrn.shape[1],
               dtrn.ctypes.data + 4 * (s0 + p), dtrn.shape[1], float(epa), 0.28, int(modscores),
               qaa.ctypes.data, daa.ctypes.data, qaa.ctypes.data, daa.ctypes.data, 0, 1, 1)
    P = np.zeros((Lq, Ld), np.float64)
    lz = ctypes.c_double()
    L.orc_map_posteriors64(ctypes.byref(mi), P.ctypes.data, ctypes.byref(lz))
    return P, lz.value


def fast_expf(a):
    """Schraudolph's exp as the MAP stage evaluates it (orc_fast_expf),
    elementwise over a float32 array: the float32 fma 12102203.16*a +
    1064631197 (exact in float64, then rounded once), truncated to int32 and
    read as a float; 0 for a <= -16."""
    a = np.asarray(a, np.float32)
    t = (np.float64(np.float32(12102203.16)) * a.astype(np.float64)
         + np.float64(np.float32(1064631197.0))).astype(np.float32)
    out = np.trunc(t.astype(np.float64)).astype(np.int32).view(np.float32)
    return np.where(np.float32(-16.0) < a, out, np.float32(0.0))


def aln_pair(query, db, p, S, btck1, maxsc, maxr, maxc, printsss=True):
    """MAPALN=0: the alignment of query vs profile p from the phase-1
    backtrack codes btck1 ([Lq][Ld], the pair's columns) and the phase-1
    maximum (raw score and its row/column). Returns the same dict fields as
    map_pair (alignment rows, counts, coordinates)."""
    L = lib()
    if not getattr(L, "_aln_bound", False):
        L.orc_aln_pair.restype = ctypes.c_int
        L.orc_aln_pair.argtypes = [ctypes.POINTER(MapIn), ctypes.c_void_p, ctypes.c_longlong,
                                   ctypes.c_float, ctypes.c_uint32, ctypes.POINTER(MapOut)]
        L._aln_bound = True
    p = int(p)
    Lq = query.npositions
    Ld = int(db.lens[p])
    s0 = int(db.starts[p])
    S = np.ascontiguousarray(S, np.float32)
    B = np.ascontiguousarray(btck1, np.uint8)
    qaa = np.ascontiguousarray(query.aa, np.int8)
    daa = np.ascontiguousarray(db.aa[s0:s0 + Ld], np.int8)
    qss = np.ascontiguousarray(query.ssstate, np.int8)
    dss = np.ascontiguousarray(db.ssstate[s0:s0 + Ld], np.int8)
    bufs = [ctypes.create_string_buffer(Lq + Ld + 2) for _ in range(5)]
    mi = MapIn(Lq, Ld, S.ctypes.data, S.ctypes.data, S.shape[1], None, 0, None, 0, 0.0, 0.0, 0,
               qaa.ctypes.data, daa.ctypes.data, qss.ctypes.data, dss.ctypes.data, int(printsss), 1, 1)
    mo = MapOut()
    for i in range(5):
        mo.aln[i] = ctypes.cast(bufs[i], ctypes.c_void_p)
    coords = ((int(maxc) & 0xffff) << 16) | (int(maxr) & 0xffff)
    L.orc_aln_pair(ctypes.byref(mi), B.ctypes.data, B.shape[1], float(maxsc), coords, ctypes.byref(mo))
    return {"aln": [b.value.decode() for b in bufs], "alnlen": mo.alnlen, "idts": mo.idts,
            "psts": mo.psts, "gaps": mo.gaps, "beg": mo.beg, "end": mo.end}


# ---------------------------------------------------------------------------
# the whole search path
def search(query, db, ss_table, db_len, n_seqs, ssswgt=0.12, ddmswgt=0.2, dstsegm=6, minpp=0.28,
           ssemodel=2, xuninf=1, nthreads=1, first_profile=0):
    """The oracle's search of `query` against `db`: score matrix, phase 1,
    statistics with E-values for a database of `db_len` positions and
    `n_seqs` profiles, MAP realignment, and the hits the reference's
    finalizer reports (log E at most the threshold, realigned), sorted by
    log E-value with ties in database order. Returns
    [(profile + first_profile, log E, (5 alignment rows))]."""
    Lq = query.npositions
    sc, ms = score_matrix(query, db, ss_table, ssswgt=ssswgt, ddmswgt=ddmswgt, dstsegm=dstsegm,
                          nthreads=nthreads)
    thld, lthld = score_threshold(Lq, db_len)
    sspace, _ = length_adjustment(Lq, db_len, n_seqs)
    rec, _ = dp1(query, db, sc, 0, 0, db.nprofiles, thld)
    hits = []
    for p in np.nonzero(rec["passed"])[0]:
        s0, Ld = int(db.starts[p]), int(db.lens[p])
        st, _ = pair_statistics(sc[:, s0:s0 + Ld], query.aa, db.aa[s0:s0 + Ld], rec["score"][p],
                                rec["psts"][p], Lq, Ld, query.eno[0], db.eno[p], sspace,
                                ssemodel=ssemodel, xuninf=xuninf)
        logE = float(np.float32(st[2]))
        if logE > lthld:
            continue
        m = map_pair(query, db, p, sc[:, s0:s0 + Ld], ms[:, s0:s0 + Ld], st[3], minpp=minpp,
                     modscores=ssswgt > 0, printsss=ssswgt > 0)
        if m["alnlen"] >= 1:
            hits.append((int(p) + first_profile, logE, tuple(m["aln"])))
    hits.sort(key=lambda h: h[1])   # stable: ties keep database order
    return hits
