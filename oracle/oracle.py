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
    """Compile the oracle (and the reference DDMS restatement when the
    reference tree is present)."""
    args = ["make", "-s", "-C", HERE, "all"]
    if force:
        subprocess.run(["make", "-s", "-C", HERE, "clean"], check=True)
    subprocess.run(args, check=True)
    if os.path.isdir(os.path.join(REFERENCE_TREE, "cother-scores-optimizer")):
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)


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
        sm_args = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_longlong, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_longlong, ctypes.c_longlong,
                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_longlong]
        L.orc_score_matrix.restype = None
        L.orc_score_matrix.argtypes = sm_args
        L.orc_score_matrix_mt.restype = None
        L.orc_score_matrix_mt.argtypes = [ctypes.c_int] + sm_args
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
                ("dstsegm", ctypes.c_int), ("initshift", ctypes.c_float)]


def logf(x: float) -> float:
    return lib().orc_logf(x)


def ddms_cell(qlist: np.ndarray, dlist: np.ndarray, dstsegm: int = 6, ddmswgt: float = 0.2):
    q = np.ascontiguousarray(qlist, dtype=np.uint8)
    d = np.ascontiguousarray(dlist, dtype=np.uint8)
    raw = ctypes.c_float()
    comp = ctypes.c_int()
    s = lib().orc_ddms_cell(q.ctypes.data, d.ctypes.data, dstsegm, ddmswgt,
                            ctypes.byref(raw), ctypes.byref(comp))
    return s, raw.value, comp.value


def score_matrix(query, db, ss_table, ssswgt=0.12, ddmswgt=0.2, dstsegm=6, initshift=0.002,
                 col0=0, ncols=None, nthreads=1):
    """(scores, modscores) [Lq][ncols] for query vs db columns [col0, col0+ncols)."""
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
    lib().orc_score_matrix_mt(int(nthreads), Lq, q_tf.ctypes.data, q_bkg.ctypes.data,
                              q_ss.ctypes.data, q_dd.ctypes.data, N, P, d_tf.ctypes.data,
                              d_bkg.ctypes.data, d_pro.ctypes.data, d_ss.ctypes.data,
                              d_dd.ctypes.data, T.ctypes.data, ctypes.byref(prm),
                              int(col0), int(ncols), sc.ctypes.data, ms.ctypes.data, int(ncols))
    return sc, ms
