"""cother_b200 -- B200-native search path of COTHER.

The search path (score matrix, phase-1 DP, statistics, MAP realignment,
hit records) runs in ``libcother_b200.so``: hand-written sm_100a CUDA
kernels behind the C ABI declared in ``include/cother_b200.h``. This module
binds that ABI with ctypes and mirrors the reference's per-worker driver
interface (``CuBatchProcessing``, src/libmycu/cupro/CuBatchProcessing.cuh:47-244)
as :class:`BatchProcessing`.

There is no CPU fallback: if the library cannot be loaded, or no GPU is
present, the calls raise.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import build as _build

__all__ = ["Options", "BatchProcessing", "CbpError", "load_library", "LIB_PATH"]

LIB_PATH = _build.LIB_MAIN

_lib = None


class CbpError(RuntimeError):
    """A failure reported by the native library (status code + message)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


TC_PLAIN, TC_BF16X3, TC_TF32X3 = 0, 1, 2   # Options.tc_form


class Options(ctypes.Structure):
    """Path options (``cbp_options``; MOptions of the reference)."""

    _fields_ = [
        ("ssswgt", ctypes.c_float), ("cvswgt", ctypes.c_float), ("ddmswgt", ctypes.c_float),
        ("dstsegm", ctypes.c_int), ("mapaln", ctypes.c_int), ("minpp", ctypes.c_float),
        ("ssemodel", ctypes.c_int), ("x_uninf", ctypes.c_int), ("eval", ctypes.c_float),
        ("nohits", ctypes.c_int), ("noalns", ctypes.c_int), ("tc_form", ctypes.c_int),
        ("autotune", ctypes.c_int), ("all_codes", ctypes.c_int),
    ]

    @classmethod
    def defaults(cls) -> "Options":
        o = cls()
        load_library().cbp_default_options(ctypes.byref(o))
        return o


def load_library(path: str | None = None):
    """Load (and bind) the native library; raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise CbpError(-1, f"native library not built: {path} (run __graft_entry__.build())")
    L = ctypes.CDLL(path)
    vp, sz, i32, f32 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_float
    sig = {
        "cbp_default_options": (None, [vp]),
        "cbp_last_error": (ctypes.c_char_p, []),
        "cbp_create": (i32, [i32, vp, vp, sz, ctypes.POINTER(vp)]),
        "cbp_destroy": (i32, [vp]),
        "cbp_set_db_details": (i32, [vp, ctypes.c_uint64, sz]),
        "cbp_set_query_len": (i32, [vp, sz]),
        "cbp_set_score_threshold": (i32, [vp, f32]),
        "cbp_set_logE_threshold": (i32, [vp, f32]),
        "cbp_set_cvs2s_map": (i32, [vp, vp, vp, sz]),
        "cbp_read_statistics": (i32, [vp, vp, sz, ctypes.POINTER(sz)]),
        "cbp_get_capacities": (i32, [vp, sz, sz] + [ctypes.POINTER(sz)] * 4),
        "cbp_transfer_chunk": (i32, [vp, vp, vp, vp]),
        "cbp_process": (i32, [vp, i32, sz, vp, vp]),
        "cbp_process_batch": (i32, [vp, sz, vp, vp, vp]),
        "cbp_ledger_choose": (i32, [vp, vp, sz, sz, sz, sz, ctypes.POINTER(sz)]),
        "cbp_server_default_config": (None, [vp]),
        "cbp_server_create": (i32, [vp, vp, vp, vp, vp, ctypes.POINTER(vp)]),
        "cbp_server_budget": (i32, [vp, ctypes.POINTER(sz)]),
        "cbp_server_submit": (i32, [vp, sz, vp, vp, ctypes.POINTER(ctypes.c_uint64)]),
        "cbp_server_wait": (i32, [vp, ctypes.c_uint64, i32, vp]),
        "cbp_server_get": (i32, [vp, ctypes.c_uint64, vp, sz, vp, sz, vp, sz]),
        "cbp_server_release": (i32, [vp, ctypes.c_uint64]),
        "cbp_server_destroy": (i32, [vp]),
        "cbp_server_last_error": (ctypes.c_char_p, []),
        "cbp_select_query": (i32, [vp, sz, ctypes.POINTER(sz)]),
        "cbp_wait_idle": (i32, [vp]),
        "cbp_read_score_matrix": (i32, [vp, vp, vp, sz, ctypes.POINTER(sz), ctypes.POINTER(sz)]),
        "cbp_set_max_slab_positions": (i32, [vp, sz]),
        "cbp_read_phase1": (i32, [vp, vp, vp, vp, vp, vp, sz, ctypes.POINTER(sz), vp,
                                  ctypes.POINTER(sz)]),
        "cbp_read_btck": (i32, [vp, vp, sz]),
        "cbp_read_slab_columns": (i32, [vp, sz, sz, vp, vp, vp, sz]),
        "cbp_read_map_fb": (i32, [vp, sz, vp, sz, ctypes.POINTER(sz)]),
        "cbp_read_fits": (i32, [vp, vp, sz, ctypes.POINTER(sz)]),
        "cbp_score_threshold": (None, [sz, ctypes.c_uint64, f32, f32, f32, ctypes.POINTER(f32),
                                       ctypes.POINTER(f32)]),
        "cbp_get_hit_records": (i32, [vp, vp, sz, ctypes.POINTER(sz)]),
        "cbp_get_search_space": (i32, [vp, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(sz)]),
        "cbp_get_alignments": (i32, [vp, vp, sz, ctypes.POINTER(sz)]),
        "cbp_get_hit_list": (i32, [vp, vp, sz, ctypes.POINTER(sz)]),
        "cbp_share_database": (i32, [vp, vp]),
        "cbp_device_memory": (i32, [i32, ctypes.POINTER(sz), ctypes.POINTER(sz)]),
        "cbp_slab_bytes": (i32, [vp, sz, sz, ctypes.POINTER(sz)]),
        "cbp_dp1_noalloc": (i32, [vp, sz, i32, vp, ctypes.c_longlong, i32, vp, vp, vp, i32, i32,
                                  ctypes.c_longlong, vp, vp, vp, vp]),
        "cbp_set_karlin_altschul": (i32, [vp, f32, f32, f32, f32, f32, f32]),
        "cbp_stage_times": (i32, [vp, vp, i32]),
        "cbp_launch_count": (i32, [vp, ctypes.POINTER(ctypes.c_uint64)]),
        "cbp_stage_launches": (i32, [vp, vp, i32]),
        "cbp_default_format_options": (None, [vp]),
        "cbp_format_hits": (i32, [vp, vp, vp, vp, sz, ctypes.POINTER(sz), ctypes.POINTER(sz)]),
        "cbp_format_hits_host": (i32, [vp, vp, vp, sz, ctypes.POINTER(sz), ctypes.POINTER(sz)]),
        "cbp_merge_hit_lists": (i32, [sz, vp, vp, vp, vp]),
        "cbp_write_report": (i32, [vp, vp, vp, vp, sz, vp, sz, ctypes.POINTER(sz)]),
        "cbp_get_tuning": (i32, [vp, sz, ctypes.POINTER(i32), ctypes.POINTER(i32), ctypes.POINTER(i32), vp, i32]),
        "cbp_set_kernels": (i32, [vp, sz, i32, i32, i32]),
        "cbp_graph_launches": (i32, [vp, ctypes.POINTER(ctypes.c_uint64)]),
        "cbp_db_open": (i32, [ctypes.c_char_p, ctypes.POINTER(vp)]),
        "cbp_db_close": (i32, [vp]),
        "cbp_db_info": (i32, [vp] + [ctypes.POINTER(ctypes.c_uint64)] * 3),
        "cbp_db_profile_lengths": (i32, [vp, vp]),
        "cbp_db_chunk": (i32, [vp, ctypes.c_uint64, ctypes.c_uint64, vp, vp, vp]),
        "cbp_db_write": (i32, [ctypes.c_char_p, vp, vp, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


# gapped Karlin-Altschul parameters of the reference's statistical
# configuration (src/env/cother.par, section [GAPPED_A_1])
GAPPED_LAMBDA = 0.561132
GAPPED_K = 0.001488


def score_threshold(query_len: int, db_len: int, evalue: float = 10.0,
                    lam: float = GAPPED_LAMBDA, K: float = GAPPED_K):
    """(score threshold, log E-value threshold) as the reference's job
    dispatcher derives them (cbp_score_threshold)."""
    a, b = ctypes.c_float(), ctypes.c_float()
    load_library().cbp_score_threshold(int(query_len), int(db_len), float(evalue), float(lam),
                                       float(K), ctypes.byref(a), ctypes.byref(b))
    return a.value, b.value


REC_FLOATS = 18
REC_FIELDS = ["score", "org_pro_no", "pro_new_dst", "psts", "beg_coords", "end_coords",
              "lambda_est", "K_est", "log_evalue", "log_evalue_pair", "min", "max", "expected",
              "entropy", "lambda", "K", "identities", "gaps"]
_REC_UINT = {"org_pro_no", "pro_new_dst", "beg_coords", "end_coords"}


def device_memory(device: int = 0):
    """(free, total) device memory in bytes."""
    f, t = ctypes.c_size_t(), ctypes.c_size_t()
    _check(load_library().cbp_device_memory(int(device), ctypes.byref(f), ctypes.byref(t)))
    return int(f.value), int(t.value)


def slab_bytes(query_len: int, positions: int, options: "Options | None" = None) -> int:
    """Working device memory of one slab of `positions` database positions
    for a query of `query_len` positions (what the slab planner charges)."""
    o = options if options is not None else Options.defaults()
    n = ctypes.c_size_t()
    _check(load_library().cbp_slab_bytes(ctypes.byref(o), int(query_len), int(positions),
                                         ctypes.byref(n)))
    return int(n.value)


def alignments_from(recs: np.ndarray, rows: np.ndarray, query_len: int, db_lens) -> list:
    """Per record: its alignment rows (query, middle, target, query SS,
    target SS) as strings, or None when it was not realigned. `rows` are the
    5 alignment rows of a search; the pair of record k ends its slot at
    newDst + Ld - 1 + (k+1) Lq (the finalizer's layout,
    src/libmycu/cupro/CuBatchProcessingFinalizerPlain.cpp:252-256)."""
    t = records_table(recs)
    out = []
    alnlen = t["log_evalue_pair"].view(np.int32)
    for k in range(len(t["score"])):
        n = int(alnlen[k])
        if n <= 0:
            out.append(None)
            continue
        p = int(t["org_pro_no"][k])
        Ld = int(db_lens[p])
        term = int(t["pro_new_dst"][k]) + k * query_len + Ld + query_len - 1
        out.append(tuple(bytes(rows[r, term - n:term]).decode() for r in range(5)))
    return out


def records_table(recs: np.ndarray) -> dict:
    """Named columns of hit records; integer fields decoded from their bits."""
    out = {}
    for i, name in enumerate(REC_FIELDS):
        col = np.ascontiguousarray(recs[:, i])
        out[name] = col.view(np.uint32).copy() if name in _REC_UINT else col.copy()
    return out


def _check(rc: int) -> None:
    if rc != 0:
        msg = load_library().cbp_last_error()
        raise CbpError(rc, msg.decode() if msg else "")


class BatchProcessing:
    """One search context on one GPU (the reference's CuBatchProcessing).

    Method names follow the reference's (TransferCPMData, SetDbDetails,
    ProcessScoreMatrix ...) in Python style.
    """

    def __init__(self, ss_table: np.ndarray, options: Options | None = None, device: int = 0,
                 dev_mem_bytes: int = 0):
        L = load_library()
        self._opt = options or Options.defaults()
        self._ss = np.ascontiguousarray(ss_table, dtype=np.float32)
        if self._ss.shape != (30, 30):
            raise ValueError("ss_table must be 30x30")
        h = ctypes.c_void_p()
        _check(L.cbp_create(device, ctypes.byref(self._opt), self._ss.ctypes.data, dev_mem_bytes,
                            ctypes.byref(h)))
        self._h = h
        self._db = None

    def close(self) -> None:
        if getattr(self, "_h", None):
            load_library().cbp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # --- settings (CuBatchProcessing::Set*) ---
    def set_db_details(self, db_len: int, n_seqs: int) -> None:
        _check(load_library().cbp_set_db_details(self._h, int(db_len), int(n_seqs)))

    def set_query_len(self, qlen: int) -> None:
        _check(load_library().cbp_set_query_len(self._h, int(qlen)))

    def set_score_threshold(self, t: float) -> None:
        _check(load_library().cbp_set_score_threshold(self._h, float(t)))

    def set_logE_threshold(self, t: float) -> None:
        _check(load_library().cbp_set_logE_threshold(self._h, float(t)))

    def capacities(self, query_len: int, expected_profile_length: int = 250) -> dict:
        """Chunk capacities for a query length (GetCurrentMaxDbPos and the
        like): max_db_pos, max_db_pros, max_pass2_pos, max_pass2_pros."""
        out = [ctypes.c_size_t() for _ in range(4)]
        _check(load_library().cbp_get_capacities(self._h, int(query_len), int(expected_profile_length),
                                                  *[ctypes.byref(x) for x in out]))
        return dict(zip(("max_db_pos", "max_db_pros", "max_pass2_pos", "max_pass2_pros"),
                        (x.value for x in out)))

    def set_cvs2s_map(self, keys, scores) -> None:
        """The context-vector score map, needed when CVSWGT > 0: keys on the
        grid of halves and their scores, as the reference's CVS2Scores
        reader leaves them (smoothed)."""
        k = np.ascontiguousarray(keys, np.float32)
        v = np.ascontiguousarray(scores, np.float32)
        if k.shape != v.shape or k.ndim != 1:
            raise ValueError("keys and scores must be 1-D arrays of equal length")
        _check(load_library().cbp_set_cvs2s_map(self._h, k.ctypes.data, v.ctypes.data, len(k)))

    def set_max_slab_positions(self, n: int) -> None:
        _check(load_library().cbp_set_max_slab_positions(self._h, int(n)))

    # --- data and processing ---
    def transfer_cpm_data(self, db) -> None:
        """Upload a database chunk (a ProfileSet) and keep it resident."""
        beg, end = db.field_tables()
        _check(load_library().cbp_transfer_chunk(self._h, beg, end, None))
        self._db = db

    def transfer_db_chunk(self, database, first: int, count: int):
        """Transfer profiles first .. first+count-1 of an opened database
        file (cother_b200.database.Database); returns their descriptions."""
        beg, end, descs = database.chunk(first, count)
        _check(load_library().cbp_transfer_chunk(self._h, beg, end, None))
        return descs

    def share_database(self, owner: "BatchProcessing") -> None:
        """Search `owner`'s resident database (same device) without a copy."""
        _check(load_library().cbp_share_database(self._h, owner._h))
        self._db = owner._db

    def process_score_matrix(self, query, query_serial: int = 0) -> None:
        """Search one query profile against the resident chunk."""
        beg, end = query.field_tables()
        _check(load_library().cbp_process(self._h, int(query_serial), int(query.npositions), beg, end))

    def process_batch(self, queries) -> None:
        """Search several query profiles in one pass over the resident chunk
        (cbp_process_batch); select_query(k) picks whose results the result
        calls return (query 0 after the call)."""
        n = len(queries)
        tables = [q.field_tables() for q in queries]
        lens = (ctypes.c_size_t * n)(*[q.npositions for q in queries])
        beg = (ctypes.c_void_p * n)(*[ctypes.cast(t[0], ctypes.c_void_p) for t in tables])
        end = (ctypes.c_void_p * n)(*[ctypes.cast(t[1], ctypes.c_void_p) for t in tables])
        _check(load_library().cbp_process_batch(self._h, n, lens, beg, end))
        self._batch = list(queries)

    def select_query(self, k: int) -> int:
        """Results of query k of the last call from now on; returns the
        call's number of queries (cbp_select_query)."""
        n = ctypes.c_size_t()
        _check(load_library().cbp_select_query(self._h, int(k), ctypes.byref(n)))
        return n.value

    def wait_idle(self) -> None:
        _check(load_library().cbp_wait_idle(self._h))

    # --- inspection ---
    def read_score_matrix(self, nrows: int, max_cols: int):
        """(scores, modscores, first_profile) of the last processed slab."""
        sc = np.zeros((nrows, max_cols), np.float32)
        ms = np.zeros((nrows, max_cols), np.float32)
        ncols = ctypes.c_size_t()
        first = ctypes.c_size_t()
        _check(load_library().cbp_read_score_matrix(self._h, sc.ctypes.data, ms.ctypes.data, max_cols,
                                                     ctypes.byref(ncols), ctypes.byref(first)))
        n = ncols.value
        return sc[:, :n], ms[:, :n], first.value

    def read_statistics(self) -> np.ndarray:
        """Hit records [npass][CBP_REC_FLOATS] of the last slab as the
        statistics stage leaves them (before the phase-2 finalizer)."""
        L = load_library()
        n = ctypes.c_size_t()
        _check(L.cbp_read_statistics(self._h, None, 0, ctypes.byref(n)))
        out = np.zeros((n.value, REC_FLOATS), np.float32)
        if n.value:
            _check(L.cbp_read_statistics(self._h, out.ctypes.data, n.value, ctypes.byref(n)))
        return out

    def read_fits(self) -> np.ndarray:
        """The precision forms: per passed pair of the last slab, the
        parameter fit in FP64 and in FP32, float64 [npass][8] (lambda, K, H,
        expected score of each; cbp_read_fits)."""
        L = load_library()
        n = ctypes.c_size_t()
        _check(L.cbp_read_fits(self._h, None, 0, ctypes.byref(n)))
        out = np.zeros((n.value, 8), np.float64)
        if n.value:
            _check(L.cbp_read_fits(self._h, out.ctypes.data, n.value, ctypes.byref(n)))
        return out

    def read_phase1(self):
        """Phase-1 records of the last slab: dict of arrays (score, psts,
        beg, end, passed) and the pass list."""
        n = self._db.nprofiles if self._db is not None else 0
        score = np.zeros(n, np.float32)
        psts = np.zeros(n, np.float32)
        beg = np.zeros(n, np.uint32)
        end = np.zeros(n, np.uint32)
        passed = np.zeros(n, np.int32)
        plist = np.zeros(n, np.int32)
        nprof, npass = ctypes.c_size_t(), ctypes.c_size_t()
        _check(load_library().cbp_read_phase1(self._h, score.ctypes.data, psts.ctypes.data,
                                               beg.ctypes.data, end.ctypes.data, passed.ctypes.data,
                                               n, ctypes.byref(nprof), plist.ctypes.data,
                                               ctypes.byref(npass)))
        k = nprof.value
        return ({"score": score[:k], "psts": psts[:k], "beg": beg[:k], "end": end[:k],
                 "passed": passed[:k]}, plist[:npass.value])

    def hit_records(self) -> np.ndarray:
        """Hit records of the last search: float32 [n][18] (CBP_REC_FLOATS);
        use :func:`records_table` for named fields."""
        L = load_library()
        n = ctypes.c_size_t()
        _check(L.cbp_get_hit_records(self._h, None, 0, ctypes.byref(n)))
        out = np.zeros((n.value, REC_FLOATS), np.float32)
        if n.value:
            _check(L.cbp_get_hit_records(self._h, out.ctypes.data, n.value, ctypes.byref(n)))
        return out

    def alignment_rows(self) -> np.ndarray:
        """The 5 alignment rows of the last search (uint8 [5][length])."""
        L = load_library()
        n = ctypes.c_size_t()
        _check(L.cbp_get_alignments(self._h, None, 0, ctypes.byref(n)))
        rows = np.zeros((5, max(n.value, 1)), np.uint8)
        if n.value:
            _check(L.cbp_get_alignments(self._h, rows.ctypes.data, rows.shape[1], ctypes.byref(n)))
        return rows[:, :n.value]

    def alignments(self, query_len: int):
        """Per hit: (query, middle, target, query SS, target SS) strings, or
        None for hits that were not realigned."""
        return alignments_from(self.hit_records(), self.alignment_rows(), query_len, self._db.lens)

    def hit_list(self, top: int | None = None) -> np.ndarray:
        """Record indices of the reported hits of the last search (log E at
        most the threshold, realigned), sorted by log E-value on the device:
        the order of the reference's finalizer. With `top`, only the first
        `top` (the top-k hits)."""
        L = load_library()
        n = ctypes.c_size_t()
        _check(L.cbp_get_hit_list(self._h, None, 0, ctypes.byref(n)))
        k = n.value if top is None else min(int(top), n.value)
        out = np.zeros(k, np.int32)
        if k:
            _check(L.cbp_get_hit_list(self._h, out.ctypes.data, k, ctypes.byref(n)))
        return out

    def search_space(self):
        ss, dl = ctypes.c_uint64(), ctypes.c_size_t()
        _check(load_library().cbp_get_search_space(self._h, ctypes.byref(ss), ctypes.byref(dl)))
        return int(ss.value), int(dl.value)

    def set_karlin_altschul(self, ungapped_lambda, ungapped_k, gapped_lambda, gapped_k,
                            gapped_alpha=0.5, gapped_beta=-1.0) -> None:
        _check(load_library().cbp_set_karlin_altschul(self._h, ungapped_lambda, ungapped_k,
                                                       gapped_lambda, gapped_k, gapped_alpha,
                                                       gapped_beta))

    def read_btck(self, nrows: int, max_cols: int):
        b = np.zeros((nrows, max_cols), np.uint8)
        _check(load_library().cbp_read_btck(self._h, b.ctypes.data, max_cols))
        return b

    def read_slab_columns(self, nrows: int, first_col: int, ncols: int):
        """(scores, modscores, btck) of slab columns [first_col,
        first_col + ncols) of the last slab (cbp_read_slab_columns)."""
        sc = np.zeros((nrows, max(ncols, 1)), np.float32)
        ms = np.zeros((nrows, max(ncols, 1)), np.float32)
        bt = np.zeros((nrows, max(ncols, 1)), np.uint8)
        _check(load_library().cbp_read_slab_columns(self._h, int(first_col), int(ncols), sc.ctypes.data,
                                                     ms.ctypes.data, bt.ctypes.data, sc.shape[1]))
        return sc[:, :ncols], ms[:, :ncols], bt[:, :ncols]

    def map_fb(self, pair: int, nrows: int) -> np.ndarray:
        """The MAP stage's forward + backward log match-state values of pair
        `pair` of the last slab's pass list, [nrows][profile length]
        (cbp_read_map_fb)."""
        L = load_library()
        n = ctypes.c_size_t()
        _check(L.cbp_read_map_fb(self._h, int(pair), None, 0, ctypes.byref(n)))
        fb = np.zeros((nrows, max(1, n.value)), np.float32)
        _check(L.cbp_read_map_fb(self._h, int(pair), fb.ctypes.data, fb.shape[1], ctypes.byref(n)))
        return fb[:, :n.value]

    def format_hits(self, descs=None, options=None):
        """Per-hit text of the last search in the finalizer's order: a list
        of (annotation, hit record) strings (cbp_format_hits)."""
        from . import report
        return report.format_hits_ctx(self._h, descs, options)

    def tuning(self, query_len: int) -> dict:
        """The kernel variants in use for this query length and the tuned
        candidates' sample times (cbp_get_tuning)."""
        L = load_library()
        r, w, d = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        ms = np.zeros(7, np.float32)
        _check(L.cbp_get_tuning(self._h, int(query_len), ctypes.byref(r), ctypes.byref(w), ctypes.byref(d),
                                ms.ctypes.data, 7))
        return {"score_rows": r.value, "order_window": w.value, "dp_warps": d.value,
                "score_candidates_ms": ms[:5].tolist(), "dp_candidates_ms": ms[5:].tolist()}

    def set_kernels(self, query_len: int, rows: int, window: int, dp_warps: int) -> None:
        """Fix the kernel variants for this query length (cbp_set_kernels)."""
        _check(load_library().cbp_set_kernels(self._h, int(query_len), rows, window, dp_warps))

    def graph_launches(self) -> int:
        """CUDA-graph launches of this context so far (cbp_graph_launches)."""
        n = ctypes.c_uint64()
        _check(load_library().cbp_graph_launches(self._h, ctypes.byref(n)))
        return n.value

    def stage_times(self) -> list:
        buf = (ctypes.c_float * 6)()
        n = load_library().cbp_stage_times(self._h, buf, 6)
        return [buf[i] for i in range(n)]

    def stage_launches(self) -> list:
        buf = (ctypes.c_uint64 * 6)()
        n = load_library().cbp_stage_launches(self._h, buf, 6)
        return [int(buf[i]) for i in range(n)]

    def launch_count(self) -> int:
        v = ctypes.c_uint64()
        _check(load_library().cbp_launch_count(self._h, ctypes.byref(v)))
        return int(v.value)
