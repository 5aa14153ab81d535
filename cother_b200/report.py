"""Text output of search results through the C ABI: the finalizer's
per-hit text (cbp_format_hits / cbp_format_hits_host), the stable merge of
a query's hit lists over database chunks (cbp_merge_hit_lists) and the
per-query report (cbp_write_report), in the reference's plain and JSON
layouts (src/libmycu/cupro/CuBatchProcessingFinalizerPlain.cpp,
CuBatchProcessingFinalizerJSON.cpp, src/libmycu/cualn/AlnWriter*.cpp)."""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import CbpError, load_library

PLAIN = 0
JSON = 1


class FormatOptions(ctypes.Structure):
    _fields_ = [("format", ctypes.c_int), ("dsclen", ctypes.c_int), ("dscwidth", ctypes.c_int),
                ("alnwidth", ctypes.c_int), ("show", ctypes.c_int)]

    @classmethod
    def defaults(cls, fmt: int = PLAIN) -> "FormatOptions":
        o = cls()
        load_library().cbp_default_format_options(ctypes.byref(o))
        o.format = fmt
        return o


class HitsInput(ctypes.Structure):
    _fields_ = [("recs", ctypes.c_void_p), ("nrecs", ctypes.c_size_t), ("rows", ctypes.c_void_p),
                ("row_stride", ctypes.c_size_t), ("row_length", ctypes.c_size_t),
                ("prof_len", ctypes.c_void_p), ("prof_eno", ctypes.c_void_p), ("prof_ss", ctypes.c_void_p),
                ("nprof", ctypes.c_size_t), ("descs", ctypes.c_void_p), ("query_len", ctypes.c_int),
                ("query_eno", ctypes.c_float), ("query_ss", ctypes.c_int), ("ssswgt", ctypes.c_float),
                ("log_evalue_threshold", ctypes.c_float), ("search_space", ctypes.c_float)]


class ReportInfo(ctypes.Structure):
    _fields_ = [("program", ctypes.c_char_p), ("version", ctypes.c_char_p), ("references", ctypes.c_void_p),
                ("query_len", ctypes.c_int), ("query_desc", ctypes.c_char_p), ("db_names", ctypes.c_void_p),
                ("n_db_names", ctypes.c_size_t), ("db_size", ctypes.c_uint64), ("db_entries", ctypes.c_uint64),
                ("log_evalue_threshold", ctypes.c_float), ("search_space", ctypes.c_float),
                ("delta_length", ctypes.c_int), ("ref_lambda", ctypes.c_float), ("ref_k", ctypes.c_float),
                ("gapped_lambda", ctypes.c_float), ("gapped_k", ctypes.c_float), ("nohits", ctypes.c_int),
                ("noalns", ctypes.c_int)]


def _cstrings(strs, keep):
    """NULL-terminated char* array (None entries stay NULL)."""
    if strs is None:
        return None
    arr = (ctypes.c_char_p * (len(strs) + 1))()
    for i, x in enumerate(strs):
        if x is not None:
            b = x.encode() if isinstance(x, str) else bytes(x)
            keep.append(b)
            arr[i] = b
    arr[len(strs)] = None
    keep.append(arr)
    return ctypes.cast(arr, ctypes.c_void_p)


def _check(L, rc):
    if rc != 0:
        raise CbpError(rc, L.cbp_last_error().decode(errors="replace"))


def _split(buf: bytes, n: int):
    parts = buf.split(b"\0")
    if len(parts) < 2 * n:
        raise CbpError(-1, "malformed hit text")
    return [(parts[2 * i].decode("latin-1"), parts[2 * i + 1].decode("latin-1")) for i in range(n)]


def format_hits_ctx(handle, descs=None, options=None):
    L = load_library()
    fo = options or FormatOptions.defaults()
    keep = []
    d = _cstrings(descs, keep)
    used, n = ctypes.c_size_t(0), ctypes.c_size_t(0)
    _check(L, L.cbp_format_hits(handle, ctypes.byref(fo), d, None, 0, ctypes.byref(used), ctypes.byref(n)))
    buf = ctypes.create_string_buffer(max(1, used.value))
    _check(L, L.cbp_format_hits(handle, ctypes.byref(fo), d, buf, used.value, ctypes.byref(used),
                                ctypes.byref(n)))
    return _split(buf.raw[:used.value], n.value)


def format_hits_host(recs: np.ndarray, rows: np.ndarray, prof_len, prof_eno, query_len: int,
                     query_eno: float, log_evalue_threshold: float, search_space: float,
                     ssswgt: float = 0.12, descs=None, prof_ss=None, query_ss: bool = True,
                     options=None):
    """Per-hit text from host records ([n][18] float32) and the 5 alignment
    rows ([5][len] uint8), without a context (cbp_format_hits_host)."""
    L = load_library()
    fo = options or FormatOptions.defaults()
    keep = []
    recs = np.ascontiguousarray(recs, np.float32).reshape(-1, 18)
    rows = np.ascontiguousarray(rows, np.uint8)
    plen = np.ascontiguousarray(prof_len, np.int32)
    peno = np.ascontiguousarray(prof_eno, np.float32)
    pss = None if prof_ss is None else np.ascontiguousarray(prof_ss, np.uint8)
    hi = HitsInput()
    hi.recs = recs.ctypes.data
    hi.nrecs = recs.shape[0]
    hi.rows = rows.ctypes.data
    hi.row_stride = rows.shape[1]
    hi.row_length = rows.shape[1]
    hi.prof_len = plen.ctypes.data
    hi.prof_eno = peno.ctypes.data
    hi.prof_ss = None if pss is None else pss.ctypes.data
    hi.nprof = plen.shape[0]
    hi.descs = _cstrings(descs, keep)
    hi.query_len = int(query_len)
    hi.query_eno = float(query_eno)
    hi.query_ss = 1 if query_ss else 0
    hi.ssswgt = float(ssswgt)
    hi.log_evalue_threshold = float(log_evalue_threshold)
    hi.search_space = float(search_space)
    used, n = ctypes.c_size_t(0), ctypes.c_size_t(0)
    _check(L, L.cbp_format_hits_host(ctypes.byref(hi), ctypes.byref(fo), None, 0, ctypes.byref(used),
                                     ctypes.byref(n)))
    buf = ctypes.create_string_buffer(max(1, used.value))
    _check(L, L.cbp_format_hits_host(ctypes.byref(hi), ctypes.byref(fo), buf, used.value, ctypes.byref(used),
                                     ctypes.byref(n)))
    return _split(buf.raw[:used.value], n.value)


def merge_hit_lists(log_evalues):
    """Stable merge of per-chunk sorted hit lists by log E-value: a list of
    (part, index) pairs (cbp_merge_hit_lists)."""
    L = load_library()
    parts = [np.ascontiguousarray(x, np.float32) for x in log_evalues]
    ptrs = (ctypes.c_void_p * max(1, len(parts)))(*[p.ctypes.data for p in parts])
    counts = (ctypes.c_size_t * max(1, len(parts)))(*[p.size for p in parts])
    total = sum(p.size for p in parts)
    part = np.zeros(max(1, total), np.int32)
    index = np.zeros(max(1, total), np.int32)
    _check(L, L.cbp_merge_hit_lists(len(parts), ptrs, counts, part.ctypes.data, index.ctypes.data))
    return list(zip(part[:total].tolist(), index[:total].tolist()))


def write_report(hits, query_len: int, db_size: int, db_entries: int, log_evalue_threshold: float,
                 search_space: float, delta_length: int, query_desc: str | None = None,
                 db_names=(), program: str | None = None, version: str | None = None,
                 references=None, ref_lambda: float = 1.116276, ref_k: float = 0.115812,
                 gapped_lambda: float = 0.561132, gapped_k: float = 0.001488,
                 nohits: int = 700, noalns: int = 700, options=None) -> str:
    """One query's report from its merged hits [(annotation, record), ...]
    (cbp_write_report)."""
    L = load_library()
    fo = options or FormatOptions.defaults()
    keep = []
    ri = ReportInfo()
    ri.program = program.encode() if program is not None else None
    ri.version = version.encode() if version is not None else None
    ri.references = _cstrings(references, keep)
    ri.query_len = int(query_len)
    ri.query_desc = query_desc.encode() if query_desc is not None else None
    ri.db_names = _cstrings(list(db_names), keep)
    ri.n_db_names = len(db_names)
    ri.db_size = int(db_size)
    ri.db_entries = int(db_entries)
    ri.log_evalue_threshold = float(log_evalue_threshold)
    ri.search_space = float(search_space)
    ri.delta_length = int(delta_length)
    ri.ref_lambda, ri.ref_k = float(ref_lambda), float(ref_k)
    ri.gapped_lambda, ri.gapped_k = float(gapped_lambda), float(gapped_k)
    ri.nohits, ri.noalns = int(nohits), int(noalns)
    ann = _cstrings([h[0] for h in hits], keep)
    rec = _cstrings([h[1] for h in hits], keep)
    used = ctypes.c_size_t(0)
    _check(L, L.cbp_write_report(ctypes.byref(ri), ctypes.byref(fo), ann, rec, len(hits), None, 0,
                                 ctypes.byref(used)))
    buf = ctypes.create_string_buffer(max(1, used.value))
    _check(L, L.cbp_write_report(ctypes.byref(ri), ctypes.byref(fo), ann, rec, len(hits), buf, used.value,
                                 ctypes.byref(used)))
    return buf.raw[:used.value].decode("latin-1")


def output_filename(outdir: str, query_name: str, query_serial: int, fmt: int = PLAIN) -> str:
    """Name of a query's output file (AlnWriter::GetOutputFilename,
    src/libmycu/cualn/AlnWriter.cpp:357-375): the query file's base name
    without an extension of at most 3 characters, "__<serial>", and .out or
    .json."""
    ext = "json" if fmt == JSON else "out"
    name = outdir
    if name and not name.endswith(os.sep):
        name += os.sep
    qn = os.path.basename(query_name)
    pos = qn.rfind(".")
    if pos >= 0 and len(qn) - pos <= 4:
        qn = qn[:pos]
    return name + qn + "__%d.%s" % (query_serial, ext)
