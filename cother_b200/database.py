"""Binary profile database files (the reference's db2bin format v2.2)
through the C ABI: write a profile set with its descriptions, open a file,
and hand chunks of it to a search context (cbp_db_*)."""
from __future__ import annotations

import ctypes

import numpy as np

from . import CbpError, load_library
from .profiles import NFIELDS


def _check(L, rc):
    if rc != 0:
        raise CbpError(rc, L.cbp_last_error().decode(errors="replace"))


def write_database(path: str, profiles, descs=None) -> None:
    """Write a ProfileSet (and one description per profile) to `path`."""
    L = load_library()
    beg, end = profiles.field_tables()
    keep = []
    d = None
    if descs is not None:
        if len(descs) != profiles.nprofiles:
            raise ValueError("one description per profile")
        arr = (ctypes.c_char_p * len(descs))()
        for i, x in enumerate(descs):
            b = x.encode() if isinstance(x, str) else bytes(x)
            keep.append(b)
            arr[i] = b
        d = arr
    _check(L, L.cbp_db_write(path.encode(), beg, end, d))


class Database:
    """An opened database file; chunks stay valid until the next chunk()."""

    def __init__(self, path: str):
        L = load_library()
        h = ctypes.c_void_p()
        _check(L, L.cbp_db_open(path.encode(), ctypes.byref(h)))
        self._h = h
        n, npos, ndst = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        _check(L, L.cbp_db_info(self._h, ctypes.byref(n), ctypes.byref(npos), ctypes.byref(ndst)))
        self.nprofiles, self.npositions, self.ndistances = n.value, npos.value, ndst.value
        self._beg = (ctypes.c_void_p * NFIELDS)()
        self._end = (ctypes.c_void_p * NFIELDS)()

    def close(self) -> None:
        if getattr(self, "_h", None):
            load_library().cbp_db_close(self._h)
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

    def lengths(self) -> np.ndarray:
        L = load_library()
        out = np.zeros(self.nprofiles, np.int32)
        _check(L, L.cbp_db_profile_lengths(self._h, out.ctypes.data))
        return out

    def chunk(self, first: int, count: int):
        """(beg, end, descriptions) of profiles first .. first+count-1."""
        L = load_library()
        d = (ctypes.c_char_p * max(1, count))()
        _check(L, L.cbp_db_chunk(self._h, first, count, self._beg, self._end, d))
        return self._beg, self._end, [d[i].decode("latin-1") for i in range(count)]

    def field(self, f: int, dtype=np.float32) -> np.ndarray:
        """A copy of field f of the current chunk."""
        b, e = self._beg[f], self._end[f]
        n = (e - b) // np.dtype(dtype).itemsize
        return np.ctypeslib.as_array((ctypes.c_char * (e - b)).from_address(b)).view(dtype)[:n].copy()

    def chunks(self, max_positions: int):
        """Ranges (first, count) of whole profiles of at most max_positions
        positions each (a profile longer than that is a chunk of its own),
        in database order."""
        lens = self.lengths()
        out, first, acc = [], 0, 0
        for k, n in enumerate(lens.tolist()):
            if k > first and acc + n > max_positions:
                out.append((first, k - first))
                first, acc = k, 0
            acc += n
        out.append((first, len(lens) - first))
        return out
