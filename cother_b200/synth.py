"""Seeded synthetic query and database profiles.

The workloads stand in for real profile databases (none can be downloaded
here). Shapes and value distributions follow the benchmark configurations
of the search path:

* query profiles carry *predicted* C-beta distance distributions (17 bins
  over 2-20 A, Dirichlet(0.3)) for every pair 3 <= |i-j| < window;
* database profiles carry *observed* distances from a C-beta random walk
  with 3.8 A steps;
* target frequencies are Dirichlet(0.5) draws mixed with the profile
  background, SS probabilities Dirichlet(1), the effective number of
  observations uniform in [1, 14];
* database lengths are lognormal (sigma 0.5) clipped to a range.

The heavy lifting (distance lists) runs in ``libcbsynth.so`` with one
random stream per profile, so results do not depend on the thread count.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import build as _build
from .profiles import NDSTSLOTS, NSSSTATES, NTRN, NUMAA, ProfileSet

_lib = None


def _synth_lib():
    global _lib
    if _lib is None:
        path = _build.LIB_SYNTH
        if not os.path.exists(path):
            _build.build_synth()
        lib = ctypes.CDLL(path)
        lib.cbs_generate.restype = ctypes.c_int
        lib.cbs_generate.argtypes = [
            ctypes.c_int, ctypes.c_longlong, ctypes.c_void_p, ctypes.c_void_p,
            ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_ulonglong,
            ctypes.c_void_p,
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
            ctypes.c_int,
        ]
        _lib = lib
    return _lib


def global_background() -> np.ndarray:
    """Fixed amino-acid background shared by all synthetic profiles."""
    rng = np.random.default_rng(20240917)
    return rng.dirichlet(np.full(NUMAA, 40.0))


def make_profiles(lens, seed: int, predicted: bool, window: int = 64,
                  prb_thld: float = 0.05, nthreads: int | None = None) -> ProfileSet:
    """Generate profiles of the given lengths."""
    lens = np.ascontiguousarray(np.asarray(lens, dtype=np.int32))
    P = int(len(lens))
    N = int(lens.sum(dtype=np.int64))
    starts = np.zeros(P, dtype=np.int64)
    if P > 1:
        starts[1:] = np.cumsum(lens[:-1], dtype=np.int64)
    bkg = np.zeros((NUMAA, P), np.float32)
    eno = np.zeros(P, np.float32)
    trn = np.zeros((NTRN, N + P), np.float32)
    tf = np.zeros((NUMAA, N), np.float32)
    ss = np.zeros((NSSSTATES, N), np.float32)
    ssstate = np.zeros(N, np.int8)
    aa = np.zeros(N, np.int8)
    dd = np.zeros((NDSTSLOTS, N), np.float32)
    addrpro = np.zeros(N, np.int32)
    gb = np.ascontiguousarray(global_background(), dtype=np.float64)
    if nthreads is None:
        nthreads = max(1, min(os.cpu_count() or 1, 32))
    rc = _synth_lib().cbs_generate(
        P, N, lens.ctypes.data, starts.ctypes.data,
        1 if predicted else 0, int(window), float(prb_thld), int(seed) & 0xFFFFFFFFFFFFFFFF,
        gb.ctypes.data,
        bkg.ctypes.data, eno.ctypes.data, trn.ctypes.data, tf.ctypes.data, ss.ctypes.data,
        ssstate.ctypes.data, aa.ctypes.data, dd.ctypes.data, addrpro.ctypes.data,
        int(nthreads))
    if rc != 0:
        raise RuntimeError(f"cbs_generate failed ({rc})")
    return ProfileSet(lens=lens, bkg=bkg, eno=eno, trn=trn, tf=tf, dd=dd, ss=ss,
                      addrpro=addrpro, aa=aa, ssstate=ssstate,
                      names=[f"synth{seed}_{i}" for i in range(P)])


def plant_homologs(query: ProfileSet, db: ProfileSet, fraction: float, seed: int,
                   noise: float = 0.3) -> np.ndarray:
    """Overwrite a seeded subset of database profiles with noisy copies of
    query segments (target frequencies, SS probabilities, transitions and
    distance lists), so that a search finds true hits. Returns the indices of
    the planted profiles."""
    rng = np.random.default_rng(seed)
    P = db.nprofiles
    k = int(round(fraction * P))
    if k <= 0:
        return np.zeros(0, np.int64)
    picks = np.sort(rng.choice(P, size=k, replace=False))
    Lq = query.npositions
    starts = db.starts
    for p in picks:
        Ld = int(db.lens[p])
        n = int(min(Ld, Lq) * rng.uniform(0.5, 1.0))
        if n < 8:
            continue
        qa = int(rng.integers(0, Lq - n + 1))
        da = int(rng.integers(0, Ld - n + 1))
        s0 = int(starts[p]) + da
        w = 1.0 - noise
        db.tf[:, s0:s0 + n] = (w * query.tf[:, qa:qa + n] + noise * db.tf[:, s0:s0 + n])
        db.ss[:, s0:s0 + n] = (w * query.ss[:, qa:qa + n] + noise * db.ss[:, s0:s0 + n])
        t0 = int(starts[p]) + int(p) + 1 + da
        db.trn[:, t0:t0 + n] = query.trn[:, qa + 1:qa + 1 + n]
        dl = query.dd[:, qa:qa + n].copy()
        jitter = rng.integers(-1, 2, size=dl[1:].shape)
        vals = dl[1:]
        keep = vals != 255.0
        vals[keep] = np.clip(vals[keep] + jitter[keep], 0, 64)
        db.dd[:, s0:s0 + n] = dl
        db.aa[s0:s0 + n] = query.aa[qa:qa + n]
        db.ssstate[s0:s0 + n] = query.ssstate[qa:qa + n]
        if query.cv is not None and db.cv is not None:
            db.cv[:, s0:s0 + n] = (np.float32(w) * query.cv[:, qa:qa + n] +
                                   np.float32(noise) * db.cv[:, s0:s0 + n])
            db.cvnorm2[s0:s0 + n], db.cvprior[s0:s0 + n] = cv_magnitudes(db.cv[:, s0:s0 + n])
    return picks


# normal-Wishart prior of context vectors (src/libpro/srcpro/TCTXVECT.cpp:26-60):
# dimension 19, kappa0 0.1, nu0 19; the log prior of a vector is
# LPFACT - (nu0+1)/2 * log(1 + kappa0/(kappa0+1) * |v|^2)
# (src/libpro/srcpro/PMProfileModel.cpp:363-387, 823-828), with LPFACT =
# lgamma(10) - lgamma(1/2) + 19/2 * (log 0.1 - log 1.1)
CV_DIM = 19
CV_LPFACT = np.float32(-10.550543)


def cv_magnitudes(cv: np.ndarray):
    """(squared norms, log prior probabilities) of context vectors [19][n]."""
    cv = np.asarray(cv, np.float32)
    norm2 = np.zeros(cv.shape[1], np.float32)
    for d in range(cv.shape[0]):
        norm2 = norm2 + cv[d] * cv[d]
    prior = CV_LPFACT - np.float32(10.0) * np.log(np.float32(1.0) + np.float32(0.1 / 1.1) * norm2)
    return norm2, prior.astype(np.float32)


def add_context_vectors(ps: ProfileSet, seed: int) -> ProfileSet:
    """Give every position of `ps` a context vector: 19 standard normal
    entries (a stand-in for the reference profile builder's mixed
    logit-normal transform of the target frequencies), with its squared norm
    and log prior probability. Seeded apart from the other fields."""
    rng = np.random.default_rng([int(seed) & 0xFFFFFFFF, 0xC5])
    ps.cv = rng.standard_normal((CV_DIM, ps.npositions), dtype=np.float32)
    ps.cvnorm2, ps.cvprior = cv_magnitudes(ps.cv)
    return ps


def lognormal_lengths(n: int, median: float, lo: int, hi: int, seed: int,
                      sigma: float = 0.5) -> np.ndarray:
    rng = np.random.default_rng(seed)
    x = rng.lognormal(mean=np.log(median), sigma=sigma, size=n)
    return np.clip(np.rint(x), lo, hi).astype(np.int32)


def uniform_lengths(n: int, lo: int, hi: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.integers(lo, hi + 1, size=n).astype(np.int32)


# Workloads of the benchmark configurations. Each entry gives the query
# lengths, the database length law and the distance window.
WORKLOADS = {
    # 1 query of length 200 vs 1,000 profiles, lognormal median 180 in [30,600]
    "q200_db1k": dict(qlens=[200], ndb=1000, law=("lognormal", 180, 30, 600), window=64),
    # 1 query of length 400 vs 50,000 profiles, lognormal median 220 in [30,1500]
    "q400_db50k": dict(qlens=[400], ndb=50000, law=("lognormal", 220, 30, 1500), window=64),
    # query-length sweep over the 50,000-profile database
    "qsweep_db50k": dict(qlens=[64, 256, 1024], ndb=50000, law=("lognormal", 220, 30, 1500), window=64),
    # 1 query of length 1,500 vs 20,000 profiles of length U(500,1500), window 128
    "q1500_db20k": dict(qlens=[1500], ndb=20000, law=("uniform", 500, 1500), window=128),
    # serving: a resident 100,000-profile database (lognormal median 220 in
    # [30,1500]); request queries have lognormal lengths, median 250 in
    # [40,1200] (serving_queries)
    "serve_db100k": dict(qlens=[250], ndb=100000, law=("lognormal", 220, 30, 1500), window=64),
}


def serving_queries(n: int, seed: int = 7):
    """`n` request queries with lognormal lengths (median 250, in [40,1200])."""
    lens = lognormal_lengths(n, 250, 40, 1200, seed=seed * 1000 + 11)
    return [make_profiles([int(L)], seed=seed * 1000 + 100 + k, predicted=True)
            for k, L in enumerate(lens)]


def db_lengths(name: str, seed: int = 7, ndb: int | None = None) -> np.ndarray:
    w = WORKLOADS[name]
    n = w["ndb"] if ndb is None else ndb
    law = w["law"]
    if law[0] == "lognormal":
        return lognormal_lengths(n, law[1], law[2], law[3], seed)
    return uniform_lengths(n, law[1], law[2], seed)


HOMOLOG_FRACTION = 0.01


def make_workload(name: str, seed: int = 7, ndb: int | None = None, qindex: int = 0,
                  homologs: float = HOMOLOG_FRACTION, db_seed: int | None = None,
                  context_vectors: bool = False):
    """(query ProfileSet, database ProfileSet) for a named workload; a
    fraction `homologs` of the database profiles are planted homologs of
    the query. The query depends on `seed` only; the database on `db_seed`
    (default `seed`), so that shards of one search can share the query.
    With `context_vectors`, both sides carry context vectors (the CVS term)."""
    w = WORKLOADS[name]
    dseed = seed if db_seed is None else db_seed
    lens = db_lengths(name, dseed, ndb)
    db = make_profiles(lens, seed=dseed * 1000 + 1, predicted=False, window=w["window"])
    q = make_profiles([w["qlens"][qindex]], seed=seed * 1000 + 2 + qindex, predicted=True,
                      window=w["window"])
    if context_vectors:
        add_context_vectors(db, dseed * 1000 + 1)
        add_context_vectors(q, seed * 1000 + 2 + qindex)
    plant_homologs(q, db, homologs, seed=dseed * 1000 + 3 + qindex)
    return q, db


def planted_indices(name: str, seed: int = 7, ndb: int | None = None, qindex: int = 0,
                    homologs: float = HOMOLOG_FRACTION, db_seed: int | None = None) -> np.ndarray:
    """Indices of the database profiles that make_workload() with the same
    arguments overwrites with planted homologs (without generating them)."""
    dseed = seed if db_seed is None else db_seed
    P = len(db_lengths(name, dseed, ndb))
    k = int(round(homologs * P))
    if k <= 0:
        return np.zeros(0, np.int64)
    rng = np.random.default_rng(dseed * 1000 + 3 + qindex)
    return np.sort(rng.choice(P, size=k, replace=False))

