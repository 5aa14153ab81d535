"""Golden fixtures from the reference's own CUDA kernels (needs a GPU).

Runs the reference's score-matrix, phase-1 DP, statistics and MAP kernels,
compiled from their sources by ``make -C oracle refgpu`` into
``oracle/_ref/librefgpu.so`` and driven by ``oracle/ref_gpu_driver.cu``, on
small seeded synthetic searches, and writes every intermediate result to
``ref_gpu_<case>.npz``. ``tests/test_ref_gpu_pin.py`` then checks the CPU
oracle against these files on any machine.

The inputs are rebuilt from their seeds by :func:`case_inputs` (the test
does the same and checks ``input_digest`` first). The reference tree is not
read at run time: only the prebuilt library and the committed fixtures
(ssss.npy, nn_weights.npy, cother_par.json) are.

Usage (on a machine with a B200):
    python tests/golden/make_ref_gpu_fixtures.py [outdir [case,case,...]]
"""
from __future__ import annotations

import ctypes
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from cother_b200 import synth  # noqa: E402
from cother_b200.profiles import NFIELDS  # noqa: E402

LIB = os.path.join(ROOT, "oracle", "_ref", "librefgpu.so")

# option sets: SSSWGT, DDMSWGT, DSTSEGM, MINPP, SSEMODEL, X_UNINF; `full`
# stores the score matrices and backtrack codes as well as the records
CASES = {
    "main": dict(ssswgt=0.12, ddmswgt=0.2, dstsegm=6, minpp=0.28, ssemodel=2, xuninf=1,
                 full=True),
    "q77": dict(ssswgt=0.12, ddmswgt=0.2, dstsegm=6, minpp=0.28, ssemodel=2, xuninf=1,
                full=True, inputs="q77"),
    "sse1": dict(ssswgt=0.12, ddmswgt=0.2, dstsegm=6, minpp=0.28, ssemodel=1, xuninf=1,
                 full=False),
    "sse0_nox": dict(ssswgt=0.12, ddmswgt=0.2, dstsegm=6, minpp=0.28, ssemodel=0, xuninf=0,
                     full=False),
    "noss": dict(ssswgt=0.0, ddmswgt=0.2, dstsegm=6, minpp=0.28, ssemodel=2, xuninf=1,
                 full=True),
    # the context-vector term at the reference's default weight, with and
    # without the SS term (inputs with context vectors)
    "cvs": dict(ssswgt=0.12, cvswgt=0.15, ddmswgt=0.2, dstsegm=6, minpp=0.28, ssemodel=2,
                xuninf=1, full=True, inputs="q64cv"),
    "cvs_only": dict(ssswgt=0.0, cvswgt=0.15, ddmswgt=0.2, dstsegm=6, minpp=0.28, ssemodel=2,
                     xuninf=1, full=True, inputs="q64cv"),
    # MAPALN=0: the phase-1 alignments are reported (no MAP realignment)
    "mapaln0": dict(ssswgt=0.12, ddmswgt=0.2, dstsegm=6, minpp=0.28, ssemodel=2, xuninf=1,
                    full=True, nomapaln=1),
    "mapaln0_cvs": dict(ssswgt=0.12, cvswgt=0.15, ddmswgt=0.2, dstsegm=6, minpp=0.28, ssemodel=2,
                        xuninf=1, full=True, inputs="q64cv", nomapaln=1),
}
# every profile passes phase 1, so that each one's phase-1 record and
# statistics are pinned; MAP realigns the pairs with log E <= LOGE_THLD
# (about half of them) and skips the rest
SCORE_THLD = -1.0e9
LOGE_THLD = 1.8


def search_space(q, db) -> float:
    """Effective search space for this query against a database of exactly
    these profiles: the length adjustment of
    libpro/srcsco/AbstractScoreMatrix.cpp:303-393 (the oracle's restatement),
    i.e. what cbp_set_db_details(N, P) gives the CUDA path."""
    from oracle import oracle as orc
    return float(orc.length_adjustment(q.npositions, db.npositions, db.nprofiles)[0])


# input sets: query length, number of profiles, length range, seed base
INPUTS = {
    "q64": dict(qlen=64, nprof=16, median=90, lo=30, hi=220, seed=611),
    "q77": dict(qlen=77, nprof=12, median=120, lo=30, hi=300, seed=711),
    "q64cv": dict(qlen=64, nprof=16, median=90, lo=30, hi=220, seed=611, cv=True),
}


def case_inputs(name: str = "q64"):
    """(query, db): a query with predicted distance lists and database
    profiles, longest first, two of them planted homologs."""
    c = INPUTS[name]
    q = synth.make_profiles([c["qlen"]], seed=c["seed"], predicted=True, nthreads=1)
    lens = synth.lognormal_lengths(c["nprof"], c["median"], c["lo"], c["hi"], seed=c["seed"] + 1)
    lens = np.sort(np.asarray(lens))[::-1].copy()
    db = synth.make_profiles(lens, seed=c["seed"] + 2, predicted=False, nthreads=1)
    if c.get("cv"):
        synth.add_context_vectors(q, c["seed"] + 10)
        synth.add_context_vectors(db, c["seed"] + 11)
    synth.plant_homologs(q, db, 2.0 / c["nprof"], seed=c["seed"] + 3)
    return q, db


def input_digest(q, db) -> str:
    h = hashlib.sha256()
    for ps in (q, db):
        for a in (ps.lens, ps.bkg, ps.eno, ps.trn, ps.tf, ps.dd, ps.ss, ps.addrpro, ps.aa,
                  ps.ssstate):
            h.update(np.ascontiguousarray(a).tobytes())
        if ps.cv is not None:
            for a in (ps.cv, ps.cvprior, ps.cvnorm2):
                h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


class Job(ctypes.Structure):
    _fields_ = [
        ("q", ctypes.c_void_p * NFIELDS), ("qsz", ctypes.c_size_t * NFIELDS),
        ("d", ctypes.c_void_p * NFIELDS), ("dsz", ctypes.c_size_t * NFIELDS),
        ("nqyposs", ctypes.c_int), ("ndbpros", ctypes.c_int), ("ndbposs", ctypes.c_int),
        ("dbpro1len", ctypes.c_int), ("qyeno", ctypes.c_float),
        ("sstab", ctypes.c_void_p), ("nnweights", ctypes.c_void_p),
        ("ssswgt", ctypes.c_float), ("ddmswgt", ctypes.c_float), ("minpp", ctypes.c_float),
        ("scorethld", ctypes.c_float), ("logevthld", ctypes.c_float),
        ("searchspace", ctypes.c_float), ("reflambda", ctypes.c_float), ("refK", ctypes.c_float),
        ("explambda", ctypes.c_float), ("expK", ctypes.c_float),
        ("dstsegm", ctypes.c_int), ("ssemodel", ctypes.c_int), ("xuninf", ctypes.c_int),
        ("scores", ctypes.c_void_p), ("modscores", ctypes.c_void_p), ("btck", ctypes.c_void_p),
        ("phase1", ctypes.c_void_p), ("stats", ctypes.c_void_p), ("final_recs", ctypes.c_void_p),
        ("alns", ctypes.c_void_p), ("alns_cap", ctypes.c_size_t),
        ("globvars", ctypes.c_uint * 4), ("dblen", ctypes.c_int), ("dbalnlen2", ctypes.c_size_t),
        ("copy_matrices", ctypes.c_int), ("stage_ms", ctypes.c_float * 4),
        ("cvswgt", ctypes.c_float), ("cvskeys", ctypes.c_void_p), ("cvsscores", ctypes.c_void_p),
        ("cvscard", ctypes.c_int), ("nomapaln", ctypes.c_int),
    ]


def run_case(L, q, db, opts):
    consts = (ctypes.c_int * 5)()
    L.refgpu_consts(consts)
    nph1, nrec, nrows, nflds, line = list(consts)
    assert nflds == NFIELDS
    j = Job()
    for name, ps in (("q", q), ("d", db)):
        beg, end = ps.field_tables()
        ptrs = getattr(j, name)
        sizes = getattr(j, name + "sz")
        for f in range(NFIELDS):
            ptrs[f] = beg[f]
            sizes[f] = (end[f] or 0) - (beg[f] or 0)
    Lq, N, P = q.npositions, db.npositions, db.nprofiles
    dblen = (N + line - 1) // line * line
    sstab = np.ascontiguousarray(np.load(os.path.join(HERE, "ssss.npy")), np.float32)
    nnw = np.ascontiguousarray(np.load(os.path.join(HERE, "nn_weights.npy")), np.float32)
    par = json.load(open(os.path.join(HERE, "cother_par.json")))
    j.nqyposs, j.ndbpros, j.ndbposs, j.dbpro1len = Lq, P, N, int(db.lens.max())
    j.qyeno = float(q.eno[0])
    j.sstab, j.nnweights = sstab.ctypes.data, nnw.ctypes.data
    j.ssswgt, j.ddmswgt, j.minpp = opts["ssswgt"], opts["ddmswgt"], opts["minpp"]
    sspace = search_space(q, db)
    j.scorethld, j.logevthld, j.searchspace = SCORE_THLD, LOGE_THLD, sspace
    j.reflambda, j.refK = par["UNGAPPED"]["Lambda"], par["UNGAPPED"]["K"]
    j.explambda, j.expK = par["GAPPED_A_1"]["Lambda"], par["GAPPED_A_1"]["K"]
    j.dstsegm, j.ssemodel, j.xuninf = opts["dstsegm"], opts["ssemodel"], opts["xuninf"]
    cvs = np.load(os.path.join(HERE, "cvs2s.npz"))
    cvkeys = np.ascontiguousarray(cvs["keys"], np.float32)
    cvscores = np.ascontiguousarray(cvs["scores"], np.float32)
    j.cvswgt = opts.get("cvswgt", 0.0)
    j.nomapaln = int(opts.get("nomapaln", 0))
    j.cvskeys, j.cvsscores, j.cvscard = cvkeys.ctypes.data, cvscores.ctypes.data, len(cvkeys)
    sc = np.zeros((Lq, dblen), np.float32)
    ms = np.zeros((Lq, dblen), np.float32)
    bt = np.zeros((Lq, dblen), np.uint8)
    ph1 = np.zeros((P, nph1), np.float32)
    st = np.zeros((P, nrec), np.float32)
    fin = np.zeros((P, nrec), np.float32)
    cap = N + P * (Lq + 1) + 2 * line
    alns = np.zeros((nrows, cap), np.uint8)
    j.scores, j.modscores, j.btck = sc.ctypes.data, ms.ctypes.data, bt.ctypes.data
    j.phase1, j.stats, j.final_recs = ph1.ctypes.data, st.ctypes.data, fin.ctypes.data
    j.alns, j.alns_cap = alns.ctypes.data, cap
    j.copy_matrices = 1
    rc = L.refgpu_run(ctypes.byref(j))
    if rc != 0:
        raise RuntimeError(L.refgpu_error().decode())
    npass = int(j.globvars[0])
    out = dict(globvars=np.array(list(j.globvars), np.uint32), dblen=np.int64(j.dblen),
               dbalnlen2=np.int64(j.dbalnlen2), phase1=ph1[:npass], stats=st[:npass],
               final=fin[:npass], alns=alns[:, :j.dbalnlen2],
               options=json.dumps(opts), scorethld=np.float32(SCORE_THLD),
               logevthld=np.float32(LOGE_THLD), searchspace=np.float32(sspace),
               digest=input_digest(q, db))
    if opts["full"]:
        out.update(scores=sc, modscores=ms, btck=bt)
    return out


def main(outdir: str, only=None) -> None:
    L = ctypes.CDLL(LIB)
    L.refgpu_error.restype = ctypes.c_char_p
    os.makedirs(outdir, exist_ok=True)
    for name, opts in CASES.items():
        if only and name not in only:
            continue
        q, db = case_inputs(opts.get("inputs", "q64"))
        out = run_case(L, q, db, opts)
        path = os.path.join(outdir, f"ref_gpu_{name}.npz")
        np.savez_compressed(path, **out)
        print(name, "passed", int(out["globvars"][0]), "alnlen", int(out["dbalnlen2"]), "->", path)


if __name__ == "__main__":
    # usage: make_ref_gpu_fixtures.py [outdir [case,case,...]]
    main(sys.argv[1] if len(sys.argv) > 1 else HERE,
         sys.argv[2].split(",") if len(sys.argv) > 2 else None)
