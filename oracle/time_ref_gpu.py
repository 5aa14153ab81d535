"""Device time of the reference's own CUDA kernels on a benchmark workload.

Measurement infrastructure, not part of the product: runs the reference's
score-matrix, phase-1, statistics and MAP kernels (built from their sources
by ``make -C oracle refgpu``, driven by ``oracle/ref_gpu_driver.cu``) on the
same seeded synthetic workload, query and options that ``bench.py`` uses for
rank 0, and prints one JSON line with the per-stage device times (CUDA
events around each stage's launches, summed over the database chunks) and
GCUPS = query length x database positions / total time. The database is
split into chunks of whole profiles as the reference's memory planner would
cap them (its kernels index a chunk's cells with 32-bit ints).

Usage (on a machine with a B200):
    python oracle/time_ref_gpu.py [--workload q400_db50k] [--seed 7] [--repeats 2]
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
# run as a script, this directory would shadow the oracle package
sys.path[:] = [p for p in sys.path if os.path.abspath(p or ".") != HERE]
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

from cother_b200 import synth  # noqa: E402
from cother_b200.profiles import NFIELDS  # noqa: E402
import make_ref_gpu_fixtures as fx  # noqa: E402
from oracle import oracle as orc  # noqa: E402


def max_chunk_positions(Lq: int, expct_prolen: int = 50) -> int:
    """The reference's cap on the positions of one database chunk
    (CuDeviceMemory::GetMaxAllowedNumDbProfilePositions,
    src/libmycu/cupro/CuDeviceMemory.cuh:658-690, DEV_EXPCT_DBPROLEN = 50)."""
    imax = 2147483647
    deplen1 = imax // Lq
    deplen2 = int(imax / 5 / (1.0 + (Lq + 2) / expct_prolen))
    indeplen1 = imax // 16 - 64
    indeplen2 = imax // 672 * expct_prolen
    return min(deplen1, deplen2, indeplen1, indeplen2)


def chunks(db, cap: int):
    """Runs of whole profiles with at most `cap` positions each."""
    out, first, n = [], 0, 0
    for p, L in enumerate(db.lens.tolist()):
        if n and n + L > cap:
            out.append((first, p - first))
            first, n = p, 0
        n += L
    out.append((first, db.nprofiles - first))
    return out


def run_chunk(L, q, db, thld, logethld, sspace, consts):
    nph1, nrec, nrows, _, line = consts
    Lq, N, P = q.npositions, db.npositions, db.nprofiles
    j = fx.Job()
    for name, ps in (("q", q), ("d", db)):
        beg, end = ps.field_tables()
        ptrs, sizes = getattr(j, name), getattr(j, name + "sz")
        for f in range(NFIELDS):
            ptrs[f] = beg[f]
            sizes[f] = (end[f] or 0) - (beg[f] or 0)
    sstab = np.ascontiguousarray(np.load(os.path.join(fx.HERE, "ssss.npy")), np.float32)
    nnw = np.ascontiguousarray(np.load(os.path.join(fx.HERE, "nn_weights.npy")), np.float32)
    par = orc.cother_par()
    j.nqyposs, j.ndbpros, j.ndbposs, j.dbpro1len = Lq, P, N, int(db.lens.max())
    j.qyeno = float(q.eno[0])
    j.sstab, j.nnweights = sstab.ctypes.data, nnw.ctypes.data
    j.ssswgt, j.ddmswgt, j.minpp = 0.12, 0.2, 0.28
    j.scorethld, j.logevthld, j.searchspace = thld, logethld, sspace
    j.reflambda, j.refK = par["UNGAPPED"]["Lambda"], par["UNGAPPED"]["K"]
    j.explambda, j.expK = par["GAPPED_A_1"]["Lambda"], par["GAPPED_A_1"]["K"]
    j.dstsegm, j.ssemodel, j.xuninf = 6, 2, 1
    ph1 = np.zeros((P, nph1), np.float32)
    st = np.zeros((P, nrec), np.float32)
    fin = np.zeros((P, nrec), np.float32)
    cap = N + P * (Lq + 1) + 2 * line
    alns = np.zeros((nrows, cap), np.uint8)
    j.phase1, j.stats, j.final_recs = ph1.ctypes.data, st.ctypes.data, fin.ctypes.data
    j.alns, j.alns_cap = alns.ctypes.data, cap
    j.copy_matrices = 0
    if L.refgpu_run(ctypes.byref(j)) != 0:
        raise RuntimeError(L.refgpu_error().decode())
    return [float(t) for t in j.stage_ms], int(j.globvars[0])


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="q400_db50k")
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--ndb", type=int, default=None)
    ap.add_argument("--repeats", type=int, default=2)
    args = ap.parse_args()
    q, db = synth.make_workload(args.workload, seed=args.seed, ndb=args.ndb)
    Lq, N, P = q.npositions, db.npositions, db.nprofiles
    L = ctypes.CDLL(fx.LIB)
    L.refgpu_error.restype = ctypes.c_char_p
    consts = (ctypes.c_int * 5)()
    L.refgpu_consts(consts)
    consts = list(consts)
    thld, logethld = orc.score_threshold(Lq, N)
    sspace = float(orc.length_adjustment(Lq, N, P)[0])
    parts = chunks(db, max_chunk_positions(Lq))
    subs = [db.subset(f, n) for f, n in parts]
    runs, passed = [], 0
    for _ in range(max(1, args.repeats)):
        tot, passed = [0.0] * 4, 0
        for sub in subs:
            ms, npass = run_chunk(L, q, sub, thld, logethld, sspace, consts)
            tot = [a + b for a, b in zip(tot, ms)]
            passed += npass
        runs.append(tot)
    last = runs[-1]
    total = sum(last)
    print(json.dumps({
        "impl": "reference-cuda-kernels", "workload": args.workload, "query_len": Lq,
        "db_profiles": P, "db_positions": N, "chunks": len(parts),
        "chunk_positions": [int(s.npositions) for s in subs], "passed_phase1": passed,
        "stage_ms": dict(zip(["score_matrix", "phase1", "statistics", "map"], last)),
        "total_ms": total, "gcups": Lq * N / (total * 1e-3) / 1e9,
        "all_runs_ms": runs,
    }))


if __name__ == "__main__":
    main()
