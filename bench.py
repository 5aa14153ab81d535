#!/usr/bin/env python3
"""Benchmark of the COTHER search path on B200.

One step = one query profile searched against the GPU-resident synthetic
database through the whole implemented pipeline. Metric: GCUPS = query
length x database positions / time.

  value  -- GCUPS from the device time of the pipeline's kernels (inputs
            already resident in HBM);
  e2e    -- GCUPS of the C-ABI call a user makes (cbp_process): host query
            buffers are packed and copied to the device and the results are
            read back inside the timed region.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Multi-GPU: launched by torchrun, one rank per GPU; every rank searches its
own database shard of the full configured size (weak scaling), no
collective on the data path; the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DEFAULT_WORKLOAD = "q400_db50k"
# DRAM bytes (read + write) per cell of one score_matrix_kernel launch,
# measured by ncu on q400 x 2,000 profiles (3.03 GB for 195.0 M cells with
# the 32-row variant: 8 B/cell of score writes plus the database lists
# re-read by each block of query rows); the traffic grows with the cells
SCORE_DRAM_BYTES_PER_CELL = 15.51


def score_traffic_per_cell(rows: int) -> float:
    """DRAM bytes per cell of the score kernel with `rows` query rows per
    block: the 8 B/cell of score writes plus the database reads, which each
    block of rows repeats (measured at 32 rows)."""
    return 8.0 + (SCORE_DRAM_BYTES_PER_CELL - 8.0) * 32.0 / rows


STAGES = ["score_matrix", "phase1_dp", "phase1_finalize", "statistics", "map_realignment", "hit_order"]
OPS_PER_DDMS_STEP = 50  # algorithmic ops of one 4-cell DDMS step (2 pair scores,
                        # 2 interpolations, 4 segment updates, 1 top-3 register)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD)
    ap.add_argument("--qindex", type=int, default=0,
                    help="which of the workload's query lengths (qsweep_db50k: 0, 1, 2 = 64, 256, 1024)")
    ap.add_argument("--ndb", type=int, default=None, help="override #database profiles (testing only)")
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-tc-forms", action="store_true",
                    help="skip the tensor-core forms measured after the timed run")
    ap.add_argument("--no-serving", action="store_true",
                    help="skip the short serving run after the timed run")
    ap.add_argument("--tc", default="plain", choices=["plain", "bf16", "tf32"],
                    help="form of the profile-profile term: FP32 CUDA cores or tensor cores "
                         "(BF16x3 / TF32x3 hi-lo split)")
    ap.add_argument("--cvswgt", type=float, default=0.0,
                    help="weight of the context-vector term (0 = off, the parity configuration; "
                         "the reference's own default is 0.15); > 0 gives the profiles context vectors")
    ap.add_argument("--ddmswgt", type=float, default=0.2,
                    help="weight of the DDMS term (the parity configuration's 0.2; 0 leaves the "
                         "profile-profile and SS terms, and the phase-1 DP dominates)")
    ap.add_argument("--serve", action="store_true",
                    help="request loop over a resident database: queries/s and p50/p99 latency")
    ap.add_argument("--rate", default="5", help="--serve: offered loads (Poisson, queries/s), comma list")
    ap.add_argument("--queries", type=int, default=12, help="--serve: requests in the timed run")
    ap.add_argument("--slots", type=int, default=3, help="--serve: concurrent batches (slots)")
    ap.add_argument("--max-batch", type=int, default=4, help="--serve: queries searched in one pass at most")
    return ap.parse_args()


def ddms_steps(L1: int, L2: int, dstsegm: int = 6) -> int:
    """Exact number of 4-cell DDMS steps for lists of lengths L1, L2."""
    if L1 < dstsegm or L2 < dstsegm:
        return 0
    n = 0
    j = L2 >> 2
    while j >= 0:
        lim = min(L1, L2 - j)
        n += (lim + 3) // 4 if lim > 0 else 0
        j -= 2
    i = L1 >> 2
    while i > 0:
        lim = min(L2, L1 - i)
        n += (lim + 3) // 4 if lim > 0 else 0
        i -= 2
    return n


def total_ddms_steps(q, db) -> int:
    hq = np.bincount(q.dd[0].astype(np.int64), minlength=100)
    hd = np.bincount(db.dd[0].astype(np.int64), minlength=100)
    tab = np.array([[ddms_steps(a, b) for b in range(100)] for a in range(100)], np.int64)
    return int(hq @ tab @ hd)


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = max(mx, float(p[2]))
            except ValueError:
                continue
            for k, n in enumerate(names):
                if p[5 + k].lower() in ("active", "1"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return None


def oracle_pipeline(q, db, ss, nthreads, db_len, nseqs, cvswgt=0.0):
    """The oracle's whole search path (score matrix, phase 1, statistics,
    MAP realignment) for the query against the profile set `db` (a sample
    of the workload's database); E-values for a database of `db_len`
    positions and `nseqs` profiles. Loads the oracle only, never the
    product library."""
    from oracle import oracle as O
    ncols = db.npositions
    sc, ms = O.score_matrix(q, db, ss, ncols=ncols, nthreads=nthreads, cvswgt=cvswgt)
    thld, lthld = O.score_threshold(q.npositions, db_len)
    sspace, _ = O.length_adjustment(q.npositions, db_len, nseqs)
    rec, _ = O.dp1(q, db, sc, 0, 0, db.nprofiles, thld)
    for p in np.nonzero(rec["passed"])[0]:
        s0, Ld = int(db.starts[p]), int(db.lens[p])
        st, _ = O.pair_statistics(sc[:, s0:s0 + Ld], q.aa, db.aa[s0:s0 + Ld], rec["score"][p],
                                  rec["psts"][p], q.npositions, Ld, q.eno[0], db.eno[p], sspace)
        if st[2] <= lthld:
            O.map_pair(q, db, p, sc[:, s0:s0 + Ld], ms[:, s0:s0 + Ld], st[3])
    return ncols


def spread_sample(db, nprof: int) -> np.ndarray:
    """`nprof` profile indices spread evenly over the whole database."""
    nprof = int(max(1, min(db.nprofiles, nprof)))
    return np.unique(np.linspace(0, db.nprofiles - 1, nprof).round().astype(np.int64))


class CpuTimer:
    """The oracle pipeline on the host cores over bounded samples of the
    workload's database (profiles spread across it), calibrated so that a
    sample takes about the requested seconds."""

    def __init__(self, q, db, ss, db_len, nseqs, cvswgt=0.0):
        self.q, self.db, self.ss = q, db, ss
        self.db_len, self.nseqs, self.cvswgt = db_len, nseqs, cvswgt
        self.rate = {}

    def _run(self, idx, nthreads):
        sub = self.db.select(idx)
        t = time.perf_counter()
        cols = oracle_pipeline(self.q, sub, self.ss, nthreads, self.db_len, self.nseqs, self.cvswgt)
        return cols, max(time.perf_counter() - t, 1e-6)

    def measure(self, seconds: float, nthreads: int):
        if nthreads not in self.rate:
            cols, dt = self._run(spread_sample(self.db, 4), nthreads)
            self.rate[nthreads] = cols / dt
        mean_len = float(self.db.lens.mean())
        idx = spread_sample(self.db, max(4, self.rate[nthreads] * seconds / mean_len))
        cols, dt = self._run(idx, nthreads)
        cells = self.q.npositions * cols
        return {"value": cells / dt / 1e9, "unit": "GCUPS", "cores": nthreads,
                "kind": "port",
                "sample": f"query {self.q.npositions} x {len(idx)} database profiles spread over "
                          f"all {self.db.nprofiles} ({cols} positions, {cells} cells, {dt:.1f} s), "
                          f"whole path (score matrix on {nthreads} threads, phase 1, statistics, "
                          f"MAP); E-values for the whole database"}


def cpu_baseline(q, db, ss, seconds: float, db_len: int, nseqs: int, cvswgt: float = 0.0):
    """The oracle (a port of the reference's kernels; the reference has no
    CPU path) on all host cores and on one core, each on a bounded sample
    of the same workload."""
    ncpu = os.cpu_count() or 1
    timer = CpuTimer(q, db, ss, db_len, nseqs, cvswgt)
    out = timer.measure(seconds * 0.6, ncpu)
    out["single_thread"] = timer.measure(seconds * 0.4, 1)
    return out


def tc_forms(cb, ss, plain_opts, q, db, db_len: int, nseqs: int, plain_digest: str) -> dict:
    """The tensor-core forms (BF16x3, TF32x3) of the whole path on the same
    query and database: GCUPS from the stages' device time over two steps
    after one warm-up, the score stage's time, and whether the top-50 hit
    list equals the plain form's."""
    out = {}
    for name, form in (("bf16x3", cb.TC_BF16X3), ("tf32x3", cb.TC_TF32X3)):
        o = cb.Options.defaults()
        for f, _ in cb.Options._fields_:
            setattr(o, f, getattr(plain_opts, f))
        o.tc_form = form
        with cb.BatchProcessing(ss, o) as bp:
            bp.transfer_cpm_data(db)
            bp.set_db_details(db_len, nseqs)
            bp.set_query_len(q.npositions)
            bp.process_score_matrix(q)
            ms, score_ms = 0.0, 0.0
            for _ in range(2):
                bp.process_score_matrix(q)
                st = bp.stage_times()
                ms += sum(st)
                score_ms += st[0]
            recs, order = bp.hit_records(), bp.hit_list()
            digest = hashlib.sha1(recs[order[:50], 1].view(np.uint32).tobytes()).hexdigest()[:16]
        out[name] = {"value": float(q.npositions) * db.npositions * 2 / (ms / 1e3) / 1e9, "unit": "GCUPS",
                     "score_matrix_ms": score_ms / 2, "top50_digest": digest,
                     "top50_same_as_plain": digest == plain_digest}
    return out


def workload_config(args, q, db, world: int) -> dict:
    """The `config` of the JSON line: the same for both arms."""
    return {"workload": args.workload, "query_len": q.npositions, "db_profiles": db.nprofiles,
            "db_positions": db.npositions, "stages": STAGES, "tc_form": args.tc,
            "cvswgt": args.cvswgt, "ddmswgt": args.ddmswgt,
            "l2": "inputs larger than L2 (database chunk > 126 MB)",
            "parallelism": f"dp{world} (database shard per GPU)"}


def reference_gpu_kernels(args):
    """Device time of the reference's own CUDA kernels (compiled from its
    sources for sm_100a into oracle/_ref) on the same workload, or None when
    they are not built. Runs after the CPU arm's timed steps."""
    lib = os.path.join(ROOT, "oracle", "_ref", "librefgpu.so")
    if not os.path.exists(lib) or args.tc != "plain" or args.cvswgt > 0:
        return None
    cmd = [sys.executable, os.path.join(ROOT, "oracle", "time_ref_gpu.py"), "--workload",
           args.workload, "--seed", str(args.seed), "--repeats", "2"]
    if args.ndb:
        cmd += ["--ndb", str(args.ndb)]
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
        line = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
        if r.returncode != 0 or not line:
            return {"unavailable": (r.stderr.strip().splitlines() or ["no output"])[-1][:300]}
        d = json.loads(line[-1])
        return {"value": d["gcups"], "unit": "GCUPS", "stage_ms": d["stage_ms"],
                "total_ms": d["total_ms"], "chunks": d["chunks"],
                "what": "the reference's own score-matrix, phase-1, statistics and MAP kernels, "
                        "compiled from its sources for sm_100a, same workload and query, device "
                        "time (oracle/time_ref_gpu.py)"}
    except Exception as e:  # a measurement beside the arm's value, never its result
        return {"unavailable": str(e)[:300]}


def run_reference(args):
    """--impl reference: the oracle port of the reference's kernels on the
    host cores (the reference has no CPU path of its own), on the same
    workload as the product arm: the full database is generated and each
    step searches the query against a bounded sample of it."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from cother_b200 import synth
    ss = np.load(os.path.join(ROOT, "tests", "golden", "ssss.npy"))
    q, db = synth.make_workload(args.workload, seed=args.seed, ndb=args.ndb, qindex=args.qindex,
                                context_vectors=args.cvswgt > 0)
    db_len, nseqs = db.npositions, db.nprofiles
    ncpu = os.cpu_count() or 1
    timer = CpuTimer(q, db, ss, db_len, nseqs, args.cvswgt)
    per_step = max(1.0, args.cpu_seconds / 3)
    vals = [timer.measure(per_step, ncpu) for _ in range(max(3, args.warmup) + args.steps)]
    timed = vals[-args.steps:] if args.steps > 0 else vals
    v = float(np.mean([x["value"] for x in timed]))
    cb = dict(timed[-1])
    cb["value"] = v
    cb["single_thread"] = timer.measure(per_step, 1)
    line = {"impl": "reference", "metric": "GCUPS", "value": v, "unit": "GCUPS", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(args, q, db, args.gpus),
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    ref_gpu = reference_gpu_kernels(args)
    if ref_gpu is not None:
        line["reference_gpu_kernels"] = ref_gpu
    print(json.dumps(line))


def serve_loads(db, ss, opts, rates, nqueries: int, slots: int, max_batch: int, seed: int):
    """Poisson arrivals of `nqueries` request queries per offered load in
    `rates` (queries/s) against the resident database `db`, served by the
    library's C++ request loop; one summary dict per load, and the loop's
    memory budget."""
    from cother_b200 import synth
    from cother_b200.serving import SearchServer, latency_summary
    loads = []
    with SearchServer(db, ss, opts, slots=slots, max_batch=max_batch) as srv:
        srv.submit(synth.serving_queries(1, seed=seed + 99)[0]).result()   # warm-up, not timed
        for li, rate in enumerate(rates):
            queries = synth.serving_queries(nqueries, seed=seed + li)
            rng = np.random.default_rng(seed + li)
            gaps = rng.exponential(1.0 / rate, nqueries)
            t0 = time.perf_counter()
            futs = []
            for k in range(nqueries):
                t0 += gaps[k]
                delay = t0 - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                futs.append(srv.submit(queries[k]))
            res = [f.result() for f in futs]
            s = latency_summary(res)
            cells = sum(q.npositions for q in queries) * db.npositions
            wall = max(r["finish"] for r in res) - min(r["arrival"] for r in res)
            loads.append({"offered_qps": rate, "queries": nqueries, "queries_per_s": s["queries_per_s"],
                          "p50_ms": s["p50_ms"], "p99_ms": s["p99_ms"], "service_p50_ms": s["service_p50_ms"],
                          "mean_batch": s["mean_batch"], "gcups": cells / wall / 1e9,
                          "query_lens": [q.npositions for q in queries]})
        budget = srv.budget
    return loads, budget


def run_serve(args):
    """--serve: Poisson arrivals of request queries against a resident
    database, served by the library's C++ request loop (concurrent slots,
    continuous batching of the waiting queries into one pass over the
    database); reports completed queries per second and the latency
    (arrival to results) for each offered load in --rate (comma list)."""
    from cother_b200 import synth
    import cother_b200 as cb
    workload = args.workload if args.workload != DEFAULT_WORKLOAD else "serve_db100k"
    ss = np.load(os.path.join(ROOT, "tests", "golden", "ssss.npy"))
    _, db = synth.make_workload(workload, seed=args.seed, ndb=args.ndb)
    rates = [float(x) for x in str(args.rate).split(",")]
    opts = cb.Options.defaults()
    opts.tc_form = {"plain": cb.TC_PLAIN, "bf16": cb.TC_BF16X3, "tf32": cb.TC_TF32X3}[args.tc]
    loads, budget = serve_loads(db, ss, opts, rates, args.queries, args.slots, args.max_batch, args.seed)
    best = max(loads, key=lambda x: x["queries_per_s"])
    print(json.dumps({
        "metric": "queries_per_s", "value": best["queries_per_s"], "unit": "queries/s",
        "n_gpus": 1, "higher_is_better": True, "p50_ms": best["p50_ms"], "p99_ms": best["p99_ms"],
        "offered_qps": best["offered_qps"], "loads": loads, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload, "db_profiles": db.nprofiles, "db_positions": db.npositions,
                   "slots": args.slots, "max_batch": args.max_batch, "tc_form": args.tc,
                   "memory_budget_bytes": budget}}))


def serving_summary(cb, ss, seed: int) -> dict:
    """A short run of the serving configuration after the timed steps: the
    resident 100,000-profile database, six Poisson requests at 20 queries/s,
    3 slots, batches of up to 4, the BF16x3 tensor-core score path."""
    from cother_b200 import synth
    _, db = synth.make_workload("serve_db100k", seed=seed)
    opts = cb.Options.defaults()
    opts.tc_form = cb.TC_BF16X3
    loads, budget = serve_loads(db, ss, opts, [20.0], 6, 3, 4, seed)
    out = dict(loads[0])
    out.update({"workload": "serve_db100k", "db_profiles": db.nprofiles, "db_positions": db.npositions,
                "slots": 3, "max_batch": 4, "tc_form": "bf16", "memory_budget_bytes": budget,
                "note": "shortened stream (6 requests); the configuration's 2,000 would take hours at "
                        "this capacity"})
    return out


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.serve:
        run_serve(args)
        return
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))

    import cother_b200 as cb
    from cother_b200 import synth
    ss = np.load(os.path.join(ROOT, "tests", "golden", "ssss.npy"))
    # one query for all ranks; each rank holds its own database shard
    q, db = synth.make_workload(args.workload, seed=args.seed, ndb=args.ndb, qindex=args.qindex,
                                db_seed=args.seed + 1000 * rank, context_vectors=args.cvswgt > 0)
    Lq, Ndb = q.npositions, db.npositions
    steps_ddms = total_ddms_steps(q, db)

    opts = cb.Options.defaults()
    opts.tc_form = {"plain": cb.TC_PLAIN, "bf16": cb.TC_BF16X3, "tf32": cb.TC_TF32X3}[args.tc]
    opts.cvswgt = args.cvswgt
    opts.ddmswgt = args.ddmswgt
    if args.ddmswgt <= 0:
        steps_ddms = 0
    bp = cb.BatchProcessing(ss, opts, device=local)
    if args.cvswgt > 0:
        cvs = np.load(os.path.join(ROOT, "tests", "golden", "cvs2s.npz"))
        bp.set_cvs2s_map(cvs["keys"], cvs["scores"])
    bp.transfer_cpm_data(db)
    db_len, nseqs = Ndb * world, db.nprofiles * world
    bp.set_db_details(db_len, nseqs)
    bp.set_query_len(Lq)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        bp.process_score_matrix(q)
    barrier()
    clk = ClockSampler(local)
    clk.start()
    stream = torch.cuda.current_stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    kern_ms, launches = 0.0, 0
    score_ms, score_launches = 0.0, 0
    stage_acc = [0.0] * len(STAGES)
    e0.record(stream)
    d2h = 0
    nhits = 0
    merged_hits = 0
    for _ in range(args.steps):
        bp.process_score_matrix(q)
        recs = bp.hit_records()
        rows = bp.alignment_rows()
        if dist is not None:
            # the path's one exchange: the shards' hit lists, merged by E-value
            from cother_b200 import sharding
            parts = sharding.gather_hits(sharding.local_hits(bp, rank * db.nprofiles, Lq))
            merged_hits = len(sharding.merge_hit_lists(parts))
        d2h = recs.nbytes + rows.nbytes
        nhits = len(recs)
        order = bp.hit_list()
        st = bp.stage_times()
        stage_acc = [a + b for a, b in zip(stage_acc, st)]
        kern_ms += sum(st)
        score_ms += st[0]
        launches += bp.launch_count()
        score_launches += bp.stage_launches()[0]
    e1.record(stream)
    e1.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    clocks = clk.stop()
    t = torch.tensor([e2e_ms, kern_ms], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_ms, kern_ms = float(t[0]), float(t[1])
    cells = float(Lq) * float(Ndb) * world
    steps = max(args.steps, 1)
    value = cells * steps / (kern_ms / 1e3) / 1e9
    e2e = cells * steps / (e2e_ms / 1e3) / 1e9

    if rank == 0:
        peaks = measured_peaks()
        rows = bp.tuning(Lq)["score_rows"]
        score_launch_ms = score_ms / max(1, score_launches)
        sm_mhz = clocks.get("sm_max_mhz") or 1965.0
        alu_peak = 148 * 128 * sm_mhz * 1e6 / 1e9  # lane-ops/s at max clock, Gop/s
        # one launch per slab; the workload here fits one slab
        ops = steps_ddms * OPS_PER_DDMS_STEP * args.steps / max(1, score_launches)
        achieved = ops / (score_launch_ms / 1e3) / 1e9  # Gop/s
        roof = {"bound": "alu", "achieved": achieved, "peak": alu_peak, "unit": "Gop/s",
                "frac": achieved / alu_peak,
                "traffic": score_traffic_per_cell(rows) * float(Lq) * Ndb,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one "
                                  "score_matrix_kernel launch at q400 x 2,000 profiles with 32 "
                                  "rows per block, scaled by cells and, for the %d-row variant "
                                  "in use, by the database reads per block "
                                  "(profiles/score_matrix_kernel_q400_db2k.md)" % rows,
                "kernel": "score_matrix_kernel",
                "peak_source": "148 SMs x 128 FP32 lanes x max SM clock (nominal issue rate)",
                "hbm_bytes_per_launch": float(Lq) * Ndb * 8,
                "hbm_peak_gbs": (peaks or {}).get("hbm_gbs")}
        if args.ddmswgt <= 0:
            # without DDMS the phase-1 DP weighs more: its ALU roofline at 37
            # algorithmic ops per cell (23 adds, 9 maxima and 5 compares of
            # the 5-state cell, CuBatchDP_init_btck.cu:303-360)
            dp_ms = stage_acc[1] / steps
            achieved = 37.0 * Lq * Ndb / (dp_ms / 1e3) / 1e9
            roof = {"bound": "alu", "achieved": achieved, "peak": alu_peak, "unit": "Gop/s",
                    "frac": achieved / alu_peak, "traffic": None, "kernel": "dp1_kernel",
                    "peak_source": "148 SMs x 128 FP32 lanes x max SM clock (nominal issue rate)",
                    "hbm_bytes_per_launch": float(Lq) * Ndb * 5,
                    "hbm_peak_gbs": (peaks or {}).get("hbm_gbs")}
        line = {"metric": "GCUPS", "value": value, "unit": "GCUPS", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": kern_ms / steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic",
                "config": workload_config(args, q, db, world),
                "e2e": {"value": e2e, "unit": "GCUPS",
                        "h2d_bytes_per_step": int(Lq * (4 * 20 + 4 * 3 + 4 * 100 + 2) + 4 * 7 * (Lq + 1)),
                        "d2h_bytes_per_step": int(d2h)},
                "hits": nhits,
                "top50_digest": hashlib.sha1(
                    recs[order[:50], 1].view(np.uint32).tobytes()).hexdigest()[:16],
                "merged_hits": merged_hits if world > 1 else None,
                "stage_ms": {k: v / steps for k, v in zip(STAGES, stage_acc)},
                "gpu_launches": launches, "graph_launches": bp.graph_launches(),
                "tuning": bp.tuning(Lq), "roofline": roof, "clocks": clocks}
        if not args.no_cpu_baseline and world == 1:
            # the host-core baseline: rank 0 of a one-GPU run only
            line["cpu_baseline"] = cpu_baseline(q, db, ss, args.cpu_seconds, db_len, nseqs, args.cvswgt)
    bp.close()
    if rank == 0:
        if world == 1 and args.tc == "plain" and not args.no_tc_forms:
            # the precision forms on the same workload, after the timed run
            line["tc_forms"] = tc_forms(cb, ss, opts, q, db, db_len, nseqs, line["top50_digest"])
        if world == 1 and not args.no_serving and args.ndb is None and args.workload == DEFAULT_WORKLOAD:
            del q, db
            line["serving"] = serving_summary(cb, ss, args.seed)
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
