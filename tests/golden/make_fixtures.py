"""Generate the committed fixtures under tests/golden/ from the reference tree.

Run in a container that has the reference checkout (default
/root/reference). The GPU box has no reference tree, so everything the
tests and the benchmark need from it is committed:

* ssss.npy       -- the SS score table of src/env/ssss (30x30, full
                    symmetric, float32 as parsed by the reference's
                    VirtScores::ReadScoresHelper, src/libpro/srcpro/VirtScores.cpp:44)
* nn_weights.npy -- the 93 parameters of the significance networks and the
                    SS18 adjustments (static table SSE_NN_WEIGHTS_ of
                    src/libmycu/cupro/CuDeviceMemory.cu:43-80)
* cother_par.json -- the [UNGAPPED] and [GAPPED_A_1] lambda, K, alpha, beta
                    of src/env/cother.par
* ddms_ref.npz   -- DDMS golden vectors: seeded list pairs and the value
                    returned by the reference's own CPU restatement
                    (cother-scores-optimizer/ddms.cxx:388-436, built by
                    oracle/Makefile into oracle/_ref/), rint(16 * top-3 sum)
* cvs2s.npz      -- the context-vector score map of src/env/cvs2s as the
                    reference's reader leaves it (keys, smoothed scores and
                    the shift; see parse_cvs2s)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
REF = os.environ.get("COTHER_REFERENCE", "/root/reference")


def parse_ssss(path):
    lines = open(path).read().splitlines()
    i = next(k for k, ln in enumerate(lines) if ln.startswith("Cardinality"))
    card = int(lines[i].split("=")[1])
    T = np.zeros((card, card), np.float32)
    for r in range(card):
        vals = [np.float32(v) for v in lines[i + 1 + r].split()]
        assert len(vals) == r + 1, (r, len(vals))
        for c, v in enumerate(vals):
            T[r, c] = v
            T[c, r] = v
    return T


CVS_PLUS = np.float32(9999.0)   # the reader's value for a '+' score (CVS2Scores.cpp:39)


def smooth_cvs_scores(keys, scos):
    """CVS2Scores::SmoothScores (src/libpro/srcpro/CVS2Scores.cpp:366-460)
    in float32: every score becomes the running average of 5 scores
    ('+' entries skipped, the first two and the trailing ones take the
    nearest full window), then keys missing from the 1/2 grid are inserted
    with the previous smoothed score. Returns (keys, scores, shift), shift
    being the number of negative keys."""
    f32 = np.float32
    n_ = len(scos)
    plus = lambda v: CVS_PLUS <= v
    smth = [f32(0)] * n_
    rwin = [f32(0)] * 5
    rsum, avg = f32(0), f32(0)
    nv = rn = nn = 0
    for n in range(n_):
        sc = scos[n]
        if nv < 2:
            nn += 1
        if not plus(sc):
            if 5 <= rn:
                rn = 0
            rsum = f32(rsum - rwin[rn])
            rwin[rn] = sc
            rn += 1
            rsum = f32(rsum + sc)
            avg = f32(rsum / f32(5))
            nv += 1
        if 5 <= nv:
            if not plus(sc):
                if nv == 5:
                    for p in range(nn):
                        smth[p] = avg
                smth[nn] = avg
                nn += 1
                while plus(scos[nn]) and nn < n:
                    smth[nn] = avg
                    nn += 1
            if n_ == n + 1:
                for p in range(nn, n_):
                    smth[p] = avg
    scos = list(scos)
    sm = f32(0)
    for n in range(n_ - 1, max(-1, n_ - 9999 - 1), -1):   # all: nSLAST = 9999
        sm = smth[n]
        scos[n] = sm
    keys = list(keys)
    incr = f32(0.5)
    pkk = f32(0)
    n = 0
    while n < len(keys):
        kk, sc = keys[n], scos[n]
        if n and kk <= pkk:
            raise ValueError("CVS keys are not sorted")
        if n and incr < f32(kk - pkk):
            pkk = f32(pkk + incr)
            keys.insert(n, pkk)
            scos.insert(n, sm)
            smth.insert(n, sm)
            n += 1
            continue
        pkk = kk
        sm = smth[n]
        if plus(sc):
            scos[n] = sm
        n += 1
    shift = next((i for i, k in enumerate(keys) if f32(0) <= k), len(keys))
    return np.array(keys, np.float32), np.array(scos, np.float32), shift


def parse_cvs2s(path):
    """The single table of src/env/cvs2s (one level of effective sequence
    numbers, read by CVS2Scores::ReadScoresHelper,
    src/libpro/srcpro/CVS2Scores.cpp:206-357), smoothed as the reader does."""
    lines = open(path).read().splitlines()
    i = next(k for k, ln in enumerate(lines) if ln.strip().startswith("Cardinality"))
    card = int(lines[i].split("=")[1])
    rest = [ln for ln in lines[i + 1:] if ln.strip() and not ln.lstrip().startswith("#")]
    keys = [np.float32(v) for v in rest[0].split()[:card]]
    scos = [CVS_PLUS if v == "+" else np.float32(v) for v in rest[1].split()[:card]]
    assert len(keys) == card and len(scos) == card
    return smooth_cvs_scores(keys, scos)


def parse_nn_weights(path):
    import re
    text = open(path).read()
    i = text.index("SSE_NN_WEIGHTS_[]")
    j = text.index("};", i)
    body = re.sub(r"//[^\n]*", "", text[i:j].split("{", 1)[1])
    vals = [np.float32(v.rstrip("f")) for v in re.findall(r"[-+]?[0-9]*\.?[0-9]+(?:[eE][-+]?[0-9]+)?f?", body)]
    w = np.array(vals, np.float32)
    assert len(w) == 93, len(w)
    return w


def parse_cother_par(path):
    out, sec = {}, None
    for ln in open(path):
        ln = ln.strip()
        if ln.startswith("["):
            sec = ln.strip("[]")
            out[sec] = {}
        elif "=" in ln and sec and not ln.startswith("#"):
            k, v = [x.strip() for x in ln.split("=", 1)]
            out[sec][k] = float(v)
    return out


def ddms_vectors(n_pairs=400, seed=99):
    from oracle import oracle as O
    from cother_b200 import synth
    O.build()
    R = O.ref_lib()
    assert R is not None, "reference DDMS library not built"
    q = synth.make_profiles([180], seed, True)
    d = synth.make_profiles([160, 90, 40], seed + 1, False)
    ql, dl = q.dd_lists(), d.dd_lists()
    rng = np.random.default_rng(seed)
    qi = rng.integers(0, len(ql), n_pairs)
    di = rng.integers(0, len(dl), n_pairs)
    out = []
    for a, b in zip(qi, di):
        x = np.full(110, 255, np.int32); x[:ql[a][0] + 1] = ql[a][:ql[a][0] + 1]
        y = np.full(110, 255, np.int32); y[:dl[b][0] + 1] = dl[b][:dl[b][0] + 1]
        out.append(R.ref_ddms_scaled_sum(x.ctypes.data, y.ctypes.data))
    return ql[qi], dl[di], np.array(out, np.float32)


if __name__ == "__main__":
    T = parse_ssss(os.path.join(REF, "src/env/ssss"))
    np.save(os.path.join(HERE, "ssss.npy"), T)
    np.save(os.path.join(HERE, "nn_weights.npy"),
            parse_nn_weights(os.path.join(REF, "src/libmycu/cupro/CuDeviceMemory.cu")))
    import json
    par = parse_cother_par(os.path.join(REF, "src/env/cother.par"))
    json.dump({k: par[k] for k in ("UNGAPPED", "GAPPED_A_1")},
              open(os.path.join(HERE, "cother_par.json"), "w"), indent=1)
    ck, cs, cshift = parse_cvs2s(os.path.join(REF, "src/env/cvs2s"))
    np.savez(os.path.join(HERE, "cvs2s.npz"), keys=ck, scores=cs, shift=np.int32(cshift))
    print("cvs2s", len(ck), "keys", float(ck[0]), "..", float(ck[-1]), "shift", cshift)
    qa, da, ref = ddms_vectors()
    np.savez_compressed(os.path.join(HERE, "ddms_ref.npz"), qlists=qa, dlists=da, ref=ref)
    print("ssss", T.shape, "ddms pairs", len(ref), "scored", int((ref != -777).sum()))
