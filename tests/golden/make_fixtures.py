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
    qa, da, ref = ddms_vectors()
    np.savez_compressed(os.path.join(HERE, "ddms_ref.npz"), qlists=qa, dlists=da, ref=ref)
    print("ssss", T.shape, "ddms pairs", len(ref), "scored", int((ref != -777).sum()))
