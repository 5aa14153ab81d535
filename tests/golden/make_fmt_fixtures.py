"""Golden vectors of the reference's description formatters.

Runs FormatDescription and FormatDescriptionJSON (src/liblib/fmtdescription.h,
compiled from the reference's source by `make -C oracle fmtref` into
oracle/_ref/libfmtref.so) on seeded descriptions and writes
tests/golden/fmt_desc_ref.json. Needs the reference checkout; the committed
JSON is what the tests read.

Usage: python tests/golden/make_fmt_fixtures.py
"""
import ctypes
import json
import os
import random
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def descriptions(seed: int = 2024, n: int = 60):
    rng = random.Random(seed)
    alphabet = "abcdefghijklmnopqrstuvwxyzABCDEFGHIJKLMNOPQRSTUVWXYZ0123456789_-.,:;()[]|"
    out = ["", " ", "single", "  leading and trailing  ", "tab\tseparated\t\twords",
           "quote \"inside\" and back\\slash / slash", "x" * 150, "a " * 80]
    while len(out) < n:
        words = []
        for _ in range(rng.randint(1, 40)):
            w = "".join(rng.choice(alphabet) for _ in range(rng.choice([1, 2, 3, 5, 8, 13, 21, 34])))
            if rng.random() < 0.1:
                w = w[:1] + rng.choice('"\\/') + w[1:]
            words.append(w)
        seps = [rng.choice([" ", " ", " ", "  ", "\t", " \t "]) for _ in words]
        s = "".join(w + sp for w, sp in zip(words, seps))
        if rng.random() < 0.5:
            s = s.rstrip()
        if rng.random() < 0.2:
            s = rng.choice([" ", "\n", "\t\r "]) + s
        out.append(s)
    return out


def main():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "fmtref"], check=True)
    L = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libfmtref.so"))
    L.ref_format_description.restype = ctypes.c_int
    L.ref_format_description.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int, ctypes.c_char, ctypes.c_void_p]
    L.ref_format_description_json.restype = ctypes.c_int
    L.ref_format_description_json.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    # the formatters mark a cut by rewriting the 3 bytes before their output
    # position, which can lie before the output they wrote: keep a margin
    pad = 16

    def fd(d, maxoutlen, indent, width, outpos, linepos, sep):
        buf = ctypes.create_string_buffer(maxoutlen * (indent + 2) + 64 + pad)
        n = L.ref_format_description(d.encode(), maxoutlen, indent, width, outpos, linepos,
                                     sep.encode() if sep else b"\0", ctypes.addressof(buf) + pad)
        return buf.raw[pad:pad + n].decode()

    def fdj(d, maxoutlen, outpos):
        buf = ctypes.create_string_buffer(2 * maxoutlen + 64 + pad)
        n = L.ref_format_description_json(d.encode(), maxoutlen, outpos, ctypes.addressof(buf) + pad)
        return buf.raw[pad:pad + n].decode()

    rng = random.Random(77)
    cases = []
    for d in descriptions():
        c = {"desc": d,
             # the finalizer's uses (CuBatchProcessingFinalizerPlain.cpp:100-123,
             # CuBatchProcessingFinalizerJSON.cpp:108-122): annotation, hit record
             "annot_plain": fd(d, 75, 0, 75, 0, 0, ""),
             "rec_plain_1024_80": fd(d, 1024, 13, 80, 0, 0, ">"),
             "rec_plain_60_30": fd(d, 60, 13, 30, 0, 0, ">"),
             "annot_json": fdj(d, 75, 0),
             "rec_json_1024": fdj(d, 1024, 0),
             "rec_json_60": fdj(d, 60, 0),
             "generic": []}
        for _ in range(6):
            m = rng.choice([3, 4, 10, 20, 75, 100, 1024])
            ind = rng.choice([0, 13])
            w = rng.choice([1, 14, 30, 75, 80, 2000])
            op = rng.choice([0, 0, 5])
            lp = rng.choice([0, 0, 7])
            sep = rng.choice(["", ">"])
            c["generic"].append({"args": [m, ind, w, op, lp, sep], "out": fd(d, m, ind, w, op, lp, sep)})
            mj = rng.choice([3, 4, 10, 20, 75, 1024])
            opj = rng.choice([0, 0, 6])
            c["generic"].append({"json_args": [mj, opj], "out": fdj(d, mj, opj)})
        cases.append(c)
    with open(os.path.join(HERE, "fmt_desc_ref.json"), "w") as f:
        json.dump(cases, f, indent=0)
    print(len(cases), "cases")


if __name__ == "__main__":
    main()
