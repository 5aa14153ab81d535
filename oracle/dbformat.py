"""Oracle (test infrastructure only): a numpy restatement of the layout of
the reference's binary profile database, format v2.2, to check the
library's writer and reader (cother_b200/csrc/dbfile.cpp) byte for byte.

  header   Db::WriteBinaryHeader (src/libpro/srcpro/Db.cpp:707-715):
           "COTHER profile bin database v" "2.5", size_t #profiles,
           uint64 #positions, uint64 #distance values
  table    CalculateAndWriteAddressTable_v2_2
           (src/libpro/srcpro/PMProfileModel.cpp:1250-1336): the file
           address of each section, in the order below
  sections BinaryWriteProfile_v2_2 (PMProfileModel.cpp:1350-1810), each the
           whole database's values of one field: lengths (int), ENOs,
           backgrounds x20 (per profile); transitions x7 (per profile and
           position: a beginning vector per profile); target frequencies x20,
           context vectors x19, CV prior, CV norm, distances x100 (slot 0 the
           count), SS probabilities x3, HDP1 probability (float), HDP1 index
           (int), residues (char), SS states (char) (per position); the end
           addresses of the descriptions (size_t); the NUL-terminated
           descriptions
"""
from __future__ import annotations

import numpy as np

SIGNATURE = b"COTHER profile bin database v"
VERSION = b"2.5"


def v22_bytes(ps, descs) -> bytes:
    """The file the reference's db2bin would write for ProfileSet `ps`
    (whose fields hold the values its reader produces)."""
    P, N = ps.nprofiles, ps.npositions
    z = np.zeros(N, np.float32)
    cv = ps.cv if ps.cv is not None else np.zeros((19, N), np.float32)
    cvp = ps.cvprior if ps.cvprior is not None else z
    cvn = ps.cvnorm2 if ps.cvnorm2 is not None else z
    sections = [np.asarray(ps.lens, np.int32), np.asarray(ps.eno, np.float32)]
    sections += [np.asarray(ps.bkg[r], np.float32) for r in range(20)]
    sections += [np.asarray(ps.trn[t], np.float32) for t in range(7)]
    sections += [np.asarray(ps.tf[r], np.float32) for r in range(20)]
    sections += [np.asarray(cv[t], np.float32) for t in range(19)]
    sections += [np.asarray(cvp, np.float32), np.asarray(cvn, np.float32)]
    sections += [np.asarray(ps.dd[t], np.float32) for t in range(100)]
    sections += [np.asarray(ps.ss[t], np.float32) for t in range(3)]
    sections += [z, np.zeros(N, np.int32), np.asarray(ps.aa, np.int8), np.asarray(ps.ssstate, np.int8)]
    nsec = len(sections) + 2
    head = len(SIGNATURE) + len(VERSION) + 24
    addr = head + 8 * nsec
    table = []
    for s in sections:
        table.append(addr)
        addr += s.nbytes
    table.append(addr)          # description end addresses
    addr += 8 * P
    table.append(addr)          # descriptions
    d = [(x or "").encode() + b"\0" for x in descs]
    ends = np.cumsum([len(x) for x in d]) + addr
    ndst = int(np.asarray(ps.dd[0], np.float64).astype(np.int64).sum())
    out = [SIGNATURE, VERSION, np.array([P, N, ndst], np.uint64).tobytes(),
           np.array(table, np.uint64).tobytes()]
    out += [s.tobytes() for s in sections]
    out += [np.asarray(ends, np.uint64).tobytes()] + d
    return b"".join(out)
