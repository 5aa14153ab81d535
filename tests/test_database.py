"""Binary profile database files (the reference's format v2.2) on the CPU:
the library's writer produces the reference layout byte for byte (as the
oracle restates it), and its reader hands out chunks whose fields equal the
profile set's, with descriptions; malformed files are rejected."""
import os

import numpy as np
import pytest

from oracle import dbformat


@pytest.fixture(scope="module")
def profile_db():
    from cother_b200 import synth
    db = synth.make_profiles([35, 120, 8, 64, 250, 31, 77], 4401, False)
    synth.add_context_vectors(db, 4402)
    descs = ["d1abc_ protein kinase", "", "x" * 300, "tab\tand \"quotes\"", "p5", "p6 / slash", "last one"]
    return db, descs


def _fields(ps):
    from cother_b200.profiles import (PMV_AA, PMV_DDVALUES, PMV_SSSPRBS, PMV_SSSTATE, PMV_TRGFRQS, PPS_BKGPRBS,
                                      PPS_ENO, PPS_LEN, PTR_TRNPRBS)
    out = {PPS_LEN: np.asarray(ps.lens, np.int32), PPS_ENO: np.asarray(ps.eno, np.float32),
           PMV_AA: np.asarray(ps.aa, np.int8), PMV_SSSTATE: np.asarray(ps.ssstate, np.int8)}
    for r in range(20):
        out[PPS_BKGPRBS + r] = np.asarray(ps.bkg[r], np.float32)
        out[PMV_TRGFRQS + r] = np.asarray(ps.tf[r], np.float32)
    for t in range(7):
        out[PTR_TRNPRBS + t] = np.asarray(ps.trn[t], np.float32)
    for t in range(100):
        out[PMV_DDVALUES + t] = np.asarray(ps.dd[t], np.float32)
    for t in range(3):
        out[PMV_SSSPRBS + t] = np.asarray(ps.ss[t], np.float32)
    return out


def test_writer_matches_reference_layout(tmp_path, profile_db):
    from cother_b200 import database
    db, descs = profile_db
    path = str(tmp_path / "db.tbin")
    database.write_database(path, db, descs)
    with open(path, "rb") as f:
        data = f.read()
    assert data == dbformat.v22_bytes(db, descs)
    assert data.startswith(b"COTHER profile bin database v2.5")


@pytest.mark.parametrize("first,count", [(0, 7), (0, 1), (2, 3), (4, 3), (6, 1)])
def test_reader_chunks_equal_profile_subsets(tmp_path, profile_db, first, count):
    from cother_b200 import database
    from cother_b200.profiles import PMV_ADDRPRO, PMV_ADDRSS, PPS_DIST
    db, descs = profile_db
    path = str(tmp_path / "db.tbin")
    database.write_database(path, db, descs)
    with database.Database(path) as d:
        assert (d.nprofiles, d.npositions) == (7, db.npositions)
        assert d.ndistances == int(np.asarray(db.dd[0]).astype(np.int64).sum())
        assert np.array_equal(d.lengths(), db.lens)
        _, _, got_descs = d.chunk(first, count)
        assert got_descs == descs[first:first + count]
        sub = db.subset(first, count)
        for f, want in _fields(sub).items():
            assert np.array_equal(d.field(f, want.dtype), want), f
        assert np.array_equal(d.field(PPS_DIST, np.uint32), np.asarray(sub.starts, np.uint32))
        assert np.array_equal(d.field(PMV_ADDRPRO, np.int32), np.repeat(np.arange(count), sub.lens))
        assert np.array_equal(d.field(PMV_ADDRSS, np.int32), np.arange(sub.npositions))


def test_chunk_planning(tmp_path, profile_db):
    from cother_b200 import database
    db, descs = profile_db
    path = str(tmp_path / "db.tbin")
    database.write_database(path, db, descs)
    with database.Database(path) as d:
        for cap in (1, 100, 200, 10**6):
            ch = d.chunks(cap)
            assert [c[0] for c in ch] == sorted(c[0] for c in ch)
            assert sum(c[1] for c in ch) == 7
            for first, count in ch:
                n = int(db.lens[first:first + count].sum())
                assert n <= cap or count == 1


def test_malformed_files_are_rejected(tmp_path, profile_db):
    from cother_b200 import CbpError, database
    db, descs = profile_db
    good = dbformat.v22_bytes(db, descs)
    cases = {
        "signature": b"XOTHER" + good[6:],
        "version": good[:29] + b"9.9" + good[32:],
        "truncated": good[: len(good) // 2],
        "header_only": good[:40],
        "length": None,
    }
    bad_len = bytearray(good)
    table0 = int(np.frombuffer(good[56:64], np.uint64)[0])
    bad_len[table0:table0 + 4] = np.int32(0).tobytes()
    cases["length"] = bytes(bad_len)
    for name, data in cases.items():
        p = tmp_path / ("bad_" + name)
        p.write_bytes(data)
        with pytest.raises(CbpError):
            database.Database(str(p))
    with pytest.raises(CbpError):
        database.Database(str(tmp_path / "missing.tbin"))
    p = tmp_path / "ok.tbin"
    p.write_bytes(good)
    with database.Database(str(p)) as d:
        with pytest.raises(CbpError):
            d.chunk(5, 3)
        with pytest.raises(CbpError):
            d.chunk(0, 0)
