"""Profile data in the reference's structure-of-arrays field layout.

The search path receives profile data as 181 parallel field arrays, one
pointer per field, exactly as the reference's per-worker driver does
(``char** pmbeg``/``char** pmend``; field indices restated from
src/libmycu/cupro/PM2DVectorFields.h:51-87). :class:`ProfileSet` owns those
arrays as numpy buffers and hands out the pointer tables that the C-ABI
(``include/cother_b200.h``) takes.

Field groups (per profile P, per position N, per transition entry N+P):

* ``bkg``     [20][P] float32  background probabilities (pps2DBkgPrbs)
* ``eno``     [P]     float32  effective number of observations (pps2DENO)
* ``lens``    [P]     int32    profile lengths (pps2DLen)
* ``dist``    [P]     uint32   first position of each profile (pps2DDist)
* ``trn``     [7][N+P] float32 log transition probabilities (ptr2DTrnPrbs);
  entry ``dist[p]+p`` holds the beginning transitions of profile p and
  ``dist[p]+p+1+k`` those of its position k
* ``tf``      [20][N] float32  target frequencies (pmv2DTrgFrqs)
* ``dd``      [100][N] float32 distance list: slot 0 = count, 1..99 values,
  255 = no data (pmv2DDDvalues)
* ``ss``      [3][N]  float32  SS state probabilities (pmv2DSSsprbs)
* ``addrpro`` [N]     int32    profile index of each position (pmv2DAddrPro)
* ``aa``      [N]     int8     amino acid codes (pmv2Daa)
* ``ssstate`` [N]     int8     SS state codes (pmv2DSSstate)

Context-vector and HDP fields are carried as zero-filled arrays: the terms
that use them are off on this path.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

# field indices (src/libmycu/cupro/PM2DVectorFields.h:51-87)
NUMAA = 20
NCVELS = 19
NSSSTATES = 3
NTRN = 7
NDSTSLOTS = 100
PPS_BKGPRBS = 0
PPS_ENO = PPS_BKGPRBS + NUMAA          # 20
PPS_LEN = PPS_ENO + 1                  # 21
PPS_DIST = PPS_LEN + 1                 # 22
PTR_TRNPRBS = PPS_DIST + 1             # 23
PMV_TRGFRQS = PTR_TRNPRBS + NTRN       # 30
PMV_CVENTRS = PMV_TRGFRQS + NUMAA      # 50
PMV_CVPRIOR = PMV_CVENTRS + NCVELS     # 69
PMV_CVNORM2 = PMV_CVPRIOR + 1          # 70
PMV_DDVALUES = PMV_CVNORM2 + 1         # 71
PMV_SSSPRBS = PMV_DDVALUES + NDSTSLOTS  # 171
PMV_HDP1PRB = PMV_SSSPRBS + NSSSTATES  # 174
PMV_HDP1IND = PMV_HDP1PRB + 1          # 175
PMV_ADDRPRO = PMV_HDP1IND + 1          # 176
PMV_ADDRCV = PMV_ADDRPRO + 1           # 177
PMV_ADDRSS = PMV_ADDRCV + 1            # 178
PMV_AA = PMV_ADDRSS + 1                # 179
PMV_SSSTATE = PMV_AA + 1               # 180
NFIELDS = PMV_SSSTATE + 1              # 181

DST_NODATA = 255.0

# amino acids are stored as letters, SS states as ' ', 'e', 'h'
# (src/liblib/alpha.cpp:12-14)
AA_ALPHABET = "ARNDCQEGHILKMFPSTWYV"
SS_CODES = " eh"


@dataclass
class ProfileSet:
    """A batch of profiles held in the reference's SoA field layout."""

    lens: np.ndarray
    bkg: np.ndarray
    eno: np.ndarray
    trn: np.ndarray
    tf: np.ndarray
    dd: np.ndarray
    ss: np.ndarray
    addrpro: np.ndarray
    aa: np.ndarray
    ssstate: np.ndarray
    names: list = field(default_factory=list)
    # context vectors (optional): [19][N] entries, their prior log
    # probabilities and squared norms [N]; zeros are passed when absent
    cv: np.ndarray | None = None
    cvprior: np.ndarray | None = None
    cvnorm2: np.ndarray | None = None
    _keep: list = field(default_factory=list, repr=False)

    def __post_init__(self):
        self.lens = np.ascontiguousarray(self.lens, dtype=np.int32)
        self.dist = np.zeros(len(self.lens), dtype=np.uint32)
        if len(self.lens) > 1:
            self.dist[1:] = np.cumsum(self.lens[:-1], dtype=np.int64).astype(np.uint32)
        self._zero_n = None

    @property
    def nprofiles(self) -> int:
        return int(len(self.lens))

    @property
    def npositions(self) -> int:
        return int(self.lens.sum(dtype=np.int64))

    @property
    def starts(self) -> np.ndarray:
        return self.dist.astype(np.int64)

    def subset(self, first: int, count: int) -> "ProfileSet":
        """Profiles [first, first+count) as a new set (copies)."""
        s0 = int(self.starts[first])
        n = int(self.lens[first:first + count].sum(dtype=np.int64))
        t0 = s0 + first
        nt = n + count
        return ProfileSet(
            lens=self.lens[first:first + count].copy(),
            bkg=np.ascontiguousarray(self.bkg[:, first:first + count]),
            eno=self.eno[first:first + count].copy(),
            trn=np.ascontiguousarray(self.trn[:, t0:t0 + nt]),
            tf=np.ascontiguousarray(self.tf[:, s0:s0 + n]),
            dd=np.ascontiguousarray(self.dd[:, s0:s0 + n]),
            ss=np.ascontiguousarray(self.ss[:, s0:s0 + n]),
            addrpro=(self.addrpro[s0:s0 + n] - first).astype(np.int32),
            aa=self.aa[s0:s0 + n].copy(),
            ssstate=self.ssstate[s0:s0 + n].copy(),
            names=list(self.names[first:first + count]) if self.names else [],
            cv=None if self.cv is None else np.ascontiguousarray(self.cv[:, s0:s0 + n]),
            cvprior=None if self.cvprior is None else self.cvprior[s0:s0 + n].copy(),
            cvnorm2=None if self.cvnorm2 is None else self.cvnorm2[s0:s0 + n].copy(),
        )

    def select(self, indices) -> "ProfileSet":
        """Profiles `indices` (in that order) as a new set (copies)."""
        idx = np.asarray(indices, dtype=np.int64)
        st = self.starts
        lens = self.lens[idx]
        pos = np.concatenate([np.arange(st[p], st[p] + self.lens[p]) for p in idx]) \
            if len(idx) else np.zeros(0, np.int64)
        tpos = np.concatenate([np.arange(st[p] + p, st[p] + p + self.lens[p] + 1) for p in idx]) \
            if len(idx) else np.zeros(0, np.int64)
        return ProfileSet(
            lens=lens.copy(),
            bkg=np.ascontiguousarray(self.bkg[:, idx]),
            eno=self.eno[idx].copy(),
            trn=np.ascontiguousarray(self.trn[:, tpos]),
            tf=np.ascontiguousarray(self.tf[:, pos]),
            dd=np.ascontiguousarray(self.dd[:, pos]),
            ss=np.ascontiguousarray(self.ss[:, pos]),
            addrpro=np.repeat(np.arange(len(idx), dtype=np.int32), lens),
            aa=self.aa[pos].copy(),
            ssstate=self.ssstate[pos].copy(),
            names=[self.names[p] for p in idx] if self.names else [],
            cv=None if self.cv is None else np.ascontiguousarray(self.cv[:, pos]),
            cvprior=None if self.cvprior is None else self.cvprior[pos].copy(),
            cvnorm2=None if self.cvnorm2 is None else self.cvnorm2[pos].copy(),
        )

    def field_tables(self):
        """(beg, end) arrays of 181 host pointers, as the reference passes them.

        Pointers stay valid while this ProfileSet is alive.
        """
        N, P = self.npositions, self.nprofiles
        if self._zero_n is None or len(self._zero_n) < N:
            self._zero_n = np.zeros(max(N, 1), dtype=np.float32)
        z = self._zero_n
        beg = (ctypes.c_void_p * NFIELDS)()
        end = (ctypes.c_void_p * NFIELDS)()

        def put(f, arr, nbytes):
            a = arr.ctypes.data
            beg[f] = a
            end[f] = a + nbytes

        for a in range(NUMAA):
            put(PPS_BKGPRBS + a, self.bkg[a], 4 * P)
        put(PPS_ENO, self.eno, 4 * P)
        put(PPS_LEN, self.lens, 4 * P)
        put(PPS_DIST, self.dist, 4 * P)
        for t in range(NTRN):
            put(PTR_TRNPRBS + t, self.trn[t], 4 * (N + P))
        for a in range(NUMAA):
            put(PMV_TRGFRQS + a, self.tf[a], 4 * N)
        if self.cv is not None:
            for c in range(NCVELS):
                put(PMV_CVENTRS + c, self.cv[c], 4 * N)
            put(PMV_CVPRIOR, self.cvprior, 4 * N)
            put(PMV_CVNORM2, self.cvnorm2, 4 * N)
        else:
            for c in range(NCVELS):
                put(PMV_CVENTRS + c, z, 4 * N)
            put(PMV_CVPRIOR, z, 4 * N)
            put(PMV_CVNORM2, z, 4 * N)
        for s in range(NDSTSLOTS):
            put(PMV_DDVALUES + s, self.dd[s], 4 * N)
        for s in range(NSSSTATES):
            put(PMV_SSSPRBS + s, self.ss[s], 4 * N)
        put(PMV_HDP1PRB, z, 4 * N)
        put(PMV_HDP1IND, z, 4 * N)
        put(PMV_ADDRPRO, self.addrpro, 4 * N)
        put(PMV_ADDRCV, z, 4 * N)
        put(PMV_ADDRSS, z, 4 * N)
        put(PMV_AA, self.aa, N)
        put(PMV_SSSTATE, self.ssstate, N)
        return beg, end

    def dd_lists(self) -> np.ndarray:
        """Distance lists as uint8 [N][100] (slot 0 = count, 255 = no data)."""
        return np.ascontiguousarray(self.dd.T).astype(np.uint8)

    def sequence(self, p: int) -> str:
        s0 = int(self.starts[p])
        return bytes(self.aa[s0:s0 + int(self.lens[p])].astype(np.uint8)).decode()
