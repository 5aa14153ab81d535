// Binary profile database files: the reference's format v2.2
// ("COTHER profile bin database v2.5", made by db2bin,
// src/db2bin/db2bin.cpp:131 -> Db::MakeBin_v2_2, src/libpro/srcpro/Db.cpp:340-385).
//
// The file is the database's structure of arrays: a header (signature,
// version, #profiles, #positions, #distance values;
// Db::WriteBinaryHeader, Db.cpp:707-715), an address table of the sections
// (CalculateAndWriteAddressTable_v2_2,
// src/libpro/srcpro/PMProfileModel.cpp:1250-1336) and one section per
// profile field -- lengths, ENOs, 20 backgrounds, 7 transitions (P+N
// entries: a beginning vector per profile), 20 target frequencies, 19
// context-vector entries, their priors and norms, 100 distance slots (slot 0
// the count), 3 SS probabilities, HDP1 probability and index, residues, SS
// states -- then the end addresses of the descriptions and the descriptions
// (BinaryWriteProfile_v2_2, PMProfileModel.cpp:1350-1810).
//
// Reading maps the file and hands out chunks of whole profiles as the 181
// begin/end field pointers that cbp_transfer_chunk takes, the stored
// sections in place and the derived fields (offsets, profile addresses, SS
// addresses) computed -- what TdDataReader::ReadDataChunkHelper assembles by
// copying (src/libmycu/cupro/TdDataReader.cpp:703-984). Writing is the
// reverse, from a field table, for databases built elsewhere than with db2bin.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "cother_b200.h"

namespace cbp {
void set_last_error(const std::string& msg);
}

namespace {

// field indices (src/libmycu/cupro/PM2DVectorFields.h:51-87)
enum {
    fBkg = 0, fENO = 20, fLen = 21, fDist = 22, fTrn = 23, fTF = 30, fCV = 50, fCVprior = 69, fCVnorm2 = 70,
    fDD = 71, fSS = 171, fHDP1prb = 174, fHDP1ind = 175, fAddrPro = 176, fAddrCV = 177, fAddrSS = 178,
    fAA = 179, fSSstate = 180, fTot = 181
};
constexpr int kNAA = 20, kNTrn = 7, kNCV = 19, kNDst = 100, kNSS = 3;
// sections of the address table in file order (v2_2_NSECTIONS,
// src/libpro/srcpro/PMProfileModel.h:42-49): one per stored field, then the
// description end addresses and the descriptions
constexpr int kNStored = 1 + 1 + kNAA + kNTrn + kNAA + kNCV + 1 + 1 + kNDst + kNSS + 1 + 1 + 1 + 1;
constexpr int kNSections = kNStored + 2;

const char kSignature[] = "COTHER profile bin database v";   // Db::patstrDBBINVER (Db.cpp:699)
const char kVersion[] = "2.5";                               // PMProfileModel::bindataversion (PMProfileModel.cpp:42)

struct Section {
    int field;      // profile field
    int per;        // 0: per profile, 1: per position, 2: per profile + per position
    int esz;        // element size
};

std::vector<Section> stored_sections()
{
    std::vector<Section> s;
    s.push_back({fLen, 0, 4});
    s.push_back({fENO, 0, 4});
    for (int r = 0; r < kNAA; r++) s.push_back({fBkg + r, 0, 4});
    for (int t = 0; t < kNTrn; t++) s.push_back({fTrn + t, 2, 4});
    for (int r = 0; r < kNAA; r++) s.push_back({fTF + r, 1, 4});
    for (int t = 0; t < kNCV; t++) s.push_back({fCV + t, 1, 4});
    s.push_back({fCVprior, 1, 4});
    s.push_back({fCVnorm2, 1, 4});
    for (int t = 0; t < kNDst; t++) s.push_back({fDD + t, 1, 4});
    for (int t = 0; t < kNSS; t++) s.push_back({fSS + t, 1, 4});
    s.push_back({fHDP1prb, 1, 4});
    s.push_back({fHDP1ind, 1, 4});
    s.push_back({fAA, 1, 1});
    s.push_back({fSSstate, 1, 1});
    return s;
}

struct DbError {
    int code;
    std::string msg;
};

size_t header_bytes() { return (sizeof(kSignature) - 1) + (sizeof(kVersion) - 1) + 8 + 8 + 8; }

}  // namespace

struct cbp_db {
    int fd = -1;
    const char* map = nullptr;
    size_t size = 0;
    uint64_t nprof = 0, npos = 0, ndst = 0;
    size_t addr[kNSections] = {};
    std::vector<long long> pstart;   // first position of each profile
    // chunk buffers of the derived fields
    std::vector<uint32_t> dist;
    std::vector<int> addrpro, addrcv, addrss;
    std::vector<const char*> descs;
    ~cbp_db()
    {
        if (map) munmap((void*)map, size);
        if (fd >= 0) close(fd);
    }
};

namespace {

template <class F>
int guarded_db(F&& f)
{
    try {
        f();
        cbp::set_last_error("");
        return CBP_OK;
    } catch (const DbError& e) {
        cbp::set_last_error(e.msg);
        return e.code;
    } catch (const std::exception& e) {
        cbp::set_last_error(e.what());
        return CBP_ERR_ARG;
    }
}

size_t section_count(const Section& s, uint64_t P, uint64_t N)
{
    return s.per == 0 ? P : s.per == 1 ? N : N + P;
}

// ReadBinaryHeader and OpenAndReadPreamble
// (src/libmycu/cupro/CuDbReader.cpp:457-519, TdDataReader.cpp:387-470)
void read_preamble(cbp_db& db)
{
    const char* p = db.map;
    const size_t need = header_bytes() + kNSections * sizeof(size_t);
    if (db.size < need) throw DbError{CBP_ERR_ARG, "database file too short for its header"};
    if (std::strncmp(p, kSignature, sizeof(kSignature) - 1))
        throw DbError{CBP_ERR_ARG, "not a binary profile database (wrong signature)"};
    p += sizeof(kSignature) - 1;
    if (std::strncmp(p, kVersion, sizeof(kVersion) - 1))
        throw DbError{CBP_ERR_ARG, "binary profile database of another version"};
    p += sizeof(kVersion) - 1;
    std::memcpy(&db.nprof, p, 8);
    std::memcpy(&db.npos, p + 8, 8);
    std::memcpy(&db.ndst, p + 16, 8);
    p += 24;
    if (db.nprof < 1) throw DbError{CBP_ERR_ARG, "invalid number of profiles"};
    if (db.npos < 1) throw DbError{CBP_ERR_ARG, "invalid database size"};
    std::memcpy(db.addr, p, sizeof(db.addr));
    const std::vector<Section> secs = stored_sections();
    for (int k = 0; k < kNSections; k++) {
        if (db.addr[k] >= db.size) throw DbError{CBP_ERR_ARG, "address table points outside the file"};
        if (k < kNStored) {
            const size_t bytes = section_count(secs[k], db.nprof, db.npos) * secs[k].esz;
            if (db.addr[k] + bytes > db.size) throw DbError{CBP_ERR_ARG, "section extends past the end of the file"};
        }
    }
    const size_t ends = db.addr[kNStored];
    if (ends + db.nprof * sizeof(size_t) > db.size)
        throw DbError{CBP_ERR_ARG, "description addresses extend past the end of the file"};
    // lengths and their sum
    const int* lens = reinterpret_cast<const int*>(db.map + db.addr[0]);
    db.pstart.resize(db.nprof + 1);
    long long acc = 0;
    for (uint64_t k = 0; k < db.nprof; k++) {
        int len;
        std::memcpy(&len, lens + k, 4);
        if (len < 1 || len >= 65536) throw DbError{CBP_ERR_ARG, "invalid profile length in the database"};
        db.pstart[k] = acc;
        acc += len;
    }
    db.pstart[db.nprof] = acc;
    if ((uint64_t)acc != db.npos) throw DbError{CBP_ERR_ARG, "profile lengths do not sum to the database size"};
    // description end addresses: increasing, within the file
    size_t prev = db.addr[kNStored + 1];
    for (uint64_t k = 0; k < db.nprof; k++) {
        size_t e;
        std::memcpy(&e, db.map + ends + k * sizeof(size_t), sizeof(size_t));
        if (e <= prev || e > db.size) throw DbError{CBP_ERR_ARG, "invalid description address"};
        if (db.map[e - 1] != '\0') throw DbError{CBP_ERR_ARG, "description not terminated"};
        prev = e;
    }
}

}  // namespace

extern "C" {

int cbp_db_open(const char* path, cbp_db** out)
{
    if (out) *out = nullptr;
    cbp_db* db = nullptr;
    const int rc = guarded_db([&] {
        if (!path || !out) throw DbError{CBP_ERR_ARG, "null argument"};
        db = new cbp_db();
        db->fd = ::open(path, O_RDONLY);
        if (db->fd < 0) throw DbError{CBP_ERR_ARG, std::string("cannot open ") + path};
        struct stat st;
        if (fstat(db->fd, &st) != 0) throw DbError{CBP_ERR_ARG, std::string("cannot stat ") + path};
        db->size = (size_t)st.st_size;
        if (db->size == 0) throw DbError{CBP_ERR_ARG, "empty database file"};
        void* m = mmap(nullptr, db->size, PROT_READ, MAP_PRIVATE, db->fd, 0);
        if (m == MAP_FAILED) throw DbError{CBP_ERR_ARG, std::string("cannot map ") + path};
        db->map = static_cast<const char*>(m);
        read_preamble(*db);
    });
    if (rc != CBP_OK) {
        delete db;
        return rc;
    }
    *out = db;
    return CBP_OK;
}

int cbp_db_close(cbp_db* db)
{
    delete db;
    return CBP_OK;
}

int cbp_db_info(cbp_db* db, uint64_t* nprofiles, uint64_t* npositions, uint64_t* ndistances)
{
    return guarded_db([&] {
        if (!db) throw DbError{CBP_ERR_ARG, "null database"};
        if (nprofiles) *nprofiles = db->nprof;
        if (npositions) *npositions = db->npos;
        if (ndistances) *ndistances = db->ndst;
    });
}

int cbp_db_profile_lengths(cbp_db* db, int32_t* lens)
{
    return guarded_db([&] {
        if (!db || !lens) throw DbError{CBP_ERR_ARG, "null argument"};
        std::memcpy(lens, db->map + db->addr[0], db->nprof * sizeof(int));
    });
}

int cbp_db_chunk(cbp_db* db, uint64_t first, uint64_t count, char** beg, char** end, const char** descs)
{
    return guarded_db([&] {
        if (!db || !beg || !end) throw DbError{CBP_ERR_ARG, "null argument"};
        if (count < 1 || first >= db->nprof || count > db->nprof - first)
            throw DbError{CBP_ERR_ARG, "profile range outside the database"};
        const uint64_t P = count;
        const long long pos0 = db->pstart[first], pos1 = db->pstart[first + count];
        const uint64_t N = (uint64_t)(pos1 - pos0);
        const std::vector<Section> secs = stored_sections();
        for (int f = 0; f < fTot; f++) beg[f] = end[f] = nullptr;
        for (int k = 0; k < kNStored; k++) {
            const Section& s = secs[k];
            const uint64_t off = s.per == 0 ? first : s.per == 1 ? (uint64_t)pos0 : first + (uint64_t)pos0;
            const char* b = db->map + db->addr[k] + off * s.esz;
            beg[s.field] = const_cast<char*>(b);
            end[s.field] = const_cast<char*>(b + section_count(s, P, N) * s.esz);
        }
        // derived fields (TdDataReader.cpp:947-975): offsets of the chunk's
        // profiles, each position's profile within the chunk, and the
        // addresses of the CV and SS data (the position itself)
        db->dist.resize(P);
        db->addrpro.resize(N);
        db->addrcv.resize(N);
        db->addrss.resize(N);
        for (uint64_t k = 0; k < P; k++) {
            const long long s0 = db->pstart[first + k] - pos0, s1 = db->pstart[first + k + 1] - pos0;
            db->dist[k] = (uint32_t)s0;
            for (long long n = s0; n < s1; n++) {
                db->addrpro[n] = (int)k;
                db->addrcv[n] = (int)n;
                db->addrss[n] = (int)n;
            }
        }
        auto put = [&](int f, const void* p, size_t bytes) {
            beg[f] = static_cast<char*>(const_cast<void*>(p));
            end[f] = beg[f] + bytes;
        };
        put(fDist, db->dist.data(), P * 4);
        put(fAddrPro, db->addrpro.data(), N * 4);
        put(fAddrCV, db->addrcv.data(), N * 4);
        put(fAddrSS, db->addrss.data(), N * 4);
        if (descs) {
            size_t prev = db->addr[kNStored + 1];
            if (first > 0)
                std::memcpy(&prev, db->map + db->addr[kNStored] + (first - 1) * sizeof(size_t), sizeof(size_t));
            for (uint64_t k = 0; k < P; k++) {
                descs[k] = db->map + prev;
                std::memcpy(&prev, db->map + db->addr[kNStored] + (first + k) * sizeof(size_t), sizeof(size_t));
            }
        }
    });
}

int cbp_db_write(const char* path, char* const* beg, char* const* end, const char* const* descs)
{
    FILE* fp = nullptr;
    const int rc = guarded_db([&] {
        if (!path || !beg || !end) throw DbError{CBP_ERR_ARG, "null argument"};
        for (int f = 0; f < fTot; f++)
            if (!beg[f] || !end[f] || end[f] < beg[f])
                throw DbError{CBP_ERR_ARG, "field " + std::to_string(f) + ": invalid begin/end pointers"};
        const uint64_t P = (uint64_t)(end[fLen] - beg[fLen]) / 4;
        const uint64_t N = (uint64_t)(end[fTF] - beg[fTF]) / 4;
        if (P < 1 || N < 1) throw DbError{CBP_ERR_ARG, "empty profile set"};
        const std::vector<Section> secs = stored_sections();
        for (const Section& s : secs)
            if ((uint64_t)(end[s.field] - beg[s.field]) != section_count(s, P, N) * s.esz)
                throw DbError{CBP_ERR_ARG, "field " + std::to_string(s.field) + " of wrong size"};
        uint64_t ndst = 0;
        for (uint64_t n = 0; n < N; n++) {
            float c;
            std::memcpy(&c, beg[fDD] + n * 4, 4);
            ndst += (uint64_t)c;
        }
        // header and address table (Db::WriteBinaryHeader,
        // CalculateAndWriteAddressTable_v2_2)
        std::vector<size_t> table(kNSections);
        size_t addr = header_bytes() + kNSections * sizeof(size_t);
        for (int k = 0; k < kNStored; k++) {
            table[k] = addr;
            addr += section_count(secs[k], P, N) * secs[k].esz;
        }
        table[kNStored] = addr;
        addr += P * sizeof(size_t);
        table[kNStored + 1] = addr;
        fp = std::fopen(path, "wb");
        if (!fp) throw DbError{CBP_ERR_ARG, std::string("cannot create ") + path};
        auto wr = [&](const void* p, size_t n) {
            if (n && std::fwrite(p, 1, n, fp) != n) throw DbError{CBP_ERR_ARG, "write failed"};
        };
        wr(kSignature, sizeof(kSignature) - 1);
        wr(kVersion, sizeof(kVersion) - 1);
        wr(&P, 8);
        wr(&N, 8);
        wr(&ndst, 8);
        wr(table.data(), table.size() * sizeof(size_t));
        for (const Section& s : secs) wr(beg[s.field], (size_t)(end[s.field] - beg[s.field]));
        size_t daddr = table[kNStored + 1];
        for (uint64_t k = 0; k < P; k++) {
            const char* d = (descs && descs[k]) ? descs[k] : "";
            daddr += std::strlen(d) + 1;
            wr(&daddr, sizeof(size_t));
        }
        for (uint64_t k = 0; k < P; k++) {
            const char* d = (descs && descs[k]) ? descs[k] : "";
            wr(d, std::strlen(d) + 1);
        }
        if (std::fclose(fp) != 0) {
            fp = nullptr;
            throw DbError{CBP_ERR_ARG, "write failed"};
        }
        fp = nullptr;
    });
    if (fp) std::fclose(fp);
    return rc;
}

}  // extern "C"
