// Seeded synthetic profile generator.
//
// Produces profile data in the structure-of-arrays field layout that the
// search path consumes (one contiguous array per field, see profile_fields.h):
// background probabilities, effective number of observations, lengths,
// position offsets, beginning and per-position transition log-probabilities,
// target frequencies, SS probabilities and SS state, amino acids, and the
// per-position inter-residue distance lists.
//
// The distance lists follow the construction that the reference's `adddist`
// tool applies to pair distances (src/adddist/adddist.cpp:546-651,
// ProcessDistancesForPosition): partners nearest in sequence are kept (at
// most 99), ordered by partner position, and gaps between partners are
// filled with penalty distances (DSTSEP6=12 or DSTGAPL=24; DSTFREE=3,
// DSTNPOS=12, DSTSEGM=6 as in src/env/options.txt).
//
// Amino acids are stored as letters and SS states as ' ', 'e', 'h' (the
// reference's text reader keeps residue letters and lower-case SS codes,
// src/libmycu/cupro/IOProfileModelTxt.cu:438,1029; src/liblib/alpha.cpp:12-14).
//
// Two distance sources are generated:
//  * "observed" (database profiles): a C-beta random walk with 3.8 A steps,
//    pairwise Euclidean distances rounded to integers;
//  * "predicted" (query profiles): per pair a 17-bin Dirichlet(0.3)
//    distribution over 2-20 A; the distance is the rounded expectation and
//    its probability is the mass of the bin holding the expectation; pairs
//    with probability < prb_thld are dropped (adddist --prb).
//
// Every profile draws from its own random stream derived from (seed,
// profile index), so the output does not depend on the thread count.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <thread>
#include <algorithm>

namespace {

constexpr int kNAA = 20;
constexpr int kNTrn = 7;         // MM MI MD IM II DM DD kept by the reader
constexpr int kNDstSlots = 100;  // slot 0 = count, 1..99 = distances
constexpr int kMaxDst = 99;
constexpr float kDstGap = 255.f;
constexpr float kLogFct = 0.4f;  // factor applied to IM, II, DM, DD log-probs
constexpr float kLog0 = -32768.f;

// optdst* options of adddist (src/env/options.txt)
constexpr int kDstFree = 3;
constexpr int kDstNPos = 12;
constexpr int kDstSegm = 6;
constexpr float kDstSep6 = 12.f;
constexpr float kDstGapL = 24.f;

struct Rng {
    uint64_t s[4];
    static uint64_t splitmix(uint64_t& x) {
        uint64_t z = (x += 0x9e3779b97f4a7c15ULL);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
        return z ^ (z >> 31);
    }
    explicit Rng(uint64_t seed) {
        uint64_t x = seed;
        for (int i = 0; i < 4; i++) s[i] = splitmix(x);
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {  // xoshiro256**
        uint64_t r = rotl(s[1] * 5, 7) * 9;
        uint64_t t = s[1] << 17;
        s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
        s[2] ^= t; s[3] = rotl(s[3], 45);
        return r;
    }
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
    double uniform_pos() { double u; do { u = uniform(); } while (u <= 0.0); return u; }
    double normal() {  // Box-Muller
        double u1 = uniform_pos(), u2 = uniform();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
    // Marsaglia & Tsang (2000) gamma sampler; alpha < 1 via the U^(1/alpha) boost.
    double gamma(double alpha) {
        if (alpha < 1.0) {
            double g = gamma(alpha + 1.0);
            return g * std::pow(uniform_pos(), 1.0 / alpha);
        }
        double d = alpha - 1.0 / 3.0, c = 1.0 / std::sqrt(9.0 * d);
        for (;;) {
            double x, v;
            do { x = normal(); v = 1.0 + c * x; } while (v <= 0.0);
            v = v * v * v;
            double u = uniform_pos();
            if (u < 1.0 - 0.0331 * x * x * x * x) return d * v;
            if (std::log(u) < 0.5 * x * x + d * (1.0 - v + std::log(v))) return d * v;
        }
    }
    void dirichlet(const double* alpha, int n, double* out) {
        double s = 0.0;
        for (int i = 0; i < n; i++) { out[i] = gamma(alpha[i]); s += out[i]; }
        if (s <= 0.0) { for (int i = 0; i < n; i++) out[i] = 1.0 / n; return; }
        for (int i = 0; i < n; i++) out[i] /= s;
    }
};

struct PairDst { int partner; float dst; };

// Turn the partners of one position into its distance list (adddist rules).
// `partners` holds (partner position, distance) for every pair with a
// distance; `plen` is the profile length.
int CompileList(int position, int plen, std::vector<PairDst>& partners, float* out /*kMaxDst*/)
{
    // nearest partners in sequence first; ties broken by partner position
    std::sort(partners.begin(), partners.end(), [position](const PairDst& a, const PairDst& b) {
        int sa = std::abs(position - a.partner), sb = std::abs(position - b.partner);
        return sa != sb ? sa < sb : a.partner < b.partner;
    });
    if ((int)partners.size() > kMaxDst) partners.resize(kMaxDst);
    std::sort(partners.begin(), partners.end(),
              [](const PairDst& a, const PairDst& b) { return a.partner < b.partner; });

    std::vector<float> v;
    v.reserve(2 * kMaxDst);
    if (!partners.empty() && kDstFree < std::abs(position - partners[0].partner))
        v.push_back(partners[0].dst);
    int maxmainsep = 1;
    float dstpen = kDstSep6;
    for (size_t i = 1; i < partners.size(); i++) {
        int posep = partners[i].partner - partners[i - 1].partner;
        int mainsepp = std::abs(position - partners[i - 1].partner);
        int mainsep = std::abs(position - partners[i].partner);
        int mainsp2 = std::max(mainsepp, mainsep);
        if (mainsep <= kDstFree) {
            if (posep > 1 && maxmainsep < mainsp2) maxmainsep = mainsp2;
            continue;
        }
        if ((posep > 1 && mainsp2 >= kDstNPos) || maxmainsep >= kDstNPos)
            v.push_back(dstpen = kDstGapL);
        else if (posep > 1 || maxmainsep > 1)
            v.push_back(dstpen = kDstSep6);
        for (int k = 2; k < posep && k < kDstSegm; k++) v.push_back(dstpen);
        v.push_back(partners[i].dst);
        maxmainsep = 1;
    }
    if ((int)v.size() > kMaxDst) {
        if (position + kMaxDst > plen)
            v.erase(v.begin(), v.begin() + (v.size() - kMaxDst));
        else
            v.resize(kMaxDst);
    }
    for (size_t i = 0; i < v.size(); i++) out[i] = v[i];
    return (int)v.size();
}

struct Fields {
    float* bkg;      // [20][P]
    float* eno;      // [P]
    float* trn;      // [7][N+P]
    float* tf;       // [20][N]
    float* ss;       // [3][N]
    int8_t* ssstate; // [N]
    int8_t* aa;      // [N]
    float* dd;       // [100][N]
    int32_t* addrpro;// [N]
};

void GenProfile(int p, int P, long long N, const int* lens, const long long* starts,
                int predicted, int window, float prb_thld, uint64_t seed,
                const double* gbkg, Fields f)
{
    Rng rng(seed * 0x100000001b3ULL + (uint64_t)p * 0x9e3779b97f4a7c15ULL + 12345);
    const int L = lens[p];
    const long long s0 = starts[p];
    const long long NT = N + P;  // transition entries

    // profile background: Dirichlet around the global background
    double a[kNAA], bk[kNAA];
    for (int i = 0; i < kNAA; i++) a[i] = 200.0 * gbkg[i];
    rng.dirichlet(a, kNAA, bk);
    for (int i = 0; i < kNAA; i++) f.bkg[(long long)i * P + p] = (float)bk[i];
    f.eno[p] = (float)(1.0 + 13.0 * rng.uniform());

    // transitions: beginning vector at entry s0+p, position k at s0+p+1+k
    for (int k = -1; k < L; k++) {
        double m3[3], am[3] = {30.0, 1.2, 1.2}, i2[2], ai[2] = {4.0, 1.0}, d2[2], ad[2] = {3.0, 1.3};
        rng.dirichlet(am, 3, m3);
        rng.dirichlet(ai, 2, i2);
        rng.dirichlet(ad, 2, d2);
        const double pr[kNTrn] = {m3[0], m3[1], m3[2], i2[0], i2[1], d2[0], d2[1]};
        const long long e = s0 + p + 1 + k;
        for (int t = 0; t < kNTrn; t++) {
            float v = (float)pr[t];
            float lv = v > 0.f ? (t > 2 ? std::log(v) * kLogFct : std::log(v)) : kLog0;
            f.trn[(long long)t * NT + e] = lv;
        }
    }

    // per-position fields
    // Dirichlet(0.5 per letter) centred on the profile background, so that
    // the target frequencies average to the background (and unrelated
    // profiles score below zero on average, as real profiles do)
    double at[kNAA];
    for (int i = 0; i < kNAA; i++) at[i] = 0.5 * kNAA * bk[i];
    for (int k = 0; k < L; k++) {
        const long long n = s0 + k;
        double tf[kNAA], sp[3];
        rng.dirichlet(at, kNAA, tf);
        int amax = 0;
        for (int i = 0; i < kNAA; i++) {
            double v = 0.7 * tf[i] + 0.3 * bk[i];
            f.tf[(long long)i * N + n] = (float)v;
            if (tf[i] > tf[amax]) amax = i;
        }
        f.aa[n] = (int8_t)"ARNDCQEGHILKMFPSTWYV"[amax];
        const double a3[3] = {1.0, 1.0, 1.0};
        rng.dirichlet(a3, 3, sp);
        int smax = 0;
        for (int i = 0; i < 3; i++) {
            f.ss[(long long)i * N + n] = (float)sp[i];
            if (sp[i] > sp[smax]) smax = i;
        }
        f.ssstate[n] = (int8_t)" eh"[smax];
        f.addrpro[n] = p;
    }

    // pair distances
    std::vector<std::vector<PairDst>> part(L);
    if (predicted) {
        const int nb = 17;
        double ab[nb], pb[nb];
        for (int i = 0; i < nb; i++) ab[i] = 0.3;
        for (int i = 0; i < L; i++)
            for (int j = i + 3; j < L && j - i < window; j++) {
                rng.dirichlet(ab, nb, pb);
                double e = 0.0;
                for (int b = 0; b < nb; b++) e += pb[b] * (2.0 + (b + 0.5) * 18.0 / nb);
                int bin = (int)((e - 2.0) * nb / 18.0);
                bin = std::min(std::max(bin, 0), nb - 1);
                if (pb[bin] < prb_thld) continue;
                float d = (float)std::lround(e);
                part[i].push_back({j, d});
                part[j].push_back({i, d});
            }
    } else {
        std::vector<double> x(3 * (size_t)L, 0.0);
        for (int i = 1; i < L; i++) {
            double u[3], nrm;
            do {
                for (int c = 0; c < 3; c++) u[c] = rng.normal();
                nrm = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
            } while (nrm < 1e-9);
            for (int c = 0; c < 3; c++) x[3 * i + c] = x[3 * (i - 1) + c] + 3.8 * u[c] / nrm;
        }
        for (int i = 0; i < L; i++)
            for (int j = i + 3; j < L && j - i < window; j++) {
                double dx = x[3 * i] - x[3 * j], dy = x[3 * i + 1] - x[3 * j + 1], dz = x[3 * i + 2] - x[3 * j + 2];
                float d = (float)std::lround(std::sqrt(dx * dx + dy * dy + dz * dz));
                if (d > 64.f) d = 64.f;
                part[i].push_back({j, d});
                part[j].push_back({i, d});
            }
    }
    float lst[kMaxDst];
    for (int k = 0; k < L; k++) {
        const long long n = s0 + k;
        int cnt = CompileList(k, L, part[k], lst);
        f.dd[n] = (float)cnt;
        for (int t = 1; t < kNDstSlots; t++)
            f.dd[(long long)t * N + n] = (t <= cnt) ? lst[t - 1] : kDstGap;
    }
}

}  // namespace

extern "C" {

// Fill the field arrays of P profiles (lengths `lens`, position offsets
// `starts`, N = total positions). `predicted` selects the distance source
// (1 = predicted distributions for queries, 0 = observed random walk).
// `gbkg` is the global background (20 values). Returns 0 on success.
int cbs_generate(int P, long long N, const int* lens, const long long* starts,
                 int predicted, int window, float prb_thld, unsigned long long seed,
                 const double* gbkg,
                 float* bkg, float* eno, float* trn, float* tf, float* ss,
                 signed char* ssstate, signed char* aa, float* dd, int* addrpro,
                 int nthreads)
{
    if (P <= 0 || N <= 0 || !lens || !starts) return 1;
    Fields f{bkg, eno, trn, tf, ss, (int8_t*)ssstate, (int8_t*)aa, dd, addrpro};
    if (nthreads < 1) nthreads = 1;
    if (nthreads > P) nthreads = P;
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; t++)
        th.emplace_back([=]() {
            for (int p = t; p < P; p += nthreads)
                GenProfile(p, P, N, lens, starts, predicted, window, prb_thld, seed, gbkg, f);
        });
    for (auto& x : th) x.join();
    return 0;
}

}  // extern "C"
