/*
 * CPU restatement of MSGseqTK v1.2.3's read-mapping hot path. TEST
 * INFRASTRUCTURE ONLY: it is the checker for the CUDA path (tests, smoke and
 * the bench's CPU-baseline leg); the product never links it.
 *
 * Citations are file:line in the reference tree (MSGseqTK src/).
 */
#include "msg_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>
#include <atomic>
#include <string>

namespace {

const double kInf = std::numeric_limits<double>::infinity();

/* DNAalphabet tables (DNAalphabet.h:37-51, DNAalphabet.cpp:74-190). */
const uint8_t kComp[16] = {0, 8, 4, 12, 2, 10, 6, 14, 1, 9, 5, 13, 3, 11, 7, 15};
const int kToInt[16] = {0, 1, 2, 0, 3, 0, 0, 0, 4, 0, 0, 0, 0, 0, 0, 0};
const uint8_t kToBasic[16] = {0, 1, 2, 2, 4, 4, 4, 4, 8, 8, 8, 8, 8, 8, 8, 15};
const uint8_t kEncodeInt[5] = {0, 1, 2, 4, 8};
const char kDecode[16] = {'$', 'A', 'C', 'M', 'G', 'R', 'S', 'V', 'T', 'W', 'Y', 'H', 'K', 'D', 'B', 'N'};
inline bool is_ambiguous(int b) { return !(b == 1 || b == 2 || b == 4 || b == 8); }  // DNAalphabet.h:135-142

enum { FWD = 1, REV = 2 };  // GLoc.h:20
enum { OP_M = 0, OP_I = 1, OP_D = 2, OP_S = 4, OP_EQ = 7, OP_X = 8 };  // SAM CIGAR codes

}  // namespace

struct orc_index {
    int64_t n;
    std::vector<uint8_t> bwt;
    int64_t B[256];
    int64_t C[256];
    std::vector<int64_t> ck;      // per 64-symbol block: counts of each nt16 code before it
    std::vector<uint64_t> sbits;  // SA-sample bit per row
    std::vector<int64_t> srank;   // ones before each 64-bit word
    std::vector<int64_t> svals;   // sample values in row order
    int64_t n_chrom;
    std::vector<int64_t> bd_start, bd_end, chr_len, chr_off;
    std::vector<uint8_t> chr_seq;
    double llk[16];
};

extern "C" orc_index* orc_index_create(int64_t n, const uint8_t* bwt, const int64_t* B16,
                                       int64_t n_samples, const int64_t* sample_rows,
                                       const int64_t* sample_vals, int64_t n_chrom,
                                       const int64_t* bd_start, const int64_t* bd_end,
                                       const int64_t* chr_len, const uint8_t* chr_seq,
                                       const int64_t* chr_off) {
    orc_index* ix = new orc_index();
    ix->n = n;
    ix->bwt.assign(bwt, bwt + n);
    std::memset(ix->B, 0, sizeof(ix->B));
    std::memset(ix->C, 0, sizeof(ix->C));
    for (int b = 0; b < 16; ++b) ix->B[b] = B16[b];
    /* FMDIndex::buildCounts (FMDIndex.cpp:118-129): C[i] for i = 0..16 */
    int64_t S = 0;
    for (int i = 0; i <= 16; ++i) { ix->C[i] = S; S += ix->B[i]; }
    const int64_t nb = n / 64 + 1;
    ix->ck.assign((size_t)(nb + 1) * 16, 0);
    int64_t run[16] = {0};
    for (int64_t k = 0; k <= nb; ++k) {
        for (int b = 0; b < 16; ++b) ix->ck[(size_t)k * 16 + b] = run[b];
        for (int64_t i = k * 64; i < std::min(n, (k + 1) * 64); ++i) run[bwt[i]]++;
    }
    const int64_t nw = n / 64 + 1;
    ix->sbits.assign(nw, 0);
    for (int64_t k = 0; k < n_samples; ++k) ix->sbits[sample_rows[k] >> 6] |= 1ULL << (sample_rows[k] & 63);
    ix->srank.assign(nw + 1, 0);
    for (int64_t w = 0; w < nw; ++w) ix->srank[w + 1] = ix->srank[w] + __builtin_popcountll(ix->sbits[w]);
    ix->svals.assign(sample_vals, sample_vals + n_samples);
    ix->n_chrom = n_chrom;
    ix->bd_start.assign(bd_start, bd_start + n_chrom);
    ix->bd_end.assign(bd_end, bd_end + n_chrom);
    ix->chr_len.assign(chr_len, chr_len + n_chrom);
    ix->chr_off.assign(chr_off, chr_off + n_chrom + 1);
    ix->chr_seq.assign(chr_seq, chr_seq + chr_off[n_chrom]);
    /* FMDIndex::loglik (FMDIndex.h:195-197) */
    for (int b = 0; b < 16; ++b)
        ix->llk[b] = std::log((double)ix->B[kToBasic[b]]) - std::log((double)n);
    return ix;
}

extern "C" void orc_index_free(orc_index* ix) { delete ix; }

/* WaveletTreeRRR::rank (WaveletTreeRRR.cpp:101-125): occurrences of b in
 * BWT[0..i], or (size_t)-1 when i >= n. */
extern "C" int64_t orc_rank(const orc_index* ix, int b, int64_t i) {
    if ((uint64_t)i >= (uint64_t)ix->n) return -1;
    const int64_t k = i >> 6;
    int64_t r = ix->ck[(size_t)k * 16 + b];
    for (int64_t x = k << 6; x <= i; ++x) r += ix->bwt[x] == b;
    return r;
}

/* FMDIndex::backExt (FMDIndex.cpp:577-610). */
extern "C" int64_t orc_back_ext(const orc_index* ix, int64_t* p, int64_t* q, int64_t* s, int b) {
    if (is_ambiguous(b)) return (*s = 0);
    int64_t sB[5], qB[5];
    const int c = kToInt[b];
    const int64_t O = orc_rank(ix, b, *p - 1);
    sB[c] = orc_rank(ix, b, *p + *s - 1) - O;
    if (sB[c] <= 0) return (*s = sB[c]);
    if (sB[c] != *s) {
        sB[0] = orc_rank(ix, 0, *p + *s - 1) - orc_rank(ix, 0, *p - 1);
        for (int j = c + 1; j <= 4; ++j)
            sB[j] = orc_rank(ix, kEncodeInt[j], *p + *s - 1) - orc_rank(ix, kEncodeInt[j], *p - 1);
        qB[0] = *q;
        qB[4] = qB[0] + sB[0];
        for (int j = 4; j > c; --j) qB[j - 1] = qB[j] + sB[j];
        *q = qB[c];
    }
    *p = ix->C[b] + O;
    *s = sB[c];
    return *s;
}

/* FMDIndex::fwdExt (FMDIndex.h:226-228). */
extern "C" int64_t orc_fwd_ext(const orc_index* ix, int64_t* p, int64_t* q, int64_t* s, int b) {
    return orc_back_ext(ix, q, p, s, kComp[b & 15]);
}

/* FMDIndex::accessSA (FMDIndex.cpp:520-527) with LF (FMDIndex.h:130-141). */
extern "C" int64_t orc_access_sa(const orc_index* ix, int64_t i) {
    int64_t dist = 0;
    while (!((ix->sbits[i >> 6] >> (i & 63)) & 1)) {
        const int b = ix->bwt[i];
        i = ix->C[b] + orc_rank(ix, b, i) - 1;
        dist++;
    }
    const int64_t w = i >> 6;
    const int64_t r1 = ix->srank[w] + __builtin_popcountll(ix->sbits[w] & (~0ULL >> (63 - (i & 63))));
    return ix->svals[r1 - 1] + dist;
}

extern "C" double orc_loglik(const orc_index* ix, int b) { return ix->llk[b & 15]; }

namespace {

struct Smem {
    int64_t from, to, p, q, s;
    double logP;
};

struct Read {
    const uint8_t* seq;
    int64_t L;
    int base(int64_t i) const { return i < L ? seq[i] : 0; }  // PrimarySeq::getBase at L is the terminator
};

/* SMEM::evaluate (SMEM.cpp:19-24) */
void smem_evaluate(const orc_index* ix, const Read& r, Smem& m) {
    m.logP = 0;
    for (int64_t i = m.from; i < m.to; ++i) m.logP += ix->llk[r.base(i)];
}

/* SMEM::fwdExt + fwdEvaluate (SMEM.h:140-145,166-170) */
void smem_fwd(const orc_index* ix, const Read& r, Smem& m) {
    orc_fwd_ext(ix, &m.p, &m.q, &m.s, r.base(m.to));
    if (m.to < r.L) m.logP += ix->llk[r.base(m.to)];
    m.to++;
}

/* SMEM::backExt + backEvaluate (SMEM.h:152-157,173-177) */
void smem_back(const orc_index* ix, const Read& r, Smem& m) {
    orc_back_ext(ix, &m.p, &m.q, &m.s, m.from > 0 ? r.base(m.from - 1) : 0);
    if (m.from > 0) m.logP += ix->llk[r.base(m.from - 1)];
    m.from--;
}

/* SMEM::loglik(from, to) (SMEM.cpp:26-40) */
double smem_loglik_range(const orc_index* ix, const Read& r, const Smem& m, int64_t from, int64_t to) {
    double ll = 0;
    if (from <= m.from && m.to <= to) {
        ll += m.logP;
        for (int64_t i = from; i < m.from; ++i) ll += ix->llk[r.base(i)];
        for (int64_t i = m.to; i < to; ++i) ll += ix->llk[r.base(i)];
    } else {
        for (int64_t i = from; i < to; ++i) ll += ix->llk[r.base(i)];
    }
    return ll;
}

double evalue_of(const orc_index* ix, double ll) { return ix->n * std::exp(ll); }  // SMEM.h:90-110

Smem smem_init(const orc_index* ix, const Read& r, int64_t from) {
    const int b = r.base(from);
    Smem m;
    m.from = from; m.to = from + 1;
    m.p = ix->C[b]; m.q = ix->C[kComp[b]]; m.s = ix->C[b + 1] - ix->C[b];
    smem_evaluate(ix, r, m);
    return m;
}

/* SMEM_LIST::findFwdBackSMEMS (SMEM.cpp:64-117) */
void find_fwd_back(const orc_index* ix, const Read& r, int64_t& from, int64_t& to, int64_t minLen,
                   double maxEvalue, int64_t minSize, std::vector<Smem>& curr) {
    std::vector<Smem> prev;
    const int b = r.base(from);
    to = from + 1;
    if (is_ambiguous(b)) return;
    Smem smem = smem_init(ix, r, from);
    Smem smem0 = smem;
    while (smem.s >= minSize) {
        smem_fwd(ix, r, smem);
        if (smem.s != smem0.s && smem0.to >= minLen &&
            (!std::isfinite(maxEvalue) ||
             evalue_of(ix, smem_loglik_range(ix, r, smem0, 0, smem0.to)) <= maxEvalue))
            prev.push_back(smem0);
        smem0 = smem;
    }
    to = smem.to;
    if (prev.empty()) { from--; return; }
    std::reverse(prev.begin(), prev.end());
    while (from >= 0 && !prev.empty()) {
        int64_t s0 = -1, nValid = 0;
        for (Smem& m : prev) {
            smem0 = m;
            smem_back(ix, r, m);
            if (m.s != smem0.s && smem0.s >= minSize && nValid == 0 && smem0.to - smem0.from >= minLen &&
                evalue_of(ix, smem0.logP) <= maxEvalue)
                curr.push_back(smem0);
            if (m.s >= minSize && m.s != s0) { s0 = m.s; nValid++; }
            else m.s = 0;
        }
        prev.erase(std::remove_if(prev.begin(), prev.end(), [](const Smem& m) { return !(m.s > 0); }), prev.end());
        from--;
    }
}

/* SMEM_LIST::findBackFwdSMEMS (SMEM.cpp:119-172) */
void find_back_fwd(const orc_index* ix, const Read& r, int64_t& from, int64_t& to, int64_t minLen,
                   double maxEvalue, int64_t minSize, std::vector<Smem>& curr) {
    const int64_t L = r.L;
    std::vector<Smem> prev;
    const int b = r.base(from);
    to = from + 1;
    if (is_ambiguous(b)) return;
    Smem smem = smem_init(ix, r, from);
    Smem smem0 = smem;
    while (smem.s >= minSize) {
        smem_back(ix, r, smem);
        if (smem.s != smem0.s && L - smem0.from >= minLen &&
            (!std::isfinite(maxEvalue) ||
             evalue_of(ix, smem_loglik_range(ix, r, smem0, smem0.from, L)) <= maxEvalue))
            prev.push_back(smem0);
        smem0 = smem;
    }
    from = smem.from;
    if (prev.empty()) { to++; return; }
    std::reverse(prev.begin(), prev.end());
    while (to <= L && !prev.empty()) {
        int64_t s0 = -1, nValid = 0;
        for (Smem& m : prev) {
            smem0 = m;
            smem_fwd(ix, r, m);
            if (m.s != smem0.s && smem0.s >= minSize && nValid == 0 && smem0.to - smem0.from >= minLen &&
                evalue_of(ix, smem0.logP) <= maxEvalue)
                curr.push_back(smem0);
            if (m.s >= minSize && m.s != s0) { s0 = m.s; nValid++; }
            else m.s = 0;
        }
        prev.erase(std::remove_if(prev.begin(), prev.end(), [](const Smem& m) { return !(m.s > 0); }), prev.end());
        to++;
    }
}

/* SMEM_LIST::findAllSMEMS (SMEM.cpp:186-215) */
std::vector<Smem> find_all_smems(const orc_index* ix, const Read& r, int64_t minLen, double maxEvalue) {
    const int64_t L = r.L;
    std::vector<Smem> curr;
    int64_t from = L / 2;
    int64_t to = from + 1;
    find_fwd_back(ix, r, from, to, minLen, maxEvalue, 1, curr);
    while (from > 0 || to < L) {
        int64_t from0 = to;
        if (from0 < L) find_fwd_back(ix, r, from0, to, minLen, maxEvalue, 1, curr);
        int64_t to0 = --from + 1;
        if (from >= 0) find_back_fwd(ix, r, from, to0, minLen, maxEvalue, 1, curr);
    }
    return curr;
}

struct Seed {
    int64_t from, to, start, end, tid, strand;
    int64_t len() const { return to - from; }
};

bool seed_less(const Seed& l, const Seed& r) {  // SeedPair.h:225-232
    return l.from != r.from ? l.from < r.from
         : l.to != r.to ? l.to < r.to
         : l.tid != r.tid ? l.tid < r.tid
         : l.strand != r.strand ? l.strand < r.strand
         : l.start != r.start ? l.start < r.start
         : l.end < r.end;
}

bool containing(const Seed& l, const Seed& r) {  // SeedPair.h:171-175
    return l.tid == r.tid && l.strand == r.strand && l.from <= r.from && l.to >= r.to &&
           l.start <= r.start && l.end >= r.end;
}

/* MetaGenome::getTid (MetaGenome.h:474-479): linear scan. */
int64_t get_tid(const orc_index* ix, int64_t pos) {
    for (int64_t t = 0; t < ix->n_chrom; ++t)
        if (ix->bd_start[t] <= pos && pos < ix->bd_end[t]) return t;
    return -1;
}

/* MetaGenome::getStrand / getLoc (MetaGenome.h:147-167) */
int get_strand(const orc_index* ix, int64_t tid, int64_t pos) {
    const int64_t st = ix->bd_start[tid], len = ix->bd_end[tid] - st;
    return st <= pos && pos < st + len / 2 ? FWD : REV;
}
int64_t get_loc(const orc_index* ix, int64_t tid, int64_t pos) {
    return get_strand(ix, tid, pos) == FWD ? pos - ix->bd_start[tid] : ix->bd_end[tid] - pos - 1;
}

/* SMEM::getSeeds (SMEM.cpp:217-269) */
void get_seeds(const orc_index* ix, const Read& r, const Smem& m, std::vector<Seed>& out) {
    const int64_t len = m.to - m.from;
    for (int64_t i = 0; i < m.s; ++i) {
        {
            const int64_t bd = orc_access_sa(ix, m.p + i);
            const int64_t tid = get_tid(ix, bd);
            const int64_t st = get_loc(ix, tid, bd);
            if (get_strand(ix, tid, bd) == FWD) out.push_back(Seed{m.from, m.from + len, st, st + len, tid, FWD});
        }
        {
            const int64_t bd = orc_access_sa(ix, m.q + i);
            const int64_t tid = get_tid(ix, bd);
            const int64_t st = get_loc(ix, tid, bd);
            if (get_strand(ix, tid, bd) == FWD) out.push_back(Seed{r.L - m.to, r.L - m.to + len, st, st + len, tid, REV});
        }
    }
}

/* SeedPair::removeRedundant (SeedPair.cpp:71-88) */
void remove_redundant(std::vector<Seed>& seeds) {
    if (seeds.size() <= 1) return;
    std::sort(seeds.begin(), seeds.end(), seed_less);
    for (size_t i = 0; i + 1 < seeds.size(); ++i)
        for (size_t j = i + 1; j < seeds.size(); ++j)
            if (containing(seeds[i], seeds[j]) || containing(seeds[j], seeds[i])) {
                seeds[i] = Seed{0, 0, 0, 0, -1, 3};
                break;
            }
    seeds.erase(std::remove_if(seeds.begin(), seeds.end(), [](const Seed& s) { return s.len() == 0; }), seeds.end());
}

/* SMEM_LIST::findSeeds (SMEM.cpp:271-305) */
std::vector<Seed> find_seeds(const orc_index* ix, const Read& r, int64_t minLen, double maxEvalue, int64_t maxNSeed) {
    std::vector<Smem> smems = find_all_smems(ix, r, minLen, maxEvalue);
    std::sort(smems.begin(), smems.end(), [](const Smem& a, const Smem& b) -> bool { return a.logP < b.logP; });
    std::vector<Seed> all;
    for (const Smem& m : smems) {
        get_seeds(ix, r, m, all);
        if ((int64_t)all.size() >= maxNSeed) break;
    }
    remove_redundant(all);
    return all;
}

/* Loc::dist (Loc.h:89-91) */
int64_t loc_dist(int64_t ls, int64_t le, int64_t rs, int64_t re) {
    const bool ov = ls < re && le > rs;
    return ov ? 0 : ls < rs ? rs - le + 1 : ls - re + 1;
}

bool compatible(const Seed& l, const Seed& r) {  // SeedPair.h:156-158
    return l.to <= r.from && l.end <= r.start && l.tid == r.tid && l.strand == r.strand;
}

int64_t n_mismatch(const Seed& l, const Seed& r) {  // SeedPair.h:136-142
    if (!compatible(l, r)) return INT64_MAX;
    return std::min(loc_dist(l.from, l.to, r.from, r.to), loc_dist(l.start, l.end, r.start, r.end));
}

int64_t n_indel(const Seed& l, const Seed& r) {  // SeedPair.h:148-153
    if (!compatible(l, r)) return INT64_MAX;
    return (r.from - l.to) - (r.start - l.end);
}

/* SeedChain::getChains / dfsSeeds (SeedChain.cpp:40-73), with the recursion
 * unrolled onto an explicit stack; visiting order is unchanged. */
void get_chains(const std::vector<Seed>& seeds, int64_t maxMM, int64_t maxIndel,
                std::vector<std::vector<int64_t>>& chains) {
    const int64_t N = (int64_t)seeds.size();
    std::vector<char> visited(N, 0);
    struct Frame { int64_t i, j; bool leaf; };
    std::vector<Frame> st;
    for (int64_t root = 0; root < N; ++root) {
        if (visited[root]) continue;
        visited[root] = 1;
        st.push_back(Frame{root, root + 1, true});
        while (!st.empty()) {
            Frame& f = st.back();
            bool descended = false;
            while (f.j < N) {
                const int64_t j = f.j++;
                if (!visited[j] && n_mismatch(seeds[f.i], seeds[j]) <= maxMM &&
                    std::llabs(n_indel(seeds[f.i], seeds[j])) <= maxIndel) {
                    f.leaf = false;
                    visited[j] = 1;
                    st.push_back(Frame{j, j + 1, true});
                    descended = true;
                    break;
                }
            }
            if (descended) continue;
            if (st.back().leaf) {
                std::vector<int64_t> c;
                for (const Frame& g : st) c.push_back(g.i);
                chains.push_back(c);
            }
            st.pop_back();
        }
    }
}

/* ScoreScheme (ScoreScheme.cpp:20-24, ScoreScheme.h:76-96) with integral values. */
struct Score {
    double sc[16][16];
    double match, mismatch, gapO, gapE;
    Score(const int32_t* s4) {
        match = s4[0]; mismatch = s4[1]; gapO = s4[2]; gapE = s4[3];
        for (int i = 0; i < 16; ++i)
            for (int j = 0; j < 16; ++j)
                sc[i][j] = (i & j) && i != 15 && j != 15 ? match : -mismatch;
    }
    double gap_penalty(int64_t len) const { return len == 0 ? 0 : gapO + gapE * len; }
};

struct Mat {
    int64_t R, Cc;
    std::vector<double> d;
    void init(int64_t r, int64_t c) { R = r; Cc = c; d.assign((size_t)r * c, -kInf); }
    double& at(int64_t i, int64_t j) { return d[(size_t)i * Cc + j]; }
};

/* Alignment::matchMax/insMax/delMax (Alignment.h:577-597), including the
 * reference's `max = del` assignment in matchMax. */
int match_max(double match, double ins, double del) {
    double mx = match;
    int s = OP_M;
    if (ins > mx) { mx = del; s = OP_I; }
    if (del > mx) s = OP_D;
    return s;
}
int ins_max(double m, double i) { return m > i ? OP_M : OP_I; }
int del_max(double m, double d) { return m > d ? OP_M : OP_D; }

struct Aligner {
    const orc_index* ix;
    const Read* read;
    std::vector<uint8_t> query;  // read or its reverse complement
    const uint8_t* target;
    int64_t target_len;
    int64_t tid, strand, qFrom, qTo, tStart, tEnd;
    /* chromosome base, or the DNAseq terminator 0 one past its end (the
     * window may reach it: getChromLength counts the terminator,
     * MetaGenome.cpp:208 with MetaGenome.h:237) */
    int tb(int64_t j) const { return j < target_len ? target[j] : 0; }
    int mode;
    const Score* ss;
    Mat M, I, D;

    int64_t qLen() const { return qTo - qFrom; }
    int64_t tLen() const { return tEnd - tStart; }

    void calc_rect(int64_t from, int64_t to, int64_t start, int64_t end) {  // Alignment.cpp:72-133
        const double o = -(ss->gapO + ss->gapE), e = -ss->gapE;
        for (int64_t t = start; t < end; ++t) {
            const int64_t j = t - tStart + 1;
            for (int64_t q = from; q < to; ++q) {
                const int64_t i = q - qFrom + 1;
                const double s = ss->sc[query[q]][tb(t)];
                double m = std::max({M.at(i - 1, j - 1) + s, D.at(i - 1, j - 1) + s, I.at(i - 1, j - 1) + s});
                if (mode == 1) m = std::max(m, 0.0);
                M.at(i, j) = m;
                I.at(i, j) = std::max(M.at(i - 1, j) + o, I.at(i - 1, j) + e);
                D.at(i, j) = std::max(M.at(i, j - 1) + o, D.at(i, j - 1) + e);
            }
        }
    }

    void calc_seed(const Seed& sd) {  // Alignment.cpp:135-171
        const double o = -(ss->gapO + ss->gapE);
        const double s = ss->match;
        const int64_t len = sd.len();
        for (int64_t a = 0; a < len; ++a)
            for (int64_t b = 0; b < len; ++b) M.at(sd.from - qFrom + 1 + a, sd.start - tStart + 1 + b) = -kInf;
        for (int64_t k = 0; k < len; ++k) {
            const int64_t i = sd.from + k - qFrom + 1, j = sd.start + k - tStart + 1;
            if (k == 0) M.at(i, j) = std::max({M.at(i - 1, j - 1) + s, D.at(i - 1, j - 1) + s, I.at(i - 1, j - 1) + s, 0.0});
            else M.at(i, j) = M.at(i - 1, j - 1) + s;
        }
        const int64_t i = sd.to - qFrom + 1, j = sd.end - tStart + 1;
        if (i <= qLen() && j <= tLen()) M.at(i, j) = M.at(i - 1, j - 1) + s;
        if (i <= qLen()) for (int64_t c = 0; c <= tLen(); ++c) I.at(i, c) = M.at(i - 1, c) + o;
        if (j <= tLen()) for (int64_t r = 0; r <= qLen(); ++r) D.at(r, j) = M.at(r, j - 1) + o;
    }
};

int64_t do_align(const orc_index* ix, const Read& r, const std::vector<Seed>& chain, int mode, const Score& ss,
                 orc_aln* out, uint32_t* cigar_buf, int64_t cigar_cap, int64_t* cigar_used, char* md_buf,
                 int64_t md_cap, int64_t* md_used) {
    Aligner a;
    a.ix = ix; a.read = &r; a.mode = mode; a.ss = &ss;
    const Seed& first = chain.front();
    const Seed& last = chain.back();
    a.tid = first.tid; a.strand = first.strand;
    a.query.resize(r.L);
    if (a.strand == FWD) std::memcpy(a.query.data(), r.seq, r.L);
    else for (int64_t i = 0; i < r.L; ++i) a.query[i] = kComp[r.seq[r.L - 1 - i]];  // PrimarySeq::revcom
    a.target = ix->chr_seq.data() + ix->chr_off[a.tid];
    a.target_len = ix->chr_len[a.tid];
    const int64_t chrLen = ix->chr_len[a.tid] + 1;  // MetaGenome::getChromLength (MetaGenome.h:237)
    a.qFrom = 0; a.qTo = r.L;
    /* Alignment::initTStart / initTEnd (Alignment.cpp:46-52) */
    a.tStart = std::max<int64_t>(0, first.start - (1 + 0.1) * (first.from - a.qFrom));
    a.tEnd = std::min<int64_t>(chrLen, last.end + (1 + 0.1) * (a.qTo - last.to));
    const int64_t R = a.qLen() + 1, Cc = a.tLen() + 1;
    a.M.init(R, Cc); a.I.init(R, Cc); a.D.init(R, Cc);
    if (mode == 0) {  // initNW (Alignment.h:599-606)
        for (int64_t j = 0; j < Cc; ++j) a.M.at(0, j) = 0;
        for (int64_t i = 0; i < R; ++i) a.I.at(i, 0) = -ss.gap_penalty(i);
    } else {  // initSW (Alignment.h:608-613)
        for (int64_t j = 0; j < Cc; ++j) a.M.at(0, j) = 0;
        for (int64_t i = 0; i < R; ++i) a.M.at(i, 0) = 0;
    }
    /* calculateScores(chain) (Alignment.cpp:54-70) */
    if (a.qFrom < first.from && a.tStart < first.start) a.calc_rect(a.qFrom, first.from, a.tStart, first.start);
    for (size_t k = 0; k < chain.size(); ++k) {
        a.calc_seed(chain[k]);
        if (k + 1 < chain.size()) a.calc_rect(chain[k].to, chain[k + 1].from, chain[k].end, chain[k + 1].start);
    }
    if (last.to < a.qTo && last.end < a.tEnd) a.calc_rect(last.to, a.qTo, last.end, a.tEnd);

    int64_t flags = 0;
    int64_t alnTo, alnEnd, alnFrom, alnStart;
    double alnScore;
    std::vector<int> path;
    const double o = ss.gapO, e = ss.gapE;
    if (mode == 0) {  // backTraceNW (Alignment.cpp:173-233)
        alnTo = R - 1; alnScore = -kInf; alnEnd = 0;
        int s = OP_M;
        for (int64_t j = 1; j < Cc; ++j) {
            if (a.M.at(alnTo, j) > alnScore) { alnScore = a.M.at(alnTo, j); alnEnd = j; s = OP_M; }
            if (a.I.at(alnTo, j) > alnScore) { alnScore = a.I.at(alnTo, j); alnEnd = j; s = OP_I; }
        }
        if (alnScore == -kInf) flags |= 1;
        int64_t i = alnTo, j = alnEnd;
        alnTo += a.qFrom; alnEnd += a.tStart;
        while (i > 0) {
            if (j < 0 || (s != OP_I && j < 1)) { flags |= 2; break; }
            path.push_back(s);
            if (s == OP_M) { s = match_max(a.M.at(i - 1, j - 1), a.I.at(i - 1, j - 1), a.D.at(i - 1, j - 1)); i--; j--; }
            else if (s == OP_I) { s = ins_max(a.M.at(i - 1, j) - o - e, a.I.at(i - 1, j) - e); i--; }
            else { s = del_max(a.M.at(i, j - 1) - o - e, a.D.at(i, j - 1) - e); j--; }
        }
        alnFrom = a.qFrom + i; alnStart = a.tStart + j;
    } else {  // backTraceSW (Alignment.cpp:235-276); maxCoeff = first max, column-major
        double best = a.M.at(0, 0); int64_t bi = 0, bj = 0;
        for (int64_t j = 0; j < Cc; ++j)
            for (int64_t i = 0; i < R; ++i)
                if (a.M.at(i, j) > best) { best = a.M.at(i, j); bi = i; bj = j; }
        alnScore = best; alnTo = bi; alnEnd = bj;
        int64_t i = alnTo, j = alnEnd;
        alnTo += a.qFrom; alnEnd += a.tStart;
        int s = OP_M;
        while (s != OP_M || a.M.at(i, j) > 0) {
            if ((s == OP_M && (i < 1 || j < 1)) || (s == OP_I && i < 1) || (s == OP_D && j < 1)) { flags |= 2; break; }
            path.push_back(s);
            if (s == OP_M) { s = match_max(a.M.at(i - 1, j - 1), a.I.at(i - 1, j - 1), a.D.at(i - 1, j - 1)); i--; j--; }
            else if (s == OP_I) { s = ins_max(a.M.at(i - 1, j) - o - e, a.I.at(i - 1, j) - e); i--; }
            else { s = del_max(a.M.at(i, j - 1) - o - e, a.D.at(i, j - 1) - e); j--; }
        }
        alnFrom = a.qFrom + i; alnStart = a.tStart + j;
    }
    std::reverse(path.begin(), path.end());

    out->tid = a.tid; out->strand = a.strand; out->t_start = a.tStart; out->t_end = a.tEnd;
    out->aln_from = alnFrom; out->aln_to = alnTo; out->aln_start = alnStart; out->aln_end = alnEnd;
    out->aln_score = alnScore; out->flags = flags;
    /* getAlnCigar (Alignment.cpp:278-303) */
    std::vector<uint32_t> cg;
    const int64_t clip5 = alnFrom - a.qFrom, clip3 = a.qTo - alnTo;
    if (clip5 > 0) cg.push_back((uint32_t)(clip5 << 4 | OP_S));
    if (!path.empty()) {
        uint32_t op = path[0], len = 1;
        for (size_t k = 1; k < path.size(); ++k) {
            if ((uint32_t)path[k] != op) { cg.push_back(len << 4 | op); len = 1; }
            else len++;
            op = path[k];
        }
        cg.push_back(len << 4 | op);
    }
    if (clip3 > 0) cg.push_back((uint32_t)(clip3 << 4 | OP_S));
    out->n_cigar = (int64_t)cg.size();
    out->cigar_off = *cigar_used;
    for (uint32_t w : cg) { if (*cigar_used < cigar_cap) cigar_buf[*cigar_used] = w; ++*cigar_used; }
    /* getAlnMDTag (Alignment.cpp:305-353) */
    std::string md;
    uint32_t prev_op = (uint32_t)-1, len = 0;
    for (int64_t k = 0, i = alnFrom, j = alnStart; k < (int64_t)path.size(); ++k) {
        const int qb = i < r.L ? a.query[i] : 0;
        const int tb = j >= 0 ? a.tb(j) : 0;
        uint32_t op = path[k];
        if (op == OP_M) op = (qb & tb) ? OP_EQ : OP_X;
        switch (op) {
            case OP_EQ: i++; j++; len++; break;
            case OP_X: md += std::to_string(len); len = 0; md.push_back(kDecode[tb]); i++; j++; break;
            case OP_I:
                if (prev_op != OP_I) md += std::to_string(len);
                len = 0;
                if (op != prev_op) md.push_back('^');
                md.push_back(kDecode[qb]);
                i++;
                break;
            case OP_D: j++; break;
            default: break;
        }
        prev_op = op;
    }
    md += std::to_string(len);
    out->md_off = *md_used;
    out->md_len = (int64_t)md.size();
    for (char ch : md) { if (*md_used < md_cap) md_buf[*md_used] = ch; ++*md_used; }
    return (int64_t)((R - 1) * (Cc - 1));
}

/* SMEM::findMEM (SMEM.cpp:42-62). The backward pass starts from the state
 * left by the failed forward extension, whose size is 0, so it never extends:
 * the returned MEM keeps `from`, ends one past the last matching base
 * (to_good + 1) with the failed state's size (0) and bi-interval, and its logP
 * includes that extra base when it lies inside the read. `to` returns to_good. */
Smem find_mem(const orc_index* ix, const Read& r, int64_t& from, int64_t& to) {
    Smem mem = smem_init(ix, r, from);
    Smem mem0 = mem;
    for (;;) {
        smem_fwd(ix, r, mem);
        if (mem.s <= 0) break;
        mem0 = mem;
    }
    to = mem0.to;
    mem0 = mem;
    for (;;) {
        smem_back(ix, r, mem);
        if (mem.s <= 0) break;
        mem0 = mem;
    }
    from = mem0.from;
    return mem0;
}

/* SMEM_LIST::findMEMS (SMEM.cpp:174-184) */
std::vector<Smem> find_mems(const orc_index* ix, const Read& r, int64_t minLen, double maxEvalue) {
    std::vector<Smem> mems;
    for (int64_t from = 0, to = 1; from < r.L; from = to + 1) {
        Smem m = find_mem(ix, r, from, to);
        if (m.to - m.from >= minLen && evalue_of(ix, m.logP) <= maxEvalue) mems.push_back(m);
    }
    return mems;
}

std::vector<Seed> seeds_from_rows(const int64_t* rows, int64_t n) {
    std::vector<Seed> v;
    for (int64_t i = 0; i < n; ++i) {
        const int64_t* s = rows + 6 * i;
        v.push_back(Seed{s[0], s[1], s[2], s[3], s[4], s[5]});
    }
    return v;
}

}  // namespace

extern "C" int64_t orc_find_smems(const orc_index* ix, const uint8_t* read, int64_t L, int64_t min_len,
                                  double max_evalue, int64_t* out, int64_t cap) {
    Read r{read, L};
    std::vector<Smem> v = find_all_smems(ix, r, min_len, max_evalue);
    for (int64_t k = 0; k < (int64_t)v.size() && k < cap; ++k) {
        int64_t* o = out + 6 * k;
        o[0] = v[k].from; o[1] = v[k].to; o[2] = v[k].p; o[3] = v[k].q; o[4] = v[k].s;
        std::memcpy(&o[5], &v[k].logP, 8);
    }
    return (int64_t)v.size();
}

extern "C" int64_t orc_find_mems(const orc_index* ix, const uint8_t* read, int64_t L, int64_t min_len,
                                 double max_evalue, int64_t* out, int64_t cap, double* loglik) {
    Read r{read, L};
    std::vector<Smem> v = find_mems(ix, r, min_len, max_evalue);
    double ll = 0;  // SMEM_LIST::loglik (SMEM.cpp:307-312)
    for (int64_t k = 0; k < (int64_t)v.size(); ++k) {
        ll += v[k].logP;
        if (k >= cap) continue;
        int64_t* o = out + 6 * k;
        o[0] = v[k].from; o[1] = v[k].to; o[2] = v[k].p; o[3] = v[k].q; o[4] = v[k].s;
        std::memcpy(&o[5], &v[k].logP, 8);
    }
    if (loglik) *loglik = ll;
    return (int64_t)v.size();
}

extern "C" int64_t orc_find_seeds(const orc_index* ix, const uint8_t* read, int64_t L, int64_t min_len,
                                  double max_evalue, int64_t max_nseed, int64_t* out, int64_t cap) {
    Read r{read, L};
    std::vector<Seed> v = find_seeds(ix, r, min_len, max_evalue, max_nseed);
    for (int64_t k = 0; k < (int64_t)v.size() && k < cap; ++k) {
        int64_t* o = out + 6 * k;
        o[0] = v[k].from; o[1] = v[k].to; o[2] = v[k].start; o[3] = v[k].end; o[4] = v[k].tid; o[5] = v[k].strand;
    }
    return (int64_t)v.size();
}

extern "C" int64_t orc_get_chains(const int64_t* seeds, int64_t n, int64_t max_mismatch, int64_t max_indel,
                                  int64_t* out_off, int64_t* out_idx, int64_t cap_chain, int64_t cap_idx) {
    std::vector<std::vector<int64_t>> chains;
    get_chains(seeds_from_rows(seeds, n), max_mismatch, max_indel, chains);
    int64_t ni = 0;
    if (cap_chain > 0) out_off[0] = 0;
    for (size_t c = 0; c < chains.size(); ++c) {
        for (int64_t x : chains[c]) { if (ni < cap_idx) out_idx[ni] = x; ++ni; }
        if ((int64_t)c + 1 <= cap_chain) out_off[c + 1] = ni;
    }
    return (int64_t)chains.size();
}

extern "C" int orc_align_chain(const orc_index* ix, const uint8_t* read, int64_t L, const int64_t* chain_seeds,
                               int64_t n_seeds, int mode, const int32_t* score4, orc_aln* out,
                               uint32_t* cigar_buf, int64_t cigar_cap, int64_t* cigar_used,
                               char* md_buf, int64_t md_cap, int64_t* md_used) {
    Read r{read, L};
    Score ss(score4);
    std::vector<Seed> chain = seeds_from_rows(chain_seeds, n_seeds);
    do_align(ix, r, chain, mode, ss, out, cigar_buf, cigar_cap, cigar_used, md_buf, md_cap, md_used);
    return 0;
}

extern "C" int64_t orc_align_read(const orc_index* ix, const uint8_t* read, int64_t L, int64_t min_len,
                                  double max_evalue, int64_t max_nseed, int mode, const int32_t* score4,
                                  orc_aln* out, int64_t cap, uint32_t* cigar_buf, int64_t cigar_cap,
                                  int64_t* cigar_used, char* md_buf, int64_t md_cap, int64_t* md_used) {
    Read r{read, L};
    Score ss(score4);
    std::vector<Seed> seeds = find_seeds(ix, r, min_len, max_evalue, max_nseed);
    if (seeds.empty()) return 0;
    /* msgseqtk-align.cpp:619-620 */
    const int64_t maxMM = (int64_t)std::ceil(L * 0.2), maxIndel = (int64_t)std::ceil(L * 0.1);
    std::vector<std::vector<int64_t>> chains;
    get_chains(seeds, maxMM, maxIndel, chains);
    int64_t k = 0;
    for (const auto& c : chains) {
        std::vector<Seed> ch;
        for (int64_t x : c) ch.push_back(seeds[x]);
        orc_aln tmp;
        do_align(ix, r, ch, mode, ss, k < cap ? &out[k] : &tmp, cigar_buf, cigar_cap, cigar_used, md_buf, md_cap, md_used);
        ++k;
    }
    return k;
}

extern "C" int64_t orc_map_batch(const orc_index* ix, int64_t n_reads, const uint8_t* reads, const int64_t* offs,
                                 int64_t min_len, double max_evalue, int64_t max_nseed, int n_threads,
                                 int64_t* n_aln_out, int64_t* n_cells_out) {
    std::atomic<int64_t> next(0), n_aln(0), n_cells(0), mapped(0);
    const int32_t score4[4] = {1, 3, 5, 2};
    auto worker = [&]() {
        Score ss(score4);
        std::vector<uint32_t> cg(1 << 16);
        std::vector<char> md(1 << 16);
        for (;;) {
            const int64_t i = next.fetch_add(1);
            if (i >= n_reads) break;
            const int64_t L = offs[i + 1] - offs[i];
            Read r{reads + offs[i], L};
            std::vector<Seed> seeds = find_seeds(ix, r, min_len, max_evalue, max_nseed);
            if (seeds.empty()) continue;
            const int64_t maxMM = (int64_t)std::ceil(L * 0.2), maxIndel = (int64_t)std::ceil(L * 0.1);
            std::vector<std::vector<int64_t>> chains;
            get_chains(seeds, maxMM, maxIndel, chains);
            int64_t kept = 0;
            for (const auto& c : chains) {
                std::vector<Seed> ch;
                for (int64_t x : c) ch.push_back(seeds[x]);
                orc_aln a;
                int64_t cu = 0, mu = 0;
                n_cells += do_align(ix, r, ch, 0, ss, &a, cg.data(), (int64_t)cg.size(), &cu, md.data(), (int64_t)md.size(), &mu);
                if (!(a.aln_score < L * 0.65)) kept++;
            }
            n_aln += kept;
            if (kept > 0) mapped++;
        }
    };
    std::vector<std::thread> th;
    const int nt = n_threads > 0 ? n_threads : 1;
    for (int t = 0; t < nt; ++t) th.emplace_back(worker);
    for (auto& t : th) t.join();
    *n_aln_out = n_aln.load();
    *n_cells_out = n_cells.load();
    return mapped.load();
}
