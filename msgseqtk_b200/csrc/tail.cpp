// Host tail of msgseqtk-align's single-end task (src/msgseqtk-align.cpp:612-628
// and its output step :538-556, :583-585): Alignment::filter, evaluate,
// calcMapQ and sort (src/Alignment.cpp:446-555, src/Alignment.h:622-633) and
// the fields exportBAM and output set (src/Alignment.cpp:429-444), on the
// alignment records the CUDA path returns. Everything is double precision in
// the reference's order of operations (no contraction: built with
// -ffp-contract=off), so log10P, postP, MAPQ and the record order are the
// reference's bit for bit; reads are spread over host threads.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/msg_b200.h"

namespace {

constexpr double kPhredScale = -10;   // quality::PHRED_SCALE (src/QualStr.h:36)
constexpr double kMaxQ = 250;         // quality::MAX_Q_SCORE (src/QualStr.h:35)
constexpr double kMinLoglikExp = -256;  // MIN_LOGLIK_EXP (src/MSGseqTKConst.h:36)
constexpr int kOpM = 0, kOpI = 1, kOpD = 2, kOpS = 4;  // SAM CIGAR op codes
constexpr int kFlagReverse = 0x10, kFlagSecondary = 0x100, kFlagUnmapped = 0x4;
// quality of every base of a read without one: PrimarySeq::fixQual pads the
// (empty) quality string to the read's length with 33 (src/PrimarySeq.h:105-109)
constexpr uint8_t kNoQual = 33;
const char kDecode[16] = {'$', 'A', 'C', 'M', 'G', 'R', 'S', 'V', 'T', 'W', 'Y', 'H', 'K', 'D', 'B', 'N'};

// Per-quality terms of Alignment::evaluate (src/Alignment.cpp:461-465):
// a matching base adds log10(1 - phredQ2P(q)), a mismatch q / PHRED_SCALE,
// with phredQ2P(q) = exp(log(10) * q / PHRED_SCALE) (src/QualStr.h:110-112).
struct QualTables {
    double match[256], mis[256];
    QualTables() {
        const double logbase = std::log(10.0);
        for (int q = 0; q < 256; ++q) {
            const double p = std::exp(logbase * q / kPhredScale);
            match[q] = std::log10(1 - p);
            mis[q] = q / kPhredScale;
        }
    }
};

const QualTables& tables() {
    static const QualTables t;
    return t;
}

struct Target {
    const uint8_t* seq;
    int64_t len;
};

struct ReadOut {
    std::vector<msg_sam_rec> rec;
    std::string md;
};

inline void put_count(std::string& s, uint32_t v) {  // boost::lexical_cast<string>(uint32_t)
    char b[10];
    int n = 0;
    do { b[n++] = (char)('0' + v % 10); v /= 10; } while (v);
    while (n) s.push_back(b[--n]);
}

// Alignment::getAlnMDTag (src/Alignment.cpp:305-353): runs of '=' as counts,
// a mismatch as the count then the target base, an insertion as the count
// (at its start) then '^' and the inserted query bases; deletions add
// nothing; the last count closes the tag.
void md_tag(const uint8_t* q, const uint8_t* t, int64_t i, int64_t j, const uint32_t* cg, int32_t nc, std::string& md) {
    int prev = -1;
    uint32_t len = 0;
    for (int32_t w = 0; w < nc; ++w) {
        const int op = cg[w] & 0xf;
        if (op == kOpS) continue;
        const uint32_t run = cg[w] >> 4;
        if (op == kOpM) {  // '=' runs counted in a tight loop; each 'X' ends one
            uint32_t r = 0;
            while (r < run) {
                while (r < run && (q[i] & t[j])) { ++i; ++j; ++len; ++r; }
                if (r == run) { prev = 7; break; }  // BAM_CEQUAL
                put_count(md, len);                 // BAM_CDIFF
                len = 0;
                md.push_back(kDecode[t[j] & 15]);
                ++i; ++j; ++r;
                prev = 8;
            }
            continue;
        }
        for (uint32_t r = 0; r < run; ++r) {
            if (op == kOpI) {
                if (prev != kOpI) {
                    put_count(md, len);
                    md.push_back('^');
                }
                len = 0;
                md.push_back(kDecode[q[i] & 15]);
                ++i;
            } else if (op == kOpD) {
                ++j;
            }
            prev = op;
        }
    }
    put_count(md, len);
}

// Alignment::evaluate (src/Alignment.cpp:446-489) over the record's path.
double evaluate(const uint8_t* q, const uint8_t* qual, int64_t L, const uint8_t* t, const msg_aln& a,
                const uint32_t* cg, const msg_tail_params& p, bool* empty) {
    const QualTables& T = tables();
    *empty = true;
    for (int32_t w = 0; w < a.n_cigar; ++w)
        if ((cg[w] & 0xf) != kOpS && (cg[w] >> 4) > 0) *empty = false;
    if (*empty) return 0;  // log10P keeps its initial 0
    double ll = 0;
    for (int64_t i = 0; i < a.aln_from; ++i) ll += -p.clip;
    int64_t i = a.aln_from, j = a.aln_start;
    int prev = -1;
    for (int32_t w = 0; w < a.n_cigar; ++w) {
        const int op = cg[w] & 0xf;
        if (op == kOpS) continue;
        const uint32_t run = cg[w] >> 4;
        if (op == kOpM) {  // query bases of an M run lie inside the read (checked)
            for (uint32_t r = 0; r < run; ++r, ++i, ++j) ll += (q[i] & t[j]) ? T.match[qual[i]] : T.mis[qual[i]];
            if (run) prev = kOpM;
            continue;
        }
        for (uint32_t r = 0; r < run; ++r) {
            const int qv = i < L ? qual[i] : 0;  // a QualStr reads its terminator at L
            switch (op) {
                case kOpI:
                    if (prev != kOpI) ll += T.mis[qv] - p.gap_open;
                    ll += -p.gap_ext;
                    ++i;
                    break;
                case kOpD:
                    if (prev != kOpD) ll += T.mis[qv] - p.gap_open;
                    ll += -p.gap_ext;
                    ++j;
                    break;
                default: break;
            }
            prev = op;
        }
    }
    for (int64_t k = a.aln_to; k < L; ++k) ll += -p.clip;
    return ll;
}

// evaluate and getAlnMDTag in one pass over the record's path (the same
// sums in the same order, the same text): the MD scan runs beside the
// dependent chain of log10P adds. For reads whose one kept record is also
// the one reported.
double evaluate_md(const uint8_t* q, const uint8_t* qual, int64_t L, const uint8_t* t, const msg_aln& a,
                   const uint32_t* cg, const msg_tail_params& p, std::string& md) {
    const QualTables& T = tables();
    double ll = 0;
    for (int64_t i = 0; i < a.aln_from; ++i) ll += -p.clip;
    int64_t i = a.aln_from, j = a.aln_start;
    int prev = -1;       // evaluate's previous op (M, I, D)
    uint32_t len = 0;    // MD: '=' bases since the last mismatch or insertion
    for (int32_t w = 0; w < a.n_cigar; ++w) {
        const int op = cg[w] & 0xf;
        if (op == kOpS) continue;
        const uint32_t run = cg[w] >> 4;
        if (op == kOpM) {
            for (uint32_t r = 0; r < run; ++r, ++i, ++j) {
                const bool eq = (q[i] & t[j]) != 0;
                ll += eq ? T.match[qual[i]] : T.mis[qual[i]];
                if (eq) {
                    ++len;
                } else {
                    put_count(md, len);
                    len = 0;
                    md.push_back(kDecode[t[j] & 15]);
                }
            }
            if (run) prev = kOpM;
            continue;
        }
        for (uint32_t r = 0; r < run; ++r) {
            const int qv = i < L ? qual[i] : 0;
            if (op == kOpI) {
                if (prev != kOpI) {
                    ll += T.mis[qv] - p.gap_open;
                    put_count(md, len);
                    md.push_back('^');
                }
                ll += -p.gap_ext;
                len = 0;
                md.push_back(kDecode[q[i] & 15]);
                ++i;
            } else if (op == kOpD) {
                if (prev != kOpD) ll += T.mis[qv] - p.gap_open;
                ll += -p.gap_ext;
                ++j;
            }
            prev = op;
        }
    }
    put_count(md, len);
    for (int64_t k = a.aln_to; k < L; ++k) ll += -p.clip;
    return ll;
}

// One read's alignments after Alignment::filter and evaluate, with the
// reverse-complemented read (PrimarySeq::revcom: bases reversed and
// complemented, quality reversed) when a record needs it.
struct Mate {
    int64_t read = 0, L = 0;
    const uint8_t* seq = nullptr;
    const uint8_t* fq = nullptr;   // forward quality (33s without one)
    std::vector<uint8_t> rc, rq;   // reverse complement; reversed quality, then 33s for reads without one
    std::vector<int64_t> keep;     // record indices kept by the filter, in record order
    std::vector<double> l10;       // log10P of each kept record
    std::vector<char> empty;       // a record without a path (evaluate skips it)
    std::vector<double> pr, post;  // calcMapQ work and posterior
    std::vector<int> mapq;
    std::vector<size_t> ord;
    std::string md1;               // MD text of the only kept record, made with its log10P
    bool has_md1 = false;
};

void mate_eval(Mate& m, int64_t r, const uint8_t* seq, const uint8_t* qual, int64_t L, const msg_aln* aln,
               int64_t k0, int64_t k1, const uint32_t* cigar, const std::vector<Target>& tg,
               const msg_tail_params& p) {
    static const uint8_t kComp[16] = {0, 8, 4, 12, 2, 10, 6, 14, 1, 9, 5, 13, 3, 11, 7, 15};
    m.read = r;
    m.seq = seq;
    m.L = L;
    m.keep.clear();
    for (int64_t k = k0; k < k1; ++k) {  // Alignment::filter (src/Alignment.cpp:548-555)
        const double score = aln[k].aln_score == INT32_MIN ? -INFINITY : (double)aln[k].aln_score;
        if (!(score < L * p.min_score_rate)) m.keep.push_back(k);
    }
    const size_t N = m.keep.size();
    if (N == 0) return;
    bool any_rev = false;
    for (int64_t k : m.keep) any_rev |= aln[k].strand == 2;
    m.rq.resize(2 * L);
    if (!qual) std::fill(m.rq.begin() + L, m.rq.end(), kNoQual);
    if (any_rev) {
        m.rc.resize(L);
        for (int64_t i = 0; i < L; ++i) {
            m.rc[i] = kComp[seq[L - 1 - i] & 15];
            m.rq[i] = qual ? qual[L - 1 - i] : kNoQual;
        }
    }
    m.fq = qual ? qual : m.rq.data() + L;
    m.l10.resize(N);
    m.empty.resize(N);
    m.has_md1 = false;
    for (size_t n = 0; n < N; ++n) {
        const msg_aln& a = aln[m.keep[n]];
        const bool rev = a.strand == 2;
        bool e;
        if (N == 1) {  // its record is reported: log10P and MD in one pass
            e = true;
            for (int32_t w = 0; w < a.n_cigar; ++w)
                if ((cigar[a.cigar_off + w] & 0xf) != kOpS && (cigar[a.cigar_off + w] >> 4) > 0) e = false;
            m.md1.clear();
            m.l10[0] = e ? 0 : evaluate_md(rev ? m.rc.data() : seq, rev ? m.rq.data() : m.fq, L, tg[a.tid].seq, a,
                                           cigar + a.cigar_off, p, m.md1);
            m.has_md1 = !e;
        } else {
            m.l10[n] = evaluate(rev ? m.rc.data() : seq, rev ? m.rq.data() : m.fq, L, tg[a.tid].seq, a,
                                cigar + a.cigar_off, p, &e);
        }
        m.empty[n] = e;
    }
}

const double kLog10e = std::log10(M_E);

// The posterior/MAPQ step shared by Alignment::calcMapQ and
// AlignmentPE::calcMapQ (src/Alignment.cpp:491-537) on log-likelihoods pr:
// shift by MIN_LOGLIK_EXP when all are below it, exp, normalise by the
// left-to-right sum (pairs: 1/N each when the sum is 0), MAPQ =
// min(round(phredP2Q(1 - postP)), 250).
void posterior(std::vector<double>& pr, std::vector<double>& post, std::vector<int>& mapq, bool pairs) {
    const size_t N = pr.size();
    post.resize(N);
    mapq.resize(N);
    double maxV = pr[0];
    for (double x : pr) if (x > maxV) maxV = x;
    const double scale = maxV != -INFINITY && maxV < kMinLoglikExp ? kMinLoglikExp - maxV : 0;
    if (N == 1 && std::isfinite(pr[0]) && pr[0] + scale < 700) {
        // exp(x + scale) is finite and above 0 (x + scale >= -256), so postP =
        // pr / pr = 1 and MAPQ = min(round(-10 * log10(0)), 250) = 250
        post[0] = 1.0;
        mapq[0] = (int)kMaxQ;
        return;
    }
    for (double& x : pr) x = std::exp(x + scale);
    double sum = 0;
    for (double x : pr) sum += x;
    for (size_t n = 0; n < N; ++n) {
        post[n] = pairs && !(sum > 0) ? 1.0 / N : pr[n] / sum;
        const double mq = kPhredScale * std::log10(1 - post[n]);
        mapq[n] = (int)(uint8_t)std::min(std::round(mq), kMaxQ);
    }
}

// The record exportBAM builds for kept alignment n of a mate (flags, MAPQ
// and pair fields are set by the caller).
msg_sam_rec export_rec(const Mate& m, size_t n, const msg_aln* aln, const uint32_t* cigar,
                       const std::vector<Target>& tg, std::string& md) {
    const msg_aln& a = aln[m.keep[n]];
    msg_sam_rec o{};
    o.read = m.read;
    o.flag = a.strand == 2 ? kFlagReverse : 0;
    o.tid = a.tid;
    o.pos = a.aln_start;
    o.as = (int32_t)std::round((double)a.aln_score);
    o.xh = (float)m.l10[n];
    o.cigar_off = a.cigar_off;
    o.n_cigar = a.n_cigar;
    o.md_off = (int64_t)md.size();
    if (m.has_md1 && n == 0)
        md += m.md1;
    else if (!m.empty[n])
        md_tag(a.strand == 2 ? m.rc.data() : m.seq, tg[a.tid].seq, a.aln_from, a.aln_start, cigar + a.cigar_off,
               a.n_cigar, md);
    o.md_len = (int32_t)((int64_t)md.size() - o.md_off);
    return o;
}

// calcMapQ + sort + output(alnList, out, maxReport, extraFlag) for one mate
// (src/Alignment.cpp:491-512, src/Alignment.h:629-633,
// src/msgseqtk-align.cpp:538-556).
void mate_out(Mate& m, const msg_aln* aln, const uint32_t* cigar, const std::vector<Target>& tg,
              const msg_tail_params& p, int extra, ReadOut& out) {
    const size_t N = m.keep.size();
    m.pr.resize(N);
    for (size_t n = 0; n < N; ++n) m.pr[n] = m.l10[n] / kLog10e;  // Alignment::loglik
    posterior(m.pr, m.post, m.mapq, false);
    m.ord.resize(N);
    for (size_t n = 0; n < N; ++n) m.ord[n] = n;
    const std::vector<double>& l10 = m.l10;
    std::sort(m.ord.begin(), m.ord.end(), [&](size_t x, size_t y) { return l10[x] > l10[y]; });
    const size_t num = p.max_report == 0 ? N : std::min<size_t>(p.max_report, N);
    for (size_t s = 0; s < num; ++s) {
        const size_t n = m.ord[s];
        msg_sam_rec o = export_rec(m, n, aln, cigar, tg, out.md);
        o.flag |= (s > 0 ? kFlagSecondary : 0) | extra;
        o.mapq = m.mapq[n];
        o.xp = (float)m.post[n];
        o.nh = (int32_t)num;
        o.xn = (int32_t)N;
        out.rec.push_back(o);
    }
}

msg_sam_rec unmapped(int64_t r, int flag) {
    msg_sam_rec u{};
    u.read = r;
    u.flag = flag;
    u.tid = -1;
    return u;
}

// Single-end task tail (src/msgseqtk-align.cpp:619-628).
void tail_se(Mate& m, const msg_aln* aln, const uint32_t* cigar, const std::vector<Target>& tg,
             const msg_tail_params& p, ReadOut& out) {
    if (m.keep.empty()) {
        out.rec.push_back(unmapped(m.read, kFlagUnmapped));  // output(read, out), :583-585
        return;
    }
    mate_out(m, aln, cigar, tg, p, 0, out);
}

// PairingScheme::pr (src/PairingScheme.cpp:18-25) with the normal pdf
// exp(-z^2 / 2) / (sd * sqrt(2 pi)), z = (x - mean) / sd.
double pairing_pr(const msg_pair_params& q, double sd, double x) {
    if (q.mean == 0) return 1;
    if (q.min_ins <= x && x <= q.max_ins) {
        const double z = (x - q.mean) / sd;
        return std::exp(-0.5 * z * z) / (sd * std::sqrt(2.0 * M_PI));
    }
    return 0;
}

struct Pair {
    size_t f, r;       // kept-record indices of the two mates
    int32_t isize;
    double l10, ll;    // AlignmentPE::log10lik and loglik
};

// Paired-end task tail (src/msgseqtk-align.cpp:703-748): AlignmentPE::getPairs,
// sort, filter, calcMapQ and output(pairList) (src/Alignment.cpp:514-581,
// src/Alignment.h:636-640, src/msgseqtk-align.cpp:558-581), or the unpaired
// records of each mate, or an unmapped pair.
void tail_pe(Mate& f, Mate& r, const msg_aln* aln, const uint32_t* cigar, const std::vector<Target>& tg,
             const msg_tail_params& p, const msg_pair_params& q, double sd, std::vector<Pair>& pairs,
             std::vector<double>& pr, std::vector<double>& post, std::vector<int>& mapq, ReadOut& out) {
    constexpr int kPaired = 0x1, kProper = 0x2, kMateUnmapped = 0x8, kRead1 = 0x40, kRead2 = 0x80;
    if (f.keep.empty() && r.keep.empty()) {  // output(fwdRead, revRead, out), :587-591
        out.rec.push_back(unmapped(f.read, kFlagUnmapped | kMateUnmapped | kPaired | kRead1));
        out.rec.push_back(unmapped(r.read, kFlagUnmapped | kMateUnmapped | kPaired | kRead2));
        return;
    }
    pairs.clear();
    for (size_t i = 0; i < f.keep.size(); ++i)  // getPairs: mates on different strands
        for (size_t j = 0; j < r.keep.size(); ++j) {
            const msg_aln& a = aln[f.keep[i]];
            const msg_aln& b = aln[r.keep[j]];
            if ((a.strand & b.strand) != 0) continue;
            Pair x;
            x.f = i;
            x.r = j;
            x.isize = a.tid != b.tid ? -1
                                     : (int32_t)(std::max(a.aln_end, b.aln_end) - std::min(a.aln_start, b.aln_start));
            const double ppr = pairing_pr(q, sd, (double)x.isize);
            x.l10 = f.l10[i] + r.l10[j] + std::log10(ppr);
            x.ll = f.l10[i] / kLog10e + r.l10[j] / kLog10e + std::log(ppr);
            pairs.push_back(x);
        }
    std::sort(pairs.begin(), pairs.end(), [](const Pair& x, const Pair& y) { return x.l10 > y.l10; });
    auto drop = [&](auto pred) { pairs.erase(std::remove_if(pairs.begin(), pairs.end(), pred), pairs.end()); };
    drop([&](const Pair& x) { return !(q.min_ins <= x.isize && x.isize <= q.max_ins); });
    auto A = [&](const Pair& x) -> const msg_aln& { return aln[f.keep[x.f]]; };
    auto B = [&](const Pair& x) -> const msg_aln& { return aln[r.keep[x.r]]; };
    if (q.no_discordant)
        drop([&](const Pair& x) { return !(A(x).tid == B(x).tid && (A(x).strand & B(x).strand) == 0); });
    if (q.no_tail_over)
        drop([&](const Pair& x) {
            const msg_aln &a = A(x), &b = B(x);
            return (a.aln_start <= b.aln_start && a.aln_end > b.aln_start) ||
                   (b.aln_start <= a.aln_start && b.aln_end > a.aln_start);
        });
    if (q.no_contain)
        drop([&](const Pair& x) {
            const msg_aln &a = A(x), &b = B(x);
            return (a.aln_start <= b.aln_start && a.aln_end >= b.aln_end) ||
                   (b.aln_start <= a.aln_start && b.aln_end >= a.aln_end);
        });
    if (q.no_overlap)
        drop([&](const Pair& x) { return A(x).aln_start < B(x).aln_end && A(x).aln_end > B(x).aln_start; });
    if (q.max_npair > 0 && (int64_t)pairs.size() > q.max_npair) pairs.resize(q.max_npair);
    if (!pairs.empty()) {
        const size_t N = pairs.size();
        pr.resize(N);
        for (size_t n = 0; n < N; ++n) pr[n] = pairs[n].ll;
        posterior(pr, post, mapq, true);
        const size_t num = p.max_report == 0 ? N : std::min<size_t>(p.max_report, N);
        for (size_t s = 0; s < num; ++s) {
            const Pair& x = pairs[s];
            const bool fwd_first = A(x).aln_start < B(x).aln_start;
            msg_sam_rec a = export_rec(f, x.f, aln, cigar, tg, out.md);  // exportFwdBAM
            msg_sam_rec b = export_rec(r, x.r, aln, cigar, tg, out.md);  // exportRevBAM
            a.flag |= kPaired | kProper | kRead1 | (s > 0 ? kFlagSecondary : 0);
            b.flag |= kPaired | kProper | kRead2 | (s > 0 ? kFlagSecondary : 0);
            a.isize = fwd_first ? x.isize : -x.isize;
            b.isize = fwd_first ? -x.isize : x.isize;
            a.mapq = b.mapq = mapq[s];
            a.nh = b.nh = (int32_t)num;
            a.xn = b.xn = (int32_t)N;
            a.xp = b.xp = (float)post[s];
            out.rec.push_back(a);
            out.rec.push_back(b);
        }
    } else if (!q.no_mixed) {
        if (!f.keep.empty()) mate_out(f, aln, cigar, tg, p, kPaired | kRead1, out);
        if (!r.keep.empty()) mate_out(r, aln, cigar, tg, p, kPaired | kRead2, out);
    }
}

}  // namespace

extern "C" void msg_tail_params_default(msg_tail_params* p) {
    if (!p) return;
    p->min_score_rate = 0.65;  // msgseqtk-align -s
    p->max_report = 1;         // -k
    p->n_threads = 0;
    p->gap_open = 5;           // ScoreScheme defaults (src/ScoreScheme.cpp:14-18)
    p->gap_ext = 2;
    p->clip = 4;
}

extern "C" void msg_pair_params_default(msg_pair_params* q) {
    if (!q) return;
    // PairingScheme after msgseqtk-align's options without -m/-d/-I/-X
    // (src/PairingScheme.h:34-37, 84-97; src/msgseqtk-align.cpp:267-300, 400)
    q->mean = 200;
    q->sd = 20;
    q->min_ins = 0;
    q->max_ins = 400;
    q->no_mixed = q->no_discordant = q->no_tail_over = q->no_contain = q->no_overlap = 0;
    q->max_npair = 0;
}

namespace {

int tail_run(const msg_mtg_view* mtg, const msg_read_batch* reads, const uint8_t* quals, const msg_aln* aln,
             const uint32_t* cigar, const int64_t* read_aln_off, const msg_tail_params* p,
             const msg_pair_params* q, msg_sam_rec* out, int64_t out_cap, char* md, int64_t md_cap, int64_t* n_out,
             int64_t* md_len) {
    if (!mtg || !reads || !read_aln_off || !p || !n_out || !md_len) return MSG_EINVAL;
    const int64_t n = reads->n_reads;
    if (n < 0 || (n > 0 && (!reads->seq || !reads->off))) return MSG_EINVAL;
    if (q && (n % 2 != 0)) return MSG_EINVAL;
    if (std::isnan(p->min_score_rate)) return MSG_EINVAL;
    // PairingScheme::updateParam (src/PairingScheme.h:72-78)
    const double sd = q ? (q->mean == 0 ? 1 : q->sd == 0 ? q->mean * 0.1 : q->sd) : 0;
    if (q && (std::isnan(q->mean) || std::isnan(sd) || std::isnan(q->min_ins) || std::isnan(q->max_ins)))
        return MSG_EINVAL;
    std::vector<Target> tg(mtg->n_chrom);
    for (int64_t t = 0; t < mtg->n_chrom; ++t) tg[t] = Target{mtg->chr_seq + mtg->chr_off[t], mtg->chr_len[t]};
    // every record must lie inside its read, its chromosome and the CIGAR array
    auto valid = [&](int64_t i) {
        const int64_t L = reads->off[i + 1] - reads->off[i];
        if (L < 0 || read_aln_off[i + 1] < read_aln_off[i]) return false;
        for (int64_t k = read_aln_off[i]; k < read_aln_off[i + 1]; ++k) {
            const msg_aln& a = aln[k];
            if (a.tid < 0 || a.tid >= mtg->n_chrom || a.aln_from < 0 || a.aln_start < 0 || a.n_cigar < 0)
                return false;
            int64_t qi = 0, tj = 0;
            for (int32_t w = 0; w < a.n_cigar; ++w) {
                const uint32_t c = cigar[a.cigar_off + w];
                const int op = c & 0xf;
                if (op == kOpM) { qi += c >> 4; tj += c >> 4; }
                else if (op == kOpI) qi += c >> 4;
                else if (op == kOpD) tj += c >> 4;
                else if (op != kOpS) return false;
            }
            if (a.aln_from + qi > L || a.aln_start + tj > tg[a.tid].len) return false;
        }
        return true;
    };
    const int64_t units = q ? n / 2 : n;
    int nt = p->n_threads > 0 ? p->n_threads : (int)std::max(1u, std::thread::hardware_concurrency());
    nt = (int)std::max<int64_t>(1, std::min<int64_t>(nt, (units + 127) / 128));
    std::vector<ReadOut> parts(nt);
    std::vector<char> bad(nt, 0);
    auto prep = [&](Mate& m, int64_t i) {
        const int64_t o = reads->off[i];
        mate_eval(m, i, reads->seq + o, quals ? quals + o : nullptr, reads->off[i + 1] - o, aln, read_aln_off[i],
                  read_aln_off[i + 1], cigar, tg, *p);
    };
    auto work = [&](int w) {
        Mate m0, m1;
        std::vector<Pair> pairs;
        std::vector<double> pr, post;
        std::vector<int> mapq;
        const int64_t a = units * w / nt, b = units * (w + 1) / nt;
        parts[w].rec.reserve((size_t)(b - a) * (q ? 2 : 1) * std::max<uint32_t>(1, p->max_report));
        parts[w].md.reserve((size_t)(b - a) * (q ? 2 : 1) * 16);
        for (int64_t u = a; u < b; ++u) {
            if (q) {
                if (!valid(2 * u) || !valid(2 * u + 1)) { bad[w] = 1; return; }
                prep(m0, 2 * u);
                prep(m1, 2 * u + 1);
                tail_pe(m0, m1, aln, cigar, tg, *p, *q, sd, pairs, pr, post, mapq, parts[w]);
            } else {
                if (!valid(u)) { bad[w] = 1; return; }
                prep(m0, u);
                tail_se(m0, aln, cigar, tg, *p, parts[w]);
            }
        }
    };
    auto run = [&](auto fn) {
        std::vector<std::thread> th;
        for (int w = 1; w < nt; ++w) th.emplace_back(fn, w);
        fn(0);
        for (auto& t : th) t.join();
    };
    run(work);
    for (char x : bad) if (x) return MSG_EINVAL;
    std::vector<int64_t> ro(nt + 1, 0), mo(nt + 1, 0);
    for (int w = 0; w < nt; ++w) {
        ro[w + 1] = ro[w] + (int64_t)parts[w].rec.size();
        mo[w + 1] = mo[w] + (int64_t)parts[w].md.size();
    }
    *n_out = ro[nt];
    *md_len = mo[nt];
    if (ro[nt] > out_cap || mo[nt] > md_cap || (ro[nt] > 0 && !out) || (mo[nt] > 0 && !md)) return MSG_EINVAL;
    run([&](int w) {  // each thread places its own records and MD text
        msg_sam_rec* o = out + ro[w];
        for (const msg_sam_rec& x : parts[w].rec) {
            *o = x;
            o->md_off += mo[w];
            ++o;
        }
        if (!parts[w].md.empty()) std::memcpy(md + mo[w], parts[w].md.data(), parts[w].md.size());
    });
    return MSG_OK;
}

}  // namespace

extern "C" int msg_tail_batch(const msg_mtg_view* mtg, const msg_read_batch* reads, const uint8_t* quals,
                              const msg_aln* aln, const uint32_t* cigar, const int64_t* read_aln_off,
                              const msg_tail_params* p, msg_sam_rec* out, int64_t out_cap, char* md, int64_t md_cap,
                              int64_t* n_out, int64_t* md_len) {
    return tail_run(mtg, reads, quals, aln, cigar, read_aln_off, p, nullptr, out, out_cap, md, md_cap, n_out, md_len);
}

extern "C" int msg_tail_pe_batch(const msg_mtg_view* mtg, const msg_read_batch* reads, const uint8_t* quals,
                                 const msg_aln* aln, const uint32_t* cigar, const int64_t* read_aln_off,
                                 const msg_tail_params* p, const msg_pair_params* q, msg_sam_rec* out,
                                 int64_t out_cap, char* md, int64_t md_cap, int64_t* n_out, int64_t* md_len) {
    if (!q) return MSG_EINVAL;
    return tail_run(mtg, reads, quals, aln, cigar, read_aln_off, p, q, out, out_cap, md, md_cap, n_out, md_len);
}
