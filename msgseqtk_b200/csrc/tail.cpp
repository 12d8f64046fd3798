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
        for (uint32_t r = 0; r < (cg[w] >> 4); ++r) {
            int o = op;
            if (op == kOpM) o = (q[i] & t[j]) ? 7 : 8;  // BAM_CEQUAL / BAM_CDIFF
            switch (o) {
                case 7: ++i; ++j; ++len; break;
                case 8:
                    put_count(md, len);
                    len = 0;
                    md.push_back(kDecode[t[j] & 15]);
                    ++i; ++j;
                    break;
                case kOpI:
                    if (prev != kOpI) put_count(md, len);
                    len = 0;
                    if (o != prev) md.push_back('^');
                    md.push_back(kDecode[q[i] & 15]);
                    ++i;
                    break;
                case kOpD: ++j; break;
                default: break;
            }
            prev = o;
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

// Per-thread buffers reused across reads.
struct Scratch {
    std::vector<uint8_t> rc, rq;
    std::vector<int64_t> keep;
    std::vector<double> l10, post, pr;
    std::vector<int> mapq;
    std::vector<char> empty;
    std::vector<size_t> ord;
};

void tail_read(int64_t r, const uint8_t* seq, const uint8_t* qual, int64_t L, const msg_aln* aln, int64_t k0,
               int64_t k1, const uint32_t* cigar, const std::vector<Target>& tg, const msg_tail_params& p,
               Scratch& sc, ReadOut& out) {
    static const uint8_t kComp[16] = {0, 8, 4, 12, 2, 10, 6, 14, 1, 9, 5, 13, 3, 11, 7, 15};
    std::vector<uint8_t>& rc = sc.rc;
    std::vector<uint8_t>& rq = sc.rq;
    // Alignment::filter (src/Alignment.cpp:548-555)
    std::vector<int64_t>& keep = sc.keep;
    keep.clear();
    for (int64_t k = k0; k < k1; ++k) {
        const double score = aln[k].aln_score == INT32_MIN ? -INFINITY : (double)aln[k].aln_score;
        if (!(score < L * p.min_score_rate)) keep.push_back(k);
    }
    if (keep.empty()) {  // output(read, out): an unmapped record (src/msgseqtk-align.cpp:583-585)
        msg_sam_rec u{};
        u.read = r;
        u.flag = kFlagUnmapped;
        u.tid = -1;
        out.rec.push_back(u);
        return;
    }
    bool any_rev = false;
    for (int64_t k : keep) any_rev |= aln[k].strand == 2;
    rq.resize(2 * L);  // reversed quality, then zeros for reads without one
    if (!qual) std::fill(rq.begin() + L, rq.end(), 0);
    if (any_rev) {  // PrimarySeq::revcom: reversed, complemented; quality reversed
        rc.resize(L);
        for (int64_t i = 0; i < L; ++i) {
            rc[i] = kComp[seq[L - 1 - i] & 15];
            rq[i] = qual ? qual[L - 1 - i] : 0;
        }
    }
    const uint8_t* fq = qual ? qual : rq.data() + L;
    const size_t N = keep.size();
    sc.l10.resize(N);
    sc.post.resize(N);
    sc.pr.resize(N);
    sc.mapq.resize(N);
    sc.empty.resize(N);
    sc.ord.resize(N);
    std::vector<double>& l10 = sc.l10;
    std::vector<double>& post = sc.post;
    std::vector<int>& mapq = sc.mapq;
    std::vector<char>& empty = sc.empty;
    for (size_t n = 0; n < N; ++n) {
        const msg_aln& a = aln[keep[n]];
        const bool rev = a.strand == 2;
        bool e;
        l10[n] = evaluate(rev ? rc.data() : seq, rev ? rq.data() : fq, L, tg[a.tid].seq, a, cigar + a.cigar_off, p,
                          &e);
        empty[n] = e;
    }
    // Alignment::calcMapQ (src/Alignment.cpp:491-512); loglik = log10lik / log10(e)
    std::vector<double>& pr = sc.pr;
    static const double log10e = std::log10(M_E);
    for (size_t n = 0; n < N; ++n) pr[n] = l10[n] / log10e;
    double maxV = pr[0];
    for (double x : pr) if (x > maxV) maxV = x;
    const double scale = maxV != -INFINITY && maxV < kMinLoglikExp ? kMinLoglikExp - maxV : 0;
    if (N == 1 && std::isfinite(pr[0]) && pr[0] + scale < 700) {
        // exp(x + scale) is finite and above 0 (x + scale >= -256), so postP = pr / pr = 1 and
        // MAPQ = min(round(-10 * log10(0)), 250) = 250
        post[0] = 1.0;
        mapq[0] = (int)kMaxQ;
    } else {
        for (double& x : pr) x = std::exp(x + scale);
        double sum = 0;
        for (double x : pr) sum += x;
        for (size_t n = 0; n < N; ++n) {
            post[n] = pr[n] / sum;
            const double mq = kPhredScale * std::log10(1 - post[n]);
            mapq[n] = (int)(uint8_t)std::min(std::round(mq), kMaxQ);
        }
    }
    // Alignment::sort (src/Alignment.h:629-633): std::sort by log10P, decreasing
    std::vector<size_t>& ord = sc.ord;
    for (size_t n = 0; n < N; ++n) ord[n] = n;
    std::sort(ord.begin(), ord.end(), [&](size_t x, size_t y) { return l10[x] > l10[y]; });
    const size_t num = p.max_report == 0 ? N : std::min<size_t>(p.max_report, N);
    for (size_t s = 0; s < num; ++s) {
        const size_t n = ord[s];
        const msg_aln& a = aln[keep[n]];
        msg_sam_rec o{};
        o.read = r;
        o.flag = (a.strand == 2 ? kFlagReverse : 0) | (s > 0 ? kFlagSecondary : 0);
        o.tid = a.tid;
        o.pos = a.aln_start;
        o.mapq = mapq[n];
        o.as = (int32_t)std::round((double)a.aln_score);
        o.xh = (float)l10[n];
        o.xp = (float)post[n];
        o.nh = (int32_t)num;
        o.xn = (int32_t)N;
        o.cigar_off = a.cigar_off;
        o.n_cigar = a.n_cigar;
        o.md_off = (int64_t)out.md.size();
        if (!empty[n]) {
            const uint8_t* q = a.strand == 2 ? rc.data() : seq;
            md_tag(q, tg[a.tid].seq, a.aln_from, a.aln_start, cigar + a.cigar_off, a.n_cigar, out.md);
        }
        o.md_len = (int32_t)((int64_t)out.md.size() - o.md_off);
        out.rec.push_back(o);
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

extern "C" int msg_tail_batch(const msg_mtg_view* mtg, const msg_read_batch* reads, const uint8_t* quals,
                              const msg_aln* aln, const uint32_t* cigar, const int64_t* read_aln_off,
                              const msg_tail_params* p, msg_sam_rec* out, int64_t out_cap, char* md, int64_t md_cap,
                              int64_t* n_out, int64_t* md_len) {
    if (!mtg || !reads || !read_aln_off || !p || !n_out || !md_len) return MSG_EINVAL;
    const int64_t n = reads->n_reads;
    if (n < 0 || (n > 0 && (!reads->seq || !reads->off))) return MSG_EINVAL;
    if (std::isnan(p->min_score_rate)) return MSG_EINVAL;
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
    int nt = p->n_threads > 0 ? p->n_threads : (int)std::max(1u, std::thread::hardware_concurrency());
    nt = (int)std::max<int64_t>(1, std::min<int64_t>(nt, (n + 255) / 256));
    std::vector<ReadOut> parts(nt);
    std::vector<char> bad(nt, 0);
    auto work = [&](int w) {
        Scratch sc;
        const int64_t a = n * w / nt, b = n * (w + 1) / nt;
        parts[w].rec.reserve((size_t)(b - a) * std::max<uint32_t>(1, p->max_report));
        for (int64_t i = a; i < b; ++i) {
            if (!valid(i)) { bad[w] = 1; return; }
            const int64_t o = reads->off[i];
            tail_read(i, reads->seq + o, quals ? quals + o : nullptr, reads->off[i + 1] - o, aln, read_aln_off[i],
                      read_aln_off[i + 1], cigar, tg, *p, sc, parts[w]);
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
