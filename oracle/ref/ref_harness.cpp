/*
 * Test-only harness around the UNMODIFIED MSGseqTK v1.2.3 sources (compiled in
 * place from the reference tree by oracle/ref/Makefile). It exposes a small
 * extern "C" surface so that Python tests can run the reference's own
 * read-mapping path as the checker for the CUDA path, and so the bench can time
 * the reference's OpenMP CPU path. Nothing in the product links this file.
 *
 * The reference keeps SMEM bi-interval fields private and its
 * SMEM::getFwdStart() getter recurses forever (SMEM.h:84-90), so this
 * translation unit alone reads SMEM members through a private->public define.
 */
#include <cstdint>
#include <cstring>
#include <vector>
#include <string>
#include <algorithm>
#include <cmath>
#include <chrono>
#include <array>
#include <set>
#include <map>
#include <unordered_map>
#include <unordered_set>
#include <iostream>
#include <sstream>
#include <fstream>
#include <regex>
#include <limits>
#include <stdexcept>
#include <utility>
#include <stack>
#include <numeric>
#include <cassert>
#ifdef _OPENMP
#include <omp.h>
#endif

#define private public
#define protected public
#include "SMEM.h"
#include "SeedChain.h"
#include "Alignment.h"
#include "ProgEnv.h"
#include "SeqIO.h"
#include "from_device.h"
#undef private
#undef protected

using namespace EGriceLab::MSGseqTK;

namespace {

struct RefDB {
    MetaGenome mtg;
    FMDIndex fmd;
};

/* Decode 2-bit-free ASCII (ACGTN...) into a reference PrimarySeq. */
PrimarySeq make_read(const uint8_t* nt16, int64_t L, const uint8_t* qual, const char* name) {
    DNAseq seq(nt16, nt16 + L);
    QualStr q;
    if (qual) q.assign(qual, qual + L);
    else q.assign(L, 30);
    return PrimarySeq(seq, name ? std::string(name) : std::string("r"), std::string(""), q);
}

}  // namespace

extern "C" {

/* Build a MetaGenome of n genomes with one chromosome each (chromosome k has
 * nt16 codes seqs[offs[k]..offs[k+1]) ), then the FMD-index the same way
 * msgseqtk-build does for a DB below the block size (msgseqtk-build.cpp:435-438):
 * FMDIndex(mtg.getBDSeq(), true, 32). */
void* ref_db_build(int64_t n_chrom, const uint8_t* seqs, const int64_t* offs) {
    RefDB* db = new RefDB();
    for (int64_t k = 0; k < n_chrom; ++k) {
        Genome g("g" + std::to_string(k), "genome" + std::to_string(k));
        DNAseq s(seqs + offs[k], seqs + offs[k + 1]);
        g.addChrom("chr" + std::to_string(k), s);
        db->mtg.addGenome(g);
    }
    db->mtg.updateIndex();
    db->fmd = FMDIndex(db->mtg.getBDSeq(), true, FMDIndex::SA_SAMPLE_RATE);
    return db;
}

/* Same DB, with the FMD-index assembled from an already decoded view (BWT,
 * base counts, SA samples) by the reference's own structures: the BWT goes
 * into WaveletTreeRRR(bwt, 0, 15, 32) exactly as the FMDIndex constructor does
 * (FMDIndex.cpp:66), SAidx into BitSeqRRR(bits, 32) (FMDIndex.cpp:477), and
 * C[] is accumulated as buildCounts does (FMDIndex.cpp:124-129). Used for
 * large synthetic DBs where divsufsort on the host would dominate the run;
 * the view equals what the constructor builds (suffix arrays are unique). */
void* ref_db_from_view(int64_t n_chrom, const uint8_t* seqs, const int64_t* offs, int64_t n, const uint8_t* bwt,
                       const int64_t* B16, int64_t n_samples, const int64_t* rows, const int64_t* vals,
                       const int64_t* gap_sa) {
    RefDB* db = new RefDB();
    for (int64_t k = 0; k < n_chrom; ++k) {
        Genome g("g" + std::to_string(k), "genome" + std::to_string(k));
        DNAseq s(seqs + offs[k], seqs + offs[k + 1]);
        g.addChrom("chr" + std::to_string(k), s);
        db->mtg.addGenome(g);
    }
    db->mtg.updateIndex();
    FMDIndex& f = db->fmd;
    for (int i = 0; i < 256; ++i) { f.B[i] = 0; f.C[i] = 0; }
    for (int i = 0; i < 16; ++i) f.B[i] = B16[i];
    int64_t S = 0;
    for (int i = 0; i <= 16; ++i) { f.C[i] = S; S += f.B[i]; }
    {
        DNAseq b(bwt, bwt + n);
        f.bwtRRR = WaveletTreeRRR(b, 0, DNAalphabet::NT16_MAX, FMDIndex::RRR_SAMPLE_RATE);
    }
    f.gapSA.assign(gap_sa, gap_sa + B16[0]);
    {
        BitStr32 bstr(n);
        for (int64_t k = 0; k < n_samples; ++k) bstr.set(rows[k]);
        f.SAidx = BitSeqRRR(bstr, FMDIndex::RRR_SAMPLE_RATE);
    }
    f.SAsampled.assign(vals, vals + n_samples);
    return db;
}

/* msgseqtk-mergedb's merge (src/msgseqtk-mergedb.cpp:235-262) of two DBs
 * built as ref_db_build does (genome names a<k> and b<k>): the MetaGenome and
 * the FMD-index of the second appended to the first (BWT merge), then
 * updateIndex and buildSA. */
void* ref_db_merge(int64_t na, const uint8_t* seqs_a, const int64_t* offs_a, int64_t nb, const uint8_t* seqs_b,
                   const int64_t* offs_b) {
    auto build = [](int64_t n, const uint8_t* seqs, const int64_t* offs, const char* tag) {
        RefDB* db = new RefDB();
        for (int64_t k = 0; k < n; ++k) {
            Genome g(tag + std::to_string(k), "genome " + std::string(tag) + std::to_string(k));
            DNAseq s(seqs + offs[k], seqs + offs[k + 1]);
            g.addChrom(std::string(tag) + "chr" + std::to_string(k), s);
            db->mtg.addGenome(g);
        }
        db->mtg.updateIndex();
        db->fmd = FMDIndex(db->mtg.getBDSeq(), true, FMDIndex::SA_SAMPLE_RATE);
        return db;
    };
    RefDB* a = build(na, seqs_a, offs_a, "a");
    RefDB* b = build(nb, seqs_b, offs_b, "b");
    a->mtg += b->mtg;
    a->fmd += b->fmd;
    delete b;
    a->mtg.updateIndex();
    a->fmd.buildSA(FMDIndex::SA_SAMPLE_RATE);
    return a;
}

void ref_db_free(void* h) { delete (RefDB*)h; }

int64_t ref_db_length(void* h) { return ((RefDB*)h)->fmd.length(); }

int64_t ref_db_num_chroms(void* h) { return ((RefDB*)h)->mtg.numChroms(); }

/* B[256] and C[256] of the FMD-index. */
void ref_db_counts(void* h, int64_t* B, int64_t* C) {
    RefDB* db = (RefDB*)h;
    for (int i = 0; i < 256; ++i) { B[i] = db->fmd.B[i]; C[i] = db->fmd.C[i]; }
}

/* The BWT as nt16 codes (FMDIndex::getBWT, FMDIndex.cpp:195). */
void ref_db_bwt(void* h, uint8_t* out) {
    DNAseq b = ((RefDB*)h)->fmd.getBWT();
    std::memcpy(out, b.data(), b.size());
}

/* The BD text (MetaGenome::getBDSeq, MetaGenome.h:333). */
void ref_db_bdseq(void* h, uint8_t* out) {
    DNAseq s = ((RefDB*)h)->mtg.getBDSeq();
    std::memcpy(out, s.data(), s.size());
}

int64_t ref_db_access_sa(void* h, int64_t i) { return ((RefDB*)h)->fmd.accessSA(i); }

int64_t ref_db_rank(void* h, int64_t b, int64_t i) { return (int64_t)((RefDB*)h)->fmd.bwtRRR.rank(b, i); }

/* The reference's own SA sample set: rows flagged in SAidx and their values. */
int64_t ref_db_sa_samples(void* h, int64_t* rows, int64_t* vals, int64_t cap) {
    RefDB* db = (RefDB*)h;
    const int64_t n = db->fmd.length();
    int64_t k = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (db->fmd.SAidx.access(i)) {
            if (k < cap) { rows[k] = i; vals[k] = db->fmd.SAsampled[db->fmd.SAidx.rank1(i) - 1]; }
            ++k;
        }
    }
    return k;
}

/* Chromosome table: BD start/end and forward length per tid. */
void ref_db_chroms(void* h, int64_t* bd_start, int64_t* bd_end, int64_t* chr_len) {
    RefDB* db = (RefDB*)h;
    for (size_t t = 0; t < db->mtg.numChroms(); ++t) {
        bd_start[t] = db->mtg.getChromBDStart(t);
        bd_end[t] = db->mtg.getChromBDEnd(t);
        chr_len[t] = db->mtg.getChromLength(t);
    }
}

/* FMDIndex::backExt on an arbitrary bi-interval; returns the new size. */
int64_t ref_back_ext(void* h, int64_t* p, int64_t* q, int64_t* s, int b) {
    return ((RefDB*)h)->fmd.backExt(*p, *q, *s, (nt16_t)b);
}

int64_t ref_fwd_ext(void* h, int64_t* p, int64_t* q, int64_t* s, int b) {
    return ((RefDB*)h)->fmd.fwdExt(*p, *q, *s, (nt16_t)b);
}

double ref_loglik(void* h, int b) { return ((RefDB*)h)->fmd.loglik((nt16_t)b); }

/* SMEM_LIST::findAllSMEMS (SMEM.cpp:186) in emission order.
 * out rows of 6: from, to, fwdStart, revStart, size, logP(bits). */
int64_t ref_find_smems(void* h, const uint8_t* read, int64_t L, int64_t min_len, double max_evalue,
                       int64_t* out, int64_t cap) {
    RefDB* db = (RefDB*)h;
    PrimarySeq r = make_read(read, L, nullptr, "r");
    SMEM_LIST smems = SMEM_LIST::findAllSMEMS(&r, &db->mtg, &db->fmd, min_len, max_evalue);
    int64_t k = 0;
    for (const SMEM& m : smems) {
        if (k < cap) {
            int64_t* o = out + 6 * k;
            o[0] = m.from; o[1] = m.to; o[2] = m.fwdStart; o[3] = m.revStart; o[4] = m.size;
            std::memcpy(&o[5], &m.logP, 8);
        }
        ++k;
    }
    return k;
}

/* SMEM_LIST::findSeeds (SMEM.cpp:271): rows of 6: from, to, start, end, tid, strand. */
int64_t ref_find_seeds(void* h, const uint8_t* read, int64_t L, int64_t min_len, double max_evalue,
                       int64_t max_nseed, int64_t* out, int64_t cap) {
    RefDB* db = (RefDB*)h;
    PrimarySeq r = make_read(read, L, nullptr, "r");
    SeedList seeds = SMEM_LIST::findSeeds(&r, &db->mtg, &db->fmd, min_len, max_evalue, max_nseed);
    int64_t k = 0;
    for (const SeedPair& s : seeds) {
        if (k < cap) {
            int64_t* o = out + 6 * k;
            o[0] = s.getFrom(); o[1] = s.getTo(); o[2] = s.getStart(); o[3] = s.getEnd();
            o[4] = s.getTid(); o[5] = (int64_t)s.getStrand();
        }
        ++k;
    }
    return k;
}

/* SeedChain::getChains (SeedChain.cpp:40) on given seeds (rows of 6 as above).
 * out_idx receives, per chain, the indices of its seeds; out_off the chain
 * offsets (n_chain + 1 entries). Returns the number of chains. */
int64_t ref_get_chains(const int64_t* seeds, int64_t n, int64_t max_mismatch, int64_t max_indel,
                       int64_t* out_off, int64_t* out_idx, int64_t cap_chain, int64_t cap_idx) {
    SeedList list;
    for (int64_t i = 0; i < n; ++i) {
        const int64_t* s = seeds + 6 * i;
        list.push_back(SeedPair(s[0], s[2], s[1] - s[0], s[4], (GLoc::STRAND)s[5], 0.0));
    }
    ChainList chains = SeedChain::getChains(list, max_mismatch, max_indel);
    int64_t nc = 0, ni = 0;
    if (cap_chain > 0) out_off[0] = 0;
    for (const SeedChain& c : chains) {
        for (const SeedPair& s : c) {
            int64_t idx = -1;
            for (int64_t i = 0; i < n; ++i) if (list[i] == s) { idx = i; break; }
            if (ni < cap_idx) out_idx[ni] = idx;
            ++ni;
        }
        ++nc;
        if (nc < cap_chain + 1 && cap_chain > 0 && nc <= cap_chain) out_off[nc] = ni;
    }
    return nc;
}

/* One alignment record as the reference builds it per chain
 * (Alignment::buildAlignments, Alignment.cpp:420), before filtering. */
struct RefAln {
    int64_t tid, strand, t_start, t_end, aln_from, aln_to, aln_start, aln_end;
    double aln_score;
    int64_t n_cigar;
    int64_t cigar_off;
    int64_t md_off;
    int64_t md_len;
};

/* Per-read SE mapping through chain DP: seeds -> chains -> alignments.
 * cigar words and MD text are appended into the given buffers. Returns the
 * number of alignments (unfiltered, chain order). */
int64_t ref_align_read(void* h, const uint8_t* read, int64_t L, int64_t min_len, double max_evalue,
                       int64_t max_nseed, int mode, RefAln* out, int64_t cap,
                       uint32_t* cigar_buf, int64_t cigar_cap, int64_t* cigar_used,
                       char* md_buf, int64_t md_cap, int64_t* md_used) {
    RefDB* db = (RefDB*)h;
    /* const, as in msgseqtk-align.cpp:603-604: the non-const revcom()
     * overload would reverse-complement the read in place */
    const PrimarySeq r = make_read(read, L, nullptr, "r");
    const PrimarySeq rc = r.revcom();
    SeedList seeds = SMEM_LIST::findSeeds(&r, &db->mtg, &db->fmd, min_len, max_evalue, max_nseed);
    if (seeds.empty()) return 0;
    const int64_t maxMismatch = std::ceil(L * Alignment::MAX_MISMATCH_RATE);
    const int64_t maxIndel = std::ceil(L * Alignment::MAX_INDEL_RATE);
    ChainList chains = SeedChain::getChains(seeds, maxMismatch, maxIndel);
    ALIGN_LIST alns = Alignment::buildAlignments(&r, &rc, db->mtg, chains,
                                                 mode == 0 ? Alignment::GLOBAL : Alignment::LOCAL);
    int64_t k = 0;
    for (const Alignment& a : alns) {
        if (k < cap) {
            RefAln& o = out[k];
            o.tid = a.tid; o.strand = a.qStrand; o.t_start = a.tStart; o.t_end = a.tEnd;
            o.aln_from = a.alnFrom; o.aln_to = a.alnTo; o.aln_start = a.alnStart; o.aln_end = a.alnEnd;
            o.aln_score = a.alnScore;
            BAM::cigar_str cg = a.getAlnCigar();
            std::string md = a.getAlnMDTag();
            o.n_cigar = cg.size();
            o.cigar_off = *cigar_used;
            for (uint32_t w : cg) { if (*cigar_used < cigar_cap) cigar_buf[*cigar_used] = w; ++*cigar_used; }
            o.md_off = *md_used;
            o.md_len = md.size();
            for (char ch : md) { if (*md_used < md_cap) md_buf[*md_used] = ch; ++*md_used; }
        }
        ++k;
    }
    return k;
}

/* The reference's SE mapping task body (msgseqtk-align.cpp:610-648) over a
 * batch of reads with OpenMP, for timing: findSeeds -> getChains ->
 * buildAlignments -> filter -> evaluate -> calcMapQ -> sort. reads are nt16
 * codes at offs[i]..offs[i+1]; quals likewise. Returns the number of reads
 * with at least one alignment kept; *seconds gets the steady_clock time. */
int64_t ref_map_batch(void* h, int64_t n_reads, const uint8_t* reads, const uint8_t* quals,
                      const int64_t* offs, int64_t min_len, double max_evalue, int64_t max_nseed,
                      double min_score_rate, int n_threads, double* seconds, int64_t* n_aln_out) {
    RefDB* db = (RefDB*)h;
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#endif
    int64_t mapped = 0, n_aln = 0;
    auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : mapped, n_aln)
    for (int64_t i = 0; i < n_reads; ++i) {
        const int64_t L = offs[i + 1] - offs[i];
        const PrimarySeq r = make_read(reads + offs[i], L, quals ? quals + offs[i] : nullptr, "r");
        const PrimarySeq rc = r.revcom();
        SeedList seeds = SMEM_LIST::findSeeds(&r, &db->mtg, &db->fmd, min_len, max_evalue, max_nseed);
        if (seeds.empty()) continue;
        const int64_t maxMismatch = std::ceil(L * Alignment::MAX_MISMATCH_RATE);
        const int64_t maxIndel = std::ceil(L * Alignment::MAX_INDEL_RATE);
        ChainList chains = SeedChain::getChains(seeds, maxMismatch, maxIndel);
        ALIGN_LIST alns = Alignment::buildAlignments(&r, &rc, db->mtg, chains, Alignment::GLOBAL);
        Alignment::filter(alns, min_score_rate);
        if (alns.empty()) continue;
        Alignment::evaluate(alns);
        Alignment::calcMapQ(alns);
        Alignment::sort(alns);
        mapped += 1;
        n_aln += (int64_t)alns.size();
    }
    auto t1 = std::chrono::steady_clock::now();
    *seconds = std::chrono::duration<double>(t1 - t0).count();
    *n_aln_out = n_aln;
    return mapped;
}

/* SMEM_LIST::findMEMS (SMEM.cpp:174-184): rows of 6 as ref_find_smems;
 * *loglik = MEM_LIST::loglik (SMEM.cpp:307-312). Returns the MEM count. */
int64_t ref_find_mems(void* h, const uint8_t* read, int64_t L, int64_t min_len, double max_evalue,
                      int64_t* out, int64_t cap, double* loglik) {
    RefDB* db = (RefDB*)h;
    PrimarySeq r = make_read(read, L, nullptr, "r");
    MEM_LIST mems = SMEM_LIST::findMEMS(&r, &db->mtg, &db->fmd, min_len, max_evalue);
    int64_t k = 0;
    for (const MEM& m : mems) {
        if (k < cap) {
            int64_t* o = out + 6 * k;
            o[0] = m.from; o[1] = m.to; o[2] = m.fwdStart; o[3] = m.revStart; o[4] = m.size;
            std::memcpy(&o[5], &m.logP, 8);
        }
        ++k;
    }
    if (loglik) *loglik = mems.loglik();
    return k;
}

/* msgseqtk-clean's per-read task body (msgseqtk-clean.cpp:425-438 single-end,
 * :462-475 paired-end when rev_reads is not NULL) over a batch with OpenMP:
 * findMEMS on the reference and on the background index, the lists' loglik,
 * lod = -refLoglik + bgLoglik, kept when lod > min_lod. Outputs may be NULL;
 * *seconds gets the steady_clock time. Returns the number of kept reads. */
int64_t ref_clean_batch(void* h_ref, void* h_bg, int64_t n_reads, const uint8_t* reads, const int64_t* offs,
                        const uint8_t* rev_reads, const int64_t* rev_offs, int64_t min_len, double max_evalue,
                        double min_lod, int n_threads, double* ref_ll, double* bg_ll, double* lod_out,
                        uint8_t* keep, double* seconds) {
    RefDB* rdb = (RefDB*)h_ref;
    RefDB* bdb = (RefDB*)h_bg;
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#endif
    int64_t kept = 0;
    auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : kept)
    for (int64_t i = 0; i < n_reads; ++i) {
        const PrimarySeq fwd = make_read(reads + offs[i], offs[i + 1] - offs[i], nullptr, "r");
        double refLoglik, bgLoglik;
        if (rev_reads) {
            const PrimarySeq rev = make_read(rev_reads + rev_offs[i], rev_offs[i + 1] - rev_offs[i], nullptr, "r");
            MEM_LIST_PE refMemsPE = SMEM_LIST::findMEMS_PE(&fwd, &rev, &rdb->mtg, &rdb->fmd, min_len, max_evalue);
            MEM_LIST_PE bgMemsPE = SMEM_LIST::findMEMS_PE(&fwd, &rev, &bdb->mtg, &bdb->fmd, min_len, max_evalue);
            refLoglik = SMEM_LIST::loglik(refMemsPE);
            bgLoglik = SMEM_LIST::loglik(bgMemsPE);
        } else {
            MEM_LIST refMems = SMEM_LIST::findMEMS(&fwd, &rdb->mtg, &rdb->fmd, min_len, max_evalue);
            MEM_LIST bgMems = SMEM_LIST::findMEMS(&fwd, &bdb->mtg, &bdb->fmd, min_len, max_evalue);
            refLoglik = refMems.loglik();
            bgLoglik = bgMems.loglik();
        }
        const double lod = -refLoglik + bgLoglik;
        if (ref_ll) ref_ll[i] = refLoglik;
        if (bg_ll) bg_ll[i] = bgLoglik;
        if (lod_out) lod_out[i] = lod;
        if (keep) keep[i] = lod > min_lod;
        kept += lod > min_lod;
    }
    auto t1 = std::chrono::steady_clock::now();
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    return kept;
}

/* ---- SAM records -----------------------------------------------------
 * Each read's SAM records as text lines, from the reference's own tail:
 * Alignment::filter/evaluate/calcMapQ/sort and exportBAM, plus the
 * per-read output step of msgseqtk-align (src/msgseqtk-align.cpp:538-556 for
 * mapped reads, :583-585 for unmapped ones), which lives in the program file
 * and is restated here. A line holds the BAM fields the shim records:
 * QNAME FLAG TID POS MAPQ CIGAR L_SEQ SEQ QUAL ISIZE then the aux tags in order,
 * float tags as the hex of their float32 value, so comparisons are exact. */
static void put_bam(const EGriceLab::SAMtools::BAM& b, std::string& out) {
    char buf[64];
    out += b.qname;
    std::snprintf(buf, sizeof buf, "\t%u\t%d\t%d\t%u\t", (unsigned)b.flag, b.tid, b.pos, (unsigned)b.mapQ);
    out += buf;
    for (uint32_t c : b.cigar) {
        std::snprintf(buf, sizeof buf, "%u%c", c >> 4, "MIDNSHP=XB"[c & 0xf]);
        out += buf;
    }
    if (b.cigar.empty()) out += "*";
    std::snprintf(buf, sizeof buf, "\t%d\t", b.l_seq);
    out += buf;
    for (uint8_t x : b.seq) { std::snprintf(buf, sizeof buf, "%x", (unsigned)x); out += buf; }
    out += "\t";
    for (uint8_t x : b.qual) { std::snprintf(buf, sizeof buf, "%02x", (unsigned)x); out += buf; }
    std::snprintf(buf, sizeof buf, "\t%d", b.isize);
    out += buf;
    for (const auto& a : b.aux) {
        out += "\t" + a.tag + ":" + a.type + ":";
        if (a.type == 'Z') out += a.str;
        else if (a.type == 'f') { std::snprintf(buf, sizeof buf, "%a", (double)(float)a.num); out += buf; }
        else { std::snprintf(buf, sizeof buf, "%lld", (long long)a.num); out += buf; }
    }
    out += "\n";
}

static void sam_read(ALIGN_LIST& alns, const PrimarySeq& read, double min_score_rate, uint32_t max_report,
                     std::string& out) {
    using EGriceLab::SAMtools::BAM;
    Alignment::filter(alns, min_score_rate);
    if (alns.empty()) {  // output(read, out)
        put_bam(BAM(read.getName(), read.length(), dna::nt16Encode(read.getSeq()), read.getQual(), BAM_FUNMAP), out);
        return;
    }
    Alignment::evaluate(alns);
    Alignment::calcMapQ(alns);
    Alignment::sort(alns);
    const size_t num_report = max_report == 0 ? alns.size() : std::min((size_t)max_report, alns.size());
    for (size_t i = 0; i < num_report; ++i) {
        BAM b = alns[i].exportBAM();
        b.setSecondaryFlag(i > 0);
        b.setAux(Alignment::NUM_REPORTED_ALIGNMENT_TAG, num_report);
        b.setAux(Alignment::NUM_TOTAL_ALIGNMENT_TAG, alns.size());
        b.setAux(Alignment::ALIGNMENT_POSTERIOR_PROB_TAG, alns[i].getPostP());
        put_bam(b, out);
    }
}

static int64_t put_out(const std::string& s, char* out, int64_t cap) {
    if ((int64_t)s.size() <= cap && out) std::memcpy(out, s.data(), s.size());
    return (int64_t)s.size();
}

/* The paired-end output steps of msgseqtk-align (src/msgseqtk-align.cpp:558-581
 * for pairs, :538-556 with extra flags for unpaired mates, :587-591 for an
 * unmapped pair), restated (they live in the program file), and its per-pair
 * tail after buildAlignments (:703-748). */
static void sam_pair_out(const PAIR_LIST& pairs, uint32_t max_report, std::string& out) {
    const size_t num = max_report == 0 ? pairs.size() : std::min<size_t>(max_report, pairs.size());
    for (size_t i = 0; i < num; ++i) {
        const AlignmentPE& pair = pairs[i];
        EGriceLab::SAMtools::BAM f = pair.exportFwdBAM(), r = pair.exportRevBAM();
        f.setSecondaryFlag(i > 0);
        r.setSecondaryFlag(i > 0);
        f.setAux(Alignment::NUM_REPORTED_ALIGNMENT_TAG, num);
        f.setAux(Alignment::NUM_TOTAL_ALIGNMENT_TAG, pairs.size());
        r.setAux(Alignment::NUM_REPORTED_ALIGNMENT_TAG, num);
        r.setAux(Alignment::NUM_TOTAL_ALIGNMENT_TAG, pairs.size());
        f.setAux(Alignment::ALIGNMENT_POSTERIOR_PROB_TAG, pair.postP);
        r.setAux(Alignment::ALIGNMENT_POSTERIOR_PROB_TAG, pair.postP);
        put_bam(f, out);
        put_bam(r, out);
    }
}

static void sam_list_out(const ALIGN_LIST& alns, uint32_t max_report, uint16_t extra, std::string& out) {
    const size_t num = max_report == 0 ? alns.size() : std::min((size_t)max_report, alns.size());
    for (size_t i = 0; i < num; ++i) {
        EGriceLab::SAMtools::BAM b = alns[i].exportBAM();
        b.setSecondaryFlag(i > 0);
        b.setFlag(b.getFlag() | extra);
        b.setAux(Alignment::NUM_REPORTED_ALIGNMENT_TAG, num);
        b.setAux(Alignment::NUM_TOTAL_ALIGNMENT_TAG, alns.size());
        b.setAux(Alignment::ALIGNMENT_POSTERIOR_PROB_TAG, alns[i].getPostP());
        put_bam(b, out);
    }
}

static void sam_pair(ALIGN_LIST& fa, ALIGN_LIST& ra, const PrimarySeq& f, const PrimarySeq& r, double min_score_rate,
                     uint32_t max_report, const int* opt, int64_t max_npair, std::string& out) {
    using EGriceLab::SAMtools::BAM;
    Alignment::filter(fa, min_score_rate);
    Alignment::filter(ra, min_score_rate);
    if (fa.empty() && ra.empty()) {  // output(fwdRead, revRead, out)
        put_bam(BAM(f.getName(), f.length(), dna::nt16Encode(f.getSeq()), f.getQual(),
                    BAM_FUNMAP | BAM_FMUNMAP | BAM_FPAIRED | BAM_FREAD1), out);
        put_bam(BAM(r.getName(), r.length(), dna::nt16Encode(r.getSeq()), r.getQual(),
                    BAM_FUNMAP | BAM_FMUNMAP | BAM_FPAIRED | BAM_FREAD2), out);
        return;
    }
    Alignment::evaluate(fa);
    Alignment::evaluate(ra);
    PAIR_LIST pairs = AlignmentPE::getPairs(fa, ra);
    AlignmentPE::sort(pairs);
    AlignmentPE::filter(pairs, opt[1], opt[2], opt[3], opt[4], max_npair);
    if (!pairs.empty()) {
        AlignmentPE::calcMapQ(pairs);
        sam_pair_out(pairs, max_report, out);
    } else if (!opt[0]) {
        if (!fa.empty()) {
            Alignment::calcMapQ(fa);
            Alignment::sort(fa);
            sam_list_out(fa, max_report, BAM_FPAIRED | BAM_FREAD1, out);
        }
        if (!ra.empty()) {
            Alignment::calcMapQ(ra);
            Alignment::sort(ra);
            sam_list_out(ra, max_report, BAM_FPAIRED | BAM_FREAD2, out);
        }
    }
}

/* AlignmentPE::ps as msgseqtk-align leaves it after its options
 * (src/msgseqtk-align.cpp:267-300, 400): mean, sd, insert range, then
 * updateParam. */
static void set_pairing(double mean, double sd, double min_ins, double max_ins) {
    AlignmentPE::ps.setMean(mean);
    AlignmentPE::ps.setSD(sd);
    AlignmentPE::ps.setRange(min_ins, max_ins);
    AlignmentPE::ps.updateParam();
}

/* SAM lines of the reference's paired-end path (src/msgseqtk-align.cpp:680-748)
 * for n_pairs pairs whose mates are reads 2i and 2i+1 of the batch (GLOBAL
 * mode). opt = {noMixed, noDiscordant, noTailOver, noContain, noOverlap}.
 * Returns the text length; written only when it fits in cap bytes. */
int64_t ref_sam_pe_batch(void* h, int64_t n_pairs, const uint8_t* reads, const uint8_t* quals, const int64_t* offs,
                         int64_t min_len, double max_evalue, int64_t max_nseed, double min_score_rate,
                         int max_report, double mean, double sd, double min_ins, double max_ins, const int* opt,
                         int64_t max_npair, char* out, int64_t cap) {
    RefDB* db = (RefDB*)h;
    set_pairing(mean, sd, min_ins, max_ins);
    std::string text;
    for (int64_t i = 0; i < n_pairs; ++i) {
        const std::string name = "p" + std::to_string(i);
        // const, so that revcom() makes a copy (the non-const overload reverses
        // in place; main_PE casts to const for the same reason)
        const PrimarySeq f = make_read(reads + offs[2 * i], offs[2 * i + 1] - offs[2 * i],
                                       quals ? quals + offs[2 * i] : nullptr, name.c_str());
        const PrimarySeq r = make_read(reads + offs[2 * i + 1], offs[2 * i + 2] - offs[2 * i + 1],
                                       quals ? quals + offs[2 * i + 1] : nullptr, name.c_str());
        const PrimarySeq rcf = f.revcom(), rcr = r.revcom();
        SeedListPE seeds = SMEM_LIST::findSeedsPE(&f, &r, &db->mtg, &db->fmd, min_len, max_evalue, max_nseed);
        ALIGN_LIST fa, ra;
        if (!(seeds.first.empty() && seeds.second.empty())) {
            const int64_t fL = f.length(), rL = r.length();
            ChainList fc = SeedChain::getChains(seeds.first, std::ceil(fL * Alignment::MAX_MISMATCH_RATE),
                                                std::ceil(fL * Alignment::MAX_INDEL_RATE));
            ChainList rch = SeedChain::getChains(seeds.second, std::ceil(rL * Alignment::MAX_MISMATCH_RATE),
                                                 std::ceil(rL * Alignment::MAX_INDEL_RATE));
            fa = Alignment::buildAlignments(&f, &rcf, db->mtg, fc, Alignment::GLOBAL);
            ra = Alignment::buildAlignments(&r, &rcr, db->mtg, rch, Alignment::GLOBAL);
        }
        sam_pair(fa, ra, f, r, min_score_rate, (uint32_t)max_report, opt, max_npair, text);
    }
    return put_out(text, out, cap);
}

/* SAM lines of the reference's single-end path (src/msgseqtk-align.cpp:600-640)
 * for n reads (GLOBAL mode). Returns the text length; the text is written
 * only when it fits in cap bytes. */
int64_t ref_sam_batch(void* h, int64_t n_reads, const uint8_t* reads, const uint8_t* quals, const int64_t* offs,
                      int64_t min_len, double max_evalue, int64_t max_nseed, double min_score_rate,
                      int max_report, char* out, int64_t cap) {
    RefDB* db = (RefDB*)h;
    std::string text;
    for (int64_t i = 0; i < n_reads; ++i) {
        const int64_t L = offs[i + 1] - offs[i];
        const std::string name = "r" + std::to_string(i);
        const PrimarySeq r = make_read(reads + offs[i], L, quals ? quals + offs[i] : nullptr, name.c_str());
        const PrimarySeq rc = r.revcom();
        SeedList seeds = SMEM_LIST::findSeeds(&r, &db->mtg, &db->fmd, min_len, max_evalue, max_nseed);
        ALIGN_LIST alns;
        if (!seeds.empty()) {
            ChainList chains = SeedChain::getChains(seeds, std::ceil(L * Alignment::MAX_MISMATCH_RATE),
                                                    std::ceil(L * Alignment::MAX_INDEL_RATE));
            alns = Alignment::buildAlignments(&r, &rc, db->mtg, chains, Alignment::GLOBAL);
        }
        sam_read(alns, r, min_score_rate, (uint32_t)max_report, text);
    }
    return put_out(text, out, cap);
}

static_assert(sizeof(msg_aln) == 88, "msg_aln layout");

/* The alignments of records k0..k1 of the CUDA library, through the adapter
 * a maintainer adds to the reference (from_device.h). */
static ALIGN_LIST records_to_alignments(RefDB* db, const PrimarySeq* r, const PrimarySeq* rc, int64_t L,
                                        const void* records, const uint32_t* cigar, int64_t k0, int64_t k1) {
    const msg_aln* rec = (const msg_aln*)records;
    ALIGN_LIST alns;
    (void)L;
    for (int64_t k = k0; k < k1; ++k)
        alns.push_back(msg_adapter::fromDevice(r, rc, db->mtg, rec[k], cigar, Alignment::GLOBAL));
    return alns;
}

/* The same lines with the alignments taken from records of the CUDA library
 * (msg_aln, include/msg_b200.h; 88 bytes each) and their CIGAR words, through
 * records_to_alignments; the reference's tail runs unchanged. */
int64_t ref_sam_from_records(void* h, int64_t n_reads, const uint8_t* reads, const uint8_t* quals,
                             const int64_t* offs, const void* records, const uint32_t* cigar,
                             const int64_t* read_aln_off, double min_score_rate, int max_report, char* out,
                             int64_t cap) {
    RefDB* db = (RefDB*)h;
    std::string text;
    for (int64_t i = 0; i < n_reads; ++i) {
        const int64_t L = offs[i + 1] - offs[i];
        const std::string name = "r" + std::to_string(i);
        const PrimarySeq r = make_read(reads + offs[i], L, quals ? quals + offs[i] : nullptr, name.c_str());
        const PrimarySeq rc = r.revcom();
        ALIGN_LIST alns = records_to_alignments(db, &r, &rc, L, records, cigar, read_aln_off[i], read_aln_off[i + 1]);
        sam_read(alns, r, min_score_rate, (uint32_t)max_report, text);
    }
    return put_out(text, out, cap);
}

/* ref_sam_pe_batch's tail on records of the CUDA library (reads 2i and 2i+1
 * of the batch are the mates of pair i), as ref_sam_from_records does for
 * single reads. */
int64_t ref_sam_pe_from_records(void* h, int64_t n_pairs, const uint8_t* reads, const uint8_t* quals,
                                const int64_t* offs, const void* records, const uint32_t* cigar,
                                const int64_t* read_aln_off, double min_score_rate, int max_report, double mean,
                                double sd, double min_ins, double max_ins, const int* opt, int64_t max_npair,
                                char* out, int64_t cap) {
    RefDB* db = (RefDB*)h;
    set_pairing(mean, sd, min_ins, max_ins);
    std::string text;
    for (int64_t i = 0; i < n_pairs; ++i) {
        const std::string name = "p" + std::to_string(i);
        const PrimarySeq m[2] = {make_read(reads + offs[2 * i], offs[2 * i + 1] - offs[2 * i],
                                     quals ? quals + offs[2 * i] : nullptr, name.c_str()),
                           make_read(reads + offs[2 * i + 1], offs[2 * i + 2] - offs[2 * i + 1],
                                     quals ? quals + offs[2 * i + 1] : nullptr, name.c_str())};
        const PrimarySeq rc[2] = {m[0].revcom(), m[1].revcom()};
        ALIGN_LIST lists[2];
        for (int x = 0; x < 2; ++x)
            lists[x] = records_to_alignments(db, &m[x], &rc[x], (int64_t)m[x].length(), records, cigar,
                                             read_aln_off[2 * i + x], read_aln_off[2 * i + x + 1]);
        sam_pair(lists[0], lists[1], m[0], m[1], min_score_rate, (uint32_t)max_report, opt, max_npair, text);
    }
    return put_out(text, out, cap);
}

/* Write the DB as msgseqtk-build does (src/msgseqtk-build.cpp:382-426):
 * program header + MetaGenome::save, MetaGenome::saveSeq, program header +
 * FMDIndex::save. Returns 0 on success. */
int ref_db_save(void* h, const char* mtg_path, const char* mgs_path, const char* fmd_path) {
    RefDB* db = (RefDB*)h;
    std::ofstream mtgOut(mtg_path, std::ios::binary), mgsOut(mgs_path, std::ios::binary),
        fmdOut(fmd_path, std::ios::binary);
    if (!mtgOut || !mgsOut || !fmdOut) return 1;
    EGriceLab::saveProgInfo(mtgOut);
    db->mtg.save(mtgOut);
    db->mtg.saveSeq(mgsOut);
    EGriceLab::saveProgInfo(fmdOut);
    db->fmd.save(fmdOut);
    return (mtgOut && mgsOut && fmdOut) ? 0 : 2;
}

/* msgseqtk-align's read loop over a FASTQ text (while hasNext: nextSeq,
 * src/SeqIO.cpp:44-51, 74-87): per read a line "name\tdesc\tSEQ\tQUAL" with
 * the nt16 codes as hex digits and the quality values as two hex digits
 * each. Returns the text length; written only when it fits in cap bytes. */
int64_t ref_fastq_parse(const char* text, int64_t len, char* out, int64_t cap) {
    std::istringstream in(std::string(text, text + len));
    SeqIO io(&in, SeqIO::FASTQ);
    std::string s;
    char buf[8];
    while (io.hasNext()) {
        const PrimarySeq r = io.nextSeq();
        s += r.getName() + "\t" + r.getDesc() + "\t";
        for (uint8_t b : r.getSeq()) { std::snprintf(buf, sizeof buf, "%x", (unsigned)b); s += buf; }
        s += "\t";
        for (uint8_t q : r.getQual()) { std::snprintf(buf, sizeof buf, "%02x", (unsigned)q); s += buf; }
        s += "\n";
    }
    return put_out(s, out, cap);
}

/* The reference reading a FASTQ text and writing back the reads whose
 * keep[i] is set (every read when keep is NULL), as msgseqtk-clean does
 * (SeqIO::nextSeq, SeqIO::writeSeq; src/msgseqtk-clean.cpp:420-435). */
int64_t ref_fastq_rewrite(const char* text, int64_t len, const uint8_t* keep, char* out, int64_t cap) {
    std::istringstream in(std::string(text, text + len));
    std::ostringstream os;
    SeqIO io(&in, SeqIO::FASTQ);
    SeqIO wo(&os, SeqIO::FASTQ);
    int64_t i = 0;
    while (io.hasNext()) {
        const PrimarySeq r = io.nextSeq();
        if (!keep || keep[i]) wo.writeSeq(r);
        ++i;
    }
    return put_out(os.str(), out, cap);
}

/* msgseqtk-clean's single-end task with --assign over a FASTQ text
 * (src/msgseqtk-clean.cpp:423-440, restated: it lives in the program file):
 * the assignment line of every read. */
int64_t ref_clean_assign(void* h_ref, void* h_bg, const char* text, int64_t len, int64_t min_len, double max_evalue,
                         char* out, int64_t cap) {
    RefDB* rdb = (RefDB*)h_ref;
    RefDB* bdb = (RefDB*)h_bg;
    std::istringstream in(std::string(text, text + len));
    SeqIO io(&in, SeqIO::FASTQ);
    std::ostringstream assignOut;
    while (io.hasNext()) {
        const PrimarySeq read = io.nextSeq();
        MEM_LIST refMems = SMEM_LIST::findMEMS(&read, &rdb->mtg, &rdb->fmd, min_len, max_evalue);
        MEM_LIST bgMems = SMEM_LIST::findMEMS(&read, &bdb->mtg, &bdb->fmd, min_len, max_evalue);
        const double refLoglik = refMems.loglik();
        const double bgLoglik = bgMems.loglik();
        const double lod = -refLoglik + bgLoglik;
        assignOut << read.getName() << "\t" << read.getDesc() << "\t" << refLoglik << "\t" << bgLoglik << "\t" << lod
                  << std::endl;
    }
    return put_out(assignOut.str(), out, cap);
}

int ref_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
