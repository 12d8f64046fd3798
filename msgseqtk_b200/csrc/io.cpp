// Host I/O around the mapping path: FASTQ records into read batches as
// msgseqtk-align's reader produces them (SeqIO::nextFastqSeq,
// src/SeqIO.cpp:74-87, with PrimarySeq's encoders, src/PrimarySeq.h:40-57,
// src/DNAseq.cpp:15-21, src/QualStr.h:39-42 and src/QualStr.cpp:15-20), and
// SAM text lines of the tail's records in the layout htslib's sam_format1
// writes for the BAM records msgseqtk-align builds.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <sstream>
#include <string>

#include "../../include/msg_b200.h"

namespace {

// DNAalphabet::sym2base (src/DNAalphabet.cpp:14-34): nt16 code of each
// character; every character not listed maps to 0.
struct SymTable {
    uint8_t code[256];
    SymTable() {
        std::memset(code, 0, sizeof code);
        const char* up = "ABCDGHKMNRSTUVWY";
        const uint8_t val[] = {1, 14, 2, 13, 4, 11, 12, 3, 15, 5, 6, 8, 8, 7, 9, 10};
        for (int i = 0; up[i]; ++i) {
            code[(unsigned char)up[i]] = val[i];
            code[(unsigned char)(up[i] - 'A' + 'a')] = val[i];
        }
        const char* dig = "01234";  // '0'-'3' as A, C, G, T and '4' as N
        const uint8_t dv[] = {1, 2, 4, 8, 15};
        for (int i = 0; dig[i]; ++i) code[(unsigned char)dig[i]] = dv[i];
    }
};

const SymTable& sym() {
    static const SymTable t;
    return t;
}

inline bool is_space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r'; }

// One line from p (up to '\n', which is consumed). Returns whether the line
// ended with a newline (false: it ran to the end of the text).
inline bool get_line(const char*& p, const char* end, const char*& a, const char*& b) {
    if (p >= end) { a = b = p; return false; }
    a = p;
    const char* nl = static_cast<const char*>(std::memchr(p, '\n', end - p));
    b = nl ? nl : end;
    p = nl ? nl + 1 : end;
    return nl != nullptr;
}

}  // namespace

extern "C" int msg_fastq_parse(const char* text, int64_t len, int at_eof, msg_fastq_batch* out, int64_t* consumed) {
    if (!out || !consumed || len < 0 || (len > 0 && !text)) return MSG_EINVAL;
    if (out->cap_reads < 0 || out->cap_bases < 0 || out->cap_text < 0) return MSG_EINVAL;
    if (!out->off || !out->name_off || (out->cap_bases > 0 && (!out->seq || !out->qual)) ||
        (out->cap_text > 0 && !out->text))
        return MSG_EINVAL;
    const uint8_t* code = sym().code;
    const char* p = text;
    const char* end = text + len;
    int64_t n = 0, nb = 0, nt = 0;
    out->off[0] = 0;
    out->name_off[0] = 0;
    *consumed = 0;
    // SeqIO::hasNext: the next character is '@'
    while (p < end && *p == '@' && n < out->cap_reads) {
        const char* q = p + 1;
        // `in >> name`: skip whitespace (newlines too), then one word
        while (q < end && is_space(*q)) ++q;
        const char* na = q;
        while (q < end && !is_space(*q)) ++q;
        const char* nz = q;
        while (q < end && is_space(*q) && *q != '\n') ++q;  // blanks before the description
        const char *da, *dz, *sa, *sz, *xa, *xz, *qa, *qz;
        bool whole = get_line(q, end, da, dz);  // description: the rest of the line
        whole = get_line(q, end, sa, sz) && whole;  // sequence
        whole = get_line(q, end, xa, xz) && whole;  // '+' line, ignored
        whole = get_line(q, end, qa, qz) && whole;  // quality
        // a record whose lines do not all end in the text waits for more
        // text, unless this is the end of the stream
        if (!whole && !at_eof) break;
        const int64_t L = sz - sa;
        const int64_t tl = (nz - na) + 1 + (dz - da) + 1;
        if (nb + L > out->cap_bases || nt + tl > out->cap_text) break;
        for (int64_t i = 0; i < L; ++i) out->seq[nb + i] = code[(unsigned char)sa[i]];
        // quality::encode: max(uint8(c - 33), MIN_Q_SCORE = 2); PrimarySeq::fixQual
        // resizes to the sequence length, padding with 33
        const int64_t QL = qz - qa;
        for (int64_t i = 0; i < L; ++i) {
            if (i < QL) {
                const uint8_t v = (uint8_t)((unsigned char)qa[i] - 33);
                out->qual[nb + i] = std::max<uint8_t>(v, 2);
            } else {
                out->qual[nb + i] = 33;
            }
        }
        nb += L;
        // name, a tab, the description, a newline
        std::memcpy(out->text + nt, na, nz - na);
        nt += nz - na;
        out->text[nt++] = '\t';
        std::memcpy(out->text + nt, da, dz - da);
        nt += dz - da;
        out->text[nt++] = '\n';
        ++n;
        out->off[n] = nb;
        out->name_off[n] = nt;
        p = q;
        *consumed = p - text;
    }
    out->n_reads = n;
    out->n_bases = nb;
    out->n_text = nt;
    return MSG_OK;
}

extern "C" int msg_sam_format(const msg_sam_rec* recs, int64_t n_recs, const char* md, const msg_read_batch* reads,
                              const uint8_t* quals, const uint32_t* cigar, const char* names, const int64_t* name_off,
                              const char* const* chrom_names, int64_t n_chrom, char* out, int64_t cap,
                              int64_t* text_len) {
    if ((n_recs > 0 && (!recs || !reads || !reads->seq || !reads->off || !names || !name_off)) || !text_len ||
        n_recs < 0 || cap < 0)
        return MSG_EINVAL;
    static const char kSeq[] = "=ACMGRSVTWYHKDBN";  // htslib's seq_nt16_str
    static const uint8_t kComp[16] = {0, 8, 4, 12, 2, 10, 6, 14, 1, 9, 5, 13, 3, 11, 7, 15};
    std::string s;
    char buf[64];
    for (int64_t k = 0; k < n_recs; ++k) {
        const msg_sam_rec& r = recs[k];
        if (r.read < 0 || r.read >= reads->n_reads) return MSG_EINVAL;
        if (r.tid >= n_chrom || (r.tid >= 0 && !chrom_names)) return MSG_EINVAL;
        const int64_t a = reads->off[r.read], L = reads->off[r.read + 1] - a;
        // QNAME: the read's name (its first word)
        const char* nm = names + name_off[r.read];
        const int64_t nl = name_off[r.read + 1] - name_off[r.read];
        const char* ne = static_cast<const char*>(std::memchr(nm, '\t', nl));
        if (!ne) ne = static_cast<const char*>(std::memchr(nm, '\n', nl));
        s.append(nm, ne ? ne - nm : nl);
        std::snprintf(buf, sizeof buf, "\t%d\t", r.flag);
        s += buf;
        s += r.tid < 0 ? "*" : chrom_names[r.tid];
        // POS and PNEXT are 1-based from BAM's 0-based fields; msgseqtk-align
        // leaves mtid -1 and mpos 0 (BAM.h:61-75): RNEXT '*', PNEXT 1
        std::snprintf(buf, sizeof buf, "\t%lld\t%d\t", (long long)r.pos + 1, r.mapq);
        s += buf;
        if (r.n_cigar == 0) s += "*";
        for (int32_t w = 0; w < r.n_cigar; ++w) {
            const uint32_t c = cigar[r.cigar_off + w];
            std::snprintf(buf, sizeof buf, "%u%c", c >> 4, "MIDNSHP=XB"[c & 0xf]);
            s += buf;
        }
        std::snprintf(buf, sizeof buf, "\t*\t1\t%d\t", r.isize);
        s += buf;
        const bool rev = (r.flag & 0x10) != 0;
        if (L == 0) s += "*";
        for (int64_t i = 0; i < L; ++i) s += kSeq[rev ? kComp[reads->seq[a + L - 1 - i] & 15] : reads->seq[a + i] & 15];
        s += '\t';
        if (L == 0) s += "*";
        else  // a read without qualities has 33 on every base (PrimarySeq::fixQual)
            for (int64_t i = 0; i < L; ++i) s += (char)((quals ? quals[rev ? a + L - 1 - i : a + i] : 33) + 33);
        if (!(r.flag & 0x4)) {
            std::snprintf(buf, sizeof buf, "\tAS:i:%d\tMD:Z:", r.as);
            s += buf;
            if (md) s.append(md + r.md_off, r.md_len);
            std::snprintf(buf, sizeof buf, "\tXH:f:%g\tNH:i:%d\tXN:i:%d\tXP:f:%g", (double)r.xh, r.nh, r.xn,
                          (double)r.xp);
            s += buf;
        }
        s += '\n';
    }
    *text_len = (int64_t)s.size();
    if ((int64_t)s.size() > cap || (!s.empty() && !out)) return MSG_EINVAL;
    if (!s.empty()) std::memcpy(out, s.data(), s.size());
    return MSG_OK;
}

extern "C" int msg_fastq_format(const msg_read_batch* reads, const uint8_t* quals, const char* text,
                                const int64_t* name_off, const uint8_t* keep, char* out, int64_t cap,
                                int64_t* text_len) {
    if (!reads || !text_len || cap < 0) return MSG_EINVAL;
    const int64_t n = reads->n_reads;
    if (n < 0 || (n > 0 && (!reads->seq || !reads->off || !text || !name_off))) return MSG_EINVAL;
    static const char kSym[] = "$ACMGRSVTWYHKDBN";  // DNAalphabet::base2sym (src/DNAalphabet.cpp:36)
    std::string s;
    for (int64_t i = 0; i < n; ++i) {
        if (keep && !keep[i]) continue;
        // SeqIO::writeFastqSeq (src/SeqIO.cpp:107-116): "@name[ desc]", the
        // decoded bases, "+", the qualities + 33, each on its own line
        const char* t = text + name_off[i];
        const int64_t tl = name_off[i + 1] - name_off[i] - 1;  // without the newline
        const char* tab = static_cast<const char*>(std::memchr(t, '\t', tl > 0 ? tl : 0));
        s += '@';
        if (tab) {
            s.append(t, tab - t);
            if (t + tl > tab + 1) {
                s += ' ';
                s.append(tab + 1, t + tl - (tab + 1));
            }
        } else {
            s.append(t, tl > 0 ? tl : 0);
        }
        s += '\n';
        const int64_t a = reads->off[i], L = reads->off[i + 1] - a;
        for (int64_t k = 0; k < L; ++k) s += kSym[reads->seq[a + k] & 15];
        s += "\n+\n";
        for (int64_t k = 0; k < L; ++k) s += (char)((quals ? quals[a + k] : 33) + 33);
        s += '\n';
    }
    *text_len = (int64_t)s.size();
    if ((int64_t)s.size() > cap || (!s.empty() && !out)) return MSG_EINVAL;
    if (!s.empty()) std::memcpy(out, s.data(), s.size());
    return MSG_OK;
}

extern "C" int msg_clean_format(const char* text, const int64_t* name_off, int64_t n, const double* ref_loglik,
                                const double* bg_loglik, const double* lod, char* out, int64_t cap,
                                int64_t* text_len) {
    if (!text_len || n < 0 || cap < 0 || (n > 0 && (!text || !name_off || !ref_loglik || !bg_loglik || !lod)))
        return MSG_EINVAL;
    // msgseqtk-clean's assignment line (src/msgseqtk-clean.cpp:436-437):
    // id, description and the three values through an ostream's defaults
    std::ostringstream os;
    for (int64_t i = 0; i < n; ++i) {
        const char* t = text + name_off[i];
        const int64_t tl = name_off[i + 1] - name_off[i] - 1;
        const char* tab = static_cast<const char*>(std::memchr(t, '\t', tl > 0 ? tl : 0));
        const std::string id = tab ? std::string(t, tab) : std::string(t, tl > 0 ? tl : 0);
        const std::string desc = tab ? std::string(tab + 1, t + tl) : std::string();
        os << id << "\t" << desc << "\t" << ref_loglik[i] << "\t" << bg_loglik[i] << "\t" << lod[i] << "\n";
    }
    const std::string s = os.str();
    *text_len = (int64_t)s.size();
    if ((int64_t)s.size() > cap || (!s.empty() && !out)) return MSG_EINVAL;
    if (!s.empty()) std::memcpy(out, s.data(), s.size());
    return MSG_OK;
}
