// BAM output of the tail's records, for callers without htslib: the binary
// header and alignment records of the SAM/BAM format specification (the
// layout htslib's bam_write1 gives the records msgseqtk-align builds,
// src/SAMtools/BAM.cpp:20-56, src/Alignment.cpp:429-444,
// src/msgseqtk-align.cpp:538-593), and BGZF compression (gzip members of at
// most 0xff00 input bytes with the 'BC' extra field giving the member's size,
// then the 28-byte end-of-file member) with members deflated on host threads.
#include <zlib.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/msg_b200.h"

namespace {

template <typename T> void put(std::string& s, T v) {  // little-endian, as BAM stores every field
    char b[sizeof(T)];
    std::memcpy(b, &v, sizeof(T));
    s.append(b, sizeof(T));
}

// Reference length of a CIGAR: M, D, N, = and X consume the target.
int64_t ref_len(const uint32_t* cg, int32_t n) {
    int64_t r = 0;
    for (int32_t w = 0; w < n; ++w) {
        const int op = cg[w] & 0xf;
        if (op == 0 || op == 2 || op == 3 || op == 7 || op == 8) r += cg[w] >> 4;
    }
    return r;
}

// The BAI bin of [beg, end) (SAM specification 5.3; depth 5, 16 kbp
// leaves), computed on end - 1 as htslib's hts_reg2bin(beg, end, 14, 5);
// an empty range (end == beg) gets the bin where beg and end - 1 first
// agree, 0 at beg == 0.
int reg2bin(int64_t beg, int64_t end) {
    --end;
    int s = 14, t = ((1 << 15) - 1) / 7;
    for (int l = 5; l > 0; --l, s += 3, t -= 1 << (l * 3))
        if ((beg >> s) == (end >> s)) return t + (int)(beg >> s);
    return 0;
}

// An integer aux field in the smallest type that holds it (c/C, s/S, i/I).
void put_int_aux(std::string& s, const char* tag, int64_t v) {
    s.append(tag, 2);
    if (v < 0) {
        if (v >= INT8_MIN) { s += 'c'; put<int8_t>(s, (int8_t)v); }
        else if (v >= INT16_MIN) { s += 's'; put<int16_t>(s, (int16_t)v); }
        else { s += 'i'; put<int32_t>(s, (int32_t)v); }
    } else {
        if (v <= UINT8_MAX) { s += 'C'; put<uint8_t>(s, (uint8_t)v); }
        else if (v <= UINT16_MAX) { s += 'S'; put<uint16_t>(s, (uint16_t)v); }
        else { s += 'I'; put<uint32_t>(s, (uint32_t)v); }
    }
}

constexpr size_t kBgzfBlock = 0xff00;  // input bytes per BGZF member (htslib's BGZF_BLOCK_SIZE)
// gzip header of a BGZF member: ID1 ID2 CM FLG(FEXTRA) MTIME(4) XFL OS XLEN(6),
// then the extra subfield 'B' 'C' SLEN(2) BSIZE (member size - 1, 2 bytes)
constexpr uint8_t kBgzfHead[16] = {31, 139, 8, 4, 0, 0, 0, 0, 0, 255, 6, 0, 'B', 'C', 2, 0};
// the empty member htslib writes at the end of a BGZF file
constexpr uint8_t kBgzfEof[28] = {31, 139, 8, 4, 0, 0, 0, 0, 0, 255, 6, 0, 66, 67, 2, 0,
                                  27, 0, 3, 0, 0, 0, 0, 0, 0, 0, 0, 0};

// One member: raw deflate of in[0..n) at `level`, CRC32 and input size.
bool bgzf_member(const uint8_t* in, size_t n, int level, std::string& out) {
    z_stream z;
    std::memset(&z, 0, sizeof z);
    if (deflateInit2(&z, level, Z_DEFLATED, -15, 8, Z_DEFAULT_STRATEGY) != Z_OK) return false;
    std::string body(deflateBound(&z, (uLong)n), '\0');
    z.next_in = const_cast<Bytef*>(in);
    z.avail_in = (uInt)n;
    z.next_out = reinterpret_cast<Bytef*>(&body[0]);
    z.avail_out = (uInt)body.size();
    const int rc = deflate(&z, Z_FINISH);
    const size_t clen = body.size() - z.avail_out;
    deflateEnd(&z);
    if (rc != Z_STREAM_END) return false;
    const size_t total = sizeof(kBgzfHead) + 2 + clen + 8;
    if (total > 65536) return false;  // BSIZE holds 16 bits
    out.assign(reinterpret_cast<const char*>(kBgzfHead), sizeof(kBgzfHead));
    put<uint16_t>(out, (uint16_t)(total - 1));
    out.append(body.data(), clen);
    put<uint32_t>(out, (uint32_t)crc32(crc32(0L, Z_NULL, 0), in, (uInt)n));
    put<uint32_t>(out, (uint32_t)n);
    return true;
}

}  // namespace

extern "C" int msg_bam_header(const char* text, int64_t text_len, const char* const* chrom_names,
                              const int64_t* chrom_len, int64_t n_chrom, uint8_t* out, int64_t cap, int64_t* len) {
    if (!len || text_len < 0 || (text_len > 0 && !text) || n_chrom < 0 || (n_chrom > 0 && (!chrom_names || !chrom_len)) ||
        cap < 0 || text_len > INT32_MAX || n_chrom > INT32_MAX)
        return MSG_EINVAL;
    std::string s("BAM\1", 4);
    put<int32_t>(s, (int32_t)text_len);
    s.append(text ? text : "", (size_t)text_len);
    put<int32_t>(s, (int32_t)n_chrom);
    for (int64_t t = 0; t < n_chrom; ++t) {
        if (!chrom_names[t] || chrom_len[t] < 0 || chrom_len[t] > INT32_MAX) return MSG_EINVAL;
        const size_t l = std::strlen(chrom_names[t]);
        put<int32_t>(s, (int32_t)(l + 1));
        s.append(chrom_names[t], l + 1);
        put<int32_t>(s, (int32_t)chrom_len[t]);
    }
    *len = (int64_t)s.size();
    if (*len > cap || !out) return MSG_EINVAL;
    std::memcpy(out, s.data(), s.size());
    return MSG_OK;
}

extern "C" int msg_bam_format(const msg_sam_rec* recs, int64_t n_recs, const char* md, const msg_read_batch* reads,
                              const uint8_t* quals, const uint32_t* cigar, const char* names, const int64_t* name_off,
                              int64_t n_chrom, uint8_t* out, int64_t cap, int64_t* len) {
    if ((n_recs > 0 && (!recs || !reads || !reads->seq || !reads->off || !names || !name_off)) || !len ||
        n_recs < 0 || cap < 0 || n_chrom < 0)
        return MSG_EINVAL;
    static const uint8_t kComp[16] = {0, 8, 4, 12, 2, 10, 6, 14, 1, 9, 5, 13, 3, 11, 7, 15};
    std::string s;
    std::string rec;
    for (int64_t k = 0; k < n_recs; ++k) {
        const msg_sam_rec& r = recs[k];
        if (r.read < 0 || r.read >= reads->n_reads || r.tid >= n_chrom || r.tid < -1 || r.n_cigar < 0 ||
            r.n_cigar > 0xffff || (r.n_cigar > 0 && !cigar) || r.pos < -1 || r.pos > INT32_MAX || r.md_len < 0 ||
            (r.md_len > 0 && !md))
            return MSG_EINVAL;
        const int64_t a = reads->off[r.read], L = reads->off[r.read + 1] - a;
        if (L < 0 || L > INT32_MAX) return MSG_EINVAL;
        // QNAME: the read's name, its text line's first field
        const char* nm = names + name_off[r.read];
        const int64_t nl = name_off[r.read + 1] - name_off[r.read];
        if (nl < 0) return MSG_EINVAL;
        const char* ne = static_cast<const char*>(std::memchr(nm, '\t', nl));
        if (!ne) ne = static_cast<const char*>(std::memchr(nm, '\n', nl));
        const int64_t qn = ne ? ne - nm : nl;
        if (qn + 1 > 255) return MSG_EINVAL;  // l_read_name is one byte
        const uint32_t* cg = r.n_cigar > 0 ? cigar + r.cigar_off : nullptr;
        // the record's bin, as the reference's BAM constructor sets it: the
        // range [pos, pos + reference length of the CIGAR)
        const int64_t rl = cg ? ref_len(cg, r.n_cigar) : 0;
        rec.clear();
        put<int32_t>(rec, r.tid);
        put<int32_t>(rec, (int32_t)r.pos);
        put<uint8_t>(rec, (uint8_t)(qn + 1));
        put<uint8_t>(rec, (uint8_t)r.mapq);
        put<uint16_t>(rec, (uint16_t)reg2bin(r.pos, r.pos + rl));
        put<uint16_t>(rec, (uint16_t)r.n_cigar);
        put<uint16_t>(rec, (uint16_t)r.flag);
        put<int32_t>(rec, (int32_t)L);
        put<int32_t>(rec, -1);  // next refID and pos: msgseqtk-align leaves them at -1 and 0 (BAM.h:61-75)
        put<int32_t>(rec, 0);
        put<int32_t>(rec, r.isize);
        rec.append(nm, (size_t)qn);
        rec += '\0';
        for (int32_t w = 0; w < r.n_cigar; ++w) put<uint32_t>(rec, cg[w]);
        // SEQ: nt16 codes, two per byte, the first in the high nibble; the
        // reverse complement and reversed qualities for records on the
        // reverse strand (the reference exports the reverse-complemented read)
        const bool rev = (r.flag & 0x10) != 0;
        auto base = [&](int64_t i) { return rev ? kComp[reads->seq[a + L - 1 - i] & 15] : reads->seq[a + i] & 15; };
        for (int64_t i = 0; i < L; i += 2)
            rec += (char)((base(i) << 4) | (i + 1 < L ? base(i + 1) : 0));
        for (int64_t i = 0; i < L; ++i)  // phred values; 33 on every base for a read without qualities
            rec += (char)(quals ? quals[rev ? a + L - 1 - i : a + i] : 33);
        if (!(r.flag & 0x4)) {  // AS, MD, XH, NH, XN, XP in the order the reference sets them
            put_int_aux(rec, "AS", r.as);
            rec.append("MDZ", 3);
            if (r.md_len > 0) rec.append(md + r.md_off, (size_t)r.md_len);
            rec += '\0';
            rec.append("XHf", 3);
            put<float>(rec, r.xh);
            put_int_aux(rec, "NH", r.nh);
            put_int_aux(rec, "XN", r.xn);
            rec.append("XPf", 3);
            put<float>(rec, r.xp);
        }
        put<int32_t>(s, (int32_t)rec.size());
        s += rec;
    }
    *len = (int64_t)s.size();
    if (*len > cap || (!s.empty() && !out)) return MSG_EINVAL;
    if (!s.empty()) std::memcpy(out, s.data(), s.size());
    return MSG_OK;
}

extern "C" int msg_bgzf_compress(const uint8_t* data, int64_t n, int level, int n_threads, int add_eof, uint8_t* out,
                                 int64_t cap, int64_t* len) {
    if (!len || n < 0 || (n > 0 && !data) || cap < 0 || level < 0 || level > 9) return MSG_EINVAL;
    const size_t nb = ((size_t)n + kBgzfBlock - 1) / kBgzfBlock;
    std::vector<std::string> part(nb);
    std::atomic<size_t> next{0};
    std::atomic<bool> bad{false};
    auto work = [&]() {
        for (size_t b; (b = next.fetch_add(1)) < nb;) {
            const size_t lo = b * kBgzfBlock, m = std::min(kBgzfBlock, (size_t)n - lo);
            if (!bgzf_member(data + lo, m, level, part[b])) bad = true;
        }
    };
    const int nt = (int)std::max<size_t>(1, std::min<size_t>(nb, (size_t)std::max(1, n_threads)));
    std::vector<std::thread> th;
    for (int t = 1; t < nt; ++t) th.emplace_back(work);
    work();
    for (auto& t : th) t.join();
    if (bad) return MSG_EINVAL;
    int64_t total = add_eof ? (int64_t)sizeof(kBgzfEof) : 0;
    for (const std::string& p : part) total += (int64_t)p.size();
    *len = total;
    if (total > cap || (total > 0 && !out)) return MSG_EINVAL;
    uint8_t* o = out;
    for (const std::string& p : part) {
        std::memcpy(o, p.data(), p.size());
        o += p.size();
    }
    if (add_eof) std::memcpy(o, kBgzfEof, sizeof(kBgzfEof));
    return MSG_OK;
}
