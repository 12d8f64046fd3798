// Reading a database written by msgseqtk-build (src/msgseqtk-build.cpp:382-426)
// into the host views msg_index_load takes: the MetaGenome (.mtg) and its
// sequences (.mgs), and the FMD-index (.fmd) whose BWT is stored as a wavelet
// tree of RRR-compressed bit sequences (libsds).
//
// File formats (all little-endian, as written by the reference on x86-64):
//   program header (.mtg, .fmd; ProgEnv.cpp:24-28): the 8 characters
//     "MSGseqTK", then three int32 version numbers (VersionSequence::save).
//   MetaGenome::save (MetaGenome.cpp:42-49): size_t #genomes; per genome
//     (Genome.cpp:66-74) id and name as size_t length + bytes, size_t
//     #chromosomes; per chromosome (Genome.cpp:23-27) name as length + bytes
//     and int64 length.
//   MetaGenome::saveSeq (.mgs, no header; Genome.cpp:29-32): per chromosome
//     its nt16 codes and one terminating 0.
//   FMDIndex::save (FMDIndex.cpp:142-150): int64 B[256], int64 C[256], the
//     wavelet tree, gapSA (size_t length + int64s), SAidx (an RRR bit
//     sequence marking sampled rows), SAsampled (size_t length + int64s).
//   WaveletTreeRRR::save (WaveletTreeRRR.cpp:14-29): size_t n, sigma,
//     height, wid, min, max, sample_rate, #OCC, OCC[#OCC], then `height`
//     RRR bit sequences, level 0 holding the symbols' top bit.
//   BitSeqRRR::save (BitSeqRRR.cpp:308-333): size_t n, ones; BitStr32 C
//     (4-bit block classes); BitStr32 O (variable-width block offsets);
//     size_t nC, wC, nO, wO; BitStr64 Csampled, Osampled; size_t nCsampled,
//     wCsampled, nOsampled, wOsampled, sample_rate.
//   BitStr::save (BitStr.h:386-392): the word width (a 32-bit field written
//     as 8 bytes, the upper 4 undefined), bit length and word count as size_t,
//     then the words; bits are numbered from the least significant bit of
//     word 0.
//
// An RRR block of 15 bits is stored as its class k (popcount) and its offset
// among the k-subsets of {0..14} listed in lexicographic order of their
// positions (the table BitSeqRRR::TableOffset builds); the offset takes
// bits(C(15, k) - 1) bits. Decoding unranks it (one thread per bit
// sequence). The wavelet tree gives the positions WaveletTreeRRR::access
// (WaveletTreeRRR.cpp:58-76) walks to; rows decoded in order reach them with
// one cursor per tree node, on several host threads.
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <thread>
#include <vector>

#include "../../include/msg_b200.h"

struct msg_db {
    // FMD-index view data
    std::vector<uint8_t> bwt;
    int64_t base_count[16] = {0};
    std::vector<int64_t> sample_rows, sample_vals;
    // MetaGenome view data
    std::vector<int64_t> bd_start, bd_end, chr_len, chr_off;
    std::vector<uint8_t> chr_seq;
    std::vector<std::string> chr_names;
};

namespace {

struct Reader {
    std::ifstream in;
    bool ok = true;
    explicit Reader(const char* path) : in(path, std::ios::binary) { ok = (bool)in; }
    template <typename T> T get() {
        T v{};
        if (ok) { in.read(reinterpret_cast<char*>(&v), sizeof(T)); ok = (bool)in; }
        return v;
    }
    void bytes(void* p, size_t n) {
        if (ok && n) { in.read(reinterpret_cast<char*>(p), (std::streamsize)n); ok = (bool)in; }
    }
    std::string str() {  // size_t length + bytes
        const uint64_t n = get<uint64_t>();
        if (!ok || n > (1u << 20)) { ok = false; return std::string(); }
        std::string s(n, '\0');
        bytes(&s[0], n);
        return s;
    }
    bool header() {  // saveProgInfo
        char name[8];
        bytes(name, 8);
        get<int32_t>(); get<int32_t>(); get<int32_t>();
        return ok && std::memcmp(name, "MSGseqTK", 8) == 0;
    }
};

// A libsds BitStr: words of `wid` bits, bits numbered from bit 0 of word 0.
struct Bits {
    uint64_t wid = 0, nbits = 0;
    std::vector<uint64_t> w;  // words widened to 64 bits when wid == 32
    bool read(Reader& r, uint64_t want_wid) {
        // BitStr::save writes its 32-bit word width with sizeof(size_t) bytes:
        // only the low 4 are the value
        wid = r.get<uint64_t>() & 0xffffffffull;
        nbits = r.get<uint64_t>();
        const uint64_t n = r.get<uint64_t>();
        if (!r.ok || wid != want_wid || n > (nbits / wid) + 2 || n * wid < nbits) return false;
        if (wid == 64) {
            w.resize(n);
            r.bytes(w.data(), n * 8);
        } else {
            std::vector<uint32_t> t(n);
            r.bytes(t.data(), n * 4);
            w.resize((n + 1) / 2, 0);
            for (uint64_t k = 0; k < n; ++k) w[k / 2] |= (uint64_t)t[k] << (32 * (k % 2));
        }
        return r.ok;
    }
    // bits [start, start + len), len <= 57
    uint64_t get(uint64_t start, int len) const {
        if (len == 0) return 0;
        const uint64_t i = start >> 6;
        const int j = (int)(start & 63);
        uint64_t v = w[i] >> j;
        if (j + len > 64 && i + 1 < w.size()) v |= w[i + 1] << (64 - j);
        return len >= 64 ? v : (v & ((1ull << len) - 1));
    }
};

int nbits_of(uint64_t x) { int b = 0; for (; x; x >>= 1) ++b; return b; }

struct Rrr {
    uint32_t binom[16][16];
    int offbits[16];
    Rrr() {
        for (int i = 0; i < 16; ++i)
            for (int j = 0; j < 16; ++j) binom[i][j] = (j == 0 || j == i) ? 1 : (j > i ? 0 : 0);
        for (int i = 1; i < 16; ++i)
            for (int j = 1; j < i; ++j) binom[i][j] = binom[i - 1][j - 1] + binom[i - 1][j];
        for (int k = 0; k < 16; ++k) offbits[k] = nbits_of(binom[15][k] - 1);
    }
    // the offset-th k-subset of {0..14} in lexicographic order, as a bitmap
    uint32_t unrank(int k, uint64_t off) const {
        if (k == 0) return 0;
        if (k == 15) return 0x7fff;
        uint32_t v = 0;
        int r = k;
        for (int i = 0; i < 15 && r > 0; ++i) {
            const uint32_t cnt = binom[14 - i][r - 1];  // subsets whose next element is i
            if (off < cnt) { v |= 1u << i; --r; }
            else off -= cnt;
        }
        return v;
    }
};

// A decoded RRR bit sequence: plain bits and a rank directory (ones before
// each 64-bit word).
struct Plain {
    uint64_t n = 0, ones = 0;
    std::vector<uint64_t> w;
    std::vector<uint64_t> dir;
    bool bit(uint64_t i) const { return (w[i >> 6] >> (i & 63)) & 1; }
    uint64_t rank1(uint64_t i) const {  // ones in [0, i]
        const uint64_t k = i >> 6;
        const int r = (int)(i & 63);
        const uint64_t m = r == 63 ? ~0ull : ((2ull << r) - 1);
        return dir[k] + (uint64_t)__builtin_popcountll(w[k] & m);
    }
};

// The stored parts of a BitSeqRRR (BitSeqRRR.cpp:308-360): block classes C
// and offsets O; decoded by decode_rrr.
struct RawRrr {
    uint64_t n = 0, ones = 0, nC = 0;
    Bits C, O;
};

bool parse_rrr(Reader& r, RawRrr& raw) {
    raw.n = r.get<uint64_t>();
    raw.ones = r.get<uint64_t>();
    Bits Cs, Os;
    if (!raw.C.read(r, 32) || !raw.O.read(r, 32)) return false;
    const uint64_t nC = r.get<uint64_t>(), wC = r.get<uint64_t>(), nO = r.get<uint64_t>(), wO = r.get<uint64_t>();
    if (!Cs.read(r, 64) || !Os.read(r, 64)) return false;
    for (int k = 0; k < 5; ++k) r.get<uint64_t>();  // nCsampled, wCsampled, nOsampled, wOsampled, sample_rate
    if (!r.ok || wC != 4 || wO != 1 || nC != (raw.n + 14) / 15 || raw.O.nbits < nO) return false;
    raw.nC = nC;
    return true;
}

bool decode_rrr(const RawRrr& raw, const Rrr& tab, Plain& out) {
    out.n = raw.n;
    out.ones = raw.ones;
    const Bits& C = raw.C;
    const Bits& O = raw.O;
    const uint64_t nC = raw.nC;
    out.w.assign((out.n + 63) / 64 + 1, 0);
    uint64_t pos = 0, ones = 0;
    for (uint64_t b = 0; b < nC; ++b) {
        const int k = (int)C.get(b * 4, 4);
        if (k > 15) return false;
        const int len = tab.offbits[k];
        if (pos + len > O.nbits) return false;
        const uint32_t v = tab.unrank(k, O.get(pos, len));
        pos += len;
        ones += (uint64_t)k;
        const uint64_t s = b * 15;  // block b holds bits s .. s+14
        const uint64_t i = s >> 6;
        const int j = (int)(s & 63);
        out.w[i] |= (uint64_t)v << j;
        if (j > 49 && i + 1 < out.w.size()) out.w[i + 1] |= (uint64_t)v >> (64 - j);
    }
    if (ones != out.ones) return false;
    if (out.n % 64) out.w[out.n / 64] &= (1ull << (out.n % 64)) - 1;  // bits past n are not part of the sequence
    out.dir.resize(out.w.size() + 1);
    uint64_t acc = 0;
    for (size_t k = 0; k < out.w.size(); ++k) { out.dir[k] = acc; acc += (uint64_t)__builtin_popcountll(out.w[k]); }
    out.dir[out.w.size()] = acc;
    return acc == out.ones;
}

bool read_i64s(Reader& r, std::vector<int64_t>& v) {
    const uint64_t n = r.get<uint64_t>();
    if (!r.ok || n > (1ull << 36)) return false;
    v.resize(n);
    r.bytes(v.data(), n * 8);
    return r.ok;
}

bool read_fmd(const char* path, int n_threads, msg_db& db) {
    Reader r(path);
    if (!r.ok || !r.header()) return false;
    int64_t B[256], C[256];
    r.bytes(B, sizeof(B));
    r.bytes(C, sizeof(C));
    // wavelet tree
    const uint64_t n = r.get<uint64_t>();
    r.get<uint64_t>();  // sigma
    const uint64_t height = r.get<uint64_t>();
    r.get<uint64_t>();  // wid
    r.get<uint64_t>();  // min
    r.get<uint64_t>();  // max
    r.get<uint64_t>();  // sample_rate
    const uint64_t nocc = r.get<uint64_t>();
    if (!r.ok || height == 0 || height > 8 || nocc > 1024) return false;
    std::vector<uint64_t> occ(nocc);
    r.bytes(occ.data(), nocc * 8);
    const Rrr tab;
    // the bit sequences are read in file order, then unranked in parallel
    std::vector<RawRrr> raw(height + 1);
    for (uint64_t l = 0; l < height; ++l)
        if (!parse_rrr(r, raw[l]) || raw[l].n != n) return false;
    std::vector<int64_t> gap_sa, sa_sampled;
    if (!read_i64s(r, gap_sa) || !parse_rrr(r, raw[height]) || !read_i64s(r, sa_sampled)) return false;
    std::vector<Plain> lv(height);
    Plain saidx;
    {
        // height + 1 jobs on at most n_threads workers
        std::vector<char> ok(height + 1, 0);
        std::atomic<uint64_t> next{0};
        auto worker = [&]() {
            for (uint64_t l; (l = next.fetch_add(1)) <= height;)
                ok[l] = decode_rrr(raw[l], tab, l < height ? lv[l] : saidx);
        };
        const uint64_t nw = std::min<uint64_t>(height + 1, (uint64_t)std::max(1, n_threads));
        std::vector<std::thread> th;
        for (uint64_t t = 1; t < nw; ++t) th.emplace_back(worker);
        worker();
        for (auto& x : th) x.join();
        for (char x : ok) if (!x) return false;
        raw.clear();
    }
    if (saidx.n != n || (saidx.ones != sa_sampled.size() && saidx.ones != sa_sampled.size() + 1)) return false;
    for (int b = 0; b < 16; ++b) db.base_count[b] = B[b];
    // BWT symbols: the walk of WaveletTreeRRR::access per row
    db.bwt.resize(n);
    std::atomic<bool> bad{false};  // set by any decode thread (relaxed: only read after join)
    // Rows are decoded in order, so the position a row reaches in a node of
    // level l + 1 is that node's start plus the rows before it that took
    // the same path: one cursor per node replaces the per-row rank queries
    // of the access walk (the 0-child of a node starts where the node does,
    // the 1-child at occ[symbol prefix]). A thread starting at row lo sets
    // its cursors with rank queries at the boundary, node by node.
    const uint64_t nodes = 1ull << height;
    std::vector<uint64_t> node_start(height * nodes, 0);  // [l * nodes + prefix]
    for (uint64_t l = 0; l + 1 < height; ++l) {
        for (uint64_t q = 0; q < (1ull << l); ++q) {
            // prefixes above the alphabet's largest symbol hold no rows: they
            // start at n, where any row would be caught as corrupt
            const uint64_t s1 = ((2 * q + 1) << (height - l - 1));
            node_start[(l + 1) * nodes + 2 * q] = node_start[l * nodes + q];
            node_start[(l + 1) * nodes + 2 * q + 1] = s1 < occ.size() ? occ[s1] : n;
        }
    }
    const int nt = std::max(1, n_threads);
    std::vector<std::vector<uint64_t>> hist(nt, std::vector<uint64_t>(nodes, 0));  // decoded symbols per thread
    auto decode = [&](int t, uint64_t lo, uint64_t hi) {
        uint64_t* hs = hist[t].data();
        std::vector<uint64_t> cur(height * nodes, 0);  // next position of each node
        std::vector<uint64_t> cnt(height * nodes, 0);  // rows before lo in each node
        cnt[0] = lo;
        for (uint64_t l = 0; l + 1 < height; ++l) {
            const Plain& p = lv[l];
            for (uint64_t q = 0; q < (1ull << l); ++q) {
                const uint64_t st = node_start[l * nodes + q], c = cnt[l * nodes + q];
                if (st + c > n) { bad.store(true, std::memory_order_relaxed); return; }
                const uint64_t ones = c > 0 ? p.rank1(st + c - 1) - (st > 0 ? p.rank1(st - 1) : 0) : 0;
                cnt[(l + 1) * nodes + 2 * q + 1] = ones;
                cnt[(l + 1) * nodes + 2 * q] = c - ones;
            }
        }
        for (uint64_t k = 0; k < height * nodes; ++k) cur[k] = node_start[k] + cnt[k];
        for (uint64_t row = lo; row < hi; ++row) {
            uint64_t q = 0, i = row;
            for (uint64_t l = 0; l < height; ++l) {
                if (i >= n) { bad.store(true, std::memory_order_relaxed); return; }
                q = 2 * q + (lv[l].bit(i) ? 1 : 0);
                if (l + 1 < height) i = cur[(l + 1) * nodes + q]++;
            }
            // a symbol without an entry in the occurrence table (at most
            // max symbol + 2 entries, WaveletTreeRRR.h:238) is not one the
            // index holds
            if (q + 1 >= occ.size()) { bad.store(true, std::memory_order_relaxed); return; }
            db.bwt[row] = (uint8_t)q;
            hs[q]++;
        }
    };
    std::vector<std::thread> th;
    const uint64_t chunk = (n + nt - 1) / nt;
    for (int t = 0; t < nt; ++t) {
        const uint64_t lo = std::min<uint64_t>(n, t * chunk), hi = std::min<uint64_t>(n, lo + chunk);
        th.emplace_back(decode, t, lo, hi);
    }
    for (auto& x : th) x.join();
    if (bad.load()) return false;
    // the decoded symbols must be the ones the occurrence table counts
    for (uint64_t q = 0; q + 1 < occ.size() && q < nodes; ++q) {
        uint64_t c = 0;
        for (int t = 0; t < nt; ++t) c += hist[t][q];
        if (c != occ[q + 1] - occ[q]) return false;
    }
    // FMDIndex::buildSA sizes SAsampled by SAidx.numOnes() (FMDIndex.cpp:495),
    // which can be one short of the marked rows; the last sample's value then
    // lies past the saved array (an index built in memory still holds it; one
    // loaded from its file reads the string's terminator). Recompute it here
    // as accessSA would have had it: walk LF from that row to the next
    // sampled row with a stored value, SA = that value + the distance.
    if (saidx.ones == sa_sampled.size() + 1) {
        auto rank = [&](uint64_t sym, uint64_t i) -> uint64_t {  // WaveletTreeRRR::rank (occurrences in [0, i])
            uint64_t start = 0, r = ~0ull;
            for (uint64_t l = 0; r != 0 && l < height; ++l) {
                const Plain& p = lv[l];
                const uint64_t before = start > 0 ? p.rank1(start - 1) : 0;
                if ((sym >> (height - l - 1)) & 1) {
                    const uint64_t masked = (sym >> (height - l - 1)) << (height - l - 1);
                    r = p.rank1(i) - before;
                    if (masked >= occ.size()) return 0;
                    start = occ[masked];
                } else {
                    r = i - start + before - p.rank1(i) + 1;
                }
                if (r == 0) return 0;
                i = r + start - 1;
            }
            return r;
        };
        uint64_t j = 0;  // the last marked row
        for (size_t k = saidx.w.size(); k-- > 0;)
            if (saidx.w[k]) { j = k * 64 + 63 - (uint64_t)__builtin_clzll(saidx.w[k]); break; }
        uint64_t i = j;
        int64_t dist = 0;
        for (;;) {
            const uint64_t b = db.bwt[i];
            if (b == 0 || dist > (int64_t)n) return false;  // a '$' row is always sampled and stored
            const uint64_t rk = rank(b, i);
            if (b >= 16 || rk == 0 || (uint64_t)C[b] + rk - 1 >= n) return false;  // inconsistent counts
            i = (uint64_t)C[b] + rk - 1;                    // LF(b, i) - 1 (FMDIndex.h:130-141)
            ++dist;
            if (saidx.bit(i) && saidx.rank1(i) - 1 < sa_sampled.size()) break;
        }
        sa_sampled.push_back(sa_sampled[saidx.rank1(i) - 1] + dist);
    }
    // sampled rows: the set bits of SAidx, in order
    db.sample_rows.clear();
    db.sample_rows.reserve(saidx.ones);
    for (size_t k = 0; k < saidx.w.size(); ++k) {
        uint64_t x = saidx.w[k];
        while (x) {
            const int b = __builtin_ctzll(x);
            db.sample_rows.push_back((int64_t)(k * 64 + b));
            x &= x - 1;
        }
    }
    db.sample_vals = std::move(sa_sampled);
    return db.sample_rows.size() == db.sample_vals.size();
}

bool read_mtg(const char* mtg_path, const char* mgs_path, msg_db& db) {
    Reader r(mtg_path);
    if (!r.ok || !r.header()) return false;
    const uint64_t ng = r.get<uint64_t>();
    if (!r.ok || ng > (1u << 28)) return false;
    int64_t bd = 0;
    for (uint64_t g = 0; g < ng; ++g) {
        r.str();  // genome id
        r.str();  // genome name
        const uint64_t nc = r.get<uint64_t>();
        if (!r.ok || nc > (1u << 28)) return false;
        for (uint64_t c = 0; c < nc; ++c) {
            db.chr_names.push_back(r.str());
            const int64_t len = r.get<int64_t>();
            if (!r.ok || len < 0) return false;
            db.chr_len.push_back(len);
            db.bd_start.push_back(bd);  // MetaGenome::updateIndex (MetaGenome.cpp:195-213)
            bd += (len + 1) * 2;
            db.bd_end.push_back(bd);
        }
    }
    Reader s(mgs_path);
    if (!s.ok) return false;
    int64_t total = 0;
    for (int64_t len : db.chr_len) total += len;
    db.chr_seq.resize(total);
    db.chr_off.assign(1, 0);
    int64_t at = 0;
    for (int64_t len : db.chr_len) {
        s.bytes(db.chr_seq.data() + at, len);
        const uint8_t term = s.get<uint8_t>();
        if (!s.ok || term != 0) return false;
        at += len;
        db.chr_off.push_back(at);
    }
    return true;
}

}  // namespace

extern "C" int msg_db_read(const char* mtg_path, const char* mgs_path, const char* fmd_path, int n_threads,
                           msg_db** db) {
    if (!mtg_path || !mgs_path || !fmd_path || !db) return MSG_EINVAL;
    *db = nullptr;
    msg_db* d = new (std::nothrow) msg_db();
    if (!d) return MSG_ENOMEM;
    try {
        if (!read_mtg(mtg_path, mgs_path, *d) || !read_fmd(fmd_path, n_threads, *d)) { delete d; return MSG_EINVAL; }
    } catch (const std::bad_alloc&) {
        delete d;
        return MSG_ENOMEM;
    }
    const int64_t n = (int64_t)d->bwt.size();
    if (d->bd_end.empty() || d->bd_end.back() != n) { delete d; return MSG_EINVAL; }
    *db = d;
    return MSG_OK;
}

extern "C" void msg_db_free(msg_db* db) { delete db; }

extern "C" int msg_db_views(const msg_db* db, msg_fmd_view* fmd, msg_mtg_view* mtg) {
    if (!db || !fmd || !mtg) return MSG_EINVAL;
    fmd->n = (int64_t)db->bwt.size();
    fmd->bwt = db->bwt.data();
    fmd->base_count = db->base_count;
    fmd->n_samples = (int64_t)db->sample_rows.size();
    fmd->sample_rows = db->sample_rows.data();
    fmd->sample_vals = db->sample_vals.data();
    mtg->n_chrom = (int64_t)db->chr_len.size();
    mtg->bd_start = db->bd_start.data();
    mtg->bd_end = db->bd_end.data();
    mtg->chr_len = db->chr_len.data();
    mtg->chr_seq = db->chr_seq.data();
    mtg->chr_off = db->chr_off.data();
    return MSG_OK;
}

// ---- Decoded image of a database (msg_db_read_cached) ----
//
// The wavelet-tree decode above costs seconds per G symbols; the image holds
// its result -- the arrays msg_db_views hands out and the chromosome names --
// so that a later run reads them back in one pass. The image is keyed by the
// three source files' sizes and 64-bit content hashes, and carries a hash of
// its own body; an image whose key or body does not match is ignored and
// written anew.
//
// Layout (little-endian): "MSGB200I", uint32 version, uint32 0; key: three
// (uint64 size, uint64 hash) for .mtg, .mgs, .fmd; int64 n, base_count[16],
// n_samples, n_chrom, total chromosome bases, name bytes; then bwt[n],
// sample_rows, sample_vals, bd_start, bd_end, chr_len, chr_off[n_chrom + 1],
// chr_seq, the names (each a uint64 length + bytes); last, the body hash.
namespace {

constexpr char kImageMagic[8] = {'M', 'S', 'G', 'B', '2', '0', '0', 'I'};
constexpr uint32_t kImageVersion = 1;

uint64_t fold64(uint64_t x) {  // splitmix64's finaliser
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

// Hash of a byte range: four lanes over consecutive 8-byte words (xor, odd
// multiply, xor-shift: a bijection of the lane per word), folded with the
// tail bytes and the length. It tells files apart; it is not meant to
// resist a deliberate collision.
uint64_t hash_range(const uint8_t* p, size_t n, uint64_t seed) {
    uint64_t l[4] = {seed ^ 0x243f6a8885a308d3ull, seed ^ 0x13198a2e03707344ull, seed ^ 0xa4093822299f31d0ull,
                     seed ^ 0x082efa98ec4e6c89ull};
    size_t i = 0;
    for (; i + 32 <= n; i += 32) {
        uint64_t w[4];
        std::memcpy(w, p + i, 32);
        for (int j = 0; j < 4; ++j) {
            l[j] = (l[j] ^ w[j]) * 0x9e3779b97f4a7c15ull;
            l[j] ^= l[j] >> 32;
        }
    }
    uint64_t h = fold64(seed ^ (uint64_t)n);
    for (; i < n; ++i) h = fold64(h ^ p[i]);
    for (int j = 0; j < 4; ++j) h = fold64(h ^ l[j]);
    return h;
}

constexpr size_t kHashChunk = 16u << 20;

// hash_range over chunks of kHashChunk bytes on up to nt threads, the chunk
// hashes folded in order (the result does not depend on nt)
uint64_t hash_par(const uint8_t* p, size_t n, int nt) {
    const size_t nc = (n + kHashChunk - 1) / kHashChunk;
    std::vector<uint64_t> ch(nc);
    std::atomic<size_t> next{0};
    auto work = [&]() {
        for (size_t k; (k = next.fetch_add(1)) < nc;)
            ch[k] = hash_range(p + k * kHashChunk, std::min(kHashChunk, n - k * kHashChunk), k);
    };
    const int w = (int)std::min<size_t>(nc, (size_t)std::max(1, nt));
    std::vector<std::thread> th;
    for (int t = 1; t < w; ++t) th.emplace_back(work);
    work();
    for (auto& x : th) x.join();
    uint64_t h = fold64(n);
    for (uint64_t x : ch) h = fold64(h ^ x);
    return h;
}

// Size and hash of a file's contents, read in chunks of kHashChunk bytes by
// up to nt threads (each with its own stream); same value as hash_par over
// the whole file.
bool hash_file(const char* path, int nt, uint64_t* size, uint64_t* hash) {
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f) return false;
    const std::streamoff end = f.tellg();
    if (end < 0) return false;
    const size_t n = (size_t)end;
    const size_t nc = (n + kHashChunk - 1) / kHashChunk;
    std::vector<uint64_t> ch(nc);
    std::atomic<size_t> next{0};
    std::atomic<bool> bad{false};
    auto work = [&]() {
        std::ifstream in(path, std::ios::binary);
        std::vector<uint8_t> buf(std::min(kHashChunk, n));
        if (!in) { bad = true; return; }
        for (size_t k; (k = next.fetch_add(1)) < nc;) {
            const size_t len = std::min(kHashChunk, n - k * kHashChunk);
            in.seekg((std::streamoff)(k * kHashChunk));
            in.read(reinterpret_cast<char*>(buf.data()), (std::streamsize)len);
            if (!in) { bad = true; return; }
            ch[k] = hash_range(buf.data(), len, k);
        }
    };
    const int w = (int)std::min<size_t>(nc, (size_t)std::max(1, nt));
    std::vector<std::thread> th;
    for (int t = 1; t < w; ++t) th.emplace_back(work);
    work();
    for (auto& x : th) x.join();
    if (bad) return false;
    uint64_t h = fold64(n);
    for (uint64_t x : ch) h = fold64(h ^ x);
    *size = n;
    *hash = h;
    return true;
}

struct ImageKey {
    uint64_t v[6] = {};
    bool operator==(const ImageKey& o) const { return std::memcmp(v, o.v, sizeof(v)) == 0; }
};

template <typename T> uint64_t vec_hash(const std::vector<T>& x, int nt) {
    return hash_par(reinterpret_cast<const uint8_t*>(x.data()), x.size() * sizeof(T), nt);
}

uint64_t body_hash(const msg_db& d, int nt) {
    uint64_t h = fold64(0x6d7367ull);
    for (uint64_t x : {vec_hash(d.bwt, nt), vec_hash(d.sample_rows, nt), vec_hash(d.sample_vals, nt),
                       vec_hash(d.bd_start, nt), vec_hash(d.bd_end, nt), vec_hash(d.chr_len, nt),
                       vec_hash(d.chr_off, nt), vec_hash(d.chr_seq, nt),
                       hash_range(reinterpret_cast<const uint8_t*>(d.base_count), sizeof(d.base_count), 16)})
        h = fold64(h ^ x);
    for (const std::string& s : d.chr_names)
        h = fold64(h ^ hash_range(reinterpret_cast<const uint8_t*>(s.data()), s.size(), 17));
    return h;
}

template <typename T> bool put(std::ofstream& o, const T* p, size_t n) {
    if (n) o.write(reinterpret_cast<const char*>(p), (std::streamsize)(n * sizeof(T)));
    return (bool)o;
}

bool write_image(const char* path, const ImageKey& key, const msg_db& d, int nt) {
    // written beside the target and renamed over it, so a reader never
    // sees a partial image
    const std::string tmp = std::string(path) + ".tmp." + std::to_string((long)getpid());
    {
        std::ofstream o(tmp, std::ios::binary | std::ios::trunc);
        if (!o) return false;
        int64_t names = 0;
        for (const std::string& s : d.chr_names) names += 8 + (int64_t)s.size();
        const uint32_t ver[2] = {kImageVersion, 0};
        const int64_t head[4] = {(int64_t)d.sample_rows.size(), (int64_t)d.chr_len.size(),
                                 (int64_t)d.chr_seq.size(), names};
        const int64_t n = (int64_t)d.bwt.size();
        bool ok = put(o, kImageMagic, 8) && put(o, ver, 2) && put(o, key.v, 6) && put(o, &n, 1) &&
                  put(o, d.base_count, 16) && put(o, head, 4) && put(o, d.bwt.data(), d.bwt.size()) &&
                  put(o, d.sample_rows.data(), d.sample_rows.size()) &&
                  put(o, d.sample_vals.data(), d.sample_vals.size()) && put(o, d.bd_start.data(), d.bd_start.size()) &&
                  put(o, d.bd_end.data(), d.bd_end.size()) && put(o, d.chr_len.data(), d.chr_len.size()) &&
                  put(o, d.chr_off.data(), d.chr_off.size()) && put(o, d.chr_seq.data(), d.chr_seq.size());
        for (const std::string& s : d.chr_names) {
            const uint64_t len = s.size();
            ok = ok && put(o, &len, 1) && put(o, s.data(), s.size());
        }
        const uint64_t bh = body_hash(d, nt);
        ok = ok && put(o, &bh, 1);
        o.close();
        if (!ok || !o) { std::remove(tmp.c_str()); return false; }
    }
    if (std::rename(tmp.c_str(), path) != 0) { std::remove(tmp.c_str()); return false; }
    return true;
}

// Reads an image whose key equals `key` and whose body hash and tables are
// consistent; false (and `d` left partly filled) for anything else.
bool read_image(const char* path, const ImageKey& key, msg_db& d, int nt) {
    std::ifstream in(path, std::ios::binary | std::ios::ate);
    if (!in) return false;
    const std::streamoff fsize = in.tellg();
    in.seekg(0);
    auto get = [&](void* p, size_t bytes) {
        if (bytes) in.read(reinterpret_cast<char*>(p), (std::streamsize)bytes);
        return (bool)in;
    };
    char magic[8];
    uint32_t ver[2];
    ImageKey k;
    int64_t n = 0, head[4];
    if (!get(magic, 8) || std::memcmp(magic, kImageMagic, 8) != 0 || !get(ver, 8) || ver[0] != kImageVersion ||
        !get(k.v, sizeof(k.v)) || !(k == key) || !get(&n, 8) || !get(d.base_count, sizeof(d.base_count)) ||
        !get(head, sizeof(head)))
        return false;
    const int64_t ns = head[0], nc = head[1], nseq = head[2], names = head[3];
    if (n <= 0 || ns < 0 || nc <= 0 || nseq < 0 || names < 8 * nc) return false;
    // the sizes must account for the file exactly
    const int64_t fixed = 8 + 8 + (int64_t)sizeof(k.v) + 8 + (int64_t)sizeof(d.base_count) + (int64_t)sizeof(head);
    const double body = (double)n + 16.0 * ns + 8.0 * (4 * nc + 1) + (double)nseq + (double)names + 8.0;
    if ((double)fixed + body != (double)fsize) return false;
    d.bwt.resize(n);
    d.sample_rows.resize(ns);
    d.sample_vals.resize(ns);
    d.bd_start.resize(nc);
    d.bd_end.resize(nc);
    d.chr_len.resize(nc);
    d.chr_off.resize(nc + 1);
    d.chr_seq.resize(nseq);
    if (!get(d.bwt.data(), n) || !get(d.sample_rows.data(), 8 * ns) || !get(d.sample_vals.data(), 8 * ns) ||
        !get(d.bd_start.data(), 8 * nc) || !get(d.bd_end.data(), 8 * nc) || !get(d.chr_len.data(), 8 * nc) ||
        !get(d.chr_off.data(), 8 * (nc + 1)) || !get(d.chr_seq.data(), nseq))
        return false;
    d.chr_names.resize(nc);
    int64_t left = names;
    for (int64_t c = 0; c < nc; ++c) {
        uint64_t len = 0;
        if (!get(&len, 8) || (int64_t)len > left - 8) return false;
        d.chr_names[c].resize(len);
        if (!get(&d.chr_names[c][0], len)) return false;
        left -= 8 + (int64_t)len;
    }
    uint64_t bh = 0;
    if (left != 0 || !get(&bh, 8) || bh != body_hash(d, nt)) return false;
    // the tables msg_db_read checks on a decode
    int64_t tot = 0;
    for (int b = 0; b < 16; ++b) {
        if (d.base_count[b] < 0) return false;
        tot += d.base_count[b];
    }
    if (tot != n || d.chr_off[0] != 0 || d.chr_off[nc] != nseq || d.bd_end[nc - 1] != n) return false;
    for (int64_t c = 0; c < nc; ++c)
        if (d.chr_off[c + 1] - d.chr_off[c] != d.chr_len[c] || d.bd_end[c] - d.bd_start[c] != 2 * (d.chr_len[c] + 1))
            return false;
    return true;
}

}  // namespace

extern "C" int msg_db_read_cached(const char* mtg_path, const char* mgs_path, const char* fmd_path,
                                  const char* image_path, int n_threads, msg_db** db, int* from_image) {
    if (!mtg_path || !mgs_path || !fmd_path || !image_path || !db) return MSG_EINVAL;
    *db = nullptr;
    if (from_image) *from_image = 0;
    const int nt = std::max(1, n_threads);
    ImageKey key;
    const char* src[3] = {mtg_path, mgs_path, fmd_path};
    try {
        for (int f = 0; f < 3; ++f)
            if (!hash_file(src[f], nt, &key.v[2 * f], &key.v[2 * f + 1])) return MSG_EINVAL;
        msg_db* d = new (std::nothrow) msg_db();
        if (!d) return MSG_ENOMEM;
        if (read_image(image_path, key, *d, nt)) {
            *db = d;
            if (from_image) *from_image = 1;
            return MSG_OK;
        }
        delete d;
    } catch (const std::bad_alloc&) {
        return MSG_ENOMEM;
    }
    const int rc = msg_db_read(mtg_path, mgs_path, fmd_path, n_threads, db);
    if (rc != MSG_OK) return rc;
    bool written = false;
    try {
        written = write_image(image_path, key, **db, nt);
    } catch (const std::bad_alloc&) {
        written = false;
    }
    if (from_image) *from_image = written ? 0 : -1;
    return MSG_OK;
}
