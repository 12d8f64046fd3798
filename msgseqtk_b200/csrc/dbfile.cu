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

// The stored parts of an .fmd file, parsed but not decoded.
struct FmdRaw {
    int64_t B[256], C[256];
    uint64_t n = 0, height = 0;
    std::vector<uint64_t> occ;          // the wavelet tree's occurrence table
    std::vector<RawRrr> raw;            // its `height` levels, then SAidx
    std::vector<int64_t> sa_sampled;
};

bool parse_fmd(const char* path, FmdRaw& f) {
    Reader r(path);
    if (!r.ok || !r.header()) return false;
    r.bytes(f.B, sizeof(f.B));
    r.bytes(f.C, sizeof(f.C));
    // wavelet tree
    f.n = r.get<uint64_t>();
    r.get<uint64_t>();  // sigma
    f.height = r.get<uint64_t>();
    r.get<uint64_t>();  // wid
    r.get<uint64_t>();  // min
    r.get<uint64_t>();  // max
    r.get<uint64_t>();  // sample_rate
    const uint64_t nocc = r.get<uint64_t>();
    if (!r.ok || f.height == 0 || f.height > 8 || nocc > 1024) return false;
    f.occ.resize(nocc);
    r.bytes(f.occ.data(), nocc * 8);
    f.raw.resize(f.height + 1);
    for (uint64_t l = 0; l < f.height; ++l)
        if (!parse_rrr(r, f.raw[l]) || f.raw[l].n != f.n) return false;
    std::vector<int64_t> gap_sa;
    return read_i64s(r, gap_sa) && parse_rrr(r, f.raw[f.height]) && read_i64s(r, f.sa_sampled);
}

// The first rows' positions in each wavelet-tree node, [l * 2^height +
// prefix]: the 0-child of a node starts where the node does, the 1-child
// at occ[symbol prefix]; prefixes above the alphabet's largest symbol hold
// no rows and start at n, where any row would be caught as corrupt.
std::vector<uint64_t> node_starts(const FmdRaw& f) {
    const uint64_t height = f.height, nodes = 1ull << height;
    std::vector<uint64_t> node_start(height * nodes, 0);
    for (uint64_t l = 0; l + 1 < height; ++l) {
        for (uint64_t q = 0; q < (1ull << l); ++q) {
            const uint64_t s1 = ((2 * q + 1) << (height - l - 1));
            node_start[(l + 1) * nodes + 2 * q] = node_start[l * nodes + q];
            node_start[(l + 1) * nodes + 2 * q + 1] = s1 < f.occ.size() ? f.occ[s1] : f.n;
        }
    }
    return node_start;
}

bool read_fmd(const char* path, int n_threads, msg_db& db) {
    FmdRaw f;
    if (!parse_fmd(path, f)) return false;
    const int64_t* B = f.B;
    const int64_t* C = f.C;
    const uint64_t n = f.n, height = f.height;
    const std::vector<uint64_t>& occ = f.occ;
    std::vector<RawRrr>& raw = f.raw;
    std::vector<int64_t>& sa_sampled = f.sa_sampled;
    const Rrr tab;
    // the bit sequences were read in file order; they are unranked in parallel
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
    const std::vector<uint64_t> node_start = node_starts(f);  // [l * nodes + prefix]
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

// ---- Decoding the BWT on the GPU (msg_db_read_device) ----
//
// The same decode as read_fmd, with its per-symbol work on the device:
//   1. each RRR bit sequence (the tree's levels and SAidx) is unranked by one
//      thread per superblock of 64 blocks (64 x 15 bits = 15 whole words, so
//      no two threads write one word); the superblock's first offset bit is
//      an exclusive sum of its blocks' offset widths;
//   2. a rank directory per sequence (ones before each word: a scan of the
//      words' popcounts);
//   3. one thread per BWT row walks the tree as WaveletTreeRRR::access does
//      (WaveletTreeRRR.cpp:58-76): the row's position in a child node is the
//      child's first row plus the rows before it in its node that took the
//      same branch -- a rank difference -- which is where the host decode's
//      per-node cursors put it;
//   4. SAidx's set bits become the sampled rows, and the last sample's value
//      (missing from files written by FMDIndex::buildSA, FMDIndex.cpp:495)
//      is recomputed by the same LF walk as on the host.
// Every index a kernel forms from file contents is checked before use; a
// file the host decode rejects is rejected here too (MSG_EINVAL).
#include <cub/cub.cuh>

namespace {

constexpr int kSbBlocks = 64;  // RRR blocks per superblock
constexpr int kSbWords = 15;   // 64-bit words of plain bits per superblock
constexpr uint32_t kDecBad = 1u;
constexpr int kFixupMaxSteps = 1 << 16;  // LF steps of the last-sample walk (about 32 expected)

// C(15, k) and the width of a class-k offset (bits of C(15, k) - 1)
__device__ __host__ inline uint32_t binom15(int k) {
    uint32_t c = 1;
    for (int i = 0; i < k; ++i) c = c * (15 - i) / (i + 1);
    return c;
}
__device__ __host__ inline int offset_bits(int k) {
    uint32_t x = binom15(k) - 1;
    int b = 0;
    for (; x; x >>= 1) ++b;
    return b;
}

// Shared tables of a block: binomial coefficients C(i, j), i, j < 16, and
// the offset widths.
struct RrrShared {
    uint32_t binom[16][16];
    int offbits[16];
};

__device__ void rrr_shared_init(RrrShared& t) {
    for (int e = threadIdx.x; e < 256; e += blockDim.x) {
        const int i = e >> 4, j = e & 15;
        uint32_t c = 0;
        if (j <= i) {
            c = 1;
            for (int k = 0; k < j; ++k) c = c * (i - k) / (k + 1);
        }
        t.binom[i][j] = c;
    }
    if (threadIdx.x < 16) t.offbits[threadIdx.x] = offset_bits(threadIdx.x);
    __syncthreads();
}

__device__ __forceinline__ int rrr_class(const uint64_t* __restrict__ cw, int64_t ncw, int64_t b) {
    const int64_t i = b >> 4;  // 16 four-bit classes per word
    return i < ncw ? (int)((cw[i] >> (4 * (b & 15))) & 15) : 0;
}

__global__ void k_rrr_sb_bits(const uint64_t* __restrict__ cw, int64_t ncw, int64_t nC, int64_t nsb,
                              uint64_t* __restrict__ sb_bits) {
    __shared__ RrrShared t;
    rrr_shared_init(t);
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < nsb; g += (int64_t)gridDim.x * blockDim.x) {
        uint64_t s = 0;
        const int64_t b0 = g * kSbBlocks, b1 = min(nC, b0 + kSbBlocks);
        for (int64_t b = b0; b < b1; ++b) s += (uint64_t)t.offbits[rrr_class(cw, ncw, b)];
        sb_bits[g] = s;
    }
}

// bits [pos, pos + len) of the offset stream, len <= 13
__device__ __forceinline__ uint64_t o_bits(const uint64_t* __restrict__ ow, int64_t now, uint64_t pos, int len) {
    if (len == 0) return 0;
    const uint64_t i = pos >> 6;
    const int j = (int)(pos & 63);
    uint64_t v = (int64_t)i < now ? ow[i] >> j : 0;
    if (j + len > 64 && (int64_t)(i + 1) < now) v |= ow[i + 1] << (64 - j);
    return v & ((1ull << len) - 1);
}

// The offset-th k-subset of {0..14} in lexicographic order, as a bitmap
// (BitSeqRRR's block encoding, as Rrr::unrank on the host).
__device__ __forceinline__ uint32_t rrr_unrank(const RrrShared& t, int k, uint64_t off) {
    if (k == 0) return 0;
    if (k == 15) return 0x7fff;
    uint32_t v = 0;
    int r = k;
    for (int i = 0; i < 15 && r > 0; ++i) {
        const uint32_t cnt = t.binom[14 - i][r - 1];
        if (off < cnt) { v |= 1u << i; --r; }
        else off -= cnt;
    }
    return v;
}

// One thread per superblock: its 64 blocks unranked into its 15 words
// (bits past n cleared), the class sum and the popcount counted.
__global__ void k_rrr_unrank(const uint64_t* __restrict__ cw, int64_t ncw, const uint64_t* __restrict__ ow, int64_t now,
                             uint64_t o_nbits, int64_t nC, int64_t nsb, const uint64_t* __restrict__ sb_pos,
                             uint64_t n_bits, uint64_t* __restrict__ out, unsigned long long* __restrict__ sums,
                             uint32_t* __restrict__ err) {
    __shared__ RrrShared t;
    rrr_shared_init(t);
    unsigned long long cls = 0, pop = 0;
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < nsb; g += (int64_t)gridDim.x * blockDim.x) {
        uint64_t wb[kSbWords];
#pragma unroll
        for (int j = 0; j < kSbWords; ++j) wb[j] = 0;
        uint64_t pos = sb_pos[g];
        const int64_t b0 = g * kSbBlocks, b1 = min(nC, b0 + kSbBlocks);
        for (int64_t b = b0; b < b1; ++b) {
            const int k = rrr_class(cw, ncw, b);
            const int len = t.offbits[k];
            if (pos + len > o_nbits) { atomicOr(err, kDecBad); break; }
            const uint32_t v = rrr_unrank(t, k, o_bits(ow, now, pos, len));
            pos += len;
            cls += (unsigned long long)k;
            const int lb = (int)(b - b0) * 15;
            const int lw = lb >> 6, sh = lb & 63;
            wb[lw] |= (uint64_t)v << sh;
            if (sh > 49) wb[lw + 1] |= (uint64_t)v >> (64 - sh);  // lw + 1 < 15: the last block ends at bit 960
        }
#pragma unroll
        for (int j = 0; j < kSbWords; ++j) {
            const uint64_t gb = (uint64_t)(g * kSbWords + j) * 64;  // first bit of the word
            uint64_t x = wb[j];
            if (gb >= n_bits) x = 0;
            else if (n_bits - gb < 64) x &= (1ull << (n_bits - gb)) - 1;
            out[g * kSbWords + j] = x;
            pop += (unsigned long long)__popcll(x);
        }
    }
    if (cls) atomicAdd(&sums[0], cls);
    if (pop) atomicAdd(&sums[1], pop);
}

__global__ void k_word_popc(const uint64_t* __restrict__ w, int64_t nw, uint64_t* __restrict__ cnt) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= nw; i += (int64_t)gridDim.x * blockDim.x)
        cnt[i] = i < nw ? (uint64_t)__popcll(w[i]) : 0;
}

struct WtLevels {
    const uint64_t* w[9];
    const uint64_t* dir[9];  // ones before each word; one entry past the last word
};

// ones in [0, x), x <= n (the directory has an entry for every word and one past)
__device__ __forceinline__ uint64_t rank_excl(const uint64_t* __restrict__ w, const uint64_t* __restrict__ dir,
                                              uint64_t x) {
    const uint64_t k = x >> 6;
    const int r = (int)(x & 63);
    return dir[k] + (r ? (uint64_t)__popcll(w[k] & ((1ull << r) - 1)) : 0);
}

__global__ void k_wt_access(WtLevels L, int height, int64_t n, const uint64_t* __restrict__ node_start, int nodes,
                            int64_t nocc, uint8_t* __restrict__ bwt, unsigned long long* __restrict__ hist,
                            uint32_t* __restrict__ err) {
    __shared__ unsigned long long s_hist[256];
    for (int e = threadIdx.x; e < 256; e += blockDim.x) s_hist[e] = 0;
    __syncthreads();
    bool any_bad = false;
    for (int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; row < n; row += (int64_t)gridDim.x * blockDim.x) {
        uint64_t i = (uint64_t)row;
        uint32_t q = 0;
        bool bad = false;
        for (int l = 0; l < height; ++l) {
            if (i >= (uint64_t)n) { bad = true; break; }
            const uint64_t* w = L.w[l];
            const uint32_t bit = (uint32_t)((w[i >> 6] >> (i & 63)) & 1);
            if (l + 1 < height) {
                const uint64_t st = node_start[l * nodes + q];
                if (st > i) { bad = true; break; }
                const uint64_t ob = rank_excl(w, L.dir[l], i) - rank_excl(w, L.dir[l], st);
                const uint32_t child = 2 * q + bit;
                const uint64_t cst = node_start[(l + 1) * nodes + child];
                i = bit ? cst + ob : cst + (i - st - ob);
                q = child;
            } else {
                q = 2 * q + bit;
            }
        }
        // a symbol without an entry in the occurrence table is not one the
        // index holds (WaveletTreeRRR.h:238)
        if (!bad && (int64_t)q + 1 >= nocc) bad = true;
        if (bad) { any_bad = true; continue; }
        bwt[row] = (uint8_t)q;
        atomicAdd(&s_hist[q], 1ull);
    }
    if (any_bad) atomicOr(err, kDecBad);
    __syncthreads();
    for (int e = threadIdx.x; e < 256; e += blockDim.x)
        if (s_hist[e]) atomicAdd(&hist[e], s_hist[e]);
}

__global__ void k_set_bit_rows(const uint64_t* __restrict__ w, const uint64_t* __restrict__ dir, int64_t nw,
                               uint64_t cap, int64_t* __restrict__ rows) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nw; k += (int64_t)gridDim.x * blockDim.x) {
        uint64_t x = w[k], at = dir[k];
        while (x) {
            const int b = __ffsll((long long)x) - 1;
            if (at < cap) rows[at] = k * 64 + b;
            ++at;
            x &= x - 1;
        }
    }
}

// WaveletTreeRRR::rank (occurrences of sym in [0, i]) over the decoded
// levels; 0 for positions outside the sequence.
__device__ uint64_t wt_rank(const WtLevels& L, int height, uint64_t n, const uint64_t* __restrict__ occ, int64_t nocc,
                            uint64_t sym, uint64_t i) {
    uint64_t start = 0, r = ~0ull;
    for (int l = 0; r != 0 && l < height; ++l) {
        if (i >= n || start > n) return 0;
        const uint64_t* w = L.w[l];
        const uint64_t* dir = L.dir[l];
        const uint64_t before = rank_excl(w, dir, start);
        const uint64_t upto = rank_excl(w, dir, i + 1);
        if ((sym >> (height - l - 1)) & 1) {
            const uint64_t masked = (sym >> (height - l - 1)) << (height - l - 1);
            r = upto - before;
            if (masked >= (uint64_t)nocc) return 0;
            start = occ[masked];
        } else {
            r = i - start + before - upto + 1;
        }
        if (r == 0) return 0;
        i = r + start - 1;
    }
    return r;
}

// The last sampled row's SA value: LF-walk from it to the next sampled row
// with a stored value (out[0] = that sample's index, out[1] = the distance).
__global__ void k_sample_fixup(WtLevels L, int height, int64_t n, const uint64_t* __restrict__ occ, int64_t nocc,
                               const int64_t* __restrict__ C, const uint8_t* __restrict__ bwt,
                               const uint64_t* __restrict__ sw, const uint64_t* __restrict__ sdir, int64_t n_stored,
                               int64_t j, int64_t* __restrict__ out, uint32_t* __restrict__ err) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    uint64_t i = (uint64_t)j;
    int64_t dist = 0;
    for (;;) {
        if (i >= (uint64_t)n || dist >= kFixupMaxSteps) { atomicOr(err, kDecBad); return; }
        const uint64_t b = bwt[i];
        if (b == 0 || b >= 16) { atomicOr(err, kDecBad); return; }  // a '$' row is always sampled and stored
        const uint64_t rk = wt_rank(L, height, (uint64_t)n, occ, nocc, b, i);
        if (rk == 0 || C[b] < 0 || (uint64_t)C[b] + rk - 1 >= (uint64_t)n) { atomicOr(err, kDecBad); return; }
        i = (uint64_t)C[b] + rk - 1;  // LF(b, i) - 1 (FMDIndex.h:130-141)
        ++dist;
        if ((sw[i >> 6] >> (i & 63)) & 1) {
            const uint64_t idx = rank_excl(sw, sdir, i + 1) - 1;
            if (idx < (uint64_t)n_stored) {
                out[0] = (int64_t)idx;
                out[1] = dist;
                return;
            }
        }
    }
}

// Device allocations of one decode, freed together.
struct DevPool {
    std::vector<void*> ptrs;
    cudaError_t err = cudaSuccess;
    template <typename T> T* get(size_t count) {
        void* p = nullptr;
        if (err == cudaSuccess) err = cudaMalloc(&p, std::max<size_t>(count * sizeof(T), 16));
        if (err != cudaSuccess) return nullptr;
        ptrs.push_back(p);
        return static_cast<T*>(p);
    }
    void release(void* p) {
        for (auto& q : ptrs)
            if (q == p) { cudaFree(q); q = nullptr; }
    }
    ~DevPool() {
        for (void* p : ptrs)
            if (p) cudaFree(p);
    }
};

int grid_for(int64_t n, int threads, int num_sms) {
    const int64_t b = (n + threads - 1) / threads;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, (int64_t)num_sms * 16));
}

// One decoded bit sequence on the device: plain words and rank directory.
struct DevBits {
    uint64_t* w = nullptr;
    uint64_t* dir = nullptr;
    int64_t nw = 0;
};

// Unranks `raw` into `out`; MSG_EINVAL when its classes, offsets or ones
// disagree with its header.
int unrank_device(const RawRrr& raw, DevPool& pool, int num_sms, cudaStream_t st, DevBits& out) {
    const int64_t nC = (int64_t)raw.nC, nsb = (nC + kSbBlocks - 1) / kSbBlocks;
    const int64_t ncw = (int64_t)raw.C.w.size(), now = (int64_t)raw.O.w.size();
    if ((uint64_t)ncw * 64 < 4 * raw.nC || (uint64_t)now * 64 < raw.O.nbits || nsb <= 0) return MSG_EINVAL;
    uint64_t* d_cw = pool.get<uint64_t>(ncw);
    uint64_t* d_ow = pool.get<uint64_t>(now);
    uint64_t* d_sb = pool.get<uint64_t>(nsb);
    uint64_t* d_pos = pool.get<uint64_t>(nsb);
    out.nw = nsb * kSbWords;
    out.w = pool.get<uint64_t>(out.nw);
    uint64_t* d_cnt = pool.get<uint64_t>(out.nw + 1);
    out.dir = pool.get<uint64_t>(out.nw + 1);
    unsigned long long* d_sums = pool.get<unsigned long long>(2);
    uint32_t* d_err = pool.get<uint32_t>(1);
    if (pool.err != cudaSuccess) return pool.err == cudaErrorMemoryAllocation ? MSG_ENOMEM : MSG_ECUDA;
    cudaError_t e = cudaMemcpyAsync(d_cw, raw.C.w.data(), ncw * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && now > 0) e = cudaMemcpyAsync(d_ow, raw.O.w.data(), now * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_sums, 0, 16, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_err, 0, 4, st);
    if (e != cudaSuccess) return MSG_ECUDA;
    k_rrr_sb_bits<<<grid_for(nsb, 256, num_sms), 256, 0, st>>>(d_cw, ncw, nC, nsb, d_sb);
    size_t tb = 0;
    if (cub::DeviceScan::ExclusiveSum(nullptr, tb, d_sb, d_pos, (int)nsb, st) != cudaSuccess) return MSG_ECUDA;
    size_t tb2 = 0;
    if (cub::DeviceScan::ExclusiveSum(nullptr, tb2, d_cnt, out.dir, (int)(out.nw + 1), st) != cudaSuccess)
        return MSG_ECUDA;
    void* d_tmp = pool.get<uint8_t>(std::max(tb, tb2));
    if (pool.err != cudaSuccess) return pool.err == cudaErrorMemoryAllocation ? MSG_ENOMEM : MSG_ECUDA;
    if (cub::DeviceScan::ExclusiveSum(d_tmp, tb, d_sb, d_pos, (int)nsb, st) != cudaSuccess) return MSG_ECUDA;
    k_rrr_unrank<<<grid_for(nsb, 128, num_sms), 128, 0, st>>>(d_cw, ncw, d_ow, now, raw.O.nbits, nC, nsb, d_pos,
                                                              raw.n, out.w, d_sums, d_err);
    k_word_popc<<<grid_for(out.nw + 1, 256, num_sms), 256, 0, st>>>(out.w, out.nw, d_cnt);
    if (cub::DeviceScan::ExclusiveSum(d_tmp, tb2, d_cnt, out.dir, (int)(out.nw + 1), st) != cudaSuccess)
        return MSG_ECUDA;
    unsigned long long sums[2] = {0, 0};
    uint32_t bad = 0;
    uint64_t total = 0;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(sums, d_sums, 16, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, d_err, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&total, out.dir + out.nw, 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return MSG_ECUDA;
    pool.release(d_cw);
    pool.release(d_ow);
    pool.release(d_sb);
    pool.release(d_pos);
    pool.release(d_cnt);
    pool.release(d_tmp);
    if (bad || sums[0] != raw.ones || sums[1] != raw.ones || total != raw.ones) return MSG_EINVAL;
    return MSG_OK;
}

int read_fmd_device(const char* path, int num_sms, cudaStream_t st, msg_db& db) {
    FmdRaw f;
    // (below 2^36 symbols the scans' item counts fit their int arguments)
    if (!parse_fmd(path, f) || f.n == 0 || f.n >= (1ull << 36)) return MSG_EINVAL;
    const uint64_t n = f.n;
    const int height = (int)f.height, nodes = 1 << height;
    DevPool pool;
    WtLevels L{};
    DevBits sa_bits;
    for (int l = 0; l <= height; ++l) {
        DevBits b;
        const int rc = unrank_device(f.raw[l], pool, num_sms, st, b);
        if (rc != MSG_OK) return rc;
        if (l < height) { L.w[l] = b.w; L.dir[l] = b.dir; }
        else sa_bits = b;
        f.raw[l] = RawRrr();  // the host copy is no longer needed
    }
    const std::vector<uint64_t> ns = node_starts(f);
    uint64_t* d_ns = pool.get<uint64_t>(ns.size());
    uint64_t* d_occ = pool.get<uint64_t>(f.occ.size() + 1);
    int64_t* d_C = pool.get<int64_t>(256);
    uint8_t* d_bwt = pool.get<uint8_t>(n);
    unsigned long long* d_hist = pool.get<unsigned long long>(256);
    uint32_t* d_err = pool.get<uint32_t>(1);
    int64_t* d_fix = pool.get<int64_t>(2);
    if (pool.err != cudaSuccess) return pool.err == cudaErrorMemoryAllocation ? MSG_ENOMEM : MSG_ECUDA;
    cudaError_t e = cudaMemcpyAsync(d_ns, ns.data(), ns.size() * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && !f.occ.empty())
        e = cudaMemcpyAsync(d_occ, f.occ.data(), f.occ.size() * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_C, f.C, sizeof(f.C), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_hist, 0, 256 * 8, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_err, 0, 4, st);
    if (e != cudaSuccess) return MSG_ECUDA;
    k_wt_access<<<grid_for((int64_t)n, 256, num_sms), 256, 0, st>>>(L, height, (int64_t)n, d_ns, nodes,
                                                                    (int64_t)f.occ.size(), d_bwt, d_hist, d_err);
    unsigned long long hist[256];
    uint32_t bad = 0;
    uint64_t marked = 0;  // SAidx's set bits
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(hist, d_hist, sizeof(hist), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, d_err, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&marked, sa_bits.dir + sa_bits.nw, 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return MSG_ECUDA;
    if (bad) return MSG_EINVAL;
    // the decoded symbols must be the ones the occurrence table counts
    for (uint64_t q = 0; q + 1 < f.occ.size() && q < (uint64_t)nodes; ++q)
        if (hist[q] != f.occ[q + 1] - f.occ[q]) return MSG_EINVAL;
    if (marked != f.sa_sampled.size() && marked != f.sa_sampled.size() + 1) return MSG_EINVAL;
    // sampled rows: SAidx's set bits, in order
    int64_t* d_rows = pool.get<int64_t>(marked);
    if (pool.err != cudaSuccess) return pool.err == cudaErrorMemoryAllocation ? MSG_ENOMEM : MSG_ECUDA;
    k_set_bit_rows<<<grid_for(sa_bits.nw, 256, num_sms), 256, 0, st>>>(sa_bits.w, sa_bits.dir, sa_bits.nw, marked,
                                                                      d_rows);
    db.sample_rows.resize(marked);
    db.bwt.resize(n);
    e = cudaGetLastError();
    if (e == cudaSuccess && marked > 0)
        e = cudaMemcpyAsync(db.sample_rows.data(), d_rows, marked * 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(db.bwt.data(), d_bwt, n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return MSG_ECUDA;
    if (marked == f.sa_sampled.size() + 1) {
        // FMDIndex::buildSA left the last sample's value out of the file: walk
        // LF from that row to the next sampled row with a stored value
        const int64_t j = db.sample_rows[marked - 1];
        int64_t fix[2] = {-1, 0};
        uint32_t fb = 0;
        e = cudaMemsetAsync(d_err, 0, 4, st);
        if (e == cudaSuccess) {
            k_sample_fixup<<<1, 32, 0, st>>>(L, height, (int64_t)n, d_occ, (int64_t)f.occ.size(), d_C, d_bwt,
                                             sa_bits.w, sa_bits.dir, (int64_t)f.sa_sampled.size(), j, d_fix, d_err);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(fix, d_fix, 16, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&fb, d_err, 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return MSG_ECUDA;
        if (fb || fix[0] < 0 || fix[0] >= (int64_t)f.sa_sampled.size()) return MSG_EINVAL;
        f.sa_sampled.push_back(f.sa_sampled[fix[0]] + fix[1]);
    }
    for (int b = 0; b < 16; ++b) db.base_count[b] = f.B[b];
    db.sample_vals = std::move(f.sa_sampled);
    return db.sample_rows.size() == db.sample_vals.size() ? MSG_OK : MSG_EINVAL;
}

}  // namespace

extern "C" int msg_db_read_device(int device, const char* mtg_path, const char* mgs_path, const char* fmd_path,
                                  msg_db** db) {
    if (!mtg_path || !mgs_path || !fmd_path || !db) return MSG_EINVAL;
    *db = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return MSG_ECUDA;
    if (device < 0 || device >= count) return MSG_EINVAL;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return MSG_ECUDA;
    if (prop.major != 10 || prop.minor != 0) return MSG_EUNSUPPORTED;
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) return MSG_ECUDA;
    if (prev != device && cudaSetDevice(device) != cudaSuccess) return MSG_ECUDA;
    int rc = MSG_OK;
    msg_db* d = new (std::nothrow) msg_db();
    cudaStream_t st = nullptr;
    if (!d) rc = MSG_ENOMEM;
    else if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) rc = MSG_ECUDA;
    try {
        if (rc == MSG_OK) rc = read_mtg(mtg_path, mgs_path, *d) ? MSG_OK : MSG_EINVAL;
        if (rc == MSG_OK) rc = read_fmd_device(fmd_path, prop.multiProcessorCount, st, *d);
    } catch (const std::bad_alloc&) {
        rc = MSG_ENOMEM;
    }
    if (st) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    if (rc == MSG_OK && (d->bd_end.empty() || d->bd_end.back() != (int64_t)d->bwt.size())) rc = MSG_EINVAL;
    if (prev >= 0 && prev != device) cudaSetDevice(prev);
    if (rc != MSG_OK) { delete d; return rc; }
    *db = d;
    return MSG_OK;
}
