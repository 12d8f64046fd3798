// Internal device-side layout and primitives of the sm_100a mapping library.
//
// Index image in HBM
//   * occurrence buckets: 32 B each (one DRAM sector), 64 BWT symbols per bucket.
//       word 0: count of '$' before the bucket (bit 31 set when the bucket
//       holds a '$' or an N)
//       words 1-3: counts of A, C, G before the bucket (T is derived)
//       words 4-5 / 6-7: the low / high bit planes of the 64 symbols' 2-bit
//       codes (A=00, C=01, G=10, T=11; '$' and N stored as A), symbol k at bit k
//     one 32 B load (2 x 128-bit) gives all five counts at any row; a count
//     inside the bucket is one masked 64-bit popcount of a plane expression.
//   * dollar rows: sorted rows whose BWT symbol is '$' (2 per chromosome).
//   * N (genomes with N runs; the reference's BWT alphabet is $,A,C,G,T plus
//     N, FMDIndex.cpp:118-133): sorted rows whose BWT symbol is N, and the
//     count of N before each bucket (absent when the BWT holds no N).
//   * full suffix array, uint32 per row (N < 2^32), so locating a row is one
//     4-byte gather instead of an LF walk.
//   * chromosome table and forward nt16 target sequences for the DP.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace msg {

constexpr int kBucketSyms = 64;

struct __align__(32) Bucket {
    uint32_t cnt[4];
    uint32_t lo[2];  // low code bit of symbols 0..31 (lo[0]) and 32..63 (lo[1])
    uint32_t hi[2];  // high code bit
};
static_assert(sizeof(Bucket) == 32, "bucket must be one 32 B sector");

// nt16 helpers (DNAalphabet.h:37-191)
__host__ __device__ inline bool is_basic(int b) { return b == 1 || b == 2 || b == 4 || b == 8; }
__host__ __device__ inline int to_int(int b) {  // $,A,C,G,T -> 0..4 (others 0)
    return b == 1 ? 1 : b == 2 ? 2 : b == 4 ? 3 : b == 8 ? 4 : 0;
}
__host__ __device__ inline int comp16(int b) {
    // reverse the 4 bits: A<->T, C<->G, IUPAC codes map accordingly, N->N, 0->0
    return ((b & 1) << 3) | ((b & 2) << 1) | ((b & 4) >> 1) | ((b & 8) >> 3);
}
__host__ __device__ inline int encode_int(int j) { return j == 1 ? 1 : j == 2 ? 2 : j == 3 ? 4 : j == 4 ? 8 : 0; }
// slot of a BWT symbol in Occ5: $,A,C,G,T -> 0..4, N -> 5
__host__ __device__ inline int occ_slot(int b) { return b == 15 ? 5 : to_int(b); }

struct IndexDev {
    const Bucket* bkt;
    const int64_t* dollar_rows;
    int64_t n_dollar;
    const int64_t* n_rows;     // sorted rows whose symbol is N
    int64_t n_n;
    const uint32_t* n_before;  // per bucket: N before it (null when n_n == 0)
    const uint32_t* sa;
    const uint8_t* text;       // the BD text (nt16 codes, '$' = 0) that the suffix array indexes, 16 bytes of slack
    const uint32_t* isa;       // inverse suffix array: isa[sa[i]] = i
    int64_t n;
    int64_t C[17];           // FMDIndex::C for nt16 codes 0..16
    const int64_t* bd_start; // per chromosome
    const int64_t* bd_end;
    const int64_t* chr_len;
    const int64_t* chr_off;
    const uint8_t* chr_seq;
    int64_t n_chrom;
};

struct Occ5 {
    int64_t c[6];  // $, A, C, G, T, N in BWT[0 .. i]
};

// Count of rows in [lo, hi) of a sorted row list, by binary search.
__device__ inline int64_t rows_between(const int64_t* rows, int64_t n, int64_t lo, int64_t hi) {
    int64_t a = 0, b = n;
    while (a < b) { int64_t m = (a + b) >> 1; if (rows[m] < lo) a = m + 1; else b = m; }
    const int64_t s = a;
    b = n;
    while (a < b) { int64_t m = (a + b) >> 1; if (rows[m] < hi) a = m + 1; else b = m; }
    return a - s;
}
// '$' rows and N rows in [lo, hi)
__device__ inline int64_t dollar_between(const IndexDev& ix, int64_t lo, int64_t hi) {
    return rows_between(ix.dollar_rows, ix.n_dollar, lo, hi);
}
__device__ inline int64_t nsym_between(const IndexDev& ix, int64_t lo, int64_t hi) {
    return ix.n_n ? rows_between(ix.n_rows, ix.n_n, lo, hi) : 0;
}

// Bits 0 .. r-1 set (r in [0, 64]): the symbols before row k*64 + r.
__device__ __forceinline__ uint64_t prefix_mask(uint32_t r) { return r >= 64 ? ~0ull : ((1ull << r) - 1ull); }

__device__ __forceinline__ uint64_t plane_lo(const uint4& w1) { return ((uint64_t)w1.y << 32) | w1.x; }
__device__ __forceinline__ uint64_t plane_hi(const uint4& w1) { return ((uint64_t)w1.w << 32) | w1.z; }

// Counts of $,A,C,G,T,N among the first r symbols of a loaded bucket k, from
// the bit planes: T = lo&hi, C = lo&~hi, G = ~lo&hi, A ('$' and N included)
// the rest; '$' and N inside the bucket from their row lists.
__device__ inline Occ5 occ5_in(const IndexDev& ix, int64_t k, int r, const uint4& w0, const uint4& w1) {
    Occ5 o;
    const uint64_t lo = plane_lo(w1), hi = plane_hi(w1), m = prefix_mask((uint32_t)r);
    const uint32_t n_t = (uint32_t)__popcll(lo & hi & m);
    const uint32_t nC = (uint32_t)__popcll(lo & ~hi & m), nG = (uint32_t)__popcll(~lo & hi & m);
    const uint32_t nA = (uint32_t)r - nC - nG - n_t;
    const int64_t j = k * kBucketSyms + r;
    const bool has_exc = (w0.x >> 31) != 0;
    int64_t d_in = 0, n_in = 0;
    if (has_exc && r > 0) {
        d_in = dollar_between(ix, k * kBucketSyms, j);
        n_in = nsym_between(ix, k * kBucketSyms, j);
    }
    o.c[0] = (int64_t)(w0.x & 0x7fffffffu) + d_in;
    o.c[1] = (int64_t)w0.y + (int64_t)nA - d_in - n_in;
    o.c[2] = (int64_t)w0.z + nC;
    o.c[3] = (int64_t)w0.w + nG;
    o.c[5] = (ix.n_before ? (int64_t)__ldg(ix.n_before + k) : 0) + n_in;
    o.c[4] = j - o.c[0] - o.c[1] - o.c[2] - o.c[3] - o.c[5];
    return o;
}

// Occurrences of $,A,C,G,T in BWT[0 .. i] for -1 <= i < n.
__device__ inline Occ5 occ5(const IndexDev& ix, int64_t i) {
    const int64_t j = i + 1;               // exclusive end
    const int64_t k = j / kBucketSyms;
    const int r = (int)(j - k * kBucketSyms);
    const uint4* p = reinterpret_cast<const uint4*>(ix.bkt + k);
    const uint4 w0 = __ldg(p), w1 = __ldg(p + 1);
    return occ5_in(ix, k, r, w0, w1);
}

// Counts at two rows; one bucket load when both fall in the same bucket.
__device__ inline void occ5_pair(const IndexDev& ix, int64_t i_lo, int64_t i_hi, Occ5& lo, Occ5& hi) {
    const int64_t ja = i_lo + 1, jb = i_hi + 1;
    const int64_t ka = ja / kBucketSyms, kb = jb / kBucketSyms;
    const uint4* pa = reinterpret_cast<const uint4*>(ix.bkt + ka);
    const uint4* pb = reinterpret_cast<const uint4*>(ix.bkt + kb);
    const uint4 a0 = __ldg(pa), a1 = __ldg(pa + 1);
    uint4 b0 = a0, b1 = a1;
    if (kb != ka) { b0 = __ldg(pb); b1 = __ldg(pb + 1); }
    lo = occ5_in(ix, ka, (int)(ja - ka * kBucketSyms), a0, a1);
    hi = occ5_in(ix, kb, (int)(jb - kb * kBucketSyms), b0, b1);
}

// BWT symbol (nt16) at row i.
__device__ inline int bwt_at(const IndexDev& ix, int64_t i) {
    const int64_t k = i / kBucketSyms;
    const int r = (int)(i - k * kBucketSyms);
    const uint32_t wl = __ldg(&ix.bkt[k].lo[r >> 5]), wh = __ldg(&ix.bkt[k].hi[r >> 5]);
    const int code = (int)(((wl >> (r & 31)) & 1u) | (((wh >> (r & 31)) & 1u) << 1));
    if (code == 0 && (__ldg(&ix.bkt[k].cnt[0]) >> 31)) {
        if (dollar_between(ix, i, i + 1)) return 0;
        if (nsym_between(ix, i, i + 1)) return 15;
    }
    return encode_int(code + 1);
}

// FMDIndex::backExt (FMDIndex.cpp:577-610). Returns the new size. The q
// update counts '$' and the bases after b, not N, as the reference does.
__device__ inline int64_t back_ext(const IndexDev& ix, int64_t& p, int64_t& q, int64_t& s, int b) {
    if (!is_basic(b)) return (s = 0);
    const int c = to_int(b);
    Occ5 lo, hi;
    occ5_pair(ix, p - 1, p + s - 1, lo, hi);
    const int64_t O = lo.c[c];
    int64_t sB[5];
#pragma unroll
    for (int j = 0; j < 5; ++j) sB[j] = hi.c[j] - lo.c[j];
    if (sB[c] <= 0) return (s = sB[c]);
    if (sB[c] != s) {
        int64_t qq = q + sB[0];  // qB[4]
        for (int j = 4; j > c; --j) qq += sB[j];
        q = qq;
    }
    p = ix.C[b] + O;
    s = sB[c];
    return s;
}

__device__ inline int64_t fwd_ext(const IndexDev& ix, int64_t& p, int64_t& q, int64_t& s, int b) {
    return back_ext(ix, q, p, s, comp16(b));
}

// Counts at row k*64 + r of a loaded bucket k, for one base (A,C,G,T: code
// 0..3), 32-bit (rows < 2^32): eq = occurrences of the base, gt = occurrences
// of the bases after it (C,G,T after A; G,T after C; T after G), dl =
// occurrences of '$', all among the rows before k*64 + r. Stored counts give
// '$', A, C, G before the bucket (T is the rest); within the bucket one masked
// 64-bit popcount per count over the bit planes: the symbols equal to the
// code are where both planes match its bits, the bases after A are lo|hi,
// after C hi, after G lo&hi. '$' and N are stored as A and removed from A's
// count; the N before the bucket come from their own table.
__device__ __forceinline__ void occ_counts(const IndexDev& ix, uint32_t k, uint32_t r, uint32_t code, const uint4& w0,
                                           const uint4& w1, uint32_t& eq, uint32_t& gt, uint32_t& dl) {
    const uint64_t lo = plane_lo(w1), hi = plane_hi(w1), m = prefix_mask(r);
    const uint64_t cl = (code & 1u) ? ~0ull : 0ull, ch = (code & 2u) ? ~0ull : 0ull;
    const uint32_t n_eq = (uint32_t)__popcll(~(lo ^ cl) & ~(hi ^ ch) & m);
    const uint64_t after = code == 0 ? (lo | hi) : code == 1 ? hi : code == 2 ? (lo & hi) : 0ull;
    const uint32_t n_gt = (uint32_t)__popcll(after & m);
    const uint32_t dollar = w0.x & 0x7fffffffu;
    uint32_t din = 0, nin = 0;
    if ((w0.x >> 31) && r > 0) {
        din = (uint32_t)dollar_between(ix, (int64_t)k * kBucketSyms, (int64_t)k * kBucketSyms + r);
        nin = (uint32_t)nsym_between(ix, (int64_t)k * kBucketSyms, (int64_t)k * kBucketSyms + r);
    }
    const uint32_t nbef = ix.n_before ? __ldg(ix.n_before + k) : 0u;
    const uint32_t all = k * (uint32_t)kBucketSyms - dollar - nbef;  // bases before the bucket
    const uint32_t a = w0.y, c = w0.z, g = w0.w;
    const uint32_t before_eq = code == 0 ? a : code == 1 ? c : code == 2 ? g : all - a - c - g;
    const uint32_t before_gt = code == 0 ? all - a : code == 1 ? all - a - c : code == 2 ? all - a - c - g : 0u;
    eq = before_eq + n_eq - (code == 0 ? din + nin : 0u);
    gt = before_gt + n_gt;
    dl = dollar + din;
}

// The two occurrence buckets a 32-bit backward extension of (p, s) reads: the
// buckets of rows p-1 and p+s-1 (one when both fall in the same bucket).
struct ExtLoad {
    uint4 a0, a1, b0, b1;
};

__device__ __forceinline__ void back_ext32_load(const IndexDev& ix, uint32_t p, uint32_t s, ExtLoad& l) {
    const uint32_t ka = p >> 6, kb = (p + s) >> 6;  // exclusive ends of rows p-1 and p+s-1
    const uint4* pa = reinterpret_cast<const uint4*>(ix.bkt + ka);
    l.a0 = __ldg(pa);
    l.a1 = __ldg(pa + 1);
    l.b0 = l.a0;
    l.b1 = l.a1;
    if (kb != ka) {
        const uint4* pb = reinterpret_cast<const uint4*>(ix.bkt + kb);
        l.b0 = __ldg(pb);
        l.b1 = __ldg(pb + 1);
    }
}

// FMDIndex::backExt (FMDIndex.cpp:577-610) on 32-bit bi-intervals from loaded
// buckets (b a basic base): the size from the base's counts at the two rows,
// and q, when the size changes, from the counts of '$' and of the bases after
// it (FMDIndex.cpp:592-604).
__device__ __forceinline__ uint32_t back_ext32_apply(const IndexDev& ix, uint32_t& p, uint32_t& q, uint32_t& s, int b,
                                                     const ExtLoad& l) {
    const uint32_t code = (uint32_t)(to_int(b) - 1);
    const uint32_t ja = p, jb = p + s;
    uint32_t oa, ga, da, ob, gb, db;
    occ_counts(ix, ja >> 6, ja & 63u, code, l.a0, l.a1, oa, ga, da);
    occ_counts(ix, jb >> 6, jb & 63u, code, l.b0, l.b1, ob, gb, db);
    const uint32_t ns = ob - oa;
    if (ns == 0) { s = 0; return 0; }
    if (ns != s) q = q + (db - da) + (gb - ga);
    p = (uint32_t)ix.C[b] + oa;
    s = ns;
    return ns;
}

__device__ inline int64_t back_ext32(const IndexDev& ix, uint32_t& p, uint32_t& q, uint32_t& s, int b) {
    if (!is_basic(b)) { s = 0; return 0; }
    ExtLoad l;
    back_ext32_load(ix, p, s, l);
    return back_ext32_apply(ix, p, q, s, b, l);
}

// Error bits of the device status word.
enum : uint32_t {
    kErrInternal = 1u,     // consistency check failed
    kErrOverflow = 2u,     // an output capacity was exceeded (host retries)
    kErrTrace = 4u,        // traceback left the matrix (reference would read out of bounds)
    kErrCodes = 8u,        // a read byte is not an nt16 code (0..15)
};

// Every byte of the reads' range [off[0], off[n]) must be an nt16 code
// (0..15, what DNAalphabet's encoder gives): the kernels index 16-entry
// tables with them. Sets kErrCodes in *status otherwise. (static: one copy
// per translation unit that launches it)
static __global__ void k_check_codes(const uint8_t* __restrict__ seq, const int64_t* __restrict__ off, int64_t n,
                              uint32_t* __restrict__ status) {
    const int64_t a = off[0], b = off[n];
    bool bad = false;
    for (int64_t i = a + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < b; i += (int64_t)gridDim.x * blockDim.x)
        bad |= __ldg(seq + i) > 15;
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(status, (uint32_t)kErrCodes);
}

}  // namespace msg
