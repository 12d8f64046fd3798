// MEM search and read cleaning on sm_100a: msgseqtk-clean's per-read task
// (src/msgseqtk-clean.cpp:413-486) -- SMEM_LIST::findMEMS (src/SMEM.cpp:174-184,
// SMEM::findMEM :42-62) against a reference and a background FMD-index, each
// list's loglik (src/SMEM.cpp:307-312) and the log-odds decision.
//
// One thread walks one (read, index) unit: a forward extension per base, two
// occurrence buckets (one 32 B sector each) per extension, no per-read state
// beyond registers, so any read length runs in place. The log-likelihood sums
// are made in the reference's order with round-to-nearest double adds, and the
// e-value test compares them against the host-derived threshold (the largest
// log-likelihood whose e-value the host's exp keeps), so results are
// bit-identical to the reference's.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "msg_ctx.cuh"

using namespace msg;

namespace msg {
int evalue_threshold(int64_t n, double max_e, double* thr, int* all);  // map.cu
}

namespace {

int64_t nblk(int64_t n, int t) { return (n + t - 1) / t; }

// The two occurrence buckets one extension of bi-interval (p, s) reads: rows
// p-1 and p+s-1 (exclusive ends p and p+s), one 32 B sector each, one load
// when both rows fall in the same bucket.
struct Bkt {
    uint4 a0, a1, b0, b1;
    uint32_t ja, jb;
};

__device__ __forceinline__ void mem_load(const IndexDev& ix, uint32_t p, uint32_t s, Bkt& k) {
    k.ja = p;
    k.jb = p + s;
    const uint32_t ka = k.ja >> 6, kb = k.jb >> 6;
    const uint4* pa = reinterpret_cast<const uint4*>(ix.bkt + ka);
    k.a0 = __ldg(pa);
    k.a1 = __ldg(pa + 1);
    k.b0 = k.a0;
    k.b1 = k.a1;
    if (kb != ka) {
        const uint4* pb = reinterpret_cast<const uint4*>(ix.bkt + kb);
        k.b0 = __ldg(pb);
        k.b1 = __ldg(pb + 1);
    }
}

// FMDIndex::backExt (src/FMDIndex.cpp:577-610) for the MEM walk, on buckets
// loaded by mem_load(p, s). Unlike the SMEM search, findMEM starts intervals
// on any read symbol, so a gap symbol (nt16 0, what the reference's encoder
// gives every unknown character) opens the '$' interval at row 0, and the
// next extension asks WaveletTreeRRR::rank(b, p - 1) with p - 1 = -1; that
// rank answers (size_t)-1 for every symbol
// (src/libsds/src/WaveletTreeRRR.cpp:102-103), i.e. -1 after the cast, which
// this function reproduces. A size of 0 stays 0.
__device__ __forceinline__ void mem_back_ext(const IndexDev& ix, const Bkt& k, uint32_t& p, uint32_t& q,
                                             uint32_t& s, int b, uint32_t& n_ext) {
    if (!is_basic(b) || s == 0) { s = 0; return; }
    n_ext++;
    const uint32_t code = (uint32_t)(to_int(b) - 1);
    uint32_t oa, ga, da, ob, gb, db;
    occ_counts(ix, k.ja >> 6, k.ja & 63u, code, k.a0, k.a1, oa, ga, da);
    occ_counts(ix, k.jb >> 6, k.jb & 63u, code, k.b0, k.b1, ob, gb, db);
    if (p == 0) {  // every count at row -1 is -1: (3 - code) bases after b
        oa = 0xffffffffu;
        da = 0xffffffffu;
        ga = 0u - (3u - code);
    }
    const uint32_t ns = ob - oa;
    if (ns == 0) { s = 0; return; }
    if (ns != s) q = q + (db - da) + (gb - ga);
    p = (uint32_t)ix.C[b] + oa;
    s = ns;
}

struct MemArgs {
    IndexDev ix0, ix1;         // reference (and background) index
    double llk0[16], llk1[16]; // FMDIndex::loglik per nt16 code of each index
    double thr0, thr1;         // e-value thresholds on the log-likelihood
    int all0, all1;            // 1: no e-value limit
    int n_set;                 // 1 (single reads) or 2 (first and second mates)
    const uint8_t* seq0;
    const int64_t* off0;
    const uint8_t* seq1;
    const int64_t* off1;
    int64_t n;                 // reads per set
    int64_t min_len;
    const int64_t* slot;       // first output row of each read (one index, one set; rows != null)
    int64_t* rows;             // 6 int64 per MEM: from, to, fwdStart, revStart, size, logP bits
    double* ll;                // per (index, set, read): MEM_LIST::loglik
    int32_t* cnt;              // per (index, set, read): MEMs kept
    unsigned long long* n_ext; // [0]: extensions; word 2 of the same buffer: error bits
};

constexpr int64_t kMemMaxLen = 0x7ffffffdll;  // `to` reaches L + 1 in 32 bits

// One SMEM_LIST::findMEMS walk (src/SMEM.cpp:174-184): the current MEM's
// start `from` and end `to`, its bi-interval (fwdStart P, revStart Q, size S)
// and log-likelihood lp, the next base nb, and the kept list's loglik/count.
// The reference's findMEM (src/SMEM.cpp:42-62) runs its backward pass from
// the state the failed forward extension left (size 0), so that pass never
// extends: each MEM keeps its start, ends one past the last matching base
// with the failed state's fields, and the next search starts there.
struct Walk {
    const uint8_t* sq;
    int32_t L, from, to;  // reads are below 2^31 - 2 bases (checked)
    uint32_t P, Q, S;
    int nb;
    double lp, ll;
    int32_t cnt;
};

// SMEM's constructor + evaluate at `from` (SMEM.h:48-54, SMEM.cpp:19-24).
__device__ __forceinline__ void walk_start(const IndexDev& ix, const double* llk, Walk& w) {
    const int b = w.sq[w.from];
    w.P = (uint32_t)ix.C[b];
    w.Q = (uint32_t)ix.C[comp16(b)];
    w.S = (uint32_t)(ix.C[b + 1] - ix.C[b]);
    w.lp = __dadd_rn(0.0, llk[b]);
    w.to = w.from + 1;
    w.nb = w.to < w.L ? w.sq[w.to] : 0;
}

// One SMEM::fwdExt + fwdEvaluate (SMEM.h:140-145,166-170); when the size
// drops to 0 the MEM ends: findMEMS's length and e-value test, then the next
// MEM starts at the end.
template <bool ROWS>
__device__ __forceinline__ void walk_step(const IndexDev& ix, const double* llk, double thr, int all, int64_t min_len,
                                          const Bkt& k, int nn, Walk& w, int64_t* __restrict__ out, uint32_t& n_ext) {
    mem_back_ext(ix, k, w.Q, w.P, w.S, comp16(w.nb), n_ext);
    if (w.to < w.L) w.lp = __dadd_rn(w.lp, llk[w.nb]);
    ++w.to;
    w.nb = nn;
    if (w.S != 0) return;
    if (w.to - w.from >= min_len && (all || w.lp <= thr)) {
        if (ROWS) {
            int64_t* o = out + 6 * (int64_t)w.cnt;
            o[0] = w.from; o[1] = w.to; o[2] = w.P; o[3] = w.Q; o[4] = 0;
            o[5] = __double_as_longlong(w.lp);
        }
        w.ll = __dadd_rn(w.ll, w.lp);
        w.cnt++;
    }
    w.from = w.to;
    if (w.from < w.L) walk_start(ix, llk, w);
}

// NW walks per thread in one flat loop: every iteration issues the bucket
// loads of all live walks, then advances each by one extension, so a thread
// keeps NW independent loads in flight and a warp's threads stay in step
// whatever their MEM lengths (nested per-MEM loops leave most lanes idle
// while the longest MEM of the warp finishes). NW == 2: a thread per read
// (or mate) against both indexes, walk j on index j; NW == 1: a thread per
// read (or mate) on index 0.
template <int NW, bool ROWS>
__global__ void __launch_bounds__(256, NW == 1 ? 4 : 3) k_mems(MemArgs a) {
    __shared__ double s_llk[2][16];
    if (threadIdx.x < 32) {
        const int b = threadIdx.x & 15;
        s_llk[threadIdx.x >> 4][b] = threadIdx.x < 16 ? a.llk0[b] : a.llk1[b];
    }
    __syncthreads();
    const int64_t per_idx = a.n * a.n_set;
    const int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    uint32_t n_ext = 0;
    if (u < per_idx) {
        const int set = u >= a.n;
        const int64_t r = u - set * a.n;
        const int64_t* of = set ? a.off1 : a.off0;
        const int64_t o0 = of[r], len = of[r + 1] - o0;
        if (len > kMemMaxLen) atomicOr(reinterpret_cast<uint32_t*>(a.n_ext) + 2, 1u);
        Walk w[NW];
#pragma unroll
        for (int j = 0; j < NW; ++j) {
            w[j].sq = (set ? a.seq1 : a.seq0) + o0;
            w[j].L = len > kMemMaxLen ? 0 : (int32_t)len;
            w[j].from = 0;
            w[j].ll = 0.0;
            w[j].cnt = 0;
            if (w[j].L > 0) walk_start(j ? a.ix1 : a.ix0, s_llk[j], w[j]);
        }
        int64_t* out = ROWS ? a.rows + 6 * a.slot[u] : nullptr;
        for (;;) {
            Bkt k[NW];
            bool live[NW];
            bool any = false;
#pragma unroll
            for (int j = 0; j < NW; ++j) {
                live[j] = w[j].from < w[j].L;
                any |= live[j];
                if (live[j]) mem_load(j ? a.ix1 : a.ix0, w[j].Q, w[j].S, k[j]);
            }
            if (!any) break;
            int nn[NW];
#pragma unroll
            for (int j = 0; j < NW; ++j) nn[j] = live[j] && w[j].to + 1 < w[j].L ? w[j].sq[w[j].to + 1] : 0;
#pragma unroll
            for (int j = 0; j < NW; ++j) {
                if (!live[j]) continue;
                if (j)
                    walk_step<ROWS>(a.ix1, s_llk[1], a.thr1, a.all1, a.min_len, k[j], nn[j], w[j], out, n_ext);
                else
                    walk_step<ROWS>(a.ix0, s_llk[0], a.thr0, a.all0, a.min_len, k[j], nn[j], w[j], out, n_ext);
            }
        }
#pragma unroll
        for (int j = 0; j < NW; ++j) {
            a.ll[j * per_idx + u] = w[j].ll;
            a.cnt[j * per_idx + u] = w[j].cnt;
        }
    }
    unsigned long long e = n_ext;
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) e += __shfl_down_sync(0xffffffffu, e, d);
    if ((threadIdx.x & 31) == 0 && e) atomicAdd(a.n_ext, e);
}

// msgseqtk-clean's decision per read (pair): refLoglik, bgLoglik (a pair's:
// first + second, SMEM_LIST::loglik(SMEM_LIST_PE), src/SMEM.h:391-393),
// lod = -refLoglik + bgLoglik, kept when lod > min_lod.
__global__ void k_clean_lod(const double* __restrict__ ll, int64_t n, int n_set, double min_lod, double* __restrict__ ref,
                            double* __restrict__ bg, double* __restrict__ lod, uint8_t* __restrict__ keep) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t per_idx = n * n_set;
    double r = ll[i], g = ll[per_idx + i];
    if (n_set == 2) {
        r = __dadd_rn(r, ll[n + i]);
        g = __dadd_rn(g, ll[per_idx + n + i]);
    }
    const double d = __dadd_rn(-r, g);
    ref[i] = r;
    bg[i] = g;
    lod[i] = d;
    keep[i] = d > min_lod;
}

// off[i] -= base for i < n (host offsets rebased to their set's first read).
__global__ void k_rebase(int64_t* __restrict__ off, int64_t n, int64_t base) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) off[i] -= base;
}

// Rows of unit i from its slot to its place in read order.
__global__ void k_compact_rows(const int64_t* __restrict__ slot, const int64_t* __restrict__ dst,
                               const int32_t* __restrict__ cnt, int64_t n, const int64_t* __restrict__ src,
                               int64_t* __restrict__ out) {
    const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= n) return;
    const int64_t m = 6 * (int64_t)cnt[w];
    const int64_t* s = src + 6 * slot[w];
    int64_t* d = out + 6 * dst[w];
    for (int64_t j = lane; j < m; j += 32) d[j] = s[j];
}

int check_mem_params(const msg_mem_params* p) {
    if (!p) return MSG_EINVAL;
    if (std::isnan(p->max_evalue) || p->max_evalue < 0) return MSG_EINVAL;
    return MSG_OK;
}

// A read set as given by the caller: host or device pointers.
struct Set {
    const uint8_t* seq;
    const int64_t* off;
};

bool check_offsets(const msg_read_batch* r) {
    if (r->n_reads < 0 || (r->n_reads > 0 && (!r->seq || !r->off))) return false;
    for (int64_t i = 0; i < r->n_reads; ++i)
        if (r->off[i + 1] < r->off[i]) return false;
    return true;
}

// Copy host read sets (1 or 2, same read count) into ctx->reads / ctx->offs:
// set k's bytes follow set k-1's, each set with its own n + 1 offsets.
int upload_sets(msg_ctx* ctx, const msg_read_batch* const* sets, int n_set, Set* dev) {
    const int64_t n = sets[0]->n_reads;
    int64_t bytes[2] = {0, 0};
    for (int k = 0; k < n_set; ++k) {
        if (!check_offsets(sets[k]) || sets[k]->n_reads != n) return ctx->fail(MSG_EINVAL, "bad read batch");
        bytes[k] = n > 0 ? sets[k]->off[n] - sets[k]->off[0] : 0;
    }
    cudaError_t e = ctx->reads.ensure(bytes[0] + bytes[1] + 16);
    if (e == cudaSuccess) e = ctx->offs.ensure(n_set * (n + 1) * 8 + 16);
    if (e != cudaSuccess) return ctx->cuda_fail(e);
    // the caller's bytes and offsets are copied as they are (straight from
    // pinned memory when the caller pinned them) and each set's offsets
    // rebased on the device; the call returns only after its last copy
    for (int k = 0; k < n_set; ++k) {
        const msg_read_batch* r = sets[k];
        uint8_t* d_seq = ctx->reads.as<uint8_t>() + (k ? bytes[0] : 0);
        int64_t* d_off = ctx->offs.as<int64_t>() + k * (n + 1);
        if (bytes[k] > 0) e = cudaMemcpyAsync(d_seq, r->seq + r->off[0], bytes[k], cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess && n > 0) e = cudaMemcpyAsync(d_off, r->off, (n + 1) * 8, cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess && n > 0 && r->off[0] != 0) {
            k_rebase<<<nblk(n + 1, 256), 256, 0, ctx->stream>>>(d_off, n + 1, r->off[0]);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess && n == 0) e = cudaMemsetAsync(d_off, 0, 8, ctx->stream);
        if (e != cudaSuccess) return ctx->cuda_fail(e);
        dev[k].seq = d_seq;
        dev[k].off = d_off;
    }
    return MSG_OK;
}

// Launch the MEM walk of n_set read sets (n reads each) against ctx's index
// and, when bg is given, bg's index too, on ctx's stream. Per-unit loglik and
// counts land in ctx->memo (ll at offset 0, counts after n_units doubles).
// With rows, host_slot gives each unit's first slot row (n_units + 1 entries).
int mem_launch(msg_ctx* ctx, const msg_ctx* bg, const Set* sets, int n_set, int64_t n, const msg_mem_params* p,
               const int64_t* d_slot, int64_t* d_rows, double** d_ll, int32_t** d_cnt) {
    const int n_idx = bg ? 2 : 1;
    const int64_t n_units = n * n_set * n_idx;
    MemArgs a{};
    a.ix0 = ctx->idx.dev;
    for (int b = 0; b < 16; ++b) a.llk0[b] = ctx->idx.llk[b];
    int rc = evalue_threshold(ctx->idx.dev.n, p->max_evalue, &a.thr0, &a.all0);
    if (rc != MSG_OK) return ctx->fail(rc, "e-value threshold");
    if (bg) {
        a.ix1 = bg->idx.dev;
        for (int b = 0; b < 16; ++b) a.llk1[b] = bg->idx.llk[b];
        rc = evalue_threshold(bg->idx.dev.n, p->max_evalue, &a.thr1, &a.all1);
        if (rc != MSG_OK) return ctx->fail(rc, "e-value threshold");
    }
    a.n_set = n_set;
    a.seq0 = sets[0].seq; a.off0 = sets[0].off;
    a.seq1 = n_set > 1 ? sets[1].seq : sets[0].seq;
    a.off1 = n_set > 1 ? sets[1].off : sets[0].off;
    a.n = n;
    a.min_len = p->min_len;
    a.slot = d_slot;
    a.rows = d_rows;
    cudaError_t e = ctx->memo.ensure(n_units * 12 + 64);
    if (e == cudaSuccess) e = ctx->status.ensure(128);
    if (e != cudaSuccess) return ctx->cuda_fail(e);
    a.ll = ctx->memo.as<double>();
    a.cnt = reinterpret_cast<int32_t*>(a.ll + n_units);
    a.n_ext = reinterpret_cast<unsigned long long*>(ctx->status.p);
    e = cudaMemsetAsync(ctx->status.p, 0, 128, ctx->stream);
    if (e != cudaSuccess) return ctx->cuda_fail(e);
    if (n > 0) {  // the walks index 16-entry tables with the read bytes: check them first
        uint32_t* codes = reinterpret_cast<uint32_t*>(ctx->status.p) + 4;
        for (int k = 0; k < n_set; ++k)
            k_check_codes<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(sets[k].seq, sets[k].off, n, codes);
        ctx->stats.n_launch += n_set;
        uint32_t h_codes = 0;
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(&h_codes, codes, 4, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) return ctx->cuda_fail(e);
        if (h_codes & kErrCodes) return ctx->fail(MSG_EINVAL, "read bytes must be nt16 codes (0..15)");
    }
    if (n_units > 0) {
        cudaStream_t st = ctx->stream;
        const int64_t g = nblk(n * n_set, 256);
        if (n_idx == 1 && d_rows) k_mems<1, true><<<g, 256, 0, st>>>(a);
        else if (n_idx == 1) k_mems<1, false><<<g, 256, 0, st>>>(a);
        else k_mems<2, false><<<g, 256, 0, st>>>(a);
        ctx->stats.n_launch++;
        e = cudaGetLastError();
        if (e != cudaSuccess) return ctx->cuda_fail(e);
    }
    *d_ll = a.ll;
    *d_cnt = a.cnt;
    return MSG_OK;
}

void stats_begin(msg_ctx* ctx, int64_t n_reads) {
    std::memset(&ctx->stats, 0, sizeof(ctx->stats));
    ctx->stats.n_reads = n_reads;
    cudaEventRecord(ctx->ev[0], ctx->stream);
}

int stats_end(msg_ctx* ctx) {
    cudaEventRecord(ctx->ev[2], ctx->stream);
    unsigned long long st[2] = {0, 0};  // extensions, error bits
    cudaError_t e = cudaMemcpyAsync(st, ctx->status.p, 16, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return ctx->cuda_fail(e);
    const unsigned long long n_ext = st[0];
    if (st[1] & 1u) return ctx->fail(MSG_EUNSUPPORTED, "a read of 2^31 - 2 bases or more");
    float t0 = 0, t1 = 0;
    cudaEventElapsedTime(&t0, ctx->ev[0], ctx->ev[1]);
    cudaEventElapsedTime(&t1, ctx->ev[0], ctx->ev[2]);
    ctx->stats.n_ext = (int64_t)n_ext;
    ctx->stats.ms_smem = t0;
    ctx->stats.ms_total = t1;
    return MSG_OK;
}

int clean_impl(msg_ctx* ref, msg_ctx* bg, const Set* sets, int n_set, int64_t n, const msg_mem_params* params,
               double min_lod, double* ref_ll, double* bg_ll, double* lod, uint8_t* keep) {
    if (std::isnan(min_lod)) return ref->fail(MSG_EINVAL, "min_lod is NaN");
    stats_begin(ref, n);
    double* d_ll;
    int32_t* d_cnt;
    int rc = mem_launch(ref, bg, sets, n_set, n, params, nullptr, nullptr, &d_ll, &d_cnt);
    if (rc != MSG_OK) return rc;
    cudaEventRecord(ref->ev[1], ref->stream);
    cudaError_t e = ref->memo2.ensure(n * 25 + 64);
    if (e != cudaSuccess) return ref->cuda_fail(e);
    double* d_out = ref->memo2.as<double>();
    uint8_t* d_keep = reinterpret_cast<uint8_t*>(d_out + 3 * n);
    if (n > 0) {
        k_clean_lod<<<nblk(n, 256), 256, 0, ref->stream>>>(d_ll, n, n_set, min_lod, d_out, d_out + n, d_out + 2 * n, d_keep);
        ref->stats.n_launch++;
        e = cudaGetLastError();
        if (e != cudaSuccess) return ref->cuda_fail(e);
    }
    double* dst[3] = {ref_ll, bg_ll, lod};
    for (int k = 0; k < 3 && n > 0; ++k)
        if (dst[k]) {
            e = cudaMemcpyAsync(dst[k], d_out + k * n, n * 8, cudaMemcpyDeviceToHost, ref->stream);
            if (e != cudaSuccess) return ref->cuda_fail(e);
        }
    if (keep && n > 0) {
        e = cudaMemcpyAsync(keep, d_keep, n, cudaMemcpyDeviceToHost, ref->stream);
        if (e != cudaSuccess) return ref->cuda_fail(e);
    }
    return stats_end(ref);
}

int clean_check(msg_ctx* ref, msg_ctx* bg, const msg_read_batch* fwd, const msg_mem_params* params) {
    if (!ref || !bg || !fwd || !params) return MSG_EINVAL;
    if (ref == bg) return ref->fail(MSG_EINVAL, "reference and background contexts must differ");
    if (!ref->idx.loaded || !bg->idx.loaded) return ref->fail(MSG_ESTATE, "no index loaded");
    if (ref->device != bg->device) return ref->fail(MSG_EINVAL, "contexts on different devices");
    if (check_mem_params(params) != MSG_OK) return ref->fail(MSG_EINVAL, "bad MEM parameters");
    if (fwd->n_reads < 0 || fwd->n_reads > INT32_MAX) return ref->fail(MSG_EINVAL, "bad read count");
    return MSG_OK;
}

}  // namespace

extern "C" void msg_mem_params_default(msg_mem_params* p) {
    if (!p) return;
    p->min_len = 17;       // SMEM::MIN_LENGTH (src/SMEM.h:204), msgseqtk-clean --min-seed
    p->max_evalue = 0.01;  // DEFAULT_MAX_EVALUE (src/msgseqtk-clean.cpp:52)
}

extern "C" int msg_mem_batch(msg_ctx* ctx, const msg_read_batch* reads, const msg_mem_params* params, double* loglik,
                             int32_t* n_mem, int64_t* rows, int64_t row_cap, int64_t* n_rows) {
    if (!ctx || !reads || !params) return MSG_EINVAL;
    if (!ctx->idx.loaded) return ctx->fail(MSG_ESTATE, "no index loaded");
    if (check_mem_params(params) != MSG_OK) return ctx->fail(MSG_EINVAL, "bad MEM parameters");
    if (rows && (!n_rows || row_cap < 0)) return MSG_EINVAL;
    const int64_t n = reads->n_reads;
    if (n < 0 || n > INT32_MAX) return ctx->fail(MSG_EINVAL, "bad read count");
    msg::DeviceGuard dg_(ctx->device);
    if (!dg_.ok) return ctx->fail(MSG_ECUDA, "cudaSetDevice");
    const msg_read_batch* sets[1] = {reads};
    Set dev[1];
    int rc = upload_sets(ctx, sets, 1, dev);
    if (rc != MSG_OK) return rc;
    // each kept MEM spans at least max(min_len, 2) of the L + 1 positions
    // [0, L] and kept MEMs do not overlap, so a read needs at most
    // (L + 1) / max(min_len, 2) rows
    std::vector<int64_t> slot;
    int64_t* d_slot = nullptr;
    int64_t* d_rows = nullptr;
    cudaError_t e;
    if (rows) {
        slot.resize(n + 1);
        const int64_t w = std::max<int64_t>(params->min_len, 2);
        slot[0] = 0;
        for (int64_t i = 0; i < n; ++i) slot[i + 1] = slot[i] + (reads->off[i + 1] - reads->off[i] + 1) / w;
        e = ctx->memrows.ensure(slot[n] * 12 * 8 + 64);  // slotted rows, then the dense copy
        if (e == cudaSuccess) e = ctx->memslot.ensure((n + 1) * 16 + 64);
        if (e != cudaSuccess) return ctx->cuda_fail(e);
        d_slot = ctx->memslot.as<int64_t>();
        d_rows = ctx->memrows.as<int64_t>();
        e = cudaMemcpyAsync(d_slot, slot.data(), (n + 1) * 8, cudaMemcpyHostToDevice, ctx->stream);
        if (e != cudaSuccess) return ctx->cuda_fail(e);
    }
    stats_begin(ctx, n);
    double* d_ll;
    int32_t* d_cnt;
    rc = mem_launch(ctx, nullptr, dev, 1, n, params, d_slot, d_rows, &d_ll, &d_cnt);
    if (rc != MSG_OK) return rc;
    cudaEventRecord(ctx->ev[1], ctx->stream);
    std::vector<int32_t> cnt(n);
    if (n > 0) {
        e = cudaMemcpyAsync(cnt.data(), d_cnt, n * 4, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess && loglik) e = cudaMemcpyAsync(loglik, d_ll, n * 8, cudaMemcpyDeviceToHost, ctx->stream);
        if (e != cudaSuccess) return ctx->cuda_fail(e);
    }
    rc = stats_end(ctx);
    if (rc != MSG_OK) return rc;
    int64_t total = 0;
    for (int64_t i = 0; i < n; ++i) total += cnt[i];
    ctx->stats.n_smem = total;
    if (n_mem && n > 0) std::memcpy(n_mem, cnt.data(), n * 4);
    if (n_rows) *n_rows = total;
    if (!rows) return MSG_OK;
    if (total > row_cap) return ctx->fail(MSG_EINVAL, "MEM rows exceed row_cap");
    if (total == 0) return MSG_OK;
    std::vector<int64_t> dst(n + 1, 0);
    for (int64_t i = 0; i < n; ++i) dst[i + 1] = dst[i] + cnt[i];
    int64_t* d_dst = d_slot + (n + 1);
    int64_t* d_dense = d_rows + slot[n] * 6;
    e = cudaMemcpyAsync(d_dst, dst.data(), (n + 1) * 8, cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) return ctx->cuda_fail(e);
    // the dense rows need total*6 int64 after the slotted ones: slot[n] >= total
    k_compact_rows<<<nblk(n * 32, 256), 256, 0, ctx->stream>>>(d_slot, d_dst, d_cnt, n, d_rows, d_dense);
    ctx->stats.n_launch++;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(rows, d_dense, total * 48, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    return e == cudaSuccess ? MSG_OK : ctx->cuda_fail(e);
}

extern "C" int msg_clean_batch(msg_ctx* ref, msg_ctx* bg, const msg_read_batch* fwd, const msg_read_batch* rev,
                               const msg_mem_params* params, double min_lod, double* ref_loglik, double* bg_loglik,
                               double* lod, uint8_t* keep) {
    int rc = clean_check(ref, bg, fwd, params);
    if (rc != MSG_OK) return rc;
    if (rev && rev->n_reads != fwd->n_reads) return ref->fail(MSG_EINVAL, "mate batches differ in size");
    msg::DeviceGuard dg_(ref->device);
    if (!dg_.ok) return ref->fail(MSG_ECUDA, "cudaSetDevice");
    const msg_read_batch* sets[2] = {fwd, rev};
    Set dev[2];
    const int n_set = rev ? 2 : 1;
    rc = upload_sets(ref, sets, n_set, dev);
    if (rc != MSG_OK) return rc;
    return clean_impl(ref, bg, dev, n_set, fwd->n_reads, params, min_lod, ref_loglik, bg_loglik, lod, keep);
}

extern "C" int msg_clean_batch_device(msg_ctx* ref, msg_ctx* bg, const msg_read_batch* dev_fwd,
                                      const msg_read_batch* dev_rev, const msg_mem_params* params, double min_lod,
                                      double* ref_loglik, double* bg_loglik, double* lod, uint8_t* keep) {
    int rc = clean_check(ref, bg, dev_fwd, params);
    if (rc != MSG_OK) return rc;
    if (dev_rev && dev_rev->n_reads != dev_fwd->n_reads) return ref->fail(MSG_EINVAL, "mate batches differ in size");
    if (dev_fwd->n_reads > 0 && (!dev_fwd->seq || !dev_fwd->off)) return MSG_EINVAL;
    if (dev_rev && dev_rev->n_reads > 0 && (!dev_rev->seq || !dev_rev->off)) return MSG_EINVAL;
    msg::DeviceGuard dg_(ref->device);
    if (!dg_.ok) return ref->fail(MSG_ECUDA, "cudaSetDevice");
    Set dev[2] = {{dev_fwd->seq, dev_fwd->off}, {dev_rev ? dev_rev->seq : nullptr, dev_rev ? dev_rev->off : nullptr}};
    return clean_impl(ref, bg, dev, dev_rev ? 2 : 1, dev_fwd->n_reads, params, min_lod, ref_loglik, bg_loglik, lod,
                      keep);
}
