// Read-mapping pipeline on sm_100a: SMEM seeding -> seed selection -> locate ->
// redundant-seed removal -> DFS chaining -> seed-guided affine DP + traceback.
//
// Every stage reproduces the reference's results exactly (integer/byte work;
// the double-precision SMEM log-likelihood sums are made in the reference's
// order with round-to-nearest adds). Kernel-to-reference mapping:
//   k_smem      SMEM_LIST::findAllSMEMS / findFwdBackSMEMS / findBackFwdSMEMS (SMEM.cpp:64-215)
//   k_select    SMEM_LIST::findSeeds sort + maxNSeed cut (SMEM.cpp:271-300)
//   k_locate    SMEM::getSeeds (SMEM.cpp:244-269) with FMDIndex::accessSA and MetaGenome::getTid/getLoc/getStrand
//   k_dedup     SeedPair::removeRedundant (SeedPair.cpp:71-88)
//   k_chain     SeedChain::getChains / dfsSeeds (SeedChain.cpp:40-73)
//   k_dp        Alignment ctor window, calculateScores(chain), backTraceNW/SW (Alignment.cpp:46-276)
//   k_cigar     Alignment::getAlnCigar (Alignment.cpp:278-303)
#include "map_kernels.cuh"
#include "smem_thread.cuh"
#include "band.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

#include <cub/cub.cuh>

#include "msg_ctx.cuh"

using namespace msg;

namespace {

int64_t nblk(int64_t n, int t) { return (n + t - 1) / t; }

}  // namespace

namespace msg {

// Largest double ll with n * exp(ll) <= max_e (the e-value test of
// SMEM::evalue, SMEM.h:102-110, made with the host's own exp exactly as the
// reference makes it). The predicate is monotone in ll, so SMEM stages compare
// the log-likelihood sum against this threshold instead of calling exp.
uint64_t dkey(double d) {
    uint64_t u;
    std::memcpy(&u, &d, 8);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
double dval(uint64_t k) {
    uint64_t u = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
    double d;
    std::memcpy(&d, &u, 8);
    return d;
}
bool evalue_ok(int64_t n, double ll, double max_e) { return (double)n * std::exp(ll) <= max_e; }

int evalue_threshold(int64_t n, double max_e, double* thr, int* all) {
    if (std::isnan(max_e) || max_e < 0) return MSG_EINVAL;
    if (std::isinf(max_e)) { *all = 1; *thr = std::numeric_limits<double>::infinity(); return MSG_OK; }
    *all = 0;
    uint64_t lo = dkey(-std::numeric_limits<double>::infinity());
    uint64_t hi = dkey(std::numeric_limits<double>::infinity());
    if (!evalue_ok(n, dval(lo), max_e)) { *thr = -std::numeric_limits<double>::infinity(); return MSG_OK; }
    while (hi - lo > 1) {  // invariant: ok(lo), !ok(hi)
        const uint64_t mid = lo + (hi - lo) / 2;
        if (evalue_ok(n, dval(mid), max_e)) lo = mid; else hi = mid;
    }
    // monotonicity check around the threshold
    for (uint64_t d = 1; d <= 4096; d <<= 1) {
        if (lo >= d && !evalue_ok(n, dval(lo - d), max_e)) return MSG_EINTERNAL;
        if (!evalue_ok(n, dval(lo + d), max_e) == false) return MSG_EINTERNAL;
    }
    *thr = dval(lo);
    return MSG_OK;
}

}  // namespace msg

namespace {

template <typename T>
cudaError_t scan_excl(msg_ctx* ctx, const T* in, T* out, int64_t n, DevBuf& tmpb) {
    size_t tb = 0;
    cudaError_t e = cub::DeviceScan::ExclusiveSum(nullptr, tb, in, out, n, ctx->stream);
    if (e != cudaSuccess) return e;
    e = tmpb.ensure(tb);
    if (e != cudaSuccess) return e;
    return cub::DeviceScan::ExclusiveSum(tmpb.p, tb, in, out, n, ctx->stream);
}

// exclusive scan of n values into n+1 offsets, the total copied to host
// memory `total` (pinned: the copy stays asynchronous) without waiting
template <typename T>
cudaError_t offsets_async(msg_ctx* ctx, T* cnt_with_room, int64_t n, T* off, DevBuf& tmpb, T* total) {
    cudaError_t e = cudaMemsetAsync(cnt_with_room + n, 0, sizeof(T), ctx->stream);
    if (e != cudaSuccess) return e;
    e = scan_excl(ctx, cnt_with_room, off, n + 1, tmpb);
    if (e != cudaSuccess) return e;
    return cudaMemcpyAsync(total, off + n, sizeof(T), cudaMemcpyDeviceToHost, ctx->stream);
}

// exclusive scan of n values into n+1 offsets; returns the total
template <typename T>
cudaError_t offsets(msg_ctx* ctx, T* cnt_with_room, int64_t n, T* off, DevBuf& tmpb, T* total) {
    cudaError_t e = offsets_async(ctx, cnt_with_room, n, off, tmpb, total);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(ctx->stream);
}

__global__ void k_i32_to_i64(const int32_t* __restrict__ a, int64_t* __restrict__ b, int64_t n) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) b[i] = a[i];
}

__global__ void k_read_len(const int64_t* __restrict__ off, int64_t n, int64_t* __restrict__ len,
                           unsigned long long* __restrict__ mx) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    unsigned long long l = 0;
    if (i < n) {
        const int64_t v = off[i + 1] - off[i];
        len[i] = v;
        l = v < 0 ? 0 : (unsigned long long)v;
    }
    for (int o = 16; o > 0; o >>= 1) l = max(l, __shfl_xor_sync(0xffffffffu, l, o));  // one atomic per warp
    if ((threadIdx.x & 31) == 0 && l > 0) atomicMax(mx, l);
}

// One warp per read.
__global__ void k_smem_read(const int64_t* __restrict__ smem_off, int64_t n_reads, int32_t* __restrict__ smem_read) {
    const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (r >= n_reads) return;
    for (int64_t k = smem_off[r] + (threadIdx.x & 31); k < smem_off[r + 1]; k += 32) smem_read[k] = (int32_t)r;
}

// (logP bits, size) of the SMEM rows of the reads in `list`, packed read by
// read at pack_off (one warp per listed read).
__global__ void k_gather_rank_keys(const int64_t* __restrict__ list, int64_t n, const int64_t* __restrict__ smem_off,
                                   const int64_t* __restrict__ pack_off, const int64_t* __restrict__ smem,
                                   int64_t* __restrict__ out) {
    const int64_t f = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (f >= n) return;
    const int64_t r = list[f], a = smem_off[r], b = smem_off[r + 1], o = pack_off[f];
    for (int64_t k = a + (threadIdx.x & 31); k < b; k += 32) {
        out[2 * (o + k - a)] = smem[6 * k + 5];
        out[2 * (o + k - a) + 1] = smem[6 * k + 4];
    }
}

// The selection flags of the listed reads' rows back to their places.
__global__ void k_scatter_sel(const int64_t* __restrict__ list, int64_t n, const int64_t* __restrict__ smem_off,
                              const int64_t* __restrict__ pack_off, const uint8_t* __restrict__ psel,
                              uint8_t* __restrict__ sel) {
    const int64_t f = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (f >= n) return;
    const int64_t r = list[f], a = smem_off[r], b = smem_off[r + 1], o = pack_off[f];
    for (int64_t k = a + (threadIdx.x & 31); k < b; k += 32) sel[k] = psel[o + k - a];
}

__global__ void k_gather_off(const int64_t* __restrict__ smem_off, const int64_t* __restrict__ smem_seed_off,
                             int64_t n_reads, int64_t* __restrict__ read_seed_off) {
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r > n_reads) return;
    read_seed_off[r] = smem_seed_off[smem_off[r]];
}

__global__ void k_aln_cig(msg_aln* __restrict__ aln, const int64_t* __restrict__ cig_off, int64_t n) {
    const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= n) return;
    aln[c].cigar_off = cig_off[c];
    aln[c].n_cigar = (int32_t)(cig_off[c + 1] - cig_off[c]);
    aln[c].pad = 0;
}

__global__ void k_keep64(const uint8_t* __restrict__ keep, int64_t n, int64_t* __restrict__ out) {
    const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c < n) out[c] = keep[c];
}

__global__ void k_compact_aln(const msg_aln* __restrict__ aln, const uint8_t* __restrict__ keep,
                              const int64_t* __restrict__ kidx, int64_t n, msg_aln* __restrict__ out,
                              int64_t* __restrict__ map) {
    const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= n || !keep[c]) return;
    out[kidx[c]] = aln[c];
    map[kidx[c]] = c;
}

// off[i] -= base for i < n (host offsets rebased to the batch's first read).
__global__ void k_rebase(int64_t* __restrict__ off, int64_t n, int64_t base) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) off[i] -= base;
}

struct Timer {
    msg_ctx* ctx;
    int k = 0;
    void mark() { cudaEventRecord(ctx->ev[k++], ctx->stream); }
    void mark_at(int i) { cudaEventRecord(ctx->ev[i], ctx->stream); }  // the DP stage's inner marks (6, 7)
    float ms(int a, int b) {
        float t = 0;
        cudaEventElapsedTime(&t, ctx->ev[a], ctx->ev[b]);
        return t;
    }
};

// Band assignment, DP class and sort key of chains c0 .. c0 + n, then the
// chains sorted by (class, area descending) into `sorted`; class sizes are
// added to counts[0 .. kDpClasses). keybuf holds 2n uint32 (keys in, out).
cudaError_t dp_sort(msg_ctx* ctx, int64_t c0, int64_t n, const int4* geo, const int64_t* area, const float* feat,
                    int mode, int fixed_w, const __nv_bfloat16* wts, const float* nrm, int8_t* band,
                    unsigned long long* counts, int64_t* keybuf, int64_t* ids, int64_t* sorted, msg_map_stats& S) {
    cudaStream_t st = ctx->stream;
    uint32_t* key = reinterpret_cast<uint32_t*>(keybuf);
    uint32_t* key2 = key + n;
    S.n_launch++, k_band_assign<<<nblk(n, 128), 128, 0, st>>>(c0, n, geo, area, feat, mode, fixed_w, wts, nrm,
                                                              ctx->dp_small_area, ctx->dp_warp_area, band, counts,
                                                              key);
    S.n_launch++, k_iota<<<nblk(n, 256), 256, 0, st>>>(c0, n, ids);
    cudaError_t e = cudaGetLastError();
    size_t tb = 0;
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(nullptr, tb, key, key2, ids, sorted, (int)n, 0, kKeyBits, st);
    if (e == cudaSuccess) e = ctx->misc.ensure(tb);
    if (e == cudaSuccess)
        e = cub::DeviceRadixSort::SortPairs(ctx->misc.p, tb, key, key2, ids, sorted, (int)n, 0, kKeyBits, st);
    return e;
}

// Blocks of a thread-per-chain DP launch: as many as are resident at once
// (the warps take chains from the launch's work counter until none is left),
// and no more than the chains need.
template <typename F>
int resident_blocks(msg_ctx* ctx, F kernel, int threads, int64_t n_max) {
    int bps = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kernel, threads, 0) != cudaSuccess || bps < 1) bps = 1;
    return (int)std::max<int64_t>(1, std::min<int64_t>(nblk(n_max, threads), (int64_t)ctx->num_sms * bps));
}

template <int K>
void launch_stripe(msg_ctx* ctx, const DpArgs& a, bool band, int64_t n_max, cudaStream_t st) {
    if (ctx->dp_stripe_blocks == 3) {
        if (band) k_dp_stripe<K, true, 3><<<resident_blocks(ctx, k_dp_stripe<K, true, 3>, kStripeThreads, n_max), kStripeThreads, 0, st>>>(a);
        else k_dp_stripe<K, false, 3><<<resident_blocks(ctx, k_dp_stripe<K, false, 3>, kStripeThreads, n_max), kStripeThreads, 0, st>>>(a);
    } else {
        if (band) k_dp_stripe<K, true, 4><<<resident_blocks(ctx, k_dp_stripe<K, true, 4>, kStripeThreads, n_max), kStripeThreads, 0, st>>>(a);
        else k_dp_stripe<K, false, 4><<<resident_blocks(ctx, k_dp_stripe<K, false, 4>, kStripeThreads, n_max), kStripeThreads, 0, st>>>(a);
    }
}

// One DP launch: over class `cls` of the class-sorted list a.list when
// cls >= 0; with cls < 0 over a.list[0 .. *a.n_list) with the kernel of class
// -cls - 1 (the fallback recomputations). n_max bounds the chains it may get.
// The thread kernels (row by row, stripes) take their chains 32 at a time
// from the class's work counter (class order: the largest first), the warp
// kernels loop over theirs (grid-stride).
void launch_dp(msg_ctx* ctx, DpArgs a, int cls, int64_t n_max, msg_map_stats& S, cudaStream_t st = nullptr) {
    const int kind = cls >= 0 ? cls : -cls - 1;
    a.cls = cls >= 0 ? cls : -1;
    a.queue = const_cast<unsigned long long*>(a.cls_n) + kCtrQueue + kind;  // the counter block is the stage's own
    if (!st) st = ctx->stream;
    S.n_launch++;
    if (kind == kDpSmall) {
        k_dp_small<<<resident_blocks(ctx, k_dp_small, 128, n_max), 128, 0, st>>>(a);
    } else if (kind == kDpStripe || kind == kDpStripeBand) {
        const bool band = kind == kDpStripeBand;
        if (ctx->dp_k == 8) launch_stripe<8>(ctx, a, band, n_max, st);
        else if (ctx->dp_k == 32) launch_stripe<32>(ctx, a, band, n_max, st);
        else launch_stripe<16>(ctx, a, band, n_max, st);
    } else {
        const int g = (int)std::min<int64_t>(nblk(n_max * 32, kDpWarps * 32), (int64_t)ctx->num_sms * 12);
        if (kind == kDpWarpBand) k_dp<true><<<g, kDpWarps * 32, 0, st>>>(a);
        else k_dp<false><<<g, kDpWarps * 32, 0, st>>>(a);
    }
}

int check_params(const msg_map_params* p, DpParams* dp) {
    if (!p) return MSG_EINVAL;
    if (p->min_len < 1 || p->max_nseed < 1 || (p->mode != 0 && p->mode != 1)) return MSG_EINVAL;
    if (std::isnan(p->max_evalue) || p->max_evalue < 0) return MSG_EINVAL;
    const double v[4] = {p->match, p->mismatch, p->gap_open, p->gap_ext};
    int32_t iv[4];
    for (int k = 0; k < 4; ++k) {
        if (!(v[k] >= 0 && v[k] <= 1 << 20) || std::floor(v[k]) != v[k]) return MSG_EUNSUPPORTED;
        iv[k] = (int32_t)v[k];
    }
    dp->match = iv[0]; dp->mismatch = iv[1]; dp->gap_o = iv[2]; dp->gap_e = iv[3]; dp->mode = p->mode;
    if (std::isnan(p->min_score_rate) || p->min_score_rate > 1) return MSG_EINVAL;
    if (p->band_mode < 0 || p->band_mode > 2) return MSG_EINVAL;
    if (p->band_mode == 1 && (p->band_w < 0 || p->band_w > 31)) return MSG_EINVAL;
    return MSG_OK;
}

}  // namespace

extern "C" void msg_map_params_default(msg_map_params* p) {
    if (!p) return;
    p->min_len = 17;
    p->max_evalue = 0.01;
    p->max_nseed = 500;
    p->mode = 0;
    p->match = 1;
    p->mismatch = 3;
    p->gap_open = 5;
    p->gap_ext = 2;
    p->min_score_rate = -1.0;
    p->band_mode = 0;
    p->band_w = 15;
}

namespace {
// Entry and exit points of map_impl for the per-stage calls: the pipeline
// starts at stage `first` from the caller's host arrays and stops after stage
// `last`, returning that stage's results in the caller's host arrays.
enum MapStage : int { kStSmem = 0, kStLocate = 1, kStChain = 2, kStAlign = 3 };
struct StageIO {
    int first = kStSmem, last = kStAlign;
    // inputs: SMEM rows (first == kStLocate), seeds (first >= kStChain), chains (first == kStAlign)
    const int64_t* smem = nullptr;
    const int64_t* smem_off = nullptr;
    const int64_t* seed = nullptr;
    const int64_t* seed_off = nullptr;
    const int32_t* chain_seed = nullptr;
    const int64_t* chain_seed_off = nullptr;
    const int64_t* read_chain_off = nullptr;
    // outputs: rows of 6 int64 (SMEMs or seeds) or chains
    int64_t* rows = nullptr;
    int64_t rows_cap = 0;
    int64_t* rows_off = nullptr;
    int64_t* n_rows = nullptr;
    int32_t* o_chain_seed = nullptr;
    int64_t o_chain_seed_cap = 0;
    int64_t* o_chain_seed_off = nullptr;
    int64_t o_chain_cap = 0;
    int64_t* o_read_chain_off = nullptr;
    int64_t* o_n_chain = nullptr;
    int64_t* o_n_chain_seed = nullptr;
};

struct BandCollect {
    float* feat;
    int32_t* label;
    int64_t cap;
    int64_t* n_chain;
};
}  // namespace

static int map_impl(msg_ctx* ctx, const uint8_t* d_seq, const int64_t* d_off, int64_t n_reads,
                    const msg_map_params* params, msg_aln_out* out, msg_stage_dump* dump,
                    const BandCollect* collect = nullptr, const StageIO* io = nullptr) {
    DpParams dpp;
    int rc = check_params(params, &dpp);
    if (rc != MSG_OK) return ctx->fail(rc, rc == MSG_EUNSUPPORTED ? "score scheme must be non-negative integers" : "bad mapping parameters");
    if (params->band_mode == 2 && !ctx->band_loaded) return ctx->fail(MSG_ESTATE, "band_mode 2 needs a band model");
    const IndexImage& im = ctx->idx;
    const IndexDev& ix = im.dev;
    double thr = 0;
    int thr_all = 0;
    rc = evalue_threshold(ix.n, params->max_evalue, &thr, &thr_all);
    if (rc != MSG_OK) return ctx->fail(rc, "e-value threshold");
    cudaStream_t st = ctx->stream;
    msg_map_stats& S = ctx->stats;
    std::memset(&S, 0, sizeof(S));
    S.n_reads = n_reads;
    Timer tm{ctx};
    auto t_host0 = std::chrono::steady_clock::now();
    tm.mark();  // 0
#define CK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) return ctx->cuda_fail(e_); } while (0)
    DevBuf& misc = ctx->misc;
    CK(ctx->status.ensure(128));
    uint32_t* d_status = ctx->status.as<uint32_t>();
    unsigned long long* d_ctr = reinterpret_cast<unsigned long long*>(d_status + 4);
    CK(cudaMemsetAsync(d_status, 0, 128, st));

    // read lengths
    CK(ctx->rcount.ensure((n_reads + 1) * sizeof(int64_t) * 8 + 64));
    int64_t* d_rlen = ctx->rcount.as<int64_t>();
    int64_t* d_cnt64 = d_rlen + (n_reads + 1);          // scratch counts (n+1)
    int64_t* d_smem_off = d_cnt64 + (n_reads + 1);      // n+1
    int64_t* d_read_seed_off = d_smem_off + (n_reads + 1);
    int64_t* d_nchain = d_read_seed_off + (n_reads + 1);
    int64_t* d_nidx = d_nchain + (n_reads + 1);
    int64_t* d_chain_off = d_nidx + (n_reads + 1);
    int64_t* d_idx_off = d_chain_off + (n_reads + 1);
    unsigned long long h_maxlen = 0;
    if (n_reads > 0) {
        uint32_t h_codes = 0;
        S.n_launch++, k_check_codes<<<ctx->num_sms * 4, 256, 0, st>>>(d_seq, d_off, n_reads, d_status);
        S.n_launch++, k_read_len<<<nblk(n_reads, 256), 256, 0, st>>>(d_off, n_reads, d_rlen, d_ctr + 2);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(&h_maxlen, d_ctr + 2, 8, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(&h_codes, d_status, 4, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (h_codes & kErrCodes) return ctx->fail(MSG_EINVAL, "read bytes must be nt16 codes (0..15)");
    }
    const int64_t Lmax = (int64_t)h_maxlen;
    const int first = io ? io->first : (int)kStSmem, last = io ? io->last : (int)kStAlign;
    int64_t h_nsmem = 0;
    int64_t* d_smem = nullptr;          // dense SMEM rows
    int64_t* d_smem_seed_cnt = nullptr; // n_smem + 1
    int64_t* d_smem_seed_off = nullptr; // n_smem + 1
    int32_t* d_smem_read = nullptr;
    int32_t* d_fill = nullptr;
    uint8_t* d_sel = nullptr;
    auto setup_sel = [&]() -> cudaError_t {
        const cudaError_t e = ctx->sel.ensure((h_nsmem + 1) * (48 + 1 + 4 + 8 + 8 + 4) + 64);
        if (e != cudaSuccess) return e;
        d_smem = ctx->sel.as<int64_t>();
        d_smem_seed_cnt = d_smem + 6 * h_nsmem;
        d_smem_seed_off = d_smem_seed_cnt + (h_nsmem + 1);
        d_smem_read = reinterpret_cast<int32_t*>(d_smem_seed_off + (h_nsmem + 1));
        d_fill = d_smem_read + (h_nsmem + 1);
        d_sel = reinterpret_cast<uint8_t*>(d_fill + (h_nsmem + 1));
        return cudaSuccess;
    };
    if (first == kStSmem) {
    // ---------------- SMEMs ----------------
    // Reads are bucketed by length: up to kThreadMaxLen bp one thread per read
    // (k_smem_thread), longer reads one warp per read with lanes over the
    // candidate list (k_smem); both launches share the batch. Each read's SMEM
    // rows go to its own slot, cap rows per 150 bases (at least cap), so long
    // reads get room in proportion (cap starts from the largest a batch of
    // this context needed). The thread kernel keeps at most kThreadPrev
    // candidates per read so that all candidate lists stay in L2; a read
    // whose list outgrows it is abandoned and mapped again by the warp
    // kernel.
    constexpr int64_t kThreadPrev = 48;
    constexpr int64_t kThreadMaxLen = 254;
    const int threads = 256;
    const int blocks = ctx->num_sms * 8;
    const int64_t n_warps = (int64_t)blocks * threads / 32;
    CK(ctx->rlist.ensure((n_reads + 1) * 8 * 5 + 64));
    int64_t* d_short = ctx->rlist.as<int64_t>();
    int64_t* d_long = d_short + (n_reads + 1);
    int64_t* d_slot = d_long + (n_reads + 1);        // slot rows per read (n + 1)
    int64_t* d_slot_off = d_slot + (n_reads + 1);    // slot offsets (n + 1)
    int64_t* d_ovf = d_slot_off + (n_reads + 1);     // reads the thread kernel abandoned
    unsigned long long h_split[2] = {0, 0};
    if (n_reads > 0) {
        CK(cudaMemsetAsync(d_ctr + 4, 0, 16, st));
        S.n_launch++, k_split_len<<<nblk(n_reads, 256), 256, 0, st>>>(d_rlen, n_reads, kThreadMaxLen, d_short, d_long,
                                                                      d_ctr + 4);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(h_split, d_ctr + 4, 16, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }
    bool thread_path = h_split[0] > 0;
    int64_t cap = std::max<int64_t>(16, ctx->smem_cap);
    // the warp kernel over `n` reads of `list` (all reads when null)
    auto run_warp = [&](const int64_t* list, int64_t n) -> cudaError_t {
        const int64_t pv_cap = Lmax + 2;
        cudaError_t e = ctx->prevw.ensure(n_warps * pv_cap * (4 + 8 + 8 + 8 + 8) + 64);
        if (e != cudaSuccess) return e;
        SmemArgs sa{};
        sa.seq = d_seq; sa.off = d_off; sa.n_reads = n; sa.min_len = params->min_len;
        sa.thr = thr; sa.thr_all = thr_all;
        for (int b = 0; b < 16; ++b) sa.llk[b] = im.llk[b];
        sa.out = ctx->smem.as<int64_t>(); sa.cap = cap; sa.out_off = d_slot_off;
        sa.list = list;
        sa.count = ctx->smem_cnt.as<int32_t>();
        char* pv = ctx->prevw.as<char>();
        sa.pv_p = reinterpret_cast<int64_t*>(pv);
        sa.pv_q = sa.pv_p + n_warps * pv_cap;
        sa.pv_s = sa.pv_q + n_warps * pv_cap;
        sa.pv_lp = reinterpret_cast<double*>(sa.pv_s + n_warps * pv_cap);
        sa.pv_pos = reinterpret_cast<int32_t*>(sa.pv_lp + n_warps * pv_cap);
        sa.pv_cap = pv_cap;
        sa.work = d_ctr + 3;
        sa.n_ext = d_ctr + 1;
        sa.status = d_status;
        e = cudaMemsetAsync(d_ctr + 3, 0, 8, st);
        if (e != cudaSuccess) return e;
        S.n_launch++, k_smem<<<blocks, threads, 0, st>>>(sa, ix);
        return cudaGetLastError();
    };
    for (int attempt = 0; attempt < 4; ++attempt) {
        int64_t h_rows = 0;
        if (n_reads > 0) S.n_launch++, k_slot_rows<<<nblk(n_reads, 256), 256, 0, st>>>(d_rlen, n_reads, cap, d_slot);
        CK(offsets(ctx, d_slot, n_reads, d_slot_off, misc, &h_rows));
        CK(ctx->smem.ensure((size_t)std::max<int64_t>(1, h_rows) * 48));
        CK(ctx->smem_cnt.ensure((n_reads + 1) * sizeof(int32_t)));
        CK(cudaMemsetAsync(d_ctr, 0, 8 * 4, st));
        CK(cudaMemsetAsync(d_ctr + 7, 0, 24, st));
        CK(cudaMemsetAsync(d_status, 0, 4, st));
        // short reads on the thread kernel
        if (thread_path) {
            // one read per thread (ctx->smem_variant 0; 5 and 6: registers
            // sized for 6 and 8 resident blocks), two per thread (1 and 2:
            // each thread keeps two extensions' loads in flight), or one per
            // thread with a pass's entries extended up to 4 (3) or 2 (4) at a
            // time
            const int var = ctx->smem_variant;
            const bool pair = var == 1 || var == 2;
            int bps = 0;
            if (var == 1) CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_smem_thread2<4>, 128, 0));
            else if (var == 2) CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_smem_thread2<3>, 128, 0));
            else if (var == 3) CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_smem_pass<4, 4>, 128, 0));
            else if (var == 4) CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_smem_pass<2, 5>, 128, 0));
            else if (var == 5) CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_smem_thread<6, false>, 128, 0));
            else if (var == 6) CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_smem_thread<8, false>, 128, 0));
            // variant 7: variant 0 with the fast-forward over unique matches
            else if (ctx->smem_ff) CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_smem_thread<5, true>, 128, 0));
            else CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_smem_thread<5, false>, 128, 0));
            const int64_t n_thr = (int64_t)ctx->num_sms * std::max(1, bps) * 128;
            const int64_t pv_cap = kThreadPrev;
            CK(ctx->prev.ensure((pair ? 2 : 1) * n_thr * pv_cap * sizeof(PrevEntry) + 64));
            SmemThreadArgs ta{};
            for (int b = 0; b < 16; ++b) ta.llk[b] = im.llk[b];
            ta.seq = d_seq; ta.off = d_off; ta.n_reads = (int64_t)h_split[0]; ta.min_len = params->min_len;
            ta.thr = thr; ta.thr_all = thr_all;
            ta.llk_min = *std::min_element(im.llk, im.llk + 16);
            ta.llk_max = *std::max_element(im.llk, im.llk + 16);
            ta.out = ctx->smem.as<int64_t>(); ta.cap = cap; ta.out_off = d_slot_off; ta.list = d_short;
            ta.count = ctx->smem_cnt.as<int32_t>();
            ta.prev = ctx->prev.as<PrevEntry>(); ta.pv_cap = pv_cap;
            ta.work = d_ctr; ta.n_ext = d_ctr + 1; ta.status = d_status;
            ta.ovf_list = d_ovf; ta.ovf_n = d_ctr + 7;
            ta.n_ffx = d_ctr + 8;
            ta.n_ffs = d_ctr + 9;
            const bool ff = var == 0 && ctx->smem_ff && ix.text && ix.isa;
            if (var == 1) S.n_launch++, k_smem_thread2<4><<<n_thr / 128, 128, 0, st>>>(ta, ix);
            else if (var == 2) S.n_launch++, k_smem_thread2<3><<<n_thr / 128, 128, 0, st>>>(ta, ix);
            else if (var == 3) S.n_launch++, k_smem_pass<4, 4><<<n_thr / 128, 128, 0, st>>>(ta, ix);
            else if (var == 4) S.n_launch++, k_smem_pass<2, 5><<<n_thr / 128, 128, 0, st>>>(ta, ix);
            else if (var == 5) S.n_launch++, k_smem_thread<6, false><<<n_thr / 128, 128, 0, st>>>(ta, ix);
            else if (var == 6) S.n_launch++, k_smem_thread<8, false><<<n_thr / 128, 128, 0, st>>>(ta, ix);
            else if (ff) S.n_launch++, k_smem_thread<5, true><<<n_thr / 128, 128, 0, st>>>(ta, ix);
            else S.n_launch++, k_smem_thread<5, false><<<n_thr / 128, 128, 0, st>>>(ta, ix);
            CK(cudaGetLastError());
        }
        // long reads (all reads when no read is short) on the warp kernel
        const int64_t n_warp_reads = thread_path ? (int64_t)h_split[1] : n_reads;
        if (n_warp_reads > 0) CK(run_warp(thread_path ? d_long : nullptr, n_warp_reads));
        uint32_t h_status = 0;
        CK(cudaMemcpyAsync(&h_status, d_status, 4, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(ctx->hpin + 9, d_ctr + 7, 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (h_status & kErrInternal) return ctx->fail(MSG_EINTERNAL, "SMEM stage consistency check failed");
        if (h_status & 0x100u) {  // reads whose candidate list outgrew the thread kernel's cap
            const int64_t n_ovf = ctx->hpin[9];
            if (!thread_path || n_ovf <= 0) return ctx->fail(MSG_EINTERNAL, "SMEM candidate list overflow");
            S.n_smem_rerun += n_ovf;
            CK(cudaMemsetAsync(d_status, 0, 4, st));
            CK(run_warp(d_ovf, n_ovf));
            uint32_t h2 = 0;
            CK(cudaMemcpyAsync(&h2, d_status, 4, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            if (h2 & (kErrInternal | 0x100u)) return ctx->fail(MSG_EINTERNAL, "SMEM stage consistency check failed");
            h_status = (h_status & ~0x100u) | h2;
        }
        if (!(h_status & kErrOverflow)) break;
        if (attempt == 3) return ctx->fail(MSG_EINTERNAL, "SMEM output overflow after resizing");
        // rerun with a per-150-base capacity that fits every read's count
        std::vector<int32_t> cnt(n_reads);
        std::vector<int64_t> len(n_reads);
        CK(cudaMemcpy(cnt.data(), ctx->smem_cnt.p, n_reads * 4, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(len.data(), d_rlen, n_reads * 8, cudaMemcpyDeviceToHost));
        for (int64_t r = 0; r < n_reads; ++r) {
            const int64_t per = std::max<int64_t>(len[r], kSlotBases);
            cap = std::max<int64_t>(cap, ((int64_t)cnt[r] * kSlotBases + per - 1) / per);
        }
        S.smem_retries++;
    }
    // later batches start from this batch's capacity (bounded: rarer reads
    // that need more still get their rerun)
    ctx->smem_cap = std::min<int64_t>(std::max(ctx->smem_cap, cap), 256);
    // the extension counts arrive with the next synchronisation
    CK(cudaMemcpyAsync(ctx->hpin + 8, d_ctr + 1, 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(ctx->hpin + 10, d_ctr + 8, 16, cudaMemcpyDeviceToHost, st));
    if (n_reads > 0) S.n_launch++, k_i32_to_i64<<<nblk(n_reads, 256), 256, 0, st>>>(ctx->smem_cnt.as<int32_t>(), d_cnt64, n_reads);
    CK(offsets(ctx, d_cnt64, n_reads, d_smem_off, misc, &h_nsmem));
    S.n_ext = ctx->hpin[8];
    S.n_ext_ff = ctx->hpin[10];
    S.n_ff_steps = ctx->hpin[11];
    CK(setup_sel());
    if (n_reads > 0) {
        S.n_launch++, k_compact_smem<<<nblk(n_reads * 32, 256), 256, 0, st>>>(ctx->smem.as<int64_t>(), d_slot_off,
                                                                             ctx->smem_cnt.as<int32_t>(), d_smem_off,
                                                                             n_reads, d_smem);
        CK(cudaGetLastError());
    }
    } else if (first == kStLocate) {  // the caller's SMEM rows (checked by the entry point)
        const int64_t o0 = io->smem_off[0];
        h_nsmem = io->smem_off[n_reads] - o0;
        CK(setup_sel());
        std::vector<int64_t> so(n_reads + 1);
        for (int64_t r = 0; r <= n_reads; ++r) so[r] = io->smem_off[r] - o0;
        if (h_nsmem > 0) CK(cudaMemcpyAsync(d_smem, io->smem + 6 * o0, h_nsmem * 48, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(d_smem_off, so.data(), (n_reads + 1) * 8, cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
    } else {
        CK(setup_sel());
    }
    S.n_smem = h_nsmem;
    tm.mark();  // 1
    if (last == kStSmem) {  // SMEM rows and per-read offsets to the caller
        *io->n_rows = h_nsmem;
        if (h_nsmem > io->rows_cap) return ctx->fail(MSG_EINVAL, "output capacity too small");
        if (h_nsmem > 0) CK(cudaMemcpyAsync(io->rows, d_smem, h_nsmem * 48, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(io->rows_off, d_smem_off, (n_reads + 1) * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        S.ms_smem = tm.ms(0, 1);
        S.ms_total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_host0).count();
        return MSG_OK;
    }

    // ---------------- selection (maxNSeed) ----------------
    int32_t* d_hflag = reinterpret_cast<int32_t*>(d_cnt64);  // reuse scratch (n int32)
    if (first == kStLocate && h_nsmem > 0) CK(cudaMemsetAsync(d_sel, 1, h_nsmem, st));  // the caller chose them
    if (first == kStSmem && n_reads > 0) {
        CK(cudaMemsetAsync(d_ctr + 6, 0, 8, st));
        S.n_launch++, k_select<<<nblk(n_reads, 256), 256, 0, st>>>(d_smem, d_smem_off, n_reads, params->max_nseed, d_sel, d_hflag,
                                                                   d_ctr + 6);
        CK(cudaGetLastError());
        unsigned long long h_nflag = 0;
        CK(cudaMemcpyAsync(&h_nflag, d_ctr + 6, 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        std::vector<int64_t> flagged;
        if (h_nflag > 0) {  // only then are the per-read flags needed on the host
            std::vector<int32_t> hflag(n_reads);
            CK(cudaMemcpyAsync(hflag.data(), d_hflag, n_reads * 4, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            for (int64_t r = 0; r < n_reads; ++r) if (hflag[r]) flagged.push_back(r);
        }
        if (!flagged.empty()) {
            // SMEM_LIST::findSeeds (SMEM.cpp:275-291): std::sort by loglik (not
            // stable; same libstdc++ algorithm on the same emission order), then
            // locate until at least maxNSeed seeds. The flagged reads' (logP,
            // size) pairs come to the host in one copy, are sorted read by read
            // on host threads, and their selections go back in one copy.
            const int64_t nf = (int64_t)flagged.size();
            std::vector<int64_t> soff(n_reads + 1), poff(nf + 1, 0);
            CK(cudaMemcpy(soff.data(), d_smem_off, (n_reads + 1) * 8, cudaMemcpyDeviceToHost));
            for (int64_t f = 0; f < nf; ++f) poff[f + 1] = poff[f] + soff[flagged[f] + 1] - soff[flagged[f]];
            const int64_t F = poff[nf];
            CK(ctx->hsort.ensure((2 * nf + 1 + 2 * F) * 8 + F + 64));
            int64_t* d_flist = ctx->hsort.as<int64_t>();
            int64_t* d_poff = d_flist + nf;
            int64_t* d_pairs = d_poff + (nf + 1);
            uint8_t* d_psel = reinterpret_cast<uint8_t*>(d_pairs + 2 * F);
            std::vector<int64_t> pairs(2 * F);
            std::vector<uint8_t> psel(F, 0);
            CK(cudaMemcpyAsync(d_flist, flagged.data(), nf * 8, cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(d_poff, poff.data(), (nf + 1) * 8, cudaMemcpyHostToDevice, st));
            S.n_launch++, k_gather_rank_keys<<<nblk(nf * 32, 256), 256, 0, st>>>(d_flist, nf, d_smem_off, d_poff, d_smem,
                                                                                 d_pairs);
            CK(cudaGetLastError());
            CK(cudaMemcpyAsync(pairs.data(), d_pairs, 2 * F * 8, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            struct HS { double lp; int64_t size; int64_t k; };
            auto sort_range = [&](int64_t f0, int64_t f1) {
                std::vector<HS> v;
                for (int64_t f = f0; f < f1; ++f) {
                    const int64_t o = poff[f], m = poff[f + 1] - o;
                    v.clear();
                    for (int64_t k = 0; k < m; ++k) {
                        HS h;
                        std::memcpy(&h.lp, &pairs[2 * (o + k)], 8);
                        h.size = pairs[2 * (o + k) + 1];
                        h.k = k;
                        v.push_back(h);
                    }
                    std::sort(v.begin(), v.end(), [](const HS& x, const HS& y) -> bool { return x.lp < y.lp; });
                    int64_t got = 0;
                    for (const HS& h : v) {
                        psel[o + h.k] = 1;
                        got += h.size;
                        if (got >= params->max_nseed) break;
                    }
                }
            };
            const int64_t nth = std::min<int64_t>(std::max(1u, std::thread::hardware_concurrency()), 16);
            if (nf < 256 || nth < 2) {
                sort_range(0, nf);
            } else {
                std::vector<std::thread> pool;
                for (int64_t t = 0; t < nth; ++t) pool.emplace_back(sort_range, nf * t / nth, nf * (t + 1) / nth);
                for (auto& th : pool) th.join();
            }
            CK(cudaMemcpyAsync(d_psel, psel.data(), F, cudaMemcpyHostToDevice, st));
            S.n_launch++, k_scatter_sel<<<nblk(nf * 32, 256), 256, 0, st>>>(d_flist, nf, d_smem_off, d_poff, d_psel, d_sel);
            CK(cudaGetLastError());
            CK(cudaStreamSynchronize(st));  // psel and the lists leave scope
            S.host_sorted = nf;
        }
    }
    int64_t h_nseed_raw = 0;
    Seed* d_seeds = nullptr;
    Seed* d_seeds2 = nullptr;
    int32_t* d_ndedup = reinterpret_cast<int32_t*>(d_cnt64);  // n int32 (flags no longer needed)
    if (first <= kStLocate) {
    if (h_nsmem > 0) {
        S.n_launch++, k_seed_counts<<<nblk(h_nsmem, 256), 256, 0, st>>>(d_smem, d_sel, h_nsmem, d_smem_seed_cnt);
        CK(cudaGetLastError());
    }
    CK(offsets(ctx, d_smem_seed_cnt, h_nsmem, d_smem_seed_off, misc, &h_nseed_raw));
    if (n_reads > 0) {
        S.n_launch++, k_gather_off<<<nblk(n_reads + 1, 256), 256, 0, st>>>(d_smem_off, d_smem_seed_off, n_reads, d_read_seed_off);
        S.n_launch++, k_smem_read<<<nblk(n_reads * 32, 256), 256, 0, st>>>(d_smem_off, n_reads, d_smem_read);
        CK(cudaGetLastError());
    }

    // ---------------- locate ----------------
    CK(ctx->seeds.ensure((h_nseed_raw + 1) * sizeof(Seed)));
    CK(ctx->seeds2.ensure((h_nseed_raw + 1) * sizeof(Seed)));
    d_seeds = ctx->seeds.as<Seed>();
    d_seeds2 = ctx->seeds2.as<Seed>();
    S.n_sa = 2 * h_nseed_raw;
    if (h_nseed_raw > 0) {
        CK(cudaMemsetAsync(d_fill, 0, (h_nsmem + 1) * 4, st));
        const int64_t g = std::min<int64_t>(nblk(h_nseed_raw, 256), (int64_t)ctx->num_sms * 32);
        S.n_launch++, k_locate<<<g, 256, 0, st>>>(ix, d_smem, d_smem_seed_off, d_smem_read, d_off, h_nsmem, h_nseed_raw, d_fill,
                                    d_seeds, d_status);
        CK(cudaGetLastError());
    }
    } else {  // the caller's seeds (checked by the entry point), already without redundant ones
        const int64_t o0 = io->seed_off[0];
        h_nseed_raw = io->seed_off[n_reads] - o0;
        CK(ctx->seeds.ensure((h_nseed_raw + 1) * sizeof(Seed)));
        CK(ctx->seeds2.ensure((h_nseed_raw + 1) * sizeof(Seed)));
        d_seeds = ctx->seeds.as<Seed>();
        d_seeds2 = ctx->seeds2.as<Seed>();
        std::vector<Seed> hs(h_nseed_raw);
        for (int64_t k = 0; k < h_nseed_raw; ++k) {
            const int64_t* x = io->seed + 6 * (o0 + k);
            hs[k].from = (int32_t)x[0]; hs[k].to = (int32_t)x[1]; hs[k].start = x[2]; hs[k].end = x[3];
            hs[k].tid = (int32_t)x[4]; hs[k].strand = (int32_t)x[5];
        }
        std::vector<int64_t> so(n_reads + 1);
        std::vector<int32_t> nd(n_reads + 1, 0);
        for (int64_t r = 0; r <= n_reads; ++r) so[r] = io->seed_off[r] - o0;
        for (int64_t r = 0; r < n_reads; ++r) nd[r] = (int32_t)(so[r + 1] - so[r]);
        if (h_nseed_raw > 0) CK(cudaMemcpyAsync(d_seeds, hs.data(), h_nseed_raw * sizeof(Seed), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(d_read_seed_off, so.data(), (n_reads + 1) * 8, cudaMemcpyHostToDevice, st));
        if (n_reads > 0) CK(cudaMemcpyAsync(d_ndedup, nd.data(), n_reads * 4, cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
    }
    tm.mark();  // 2

    // ---------------- redundant-seed removal ----------------
    if (first <= kStLocate && n_reads > 0) {
        S.n_launch++, k_dedup<<<nblk(n_reads * 32, 128), 128, 0, st>>>(d_read_seed_off, n_reads, d_seeds, d_seeds2, d_seeds, d_ndedup);
        CK(cudaGetLastError());
    }
    // per read, its seeds after removeRedundant as rows of 6 int64 (rows
    // beyond cap are counted, not written)
    auto seeds_to_host = [&](int64_t* rows, int64_t cap, int64_t* roff, int64_t* total) -> cudaError_t {
        std::vector<int64_t> rso(n_reads + 1);
        std::vector<int32_t> nd(n_reads);
        std::vector<Seed> hs(h_nseed_raw);
        cudaError_t e = cudaMemcpyAsync(rso.data(), d_read_seed_off, (n_reads + 1) * 8, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess && n_reads > 0) e = cudaMemcpyAsync(nd.data(), d_ndedup, n_reads * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess && h_nseed_raw > 0)
            e = cudaMemcpyAsync(hs.data(), d_seeds, h_nseed_raw * sizeof(Seed), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return e;
        int64_t k = 0;
        for (int64_t r = 0; r < n_reads; ++r) {
            if (roff) roff[r] = k;
            for (int32_t j = 0; j < nd[r]; ++j, ++k) {
                if (rows && k < cap) {
                    const Seed& x = hs[rso[r] + j];
                    int64_t* o = rows + 6 * k;
                    o[0] = x.from; o[1] = x.to; o[2] = x.start; o[3] = x.end; o[4] = x.tid; o[5] = x.strand;
                }
            }
        }
        if (roff) roff[n_reads] = k;
        *total = k;
        return cudaSuccess;
    };
    if (last == kStLocate) {
        int64_t tot = 0;
        CK(seeds_to_host(io->rows, io->rows_cap, io->rows_off, &tot));
        *io->n_rows = tot;
        if (tot > io->rows_cap) return ctx->fail(MSG_EINVAL, "output capacity too small");
        S.n_seed = h_nseed_raw;
        S.ms_smem = tm.ms(0, 1);
        S.ms_locate = tm.ms(1, 2);
        S.ms_total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_host0).count();
        return MSG_OK;
    }

    // ---------------- chains ----------------
    int64_t h_nchain = 0, h_nidx = 0;
    int64_t* d_cidx_off = nullptr;
    int64_t* d_cidx = nullptr;
    int32_t* d_clen = nullptr;
    int32_t* d_cread = nullptr;
    auto setup_chainidx = [&]() -> cudaError_t {
        const cudaError_t e = ctx->chainidx.ensure((h_nchain + 1) * (8 + 4 + 4) + (h_nidx + 1) * 8 + 64);
        if (e != cudaSuccess) return e;
        d_cidx_off = ctx->chainidx.as<int64_t>();
        d_cidx = d_cidx_off + (h_nchain + 1);
        d_clen = reinterpret_cast<int32_t*>(d_cidx + (h_nidx + 1));
        d_cread = d_clen + (h_nchain + 1);
        return cudaSuccess;
    };
    if (first <= kStChain) {
    CK(ctx->chains.ensure((h_nseed_raw + 1) * (1 + 4 + 4) + 64));
    uint8_t* d_vis = ctx->chains.as<uint8_t>();
    int32_t* d_stki = reinterpret_cast<int32_t*>(d_vis + ((h_nseed_raw + 1 + 15) / 16) * 16);
    int32_t* d_stkj = d_stki + (h_nseed_raw + 1);
    if (n_reads > 0) {
        S.n_launch++, k_chain<<<nblk(n_reads, 128), 128, 0, st>>>(d_read_seed_off, d_ndedup, d_rlen, n_reads, d_seeds, d_vis, d_stki,
                                                   d_stkj, 0, d_nchain, d_nidx, nullptr, nullptr, nullptr, nullptr,
                                                   nullptr, nullptr);
        S.n_launch++, k_chain_warp<<<ctx->num_sms * 8, 128, 0, st>>>(d_read_seed_off, d_ndedup, d_rlen, n_reads, d_seeds, d_vis,
                                                   d_stki, d_stkj, 0, d_nchain, d_nidx, nullptr, nullptr, nullptr,
                                                   nullptr, nullptr, nullptr);
        CK(cudaGetLastError());
    }
    CK(offsets_async(ctx, d_nchain, n_reads, d_chain_off, misc, ctx->hpin));
    CK(offsets_async(ctx, d_nidx, n_reads, d_idx_off, misc, ctx->hpin + 1));
    CK(cudaStreamSynchronize(st));
    h_nchain = ctx->hpin[0];
    h_nidx = ctx->hpin[1];
    CK(setup_chainidx());
    if (n_reads > 0 && h_nchain > 0) {
        S.n_launch++, k_chain<<<nblk(n_reads, 128), 128, 0, st>>>(d_read_seed_off, d_ndedup, d_rlen, n_reads, d_seeds, d_vis, d_stki,
                                                   d_stkj, 1, nullptr, nullptr, d_chain_off, d_idx_off, d_cidx_off,
                                                   d_clen, d_cread, d_cidx);
        S.n_launch++, k_chain_warp<<<ctx->num_sms * 8, 128, 0, st>>>(d_read_seed_off, d_ndedup, d_rlen, n_reads, d_seeds, d_vis,
                                                   d_stki, d_stkj, 1, nullptr, nullptr, d_chain_off, d_idx_off,
                                                   d_cidx_off, d_clen, d_cread, d_cidx);
        CK(cudaGetLastError());
    }
    } else {  // the caller's chains (checked by the entry point): seed indices local to each read
        const int64_t c0 = io->read_chain_off[0];
        h_nchain = io->read_chain_off[n_reads] - c0;
        const int64_t i0 = io->chain_seed_off[c0];
        h_nidx = io->chain_seed_off[c0 + h_nchain] - i0;
        CK(setup_chainidx());
        std::vector<int64_t> coff(n_reads + 1), cio(h_nchain + 1), cix(h_nidx + 1);
        std::vector<int32_t> cl(h_nchain + 1), cr(h_nchain + 1);
        const int64_t so0 = io->seed_off[0];
        for (int64_t r = 0; r <= n_reads; ++r) coff[r] = io->read_chain_off[r] - c0;
        for (int64_t r = 0; r < n_reads; ++r) {
            for (int64_t c = coff[r]; c < coff[r + 1]; ++c) {
                const int64_t a = io->chain_seed_off[c0 + c] - i0, b = io->chain_seed_off[c0 + c + 1] - i0;
                cio[c] = a;
                cl[c] = (int32_t)(b - a);
                cr[c] = (int32_t)r;
                for (int64_t k = a; k < b; ++k) cix[k] = (io->seed_off[r] - so0) + io->chain_seed[i0 + k];
            }
        }
        CK(cudaMemcpyAsync(d_chain_off, coff.data(), (n_reads + 1) * 8, cudaMemcpyHostToDevice, st));
        if (h_nchain > 0) {
            CK(cudaMemcpyAsync(d_cidx_off, cio.data(), h_nchain * 8, cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(d_clen, cl.data(), h_nchain * 4, cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(d_cread, cr.data(), h_nchain * 4, cudaMemcpyHostToDevice, st));
        }
        if (h_nidx > 0) CK(cudaMemcpyAsync(d_cidx, cix.data(), h_nidx * 8, cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
    }
    S.n_chain = h_nchain;
    tm.mark();  // 3
    if (last == kStChain) {  // chains as seed indices within each read's seed list
        *io->o_n_chain = h_nchain;
        *io->o_n_chain_seed = h_nidx;
        if (h_nchain > io->o_chain_cap || h_nidx > io->o_chain_seed_cap)
            return ctx->fail(MSG_EINVAL, "output capacity too small");
        std::vector<int64_t> cio(h_nchain + 1), cix(h_nidx + 1), rso(n_reads + 1);
        std::vector<int32_t> cl(h_nchain + 1), cr(h_nchain + 1);
        CK(cudaMemcpyAsync(io->o_read_chain_off, d_chain_off, (n_reads + 1) * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(rso.data(), d_read_seed_off, (n_reads + 1) * 8, cudaMemcpyDeviceToHost, st));
        if (h_nchain > 0) {
            CK(cudaMemcpyAsync(cio.data(), d_cidx_off, h_nchain * 8, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(cl.data(), d_clen, h_nchain * 4, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(cr.data(), d_cread, h_nchain * 4, cudaMemcpyDeviceToHost, st));
        }
        if (h_nidx > 0) CK(cudaMemcpyAsync(cix.data(), d_cidx, h_nidx * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        int64_t k = 0;
        for (int64_t c = 0; c < h_nchain; ++c) {
            io->o_chain_seed_off[c] = k;
            for (int32_t j = 0; j < cl[c]; ++j, ++k) io->o_chain_seed[k] = (int32_t)(cix[cio[c] + j] - rso[cr[c]]);
        }
        io->o_chain_seed_off[h_nchain] = k;
        S.n_seed = h_nseed_raw;
        S.ms_smem = tm.ms(0, 1);
        S.ms_locate = tm.ms(1, 2);
        S.ms_chain = tm.ms(2, 3);
        S.ms_total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_host0).count();
        return MSG_OK;
    }

    // ---------------- DP ----------------
    if (h_nchain >= INT32_MAX) return ctx->fail(MSG_EINVAL, "too many chains in one batch");
    const int64_t NC = h_nchain + 1;
    CK(ctx->dpinfo.ensure(NC * 8 * 16 + 256));  // 16 arrays of NC int64 + counters
    int64_t* d_ts = ctx->dpinfo.as<int64_t>();
    int64_t* d_te = d_ts + NC;
    int64_t* d_cells = d_te + NC;
    int64_t* d_pcap = d_cells + NC;
    int64_t* d_rect_off = d_pcap + NC;
    int64_t* d_path_off = d_rect_off + NC;
    int64_t* d_dpcells = d_path_off + NC;
    int64_t* d_ncig = d_dpcells + NC;
    int64_t* d_area = d_ncig + NC;
    int64_t* d_sorted = d_area + NC;    // chains of the range sorted by DP class and area
    int64_t* d_fbw = d_sorted + NC;     // warp-path chains whose banded result was not certified
    int64_t* d_fb = d_fbw + NC;         // stripe-path chains whose banded result was not certified (keys first)
    int64_t* d_kidx = d_fb + NC;        // kept-record index per chain (n + 1)
    int64_t* d_map = d_kidx + NC;       // chain of each kept record
    int64_t* d_tbl = d_map + 2 * NC;    // chains traced back by k_traceback
    // counters: class sizes, fallback lists, traceback list, band statistics (kCtr*)
    unsigned long long* d_ctr2 = reinterpret_cast<unsigned long long*>(d_tbl + NC);
    unsigned long long* d_bstat = d_ctr2 + kCtrStat;
    CK(ctx->geobuf.ensure(NC * sizeof(int4) + NC * kFeat * sizeof(float) + 64));
    int4* d_geo = ctx->geobuf.as<int4>();
    float* d_feat = reinterpret_cast<float*>(d_geo + NC);
    CK(ctx->bandbuf.ensure(NC * 4 + NC * 8 + 64));
    int8_t* d_band = ctx->bandbuf.as<int8_t>();                       // 2 per chain
    uint8_t* d_keep = reinterpret_cast<uint8_t*>(d_band + 2 * NC);    // 1 per chain
    uint8_t* d_probe = d_keep + NC;                                   // 1 per chain
    int64_t* d_pcells = reinterpret_cast<int64_t*>(ctx->bandbuf.as<uint8_t>() + (NC * 4 + 7) / 8 * 8);
    const bool learned = params->band_mode == 2 && dpp.mode == 0;
    int64_t h_cells = 0, h_pathtot = 0;
    if (h_nchain > 0) {
        S.n_launch++, k_dp_prep<<<nblk(h_nchain, 256), 256, 0, st>>>(ix, d_seeds, d_cidx_off, d_clen, d_cread, d_cidx, d_off, h_nchain,
                                                       d_ts, d_te, d_cells, d_pcap, d_dpcells, d_area, d_geo);
        CK(cudaGetLastError());
        if (learned || collect) {
            S.n_launch++, k_chain_features<<<nblk(h_nchain, 128), 128, 0, st>>>(ix, d_seeds, d_cidx_off, d_clen, d_cread, d_cidx,
                                                                   d_off, d_seq, d_chain_off, d_geo, h_nchain, dpp, d_feat);
            CK(cudaGetLastError());
        }
        // total reference cells for the stats
        size_t tb = 0;
        CK(cub::DeviceReduce::Sum(nullptr, tb, d_dpcells, d_ncig, h_nchain, st));
        CK(misc.ensure(tb));
        CK(cub::DeviceReduce::Sum(misc.p, tb, d_dpcells, d_ncig, h_nchain, st));
        CK(cudaMemcpyAsync(&S.dp_cells, d_ncig, 8, cudaMemcpyDeviceToHost, st));
    }
    CK(offsets_async(ctx, d_cells, h_nchain, d_rect_off, misc, ctx->hpin + 2));  // d_cells holds bytes per chain
    CK(offsets_async(ctx, d_pcap, h_nchain, d_path_off, misc, ctx->hpin + 3));
    CK(cudaStreamSynchronize(st));
    h_cells = ctx->hpin[2];
    h_pathtot = ctx->hpin[3];
    tm.mark_at(6);  // chains prepared and storage sized
    const int64_t aux_bytes = ((2 * (h_nidx + 1) + h_nchain + 1) * sizeof(int32_t) + 15) / 16 * 16;
    // Rectangle storage of at most scratch_limit bytes at a time: when the
    // batch needs more (long reads with large flanks), the DP runs over
    // consecutive ranges of chains that fit (a single larger chain alone).
    const int64_t kScratchBudget = ctx->scratch_limit;
    std::vector<int64_t> bounds{0, h_nchain};
    int64_t rect_cap = h_cells;
    if (h_cells > kScratchBudget && h_nchain > 0) {
        std::vector<int64_t> ro(h_nchain + 1);
        CK(cudaMemcpy(ro.data(), d_rect_off, (h_nchain + 1) * 8, cudaMemcpyDeviceToHost));
        bounds.assign(1, 0);
        rect_cap = 0;
        int64_t c0 = 0;
        for (int64_t c = 1; c <= h_nchain; ++c) {
            if (c == h_nchain || (ro[c + 1] - ro[c0] > kScratchBudget && c > c0)) {
                bounds.push_back(c);
                rect_cap = std::max(rect_cap, ro[c] - ro[c0]);
                c0 = c;
            }
        }
    }
    CK(ctx->scratch.ensure(rect_cap + 64 + aux_bytes + (2 * h_nidx + h_nchain + 1) * sizeof(int4)));
    std::vector<int64_t> h_rect_off(bounds.size(), 0);  // bounds[0] = 0 starts at offset 0
    for (size_t b = 1; b < bounds.size(); ++b)
        CK(cudaMemcpy(&h_rect_off[b], d_rect_off + bounds[b], 8, cudaMemcpyDeviceToHost));
    const int64_t P16 = ((h_pathtot + 1 + 15) / 16) * 16;
    CK(ctx->path.ensure(P16 + (h_nchain + 1) * 4 + 64));
    CK(ctx->alnbuf.ensure((h_nchain + 1) * sizeof(msg_aln)));
    uint8_t* d_scr = ctx->scratch.as<uint8_t>();
    int32_t* d_aux = reinterpret_cast<int32_t*>(d_scr + (rect_cap + 64) / 16 * 16);
    int4* d_sdbuf = reinterpret_cast<int4*>(reinterpret_cast<uint8_t*>(d_aux) + aux_bytes);
    uint8_t* d_path = ctx->path.as<uint8_t>();
    int32_t* d_plen = reinterpret_cast<int32_t*>(d_path + P16);
    msg_aln* d_aln = ctx->alnbuf.as<msg_aln>();
    DpArgs da{};
    da.ix = ix; da.seeds = d_seeds; da.chain_idx_off = d_cidx_off; da.chain_len = d_clen; da.chain_read = d_cread;
    da.chain_idx = d_cidx; da.n_chain = h_nchain; da.rseq = d_seq; da.roff = d_off; da.t_start = d_ts;
    da.t_end = d_te; da.scr_off = d_rect_off; da.scr = d_scr; da.aux = d_aux; da.sdbuf = d_sdbuf;
    da.path_off = d_path_off; da.path = d_path; da.path_len = d_plen; da.aln = d_aln;
    da.pp = dpp; da.status = d_status;
    da.band = d_band; da.min_rate = params->min_score_rate; da.keep = d_keep; da.fb_list = d_fb;
    da.fb_n = d_ctr2 + 2; da.bstat = d_bstat;
    da.tb_list = d_tbl; da.tb_n = d_ctr2 + kCtrTrace;
    da.lanes16 = ctx->dp_lanes == 16;
    da.cls_n = d_ctr2; da.cls = -1;
    const __nv_bfloat16* d_wts = ctx->band_wts.as<__nv_bfloat16>();
    const float* d_nrm = ctx->band_nrm.as<float>();

    if (collect) {
        // Certificate of every banded class on every chain; cost per class in cells.
        if (bounds.size() > 2) return ctx->fail(MSG_EINVAL, "batch too large for one collection; split it");
        if (collect->cap < h_nchain) { *collect->n_chain = h_nchain; return ctx->fail(MSG_EINVAL, "capacity too small"); }
        *collect->n_chain = h_nchain;
        if (h_nchain == 0) return MSG_OK;
        std::vector<int64_t> area(h_nchain), best(h_nchain);
        std::vector<int32_t> lab(h_nchain, kCls - 1);
        std::vector<uint8_t> eligible(h_nchain, 0);
        std::vector<uint8_t> pr(h_nchain);
        std::vector<int64_t> pc(h_nchain);
        CK(cudaMemcpyAsync(area.data(), d_area, h_nchain * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(collect->feat, d_feat, h_nchain * kFeat * sizeof(float), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        for (int64_t c = 0; c < h_nchain; ++c) best[c] = area[c];
        da.probe = d_probe; da.probe_cells = d_pcells;
        for (int cls = kCls - 2; cls >= 0; --cls) {  // wider classes first: ties keep the wider one
            CK(cudaMemsetAsync(d_ctr2, 0, kCtrWords * 8, st));
            CK(cudaMemsetAsync(d_probe, 3, h_nchain, st));  // 3: not banded at this class
            CK(cudaMemcpyAsync(d_pcells, d_area, h_nchain * 8, cudaMemcpyDeviceToDevice, st));
            CK(dp_sort(ctx, 0, h_nchain, d_geo, d_area, d_feat, 1, band_width(cls), nullptr, nullptr, d_band,
                       d_ctr2, d_fb, d_kidx, d_sorted, S));
            da.list = d_sorted;
            launch_dp(ctx, da, kDpStripeBand, h_nchain, S);
            launch_dp(ctx, da, kDpWarpBand, h_nchain, S);
            CK(cudaGetLastError());
            CK(cudaMemcpyAsync(pr.data(), d_probe, h_nchain, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(pc.data(), d_pcells, h_nchain * 8, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            for (int64_t c = 0; c < h_nchain; ++c) {
                if (pr[c] == 3) continue;
                eligible[c] = 1;
                const int64_t cost = pr[c] ? pc[c] : pc[c] + area[c];
                if (cost < best[c]) { best[c] = cost; lab[c] = cls; }
            }
        }
        for (int64_t c = 0; c < h_nchain; ++c) if (!eligible[c]) lab[c] = -1;
        std::memcpy(collect->label, lab.data(), h_nchain * sizeof(int32_t));
        uint32_t h_status = 0;
        CK(cudaMemcpyAsync(&h_status, d_status, 4, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (h_status & kErrInternal) return ctx->fail(MSG_EINTERNAL, "device consistency check failed");
        return MSG_OK;
    }

    const bool filtering = params->min_score_rate >= 0;
    if (h_nchain > 0) CK(cudaMemsetAsync(d_ctr2, 0, kCtrWords * 8, st));
    for (size_t ch = 0; ch + 1 < bounds.size(); ++ch) {
        const int64_t c0 = bounds[ch], nch = bounds[ch + 1] - bounds[ch];
        if (nch <= 0) continue;
        if (ch > 0) {  // lists and work counters start again; statistics accumulate
            CK(cudaMemsetAsync(d_ctr2, 0, kCtrStat * 8, st));
            CK(cudaMemsetAsync(d_ctr2 + kCtrQueue, 0, (kCtrWords - kCtrQueue) * 8, st));
        }
        da.scr_base = h_rect_off[ch];
        da.band = d_band;
        const int bmode = dpp.mode != 0 ? 0 : params->band_mode;
        CK(dp_sort(ctx, c0, nch, d_geo, d_area, d_feat, bmode, params->band_w, d_wts, d_nrm, d_band, d_ctr2, d_fb,
                   d_kidx, d_sorted, S));
        da.list = d_sorted;
        if (ch == 0) tm.mark_at(7);  // first range's classes assigned and sorted
        // Every launch is sized for the range; each reads its class's part of
        // the sorted list on the device, so no host round trip is needed.
        // The classes run side by side: row-by-row, stripe and banded-stripe
        // launches on three streams forked from the context's, the warp
        // launches on the context's own; a launch's last blocks (its largest
        // chains) then overlap the other launches' work. Chains of different
        // classes touch disjoint storage.
        CK(ctx->dp_streams_ready());
        CK(cudaEventRecord(ctx->dp_ev[0], st));
        for (int q = 0; q < 3; ++q) CK(cudaStreamWaitEvent(ctx->dp_side[q], ctx->dp_ev[0], 0));
        da.fb_list = d_fb; da.fb_n = d_ctr2 + kCtrFbStripe;
        launch_dp(ctx, da, kDpSmall, nch, S, ctx->dp_side[0]);
        launch_dp(ctx, da, kDpStripe, nch, S, ctx->dp_side[1]);
        launch_dp(ctx, da, kDpWarp, nch, S);
        if (bmode != 0) {
            launch_dp(ctx, da, kDpStripeBand, nch, S, ctx->dp_side[2]);
            da.fb_list = d_fbw; da.fb_n = d_ctr2 + kCtrFbWarp;
            launch_dp(ctx, da, kDpWarpBand, nch, S);
            // banded chains without a certificate, on the whole cell set: few
            // chains, mostly large, so a warp each (a thread each would leave
            // the launch waiting on its largest chain); each after the launch
            // that lists them, on its stream
            DpArgs fb = da;
            fb.band = nullptr;
            fb.list = d_fb; fb.n_list = d_ctr2 + kCtrFbStripe;
            launch_dp(ctx, fb, -kDpWarp - 1, nch, S, ctx->dp_side[2]);
            fb.list = d_fbw; fb.n_list = d_ctr2 + kCtrFbWarp;
            launch_dp(ctx, fb, -kDpWarp - 1, nch, S);
        }
        CK(cudaGetLastError());
        for (int q = 0; q < 3; ++q) {
            CK(cudaEventRecord(ctx->dp_ev[1 + q], ctx->dp_side[q]));
            CK(cudaStreamWaitEvent(st, ctx->dp_ev[1 + q], 0));
        }
        S.n_launch++, k_traceback<<<nblk(nch, 128), 128, 0, st>>>(da);
        CK(cudaGetLastError());
        if (bounds.size() > 2) {  // chains per class of this range, for the statistics
            unsigned long long w[kDpClasses];
            CK(cudaMemcpy(w, d_ctr2, sizeof(w), cudaMemcpyDeviceToHost));
            S.n_dp_warp += (int64_t)(w[kDpWarp] + w[kDpWarpBand]);
            for (int q = 0; q < kDpClasses; ++q) S.n_dp_class[q] += (int64_t)w[q];
        }
    }
    tm.mark();  // 4
    // Alignment::filter on the device: compact the kept records.
    int64_t h_nrec = h_nchain;
    msg_aln* d_rec = d_aln;
    const int64_t* d_rmap = nullptr;
    const int64_t* d_roff = d_chain_off;
    if (filtering && h_nchain > 0) {
        S.n_launch++, k_keep64<<<nblk(h_nchain, 256), 256, 0, st>>>(d_keep, h_nchain, d_ncig);
        CK(offsets(ctx, d_ncig, h_nchain, d_kidx, misc, &h_nrec));
        CK(ctx->alnbuf2.ensure((h_nrec + 1) * sizeof(msg_aln)));
        CK(ctx->recoff.ensure((n_reads + 1) * 8));
        d_rec = ctx->alnbuf2.as<msg_aln>();
        S.n_launch++, k_compact_aln<<<nblk(h_nchain, 256), 256, 0, st>>>(d_aln, d_keep, d_kidx, h_nchain, d_rec, d_map);
        S.n_launch++, k_gather_off<<<nblk(n_reads + 1, 256), 256, 0, st>>>(d_chain_off, d_kidx, n_reads, ctx->recoff.as<int64_t>());
        CK(cudaGetLastError());
        d_rmap = d_map;
        d_roff = ctx->recoff.as<int64_t>();
    }
    int64_t h_ncig = 0;
    if (h_nrec > 0) {
        S.n_launch++, k_cigar<<<nblk(h_nrec, 256), 256, 0, st>>>(h_nrec, d_rec, d_rmap, d_off, d_path_off, d_plen, d_path, 0, d_ncig,
                                                   nullptr, nullptr);
        CK(cudaGetLastError());
    }
    int64_t* d_cig_off = d_cells;  // reuse: cells no longer needed after the scan
    CK(offsets(ctx, d_ncig, h_nrec, d_cig_off, misc, &h_ncig));
    CK(ctx->cigbuf.ensure((h_ncig + 1) * 4));
    if (h_nrec > 0) {
        S.n_launch++, k_cigar<<<nblk(h_nrec, 256), 256, 0, st>>>(h_nrec, d_rec, d_rmap, d_off, d_path_off, d_plen, d_path, 1, nullptr,
                                                   d_cig_off, ctx->cigbuf.as<uint32_t>());
        S.n_launch++, k_aln_cig<<<nblk(h_nrec, 256), 256, 0, st>>>(d_rec, d_cig_off, h_nrec);
        CK(cudaGetLastError());
    }
    tm.mark();  // 5
    uint32_t h_status = 0;
    unsigned long long h_ctr2[kCtrWords] = {0};
    const unsigned long long* h_bstat = h_ctr2 + kCtrStat;
    CK(cudaMemcpyAsync(&h_status, d_status, 4, cudaMemcpyDeviceToHost, st));
    if (h_nchain > 0) CK(cudaMemcpyAsync(h_ctr2, d_ctr2, sizeof(h_ctr2), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (h_status & kErrInternal) return ctx->fail(MSG_EINTERNAL, "device consistency check failed");
    S.n_aln = h_nrec;
    S.n_band_fallback = (int64_t)h_bstat[0];
    S.n_band_exact = (int64_t)h_bstat[1];
    S.n_band_drop = (int64_t)h_bstat[2];
    S.dp_cells_done = 0;
    for (int q = 0; q < kDpClasses; ++q) {
        S.dp_class_cells[q] = (int64_t)h_bstat[3 + q];
        S.dp_cells_done += S.dp_class_cells[q];
    }
    S.n_filtered = h_nchain - h_nrec;
    if (bounds.size() <= 2) {
        S.n_dp_warp = (int64_t)(h_ctr2[kDpWarp] + h_ctr2[kDpWarpBand]);
        for (int q = 0; q < kDpClasses; ++q) S.n_dp_class[q] = (int64_t)h_ctr2[q];
    }
    S.ms_smem = tm.ms(0, 1);
    S.ms_locate = tm.ms(1, 2);
    S.ms_chain = tm.ms(2, 3);
    S.ms_dp = tm.ms(3, 5);
    if (h_nchain > 0) {  // the DP stage by part (one range: exact; several: the first range's sort ends part 1)
        S.ms_dp_part[0] = tm.ms(3, 6);  // prep, features, sizes
        S.ms_dp_part[1] = tm.ms(6, 7);  // band classes and the class sort
        S.ms_dp_part[2] = tm.ms(7, 4);  // fills and tracebacks
        S.ms_dp_part[3] = tm.ms(4, 5);  // filter and CIGARs
    }

    // ---------------- results ----------------
    out->n_aln = h_nrec;
    out->n_cigar = h_ncig;
    ctx->res_aln = d_rec;
    ctx->res_cigar = ctx->cigbuf.as<uint32_t>();
    ctx->res_off = d_roff;
    const bool on_device = !out->aln && !out->cigar && !out->read_aln_off;
    if (!on_device) {
        if (h_nrec > out->aln_cap || h_ncig > out->cigar_cap) return ctx->fail(MSG_EINVAL, "output capacity too small");
        if (h_nrec > 0) {
            if (!out->aln || !out->cigar) return ctx->fail(MSG_EINVAL, "null output buffer");
            CK(cudaMemcpyAsync(out->aln, d_rec, h_nrec * sizeof(msg_aln), cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(out->cigar, ctx->cigbuf.p, h_ncig * 4, cudaMemcpyDeviceToHost, st));
        }
        if (out->read_aln_off)
            CK(cudaMemcpyAsync(out->read_aln_off, d_roff, (n_reads + 1) * 8, cudaMemcpyDeviceToHost, st));
    }
    if (dump) {
        dump->n_smem = h_nsmem;
        if (dump->smem && h_nsmem <= dump->smem_cap)
            CK(cudaMemcpyAsync(dump->smem, d_smem, h_nsmem * 48, cudaMemcpyDeviceToHost, st));
        if (dump->smem_off) CK(cudaMemcpyAsync(dump->smem_off, d_smem_off, (n_reads + 1) * 8, cudaMemcpyDeviceToHost, st));
        // dense seeds per read after removeRedundant
        int64_t k = 0;
        CK(seeds_to_host(dump->seed, dump->seed_cap, dump->seed_off, &k));
        dump->n_seed = k;
    }
    CK(cudaStreamSynchronize(st));
    S.n_seed = h_nseed_raw;
    S.ms_total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_host0).count();
#undef CK
    return MSG_OK;
}

extern "C" int msg_map_batch_device(msg_ctx* ctx, const msg_read_batch* reads, const msg_map_params* params,
                                    msg_aln_out* out, msg_stage_dump* dump) {
    if (!ctx || !reads || !params || !out) return MSG_EINVAL;
    if (!ctx->idx.loaded) return ctx->fail(MSG_ESTATE, "no index loaded");
    if (reads->n_reads < 0 || (reads->n_reads > 0 && (!reads->seq || !reads->off))) return MSG_EINVAL;
    if (reads->n_reads > INT32_MAX) return MSG_EINVAL;
    msg::DeviceGuard dg_(ctx->device);
    if (!dg_.ok) return ctx->fail(MSG_ECUDA, "cudaSetDevice");
    return map_impl(ctx, reads->seq, reads->off, reads->n_reads, params, out, dump);
}

// Copy a host read batch into the context's device buffers.
static int upload_reads(msg_ctx* ctx, const msg_read_batch* reads) {
    const int64_t n = reads->n_reads;
    if (n < 0 || (n > 0 && (!reads->seq || !reads->off))) return MSG_EINVAL;
    if (n > INT32_MAX) return MSG_EINVAL;
    for (int64_t i = 0; i < n; ++i)
        if (reads->off[i + 1] < reads->off[i]) return MSG_EINVAL;
    const int64_t bytes = n > 0 ? reads->off[n] - reads->off[0] : 0;
    cudaError_t e = ctx->reads.ensure(bytes + 16);
    if (e != cudaSuccess) return ctx->cuda_fail(e);
    e = ctx->offs.ensure((n + 1) * 8);
    if (e != cudaSuccess) return ctx->cuda_fail(e);
    // the caller's buffers are copied as they are (straight from pinned
    // memory when the caller pinned them) and the offsets rebased to the
    // first read on the device; the copies complete before the call returns
    if (bytes > 0) {
        e = cudaMemcpyAsync(ctx->reads.p, reads->seq + reads->off[0], bytes, cudaMemcpyHostToDevice, ctx->stream);
        if (e != cudaSuccess) return ctx->cuda_fail(e);
    }
    if (n > 0) {
        e = cudaMemcpyAsync(ctx->offs.p, reads->off, (n + 1) * 8, cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess && reads->off[0] != 0) {
            k_rebase<<<nblk(n + 1, 256), 256, 0, ctx->stream>>>(ctx->offs.as<int64_t>(), n + 1, reads->off[0]);
            e = cudaGetLastError();
        }
    } else {
        e = cudaMemsetAsync(ctx->offs.p, 0, 8, ctx->stream);
    }
    return e == cudaSuccess ? MSG_OK : ctx->cuda_fail(e);
}

extern "C" int msg_map_batch(msg_ctx* ctx, const msg_read_batch* reads, const msg_map_params* params,
                             msg_aln_out* out, msg_stage_dump* dump) {
    if (!ctx || !reads || !params || !out) return MSG_EINVAL;
    if (!ctx->idx.loaded) return ctx->fail(MSG_ESTATE, "no index loaded");
    msg::DeviceGuard dg_(ctx->device);
    if (!dg_.ok) return ctx->fail(MSG_ECUDA, "cudaSetDevice");
    const int rc = upload_reads(ctx, reads);
    if (rc != MSG_OK) return rc;
    return map_impl(ctx, ctx->reads.as<uint8_t>(), ctx->offs.as<int64_t>(), reads->n_reads, params, out, dump);
}

extern "C" int msg_map_batches(msg_ctx* ctx, int64_t n_batches, const msg_read_batch* reads,
                               const msg_map_params* params, msg_aln_out* outs) {
    if (!ctx || n_batches < 0 || (n_batches > 0 && (!reads || !outs)) || !params) return MSG_EINVAL;
    if (!ctx->idx.loaded) return ctx->fail(MSG_ESTATE, "no index loaded");
    for (int64_t k = 0; k < n_batches; ++k) {
        const msg_read_batch& r = reads[k];
        if (r.n_reads < 0 || r.n_reads > INT32_MAX || (r.n_reads > 0 && (!r.seq || !r.off))) return MSG_EINVAL;
        for (int64_t i = 0; i < r.n_reads; ++i)
            if (r.off[i + 1] < r.off[i]) return MSG_EINVAL;
        if (!outs[k].aln || !outs[k].cigar) return ctx->fail(MSG_EINVAL, "null output buffer");
    }
    msg::DeviceGuard dg_(ctx->device);
    if (!dg_.ok) return ctx->fail(MSG_ECUDA, "cudaSetDevice");
#define CK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { cudaStreamSynchronize(ctx->cstream); return ctx->cuda_fail(e_); } } while (0)
    if (!ctx->cstream) {
        if (cudaStreamCreateWithFlags(&ctx->cstream, cudaStreamNonBlocking) != cudaSuccess)
            return ctx->fail(MSG_ECUDA, "copy stream");
        for (cudaEvent_t& e : ctx->pev) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    }
    cudaStream_t cs = ctx->cstream, st = ctx->stream;
    // batch k's reads into input slot k % 2 on the copy stream; the slot's
    // previous batch (k - 2) finished before batch k - 1 started
    auto upload = [&](int64_t k) -> cudaError_t {
        const msg_read_batch& r = reads[k];
        const int sl = (int)(k & 1);
        const int64_t n = r.n_reads;
        const int64_t bytes = n > 0 ? r.off[n] - r.off[0] : 0;
        cudaError_t e = ctx->in_seq[sl].ensure(bytes + 16);
        if (e == cudaSuccess) e = ctx->in_off[sl].ensure((n + 1) * 8);
        if (e != cudaSuccess) return e;
        if (bytes > 0) e = cudaMemcpyAsync(ctx->in_seq[sl].p, r.seq + r.off[0], bytes, cudaMemcpyHostToDevice, cs);
        if (e != cudaSuccess) return e;
        if (n > 0) {
            e = cudaMemcpyAsync(ctx->in_off[sl].p, r.off, (n + 1) * 8, cudaMemcpyHostToDevice, cs);
            if (e == cudaSuccess && r.off[0] != 0) {
                k_rebase<<<nblk(n + 1, 256), 256, 0, cs>>>(ctx->in_off[sl].as<int64_t>(), n + 1, r.off[0]);
                e = cudaGetLastError();
            }
        } else {
            e = cudaMemsetAsync(ctx->in_off[sl].p, 0, 8, cs);
        }
        if (e == cudaSuccess) e = cudaEventRecord(ctx->pev[sl], cs);
        return e;
    };
    int status = MSG_OK;
    if (n_batches > 0) CK(upload(0));
    for (int64_t k = 0; k < n_batches; ++k) {
        const int sl = (int)(k & 1);
        // the device buffers of the next batch's upload are not reallocated
        // while this batch runs: upload k + 1 goes to the other slot
        if (k + 1 < n_batches) CK(upload(k + 1));
        CK(cudaStreamWaitEvent(st, ctx->pev[sl], 0));
        msg_aln_out dev{};  // results stay on the device
        const int rc = map_impl(ctx, ctx->in_seq[sl].as<uint8_t>(), ctx->in_off[sl].as<int64_t>(), reads[k].n_reads,
                                params, &dev, nullptr);
        if (rc != MSG_OK) { cudaStreamSynchronize(cs); return rc; }
        msg_aln_out& o = outs[k];
        o.n_aln = dev.n_aln;
        o.n_cigar = dev.n_cigar;
        if (dev.n_aln > o.aln_cap || dev.n_cigar > o.cigar_cap) { status = MSG_EINVAL; continue; }
        // stage the records (the next batch overwrites the context's result
        // buffers) and copy them back on the copy stream while it runs
        const int64_t n = reads[k].n_reads;
        const size_t ab = dev.n_aln * sizeof(msg_aln), cb = dev.n_cigar * 4, ob = (n + 1) * 8;
        CK(cudaStreamWaitEvent(st, ctx->pev[4 + sl], 0));  // slot's download from batch k - 2 done
        if (ab + cb + ob + 64 > ctx->stage[sl].cap) CK(cudaStreamSynchronize(cs));  // before the slot is replaced
        CK(ctx->stage[sl].ensure(ab + cb + ob + 64));
        char* sg = ctx->stage[sl].as<char>();
        if (ab) CK(cudaMemcpyAsync(sg, ctx->res_aln, ab, cudaMemcpyDeviceToDevice, st));
        if (cb) CK(cudaMemcpyAsync(sg + ab, ctx->res_cigar, cb, cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(sg + ab + cb, ctx->res_off, ob, cudaMemcpyDeviceToDevice, st));
        CK(cudaEventRecord(ctx->pev[2 + sl], st));
        CK(cudaStreamWaitEvent(cs, ctx->pev[2 + sl], 0));
        if (ab) CK(cudaMemcpyAsync(o.aln, sg, ab, cudaMemcpyDeviceToHost, cs));
        if (cb) CK(cudaMemcpyAsync(o.cigar, sg + ab, cb, cudaMemcpyDeviceToHost, cs));
        if (o.read_aln_off) CK(cudaMemcpyAsync(o.read_aln_off, sg + ab + cb, ob, cudaMemcpyDeviceToHost, cs));
        CK(cudaEventRecord(ctx->pev[4 + sl], cs));
    }
    CK(cudaStreamSynchronize(cs));
    CK(cudaStreamSynchronize(st));
#undef CK
    if (status != MSG_OK) return ctx->fail(status, "output capacity too small");
    return MSG_OK;
}

// ---------------------------------------------------------------------------
// The mapping task one stage at a time (the reference's operator boundaries).
// The caller's arrays are checked on the host first so that no kernel indexes
// memory through them: offsets ascend, SMEM rows address suffix-array rows of
// the index, seeds lie in their read and chromosome, chains list seeds of
// their own read in ascending, non-overlapping order.
// ---------------------------------------------------------------------------
namespace {
bool offsets_ok(const int64_t* off, int64_t n) {
    if (!off || off[0] < 0) return false;
    for (int64_t i = 0; i < n; ++i)
        if (off[i + 1] < off[i]) return false;
    return true;
}

int64_t read_len_of(const msg_read_batch* reads, int64_t r) { return reads->off[r + 1] - reads->off[r]; }

bool reads_ok(const msg_read_batch* reads) {
    const int64_t n = reads->n_reads;
    return n >= 0 && n <= INT32_MAX && (n == 0 || (reads->seq && offsets_ok(reads->off, n)));
}

bool seeds_ok(const msg_ctx* ctx, const msg_read_batch* reads, const int64_t* seed, const int64_t* seed_off) {
    const int64_t n = reads->n_reads;
    if (!offsets_ok(seed_off, n) || (seed_off[n] > seed_off[0] && !seed)) return false;
    const int64_t* chr_len = ctx->idx.chr_len_host.data();
    const int64_t nc = (int64_t)ctx->idx.chr_len_host.size();
    for (int64_t r = 0; r < n; ++r) {
        const int64_t L = read_len_of(reads, r);
        for (int64_t k = seed_off[r]; k < seed_off[r + 1]; ++k) {
            const int64_t* x = seed + 6 * k;  // from, to, start, end, tid, strand
            if (!(0 <= x[0] && x[0] < x[1] && x[1] <= L && x[4] >= 0 && x[4] < nc && (x[5] == 1 || x[5] == 2)))
                return false;
            if (!(0 <= x[2] && x[2] < x[3] && x[3] <= chr_len[x[4]] && x[3] - x[2] == x[1] - x[0])) return false;
        }
    }
    return true;
}

bool chains_ok(const msg_ctx* ctx, const msg_read_batch* reads, const int64_t* seed, const int64_t* seed_off,
               const int32_t* chain_seed, const int64_t* chain_seed_off, const int64_t* read_chain_off) {
    const int64_t n = reads->n_reads;
    if (!seeds_ok(ctx, reads, seed, seed_off) || !offsets_ok(read_chain_off, n) || !chain_seed_off) return false;
    const int64_t c0 = read_chain_off[0], nch = read_chain_off[n] - c0;
    if (nch >= INT32_MAX || !offsets_ok(chain_seed_off + c0, nch)) return false;
    if (chain_seed_off[c0 + nch] > chain_seed_off[c0] && !chain_seed) return false;
    for (int64_t r = 0; r < n; ++r) {
        const int64_t ns = seed_off[r + 1] - seed_off[r];
        for (int64_t c = read_chain_off[r]; c < read_chain_off[r + 1]; ++c) {
            const int64_t a = chain_seed_off[c], b = chain_seed_off[c + 1];
            if (b <= a) return false;  // a chain holds at least one seed
            for (int64_t k = a; k < b; ++k) {
                if (chain_seed[k] < 0 || chain_seed[k] >= ns) return false;
                if (k > a) {
                    const int64_t* l = seed + 6 * (seed_off[r] + chain_seed[k - 1]);
                    const int64_t* q = seed + 6 * (seed_off[r] + chain_seed[k]);
                    if (!(chain_seed[k] > chain_seed[k - 1] && l[1] <= q[0] && l[3] <= q[2] && l[4] == q[4] &&
                          l[5] == q[5]))
                        return false;
                }
            }
        }
    }
    return true;
}

int stage_call(msg_ctx* ctx, const msg_read_batch* reads, const msg_map_params* params, StageIO& io,
               msg_aln_out* out) {
    msg::DeviceGuard dg_(ctx->device);
    if (!dg_.ok) return ctx->fail(MSG_ECUDA, "cudaSetDevice");
    const int rc = upload_reads(ctx, reads);
    if (rc != MSG_OK) return rc;
    msg_map_params dflt;
    msg_map_params_default(&dflt);
    msg_aln_out none{};
    return map_impl(ctx, ctx->reads.as<uint8_t>(), ctx->offs.as<int64_t>(), reads->n_reads, params ? params : &dflt,
                    out ? out : &none, nullptr, nullptr, &io);
}
}  // namespace

extern "C" int msg_seed_batch(msg_ctx* ctx, const msg_read_batch* reads, const msg_map_params* params,
                              int64_t* smem, int64_t smem_cap, int64_t* smem_off, int64_t* n_smem) {
    if (!ctx || !reads || !params || !smem_off || !n_smem || smem_cap < 0 || (smem_cap > 0 && !smem))
        return MSG_EINVAL;
    if (!ctx->idx.loaded) return ctx->fail(MSG_ESTATE, "no index loaded");
    if (!reads_ok(reads)) return MSG_EINVAL;
    StageIO io;
    io.first = kStSmem; io.last = kStSmem;
    io.rows = smem; io.rows_cap = smem_cap; io.rows_off = smem_off; io.n_rows = n_smem;
    return stage_call(ctx, reads, params, io, nullptr);
}

extern "C" int msg_locate_batch(msg_ctx* ctx, const msg_read_batch* reads, const int64_t* smem,
                                const int64_t* smem_off, int64_t* seed, int64_t seed_cap, int64_t* seed_off,
                                int64_t* n_seed) {
    if (!ctx || !reads || !seed_off || !n_seed || seed_cap < 0 || (seed_cap > 0 && !seed)) return MSG_EINVAL;
    if (!ctx->idx.loaded) return ctx->fail(MSG_ESTATE, "no index loaded");
    if (!reads_ok(reads)) return MSG_EINVAL;
    const int64_t n = reads->n_reads;
    if (!offsets_ok(smem_off, n) || (smem_off[n] > smem_off[0] && !smem)) return ctx->fail(MSG_EINVAL, "bad SMEM offsets");
    const int64_t nbwt = ctx->idx.dev.n;
    for (int64_t r = 0; r < n; ++r) {
        const int64_t L = read_len_of(reads, r);
        for (int64_t k = smem_off[r]; k < smem_off[r + 1]; ++k) {
            const int64_t* x = smem + 6 * k;  // from, to, fwdStart, revStart, size, logP
            if (!(0 <= x[0] && x[0] < x[1] && x[1] <= L && x[4] >= 0 && x[2] >= 0 && x[3] >= 0 &&
                  x[4] <= nbwt && x[2] <= nbwt - x[4] && x[3] <= nbwt - x[4]))
                return ctx->fail(MSG_EINVAL, "an SMEM row lies outside its read or the index");
        }
    }
    StageIO io;
    io.first = kStLocate; io.last = kStLocate;
    io.smem = smem; io.smem_off = smem_off;
    io.rows = seed; io.rows_cap = seed_cap; io.rows_off = seed_off; io.n_rows = n_seed;
    return stage_call(ctx, reads, nullptr, io, nullptr);
}

extern "C" int msg_chain_batch(msg_ctx* ctx, const msg_read_batch* reads, const int64_t* seed, const int64_t* seed_off,
                               int32_t* chain_seed, int64_t chain_seed_cap, int64_t* chain_seed_off,
                               int64_t chain_cap, int64_t* read_chain_off, int64_t* n_chain, int64_t* n_chain_seed) {
    if (!ctx || !reads || !read_chain_off || !n_chain || !n_chain_seed || chain_cap < 0 || chain_seed_cap < 0 ||
        !chain_seed_off || (chain_seed_cap > 0 && !chain_seed))
        return MSG_EINVAL;
    if (!ctx->idx.loaded) return ctx->fail(MSG_ESTATE, "no index loaded");
    if (!reads_ok(reads)) return MSG_EINVAL;
    if (!seeds_ok(ctx, reads, seed, seed_off)) return ctx->fail(MSG_EINVAL, "a seed lies outside its read or chromosome");
    StageIO io;
    io.first = kStChain; io.last = kStChain;
    io.seed = seed; io.seed_off = seed_off;
    io.o_chain_seed = chain_seed; io.o_chain_seed_cap = chain_seed_cap; io.o_chain_seed_off = chain_seed_off;
    io.o_chain_cap = chain_cap; io.o_read_chain_off = read_chain_off; io.o_n_chain = n_chain;
    io.o_n_chain_seed = n_chain_seed;
    return stage_call(ctx, reads, nullptr, io, nullptr);
}

extern "C" int msg_align_batch(msg_ctx* ctx, const msg_read_batch* reads, const int64_t* seed, const int64_t* seed_off,
                               const int32_t* chain_seed, const int64_t* chain_seed_off, const int64_t* read_chain_off,
                               const msg_map_params* params, msg_aln_out* out) {
    if (!ctx || !reads || !params || !out) return MSG_EINVAL;
    if (!ctx->idx.loaded) return ctx->fail(MSG_ESTATE, "no index loaded");
    if (!reads_ok(reads)) return MSG_EINVAL;
    if (!chains_ok(ctx, reads, seed, seed_off, chain_seed, chain_seed_off, read_chain_off))
        return ctx->fail(MSG_EINVAL, "a chain or seed does not fit its read, chromosome or seed list");
    StageIO io;
    io.first = kStAlign; io.last = kStAlign;
    io.seed = seed; io.seed_off = seed_off;
    io.chain_seed = chain_seed; io.chain_seed_off = chain_seed_off; io.read_chain_off = read_chain_off;
    return stage_call(ctx, reads, params, io, out);
}

// ---------------------------------------------------------------------------
// Band model: parameters, training data, training and gradient check.
// ---------------------------------------------------------------------------
namespace {
uint64_t splitmix64(uint64_t& x) {
    uint64_t z = (x += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
double unit01(uint64_t& x) { return ((splitmix64(x) >> 11) + 0.5) * (1.0 / 9007199254740992.0); }

// Weights (kNTrain floats at w) into bf16 on the device; mean/scale into nrm.
int put_model(msg_ctx* ctx, const float* params, msg::DevBuf& wts, msg::DevBuf& nrm) {
    cudaStream_t st = ctx->stream;
    cudaError_t e = wts.ensure(kNTrain * sizeof(__nv_bfloat16));
    if (e == cudaSuccess) e = nrm.ensure(2 * kFeat * sizeof(float));
    if (e == cudaSuccess) e = ctx->tr_g.ensure(kNTrain * sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpyAsync(nrm.p, params, 2 * kFeat * sizeof(float), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->tr_g.p, params + kOffW1, kNTrain * sizeof(float), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return ctx->cuda_fail(e);
    k_to_bf16<<<nblk(kNTrain, 256), 256, 0, st>>>(kNTrain, ctx->tr_g.as<float>(), wts.as<__nv_bfloat16>());
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e == cudaSuccess ? MSG_OK : ctx->cuda_fail(e);
}

bool params_ok(const float* params) {
    for (int k = 0; k < kNParams; ++k) if (!std::isfinite(params[k])) return false;
    for (int k = 0; k < kFeat; ++k) if (!(params[kOffSd + k] > 0)) return false;
    return true;
}

// Normalised features of n samples into ctx->tr_x, labels into tr_y.
int put_samples(msg_ctx* ctx, const float* feat, const int32_t* label, int64_t n, const float* nrm_host) {
    cudaStream_t st = ctx->stream;
    cudaError_t e = ctx->tr_x.ensure(n * kFeat * sizeof(float) * 2 + 64);
    if (e == cudaSuccess) e = ctx->tr_y.ensure(n * sizeof(int32_t) + 64);
    if (e == cudaSuccess) e = ctx->tr_loss.ensure(2 * kFeat * sizeof(float) + 64);
    if (e != cudaSuccess) return ctx->cuda_fail(e);
    float* raw = ctx->tr_x.as<float>() + n * kFeat;
    float* d_nrm = ctx->tr_loss.as<float>() + 16;
    e = cudaMemcpyAsync(raw, feat, n * kFeat * sizeof(float), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->tr_y.p, label, n * sizeof(int32_t), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_nrm, nrm_host, 2 * kFeat * sizeof(float), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return ctx->cuda_fail(e);
    k_normalize<<<nblk(n * kFeat, 256), 256, 0, st>>>(n, raw, d_nrm, ctx->tr_x.as<float>());
    e = cudaGetLastError();
    return e == cudaSuccess ? MSG_OK : ctx->cuda_fail(e);
}

int grad_smem_ready(msg_ctx* ctx) {
    const cudaError_t e = cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGradSmem);
    return e == cudaSuccess ? MSG_OK : ctx->cuda_fail(e);
}
}  // namespace

extern "C" int msg_band_model_set(msg_ctx* ctx, const float* params, int64_t n_params) {
    if (!ctx || !params || n_params != kNParams) return MSG_EINVAL;
    if (!params_ok(params)) return ctx->fail(MSG_EINVAL, "non-finite parameter or non-positive feature scale");
    msg::DeviceGuard dg_(ctx->device);
    if (!dg_.ok) return ctx->fail(MSG_ECUDA, "cudaSetDevice");
    const int rc = put_model(ctx, params, ctx->band_wts, ctx->band_nrm);
    if (rc == MSG_OK) ctx->band_loaded = true;
    return rc;
}

extern "C" int msg_band_collect(msg_ctx* ctx, const msg_read_batch* reads, const msg_map_params* params, float* feat,
                                int32_t* label, int64_t cap, int64_t* n_chain) {
    if (!ctx || !reads || !params || !n_chain || cap < 0 || (cap > 0 && (!feat || !label))) return MSG_EINVAL;
    if (!ctx->idx.loaded) return ctx->fail(MSG_ESTATE, "no index loaded");
    msg::DeviceGuard dg_(ctx->device);
    if (!dg_.ok) return ctx->fail(MSG_ECUDA, "cudaSetDevice");
    int rc = upload_reads(ctx, reads);
    if (rc != MSG_OK) return rc;
    BandCollect bc{feat, label, cap, n_chain};
    msg_aln_out out{};
    return map_impl(ctx, ctx->reads.as<uint8_t>(), ctx->offs.as<int64_t>(), reads->n_reads, params, &out, nullptr, &bc);
}

extern "C" int msg_band_grad(msg_ctx* ctx, const float* params, const float* feat, const int32_t* label, int64_t n,
                             float* grad, float* loss) {
    if (!ctx || !params || !feat || !label || n <= 0 || n > INT32_MAX || !grad || !loss) return MSG_EINVAL;
    if (!params_ok(params)) return ctx->fail(MSG_EINVAL, "non-finite parameter or non-positive feature scale");
    for (int64_t k = 0; k < n; ++k) if (label[k] < 0 || label[k] >= kCls) return MSG_EINVAL;
    msg::DeviceGuard dg_(ctx->device);
    if (!dg_.ok) return ctx->fail(MSG_ECUDA, "cudaSetDevice");
    int rc = grad_smem_ready(ctx);
    if (rc != MSG_OK) return rc;
    msg::DevBuf& wts = ctx->tr_ord;  // bf16 weights of this call
    rc = put_model(ctx, params, wts, ctx->tr_m);
    if (rc != MSG_OK) return rc;
    rc = put_samples(ctx, feat, label, n, params);
    if (rc != MSG_OK) return rc;
    cudaStream_t st = ctx->stream;
    float* d_loss = ctx->tr_loss.as<float>();
    cudaError_t e = cudaMemsetAsync(ctx->tr_g.p, 0, kNTrain * sizeof(float), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_loss, 0, sizeof(float), st);
    if (e != cudaSuccess) return ctx->cuda_fail(e);
    k_mlp_grad<<<(unsigned)nblk(n, kTile), kTile, kGradSmem, st>>>(ctx->tr_x.as<float>(), ctx->tr_y.as<int32_t>(), nullptr, 0,
                                                              n, wts.as<__nv_bfloat16>(), (float)(1.0 / (double)n),
                                                              ctx->tr_g.as<float>(), d_loss);
    e = cudaGetLastError();
    float h_loss = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(grad, ctx->tr_g.p, kNTrain * sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_loss, d_loss, sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return ctx->cuda_fail(e);
    *loss = (float)((double)h_loss / (double)n);
    return MSG_OK;
}

extern "C" int msg_band_train(msg_ctx* ctx, const float* feat, const int32_t* label, int64_t n,
                              const msg_band_train_params* tp, float* params, float* loss) {
    if (!ctx || !feat || !label || !tp || !params || n <= 0 || n > INT32_MAX) return MSG_EINVAL;
    if (tp->epochs <= 0 || tp->batch <= 0 || !(tp->lr > 0)) return MSG_EINVAL;
    for (int64_t k = 0; k < n; ++k) if (label[k] < 0 || label[k] >= kCls) return MSG_EINVAL;
    msg::DeviceGuard dg_(ctx->device);
    if (!dg_.ok) return ctx->fail(MSG_ECUDA, "cudaSetDevice");
    // feature mean and scale from the data
    for (int i = 0; i < kFeat; ++i) {
        double m = 0, v = 0;
        for (int64_t k = 0; k < n; ++k) m += feat[k * kFeat + i];
        m /= (double)n;
        for (int64_t k = 0; k < n; ++k) { const double d = feat[k * kFeat + i] - m; v += d * d; }
        const double sd = std::sqrt(v / (double)n);
        params[kOffMu + i] = (float)m;
        params[kOffSd + i] = sd > 1e-6 ? (float)sd : 1.0f;
    }
    // He-normal initialisation (Box-Muller on splitmix64), zero biases
    uint64_t rs = tp->seed;
    auto normal = [&]() { return std::sqrt(-2.0 * std::log(unit01(rs))) * std::cos(6.283185307179586 * unit01(rs)); };
    for (int k = kOffW1; k < kNParams; ++k) params[k] = 0.0f;
    for (int k = 0; k < kHid * kFeat; ++k) params[kOffW1 + k] = (float)(normal() * std::sqrt(2.0 / kFeat));
    for (int k = 0; k < kHid * kHid; ++k) params[kOffW2 + k] = (float)(normal() * std::sqrt(2.0 / kHid));
    for (int k = 0; k < kCls * kHid; ++k) params[kOffW3 + k] = (float)(normal() * std::sqrt(1.0 / kHid));
    int rc = grad_smem_ready(ctx);
    if (rc != MSG_OK) return rc;
    rc = put_samples(ctx, feat, label, n, params);
    if (rc != MSG_OK) return rc;
    cudaStream_t st = ctx->stream;
    cudaError_t e = ctx->tr_w.ensure(kNTrain * sizeof(float));
    if (e == cudaSuccess) e = ctx->tr_m.ensure(2 * kNTrain * sizeof(float));
    if (e == cudaSuccess) e = ctx->tr_ord.ensure(n * sizeof(int32_t) + kNTrain * sizeof(__nv_bfloat16) + 64);
    if (e == cudaSuccess) e = ctx->tr_g.ensure(kNTrain * sizeof(float));
    if (e != cudaSuccess) return ctx->cuda_fail(e);
    float* d_w = ctx->tr_w.as<float>();
    float* d_m = ctx->tr_m.as<float>();
    float* d_v = d_m + kNTrain;
    int32_t* d_ord = ctx->tr_ord.as<int32_t>();
    __nv_bfloat16* d_wb = reinterpret_cast<__nv_bfloat16*>(ctx->tr_ord.as<uint8_t>() + (n * sizeof(int32_t) + 15) / 16 * 16);
    float* d_loss = ctx->tr_loss.as<float>();
    e = cudaMemcpyAsync(d_w, params + kOffW1, kNTrain * sizeof(float), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_m, 0, 2 * kNTrain * sizeof(float), st);
    if (e != cudaSuccess) return ctx->cuda_fail(e);
    k_to_bf16<<<nblk(kNTrain, 256), 256, 0, st>>>(kNTrain, d_w, d_wb);
    std::vector<int32_t> ord(n);
    for (int64_t k = 0; k < n; ++k) ord[k] = (int32_t)k;
    const float b1 = 0.9f, b2 = 0.999f;
    double p1 = 1.0, p2 = 1.0;
    for (int ep = 0; ep < tp->epochs; ++ep) {
        for (int64_t k = n - 1; k > 0; --k) std::swap(ord[k], ord[splitmix64(rs) % (uint64_t)(k + 1)]);
        e = cudaMemcpyAsync(d_ord, ord.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(d_loss, 0, sizeof(float), st);
        if (e != cudaSuccess) return ctx->cuda_fail(e);
        for (int64_t b0 = 0; b0 < n; b0 += tp->batch) {
            const int64_t b1e = std::min<int64_t>(n, b0 + tp->batch);
            e = cudaMemsetAsync(ctx->tr_g.p, 0, kNTrain * sizeof(float), st);
            if (e != cudaSuccess) return ctx->cuda_fail(e);
            k_mlp_grad<<<(unsigned)nblk(b1e - b0, kTile), kTile, kGradSmem, st>>>(
                ctx->tr_x.as<float>(), ctx->tr_y.as<int32_t>(), d_ord, b0, b1e, d_wb, (float)(1.0 / (double)(b1e - b0)),
                ctx->tr_g.as<float>(), d_loss);
            p1 *= b1;
            p2 *= b2;
            k_adam<<<nblk(kNTrain, 256), 256, 0, st>>>(kNTrain, d_w, d_wb, ctx->tr_g.as<float>(), d_m, d_v, tp->lr, b1, b2,
                                                       1e-8f, (float)(1.0 - p1), (float)(1.0 - p2));
        }
        e = cudaGetLastError();
        float h_loss = 0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(&h_loss, d_loss, sizeof(float), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return ctx->cuda_fail(e);
        if (loss) loss[ep] = (float)((double)h_loss / (double)n);
    }
    e = cudaMemcpyAsync(params + kOffW1, d_w, kNTrain * sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return ctx->cuda_fail(e);
    return msg_band_model_set(ctx, params, kNParams);
}

extern "C" int msg_result_device(const msg_ctx* ctx, const msg_aln** aln, const uint32_t** cigar,
                                 const int64_t** read_aln_off) {
    if (!ctx) return MSG_EINVAL;
    if (aln) *aln = ctx->res_aln;
    if (cigar) *cigar = ctx->res_cigar;
    if (read_aln_off) *read_aln_off = ctx->res_off;
    return MSG_OK;
}

extern "C" int msg_ctx_set_scratch_limit(msg_ctx* ctx, int64_t bytes) {
    if (!ctx || bytes <= 0) return MSG_EINVAL;
    ctx->scratch_limit = bytes;
    return MSG_OK;
}

extern "C" int msg_ctx_set_dp_shape(msg_ctx* ctx, int32_t stripe_rows, int64_t small_area, int64_t warp_area) {
    if (!ctx || (stripe_rows != 8 && stripe_rows != 16 && stripe_rows != 32) || small_area < 0 || warp_area < 0)
        return MSG_EINVAL;
    ctx->dp_k = stripe_rows;
    ctx->dp_small_area = small_area;
    ctx->dp_warp_area = warp_area;
    return MSG_OK;
}

extern "C" int msg_ctx_set_dp_occupancy(msg_ctx* ctx, int32_t blocks) {
    if (!ctx || (blocks != 3 && blocks != 4)) return MSG_EINVAL;
    ctx->dp_stripe_blocks = blocks;
    return MSG_OK;
}

extern "C" int msg_ctx_set_dp_lanes(msg_ctx* ctx, int32_t bits) {
    if (!ctx || (bits != 16 && bits != 32)) return MSG_EINVAL;
    ctx->dp_lanes = bits;
    return MSG_OK;
}

extern "C" int msg_ctx_set_smem_shape(msg_ctx* ctx, int32_t variant) {
    if (!ctx || variant < 0 || variant > 7) return MSG_EINVAL;
    ctx->smem_ff = variant == 7;
    ctx->smem_variant = variant == 7 ? 0 : variant;
    return MSG_OK;
}

extern "C" int msg_autotune(msg_ctx* ctx, const msg_read_batch* sample, const msg_map_params* params,
                            msg_tune* result) {
    if (!ctx || !sample || !params || !result) return MSG_EINVAL;
    if (!ctx->idx.loaded) return ctx->fail(MSG_ESTATE, "no index loaded");
    msg::DeviceGuard dg_(ctx->device);
    if (!dg_.ok) return ctx->fail(MSG_ECUDA, "cudaSetDevice");
    int rc = upload_reads(ctx, sample);
    if (rc != MSG_OK) return rc;
    int n_tried = 0;
    // stage times of one shape: an untimed run, then the timed one
    int best_lanes = 16, best_blocks = 3;
    auto time_shape = [&](int var, int k, int64_t small, int64_t warp, double* ms_smem, double* ms_dp) -> int {
        ctx->dp_lanes = best_lanes;
        ctx->dp_stripe_blocks = best_blocks;
        ctx->smem_ff = var == 7;
        ctx->smem_variant = var == 7 ? 0 : var;
        ctx->dp_k = k;
        ctx->dp_small_area = small;
        ctx->dp_warp_area = warp;
        for (int rep = 0; rep < 2; ++rep) {
            msg_aln_out dev{};  // results stay on the device
            const int r = map_impl(ctx, ctx->reads.as<uint8_t>(), ctx->offs.as<int64_t>(), sample->n_reads, params,
                                   &dev, nullptr);
            if (r != MSG_OK) return r;
        }
        ++n_tried;
        *ms_smem = ctx->stats.ms_smem;
        *ms_dp = ctx->stats.ms_dp;
        return MSG_OK;
    };
    int best_var = 0, best_k = 16;
    int64_t best_small = 64, best_warp = 262144;
    double best_smem = 0, best_dp = 0, ts = 0, td = 0;
    if ((rc = time_shape(best_var, best_k, best_small, best_warp, &best_smem, &best_dp)) != MSG_OK) return rc;
    const double smem_default = best_smem, dp_default = best_dp;
    for (int var : {1, 2, 3, 4, 5, 6, 7}) {
        if ((rc = time_shape(var, best_k, best_small, best_warp, &ts, &td)) != MSG_OK) return rc;
        if (ts < best_smem) { best_smem = ts; best_var = var; }
    }
    for (int64_t warp : {4096ll, 16384ll, 65536ll}) {
        if ((rc = time_shape(best_var, best_k, best_small, warp, &ts, &td)) != MSG_OK) return rc;
        if (td < best_dp) { best_dp = td; best_warp = warp; }
    }
    for (int k : {8, 32}) {
        if ((rc = time_shape(best_var, k, best_small, best_warp, &ts, &td)) != MSG_OK) return rc;
        if (td < best_dp) { best_dp = td; best_k = k; }
    }
    for (int64_t small : {0ll, 256ll, 1024ll}) {
        if ((rc = time_shape(best_var, best_k, small, best_warp, &ts, &td)) != MSG_OK) return rc;
        if (td < best_dp) { best_dp = td; best_small = small; }
    }
    best_lanes = 32;  // the 32-bit fill for every stripe chain
    if ((rc = time_shape(best_var, best_k, best_small, best_warp, &ts, &td)) != MSG_OK) return rc;
    if (td < best_dp) best_dp = td;
    else best_lanes = 16;
    best_blocks = best_blocks == 3 ? 4 : 3;  // the other register budget of the stripe kernel
    if ((rc = time_shape(best_var, best_k, best_small, best_warp, &ts, &td)) != MSG_OK) return rc;
    if (td < best_dp) best_dp = td;
    else best_blocks = best_blocks == 3 ? 4 : 3;
    ctx->dp_lanes = best_lanes;
    ctx->dp_stripe_blocks = best_blocks;
    ctx->smem_ff = best_var == 7;
    ctx->smem_variant = best_var == 7 ? 0 : best_var;
    ctx->dp_k = best_k;
    ctx->dp_small_area = best_small;
    ctx->dp_warp_area = best_warp;
    result->stripe_rows = best_k;
    result->small_area = best_small;
    result->warp_area = best_warp;
    result->ms_dp = best_dp;
    result->ms_dp_default = dp_default;
    result->smem_variant = best_var;
    result->dp_lanes = best_lanes;
    result->dp_stripe_blocks = best_blocks;
    result->ms_smem = best_smem;
    result->ms_smem_default = smem_default;
    result->n_tried = n_tried;
    return MSG_OK;
}

extern "C" int msg_ctx_stream(const msg_ctx* ctx, void** stream) {
    if (!ctx || !stream) return MSG_EINVAL;
    *stream = (void*)ctx->stream;
    return MSG_OK;
}

extern "C" int msg_last_stats(const msg_ctx* ctx, msg_map_stats* stats) {
    if (!ctx || !stats) return MSG_EINVAL;
    *stats = ctx->stats;
    return MSG_OK;
}

// ---------------------------------------------------------------------------
// Seeding without device allocation. The per-warp candidate lists and the
// launch counters of k_smem live in one file-scope device array, so this entry
// point needs no cudaMalloc/cudaFree (nor any allocating library routine).
// ---------------------------------------------------------------------------
namespace {
constexpr int64_t kStaticMaxReadLen = MSG_NOALLOC_MAX_READ_LEN;
constexpr int64_t kStaticWarps = MSG_NOALLOC_WARPS;
constexpr int64_t kStaticPvCap = kStaticMaxReadLen + 2;
constexpr size_t kStaticHdr = 256;  // work counter, extension counter, max read length, status word
constexpr size_t kStaticBytes = kStaticHdr + (size_t)kStaticWarps * kStaticPvCap * (8 + 8 + 8 + 8 + 4);

__global__ void k_maxlen(const int64_t* __restrict__ off, int64_t n, unsigned long long* __restrict__ mx) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t l = off[i + 1] - off[i];
    atomicMax(mx, (unsigned long long)(l < 0 ? 0 : l));
}
}  // namespace

// Shared by every call on a device: contents persist between calls, so the
// header is cleared at the start of each call; calls that overlap on the GPU
// race on it.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kStaticBytes];

// Device address of g_noalloc_scratch per device ordinal. In host code the
// array's name is only a host-side stand-in, so the address is looked up with
// cudaGetSymbolAddress on the first call on each device (with that device
// current) and cached.
static void* g_noalloc_addr[256] = {nullptr};

extern "C" int msg_smem_batch_noalloc(msg_ctx* ctx, int64_t n_reads, const uint8_t* d_seq, const int64_t* d_off,
                                      const msg_map_params* params, int64_t* d_smem, int64_t cap_per_read,
                                      int32_t* d_count) {
    if (!ctx || !params || n_reads < 0 || cap_per_read < 0) return MSG_EINVAL;
    if (n_reads > 0 && (!d_seq || !d_off || !d_count || (cap_per_read > 0 && !d_smem))) return MSG_EINVAL;
    if (!ctx->idx.loaded) return ctx->fail(MSG_ESTATE, "no index loaded");
    DpParams dpp;
    int rc = check_params(params, &dpp);
    if (rc != MSG_OK) return ctx->fail(rc, "bad mapping parameters");
    double thr = 0;
    int thr_all = 0;
    rc = evalue_threshold(ctx->idx.dev.n, params->max_evalue, &thr, &thr_all);
    if (rc != MSG_OK) return ctx->fail(rc, "e-value threshold");
    if (ctx->device < 0 || ctx->device >= 256) return MSG_EINVAL;
    msg::DeviceGuard dg_(ctx->device);
    if (!dg_.ok) return ctx->fail(MSG_ECUDA, "cudaSetDevice");
    cudaError_t e = cudaSuccess;
    if (!g_noalloc_addr[ctx->device]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) return ctx->cuda_fail(e == cudaSuccess ? cudaErrorInvalidSymbol : e);
        g_noalloc_addr[ctx->device] = p;
    }
    unsigned char* base = static_cast<unsigned char*>(g_noalloc_addr[ctx->device]);
    unsigned long long* hdr = reinterpret_cast<unsigned long long*>(base);
    uint32_t* status = reinterpret_cast<uint32_t*>(hdr + 3);
    cudaStream_t st = ctx->stream;
    if (n_reads == 0) return MSG_OK;
    e = cudaMemsetAsync(base, 0, kStaticHdr, st);
    if (e != cudaSuccess) return ctx->cuda_fail(e);
    k_maxlen<<<nblk(n_reads, 256), 256, 0, st>>>(d_off, n_reads, hdr + 2);
    k_check_codes<<<ctx->num_sms * 4, 256, 0, st>>>(d_seq, d_off, n_reads, status);
    unsigned long long maxlen = 0;
    uint32_t codes = 0;
    e = cudaMemcpyAsync(&maxlen, hdr + 2, sizeof(maxlen), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&codes, status, sizeof(codes), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return ctx->cuda_fail(e);
    if ((int64_t)maxlen > kStaticMaxReadLen)
        return ctx->fail(MSG_EINVAL, "a read is longer than MSG_NOALLOC_MAX_READ_LEN");
    if (codes & kErrCodes) return ctx->fail(MSG_EINVAL, "read bytes must be nt16 codes (0..15)");
    SmemArgs sa{};
    sa.seq = d_seq; sa.off = d_off; sa.n_reads = n_reads; sa.min_len = params->min_len;
    sa.thr = thr; sa.thr_all = thr_all;
    for (int b = 0; b < 16; ++b) sa.llk[b] = ctx->idx.llk[b];
    sa.out = d_smem; sa.cap = cap_per_read; sa.count = d_count;
    unsigned char* pv = base + kStaticHdr;
    const int64_t slots = kStaticWarps * kStaticPvCap;
    sa.pv_p = reinterpret_cast<int64_t*>(pv);
    sa.pv_q = sa.pv_p + slots;
    sa.pv_s = sa.pv_q + slots;
    sa.pv_lp = reinterpret_cast<double*>(sa.pv_s + slots);
    sa.pv_pos = reinterpret_cast<int32_t*>(sa.pv_lp + slots);
    sa.pv_cap = kStaticPvCap;
    sa.work = hdr;
    sa.n_ext = hdr + 1;
    sa.status = status;
    const int blocks = (int)std::min<int64_t>(ctx->num_sms, kStaticWarps / 8);  // 8 warps per 256-thread block
    k_smem<<<blocks, 256, 0, st>>>(sa, ctx->idx.dev);
    e = cudaGetLastError();
    if (e != cudaSuccess) return ctx->cuda_fail(e);
    uint32_t h_status = 0;
    e = cudaMemcpyAsync(&h_status, status, sizeof(h_status), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return ctx->cuda_fail(e);
    if (h_status & kErrInternal) return ctx->fail(MSG_EINTERNAL, "SMEM stage consistency check failed");
    if (h_status & kErrOverflow) return ctx->fail(MSG_EINVAL, "output capacity too small; d_count holds the needed counts");
    return MSG_OK;
}
