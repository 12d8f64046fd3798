// Device kernels of the mapping pipeline (included by map.cu only).
#pragma once
#include <cstdint>

#include "../../include/msg_b200.h"
#include "msg_internal.cuh"

namespace msg {

constexpr int32_t NEG = -(1 << 30);  // the reference's -inf; absorbing under sat_add / add_s
enum { FWD = 1, REV = 2 };
enum { OP_M = 0, OP_I = 1, OP_D = 2, OP_S = 4 };

struct Seed {
    int32_t from, to, tid, strand;
    int64_t start, end;
};
static_assert(sizeof(Seed) == 32, "seed layout");

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ unsigned lanemask_lt() { return (1u << lane_id()) - 1u; }

// ======================================================================
// SMEM stage: one warp per read, lanes over the `prev` candidate list.
// ======================================================================

struct SmemArgs {
    const uint8_t* seq;
    const int64_t* off;
    int64_t n_reads;
    int64_t min_len;
    double thr;        // largest log-likelihood whose e-value passes (host-computed)
    int thr_all;       // 1 when max_evalue is +inf: every SMEM passes
    double llk[16];
    int64_t* out;      // 6 x int64 rows; read r's slot starts at row out_off[r] (r * cap when null)
    int64_t cap;       // slot rows when out_off is null
    const int64_t* out_off;  // per-read slot offsets (n + 1), or null
    const int64_t* list;     // reads handled by this launch (read k when null)
    int32_t* count;    // per read: SMEMs emitted (may exceed its slot)
    int32_t* pv_pos;   // per-warp prev lists, pv_cap entries each
    int64_t* pv_p;
    int64_t* pv_q;
    int64_t* pv_s;
    double* pv_lp;
    int64_t pv_cap;
    unsigned long long* work;
    unsigned long long* n_ext;
    uint32_t* status;
};

struct SmemState {
    int64_t from, to, p, q, s;
    double lp;
};

struct WarpSmem {
    const SmemArgs* a;
    const IndexDev* ix;
    const uint8_t* rd;
    int64_t L;
    int64_t* out;
    int32_t n_out;
    int64_t cap_r;     // rows of this read's slot
    int32_t* pv_pos;
    int64_t *pv_p, *pv_q, *pv_s;
    double* pv_lp;
    unsigned long long ext;

    __device__ int base(int64_t i) const { return (i >= 0 && i < L) ? (int)__ldg(rd + i) : 0; }

    __device__ void emit(bool cand, int64_t from, int64_t to, int64_t p, int64_t q, int64_t s, double lp) {
        const unsigned m = __ballot_sync(0xffffffffu, cand);
        if (cand) {
            const int64_t k = n_out + __popc(m & lanemask_lt());
            if (k < cap_r) {
                int64_t* o = out + 6 * k;
                o[0] = from; o[1] = to; o[2] = p; o[3] = q; o[4] = s;
                o[5] = __double_as_longlong(lp);
            }
        }
        n_out += __popc(m);
    }

    __device__ void reverse_prev(int n) {
        for (int k = lane_id(); k < n / 2; k += 32) {
            const int o = n - 1 - k;
            int32_t t0 = pv_pos[k]; pv_pos[k] = pv_pos[o]; pv_pos[o] = t0;
            int64_t t1 = pv_p[k]; pv_p[k] = pv_p[o]; pv_p[o] = t1;
            int64_t t2 = pv_q[k]; pv_q[k] = pv_q[o]; pv_q[o] = t2;
            int64_t t3 = pv_s[k]; pv_s[k] = pv_s[o]; pv_s[o] = t3;
            double t4 = pv_lp[k]; pv_lp[k] = pv_lp[o]; pv_lp[o] = t4;
        }
        __syncwarp();
    }

    // One lockstep extension of every prev entry. All entries share the outer
    // end `fixed`; pv_pos holds each entry's other end. dir 0: backward
    // extension by base b (findFwdBackSMEMS loop, SMEM.cpp:92-115); dir 1:
    // forward extension (findBackFwdSMEMS loop, SMEM.cpp:147-170). Emits the
    // SMEMs the reference pushes to `curr` and compacts the survivors.
    __device__ int step_prev(int n_prev, int dir, int64_t fixed, int b, bool add_ll) {
        int64_t carry_size = -1;
        bool found_valid = false;
        int n_keep = 0;
        const double llb = a->llk[b & 15];
        for (int base_k = 0; base_k < n_prev; base_k += 32) {
            const int k = base_k + lane_id();
            const bool act = k < n_prev;
            int32_t pos = 0;
            int64_t p = 0, q = 0, s = 0, p_old = 0, q_old = 0, s_old = 0;
            double lp = 0, lp_old = 0;
            if (act) {
                pos = pv_pos[k]; p = pv_p[k]; q = pv_q[k]; s = pv_s[k]; lp = pv_lp[k];
                p_old = p; q_old = q; s_old = s; lp_old = lp;
                if (is_basic(b)) ext++;
                if (dir == 0) back_ext(*ix, p, q, s, b); else fwd_ext(*ix, p, q, s, b);
                if (add_ll) lp = __dadd_rn(lp, llb);
            }
            const int64_t up = __shfl_up_sync(0xffffffffu, s, 1);
            const int64_t sp = lane_id() == 0 ? carry_size : up;
            const bool valid = act && s >= 1 && (k == 0 || s != sp);
            if (act && k > 0 && s >= 1 && s < sp) atomicOr(a->status, kErrInternal);  // sizes never decrease along prev
            const unsigned vb = __ballot_sync(0xffffffffu, valid);
            const int limit = vb ? __ffs(vb) - 1 : 31;
            const int64_t e_from = dir == 0 ? fixed : (int64_t)pos;
            const int64_t e_to = dir == 0 ? (int64_t)pos : fixed;
            const bool sig = a->thr_all || lp_old <= a->thr;
            const bool cand = act && !found_valid && lane_id() <= limit && s != s_old && s_old >= 1 &&
                              (e_to - e_from) >= a->min_len && sig;
            emit(cand, e_from, e_to, p_old, q_old, s_old, lp_old);
            if (vb) found_valid = true;
            __syncwarp();
            if (valid) {
                const int w = n_keep + __popc(vb & lanemask_lt());
                pv_pos[w] = pos; pv_p[w] = p; pv_q[w] = q; pv_s[w] = s; pv_lp[w] = lp;
            }
            n_keep += __popc(vb);
            const int last = min(31, n_prev - 1 - base_k);
            carry_size = __shfl_sync(0xffffffffu, s, last);
            __syncwarp();
        }
        return n_keep;
    }

    __device__ void push_prev(int& n, const SmemState& m, int32_t pos) {
        if (n < a->pv_cap) {
            pv_pos[n] = pos; pv_p[n] = m.p; pv_q[n] = m.q; pv_s[n] = m.s; pv_lp[n] = m.lp;
        } else {
            atomicOr(a->status, kErrInternal);
        }
        ++n;
    }

    __device__ SmemState init_at(int64_t from) const {
        const int b = base(from);
        SmemState m;
        m.from = from; m.to = from + 1;
        m.p = ix->C[b]; m.q = ix->C[comp16(b)]; m.s = ix->C[b + 1] - ix->C[b];
        m.lp = __dadd_rn(0.0, a->llk[b]);  // SMEM::evaluate (SMEM.cpp:19-24)
        return m;
    }

    // SMEM_LIST::findFwdBackSMEMS (SMEM.cpp:64-117). from/to are in/out.
    __device__ void fwd_back(int64_t& from, int64_t& to) {
        const int b = base(from);
        to = from + 1;
        if (!is_basic(b)) return;
        int n_prev = 0;
        int64_t end_to = 0;
        if (lane_id() == 0) {
            SmemState m = init_at(from), m0 = m;
            while (m.s >= 1) {
                const int nb = base(m.to);  // getBase(L) is the read's terminator, 0
                if (is_basic(nb)) ext++;
                fwd_ext(*ix, m.p, m.q, m.s, nb);
                if (m.to < L) m.lp = __dadd_rn(m.lp, a->llk[nb]);
                m.to++;
                if (m.s != m0.s && m0.to >= a->min_len) {
                    bool sig = a->thr_all != 0;
                    if (!sig) {  // SMEM::loglik(0, to) (SMEM.cpp:26-40); partial sums never increase
                        double ll = __dadd_rn(0.0, m0.lp);
                        sig = ll <= a->thr;
                        for (int64_t i = 0; i < m0.from && !sig; ++i) {
                            ll = __dadd_rn(ll, a->llk[base(i)]);
                            sig = ll <= a->thr;
                        }
                    }
                    if (sig) push_prev(n_prev, m0, (int32_t)m0.to);
                }
                m0 = m;
            }
            end_to = m.to;
        }
        n_prev = __shfl_sync(0xffffffffu, n_prev, 0);
        to = __shfl_sync(0xffffffffu, end_to, 0);
        __syncwarp();
        if (n_prev > a->pv_cap) return;
        if (n_prev == 0) { from--; return; }
        reverse_prev(n_prev);
        while (from >= 0 && n_prev > 0) {
            const int b2 = from > 0 ? base(from - 1) : 0;
            n_prev = step_prev(n_prev, 0, from, b2, from > 0);
            from--;
        }
    }

    // SMEM_LIST::findBackFwdSMEMS (SMEM.cpp:119-172). from/to are in/out.
    __device__ void back_fwd(int64_t& from, int64_t& to) {
        const int b = base(from);
        to = from + 1;
        if (!is_basic(b)) return;
        int n_prev = 0;
        int64_t end_from = 0;
        if (lane_id() == 0) {
            SmemState m = init_at(from), m0 = m;
            while (m.s >= 1) {
                const int nb = m.from > 0 ? base(m.from - 1) : 0;
                if (is_basic(nb)) ext++;
                back_ext(*ix, m.p, m.q, m.s, nb);
                if (m.from > 0) m.lp = __dadd_rn(m.lp, a->llk[nb]);
                m.from--;
                if (m.s != m0.s && L - m0.from >= a->min_len) {
                    bool sig = a->thr_all != 0;
                    if (!sig) {  // SMEM::loglik(from, L); partial sums never increase
                        double ll = __dadd_rn(0.0, m0.lp);
                        sig = ll <= a->thr;
                        for (int64_t i = m0.to; i < L && !sig; ++i) {
                            ll = __dadd_rn(ll, a->llk[base(i)]);
                            sig = ll <= a->thr;
                        }
                    }
                    if (sig) push_prev(n_prev, m0, (int32_t)m0.from);
                }
                m0 = m;
            }
            end_from = m.from;
        }
        n_prev = __shfl_sync(0xffffffffu, n_prev, 0);
        from = __shfl_sync(0xffffffffu, end_from, 0);
        __syncwarp();
        if (n_prev > a->pv_cap) return;
        if (n_prev == 0) { to++; return; }
        reverse_prev(n_prev);
        while (to <= L && n_prev > 0) {
            const int b2 = base(to);
            n_prev = step_prev(n_prev, 1, to, b2, to < L);
            to++;
        }
    }

    // SMEM_LIST::findAllSMEMS (SMEM.cpp:186-215)
    __device__ void find_all() {
        int64_t from = L / 2;
        int64_t to = from + 1;
        fwd_back(from, to);
        while (from > 0 || to < L) {
            int64_t from0 = to;
            if (from0 < L) fwd_back(from0, to);
            from -= 1;
            int64_t to0 = from + 1;
            if (from >= 0) back_fwd(from, to0);
        }
    }
};

__global__ void __launch_bounds__(256) k_smem(SmemArgs a, IndexDev ix) {
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    WarpSmem w;
    w.a = &a;
    w.ix = &ix;
    w.pv_pos = a.pv_pos + warp * a.pv_cap;
    w.pv_p = a.pv_p + warp * a.pv_cap;
    w.pv_q = a.pv_q + warp * a.pv_cap;
    w.pv_s = a.pv_s + warp * a.pv_cap;
    w.pv_lp = a.pv_lp + warp * a.pv_cap;
    w.ext = 0;
    for (;;) {
        unsigned long long r = 0;
        if (lane_id() == 0) r = atomicAdd(a.work, 1ull);
        r = __shfl_sync(0xffffffffu, r, 0);
        if ((int64_t)r >= a.n_reads) break;
        if (a.list) r = (unsigned long long)a.list[r];
        const int64_t o0 = a.off[r];
        w.rd = a.seq + o0;
        w.L = a.off[r + 1] - o0;
        const int64_t slot = a.out_off ? a.out_off[r] : (int64_t)r * a.cap;
        w.cap_r = a.out_off ? a.out_off[r + 1] - slot : a.cap;
        w.out = a.out + 6 * slot;
        w.n_out = 0;
        if (w.L > 0) w.find_all();
        if (lane_id() == 0) {
            a.count[r] = w.n_out;
            if (w.n_out > w.cap_r) atomicOr(a.status, kErrOverflow);
        }
    }
    // lanes count their own extensions
    unsigned long long e = w.ext;
    for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
    if (lane_id() == 0 && e) atomicAdd(a.n_ext, e);
}

// Copy each read's SMEMs from its slot (slot_off) into a dense array (read r
// at smem_off[r]). One warp per read.
__global__ void k_compact_smem(const int64_t* __restrict__ src, const int64_t* __restrict__ slot_off,
                               const int32_t* __restrict__ count, const int64_t* __restrict__ smem_off,
                               int64_t n_reads, int64_t* __restrict__ dst) {
    const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (r >= n_reads) return;
    const int64_t n = min((int64_t)count[r], slot_off[r + 1] - slot_off[r]);
    for (int64_t j = lane_id(); j < 6 * n; j += 32) dst[6 * smem_off[r] + j] = src[6 * slot_off[r] + j];
}

// Reads up to max_len bp into `short_list`, longer ones into `long_list`.
__global__ void k_split_len(const int64_t* __restrict__ len, int64_t n, int64_t max_len,
                            int64_t* __restrict__ short_list, int64_t* __restrict__ long_list,
                            unsigned long long* __restrict__ counts) {
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= n) return;
    if (len[r] <= max_len) short_list[atomicAdd(&counts[0], 1ull)] = r;
    else long_list[atomicAdd(&counts[1], 1ull)] = r;
}

// SMEM slot rows per read: cap per 150 bases, at least cap.
constexpr int64_t kSlotBases = 150;
__global__ void k_slot_rows(const int64_t* __restrict__ len, int64_t n, int64_t cap, int64_t* __restrict__ rows) {
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r < n) rows[r] = max(cap, (len[r] * cap + kSlotBases - 1) / kSlotBases);
}

// ======================================================================
// Seed selection: SMEM_LIST::findSeeds locates SMEMs in ascending loglik
// order and stops after the SMEM that brings the located count to maxNSeed
// (SMEM.cpp:275-300). Every SMEM contributes exactly `size` seeds
// (assert at SMEM.cpp:267), so when all but the smallest SMEM hold fewer than
// maxNSeed seeds the order cannot matter and all are selected. Otherwise the
// read is flagged for the host, which runs the same std::sort.
// ======================================================================
__global__ void k_select(const int64_t* __restrict__ smem, const int64_t* __restrict__ smem_off, int64_t n_reads,
                         int64_t max_nseed, uint8_t* __restrict__ sel, int32_t* __restrict__ host_flag,
                         unsigned long long* __restrict__ n_flagged) {
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= n_reads) return;
    const int64_t a = smem_off[r], b = smem_off[r + 1];
    int64_t tot = 0, mn = INT64_MAX;
    for (int64_t k = a; k < b; ++k) {
        const int64_t s = smem[6 * k + 4];
        tot += s;
        mn = min(mn, s);
    }
    const bool all = (b == a) || (tot - mn < max_nseed);
    for (int64_t k = a; k < b; ++k) sel[k] = all ? 1 : 0;
    host_flag[r] = all ? 0 : 1;
    if (!all) atomicAdd(n_flagged, 1ull);
}

__global__ void k_seed_counts(const int64_t* __restrict__ smem, const uint8_t* __restrict__ sel, int64_t n,
                              int64_t* __restrict__ cnt) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    cnt[k] = sel[k] ? smem[6 * k + 4] : 0;
}

// ======================================================================
// Locate: SMEM::getSeeds over the selected SMEMs. One thread per SA-row
// pair (fwdStart + i, revStart + i); the full suffix array is resident, so
// accessSA is a single gather. getTid's linear scan over disjoint chromosome
// spans equals a binary search over their starts.
// ======================================================================
__device__ __forceinline__ int64_t chrom_of(const IndexDev& ix, int64_t pos) {
    int64_t a = 0, b = ix.n_chrom;
    while (b - a > 1) {
        const int64_t m = (a + b) >> 1;
        if (__ldg(ix.bd_start + m) <= pos) a = m; else b = m;
    }
    return a;
}

__global__ void k_locate(IndexDev ix, const int64_t* __restrict__ smem, const int64_t* __restrict__ smem_seed_off,
                         const int32_t* __restrict__ smem_read, const int64_t* __restrict__ read_off, int64_t n_smem,
                         int64_t total, int32_t* __restrict__ fill, Seed* __restrict__ seeds,
                         uint32_t* __restrict__ status) {
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < total; g += (int64_t)gridDim.x * blockDim.x) {
        int64_t a = 0, b = n_smem;  // last k with smem_seed_off[k] <= g
        while (b - a > 1) {
            const int64_t m = (a + b) >> 1;
            if (smem_seed_off[m] <= g) a = m; else b = m;
        }
        const int64_t k = a;
        const int64_t i = g - smem_seed_off[k];
        const int64_t* m = smem + 6 * k;
        const int64_t from = m[0], to = m[1], len = to - from;
        const int32_t r = smem_read[k];
        const int64_t L = read_off[r + 1] - read_off[r];
        for (int side = 0; side < 2; ++side) {
            const int64_t row = (side == 0 ? m[2] : m[3]) + i;
            const int64_t bd = (int64_t)__ldg(ix.sa + row);
            const int64_t tid = chrom_of(ix, bd);
            const int64_t st = ix.bd_start[tid], en = ix.bd_end[tid];
            const bool fwd = st <= bd && bd < st + (en - st) / 2;
            if (!fwd) continue;
            const int64_t loc = bd - st;
            const int32_t slot = atomicAdd(&fill[k], 1);
            if (slot >= m[4]) { atomicOr(status, kErrInternal); continue; }
            Seed s;
            if (side == 0) { s.from = (int32_t)from; s.to = (int32_t)to; s.strand = FWD; }
            else { s.from = (int32_t)(L - to); s.to = (int32_t)(L - to + len); s.strand = REV; }
            s.tid = (int32_t)tid;
            s.start = loc;
            s.end = loc + len;
            seeds[smem_seed_off[k] + slot] = s;
        }
    }
}

// ======================================================================
// Redundant-seed removal, one warp per read: rank sort by SeedPair's
// operator< (SeedPair.h:225-232), then a seed is dropped when any later seed
// contains it or is contained by it (SeedPair::approxEqual, SeedPair.h:171-185).
// ======================================================================
__device__ __forceinline__ bool seed_less(const Seed& l, const Seed& r) {
    if (l.from != r.from) return l.from < r.from;
    if (l.to != r.to) return l.to < r.to;
    if (l.tid != r.tid) return l.tid < r.tid;
    if (l.strand != r.strand) return l.strand < r.strand;
    if (l.start != r.start) return l.start < r.start;
    return l.end < r.end;
}
__device__ __forceinline__ bool containing(const Seed& l, const Seed& r) {
    return l.tid == r.tid && l.strand == r.strand && l.from <= r.from && l.to >= r.to && l.start <= r.start &&
           l.end >= r.end;
}

__global__ void k_dedup(const int64_t* __restrict__ read_seed_off, int64_t n_reads, const Seed* __restrict__ in,
                        Seed* __restrict__ tmp, Seed* __restrict__ out, int32_t* __restrict__ n_out) {
    const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (r >= n_reads) return;
    const int64_t a = read_seed_off[r];
    const int64_t n = read_seed_off[r + 1] - a;
    for (int64_t i = lane_id(); i < n; i += 32) {
        const Seed si = in[a + i];
        int64_t rank = 0;
        for (int64_t j = 0; j < n; ++j) {
            const Seed sj = in[a + j];
            if (seed_less(sj, si) || (j < i && !seed_less(si, sj))) rank++;
        }
        tmp[a + rank] = si;
    }
    __syncwarp();
    int64_t kept = 0;
    for (int64_t base = 0; base < n; base += 32) {
        const int64_t i = base + lane_id();
        bool keep = false;
        Seed si;
        if (i < n) {
            si = tmp[a + i];
            keep = true;
            for (int64_t j = i + 1; j < n; ++j) {
                const Seed sj = tmp[a + j];
                if (containing(si, sj) || containing(sj, si)) { keep = false; break; }
            }
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (keep) out[a + kept + __popc(m & lanemask_lt())] = si;
        kept += __popc(m);
    }
    if (lane_id() == 0) n_out[r] = (int32_t)kept;
}

// ======================================================================
// Chaining: SeedChain::getChains / dfsSeeds with the recursion on an explicit
// stack; same visiting order. One thread per read, two passes (count, emit).
// ======================================================================
__device__ __forceinline__ int64_t loc_dist(int64_t ls, int64_t le, int64_t rs, int64_t re) {  // Loc.h:89-91
    const bool ov = ls < re && le > rs;
    return ov ? 0 : ls < rs ? rs - le + 1 : ls - re + 1;
}

__device__ __forceinline__ bool chain_ok(const Seed& l, const Seed& r, int64_t max_mm, int64_t max_indel) {
    // SeedPair::isCompatitable / nMismatch / nIndel (SeedPair.h:136-158)
    if (!(l.to <= r.from && l.end <= r.start && l.tid == r.tid && l.strand == r.strand)) return false;
    const int64_t mm = min(loc_dist(l.from, l.to, r.from, r.to), loc_dist(l.start, l.end, r.start, r.end));
    if (mm > max_mm) return false;
    int64_t ind = (int64_t)(r.from - l.to) - (r.start - l.end);
    if (ind < 0) ind = -ind;
    return ind <= max_indel;
}

// Reads with more seeds than this chain on a warp each (k_chain_warp), the
// others on a thread each (k_chain).
constexpr int64_t kChainThreadSeeds = 32;

__global__ void k_chain(const int64_t* __restrict__ read_seed_off, const int32_t* __restrict__ n_seed,
                        const int64_t* __restrict__ read_len, int64_t n_reads, const Seed* __restrict__ seeds,
                        uint8_t* __restrict__ visited, int32_t* __restrict__ stk_i, int32_t* __restrict__ stk_j,
                        int pass, int64_t* __restrict__ n_chain, int64_t* __restrict__ n_idx,
                        const int64_t* __restrict__ chain_off, const int64_t* __restrict__ idx_off,
                        int64_t* __restrict__ chain_idx_off, int32_t* __restrict__ chain_len,
                        int32_t* __restrict__ chain_read, int64_t* __restrict__ chain_idx) {
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= n_reads) return;
    const int64_t a = read_seed_off[r];
    const int64_t N = n_seed[r];
    if (N > kChainThreadSeeds) return;  // k_chain_warp's
    const int64_t L = read_len[r];
    // msgseqtk-align.cpp:619-620
    const int64_t max_mm = (int64_t)ceil(__dmul_rn((double)L, 0.2));
    const int64_t max_indel = (int64_t)ceil(__dmul_rn((double)L, 0.1));
    uint8_t* vis = visited + a;
    int32_t* si = stk_i + a;
    int32_t* sj = stk_j + a;
    for (int64_t i = 0; i < N; ++i) vis[i] = 0;
    int64_t nc = 0, ni = 0;
    int64_t c_base = pass ? chain_off[r] : 0;
    int64_t i_base = pass ? idx_off[r] : 0;
    for (int64_t root = 0; root < N; ++root) {
        if (vis[root]) continue;
        vis[root] = 1;
        int depth = 0;
        si[0] = (int32_t)root; sj[0] = (int32_t)(root + 1);
        // leaf flag kept in the sign of stk_j: negative once a child was taken
        while (depth >= 0) {
            const int64_t i = si[depth];
            int64_t j = sj[depth] < 0 ? -(int64_t)sj[depth] - 1 : sj[depth];
            const bool had_child = sj[depth] < 0;
            bool descended = false;
            const Seed s_i = seeds[a + i];
            while (j < N) {
                const int64_t jj = j++;
                if (!vis[jj] && chain_ok(s_i, seeds[a + jj], max_mm, max_indel)) {
                    sj[depth] = (int32_t)(-(j) - 1);  // resume at j, child taken
                    vis[jj] = 1;
                    ++depth;
                    si[depth] = (int32_t)jj;
                    sj[depth] = (int32_t)(jj + 1);
                    descended = true;
                    break;
                }
            }
            if (descended) continue;
            if (!had_child) {  // leaf: emit the current stack as a chain
                if (pass) {
                    chain_idx_off[c_base + nc] = i_base + ni;
                    chain_len[c_base + nc] = depth + 1;
                    chain_read[c_base + nc] = (int32_t)r;
                    for (int d = 0; d <= depth; ++d) chain_idx[i_base + ni + d] = a + si[d];
                }
                nc++;
                ni += depth + 1;
            }
            --depth;
        }
    }
    if (!pass) { n_chain[r] = nc; n_idx[r] = ni; }
}

// SeedChain::getChains / dfsSeeds (SeedChain.cpp:40-73) for reads with more
// than kChainThreadSeeds seeds, one warp per read: the DFS is k_chain's
// (same order, same chains), but each search for the next unvisited
// compatible seed tests 32 candidates at once and takes the first by ballot,
// which turns the serial O(N^2) scans of seed-rich reads (repeats) into
// N^2 / 32 steps. Lane 0 keeps the stack and visited flags in memory; the
// warp keeps depth and the resume point in registers.
__global__ void k_chain_warp(const int64_t* __restrict__ read_seed_off, const int32_t* __restrict__ n_seed,
                             const int64_t* __restrict__ read_len, int64_t n_reads, const Seed* __restrict__ seeds,
                             uint8_t* __restrict__ visited, int32_t* __restrict__ stk_i, int32_t* __restrict__ stk_j,
                             int pass, int64_t* __restrict__ n_chain, int64_t* __restrict__ n_idx,
                             const int64_t* __restrict__ chain_off, const int64_t* __restrict__ idx_off,
                             int64_t* __restrict__ chain_idx_off, int32_t* __restrict__ chain_len,
                             int32_t* __restrict__ chain_read, int64_t* __restrict__ chain_idx) {
    const int lane = threadIdx.x & 31;
    const int64_t n_warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; r < n_reads; r += n_warps) {
        const int64_t N = n_seed[r];
        if (N <= kChainThreadSeeds) continue;
        const int64_t a = read_seed_off[r];
        const int64_t L = read_len[r];
        const int64_t max_mm = (int64_t)ceil(__dmul_rn((double)L, 0.2));  // msgseqtk-align.cpp:619-620
        const int64_t max_indel = (int64_t)ceil(__dmul_rn((double)L, 0.1));
        uint8_t* vis = visited + a;
        int32_t* si = stk_i + a;
        const Seed* sd = seeds + a;
        for (int64_t i = lane; i < N; i += 32) vis[i] = 0;
        __syncwarp();
        int64_t nc = 0, ni = 0;
        const int64_t c_base = pass ? chain_off[r] : 0;
        const int64_t i_base = pass ? idx_off[r] : 0;
        for (int64_t root = 0; root < N; ++root) {
            if (vis[root]) continue;  // every lane reads the same flag
            __syncwarp();
            if (lane == 0) { vis[root] = 1; si[0] = (int32_t)root; }
            int depth = 0;
            int64_t j = root + 1;   // resume point of the top frame
            bool had_child = false; // the top frame has descended once
            // resume points and child flags of the frames below, on the stack
            int32_t* sj = stk_j + a;
            __syncwarp();
            while (depth >= 0) {
                const int64_t i = si[depth];
                const Seed s_i = sd[i];
                int64_t found = -1;
                for (int64_t base = j; base < N; base += 32) {
                    const int64_t jj = base + lane;
                    const bool ok = jj < N && !vis[jj] && chain_ok(s_i, sd[jj], max_mm, max_indel);
                    const unsigned m = __ballot_sync(0xffffffffu, ok);
                    if (m) { found = base + __ffs(m) - 1; break; }
                }
                if (found >= 0) {  // descend
                    if (lane == 0) {
                        sj[depth] = (int32_t)(-(found + 1) - 1);  // resume after it, child taken
                        vis[found] = 1;
                        si[depth + 1] = (int32_t)found;
                    }
                    __syncwarp();
                    ++depth;
                    j = found + 1;
                    had_child = false;
                    continue;
                }
                if (!had_child) {  // leaf: emit the current stack as a chain
                    if (pass) {
                        if (lane == 0) {
                            chain_idx_off[c_base + nc] = i_base + ni;
                            chain_len[c_base + nc] = depth + 1;
                            chain_read[c_base + nc] = (int32_t)r;
                        }
                        for (int d = lane; d <= depth; d += 32) chain_idx[i_base + ni + d] = a + si[d];
                    }
                    nc++;
                    ni += depth + 1;
                }
                --depth;
                if (depth >= 0) {  // back to the frame below: its resume point and child flag
                    const int32_t v = sj[depth];
                    had_child = v < 0;
                    j = v < 0 ? -(int64_t)v - 1 : v;
                }
                __syncwarp();
            }
        }
        if (!pass && lane == 0) { n_chain[r] = nc; n_idx[r] = ni; }
        __syncwarp();
    }
}

// ======================================================================
// DP. The reference fills three (L+1) x (tLen+1) double matrices with -inf and
// writes them in a fixed order (Alignment.cpp:54-171): 5' rectangle, then per
// seed [clear its block, diagonal, the cell past it, I.row(to+1) = M.row(to)+o,
// D.col(end+1) = M.col(end)+o], the gap rectangle to the next seed, and the 3'
// rectangle. Rectangles and seed blocks are disjoint, so the final value of
// any cell is given by the last region in that order that writes it; a query
// made while computing region m only looks at regions written before m, which
// is the state the reference saw at that point. No rectangle's boundary lies
// inside another rectangle, so rectangles are filled from derived values only.
//
// Per rectangle cell only a 1-byte traceback code is stored (the decisions the
// reference's matchMax/insMax/delMax would take there, and M > 0 for local
// mode); full M/I/D values are kept for the rectangle's last row and column,
// the only rectangle cells a traceback can reach from outside.
// ======================================================================
__device__ __forceinline__ int32_t sat_add(int32_t a, int32_t b) {  // a + b for b <= 0, -inf absorbing
    return a == NEG ? NEG : max(a + b, NEG);
}
__device__ __forceinline__ int32_t add_s(int32_t a, int32_t s) { return a == NEG ? NEG : a + s; }

// 16-bit lanes of the two-stripe fill (fill_rect_stripe16): a finite value v
// is held as v + kBias16 (> 0) and -inf as 0, two per 32-bit register. Then
// max(x + g, 0) keeps -inf exact for a gap term (g < 0), and
// min(x + x, max(x + s, 0)) for M's score s: x = 0 stays 0, while a finite
// x (> |s|) gives x + s, as 2x >= x + s. Exact when every finite value of the
// chain lies within (-kBias16 + W, kBias16), W the largest one-step change of
// a score: any finite value is a path's score of at most L + T steps, so
// (L + T + 1) * W < kBias16 suffices (fits16).
constexpr int32_t kBias16 = 8192;
__device__ __forceinline__ uint32_t to16(int32_t v) { return v == NEG ? 0u : (uint32_t)(v + kBias16); }
__device__ __forceinline__ int32_t from16(uint32_t u) { return u == 0u ? NEG : (int32_t)u - kBias16; }
__device__ __forceinline__ uint32_t pack16(int32_t x) { return ((uint32_t)x & 0xFFFFu) * 0x10001u; }
__device__ __forceinline__ uint32_t pk16(uint32_t lo, uint32_t hi) { return __byte_perm(lo, hi, 0x5410); }
// 0xFFFF in each 16-bit half of x whose top bit (bit 15, bit 31) is set, else
// 0: prmt's sign-replicating byte selects (nibble 8 + byte index).
__device__ __forceinline__ uint32_t halfmask16(uint32_t x) {
    uint32_t r;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(x), "r"(0u), "r"(0xBB99u));
    return r;
}

struct DpParams {
    int32_t match, mismatch, gap_o, gap_e;
    int32_t mode;  // 0 NW, 1 SW
};

constexpr int kDpWarps = 4;       // warps per block in k_dp
constexpr int kDpClassWarp = 3;   // DP class of the unbanded warp launch (DpClass::kDpWarp)
constexpr int kStripeThreads = 128;  // threads per block in k_dp_stripe (the stride of its score tables)
constexpr int kSmemSeeds = 64;    // chain seeds cached in shared memory per warp (else global)

__device__ __forceinline__ int match_max(int32_t m, int32_t i, int32_t d) {  // Alignment.h:577-589
    int32_t mx = m;
    int s = OP_M;
    if (i > mx) { mx = d; s = OP_I; }
    if (d > mx) s = OP_D;
    return s;
}

// Storage of one rectangle (16-byte aligned, a multiple of 16 bytes):
// traceback codes, then a row buffer of C + 1 entries of 16 bytes (the
// bottom row of the previous stripe: M, I, D; the warp and row fills use
// the first 12 bytes per column of it as 3 int32 per column), then M, I, D
// of the last row and of the last column. Code layouts: the warp and row
// fills keep stripes of 32 rows skewed along anti-diagonals (code of row rr,
// column cc at ((rr / 32) * (C + 31) + cc + rr % 32) * 32 + rr % 32); the
// register-stripe fill keeps stripes of K rows column by column (code at
// ((rr / K) * C + cc) * K + rr % K), which fits in the same space for K <= 32.
struct RectGeo {
    int64_t r0, c0, R, C;
    uint8_t* code;
    int32_t* rowbuf;  // (C + 1) x 4
    int32_t* lastrow; // C x 3
    int32_t* lastcol; // R x 3
};

__device__ __forceinline__ int64_t rect_bytes(int64_t R, int64_t C) {
    if (R <= 0 || C <= 0) return 0;
    const int64_t stripes = (R + 31) / 32;
    const int64_t code = ((stripes * (C + 31) * 32) + 15) / 16 * 16;
    return (code + ((C + 1) * 4 + C * 3 + R * 3) * 4 + 16 + 15) / 16 * 16;
}

// Boundary cells of one rectangle, with the closed forms' constants taken
// once (ChainCtx::bnd_info) and held in registers: the per-cell queries then
// read nothing from the chain context.
struct RectBnd {
    int kind;            // 0: the 5' rectangle, 1: the rectangle after seed p (closed form), 2: region rule
    int m;
    int nw;
    int32_t go, ge;      // gap open and extension
    int32_t E, Eo;       // kind 1: the seed's final diagonal value, and E + o
    int64_t q1, t1;      // kind 1: the seed's last row and column
};

struct ChainCtx {
    const int4* sd;             // per seed: qf, qt, ts, te (window-relative)
    const int32_t* rbnd;        // row boundaries b[0..2n+1]: 0, qf_0, qt_0, ..., qf_n-1, qt_n-1, L
    const int32_t* cbnd;        // column boundaries: 0, ts_0, te_0, ..., T
    int32_t n;                  // seeds in the chain
    int64_t L, T;               // query length, window length
    const uint8_t* rd;          // the read
    int rev;                    // the query is the read's reverse complement (PrimarySeq::revcom)
    const uint8_t* target;      // chromosome + t_start
    int64_t target_avail;       // chromosome bases available from t_start (beyond: terminator 0)
    uint8_t* scratch;           // rectangle storage of this chain
    int32_t* diag;              // per seed: first diagonal value
    int32_t* roff;              // per rectangle index (0..n): byte offset in scratch
    DpParams pp;
    uint32_t* status;
    int kst = 0;                // rows per stripe of the code layout (0: the 32-row skewed layout)
    int sep = 0;                // seeds in order without overlap, each of 2 or more bases (see boundary)
    uint32_t* stab = nullptr;   // register-stripe fill: this thread's score table, 16 words at stride kStripeThreads

    __device__ int64_t qf(int k) const { return sd[k].x; }
    __device__ int64_t qt(int k) const { return sd[k].y; }
    __device__ int64_t ts(int k) const { return sd[k].z; }
    __device__ int64_t te(int k) const { return sd[k].w; }
    __device__ int tb(int64_t t) const { return t < target_avail ? (int)__ldg(target + t) : 0; }
    // query base i (0-based): the read, or its reverse complement read backwards
    __device__ __forceinline__ int qbase(int64_t i) const { return rev ? comp16(rd[L - 1 - i]) : (int)rd[i]; }
    // ScoreScheme::getScore (ScoreScheme.cpp:20-24)
    __device__ int32_t score(int qb, int tbb) const {
        return ((qb & tbb) && qb != 15 && tbb != 15) ? pp.match : -pp.mismatch;
    }
    // row/column boundaries: b[0]=0, b[2k+1]=qf_k, b[2k+2]=qt_k, b[2n+1]=L
    __device__ int64_t rb(int m) const { return rbnd[m]; }
    __device__ int64_t cb(int m) const { return cbnd[m]; }
    // segment of matrix row i >= 1: smallest m with i <= b[m+1]
    __device__ int row_seg(int64_t i) const {
        int lo = 0, hi = 2 * n;
        while (lo < hi) { const int mid = (lo + hi) >> 1; if (i <= rbnd[mid + 1]) hi = mid; else lo = mid + 1; }
        return lo;
    }
    __device__ int col_seg(int64_t j) const {
        int lo = 0, hi = 2 * n;
        while (lo < hi) { const int mid = (lo + hi) >> 1; if (j <= cbnd[mid + 1]) hi = mid; else lo = mid + 1; }
        return lo;
    }
    __device__ RectGeo rect(int m) const {
        RectGeo g;
        g.r0 = rb(m); g.c0 = cb(m);
        g.R = rb(m + 1) - g.r0; g.C = cb(m + 1) - g.c0;
        uint8_t* base = scratch + roff[m >> 1];
        const int64_t stripes = (g.R + 31) / 32;
        g.code = base;
        int32_t* ints = reinterpret_cast<int32_t*>(base + ((stripes * (g.C + 31) * 32) + 15) / 16 * 16);
        g.rowbuf = ints;
        g.lastrow = ints + (g.C + 1) * 4;
        g.lastcol = g.lastrow + g.C * 3;
        return g;
    }
    __device__ uint8_t code_at(const RectGeo& g, int64_t i, int64_t j) const {
        const int64_t rr = i - g.r0 - 1, cc = j - g.c0 - 1;
        if (kst) return g.code[((rr / kst) * g.C + cc) * kst + rr % kst];
        const int64_t stripe = rr >> 5, lane = rr & 31;
        return g.code[(stripe * (g.C + 31) + cc + lane) * 32 + lane];
    }
    // stored value of a rectangle cell (its last row or column)
    __device__ int32_t rect_val(int m, int which, int64_t i, int64_t j) const {
        const RectGeo g = rect(m);
        if (i == g.r0 + g.R) return g.lastrow[(j - g.c0 - 1) * 3 + which];
        if (j == g.c0 + g.C) return g.lastcol[(i - g.r0 - 1) * 3 + which];
        atomicOr(status, kErrInternal);
        return NEG;
    }
    __device__ int seed_by_qt(int64_t v) const {
        int lo = 0, hi = n - 1;
        while (lo <= hi) { const int mid = (lo + hi) >> 1; const int64_t x = qt(mid); if (x == v) return mid; if (x < v) lo = mid + 1; else hi = mid - 1; }
        return -1;
    }
    __device__ int seed_by_te(int64_t v) const {
        int lo = 0, hi = n - 1;
        while (lo <= hi) { const int mid = (lo + hi) >> 1; const int64_t x = te(mid); if (x == v) return mid; if (x < v) lo = mid + 1; else hi = mid - 1; }
        return -1;
    }
    // Final value of M(i,j) as seen by region `stage` (regions < stage written).
    __device__ int32_t M(int64_t i, int64_t j, int stage) const {
        if (i >= 1 && j >= 1) {
            const int mr = row_seg(i);
            if (mr == col_seg(j) && mr < stage) {
                if (!(mr & 1)) return rect_val(mr, 0, i, j);
                const int k = (mr - 1) >> 1;
                if (i - qf(k) == j - ts(k)) return diag[k] + (int32_t)(i - qf(k) - 1) * pp.match;
                return NEG;
            }
            const int k = seed_by_qt(i - 1);  // the cell past seed k (Alignment.cpp:157-160)
            if (k >= 0 && 2 * k + 1 < stage && te(k) + 1 == j) return diag[k] + (int32_t)(qt(k) - qf(k)) * pp.match;
        }
        if (pp.mode == 0) return i == 0 ? 0 : NEG;
        return (i == 0 || j == 0) ? 0 : NEG;
    }
    __device__ int32_t I(int64_t i, int64_t j, int stage) const {
        if (i >= 1 && j >= 1) {
            const int mr = row_seg(i);
            if (mr == col_seg(j) && mr < stage && !(mr & 1)) return rect_val(mr, 1, i, j);
        }
        if (i >= 1) {
            const int k = seed_by_qt(i - 1);  // I.row(to+1) = M.row(to) + o (Alignment.cpp:161-163)
            if (k >= 0 && 2 * k + 1 < stage) return sat_add(M(i - 1, j, 2 * k + 2), -(pp.gap_o + pp.gap_e));
        }
        if (pp.mode == 0 && j == 0) return i == 0 ? 0 : -(pp.gap_o + pp.gap_e * (int32_t)i);  // initNW
        return NEG;
    }
    __device__ int32_t D(int64_t i, int64_t j, int stage) const {
        if (i >= 1 && j >= 1) {
            const int mr = row_seg(i);
            if (mr == col_seg(j) && mr < stage && !(mr & 1)) return rect_val(mr, 2, i, j);
        }
        if (j >= 1) {
            const int k = seed_by_te(j - 1);  // D.col(end+1) = M.col(end) + o (Alignment.cpp:165-169)
            if (k >= 0 && 2 * k + 1 < stage) return sat_add(M(i, j - 1, 2 * k + 2), -(pp.gap_o + pp.gap_e));
        }
        return NEG;
    }

    // M, I, D (or M, D) of a boundary cell, out of line: the band fill reads
    // boundaries at a handful of cells, and inlining each query at each of
    // its sites would bloat the banded kernel's code.
    __device__ __noinline__ int3 MID(int64_t i, int64_t j, int stage) const {
        return make_int3(M(i, j, stage), I(i, j, stage), D(i, j, stage));
    }
    __device__ __noinline__ int2 MD(int64_t i, int64_t j, int stage) const {
        return make_int2(M(i, j, stage), D(i, j, stage));
    }

    // M, I, D of a boundary cell (top row or left column) of rectangle m,
    // with closed forms for the two common cases and the region rule for the
    // rest:
    //  * the 5' rectangle (m == 0): no region is written before it, so its
    //    boundary holds the initialised matrices (initNW/initSW,
    //    Alignment.h:599-613): row 0 M = 0 (I(0,0) = 0 in NW); column 0
    //    I = -gapPenalty(i) in NW, M = 0 in SW; the rest -inf;
    //  * the rectangle after seed p (m == 2p + 2: a gap or the 3'
    //    rectangle) of a one-seed chain, or of a chain whose seeds are in
    //    order without overlap (qf_k >= qt_k-1, ts_k >= te_k-1) and at least
    //    2 bases long (sep): its top row is the seed's last row qt and its
    //    left column the seed's last column te; every cell there is -inf but
    //    the seed's last diagonal cell (qt, te) with M = E (the seed's final
    //    diagonal value), D(qt, te + 1) = E + o from the whole-column
    //    overwrite and I(qt + 1, te) = E + o from the whole-row overwrite
    //    (Alignment.cpp:161-169). No other region reaches those cells: the
    //    earlier seeds' blocks, cells past them, row and column overwrites
    //    and rectangles all lie in rows before qt and columns before te, as
    //    the region rule confirms cell by cell.
    // OUTLINE: the region rule through the out-of-line MID (else inlined).
    // (bnd_info takes the constants of a rectangle once, bnd_at answers a
    // cell from them)
    template <bool OUTLINE = true>
    __device__ __forceinline__ int3 boundary(int m, int64_t i, int64_t j) const {
        return bnd_at<OUTLINE>(bnd_info(m), i, j);
    }

    __device__ __forceinline__ RectBnd bnd_info(int m) const {
        RectBnd b;
        b.m = m;
        b.nw = pp.mode == 0;
        b.go = pp.gap_o; b.ge = pp.gap_e;
        b.E = 0; b.Eo = 0; b.q1 = 0; b.t1 = 0;
        if (m == 0) {
            b.kind = 0;
        } else if (!(m & 1) && (n == 1 || sep)) {
            const int p = (m >> 1) - 1;
            b.kind = 1;
            b.q1 = qt(p); b.t1 = te(p);
            b.E = diag[p] + (int32_t)(b.q1 - qf(p) - 1) * pp.match;
            b.Eo = sat_add(b.E, -(pp.gap_o + pp.gap_e));
        } else {
            b.kind = 2;
        }
        return b;
    }
    // boundary(m, i, j) from the constants of bnd_info(m)
    template <bool OUTLINE = true>
    __device__ __forceinline__ int3 bnd_at(const RectBnd& b, int64_t i, int64_t j) const {
        if (b.kind == 0) {
            if (i == 0) return make_int3(0, (b.nw && j == 0) ? 0 : NEG, NEG);
            return make_int3(b.nw ? NEG : 0, b.nw ? -(b.go + b.ge * (int32_t)i) : NEG, NEG);  // j == 0
        }
        if (b.kind == 1) {
            if (i == b.q1 && j == b.t1) return make_int3(b.E, NEG, NEG);
            if (i == b.q1 && j == b.t1 + 1) return make_int3(NEG, NEG, b.Eo);
            if (j == b.t1 && i == b.q1 + 1) return make_int3(NEG, b.Eo, NEG);
            return make_int3(NEG, NEG, NEG);
        }
        if constexpr (OUTLINE) return MID(i, j, b.m);
        else return make_int3(M(i, j, b.m), I(i, j, b.m), D(i, j, b.m));
    }

    // Single-thread fill of rectangle m, row by row, into the same code layout
    // (rowbuf holds the row above). With w >= 0 only the cells within w
    // diagonals of the adjacent seed's diagonal are computed (the 5' rectangle
    // ends on it, the 3' rectangle starts on it); the other cells count as
    // -inf and their stored last-row/last-column values are -inf. Returns the
    // number of cells computed.
    __device__ __forceinline__ int64_t fill_rect_thread(int m, int w, int32_t& best, int64_t& bkey) {
        const RectGeo g = rect(m);
        const RectBnd bi = bnd_info(m);
        if (g.R <= 0 || g.C <= 0) return 0;
        const int32_t o = -(pp.gap_o + pp.gap_e), e = -pp.gap_e;
        const bool banded = w >= 0;
        const int64_t dg = m == 0 ? g.C - g.R : 0;  // diagonal offset (column - row) of the seed's diagonal
        if (banded) {
            for (int64_t c = 0; c < 3 * g.C; ++c) g.lastrow[c] = NEG;
            for (int64_t c = 0; c < 3 * g.R; ++c) g.lastcol[c] = NEG;
        }
        int64_t plo = 0, phi = g.C - 1;  // columns of the row above held in rowbuf
        if (banded) { plo = max((int64_t)0, dg - w - 1); phi = min(g.C - 1, dg + w); }
        for (int64_t c = plo; c <= phi; ++c) {  // the top boundary row
            const int3 v = bnd_at<false>(bi, g.r0, g.c0 + 1 + c);
            g.rowbuf[c * 3] = v.x;
            g.rowbuf[c * 3 + 1] = v.y;
            g.rowbuf[c * 3 + 2] = v.z;
        }
        int64_t cells = 0;
        int64_t lrow = -1;         // matrix row whose left boundary cell (lrow, c0) is cached
        int32_t lm = NEG, li = NEG, ld = NEG;
        for (int64_t rr = 0; rr < g.R; ++rr) {
            const int64_t lo = banded ? max((int64_t)0, rr + dg - w) : 0;
            const int64_t hi = banded ? min(g.C - 1, rr + dg + w) : g.C - 1;
            if (lo > hi) { plo = 1; phi = 0; continue; }
            const int64_t i = g.r0 + 1 + rr;
            int32_t ml = NEG, dl = NEG, dm = NEG, di = NEG, dd = NEG;
            if (lo == 0) {
                if (lrow == i - 1) { dm = lm; di = li; dd = ld; }
                else { const int3 v = bnd_at<false>(bi, i - 1, g.c0); dm = v.x; di = v.y; dd = v.z; }
                const int3 v = bnd_at<false>(bi, i, g.c0);
                lm = v.x; li = v.y; ld = v.z;
                lrow = i;
                ml = lm; dl = ld;
            } else if (lo - 1 >= plo && lo - 1 <= phi) {
                dm = g.rowbuf[(lo - 1) * 3]; di = g.rowbuf[(lo - 1) * 3 + 1]; dd = g.rowbuf[(lo - 1) * 3 + 2];
            }
            const int qb = qbase(i - 1);
            const int64_t lane = rr & 31;
            uint8_t* code_base = g.code + (rr >> 5) * (g.C + 31) * 32;
            for (int64_t c = lo; c <= hi; ++c) {
                int32_t um = NEG, ui = NEG, ud = NEG;
                if (c >= plo && c <= phi) { um = g.rowbuf[c * 3]; ui = g.rowbuf[c * 3 + 1]; ud = g.rowbuf[c * 3 + 2]; }
                const int64_t j = g.c0 + 1 + c;
                const int s = score(qb, tb(j - 1));
                const int32_t mx = max(max(dm, dd), di);
                int32_t mv = add_s(mx, s);
                if (pp.mode == 1) mv = max(mv, 0);
                const int32_t a1 = sat_add(um, o), a2 = sat_add(ui, e);
                const int32_t iv = max(a1, a2);
                const int32_t b1 = sat_add(ml, o), b2 = sat_add(dl, e);
                const int32_t dv = max(b1, b2);
                code_base[(c + lane) * 32 + lane] = (uint8_t)(match_max(dm, di, dd) | ((a1 > a2) ? 4 : 0) |
                                                            ((b1 > b2) ? 8 : 0) | (mv > 0 ? 16 : 0));
                if (rr == g.R - 1) { g.lastrow[c * 3] = mv; g.lastrow[c * 3 + 1] = iv; g.lastrow[c * 3 + 2] = dv; }
                if (c == g.C - 1) { g.lastcol[rr * 3] = mv; g.lastcol[rr * 3 + 1] = iv; g.lastcol[rr * 3 + 2] = dv; }
                if (pp.mode == 1) {
                    const int64_t key = j * (L + 1) + i;
                    if (mv > best || (mv == best && key < bkey)) { best = mv; bkey = key; }
                }
                dm = um; di = ui; dd = ud;
                g.rowbuf[c * 3] = mv; g.rowbuf[c * 3 + 1] = iv; g.rowbuf[c * 3 + 2] = dv;
                ml = mv; dl = dv;
            }
            cells += hi - lo + 1;
            plo = lo; phi = hi;
        }
        return cells;
    }

    // Register-stripe fill of rectangle m by one thread (Alignment::
    // calculateScoresNW/SW, Alignment.cpp:72-133, cell for cell as
    // fill_rect_thread): stripes of K rows, column by column. The previous
    // column's M, I, D of the stripe's rows stay in registers; the row above
    // the stripe comes from the row buffer (one 16-byte load per column) and
    // the stripe's bottom row goes back to it; a column's K traceback codes
    // leave in one store. Cell updates use Blackwell's integer DP
    // instructions: __vimax3_s32 for M's three-way maximum and
    // __viaddmax_s32 for the saturating gap terms max(x + g, -inf), which
    // keep -inf absorbing. The score of a cell is one bit of a per-stripe
    // table (bit k of stab[t * kStripeThreads]: row k's query base matches
    // target code t). BANDED: only the cells within w diagonals of the
    // adjacent seed's diagonal are computed, the others count as -inf
    // (boundary cells next to band cells are read exactly), as
    // fill_rect_thread does with w >= 0.
    // Returns the number of cells evaluated (for a band: its stripes' columns
    // times their rows).
    template <int K, bool LOCAL, bool BANDED>
    __device__ __noinline__ int64_t fill_rect_stripe(int m, int w, int32_t& best, int64_t& bkey) {
        static_assert(K == 8 || K == 16 || K == 32, "stripe height");
        const RectGeo g = rect(m);
        if (g.R <= 0 || g.C <= 0) return 0;
        const int R = (int)g.R, C = (int)g.C;
        const int32_t o = -(pp.gap_o + pp.gap_e), e = -pp.gap_e;
        const int32_t smt = pp.match, smm = -pp.mismatch;
        int4* rb4 = reinterpret_cast<int4*>(g.rowbuf);
        const int dg = m == 0 ? C - R : 0;  // column - row of the seed's diagonal in this rectangle
        if (BANDED) {
            for (int c = 0; c < 3 * C; ++c) g.lastrow[c] = NEG;
            for (int c = 0; c < 3 * R; ++c) g.lastcol[c] = NEG;
        }
        const RectBnd bi = bnd_info(m);
        auto bnd = [&](int64_t i, int64_t j) -> int3 { return bnd_at(bi, i, j); };
        // the context's fields the column loop reads, in registers (the
        // context itself lives in local memory)
        const uint8_t* const tgt = target + g.c0;
        const int64_t tgt_n = target_avail - g.c0;
        uint32_t* const tab = stab;
        const int64_t Lq = L;
        int plo = 0, phi = C - 1;  // columns of the row buffer that hold the row above
        if (BANDED) { plo = max(0, dg - w - 1); phi = min(C - 1, dg + w); }
        for (int c = plo; c <= phi; ++c) {  // the top boundary row
            const int3 v = bnd(g.r0, g.c0 + 1 + c);
            rb4[c] = make_int4(v.x, v.y, v.z, 0);
        }
        int64_t cells = 0;
        const int nsp = (R + K - 1) / K;
        for (int sp = 0; sp < nsp; ++sp) {
            const int rr0 = sp * K;
            const int nrow = min(K, R - rr0);
            int clo = 0, chi = C - 1;
            if (BANDED) { clo = max(0, rr0 + dg - w); chi = min(C - 1, rr0 + nrow - 1 + dg + w); }
            if (clo > chi) { plo = 1; phi = 0; continue; }
            const int64_t i0 = g.r0 + 1 + rr0;  // matrix row of the stripe's first row
            {
                uint32_t tbits[16];
#pragma unroll
                for (int t = 0; t < 16; ++t) tbits[t] = 0;
                for (int k = 0; k < nrow; ++k) {
                    const int q = qbase(i0 - 1 + k);
                    if (q == 15) continue;  // N scores a mismatch against everything
#pragma unroll
                    for (int t = 1; t < 15; ++t) tbits[t] |= (q & t) ? (1u << k) : 0u;
                }
#pragma unroll
                for (int t = 0; t < 16; ++t) tab[t * kStripeThreads] = tbits[t];
            }
            // the previous column's values of the stripe's rows: the left
            // boundary (column c0) when the stripe starts at column 0
            int32_t Mp[K], Ip[K], Dp[K];
#pragma unroll
            for (int k = 0; k < K; ++k) {
                Mp[k] = NEG; Ip[k] = NEG; Dp[k] = NEG;
                if (clo == 0 && k < nrow) {
                    const int3 v = bnd(i0 + k, g.c0);
                    Mp[k] = v.x; Ip[k] = v.y; Dp[k] = v.z;
                }
            }
            // diagonal neighbour of the stripe's first row at column clo
            int32_t dM = NEG, dI = NEG, dD = NEG;
            if (clo == 0) {
                const int3 v = bnd(i0 - 1, g.c0);
                dM = v.x; dI = v.y; dD = v.z;
            } else if (clo - 1 >= plo && clo - 1 <= phi) {
                const int4 v = rb4[clo - 1];
                dM = v.x; dI = v.y; dD = v.z;
            }
            uint8_t* code = g.code + (int64_t)sp * C * K;
            const bool last = sp == nsp - 1;
            // the row above and the target base of a column are loaded one
            // column ahead, so that their latency overlaps a column's cells
            auto up_of = [&](int c) -> int4 {
                return (!BANDED || (c >= plo && c <= phi)) ? rb4[c] : make_int4(NEG, NEG, NEG, 0);
            };
            auto tbase = [&](int c) -> int { return c < tgt_n ? (int)__ldg(tgt + c) : 0; };
            int4 up_next = up_of(clo);
            int tb_next = tbase(clo);
            for (int cc = clo; cc <= chi; ++cc) {
                const int4 up = up_next;
                const uint32_t tm = tab[(tb_next & 15) * kStripeThreads];
                if (cc < chi) {
                    up_next = up_of(cc + 1);
                    tb_next = tbase(cc + 1);
                }
                const int64_t j = g.c0 + 1 + cc;
                int32_t uM = up.x, uI = up.y;
                uint32_t wd[K / 4];
#pragma unroll
                for (int q = 0; q < K / 4; ++q) wd[q] = 0;
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    const int32_t s = ((tm >> k) & 1u) ? smt : smm;
                    const int32_t mx = __vimax3_s32(dM, dD, dI);
                    int32_t mv = mx == NEG ? NEG : mx + s;
                    if (LOCAL) mv = max(mv, 0);
                    const int32_t a1 = __viaddmax_s32(uM, o, NEG), a2 = __viaddmax_s32(uI, e, NEG);
                    int32_t iv = max(a1, a2);
                    const int32_t b1 = __viaddmax_s32(Mp[k], o, NEG), b2 = __viaddmax_s32(Dp[k], e, NEG);
                    int32_t dv = max(b1, b2);
                    // matchMax with its quirk (I wins over M, then D only
                    // when I does not), insMax, delMax, M > 0
                    uint32_t cd = dI > dM ? (uint32_t)OP_I : (dD > dM ? (uint32_t)OP_D : (uint32_t)OP_M);
                    cd |= (a1 > a2 ? 4u : 0u) | (b1 > b2 ? 8u : 0u);
                    if (LOCAL) cd |= mv > 0 ? 16u : 0u;
                    if (BANDED) {
                        if ((unsigned)(cc - (rr0 + k) - dg + w) > (unsigned)(2 * w)) { mv = NEG; iv = NEG; dv = NEG; }
                    }
                    if (LOCAL && k < nrow) {
                        const int64_t key = j * (Lq + 1) + (i0 + k);
                        if (mv > best || (mv == best && key < bkey)) { best = mv; bkey = key; }
                    }
                    wd[k >> 2] |= cd << (8 * (k & 3));
                    dM = Mp[k]; dI = Ip[k]; dD = Dp[k];
                    Mp[k] = mv; Ip[k] = iv; Dp[k] = dv;
                    uM = mv; uI = iv;
                }
                if constexpr (K == 8) {
                    *reinterpret_cast<uint2*>(code + (int64_t)cc * K) = make_uint2(wd[0], wd[1]);
                } else {
#pragma unroll
                    for (int q = 0; q < K / 16; ++q)
                        reinterpret_cast<uint4*>(code + (int64_t)cc * K)[q] =
                            make_uint4(wd[4 * q], wd[4 * q + 1], wd[4 * q + 2], wd[4 * q + 3]);
                }
                dM = up.x; dI = up.y; dD = up.z;  // (stripe row - 1, cc): the next column's diagonal
                if (nrow == K) rb4[cc] = make_int4(Mp[K - 1], Ip[K - 1], Dp[K - 1], 0);
                if (last) {
                    int32_t lm = Mp[0], li = Ip[0], ld = Dp[0];
#pragma unroll
                    for (int k = 1; k < K; ++k)
                        if (k < nrow) { lm = Mp[k]; li = Ip[k]; ld = Dp[k]; }
                    g.lastrow[cc * 3] = lm; g.lastrow[cc * 3 + 1] = li; g.lastrow[cc * 3 + 2] = ld;
                }
            }
            if (chi == C - 1) {
#pragma unroll
                for (int k = 0; k < K; ++k)
                    if (k < nrow) {
                        int32_t* lc = g.lastcol + (int64_t)(rr0 + k) * 3;
                        lc[0] = Mp[k]; lc[1] = Ip[k]; lc[2] = Dp[k];
                    }
            }
            cells += (int64_t)nrow * (chi - clo + 1);  // cells evaluated (a band's stripe is a parallelogram)
            if (BANDED) { plo = clo; phi = chi; }
        }
        return cells;
    }

    // Two-stripe fill in 16-bit lanes (GLOBAL mode; the chain fits16): one
    // thread fills 32 rows at a time as two 16-row stripes held in the two
    // halves of 16 registers per matrix, the lower stripe one column behind
    // the upper, so that within an iteration the halves are independent (the
    // lower stripe's row above is the upper stripe's last row, finished one
    // iteration earlier; an extra iteration ends the lower stripe, the first
    // one starts it from the left boundary). Each instruction updates two
    // cells: __vibmax_s16x2 gives a maximum with its comparison outcomes (the
    // traceback code bits), __viaddmax_s16x2 / __viaddmin_s16x2 the gap and
    // score terms. A cell's score comes from its row's bit in the stripe
    // table word of its column's target code (bits 0-15 upper rows, 16-31
    // lower rows), moved to a byte's top bit and widened to a 16-bit mask by
    // a byte permute. BANDED (w >= 0): only the cells within w diagonals of
    // the adjacent seed's diagonal count, the others are -inf (masked to 0
    // through a per-column bitmap of the rows in band), as fill_rect_stripe
    // does; each half runs over its own band's columns. (The dispatcher
    // keeps banded flanks on the 32-bit fill: a band of 2w+1 diagonals
    // leaves each lagged half idle for 17 of the pair's 2w+33 columns, and
    // measured on the 1 M-read workload the 16-bit banded form made the DP
    // stage slower, 19.5 against 18.3 ms.) Codes and last
    // row/column go where fill_rect_stripe<16> puts them (the last row and
    // column in 32-bit values), so the traceback reads both alike. The row
    // buffer holds 16-bit values here. Returns the cells evaluated.
    template <bool BANDED, int KH>
    __device__ __noinline__ int64_t fill_rect_stripe16(int m, int w) {
        static_assert(KH == 4 || KH == 8 || KH == 16, "rows per half");
        constexpr int K = KH;
        const RectGeo g = rect(m);
        const RectBnd bi = bnd_info(m);
        if (g.R <= 0 || g.C <= 0) return 0;
        const int R = (int)g.R, C = (int)g.C;
        const uint32_t O2 = pack16(-(pp.gap_o + pp.gap_e)), E2 = pack16(-pp.gap_e);
        const uint32_t SMM2 = pack16(-pp.mismatch), SX2 = SMM2 ^ pack16(pp.match);
        int4* rb4 = reinterpret_cast<int4*>(g.rowbuf);
        const uint8_t* const tgt = target + g.c0;
        const int64_t tgt_n = target_avail - g.c0;
        uint32_t* const tab = stab;
        auto tbase = [&](int c) -> int { return c < tgt_n ? (int)__ldg(tgt + c) : 0; };
        const int dg = m == 0 ? C - R : 0;  // column - row of the seed's diagonal in this rectangle
        if (BANDED) {
            for (int c = 0; c < 3 * C; ++c) g.lastrow[c] = NEG;
            for (int c = 0; c < 3 * R; ++c) g.lastcol[c] = NEG;
        }
        int plo = 0, phi = C - 1;  // columns of the row buffer that hold the row above
        if (BANDED) { plo = max(0, dg - w - 1); phi = min(C - 1, dg + w); }
        for (int c = plo; c <= phi; ++c) {  // the top boundary row
            const int3 v = bnd_at(bi, g.r0, g.c0 + 1 + c);
            rb4[c] = make_int4((int)to16(v.x), (int)to16(v.y), (int)to16(v.z), 0);
        }
        int64_t cells = 0;
        const int nds = (R + 2 * K - 1) / (2 * K);
        for (int ds = 0; ds < nds; ++ds) {
            const int rr0 = ds * 2 * K;
            const int nlo = min(K, R - rr0), nhi = max(0, min(K, R - rr0 - K));
            const int64_t i0 = g.r0 + 1 + rr0;  // matrix row of the upper stripe's first row
            // columns of each half: all, or its rows' band
            int clo = 0, chi = C - 1, hlo = 0, hhi = nhi > 0 ? C - 1 : -1;
            if (BANDED) {
                clo = max(0, rr0 + dg - w); chi = min(C - 1, rr0 + nlo - 1 + dg + w);
                if (nhi > 0) { hlo = max(0, rr0 + K + dg - w); hhi = min(C - 1, rr0 + K + nhi - 1 + dg + w); }
                if (clo > chi) { plo = 1; phi = 0; continue; }  // no band cell left in this rectangle
            }
            {
                uint32_t tbits[16];
#pragma unroll
                for (int t = 0; t < 16; ++t) tbits[t] = 0;
                for (int k = 0; k < nlo + nhi; ++k) {
                    const int q = qbase(i0 - 1 + k);
                    if (q == 15) continue;  // N scores a mismatch against everything
                    const uint32_t bit = 1u << (k < K ? k : 16 + k - K);  // upper rows from bit 0, lower from bit 16
#pragma unroll
                    for (int t = 1; t < 15; ++t) tbits[t] |= (q & t) ? bit : 0u;
                }
#pragma unroll
                for (int t = 0; t < 16; ++t) tab[t * kStripeThreads] = tbits[t];
            }
            // the left boundary (column c0) of the pair's rows when the band
            // reaches it, parked in the rectangle's last-column slots until
            // the loop reads it (those slots get their final values at the
            // last column); -inf (0) left of a band
            const bool left = clo == 0;
            if (left) {
                for (int k = 0; k < nlo + nhi; ++k) {
                    const int3 v = bnd_at(bi, i0 + k, g.c0);
                    int32_t* lc = g.lastcol + (int64_t)(rr0 + k) * 3;
                    lc[0] = v.x; lc[1] = v.y; lc[2] = v.z;
                }
            }
            uint32_t Mp[K], Ip[K], Dp[K];
#pragma unroll
            for (int k = 0; k < K; ++k) {
                Mp[k] = 0u; Ip[k] = 0u; Dp[k] = 0u;
                if (left && k < nlo) {
                    int32_t* lc = g.lastcol + (int64_t)(rr0 + k) * 3;
                    Mp[k] = to16(lc[0]); Ip[k] = to16(lc[1]); Dp[k] = to16(lc[2]);
                    if (BANDED) { lc[0] = NEG; lc[1] = NEG; lc[2] = NEG; }  // a band may not reach the last column
                }
            }
            // diagonal inputs of row 0 of each half at the next iteration:
            // upper (row above the pair, previous column), lower (upper
            // stripe's last row two columns back)
            uint32_t dlM = 0u, dlI = 0u, dlD = 0u;
            if (left) {
                const int3 cv = bnd_at(bi, i0 - 1, g.c0);
                dlM = to16(cv.x); dlI = to16(cv.y); dlD = to16(cv.z);
            } else if (clo - 1 >= plo && clo - 1 <= phi) {
                const int4 v = rb4[clo - 1];
                dlM = (uint32_t)v.x; dlI = (uint32_t)v.y; dlD = (uint32_t)v.z;
            }
            uint32_t dhM = 0u, dhI = 0u, dhD = 0u;
            // codes in 16-row stripes: a pair of 16-row halves fills stripes
            // 2ds and 2ds+1; smaller halves share one stripe, the upper at
            // byte b0 of each column, the lower right after it
            uint8_t* const code_lo = K == 16 ? g.code + (int64_t)(2 * ds) * C * 16
                                             : g.code + (int64_t)(rr0 / 16) * C * 16 + (rr0 % 16);
            uint8_t* const code_hi = K == 16 ? code_lo + (int64_t)C * 16 : code_lo + K;
            auto store_codes = [&](uint8_t* p, const uint32_t* wv) {
                if constexpr (K == 16) *reinterpret_cast<uint4*>(p) = make_uint4(wv[0], wv[1], wv[2], wv[3]);
                else if constexpr (K == 8) *reinterpret_cast<uint2*>(p) = make_uint2(wv[0], wv[1]);
                else *reinterpret_cast<uint32_t*>(p) = wv[0];
            };
            const bool last = ds == nds - 1;
            const int lr = R - 1 - rr0;  // the rectangle's last row within this pair (last pair)
            const int cend = nhi > 0 ? max(chi, hhi + 1) : chi;  // last iteration
            auto up_of = [&](int c) -> int4 {
                return (!BANDED || (c >= plo && c <= phi)) ? rb4[c] : make_int4(0, 0, 0, 0);
            };
            int4 up_next = up_of(clo);
            int tb_next = tbase(clo);
            uint32_t tprev = clo > 0 ? tab[(tbase(clo - 1) & 15) * kStripeThreads] : 0u;
            for (int cc = clo; cc <= cend; ++cc) {
                const int4 up = up_next;  // upper stripe: the row above at column cc (cc <= chi)
                const uint32_t tw = tab[(tb_next & 15) * kStripeThreads];
                if (cc + 1 <= min(chi, C - 1)) {
                    up_next = up_of(cc + 1);
                    tb_next = tbase(cc + 1);
                } else {
                    up_next = make_int4(0, 0, 0, 0);
                    tb_next = cc + 1 < C ? tbase(cc + 1) : 0;
                }
                const uint32_t cw = (tw & 0xFFFFu) | (tprev & 0xFFFF0000u);
                tprev = tw;
                // rows in band at this iteration: upper rows at column cc,
                // lower rows at column cc - 1 (bits 0-15, 16-31)
                uint32_t band = 0xFFFFFFFFu;
                if (BANDED) {
                    // row k of a half is in band when its column minus its row
                    // minus dg lies in [-w, w]
                    const int bl = cc - rr0 - dg + w, bh = cc - 1 - rr0 - K - dg + w;
                    const int l0 = max(0, bl - 2 * w), l1 = min(K - 1, bl);
                    const int h0 = max(0, bh - 2 * w), h1 = min(K - 1, bh);
                    const uint32_t ml = (l0 <= l1 && cc <= chi) ? ((0xFFFFu >> (15 - l1 + l0)) << l0) : 0u;
                    const uint32_t mh = (h0 <= h1 && cc - 1 >= hlo && cc - 1 <= hhi) ? ((0xFFFFu >> (15 - h1 + h0)) << h0) : 0u;
                    band = ml | (mh << 16);
                }
                uint32_t uM = pk16((uint32_t)up.x, Mp[K - 1]), uI = pk16((uint32_t)up.y, Ip[K - 1]);
                uint32_t dM = pk16(dlM, dhM), dI = pk16(dlI, dhI), dD = pk16(dlD, dhD);
                dlM = (uint32_t)up.x; dlI = (uint32_t)up.y; dlD = (uint32_t)up.z;
                dhM = Mp[K - 1]; dhI = Ip[K - 1]; dhD = Dp[K - 1];
                uint32_t wl[K / 4], wh[K / 4];
#pragma unroll
                for (int q = 0; q < K / 4; ++q) { wl[q] = 0u; wh[q] = 0u; }
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    const uint32_t msk = halfmask16(cw << (15 - k));
                    const uint32_t s2 = (msk & SX2) ^ SMM2;
                    bool aIh, aIl, aDh, aDl, bIh, bIl, bDh, bDl;
                    const uint32_t t1 = __vibmax_s16x2(dM, dI, &aIh, &aIl);
                    const uint32_t mx = __vibmax_s16x2(t1, dD, &aDh, &aDl);
                    uint32_t mv = __viaddmin_s16x2(mx, mx, __viaddmax_s16x2(mx, s2, 0u));
                    const uint32_t a1 = __viaddmax_s16x2(uM, O2, 0u);
                    uint32_t iv = __vibmax_s16x2(__viaddmax_s16x2(uI, E2, 0u), a1, &bIh, &bIl);
                    const uint32_t b1 = __viaddmax_s16x2(Mp[k], O2, 0u);
                    uint32_t dv = __vibmax_s16x2(__viaddmax_s16x2(Dp[k], E2, 0u), b1, &bDh, &bDl);
                    if (BANDED) {  // cells outside the band are -inf
                        const uint32_t in = halfmask16(band << (15 - k));
                        mv &= in; iv &= in; dv &= in;
                    }
                    // matchMax (I over M, then D only when I does not win), insMax, delMax
                    const uint32_t cl = (aIl ? (aDl ? 0u : 2u) : 1u) | (bIl ? 0u : 4u) | (bDl ? 0u : 8u);
                    const uint32_t ch = (aIh ? (aDh ? 0u : 2u) : 1u) | (bIh ? 0u : 4u) | (bDh ? 0u : 8u);
                    wl[k >> 2] |= cl << (8 * (k & 3));
                    wh[k >> 2] |= ch << (8 * (k & 3));
                    dM = Mp[k]; dI = Ip[k]; dD = Dp[k];
                    Mp[k] = mv; Ip[k] = iv; Dp[k] = dv;
                    uM = mv; uI = iv;
                }
                if (cc <= chi) {  // upper stripe: column cc
                    store_codes(code_lo + (int64_t)cc * 16, wl);
                    if (last && lr < K) {
                        uint32_t lm = Mp[0], li = Ip[0], ld = Dp[0];
#pragma unroll
                        for (int k = 1; k < K; ++k)
                            if (k == lr) { lm = Mp[k]; li = Ip[k]; ld = Dp[k]; }
                        g.lastrow[cc * 3] = from16(lm & 0xFFFFu);
                        g.lastrow[cc * 3 + 1] = from16(li & 0xFFFFu);
                        g.lastrow[cc * 3 + 2] = from16(ld & 0xFFFFu);
                    }
                    if (cc == C - 1) {
#pragma unroll
                        for (int k = 0; k < K; ++k)
                            if (k < nlo) {
                                int32_t* lc = g.lastcol + (int64_t)(rr0 + k) * 3;
                                lc[0] = from16(Mp[k] & 0xFFFFu); lc[1] = from16(Ip[k] & 0xFFFFu); lc[2] = from16(Dp[k] & 0xFFFFu);
                            }
                    }
                }
                if (nhi > 0) {
                    if (cc == clo) {  // the lower stripe starts from its left boundary (-inf left of a band)
#pragma unroll
                        for (int k = 0; k < K; ++k) {
                            uint32_t hm = 0u, hi = 0u, hd = 0u;
                            if (left && k < nhi) {
                                int32_t* lc = g.lastcol + (int64_t)(rr0 + K + k) * 3;
                                hm = to16(lc[0]); hi = to16(lc[1]); hd = to16(lc[2]);
                                if (BANDED) { lc[0] = NEG; lc[1] = NEG; lc[2] = NEG; }
                            }
                            Mp[k] = pk16(Mp[k], hm); Ip[k] = pk16(Ip[k], hi); Dp[k] = pk16(Dp[k], hd);
                        }
                    } else if (cc - 1 >= hlo && cc - 1 <= hhi) {  // lower stripe: column cc - 1
                        const int c1 = cc - 1;
                        store_codes(code_hi + (int64_t)c1 * 16, wh);
                        if (nhi == K)
                            rb4[c1] = make_int4((int)(Mp[K - 1] >> 16), (int)(Ip[K - 1] >> 16), (int)(Dp[K - 1] >> 16), 0);
                        if (last && lr >= K) {
                            uint32_t lm = Mp[0], li = Ip[0], ld = Dp[0];
#pragma unroll
                            for (int k = 1; k < K; ++k)
                                if (k == lr - K) { lm = Mp[k]; li = Ip[k]; ld = Dp[k]; }
                            g.lastrow[c1 * 3] = from16(lm >> 16);
                            g.lastrow[c1 * 3 + 1] = from16(li >> 16);
                            g.lastrow[c1 * 3 + 2] = from16(ld >> 16);
                        }
                        if (c1 == C - 1) {
#pragma unroll
                            for (int k = 0; k < K; ++k)
                                if (k < nhi) {
                                    int32_t* lc = g.lastcol + (int64_t)(rr0 + K + k) * 3;
                                    lc[0] = from16(Mp[k] >> 16); lc[1] = from16(Ip[k] >> 16); lc[2] = from16(Dp[k] >> 16);
                                }
                        }
                    }
                }
            }
            cells += (int64_t)nlo * (chi - clo + 1) + (nhi > 0 ? (int64_t)nhi * (hhi - hlo + 1) : 0);
            if (BANDED) { plo = hhi >= 0 && nhi > 0 ? hlo : clo; phi = nhi > 0 ? hhi : chi; }
        }
        return cells;
    }

    // Warp fill of the band of rectangle m (m = 0 or 2n; GLOBAL mode): the
    // 2w+1 diagonals within w of the adjacent seed's diagonal. Position
    // p = lane + 32 h (h < NP) of row rr is column rr + dg - w + p; one row is
    // one step. M and I read the previous row at p and p + 1 (registers and a
    // shuffle); D runs along the row, D(p) = max(M(p-1) + o, D(p-1) + e), which
    // unrolls to a prefix maximum over the row of M(k) + o - e k (plus the left
    // boundary's contribution at column 0). Boundary cells next to band cells
    // are read exactly; cells outside the band count as -inf. Codes and the
    // last row/column go to the same places as the whole-rectangle fills.
    // Returns the number of cells computed.
    template <int NP>
    __device__ int64_t fill_rect_band(int m, int w) {
        const RectGeo g = rect(m);
        if (g.R <= 0 || g.C <= 0) return 0;
        const int lane = lane_id();
        const unsigned FULL = 0xffffffffu;
        const int32_t o = -(pp.gap_o + pp.gap_e), e = -pp.gap_e;
        const int64_t dg = m == 0 ? g.C - g.R : 0;
        const int NB = 2 * w + 1;
        constexpr int32_t VNEG = INT32_MIN + (1 << 26);  // "no path" in the prefix maximum, far below NEG
        for (int64_t c = lane; c < 3 * g.C; c += 32) g.lastrow[c] = NEG;
        for (int64_t c = lane; c < 3 * g.R; c += 32) g.lastcol[c] = NEG;
        // row -1 is the top boundary row: position p there is column dg - w + p - 1
        int32_t pm[NP], pi[NP], pd[NP];
#pragma unroll
        for (int h = 0; h < NP; ++h) {
            const int p = lane + 32 * h;
            const int64_t c = dg - w + p - 1;
            pm[h] = pi[h] = pd[h] = NEG;
            if (p <= NB && c >= -1 && c <= g.C - 1) {
                const int3 v = MID(g.r0, g.c0 + 1 + c, m);
                pm[h] = v.x; pi[h] = v.y; pd[h] = v.z;
            }
        }
        __syncwarp();
        int64_t cells = 0;
        for (int64_t rr = 0; rr < g.R; ++rr) {
            const int64_t i = g.r0 + 1 + rr;
            const int qb = qbase(i - 1);
            const int64_t lr = rr & 31;
            uint8_t* code_base = g.code + (rr >> 5) * (g.C + 31) * 32;
            int32_t um[NP], ui[NP], mv[NP], iv[NP], U[NP], b1s[NP], b2s[NP];
            uint8_t code[NP];
            bool valid[NP], at0[NP];
            int64_t col[NP];
#pragma unroll
            for (int h = 0; h < NP; ++h) {  // up neighbours: previous row at p + 1
                const int32_t a_m = __shfl_down_sync(FULL, pm[h], 1);
                const int32_t a_i = __shfl_down_sync(FULL, pi[h], 1);
                int32_t n_m = NEG, n_i = NEG;
                if (h + 1 < NP) {
                    n_m = __shfl_sync(FULL, pm[h + 1 < NP ? h + 1 : h], 0);
                    n_i = __shfl_sync(FULL, pi[h + 1 < NP ? h + 1 : h], 0);
                }
                um[h] = lane < 31 ? a_m : n_m;
                ui[h] = lane < 31 ? a_i : n_i;
            }
#pragma unroll
            for (int h = 0; h < NP; ++h) {
                const int p = lane + 32 * h;
                const int64_t c = rr + dg - w + p;
                col[h] = c;
                valid[h] = p < NB && c >= 0 && c < g.C;
                at0[h] = valid[h] && c == 0;
                int32_t dm = pm[h], di = pi[h], dd = pd[h];
                if (at0[h]) { const int3 v = MID(i - 1, g.c0, m); dm = v.x; di = v.y; dd = v.z; }
                int32_t mvv = NEG, ivv = NEG;
                uint8_t cd = 0;
                U[h] = VNEG;
                b1s[h] = b2s[h] = NEG;
                if (valid[h]) {
                    const int64_t j = g.c0 + 1 + c;
                    const int sc = score(qb, tb(j - 1));
                    mvv = add_s(max(max(dm, dd), di), sc);
                    const int32_t a1 = sat_add(um[h], o), a2 = sat_add(ui[h], e);
                    ivv = max(a1, a2);
                    cd = (uint8_t)(match_max(dm, di, dd) | ((a1 > a2) ? 4 : 0) | (mvv > 0 ? 16 : 0));
                    U[h] = mvv + o - e * p;
                    if (at0[h]) {  // left boundary column
                        const int2 l = MD(i, g.c0, m);
                        const int32_t b1 = sat_add(l.x, o), b2 = sat_add(l.y, e);
                        b1s[h] = b1; b2s[h] = b2;
                        U[h] = max(U[h], max(b1, b2) + e - e * p);
                    }
                }
                mv[h] = mvv; iv[h] = ivv; code[h] = cd;
            }
            // inclusive prefix maximum of U over positions
            int32_t P[NP];
#pragma unroll
            for (int h = 0; h < NP; ++h) {
                int32_t x = U[h];
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const int32_t y = __shfl_up_sync(FULL, x, d);
                    if (lane >= d) x = max(x, y);
                }
                if (h > 0) x = max(x, __shfl_sync(FULL, P[h > 0 ? h - 1 : 0], 31));
                P[h] = x;
            }
            int32_t dv[NP];
#pragma unroll
            for (int h = 0; h < NP; ++h) {
                const int p = lane + 32 * h;
                const int32_t t1 = __shfl_up_sync(FULL, P[h], 1);
                const int32_t t2 = h > 0 ? __shfl_sync(FULL, P[h > 0 ? h - 1 : 0], 31) : VNEG;
                const int32_t ex = lane > 0 ? t1 : t2;  // max over positions < p
                int32_t dvv = NEG;
                if (valid[h]) {
                    if (at0[h]) dvv = max(b1s[h], b2s[h]);
                    else dvv = (int32_t)max((int64_t)NEG, (int64_t)e * (p - 1) + (int64_t)ex);
                }
                dv[h] = dvv;
            }
#pragma unroll
            for (int h = 0; h < NP; ++h) {  // delMax bit from the left neighbour
                const int32_t lmA = __shfl_up_sync(FULL, mv[h], 1), ldA = __shfl_up_sync(FULL, dv[h], 1);
                int32_t lmB = NEG, ldB = NEG;
                if (h > 0) {
                    lmB = __shfl_sync(FULL, mv[h > 0 ? h - 1 : 0], 31);
                    ldB = __shfl_sync(FULL, dv[h > 0 ? h - 1 : 0], 31);
                }
                const int32_t lm = lane > 0 ? lmA : lmB, ld = lane > 0 ? ldA : ldB;
                if (valid[h]) {
                    const int p = lane + 32 * h;
                    int32_t b1 = b1s[h], b2 = b2s[h];
                    if (!at0[h]) {
                        if (p >= 1 && col[h] >= 1) { b1 = sat_add(lm, o); b2 = sat_add(ld, e); }
                        else { b1 = NEG; b2 = NEG; }
                    }
                    const uint8_t cd = (uint8_t)(code[h] | ((b1 > b2) ? 8 : 0));
                    const int64_t c = col[h];
                    code_base[(c + lr) * 32 + lr] = cd;
                    if (rr == g.R - 1) { g.lastrow[c * 3] = mv[h]; g.lastrow[c * 3 + 1] = iv[h]; g.lastrow[c * 3 + 2] = dv[h]; }
                    if (c == g.C - 1) { g.lastcol[rr * 3] = mv[h]; g.lastcol[rr * 3 + 1] = iv[h]; g.lastcol[rr * 3 + 2] = dv[h]; }
                }
                cells += __popc(__ballot_sync(FULL, valid[h]));
                pm[h] = valid[h] ? mv[h] : NEG;
                pi[h] = valid[h] ? iv[h] : NEG;
                pd[h] = valid[h] ? dv[h] : NEG;
            }
        }
        __syncwarp();
        return cells;
    }

    // Warp fill of rectangle m (Alignment::calculateScoresNW/SW,
    // Alignment.cpp:72-133): stripes of 32 rows, lane = row, one column per
    // step along the anti-diagonal wavefront; values travel by shuffles.
    // Returns this lane's best (M, column-major key) for local mode.
    __device__ __forceinline__ void fill_rect(int m, int32_t& best, int64_t& bkey) {
        const RectGeo g = rect(m);
        if (g.R <= 0 || g.C <= 0) return;
        const int lane = lane_id();
        const int32_t o = -(pp.gap_o + pp.gap_e), e = -pp.gap_e;
        const int64_t stripes = (g.R + 31) / 32;
        // top boundary row (r0, c0+1 .. c0+C) into the stripe hand-off buffer
        for (int64_t c = lane; c < g.C; c += 32) {
            const int64_t j = g.c0 + 1 + c;
            g.rowbuf[c * 3] = M(g.r0, j, m);
            g.rowbuf[c * 3 + 1] = I(g.r0, j, m);
            g.rowbuf[c * 3 + 2] = D(g.r0, j, m);
        }
        __syncwarp();
        for (int64_t sp = 0; sp < stripes; ++sp) {
            const int64_t rr = sp * 32 + lane;
            const bool row_ok = rr < g.R;
            const int64_t i = g.r0 + 1 + rr;
            // left boundary (column c0) of this row and of the row above
            int32_t ml = NEG, dl = NEG, md0 = NEG, id0 = NEG, dd0 = NEG;
            if (row_ok) {
                ml = M(i, g.c0, m); dl = D(i, g.c0, m);
                md0 = M(i - 1, g.c0, m); id0 = I(i - 1, g.c0, m); dd0 = D(i - 1, g.c0, m);
            }
            const int qb = row_ok ? qbase(i - 1) : 0;
            int32_t pm = NEG, pi = NEG, pd = NEG;       // this lane's output of the previous step
            int32_t um = NEG, ui = NEG, ud = NEG;       // up neighbour (i-1, j) of the current step
            int32_t dm = md0, di = id0, dd = dd0;       // diagonal neighbour (i-1, j-1)
            int tcur = 0;                               // target base of this lane's column
            uint8_t* code_base = g.code + sp * (g.C + 31) * 32;
            const int rows_here = (int)min((int64_t)32, g.R - sp * 32);  // the last lane with a row
            const int C = (int)g.C;
            // Lane 0's inputs for the next 32 steps (the row above from rowbuf,
            // the target bases of columns t .. t+31) are loaded together, one
            // column per lane, and handed to lane 0 by shuffles; the other lanes
            // take theirs from the lane before.
            int32_t pre_m = NEG, pre_i = NEG, pre_d = NEG;
            int pre_t = 0;
            for (int t = 0; t < C + rows_here - 1; ++t) {
                if ((t & 31) == 0) {
                    const int cc = t + lane;
                    pre_m = pre_i = pre_d = NEG;
                    pre_t = 0;
                    if (cc < C) {
                        pre_m = g.rowbuf[cc * 3]; pre_i = g.rowbuf[cc * 3 + 1]; pre_d = g.rowbuf[cc * 3 + 2];
                        pre_t = tb(g.c0 + cc);
                    }
                }
                const int c = t - lane;
                const int32_t sm_ = __shfl_up_sync(0xffffffffu, pm, 1);
                const int32_t si_ = __shfl_up_sync(0xffffffffu, pi, 1);
                const int32_t sd_ = __shfl_up_sync(0xffffffffu, pd, 1);
                const int st_ = __shfl_up_sync(0xffffffffu, tcur, 1);
                const int32_t r_m = __shfl_sync(0xffffffffu, pre_m, t & 31);
                const int32_t r_i = __shfl_sync(0xffffffffu, pre_i, t & 31);
                const int32_t r_d = __shfl_sync(0xffffffffu, pre_d, t & 31);
                const int r_t = __shfl_sync(0xffffffffu, pre_t, t & 31);
                const bool act = row_ok && c >= 0 && c < C;
                if (lane == 0) {
                    if (act) { um = r_m; ui = r_i; ud = r_d; }
                    tcur = r_t;
                } else {
                    um = sm_; ui = si_; ud = sd_;
                    tcur = st_;
                }
                if (act) {
                    const int64_t j = g.c0 + 1 + c;
                    const int32_t lm = c == 0 ? ml : pm;
                    const int32_t ld = c == 0 ? dl : pd;
                    const int s = score(qb, tcur);
                    const int32_t mx = max(max(dm, dd), di);
                    int32_t mv = add_s(mx, s);
                    if (pp.mode == 1) mv = max(mv, 0);
                    const int32_t a1 = sat_add(um, o), a2 = sat_add(ui, e);
                    const int32_t iv = max(a1, a2);
                    const int32_t b1 = sat_add(lm, o), b2 = sat_add(ld, e);
                    const int32_t dv = max(b1, b2);
                    const uint8_t code = (uint8_t)(match_max(dm, di, dd) | ((a1 > a2) ? 4 : 0) |
                                                   ((b1 > b2) ? 8 : 0) | (mv > 0 ? 16 : 0));
                    code_base[(c + lane) * 32 + lane] = code;
                    if (rr == g.R - 1) { g.lastrow[c * 3] = mv; g.lastrow[c * 3 + 1] = iv; g.lastrow[c * 3 + 2] = dv; }
                    if (c == C - 1) { g.lastcol[rr * 3] = mv; g.lastcol[rr * 3 + 1] = iv; g.lastcol[rr * 3 + 2] = dv; }
                    if (lane == 31) { g.rowbuf[c * 3] = mv; g.rowbuf[c * 3 + 1] = iv; g.rowbuf[c * 3 + 2] = dv; }
                    if (pp.mode == 1) {
                        const int64_t key = j * (L + 1) + i;
                        if (mv > best || (mv == best && key < bkey)) { best = mv; bkey = key; }
                    }
                    pm = mv; pi = iv; pd = dv;
                }
                // the up neighbour of this step is the diagonal of the next
                if (act) { dm = um; di = ui; dd = ud; }
            }
            __syncwarp();
        }
    }
};

struct DpArgs {
    IndexDev ix;
    const Seed* seeds;
    const int64_t* chain_idx_off;
    const int32_t* chain_len;
    const int32_t* chain_read;
    const int64_t* chain_idx;
    int64_t n_chain;
    const uint8_t* rseq;
    const int64_t* roff;
    const int64_t* t_start;
    const int64_t* t_end;
    const int64_t* scr_off;     // per chain, byte offset of its rectangle storage
    uint8_t* scr;               // rectangle storage of the chains of this launch
    int64_t scr_base;           // scr_off of the first chain of this launch
    int32_t* aux;               // per chain at 2 * chain_idx_off + chain index: diag (n) and rect offsets (n + 1)
    int4* sdbuf;                // per chain seed geometry when n > kSmemSeeds (at chain_idx_off)
    const int64_t* path_off;    // per chain, capacity L + tLen + 1
    uint8_t* path;
    int32_t* path_len;
    msg_aln* aln;
    DpParams pp;
    uint32_t* status;
    // Chains handled by this launch: with cls >= 0, the cls-th range of the
    // class-sorted list `list` (range lengths cls_n[0..], on the device);
    // otherwise list[0 .. *n_list).
    const int64_t* list;
    const unsigned long long* n_list;
    const unsigned long long* cls_n;
    int cls;
    unsigned long long* queue;            // thread kernels: chains of the launch handed out so far
    int lanes16;                          // stripe chains may use the 16-bit two-stripe fill
    int64_t* tb_list;                     // chains whose traceback k_traceback runs
    unsigned long long* tb_n;
    // Banded flanks (GLOBAL mode). band[2c], band[2c+1]: half-width of the 5'
    // and 3' rectangle's band, -1 for the whole rectangle.
    const int8_t* band;
    double min_rate;                      // Alignment::filter rate; < 0: keep every record
    uint8_t* keep;                        // per chain: the record survives the filter
    int64_t* fb_list;                     // chains whose banded result was not certified
    unsigned long long* fb_n;
    unsigned long long* bstat;            // banded, exact, dropped, fallback, cells computed
    uint8_t* probe;                       // non-null: certificate only (0 none, 1 exact, 2 below the filter)
    int64_t* probe_cells;
};

// Alignment::filter (Alignment.cpp:548-555): alnScore < readLen * minScoreRate.
__device__ __forceinline__ bool below_filter(int64_t score, int64_t L, double rate) {
    return rate >= 0 && (double)score < __dmul_rn((double)L, rate);
}

// Alignment ctor window (Alignment.cpp:46-52): tStart = max(0, (int64)(start - 1.1*from)),
// tEnd = min(chrLen, (int64)(end + 1.1*(qTo - to))) with chrLen counting the
// chromosome's terminator (MetaGenome.h:237 over MetaGenome.cpp:208).
__global__ void k_dp_prep(IndexDev ix, const Seed* __restrict__ seeds, const int64_t* __restrict__ chain_idx_off,
                          const int32_t* __restrict__ chain_len, const int32_t* __restrict__ chain_read,
                          const int64_t* __restrict__ chain_idx, const int64_t* __restrict__ roff, int64_t n_chain,
                          int64_t* __restrict__ t_start, int64_t* __restrict__ t_end, int64_t* __restrict__ bytes,
                          int64_t* __restrict__ pathcap, int64_t* __restrict__ dpcells, int64_t* __restrict__ area_out,
                          int4* __restrict__ geo) {
    const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= n_chain) return;
    const int64_t* idx = chain_idx + chain_idx_off[c];
    const int n = chain_len[c];
    const Seed f = seeds[idx[0]], l = seeds[idx[n - 1]];
    const int64_t r = chain_read[c];
    const int64_t L = roff[r + 1] - roff[r];
    const int64_t chr_len = ix.chr_len[f.tid] + 1;
    const double k11 = 1.0 + 0.1;
    const double ts = __dsub_rn((double)f.start, __dmul_rn(k11, (double)f.from));
    const double te = __dadd_rn((double)l.end, __dmul_rn(k11, (double)(L - l.to)));
    const int64_t tS = max((int64_t)0, (int64_t)ts);
    const int64_t tE = min(chr_len, (int64_t)te);
    t_start[c] = tS;
    t_end[c] = tE;
    const int64_t T = tE - tS;
    int64_t area = 0, diag = 0, by = 0;
    {   // 5' rectangle, gaps, 3' rectangle (Alignment.cpp:54-70)
        const int64_t a0 = f.from, b0 = f.start - tS;
        if (a0 > 0 && b0 > 0) area += a0 * b0;
        by += rect_bytes(a0, b0);
        for (int k = 0; k < n; ++k) {
            const Seed s = seeds[idx[k]];
            diag += s.to - s.from;
            if (k + 1 < n) {
                const Seed t = seeds[idx[k + 1]];
                const int64_t R = t.from - s.to, C = t.start - s.end;
                if (R > 0 && C > 0) area += R * C;
                by += rect_bytes(R, C);
            }
        }
        const int64_t R = L - l.to, C = tE - l.end;
        if (R > 0 && C > 0) area += R * C;
        by += rect_bytes(R, C);
    }
    bytes[c] = by;
    pathcap[c] = L + T + 1;
    dpcells[c] = area + diag;
    if (area_out) area_out[c] = area;
    if (geo) geo[c] = make_int4((int)f.from, (int)(f.start - tS), (int)(L - l.to), (int)(tE - l.end));
}

// One chain: a warp (WARP = true; lanes share the rectangle wavefront and the
// last-row scan) or a single thread (chains whose rectangles are all small).
// Traceback of one chain (Alignment::backTraceNW/SW, Alignment.cpp:173-276)
// from the end cell (aln_to, aln_end) in state s0, writing the reversed path
// and the alignment record.
__device__ __forceinline__ void dp_traceback(const DpArgs& a, int64_t c, const ChainCtx& xc, int64_t r, const Seed& f,
                                             int64_t t_start, int64_t aln_to, int64_t aln_end, int s0, int32_t best,
                                             int32_t flags) {
    const ChainCtx x = xc;  // a copy of its own, which registers can hold (the caller's lives in memory)
    const int stage = 2 * x.n + 2;
    uint8_t* path = a.path + a.path_off[c];
    const int32_t go = a.pp.gap_o, ge = a.pp.gap_e;
    int64_t i = aln_to, j = aln_end;
    int s = s0;
    int64_t np = 0;
    const int64_t cap = x.L + x.T + 1;
    int cur_m = -1;  // rectangle holding (i, j), if any
    RectGeo g{};
    for (;;) {
        // locate (i, j): inside a rectangle -> traceback codes
        bool in_rect = false;
        if (i >= 1 && j >= 1) {
            if (cur_m >= 0 && i > g.r0 && i <= g.r0 + g.R && j > g.c0 && j <= g.c0 + g.C) in_rect = true;
            else {
                const int mr = x.row_seg(i);
                if (mr == x.col_seg(j) && !(mr & 1)) { cur_m = mr; g = x.rect(mr); in_rect = true; }
            }
        }
        const uint8_t code = in_rect ? x.code_at(g, i, j) : 0;
        if (a.pp.mode == 0) { if (!(i > 0)) break; }
        else {
            const bool mpos = in_rect ? ((code >> 4) & 1) : (x.M(i, j, stage) > 0);
            if (!(s != OP_M || mpos)) break;
        }
        const bool ok = (s == OP_M) ? (i >= 1 && j >= 1) : (s == OP_I) ? (i >= 1) : (j >= 1);
        if (!ok || np >= cap) { flags |= 2; break; }
        if (s == OP_M && !in_rect && (a.pp.mode == 0 || a.pp.match >= 1)) {
            // Inside a seed block, diagonal cells d >= 1 have I = D = -inf
            // (no I-row or D-column overwrite reaches past the block's first
            // row/column), so matchMax keeps M: walk straight to d = 1.
            const int mr = x.row_seg(i);
            if ((mr & 1) && mr == x.col_seg(j)) {
                const int k = (mr - 1) >> 1;
                const int64_t d = i - x.qf(k) - 1;
                if (d == j - x.ts(k) - 1 && d >= 2 && np + d - 1 <= cap) {
                    for (int64_t q = 0; q < d - 1; ++q) path[np + q] = (uint8_t)OP_M;
                    np += d - 1;
                    i -= d - 1;
                    j -= d - 1;
                    continue;
                }
            }
        }
        path[np++] = (uint8_t)s;
        if (s == OP_M) {
            s = in_rect ? (code & 3) : match_max(x.M(i - 1, j - 1, stage), x.I(i - 1, j - 1, stage), x.D(i - 1, j - 1, stage));
            i--; j--;
        } else if (s == OP_I) {
            const bool mm = in_rect ? ((code >> 2) & 1)
                                    : sat_add(x.M(i - 1, j, stage), -(go + ge)) > sat_add(x.I(i - 1, j, stage), -ge);
            s = mm ? OP_M : OP_I;
            i--;
        } else {
            const bool mm = in_rect ? ((code >> 3) & 1)
                                    : sat_add(x.M(i, j - 1, stage), -(go + ge)) > sat_add(x.D(i, j - 1, stage), -ge);
            s = mm ? OP_M : OP_D;
            j--;
        }
    }
    a.path_len[c] = (int32_t)np;
    msg_aln& o = a.aln[c];
    o.read = r;
    o.tid = f.tid;
    o.strand = f.strand;
    o.t_start = t_start;
    o.t_end = a.t_end[c];
    o.aln_from = i;
    o.aln_to = aln_to;
    o.aln_start = t_start + j;
    o.aln_end = t_start + aln_end;
    o.aln_score = best == NEG ? INT32_MIN : best;
    o.flags = flags;
    if (flags & 2) atomicOr(a.status, kErrTrace);
    if (a.keep) a.keep[c] = (best == NEG || below_filter(best, x.L, a.min_rate)) && a.min_rate >= 0 ? 0 : 1;
}

// KST > 0 (thread path): rectangles filled by fill_rect_stripe<KST>, codes
// in its stripe layout; KST == 0: fill_rect_thread (thread) or the warp fills.
template <bool WARP, bool BAND, int KST = 0>
__device__ __forceinline__ void dp_chain(const DpArgs& a, int64_t c, int4* sd, int32_t* rbnd, int32_t* cbnd,
                                         int4* gsd, uint32_t* stab = nullptr) {
    const int lane = WARP ? lane_id() : 0;
    const int stride = WARP ? 32 : 1;
    ChainCtx x;
    const int64_t* idx = a.chain_idx + a.chain_idx_off[c];
    x.n = a.chain_len[c];
    const int64_t r = a.chain_read[c];
    x.L = a.roff[r + 1] - a.roff[r];
    const int64_t t_start = a.t_start[c];
    x.T = a.t_end[c] - t_start;
    const Seed f = a.seeds[idx[0]];
    const int64_t chr_len = a.ix.chr_len[f.tid];
    x.target = a.ix.chr_seq + a.ix.chr_off[f.tid] + t_start;
    x.target_avail = chr_len - t_start;
    x.scratch = a.scr + (a.scr_off[c] - a.scr_base);
    int32_t* aux = a.aux + 2 * a.chain_idx_off[c] + c;
    x.diag = aux;
    x.roff = aux + x.n;
    x.pp = a.pp;
    x.status = a.status;
    // unbanded stripe chains in GLOBAL mode whose values fit 16-bit lanes
    // run the two-stripe 16-bit fill (codes in 16-row stripes)
    const int64_t w1 = max(max(a.pp.match, a.pp.mismatch), a.pp.gap_o + a.pp.gap_e);
    // (a banded chain keeps its banded flank in 32-bit stripes of KST rows,
    // so its other rectangles share the 16-row code layout only when KST is 16)
    const bool use16 = !WARP && KST > 0 && a.lanes16 && a.pp.mode == 0 && (x.L + x.T + 1) * w1 < kBias16 &&
                       (!BAND || KST == 16);
    x.kst = use16 ? 16 : KST;
    x.stab = stab;
    // geometry in sd/rbnd/cbnd; a warp working in shared memory also leaves a
    // copy in the chain's global slot (gsd) for k_traceback
    int32_t* grb = reinterpret_cast<int32_t*>(gsd + x.n);
    int32_t* gcb = grb + 2 * x.n + 2;
    const bool copy = WARP && gsd != sd;
    for (int k = lane; k < x.n; k += stride) {
        const Seed s = a.seeds[idx[k]];
        const int4 g = make_int4(s.from, s.to, (int)(s.start - t_start), (int)(s.end - t_start));
        sd[k] = g;
        rbnd[2 * k + 1] = g.x; rbnd[2 * k + 2] = g.y;
        cbnd[2 * k + 1] = g.z; cbnd[2 * k + 2] = g.w;
        if (copy) {
            gsd[k] = g;
            grb[2 * k + 1] = g.x; grb[2 * k + 2] = g.y;
            gcb[2 * k + 1] = g.z; gcb[2 * k + 2] = g.w;
        }
    }
    if (lane == 0) {
        rbnd[0] = 0; cbnd[0] = 0;
        rbnd[2 * x.n + 1] = (int32_t)x.L; cbnd[2 * x.n + 1] = (int32_t)x.T;
        if (copy) {
            grb[0] = 0; gcb[0] = 0;
            grb[2 * x.n + 1] = (int32_t)x.L; gcb[2 * x.n + 1] = (int32_t)x.T;
        }
    }
    x.sd = sd;
    x.rbnd = rbnd;
    x.cbnd = cbnd;
    if (WARP) __syncwarp();
    {
        bool sep = true;
        for (int k = 0; k < x.n && sep; ++k) {
            const int4 g = sd[k];
            sep = g.y - g.x >= 2 && (k == 0 || (g.x >= sd[k - 1].y && g.z >= sd[k - 1].w));
        }
        x.sep = sep;
    }
    x.rd = a.rseq + a.roff[r];
    x.rev = f.strand != FWD;
    if (WARP) __syncwarp();
    if (lane == 0) {  // byte offsets of rectangles 0..n in this chain's storage
        int64_t off = 0;
        for (int q = 0; q <= x.n; ++q) {
            const int m = 2 * q;
            x.roff[q] = (int32_t)off;
            off += rect_bytes(x.rb(m + 1) - x.rb(m), x.cb(m + 1) - x.cb(m));
        }
    }
    if (WARP) __syncwarp();
    int32_t best = 0;       // local mode: M(0,0) = 0 is the first candidate
    int64_t bkey = 0;
    // band half-widths of the 5' and 3' rectangles (GLOBAL mode)
    const bool may_band = BAND && a.band && a.pp.mode == 0;
    const int w5 = may_band ? a.band[2 * c] : -1;
    const int w3 = may_band ? a.band[2 * c + 1] : -1;
    const bool banded = BAND && (w5 >= 0 || w3 >= 0);
    if (a.probe && !banded) return;  // certificate probe: the whole cell set needs no certificate
    int64_t cells = 0;
    int32_t x5 = NEG;       // best state value where the 5' rectangle meets the first seed
    auto fill = [&](int m, int w) {
        if constexpr (!WARP && KST > 0) {
            if constexpr (BAND) {
                if (w >= 0) {  // banded flanks in 32-bit stripes (see fill_rect_stripe16)
                    cells += x.template fill_rect_stripe<KST, false, true>(m, w, best, bkey);
                    return;
                }
            }
            // (halves of 4 or 8 rows for small rectangles lay their codes out
            // alike, but choosing them per rectangle made the lanes of a warp
            // call different fills: DP 19.2 against 17.1 ms per 1 M reads)
            if (use16) cells += x.template fill_rect_stripe16<false, 16>(m, -1);
            else if (x.pp.mode == 1) cells += x.template fill_rect_stripe<KST, true, false>(m, -1, best, bkey);
            else cells += x.template fill_rect_stripe<KST, false, false>(m, -1, best, bkey);
        } else if constexpr (!WARP) {
            cells += x.fill_rect_thread(m, w, best, bkey);
        } else {
            if constexpr (BAND) {
                if (w >= 0) {
                    cells += w <= 15 ? x.template fill_rect_band<1>(m, w) : x.template fill_rect_band<2>(m, w);
                    return;
                }
            }
            x.fill_rect(m, best, bkey);
            const int64_t R = x.rb(m + 1) - x.rb(m), C = x.cb(m + 1) - x.cb(m);
            if (R > 0 && C > 0) cells += R * C;
        }
    };
    // 5' rectangle, then per seed its first diagonal cell and the rectangle after it
    for (int q = 0; q <= x.n; ++q) {
        if (q > 0) {
            const int k = q - 1, m = 2 * k + 1;
            if (lane == 0) {  // first diagonal cell (Alignment.cpp:146-153): max(M,D,I + s, 0)
                const int64_t i = x.qf(k), j = x.ts(k);
                // (i, j) is the last cell of the rectangle before the seed when
                // it has cells: its stored last row holds the values
                const RectGeo gp = x.rect(2 * k);
                int32_t mx;
                if (gp.R > 0 && gp.C > 0) {
                    const int32_t* v = gp.lastrow + (gp.C - 1) * 3;
                    mx = max(max(v[0], v[2]), v[1]);
                } else {
                    mx = max(max(x.M(i, j, m), x.D(i, j, m)), x.I(i, j, m));
                }
                x.diag[k] = max(add_s(mx, a.pp.match), 0);
                if (k == 0) x5 = mx;
            }
            if (WARP) __syncwarp();
        }
        fill(2 * q, q == 0 ? w5 : q == x.n ? w3 : -1);
    }
    if (WARP) __syncwarp();
    // cells per DP class (the fallback recomputations count with the warp class)
    if (a.bstat && cells && lane == 0) atomicAdd(a.bstat + 3 + (a.cls >= 0 ? a.cls : kDpClassWarp), (unsigned long long)cells);
    const int stage = 2 * x.n + 2;
    auto reduce = [&]() {
        if (WARP) {
            for (int o = 16; o > 0; o >>= 1) {
                const int32_t ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int64_t ok = __shfl_xor_sync(0xffffffffu, bkey, o);
                if (ob > best || (ob == best && ok < bkey)) { best = ob; bkey = ok; }
            }
        }
    };
    // ---- traceback ----
    int64_t aln_to = 0, aln_end = 0;
    int s0 = OP_M;
    int32_t flags = 0;
    if (a.pp.mode == 0) {  // backTraceNW: scan the last row, M before I, first strict max
        // Finite cells of row L are the 3' rectangle's last row plus at most
        // these: the last seed's diagonal cell when it ends at L, the cell
        // past a seed ending at L-1, and the I-row copy of that seed's finite
        // M cells (its diagonal end and the previous seed's past cell). Every
        // other cell is -inf and cannot win a strict comparison.
        best = NEG;
        bkey = INT64_MAX;
        auto consider = [&](int64_t j) {
            const int32_t vm = x.M(x.L, j, stage), vi = x.I(x.L, j, stage);
            if (vm > best || (vm == best && vm != NEG && 2 * j < bkey)) { best = vm; bkey = 2 * j; }
            if (vi > best || (vi == best && vi != NEG && 2 * j + 1 < bkey)) { best = vi; bkey = 2 * j + 1; }
        };
        const RectGeo g3 = x.rect(2 * x.n);
        if (g3.R > 0 && g3.C > 0) {
            for (int64_t c = lane; c < g3.C; c += stride) {
                const int64_t j = g3.c0 + 1 + c;
                const int32_t vm = g3.lastrow[c * 3], vi = g3.lastrow[c * 3 + 1];
                if (vm > best || (vm == best && vm != NEG && 2 * j < bkey)) { best = vm; bkey = 2 * j; }
                if (vi > best || (vi == best && vi != NEG && 2 * j + 1 < bkey)) { best = vi; bkey = 2 * j + 1; }
            }
        }
        if (lane == 0) {
            const int kl = x.n - 1;
            if (x.qf(kl) < x.L && x.L <= x.qt(kl)) consider(x.ts(kl) + (x.L - x.qf(kl)));
            const int k = x.seed_by_qt(x.L - 1);
            if (k >= 0) {
                if (x.te(k) + 1 <= x.T) consider(x.te(k) + 1);
                if (x.te(k) >= 1) consider(x.te(k));
                if (k >= 1 && x.te(k - 1) + 1 >= 1 && x.te(k - 1) + 1 <= x.T) consider(x.te(k - 1) + 1);
            }
        }
        reduce();
        if (banded) {
            // Score-bound certificate. A path through a cell outside a band
            // shifts its diagonal by more than w before (5') or after (3') the
            // seed, so it pays at least one gap of length w+1 and gains at most
            // `match` per remaining row: in the 5' rectangle it reaches the
            // first seed with at most ub5, in the 3' rectangle it ends with at
            // most E + ub3 (E: the last seed's final diagonal value, through
            // which every complete path passes). If both bounds are strictly
            // below what the banded paths reach, every cell value the traceback
            // and the last-row scan compare is the full one (ties included),
            // so the result is the reference's. Otherwise, since the DP is
            // monotone and shifts by at most d when an input grows by d, the
            // full score is at most s_ub; a chain below the filter's threshold
            // is dropped, any other is recomputed on the whole cell set.
            const int64_t mt = a.pp.match, go = a.pp.gap_o, ge = a.pp.gap_e;
            const int kl = x.n - 1;
            const int64_t E = (int64_t)x.diag[kl] + (x.qt(kl) - x.qf(kl) - 1) * mt;
            bool ok = true;
            int64_t d5 = 0;
            if (w5 >= 0) {
                const int64_t ub5 = mt * x.qf(0) - go - ge * (w5 + 1);
                ok = ok && ub5 < (int64_t)x5;
                d5 = max((int64_t)0, ub5 - (int64_t)x5);
            }
            int64_t ub3 = INT64_MIN;
            if (w3 >= 0) {
                ub3 = E + mt * (x.L - x.qt(kl)) - go - ge * (w3 + 1);
                ok = ok && best != NEG && ub3 < (int64_t)best;
            }
            int res = 1;
            if (!ok) {
                int64_t s_ub = best == NEG ? INT64_MIN : (int64_t)best + d5;
                if (w3 >= 0) s_ub = max(s_ub, ub3 + d5);
                res = (s_ub > (int64_t)NEG && below_filter(s_ub, x.L, a.min_rate)) ? 2 : 0;
            }
            if (WARP) res = __shfl_sync(0xffffffffu, res, 0);  // x5 is lane 0's
            if (a.probe) {
                if (lane == 0) {
                    a.probe[c] = (uint8_t)res;
                    a.probe_cells[c] = cells;
                }
                return;
            }
            if (a.bstat && lane == 0) atomicAdd(a.bstat + res, 1ull);  // [0] recomputed, [1] exact, [2] dropped
            if (res == 2) { if (lane == 0) a.keep[c] = 0; return; }
            if (res == 0) {
                if (lane == 0) a.fb_list[atomicAdd(a.fb_n, 1ull)] = c;
                return;
            }
        }
        aln_to = x.L;
        if (best == NEG) { aln_end = 0; s0 = OP_M; flags |= 1; }
        else { aln_end = bkey >> 1; s0 = (bkey & 1) ? OP_I : OP_M; }
    } else {  // backTraceSW: Eigen maxCoeff, first max in column-major order
        auto consider = [&](int64_t i, int64_t j, int32_t v) {
            const int64_t key = j * (x.L + 1) + i;
            if (v > best || (v == best && key < bkey)) { best = v; bkey = key; }
        };
        for (int k = 0; k < x.n; ++k) {
            const int64_t len = x.qt(k) - x.qf(k);
            for (int64_t d = lane; d < len; d += stride) {
                const int64_t i = x.qf(k) + 1 + d, j = x.ts(k) + 1 + d;
                consider(i, j, x.M(i, j, stage));
            }
            if (lane == 0) {
                const int64_t i = x.qt(k) + 1, j = x.te(k) + 1;
                if (i <= x.L && j <= x.T) {
                    const int mr = x.row_seg(i);
                    if (!(mr == x.col_seg(j) && !(mr & 1))) consider(i, j, x.M(i, j, stage));
                }
            }
        }
        reduce();
        aln_to = bkey % (x.L + 1);
        aln_end = bkey / (x.L + 1);
        s0 = OP_M;
    }
    if constexpr (WARP || KST > 0) {
        // Hand the start of the traceback to k_traceback (one thread per
        // chain): the record carries the end cell, the score and flags, and
        // `pad` the starting state (bits 0-7) and the stripe height of the
        // code layout (bits 8-15). A stripe chain's thread leaves the serial
        // walk to that launch too: the fill kernel then holds no traceback
        // code, and its next chain starts at once.
        if (lane == 0) {
            msg_aln& o = a.aln[c];
            o.aln_to = aln_to;
            o.aln_end = aln_end;
            o.aln_score = best;
            o.flags = flags;
            o.pad = s0 | (x.kst << 8);
            a.tb_list[atomicAdd(a.tb_n, 1ull)] = c;
        }
    } else {
        dp_traceback(a, c, x, r, f, t_start, aln_to, aln_end, s0, best, flags);
    }
}


// The next 32 items of a launch's list for the calling warp, from its work
// counter (one atomic per warp); a value >= n when none is left. Every lane
// of the warp calls it.
__device__ __forceinline__ int64_t dp_take32(const DpArgs& a) {
    unsigned long long b = 0;
    if ((threadIdx.x & 31) == 0) b = atomicAdd(a.queue, 32ull);
    return (int64_t)__shfl_sync(0xffffffffu, b, 0);
}

// First entry and length of the chains of a launch (DpArgs::list).
__device__ __forceinline__ void dp_range(const DpArgs& a, int64_t& first, int64_t& n) {
    first = 0;
    if (a.cls >= 0) {
        for (int q = 0; q < a.cls; ++q) first += (int64_t)a.cls_n[q];
        n = (int64_t)a.cls_n[a.cls];
    } else {
        n = (int64_t)*a.n_list;
    }
}

// One warp per chain (grid-stride over the launch's chains). BAND: chains
// with a banded flank (GLOBAL mode); kept apart so that each kernel holds
// only the fills it runs.
template <bool BAND>
__global__ void __launch_bounds__(kDpWarps * 32, BAND ? 4 : 6) k_dp(DpArgs a) {
    __shared__ int4 s_sd[kDpWarps][kSmemSeeds];
    __shared__ int32_t s_bnd[kDpWarps][2][2 * kSmemSeeds + 2];
    const int w = threadIdx.x >> 5;
    int64_t first, n_items;
    dp_range(a, first, n_items);
    const int64_t n_warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t wi = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; wi < n_items; wi += n_warps) {
        const int64_t c = a.list[first + wi];
        const int n = a.chain_len[c];
        int4* gbase = a.sdbuf + 2 * a.chain_idx_off[c] + c;  // 2n+1 int4 per chain when not in shared memory
        const bool in_smem = n <= kSmemSeeds;
        int4* sd = in_smem ? s_sd[w] : gbase;
        int32_t* rbnd = in_smem ? s_bnd[w][0] : reinterpret_cast<int32_t*>(gbase + n);
        int32_t* cbnd = in_smem ? s_bnd[w][1] : rbnd + 2 * n + 2;
        dp_chain<true, BAND>(a, c, sd, rbnd, cbnd, gbase);
        __syncwarp();
    }
}

// Chains whose rectangles are all small: one thread each, row by row.
__global__ void __launch_bounds__(128) k_dp_small(DpArgs a) {
    int64_t first, n_items;
    dp_range(a, first, n_items);
    for (int64_t b = dp_take32(a); b < n_items; b = dp_take32(a)) {
        const int64_t t = b + (threadIdx.x & 31);
        if (t >= n_items) continue;
        const int64_t c = a.list[first + t];
        const int n = a.chain_len[c];
        int4* gbase = a.sdbuf + 2 * a.chain_idx_off[c] + c;
        int32_t* rbnd = reinterpret_cast<int32_t*>(gbase + n);
        dp_chain<false, false>(a, c, gbase, rbnd, rbnd + 2 * n + 2, gbase);
    }
}

// Mid-size chains: one thread each, rectangles in register stripes of K rows
// (fill_rect_stripe); k_traceback walks them back. BAND: chains with a
// banded flank. MINB: resident blocks per SM the registers are sized for (4:
// 128 registers, the 16-bit fill spills; 3: 168, none spills).
template <int K, bool BAND, int MINB>
__global__ void __launch_bounds__(kStripeThreads, MINB) k_dp_stripe(DpArgs a) {
    __shared__ uint32_t s_tab[16 * kStripeThreads];  // per-thread score tables, word t of thread x at t * 128 + x
    int64_t first, n_items;
    dp_range(a, first, n_items);
    for (int64_t b = dp_take32(a); b < n_items; b = dp_take32(a)) {
        const int64_t t = b + (threadIdx.x & 31);
        if (t >= n_items) continue;
        const int64_t c = a.list[first + t];
        const int n = a.chain_len[c];
        int4* gbase = a.sdbuf + 2 * a.chain_idx_off[c] + c;
        int32_t* rbnd = reinterpret_cast<int32_t*>(gbase + n);
        dp_chain<false, BAND, K>(a, c, gbase, rbnd, rbnd + 2 * n + 2, gbase, s_tab + threadIdx.x);
    }
}

// Tracebacks of the chains filled by the warp and stripe kernels, one thread
// each (a traceback is a serial walk; a warp per chain would leave 31 lanes
// idle).
__global__ void __launch_bounds__(128, 6) k_traceback(DpArgs a) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)*a.tb_n) return;
    const int64_t c = a.tb_list[t];
    ChainCtx x;
    const int64_t* idx = a.chain_idx + a.chain_idx_off[c];
    x.n = a.chain_len[c];
    const int64_t r = a.chain_read[c];
    x.L = a.roff[r + 1] - a.roff[r];
    const int64_t t_start = a.t_start[c];
    x.T = a.t_end[c] - t_start;
    const Seed f = a.seeds[idx[0]];
    x.target = a.ix.chr_seq + a.ix.chr_off[f.tid] + t_start;
    x.target_avail = a.ix.chr_len[f.tid] - t_start;
    x.scratch = a.scr + (a.scr_off[c] - a.scr_base);
    int32_t* aux = a.aux + 2 * a.chain_idx_off[c] + c;
    x.diag = aux;
    x.roff = aux + x.n;
    x.pp = a.pp;
    x.status = a.status;
    int4* gbase = a.sdbuf + 2 * a.chain_idx_off[c] + c;
    x.sd = gbase;
    x.rbnd = reinterpret_cast<int32_t*>(gbase + x.n);
    x.cbnd = x.rbnd + 2 * x.n + 2;
    x.rd = a.rseq + a.roff[r];
    x.rev = f.strand != FWD;
    const msg_aln h = a.aln[c];
    x.kst = h.pad >> 8;
    dp_traceback(a, c, x, r, f, t_start, h.aln_to, h.aln_end, h.pad & 0xff, h.aln_score, h.flags);
}

// CIGAR runs (Alignment::getAlnCigar): 5' clip, the reversed path in runs, 3' clip.
// Record k belongs to chain map[k] (k itself when map is null).
__global__ void k_cigar(int64_t n_rec, const msg_aln* __restrict__ aln, const int64_t* __restrict__ map,
                        const int64_t* __restrict__ roff, const int64_t* __restrict__ path_off,
                        const int32_t* __restrict__ path_len, const uint8_t* __restrict__ path, int pass,
                        int64_t* __restrict__ n_cig, const int64_t* __restrict__ cig_off, uint32_t* __restrict__ cig) {
    const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= n_rec) return;
    const msg_aln& a = aln[c];
    const int64_t ch = map ? map[c] : c;
    const int64_t L = roff[a.read + 1] - roff[a.read];
    const uint8_t* p = path + path_off[ch];
    const int64_t np = path_len[ch];
    int64_t k = 0;
    uint32_t* out = pass ? cig + cig_off[c] : nullptr;
    if (a.aln_from > 0) { if (pass) out[k] = (uint32_t)(a.aln_from << 4 | OP_S); ++k; }
    if (np > 0) {
        uint32_t op = p[np - 1], len = 1;
        for (int64_t t = np - 2; t >= 0; --t) {
            if (p[t] != op) { if (pass) out[k] = len << 4 | op; ++k; len = 1; }
            else len++;
            op = p[t];
        }
        if (pass) out[k] = len << 4 | op;
        ++k;
    }
    if (L - a.aln_to > 0) { if (pass) out[k] = (uint32_t)((L - a.aln_to) << 4 | OP_S); ++k; }
    if (!pass) n_cig[c] = k;
}

}  // namespace msg
