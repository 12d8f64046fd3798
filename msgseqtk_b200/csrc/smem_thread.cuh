// SMEM search with one thread per read (included by map.cu after
// map_kernels.cuh). The reference's findAllSMEMS / findFwdBackSMEMS /
// findBackFwdSMEMS control flow (SMEM.cpp:64-215) is unrolled into a state
// machine whose every step performs exactly one bi-interval extension, so the
// occurrence-bucket loads of all 32 reads of a warp issue together. Candidate
// lists (`prev`) live in per-thread global scratch; their processing follows
// the reference's sequential loop entry by entry (validity by the running
// size s0, emission while nValid == 0, in-place compaction).
#pragma once
#include <math_constants.h>

#include "map_kernels.cuh"

namespace msg {

// Interval bounds and sizes are below 2^32 (the index holds fewer than 2^32
// rows) and read positions below 2^31, so the per-thread state is 32-bit.
struct PrevEntry {
    double lp;
    uint32_t p, q, s;
    int32_t pos;  // `to` (fwd-back) or `from` (back-fwd) of the entry
};

struct SmemState32 {
    double lp;
    int32_t from, to;
    uint32_t p, q, s;
};

struct SmemThreadArgs {
    const uint8_t* seq;
    const int64_t* off;
    int64_t n_reads;
    int64_t min_len;
    double thr;
    int thr_all;
    int64_t* out;
    int64_t cap;
    int32_t* count;
    PrevEntry* prev;        // pv_cap entries per thread
    int64_t pv_cap;
    unsigned long long* work;
    unsigned long long* n_ext;
    uint32_t* status;
};

__constant__ double c_llk[16];

enum SmemPhase : int {
    PH_NEXT_READ = 0,
    PH_OUTER_LOOP,      // while (from > 0 || to < L)
    PH_OUTER_BACK,      // --from; back-fwd call
    PH_FB_WALK,         // forward walk of findFwdBackSMEMS
    PH_FB_ITER,         // start of one backward pass over prev
    PH_FB_ENTRY,        // one prev entry of that pass
    PH_BF_WALK,         // backward walk of findBackFwdSMEMS
    PH_BF_ITER,
    PH_BF_ENTRY,
    PH_DONE
};

struct ThreadSmem {
    const uint8_t* rd;
    int64_t* out;
    int32_t L;
    int32_t n_out;
    int32_t r;
    // findAllSMEMS variables and the call in progress
    int32_t from, to;
    int32_t site;           // 0: first FB(from,to)  1: FB(from0,to)  2: BF(from,to0)
    int32_t cf, ct;         // the called function's from/to
    // walk state
    SmemState32 m, m0;
    int32_t n_prev;
    int32_t pv_base;        // the list is pv[pv_base .. pv_base + n_prev), longest first
    int32_t ovf;            // a push found the list full: this read is abandoned (the batch reruns)
    // pass over prev
    int32_t k, n_keep, n_valid;
    uint32_t s0;            // running size; 0 stands for the reference's -1 (sizes compared are >= 1)
    int32_t b2;
    PrevEntry e0, e_next;   // entry being extended, and the next one (loaded early)
    int32_t phase;
    unsigned long long ext;

    __device__ int base(int32_t i) const { return (i >= 0 && i < L) ? (int)__ldg(rd + i) : 0; }
};

__device__ __forceinline__ void smem_emit(ThreadSmem& t, const SmemThreadArgs& a, int32_t from, int32_t to,
                                          const PrevEntry& e) {
    if (t.n_out < a.cap) {
        int64_t* o = t.out + 6 * (int64_t)t.n_out;
        o[0] = from; o[1] = to; o[2] = e.p; o[3] = e.q; o[4] = e.s;
        o[5] = __double_as_longlong(e.lp);
    }
    t.n_out++;
}

// Returns from the FB/BF call in progress to findAllSMEMS.
__device__ __forceinline__ void smem_return(ThreadSmem& t) {
    if (t.site == 0) { t.from = t.cf; t.to = t.ct; t.phase = PH_OUTER_LOOP; }
    else if (t.site == 1) { t.to = t.ct; t.phase = PH_OUTER_BACK; }
    else { t.from = t.cf; t.phase = PH_OUTER_LOOP; }
}

__device__ __forceinline__ SmemState32 smem_init_state(const ThreadSmem& t, const IndexDev& ix, int32_t from) {
    const int b = t.base(from);
    SmemState32 m;
    m.from = from; m.to = from + 1;
    m.p = (uint32_t)ix.C[b]; m.q = (uint32_t)ix.C[comp16(b)]; m.s = (uint32_t)(ix.C[b + 1] - ix.C[b]);
    m.lp = __dadd_rn(0.0, c_llk[b]);
    return m;
}

// Enter FB(cf, ct) (SMEM.cpp:64-77).
__device__ __forceinline__ void smem_call_fb(ThreadSmem& t, const IndexDev& ix, int site, int32_t cf) {
    t.site = site;
    t.cf = cf;
    const int b = t.base(cf);
    t.ct = cf + 1;
    if (!is_basic(b)) { smem_return(t); return; }
    t.m = smem_init_state(t, ix, cf);
    t.m0 = t.m;
    t.n_prev = 0;
    t.phase = PH_FB_WALK;
}

// Enter BF(cf, ct) (SMEM.cpp:119-132).
__device__ __forceinline__ void smem_call_bf(ThreadSmem& t, const IndexDev& ix, int32_t cf) {
    t.site = 2;
    t.cf = cf;
    const int b = t.base(cf);
    t.ct = cf + 1;
    if (!is_basic(b)) { smem_return(t); return; }
    t.m = smem_init_state(t, ix, cf);
    t.m0 = t.m;
    t.n_prev = 0;
    t.phase = PH_BF_WALK;
}

// Advance the state machine until an extension is needed. On return with
// true, (P,Q,S,B) is a backward extension to perform (forward extensions are
// expressed as backward ones on the swapped interval).
__device__ bool smem_advance(ThreadSmem& t, const SmemThreadArgs& a, const IndexDev& ix, PrevEntry* pv,
                             uint32_t& P, uint32_t& Q, uint32_t& S, int& B) {
    for (;;) {
        switch (t.phase) {
            case PH_OUTER_LOOP:
                if (!(t.from > 0 || t.to < t.L)) { t.phase = PH_DONE; return false; }
                if (t.to < t.L) { smem_call_fb(t, ix, 1, t.to); continue; }
                t.phase = PH_OUTER_BACK;
                continue;
            case PH_OUTER_BACK:
                t.from -= 1;
                if (t.from >= 0) { smem_call_bf(t, ix, t.from); continue; }
                t.phase = PH_OUTER_LOOP;
                continue;
            case PH_FB_WALK:
                if (t.m.s >= 1) {  // fwdExt with the base at `to` (0 past the read end)
                    const int nb = t.base(t.m.to);
                    P = t.m.q; Q = t.m.p; S = t.m.s; B = comp16(nb);
                    return true;
                }
                t.ct = t.m.to;
                if (t.ovf) { t.phase = PH_DONE; return false; }
                if (t.n_prev == 0) { t.cf--; smem_return(t); continue; }
                t.pv_base = (int32_t)a.pv_cap - t.n_prev;
                t.phase = PH_FB_ITER;
                continue;
            case PH_FB_ITER:
                if (!(t.cf >= 0 && t.n_prev > 0)) { smem_return(t); continue; }
                t.k = 0; t.n_keep = 0; t.s0 = 0; t.n_valid = 0;
                t.b2 = t.cf > 0 ? t.base(t.cf - 1) : 0;
                t.e_next = pv[t.pv_base];
                t.phase = PH_FB_ENTRY;
                continue;
            case PH_FB_ENTRY:
                if (t.k == t.n_prev) { t.n_prev = t.n_keep; t.cf--; t.phase = PH_FB_ITER; continue; }
                t.e0 = t.e_next;
                if (t.k + 1 < t.n_prev) t.e_next = pv[t.pv_base + t.k + 1];
                P = t.e0.p; Q = t.e0.q; S = t.e0.s; B = t.b2;
                return true;
            case PH_BF_WALK:
                if (t.m.s >= 1) {
                    const int nb = t.m.from > 0 ? t.base(t.m.from - 1) : 0;
                    P = t.m.p; Q = t.m.q; S = t.m.s; B = nb;
                    return true;
                }
                t.cf = t.m.from;
                if (t.ovf) { t.phase = PH_DONE; return false; }
                if (t.n_prev == 0) { t.ct++; smem_return(t); continue; }
                t.pv_base = (int32_t)a.pv_cap - t.n_prev;
                t.phase = PH_BF_ITER;
                continue;
            case PH_BF_ITER:
                if (!(t.ct <= t.L && t.n_prev > 0)) { smem_return(t); continue; }
                t.k = 0; t.n_keep = 0; t.s0 = 0; t.n_valid = 0;
                t.b2 = t.base(t.ct);
                t.e_next = pv[t.pv_base];
                t.phase = PH_BF_ENTRY;
                continue;
            case PH_BF_ENTRY:
                if (t.k == t.n_prev) { t.n_prev = t.n_keep; t.ct++; t.phase = PH_BF_ITER; continue; }
                t.e0 = t.e_next;
                if (t.k + 1 < t.n_prev) t.e_next = pv[t.pv_base + t.k + 1];
                P = t.e0.q; Q = t.e0.p; S = t.e0.s; B = comp16(t.b2);
                return true;
            default:
                return false;
        }
    }
}

// SMEM::loglik(from, to) <= thr for the two ranges the walks test
// (SMEM.cpp:79-81, 134-136): lp plus the bases outside [m.from, m.to) added in
// read order. Every term is <= 0 and round-to-nearest of a + b with b <= 0
// never exceeds a, so the running sum never increases: the exact sequential
// sum is <= thr as soon as a partial sum is.
__device__ __forceinline__ bool smem_sig(const ThreadSmem& t, const SmemThreadArgs& a, double lp, bool left,
                                         int32_t lim) {
    if (a.thr_all) return true;
    double ll = __dadd_rn(0.0, lp);
    if (ll <= a.thr) return true;
    if (left) {
        for (int32_t i = 0; i < lim; ++i) {
            ll = __dadd_rn(ll, c_llk[t.base(i)]);
            if (ll <= a.thr) return true;
        }
    } else {
        for (int32_t i = lim; i < t.L; ++i) {
            ll = __dadd_rn(ll, c_llk[t.base(i)]);
            if (ll <= a.thr) return true;
        }
    }
    return false;
}

// The walks push candidates shortest first; storing them downward from the
// top of the thread's list leaves pv[pv_base ..] longest first, which is the
// order the reference gets from std::reverse (SMEM.cpp:90, 145).
__device__ __forceinline__ void smem_push(ThreadSmem& t, const SmemThreadArgs& a, PrevEntry* pv, const SmemState32& m,
                                          int32_t pos) {
    if (t.n_prev < a.pv_cap) {
        PrevEntry e;
        e.p = m.p; e.q = m.q; e.s = m.s; e.lp = m.lp; e.pos = pos;
        pv[a.pv_cap - 1 - t.n_prev] = e;
        t.n_prev++;
    } else {
        atomicOr(a.status, 0x100u);  // list longer than the cap: the batch reruns on the warp kernel
        t.ovf = 1;
    }
}

// Apply the result of the extension requested by smem_advance.
__device__ __forceinline__ void smem_apply(ThreadSmem& t, const SmemThreadArgs& a, PrevEntry* pv, uint32_t P, uint32_t Q,
                                           uint32_t S) {
    switch (t.phase) {
        case PH_FB_WALK: {  // SMEM.cpp:79-86
            t.m.q = (uint32_t)P; t.m.p = (uint32_t)Q; t.m.s = (uint32_t)S;
            const int nb = t.base(t.m.to);
            if (t.m.to < t.L) t.m.lp = __dadd_rn(t.m.lp, c_llk[nb]);
            t.m.to++;
            if (t.m.s != t.m0.s && t.m0.to >= a.min_len && smem_sig(t, a, t.m0.lp, true, t.m0.from))
                smem_push(t, a, pv, t.m0, t.m0.to);
            t.m0 = t.m;
            break;
        }
        case PH_BF_WALK: {  // SMEM.cpp:134-141
            t.m.p = (uint32_t)P; t.m.q = (uint32_t)Q; t.m.s = (uint32_t)S;
            if (t.m.from > 0) t.m.lp = __dadd_rn(t.m.lp, c_llk[t.base(t.m.from - 1)]);
            t.m.from--;
            if (t.m.s != t.m0.s && t.L - t.m0.from >= a.min_len && smem_sig(t, a, t.m0.lp, false, t.m0.to))
                smem_push(t, a, pv, t.m0, t.m0.from);
            t.m0 = t.m;
            break;
        }
        case PH_FB_ENTRY:
        case PH_BF_ENTRY: {  // SMEM.cpp:97-112 / 152-167
            const bool fb = t.phase == PH_FB_ENTRY;
            PrevEntry e = t.e0;
            if (fb) { e.p = (uint32_t)P; e.q = (uint32_t)Q; } else { e.q = (uint32_t)P; e.p = (uint32_t)Q; }
            e.s = (uint32_t)S;
            const bool add = fb ? (t.cf > 0) : (t.ct < t.L);
            if (add) e.lp = __dadd_rn(e.lp, c_llk[t.b2]);
            const int32_t e_from = fb ? t.cf : t.e0.pos;
            const int32_t e_to = fb ? t.e0.pos : t.ct;
            if (e.s != t.e0.s && t.e0.s >= 1 && t.n_valid == 0 && e_to - e_from >= a.min_len &&
                (a.thr_all || t.e0.lp <= a.thr))
                smem_emit(t, a, e_from, e_to, t.e0);
            if (e.s >= 1 && e.s != t.s0) {
                t.s0 = e.s;
                t.n_valid++;
                pv[t.pv_base + t.n_keep++] = e;
            }
            t.k++;
            break;
        }
        default:
            break;
    }
}

__global__ void __launch_bounds__(128) k_smem_thread(SmemThreadArgs a, IndexDev ix) {
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    PrevEntry* pv = a.prev + tid * a.pv_cap;
    ThreadSmem t;
    t.phase = PH_NEXT_READ;
    t.ext = 0;
    t.n_out = 0;
    t.r = -1;
    bool alive = true;  // this lane still has reads to take
    for (;;) {
        uint32_t P = 0, Q = 0, S = 0;
        int B = 0;
        bool have = false;
        while (alive && !have) {
            if (t.phase == PH_NEXT_READ || t.phase == PH_DONE) {
                if (t.phase == PH_DONE) {
                    a.count[t.r] = t.n_out;
                    if (t.n_out > a.cap) atomicOr(a.status, kErrOverflow);
                }
                const unsigned long long r = atomicAdd(a.work, 1ull);
                if ((int64_t)r >= a.n_reads) { alive = false; break; }
                t.r = (int32_t)r;
                const int64_t o0 = a.off[r];
                t.rd = a.seq + o0;
                t.L = (int32_t)(a.off[r + 1] - o0);
                t.out = a.out + 6 * (int64_t)r * a.cap;
                t.n_out = 0;
                t.ovf = 0;
                if (t.L <= 0) { t.phase = PH_DONE; continue; }
                t.from = t.L / 2;  // SMEM.cpp:189-191
                t.to = t.from + 1;
                smem_call_fb(t, ix, 0, t.from);
                continue;
            }
            have = smem_advance(t, a, ix, pv, P, Q, S, B);
        }
        // Reconverge the warp so that every lane with a pending extension
        // issues its bucket loads in the same instructions.
        __syncwarp();
        if (!__any_sync(0xffffffffu, alive)) break;
        if (have) {
            if (is_basic(B)) t.ext++;
            back_ext32(ix, P, Q, S, B);
        }
        __syncwarp();
        if (have) smem_apply(t, a, pv, P, Q, S);
    }
    if (t.ext) atomicAdd(a.n_ext, t.ext);
}

}  // namespace msg
