// SMEM search with one thread per read (included by map.cu after
// map_kernels.cuh). The reference's findAllSMEMS / findFwdBackSMEMS /
// findBackFwdSMEMS control flow (SMEM.cpp:64-215) is unrolled into a state
// machine whose every step performs exactly one bi-interval extension, so the
// occurrence-bucket loads of all 32 reads of a warp issue together. Candidate
// lists (`prev`) live in per-thread global scratch; their processing follows
// the reference's sequential loop entry by entry (validity by the running
// size s0, emission while nValid == 0, in-place compaction).
//
// findFwdBackSMEMS and findBackFwdSMEMS are mirror images: a walk that
// extends one end of the interval until it fails, then passes over the
// candidates that extend the other end. Both run on one code path here, with
// a direction flag `fb` and intervals kept "oriented", i.e. with the two
// bounds ordered so that the extension at hand is always a backward one
// (fwdExt(p, q) = backExt(q, p), FMDIndex.h:226-228): the walk's interval is
// (q, p) in a forward-then-backward call and (p, q) otherwise, and candidates
// are stored the other way round. Lanes of a warp in either kind of call then
// execute the same instructions.
#pragma once
#include <math_constants.h>

#include "map_kernels.cuh"

namespace msg {

// Interval bounds and sizes are below 2^32 (the index holds fewer than 2^32
// rows) and read positions below 2^31, so the per-thread state is 32-bit.
struct PrevEntry {
    double lp;
    uint32_t p, q, s;  // p, q in candidate orientation (see above)
    int32_t pos;       // `to` (fwd-back) or `from` (back-fwd) of the entry
};

struct SmemThreadArgs {
    const uint8_t* seq;
    const int64_t* off;
    int64_t n_reads;
    int64_t min_len;
    double thr;
    int thr_all;
    double llk_min, llk_max;  // extremes of the per-base log-likelihoods
    double llk[16];           // FMDIndex::loglik per nt16 code (by value: each context's own table)
    int64_t* out;
    int64_t cap;            // slot rows when out_off is null
    const int64_t* out_off; // per-read slot offsets (n + 1), or null: slot r at row r * cap
    const int64_t* list;    // reads handled by this launch (read k when null)
    int32_t* count;
    PrevEntry* prev;        // pv_cap entries per thread
    int64_t pv_cap;
    unsigned long long* work;
    unsigned long long* n_ext;
    unsigned long long* n_ffx;   // extensions replaced by the fast-forward over unique matches
    unsigned long long* n_ffs;   // fast-forward steps (one word or 16-byte text chunk loaded each)
    uint32_t* status;
    int64_t* ovf_list;      // reads abandoned because their candidate list outgrew pv_cap (rerun on k_smem)
    unsigned long long* ovf_n;
};

// per-block copy of the argument table: lanes index it by their own bases,
// which shared memory serves in one pass where the parameter (constant) bank
// would serialise
__shared__ double s_llk[16];

// Steps one read's state machine may take: at most 2L calls, each a walk of
// at most L extensions and at most L passes over at most pv_cap (48)
// candidates -- under 6.4 M for a 254-base read (about 500 on average); a
// read that exceeds the bound sets kErrInternal and ends, so a defect fails
// the batch loudly instead of running without end.
constexpr int32_t kSmemMaxSteps = 1 << 23;

enum SmemPhase : int {
    PH_NEXT_READ = 0,
    PH_OUTER_LOOP,      // while (from > 0 || to < L)
    PH_OUTER_BACK,      // --from; back-fwd call
    PH_WALK,            // the walk of either call
    PH_ITER,            // start of one pass over prev
    PH_ENTRY,           // one prev entry of that pass
    PH_DONE
};

struct ThreadSmem {
    const uint8_t* rd;
    int64_t* out;
    int32_t L;
    int32_t n_out;
    int32_t cap_r;          // rows of this read's slot
    int32_t r;
    // findAllSMEMS variables and the call in progress
    int32_t from, to;
    int32_t site;           // 0: first FB(from,to)  1: FB(from0,to)  2: BF(from,to0)
    int32_t fb;             // the call in progress is findFwdBackSMEMS
    int32_t cf, ct;         // the called function's from/to
    // walk state: oriented interval (wp, wq, s), log-likelihood, read range
    double lp;
    uint32_t wp, wq, s;
    int32_t mfrom, mto;
    // the walk's previous state (same range end on the fixed side)
    double lp0;
    uint32_t wp0, wq0, s0w;
    int32_t n_prev;
    int32_t pv_base;        // the list is pv[pv_base .. pv_base + n_prev), longest first
    int32_t ovf;            // a push found the list full: this read is abandoned (the warp kernel reruns it)
    // pass over prev
    int32_t k, n_keep, n_valid;
    uint32_t s0;            // running size; 0 stands for the reference's -1 (sizes compared are >= 1)
    int32_t b2;
    PrevEntry e0, e_next;   // entry being extended, and the next one (loaded early)
    int32_t phase;
    unsigned long long ext;
    int32_t steps;          // state-machine steps of the read in progress (bounded by kSmemMaxSteps)
    // fast-forward over a unique match (interval size 1): 0 none, 1 suffix
    // array word of the row, 2 text chunks, 3 inverse-suffix-array word
    int32_t ffst;
    int32_t ffent;          // the fast-forward extends the pass's single entry (else the walk)
    int32_t ffm;            // bases matched so far
    int32_t ffdone;         // a fast-forward just ended: the next extension is an ordinary one
    uint32_t ffp;           // the row at the start
    uint32_t ffpos;         // text position of its string (sa[ffp])
    unsigned long long ffx, ffs;

    __device__ int base(int32_t i) const { return (i >= 0 && i < L) ? (int)__ldg(rd + i) : 0; }
};

// Fast-forward over a unique match. While a walk's interval (or a pass's
// single candidate) has size 1, its string occurs once in the BD text, at
// sa[P], and extending it backward by base B keeps size 1 exactly when the
// text has B just before that occurrence (the row's BWT symbol); the new row
// is then the inverse suffix array at that position and q does not change
// (backExt only moves q when the size changes, FMDIndex.cpp:592-604). So a
// run of such extensions is the common prefix of the read's next bases and
// the text read backward from sa[P] - 1, and one inverse-suffix-array lookup
// gives the final row. Only basic read bases inside the read are taken; the
// extension that ends the run is an ordinary one. The run's steps (the
// suffix-array word, 16-byte text chunks, the inverse word) are steps of the
// state machine, so that their loads issue with the other lanes' bucket
// loads.
//
// Read position of the i-th base of a run (walk: at `to` going forward for
// findFwdBackSMEMS, before `from` going backward otherwise; pass: before cf
// or at ct), -1 past the read.
__device__ __forceinline__ int32_t ff_read_pos(const ThreadSmem& t, int32_t i) {
    int32_t pos;
    if (!t.ffent) pos = t.fb ? t.mto + i : t.mfrom - 1 - i;
    else pos = t.fb ? t.cf - 1 - i : t.ct + i;
    return (pos >= 0 && pos < t.L) ? pos : -1;
}
// The oriented base the i-th extension of the run prepends (-1: not a basic
// base inside the read): complemented when it extends the reverse strand.
__device__ __forceinline__ int ff_base(const ThreadSmem& t, int32_t i) {
    const int32_t pos = ff_read_pos(t, i);
    if (pos < 0) return -1;
    const int b = t.base(pos);
    if (!is_basic(b)) return -1;
    return (t.ffent ? !t.fb : t.fb) ? comp16(b) : b;
}

__device__ __forceinline__ uint32_t byte_of16(const uint4& v, int j) {
    const uint32_t w = j < 8 ? (j < 4 ? v.x : v.y) : (j < 12 ? v.z : v.w);
    return (w >> ((j & 3) * 8)) & 0xFFu;
}

__device__ __forceinline__ void smem_emit(ThreadSmem& t, const SmemThreadArgs& a, int32_t from, int32_t to,
                                          uint32_t p, uint32_t q, uint32_t s, double lp) {
    if (t.n_out < t.cap_r) {
        int64_t* o = t.out + 6 * (int64_t)t.n_out;
        o[0] = from; o[1] = to; o[2] = p; o[3] = q; o[4] = s;
        o[5] = __double_as_longlong(lp);
    }
    t.n_out++;
}

// Returns from the FB/BF call in progress to findAllSMEMS.
__device__ __forceinline__ void smem_return(ThreadSmem& t) {
    if (t.site == 0) { t.from = t.cf; t.to = t.ct; t.phase = PH_OUTER_LOOP; }
    else if (t.site == 1) { t.to = t.ct; t.phase = PH_OUTER_BACK; }
    else { t.from = t.cf; t.phase = PH_OUTER_LOOP; }
}

// Enter FB(cf, cf + 1) (SMEM.cpp:64-77) when fb, else BF(cf, cf + 1) (SMEM.cpp:119-132).
__device__ __forceinline__ void smem_call(ThreadSmem& t, const IndexDev& ix, int site, int fb, int32_t cf) {
    t.site = site;
    t.fb = fb;
    t.cf = cf;
    t.ct = cf + 1;
    const int b = t.base(cf);
    if (!is_basic(b)) { smem_return(t); return; }
    const uint32_t p = (uint32_t)ix.C[b], q = (uint32_t)ix.C[comp16(b)];
    t.wp = fb ? q : p;
    t.wq = fb ? p : q;
    t.s = (uint32_t)(ix.C[b + 1] - ix.C[b]);
    t.lp = __dadd_rn(0.0, s_llk[b]);
    t.mfrom = cf;
    t.mto = cf + 1;
    t.wp0 = t.wp; t.wq0 = t.wq; t.s0w = t.s; t.lp0 = t.lp;
    t.n_prev = 0;
    t.phase = PH_WALK;
}

// Advance the state machine until an extension is needed. On return with
// true, (P,Q,S,B) is the backward extension to perform.
// FF: runs over unique matches become fast-forward steps (k_smem_thread).
template <bool FF = false>
__device__ bool smem_advance(ThreadSmem& t, const SmemThreadArgs& a, const IndexDev& ix, PrevEntry* pv,
                             uint32_t& P, uint32_t& Q, uint32_t& S, int& B) {
    if (FF && t.ffst != 0) return true;  // a fast-forward run in progress takes its next step
    if (++t.steps > kSmemMaxSteps) {  // no read needs this many: a broken state machine ends the read
        atomicOr(a.status, kErrInternal);
        t.phase = PH_DONE;
        return false;
    }
    for (;;) {
        switch (t.phase) {
            case PH_OUTER_LOOP:
                if (!(t.from > 0 || t.to < t.L)) { t.phase = PH_DONE; return false; }
                if (t.to < t.L) { smem_call(t, ix, 1, 1, t.to); continue; }
                t.phase = PH_OUTER_BACK;
                continue;
            case PH_OUTER_BACK:
                t.from -= 1;
                if (t.from >= 0) { smem_call(t, ix, 2, 0, t.from); continue; }
                t.phase = PH_OUTER_LOOP;
                continue;
            case PH_WALK:
                if (t.s >= 1) {  // extend at `to` (fb, the base past the read is 0) or before `from`
                    if (FF && t.s == 1 && !t.ffdone) {
                        t.ffent = 0;
                        if (ff_base(t, 0) >= 0) {  // a run over a unique match starts
                            t.ffst = 1; t.ffm = 0; t.ffp = t.wp;
                            return true;
                        }
                    }
                    const int nb = t.fb ? t.base(t.mto) : t.base(t.mfrom - 1);
                    P = t.wp; Q = t.wq; S = t.s; B = t.fb ? comp16(nb) : nb;
                    return true;
                }
                if (t.fb) t.ct = t.mto; else t.cf = t.mfrom;
                if (t.ovf) { t.phase = PH_DONE; return false; }
                if (t.n_prev == 0) {
                    if (t.fb) t.cf--; else t.ct++;
                    smem_return(t);
                    continue;
                }
                t.pv_base = (int32_t)a.pv_cap - t.n_prev;
                t.phase = PH_ITER;
                continue;
            case PH_ITER: {
                // passes extend the other end: before cf (fb) or at ct (bf)
                const bool more = t.fb ? t.cf >= 0 : t.ct <= t.L;
                if (!(more && t.n_prev > 0)) { smem_return(t); continue; }
                if (FF && t.n_prev == 1 && !t.ffdone) {
                    const PrevEntry e = pv[t.pv_base];
                    t.ffent = 1;
                    if (e.s == 1 && ff_base(t, 0) >= 0) {  // the single candidate's run over a unique match
                        t.e0 = e;
                        t.ffst = 1; t.ffm = 0; t.ffp = e.p;
                        return true;
                    }
                }
                t.k = 0; t.n_keep = 0; t.s0 = 0; t.n_valid = 0;
                t.b2 = t.fb ? (t.cf > 0 ? t.base(t.cf - 1) : 0) : t.base(t.ct);
                t.e_next = pv[t.pv_base];
                t.phase = PH_ENTRY;
                continue;
            }
            case PH_ENTRY:
                if (t.k == t.n_prev) {
                    t.n_prev = t.n_keep;
                    if (t.fb) t.cf--; else t.ct++;
                    t.phase = PH_ITER;
                    continue;
                }
                t.e0 = t.e_next;
                if (t.k + 1 < t.n_prev) t.e_next = pv[t.pv_base + t.k + 1];
                P = t.e0.p; Q = t.e0.q; S = t.e0.s; B = t.fb ? t.b2 : comp16(t.b2);
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
// sum is <= thr as soon as a partial sum is. Each of the n terms lies in
// [llk_min, llk_max], so the sum lies within n of them of the start, up to a
// rounding error of about n * 2^-53 times the magnitudes (below 1e-10 for
// reads of a few hundred bases): bounds clear of thr by 1e-6 decide at once,
// and only the rest is summed term by term.
__device__ __forceinline__ bool smem_sig(const ThreadSmem& t, const SmemThreadArgs& a, double lp, int32_t i0,
                                         int32_t i1) {
    if (a.thr_all) return true;
    double ll = __dadd_rn(0.0, lp);
    if (ll <= a.thr) return true;
    const double n = (double)max(i1 - i0, 0);
    if (ll + n * a.llk_max <= a.thr - 1e-6) return true;
    if (ll + n * a.llk_min > a.thr + 1e-6) return false;
    for (int32_t i = i0; i < i1; ++i) {
        ll = __dadd_rn(ll, s_llk[t.base(i)]);
        if (ll <= a.thr) return true;
    }
    return false;
}

// The walks push candidates shortest first; storing them downward from the
// top of the thread's list leaves pv[pv_base ..] longest first, which is the
// order the reference gets from std::reverse (SMEM.cpp:90, 145).
__device__ __forceinline__ void smem_push(ThreadSmem& t, const SmemThreadArgs& a, PrevEntry* pv, int32_t pos) {
    if (t.n_prev < a.pv_cap) {
        PrevEntry e;
        e.p = t.wq0; e.q = t.wp0;  // candidate orientation is the walk's, swapped
        e.s = t.s0w; e.lp = t.lp0; e.pos = pos;
        pv[a.pv_cap - 1 - t.n_prev] = e;
        t.n_prev++;
    } else {
        atomicOr(a.status, 0x100u);  // list longer than the cap: this read reruns on the warp kernel
        t.ovf = 1;
    }
}

// One entry of a pass over prev (SMEM.cpp:97-112 (fb) / 152-167 (bf)): e0 is
// the entry before its extension, (P, Q, S) the extension's result.
__device__ __forceinline__ void smem_apply_entry(ThreadSmem& t, const SmemThreadArgs& a, PrevEntry* pv,
                                                 const PrevEntry& e0, uint32_t P, uint32_t Q, uint32_t S) {
    const bool fb = t.fb;
    PrevEntry e = e0;
    e.p = P; e.q = Q; e.s = S;
    const bool add = fb ? (t.cf > 0) : (t.ct < t.L);
    if (add) e.lp = __dadd_rn(e.lp, s_llk[t.b2]);
    const int32_t e_from = fb ? t.cf : e0.pos;
    const int32_t e_to = fb ? e0.pos : t.ct;
    if (e.s != e0.s && e0.s >= 1 && t.n_valid == 0 && e_to - e_from >= a.min_len && (a.thr_all || e0.lp <= a.thr))
        smem_emit(t, a, e_from, e_to, fb ? e0.p : e0.q, fb ? e0.q : e0.p, e0.s, e0.lp);
    if (e.s >= 1 && e.s != t.s0) {
        t.s0 = e.s;
        t.n_valid++;
        pv[t.pv_base + t.n_keep++] = e;
    }
    t.k++;
}

// Apply the result of the extension requested by smem_advance.
__device__ __forceinline__ void smem_apply(ThreadSmem& t, const SmemThreadArgs& a, PrevEntry* pv, uint32_t P, uint32_t Q,
                                           uint32_t S) {
    t.ffdone = 0;
    if (t.phase == PH_WALK) {  // SMEM.cpp:79-86 (fb) / 134-141 (bf)
        const bool fb = t.fb;
        t.wp = P; t.wq = Q; t.s = S;
        const int32_t np = fb ? t.mto : t.mfrom - 1;  // the base just added
        if (np >= 0 && np < t.L) t.lp = __dadd_rn(t.lp, s_llk[t.base(np)]);
        if (fb) t.mto++; else t.mfrom--;
        if (t.s != t.s0w) {
            // the previous state: its moving end is one step back
            const int32_t f0 = fb ? t.mfrom : t.mfrom + 1;
            const int32_t t0 = fb ? t.mto - 1 : t.mto;
            const bool long_enough = fb ? t0 >= a.min_len : t.L - f0 >= a.min_len;
            if (long_enough && (fb ? smem_sig(t, a, t.lp0, 0, f0) : smem_sig(t, a, t.lp0, t0, t.L)))
                smem_push(t, a, pv, fb ? t0 : f0);
        }
        t.wp0 = t.wp; t.wq0 = t.wq; t.s0w = t.s; t.lp0 = t.lp;
    } else if (t.phase == PH_ENTRY) {
        smem_apply_entry(t, a, pv, t.e0, P, Q, S);
    }
}

// One step of a fast-forward run with its loaded word (w.x for the
// suffix-array and inverse words, all of w for a text chunk).
__device__ __forceinline__ void smem_ff_apply(ThreadSmem& t, const SmemThreadArgs& a, PrevEntry* pv, const uint4& w) {
    t.ffs++;
    if (t.ffst == 1) {  // the string's text position
        t.ffpos = w.x;
        t.ffst = 2;
    } else if (t.ffst == 2) {  // compare the chunk holding text position ffpos - 1 - ffm, downward
        const uint32_t cb = (t.ffpos - 1u - (uint32_t)t.ffm) & ~15u;  // where this step's chunk starts
        for (;;) {
            if ((int64_t)t.ffpos - 1 - t.ffm < 0) { t.ffst = 3; break; }  // the text starts here
            const uint32_t x = t.ffpos - 1u - (uint32_t)t.ffm;
            if (x < cb) return;  // chunk done: the next step loads the one below
            const int b = ff_base(t, t.ffm);
            if (b < 0 || b != (int)byte_of16(w, (int)(x - cb))) { t.ffst = 3; break; }
            t.ffm++;
        }
        if (t.ffm == 0) { t.ffst = 0; t.ffdone = 1; }  // nothing to skip: the ordinary extension follows
    } else {  // the final row: commit the run's ffm extensions
        const int32_t m = t.ffm;
        if (!t.ffent) {  // SMEM.cpp:79-86 (fb) / 134-141 (bf), m times with the size staying 1
            for (int32_t i = 0; i < m; ++i) t.lp = __dadd_rn(t.lp, s_llk[t.base(ff_read_pos(t, i))]);
            t.wp = w.x;
            if (t.fb) t.mto += m; else t.mfrom -= m;
            t.wp0 = t.wp; t.wq0 = t.wq; t.s0w = t.s; t.lp0 = t.lp;
        } else {  // SMEM.cpp:97-112 (fb) / 152-167 (bf), m passes keeping the single entry
            PrevEntry e = t.e0;
            for (int32_t i = 0; i < m; ++i) e.lp = __dadd_rn(e.lp, s_llk[t.base(ff_read_pos(t, i))]);
            e.p = w.x;
            pv[t.pv_base] = e;
            if (t.fb) t.cf -= m; else t.ct += m;
        }
        t.ffx += (unsigned long long)m;
        t.ffst = 0;
        t.ffdone = 1;
    }
}

// Finish the read in progress (its count) and start the next one from the
// batch's work counter; false when the batch has no read left.
__device__ __forceinline__ bool smem_next_read(ThreadSmem& t, const SmemThreadArgs& a, const IndexDev& ix) {
    if (t.phase == PH_DONE) {
        if (t.ovf) {  // abandoned: the warp kernel maps it again
            a.ovf_list[atomicAdd(a.ovf_n, 1ull)] = t.r;
        } else {
            a.count[t.r] = t.n_out;
            if (t.n_out > t.cap_r) atomicOr(a.status, kErrOverflow);
        }
    }
    unsigned long long r = atomicAdd(a.work, 1ull);
    if ((int64_t)r >= a.n_reads) return false;
    if (a.list) r = (unsigned long long)a.list[r];
    t.r = (int32_t)r;
    const int64_t o0 = a.off[r];
    t.rd = a.seq + o0;
    t.L = (int32_t)(a.off[r + 1] - o0);
    const int64_t slot = a.out_off ? a.out_off[r] : (int64_t)r * a.cap;
    t.cap_r = (int32_t)(a.out_off ? a.out_off[r + 1] - slot : a.cap);
    t.out = a.out + 6 * slot;
    t.n_out = 0;
    t.ovf = 0;
    t.ffst = 0;
    t.ffdone = 0;
    t.steps = 0;
    if (t.L <= 0) { t.phase = PH_DONE; return true; }
    t.from = t.L / 2;  // SMEM.cpp:189-191
    t.to = t.from + 1;
    smem_call(t, ix, 0, 1, t.from);
    return true;
}

// MINB: resident blocks of 128 threads per SM the registers are sized for;
// FF: with the fast-forward over unique matches (the index's text and
// inverse suffix array).
template <int MINB, bool FF>
__global__ void __launch_bounds__(128, MINB) k_smem_thread(SmemThreadArgs a, IndexDev ix) {
    if (threadIdx.x < 16) s_llk[threadIdx.x] = a.llk[threadIdx.x];
    __syncthreads();
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    PrevEntry* pv = a.prev + tid * a.pv_cap;
    ThreadSmem t;
    t.phase = PH_NEXT_READ;
    t.ext = 0;
    t.ffx = 0;
    t.ffs = 0;
    t.ffst = 0;
    t.n_out = 0;
    t.r = -1;
    bool alive = true;  // this lane still has reads to take
    for (;;) {
        uint32_t P = 0, Q = 0, S = 0;
        int B = 0;
        bool have = false;
        while (alive && !have) {
            if (t.phase == PH_NEXT_READ || t.phase == PH_DONE) {
                alive = smem_next_read(t, a, ix);
                continue;
            }
            have = smem_advance<FF>(t, a, ix, pv, P, Q, S, B);
        }
        // Reconverge the warp so that every lane with a pending extension
        // issues its bucket loads in the same instructions.
        __syncwarp();
        if (!__any_sync(0xffffffffu, alive)) break;
        // a fast-forward step's word is requested first, so that its load is
        // in flight while the other lanes' extensions wait on theirs
        const bool ff = FF && have && t.ffst != 0;
        uint4 w = make_uint4(0u, 0u, 0u, 0u);
        if (ff) {
            if (t.ffst == 1) {
                w.x = __ldg(ix.sa + t.ffp);
            } else if (t.ffst == 2) {
                const int64_t x = (int64_t)t.ffpos - 1 - t.ffm;
                if (x >= 0) w = __ldg(reinterpret_cast<const uint4*>(ix.text + (x & ~(int64_t)15)));
            } else {
                w.x = __ldg(ix.isa + (t.ffpos - (uint32_t)t.ffm));
            }
        }
        if (have && !ff) {
            if (is_basic(B)) t.ext++;
            back_ext32(ix, P, Q, S, B);
        }
        __syncwarp();
        if (ff) smem_ff_apply(t, a, pv, w);
        else if (have) smem_apply(t, a, pv, P, Q, S);
    }
    if (t.ext) atomicAdd(a.n_ext, t.ext);
    if (FF && t.ffx) atomicAdd(a.n_ffx, t.ffx);
    if (FF && t.ffs) atomicAdd(a.n_ffs, t.ffs);
}

// Two reads per thread, each with its own state machine and candidate list:
// an iteration advances both to their next extension, issues the bucket loads
// of both, then finishes both, so that a thread has two extensions' loads in
// flight instead of one. Same per-read results as k_smem_thread. MINB: blocks
// of 128 threads per SM the registers are sized for (4: spills a little; 3:
// fewer resident threads).
template <int MINB>
__global__ void __launch_bounds__(128, MINB) k_smem_thread2(SmemThreadArgs a, IndexDev ix) {
    if (threadIdx.x < 16) s_llk[threadIdx.x] = a.llk[threadIdx.x];
    __syncthreads();
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    PrevEntry* pv[2] = {a.prev + (2 * tid) * a.pv_cap, a.prev + (2 * tid + 1) * a.pv_cap};
    ThreadSmem t[2];
    bool alive[2] = {true, true};
#pragma unroll
    for (int u = 0; u < 2; ++u) {
        t[u].phase = PH_NEXT_READ;
        t[u].ext = 0;
        t[u].n_out = 0;
        t[u].r = -1;
    }
    for (;;) {
        uint32_t P[2] = {0, 0}, Q[2] = {0, 0}, S[2] = {0, 0};
        int B[2] = {0, 0};
        bool have[2] = {false, false};
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            while (alive[u] && !have[u]) {
                if (t[u].phase == PH_NEXT_READ || t[u].phase == PH_DONE) {
                    alive[u] = smem_next_read(t[u], a, ix);
                    continue;
                }
                have[u] = smem_advance(t[u], a, ix, pv[u], P[u], Q[u], S[u], B[u]);
            }
        }
        __syncwarp();
        if (!__any_sync(0xffffffffu, alive[0] || alive[1])) break;
        ExtLoad l[2];
#pragma unroll
        for (int u = 0; u < 2; ++u)
            if (have[u] && is_basic(B[u])) back_ext32_load(ix, P[u], S[u], l[u]);
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            if (!have[u]) continue;
            if (is_basic(B[u])) {
                t[u].ext++;
                back_ext32_apply(ix, P[u], Q[u], S[u], B[u], l[u]);
            } else {
                S[u] = 0;
            }
        }
        __syncwarp();
#pragma unroll
        for (int u = 0; u < 2; ++u)
            if (have[u]) smem_apply(t[u], a, pv[u], P[u], Q[u], S[u]);
    }
    const unsigned long long e = t[0].ext + t[1].ext;
    if (e) atomicAdd(a.n_ext, e);
}

// 16 bytes from global to shared memory without passing through registers
// (cp.async: the copy is in flight until cp_async_wait_all).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// One read per thread, like k_smem_thread, but a step of a pass over the
// candidate list extends up to NB entries at once: the entries of one pass
// are independent (each is extended by the same base; only the bookkeeping
// after each extension -- running size, emission, compaction -- is ordered),
// so their bucket loads are issued together and their results applied in
// list order afterwards. The buckets land in shared memory (cp.async), four
// 16-byte words per extension at [4 j + w][thread], so a thread holds no
// registers for the loads in flight. The walks stay one extension per step
// (each depends on the previous). Same per-read results as k_smem_thread.
// MINB: resident blocks of 128 threads per SM the registers are sized for.
template <int NB, int MINB>
__global__ void __launch_bounds__(128, MINB) k_smem_pass(SmemThreadArgs a, IndexDev ix) {
    __shared__ uint4 s_bk[NB * 4][128];
    if (threadIdx.x < 16) s_llk[threadIdx.x] = a.llk[threadIdx.x];
    __syncthreads();
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int x = threadIdx.x;
    PrevEntry* pv = a.prev + tid * a.pv_cap;
    ThreadSmem t;
    t.phase = PH_NEXT_READ;
    t.ext = 0;
    t.n_out = 0;
    t.r = -1;
    bool alive = true;
    for (;;) {
        uint32_t P = 0, Q = 0, S = 0;
        int B = 0;
        bool have = false;
        while (alive && !have) {
            if (t.phase == PH_NEXT_READ || t.phase == PH_DONE) {
                alive = smem_next_read(t, a, ix);
                continue;
            }
            have = smem_advance(t, a, ix, pv, P, Q, S, B);
        }
        __syncwarp();
        if (!__any_sync(0xffffffffu, alive)) break;
        // this step's extensions: the walk's one, or entries k .. k+nb-1 of a pass
        // (entries 1.. keep only p and s in registers; they are read whole
        // again when applied: the batch writes only positions below them)
        int nb = 0;
        uint32_t Ep[NB], Es[NB];
        Ep[0] = P; Es[0] = S;
        if (have) {
            nb = 1;
            if (t.phase == PH_ENTRY) {
                nb = min(NB, t.n_prev - t.k);
#pragma unroll
                for (int j = 1; j < NB; ++j) {
                    if (j < nb) {
                        const PrevEntry& e = j == 1 ? t.e_next : pv[t.pv_base + t.k + j];
                        Ep[j] = e.p;
                        Es[j] = e.s;
                    }
                }
            }
        }
        const bool basic = is_basic(B);
        if (basic) {
#pragma unroll
            for (int j = 0; j < NB; ++j) {
                if (j < nb) {
                    const uint32_t p = Ep[j], sz = Es[j];
                    const uint32_t ka = p >> 6, kb = (p + sz) >> 6;
                    const uint4* ga = reinterpret_cast<const uint4*>(ix.bkt + ka);
                    cp_async16(&s_bk[4 * j][x], ga);
                    cp_async16(&s_bk[4 * j + 1][x], ga + 1);
                    if (kb != ka) {
                        const uint4* gb = reinterpret_cast<const uint4*>(ix.bkt + kb);
                        cp_async16(&s_bk[4 * j + 2][x], gb);
                        cp_async16(&s_bk[4 * j + 3][x], gb + 1);
                    }
                }
            }
        }
        cp_async_wait_all();
        __syncwarp();
#pragma unroll
        for (int j = 0; j < NB; ++j) {
            if (j < nb) {
                const bool entry = t.phase == PH_ENTRY;
                const PrevEntry e0 = !entry ? PrevEntry{} : j == 0 ? t.e0 : pv[t.pv_base + t.k];
                uint32_t p = Ep[j], q = j == 0 ? Q : e0.q, sz = Es[j];
                if (basic) {
                    t.ext++;
                    ExtLoad l;
                    l.a0 = s_bk[4 * j][x];
                    l.a1 = s_bk[4 * j + 1][x];
                    if (((p + sz) >> 6) != (p >> 6)) {
                        l.b0 = s_bk[4 * j + 2][x];
                        l.b1 = s_bk[4 * j + 3][x];
                    } else {
                        l.b0 = l.a0;
                        l.b1 = l.a1;
                    }
                    back_ext32_apply(ix, p, q, sz, B, l);
                } else {
                    sz = 0;
                }
                if (entry) smem_apply_entry(t, a, pv, e0, p, q, sz);
                else smem_apply(t, a, pv, p, q, sz);
            }
        }
        // the entry after the batch, for the next step (the batch wrote only
        // positions below it)
        if (have && t.phase == PH_ENTRY && nb > 1 && t.k < t.n_prev) t.e_next = pv[t.pv_base + t.k];
    }
    if (t.ext) atomicAdd(a.n_ext, t.ext);
}

}  // namespace msg
