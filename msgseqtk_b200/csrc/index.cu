// Index image construction on the device (msg_index_load) and the
// single-operation parity entry points (occ / bi-extension / SA queries).
#include <algorithm>
#include <cstring>
#include <vector>

#include <cub/cub.cuh>

#include "msg_ctx.cuh"

namespace msg {

// One thread per bucket: pack 64 nt16 BWT symbols into the two bit planes of
// their 2-bit codes and count $, A, C, G, N locally ('$' and N are stored as A).
__global__ void k_pack_buckets(const uint8_t* __restrict__ bwt, int64_t n, int64_t nb, Bucket* __restrict__ bkt,
                               uint32_t* __restrict__ cd, uint32_t* __restrict__ ca, uint32_t* __restrict__ cc,
                               uint32_t* __restrict__ cg, uint32_t* __restrict__ cn, uint32_t* __restrict__ bad) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= nb) return;
    uint32_t plo[2], phi[2];
    uint32_t nd = 0, na = 0, nc = 0, ng = 0, nn = 0;
    const int64_t base = k * kBucketSyms;
    for (int w = 0; w < 2; ++w) {
        uint32_t xl = 0, xh = 0;
        for (int t = 0; t < 32; ++t) {
            const int64_t i = base + w * 32 + t;
            int code = 0;
            if (i < n) {
                const int b = bwt[i];
                switch (b) {
                    case 0: nd++; code = 0; break;
                    case 1: na++; code = 0; break;
                    case 2: nc++; code = 1; break;
                    case 4: ng++; code = 2; break;
                    case 8: code = 3; break;
                    case 15: nn++; code = 0; break;
                    default: atomicOr(bad, 1u); break;
                }
            }
            xl |= (uint32_t)(code & 1) << t;
            xh |= (uint32_t)(code >> 1) << t;
        }
        plo[w] = xl;
        phi[w] = xh;
    }
    for (int w = 0; w < 2; ++w) { bkt[k].lo[w] = plo[w]; bkt[k].hi[w] = phi[w]; }
    cd[k] = nd; ca[k] = na; cc[k] = nc; cg[k] = ng; cn[k] = nn;
}

// Counts before each bucket; bit 31 of the '$' count flags a bucket holding a
// '$' or an N (exc: '$' and N in the bucket).
__global__ void k_fill_counts(int64_t nb, Bucket* __restrict__ bkt, const uint32_t* __restrict__ cd,
                              const uint32_t* __restrict__ ca, const uint32_t* __restrict__ cc,
                              const uint32_t* __restrict__ cg, const uint32_t* __restrict__ exc) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= nb) return;
    bkt[k].cnt[0] = cd[k] | (exc[k] ? 0x80000000u : 0u);
    bkt[k].cnt[1] = ca[k];
    bkt[k].cnt[2] = cc[k];
    bkt[k].cnt[3] = cg[k];
}

__global__ void k_add_u32(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b, int64_t n,
                          uint32_t* __restrict__ out) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k < n) out[k] = a[k] + b[k];
}

// Rows whose BWT symbol is `sym`, in any order.
__global__ void k_collect_rows(const uint8_t* __restrict__ bwt, int64_t n, int sym, int64_t* __restrict__ rows,
                               unsigned long long* __restrict__ cnt, int64_t cap) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (bwt[i] == sym) {
            const unsigned long long s = atomicAdd(cnt, 1ull);
            if ((int64_t)s < cap) rows[s] = i;
        }
    }
}

__global__ void k_mark_starts(const int64_t* __restrict__ rows, int64_t m, uint32_t* __restrict__ bits) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= m) return;
    const int64_t r = rows[k];
    atomicOr(&bits[r >> 5], 1u << (r & 31));
}

// Recover the full suffix array: every start row (an SA sample or a row whose
// suffix begins with '$') holds a known value; walking LF from it visits the
// rows of the preceding text positions until the next start row. LF never
// crosses a '$' because rows whose BWT symbol is '$' are SA samples
// (FMDIndex.cpp:465-480) and end every walk.
// The BD text from the BWT and the suffix array (text[sa[i] - 1] = bwt[i],
// cyclically), and the inverse suffix array.
__global__ void k_text_isa(const uint8_t* __restrict__ bwt, const uint32_t* __restrict__ sa, int64_t n,
                           uint8_t* __restrict__ text, uint32_t* __restrict__ isa) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = sa[i];
        isa[p] = (uint32_t)i;
        text[p == 0 ? n - 1 : p - 1] = bwt[i];
    }
}

__global__ void k_recover_sa(IndexDev ix, const int64_t* __restrict__ rows, const int64_t* __restrict__ vals,
                             int64_t m, const uint32_t* __restrict__ start_bits, uint32_t* __restrict__ sa,
                             uint32_t* __restrict__ err, int64_t max_walk) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= m) return;
    int64_t row = rows[k];
    int64_t val = vals[k];
    sa[row] = (uint32_t)val;
    for (int64_t step = 0; step < max_walk; ++step) {
        const int b = bwt_at(ix, row);
        if (b == 0) return;
        const Occ5 o = occ5(ix, row);
        const int64_t nxt = ix.C[b] + o.c[occ_slot(b)] - 1;
        if ((start_bits[nxt >> 5] >> (nxt & 31)) & 1u) return;
        val -= 1;
        row = nxt;
        sa[row] = (uint32_t)val;
    }
    atomicOr(err, kErrInternal);
}

// FMDIndex::accessSA (FMDIndex.cpp:520-527) for the rows of '$'-suffixes
// [0, d): LF-walk over base symbols until a sampled row, whose value plus the
// steps walked is the row's value. Used when those rows are not in the order
// a whole-text suffix sort gives them (databases merged by the reference's
// BWT merge, FMDIndex::append); a walk never meets a '$' because rows whose
// symbol is '$' are samples.
__global__ void k_dollar_sa(IndexDev ix, const int64_t* __restrict__ srows, const int64_t* __restrict__ svals,
                            int64_t ns, int64_t d, int64_t* __restrict__ out, uint32_t* __restrict__ err,
                            int64_t max_walk) {
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= d) return;
    int64_t row = r, dist = 0;
    for (int64_t step = 0; step <= max_walk; ++step) {
        int64_t lo = 0, hi = ns;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (srows[mid] < row) lo = mid + 1; else hi = mid;
        }
        if (lo < ns && srows[lo] == row) {
            out[r] = svals[lo] + dist;
            return;
        }
        const int b = bwt_at(ix, row);
        if (b == 0) break;
        const Occ5 o = occ5(ix, row);
        row = ix.C[b] + o.c[occ_slot(b)] - 1;
        ++dist;
    }
    atomicOr(err, kErrInternal);
}

__global__ void k_occ_query(IndexDev ix, int64_t cnt, const uint8_t* __restrict__ b, const int64_t* __restrict__ i,
                            int64_t* __restrict__ out) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= cnt) return;
    const int64_t pos = i[k];
    if (pos < 0 || pos >= ix.n) { out[k] = -1; return; }
    const Occ5 o = occ5(ix, pos);
    const int s = b[k];
    out[k] = (s == 0 || s == 15 || is_basic(s)) ? o.c[occ_slot(s)] : 0;
}

__global__ void k_ext_query(IndexDev ix, int64_t cnt, int dir, const uint8_t* __restrict__ b, int64_t* __restrict__ p,
                            int64_t* __restrict__ q, int64_t* __restrict__ s, int64_t* __restrict__ ret) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= cnt) return;
    int64_t P = p[k], Q = q[k], S = s[k];
    ret[k] = dir == 0 ? back_ext(ix, P, Q, S, b[k]) : fwd_ext(ix, P, Q, S, b[k]);
    p[k] = P; q[k] = Q; s[k] = S;
}

__global__ void k_sa_query(IndexDev ix, int64_t cnt, const int64_t* __restrict__ rows, int64_t* __restrict__ out) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= cnt) return;
    out[k] = ix.sa[rows[k]];
}

}  // namespace msg

using namespace msg;

static int64_t blocks_for(int64_t n, int t) { return (n + t - 1) / t; }

extern "C" int msg_index_load(msg_ctx* ctx, const msg_fmd_view* fmd, const msg_mtg_view* mtg) {
    if (!ctx || !fmd || !mtg || !fmd->bwt || !fmd->base_count || !fmd->sample_rows || !fmd->sample_vals ||
        !mtg->bd_start || !mtg->bd_end || !mtg->chr_len || !mtg->chr_seq || !mtg->chr_off)
        return MSG_EINVAL;
    msg::DeviceGuard dg_(ctx->device);
    if (!dg_.ok) return ctx->fail(MSG_ECUDA, "cudaSetDevice");
    const int64_t n = fmd->n;
    if (n <= 0 || fmd->n_samples <= 0 || mtg->n_chrom <= 0) return MSG_EINVAL;
    if (n >= (int64_t)0xFFFFFFFFll) return ctx->fail(MSG_EUNSUPPORTED, "BWT length must be below 2^32");
    const int64_t* B = fmd->base_count;
    int64_t tot = 0;
    for (int b = 0; b < 16; ++b) {
        if (B[b] < 0) return MSG_EINVAL;
        // FMDIndex::buildCounts rejects IUPAC-extended codes (FMDIndex.cpp:130-133)
        if (B[b] > 0 && !(b == 0 || b == 1 || b == 2 || b == 4 || b == 8 || b == 15))
            return ctx->fail(MSG_EINVAL, "BWT symbols other than $,A,C,G,T,N (IUPAC-extended codes)");
        tot += B[b];
    }
    if (tot != n) return MSG_EINVAL;
    for (int64_t t = 0; t < mtg->n_chrom; ++t)
        if (mtg->chr_len[t] <= 0 || mtg->bd_end[t] - mtg->bd_start[t] != 2 * (mtg->chr_len[t] + 1) ||
            mtg->chr_off[t + 1] - mtg->chr_off[t] != mtg->chr_len[t] || (t > 0 && mtg->bd_start[t] != mtg->bd_end[t - 1]))
            return ctx->fail(MSG_EINVAL, "inconsistent chromosome table");
    if (mtg->bd_start[0] != 0 || mtg->bd_end[mtg->n_chrom - 1] != n || B[0] != 2 * mtg->n_chrom)
        return ctx->fail(MSG_EINVAL, "chromosome table does not cover the BWT");

    ctx->index_free();
    IndexImage& im = ctx->idx;
    IndexDev& ix = im.dev;
    std::memset(&ix, 0, sizeof(ix));
    ix.n = n;
    int64_t S = 0;
    for (int i = 0; i <= 16; ++i) { ix.C[i] = S; S += i < 16 ? B[i] : 0; }  // FMDIndex.cpp:124-129
    for (int b = 0; b < 16; ++b) im.B[b] = B[b];

    cudaStream_t st = ctx->stream;
    const int64_t nb = n / kBucketSyms + 1;
    uint8_t* d_bwt = nullptr;
    uint32_t* tmp = nullptr;
    uint32_t* d_bad = nullptr;
    int rc = MSG_OK;
#define CK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { rc = ctx->cuda_fail(e_); goto done; } } while (0)
    CK(cudaMalloc(&im.bkt, nb * sizeof(Bucket)));
    CK(cudaMalloc(&d_bwt, n));
    CK(cudaMemcpyAsync(d_bwt, fmd->bwt, n, cudaMemcpyHostToDevice, st));
    CK(cudaMalloc(&tmp, 11 * nb * sizeof(uint32_t) + 16));
    CK(cudaMalloc(&d_bad, sizeof(uint32_t)));
    CK(cudaMemsetAsync(d_bad, 0, sizeof(uint32_t), st));
    {
        uint32_t* cd = tmp; uint32_t* ca = tmp + nb; uint32_t* cc = tmp + 2 * nb; uint32_t* cg = tmp + 3 * nb;
        uint32_t* sd = tmp + 4 * nb; uint32_t* sa_ = tmp + 5 * nb; uint32_t* sc = tmp + 6 * nb; uint32_t* sg = tmp + 7 * nb;
        uint32_t* ld = tmp + 8 * nb;
        uint32_t* cn = tmp + 9 * nb; uint32_t* sn = tmp + 10 * nb;
        k_pack_buckets<<<blocks_for(nb, 256), 256, 0, st>>>(d_bwt, n, nb, im.bkt, cd, ca, cc, cg, cn, d_bad);
        CK(cudaGetLastError());
        k_add_u32<<<blocks_for(nb, 256), 256, 0, st>>>(cd, cn, nb, ld);  // '$' and N of each bucket
        CK(cudaGetLastError());
        size_t tb = 0;
        CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, cd, sd, (int)nb, st));
        void* dt = nullptr;
        CK(cudaMalloc(&dt, tb));
        CK(cub::DeviceScan::ExclusiveSum(dt, tb, cd, sd, (int)nb, st));
        CK(cub::DeviceScan::ExclusiveSum(dt, tb, ca, sa_, (int)nb, st));
        CK(cub::DeviceScan::ExclusiveSum(dt, tb, cc, sc, (int)nb, st));
        CK(cub::DeviceScan::ExclusiveSum(dt, tb, cg, sg, (int)nb, st));
        k_fill_counts<<<blocks_for(nb, 256), 256, 0, st>>>(nb, im.bkt, sd, sa_, sc, sg, ld);
        CK(cudaGetLastError());
        if (B[15] > 0) {  // N before each bucket
            CK(cub::DeviceScan::ExclusiveSum(dt, tb, cn, sn, (int)nb, st));
            CK(cudaMalloc(&im.n_before, nb * sizeof(uint32_t)));
            CK(cudaMemcpyAsync(im.n_before, sn, nb * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
        }
        CK(cudaStreamSynchronize(st));
        cudaFree(dt);
    }
    {
        uint32_t bad = 0;
        CK(cudaMemcpy(&bad, d_bad, sizeof(uint32_t), cudaMemcpyDeviceToHost));
        if (bad) { rc = ctx->fail(MSG_EINVAL, "BWT holds symbols other than $,A,C,G,T,N"); goto done; }
    }
    // N rows of the BWT (sorted)
    if (B[15] > 0) {
        const int64_t nn = B[15];
        CK(cudaMalloc(&im.n_rows, nn * sizeof(int64_t)));
        unsigned long long* ncnt = reinterpret_cast<unsigned long long*>(tmp);
        CK(cudaMemsetAsync(ncnt, 0, sizeof(unsigned long long), st));
        k_collect_rows<<<ctx->num_sms * 8, 256, 0, st>>>(d_bwt, n, 15, im.n_rows, ncnt, nn);
        CK(cudaGetLastError());
        unsigned long long got = 0;
        CK(cudaMemcpyAsync(&got, ncnt, sizeof(got), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if ((int64_t)got != nn) { rc = ctx->fail(MSG_EINVAL, "number of N in the BWT differs from B[15]"); goto done; }
        std::vector<int64_t> nrows(nn);
        CK(cudaMemcpy(nrows.data(), im.n_rows, nn * sizeof(int64_t), cudaMemcpyDeviceToHost));
        std::sort(nrows.begin(), nrows.end());
        CK(cudaMemcpy(im.n_rows, nrows.data(), nn * sizeof(int64_t), cudaMemcpyHostToDevice));
        ix.n_rows = im.n_rows;
        ix.n_n = nn;
        ix.n_before = im.n_before;
    }
    // '$' rows of the BWT
    {
        const int64_t nd = B[0];
        CK(cudaMalloc(&im.dollar_rows, nd * sizeof(int64_t)));
        unsigned long long* dcnt = reinterpret_cast<unsigned long long*>(tmp);
        CK(cudaMemsetAsync(dcnt, 0, sizeof(unsigned long long), st));
        k_collect_rows<<<ctx->num_sms * 8, 256, 0, st>>>(d_bwt, n, 0, im.dollar_rows, dcnt, nd);
        CK(cudaGetLastError());
        unsigned long long got = 0;
        CK(cudaMemcpyAsync(&got, dcnt, sizeof(got), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if ((int64_t)got != nd) { rc = ctx->fail(MSG_EINVAL, "number of '$' in the BWT differs from B[0]"); goto done; }
        std::vector<int64_t> drows(nd);
        CK(cudaMemcpy(drows.data(), im.dollar_rows, nd * sizeof(int64_t), cudaMemcpyDeviceToHost));
        std::sort(drows.begin(), drows.end());
        CK(cudaMemcpy(im.dollar_rows, drows.data(), nd * sizeof(int64_t), cudaMemcpyHostToDevice));
        ix.bkt = im.bkt;
        ix.dollar_rows = im.dollar_rows;
        ix.n_dollar = nd;
        // Start rows: the SA samples plus the rows of '$'-suffixes [0, B[0]).
        // Row 0 is the final '$' (value n-1); the other '$'-suffixes sort as
        // the strand starts that follow them: the k-th BWT-'$' row in row
        // order, skipping the one holding text position 0, gives row k its
        // value minus one.
        const int64_t ns = fmd->n_samples;
        std::vector<int64_t> srows(fmd->sample_rows, fmd->sample_rows + ns);
        std::vector<int64_t> svals(fmd->sample_vals, fmd->sample_vals + ns);
        for (int64_t k = 1; k < ns; ++k)
            if (srows[k] <= srows[k - 1]) { rc = ctx->fail(MSG_EINVAL, "SA sample rows must be ascending"); goto done; }
        std::vector<int64_t> frows, fvals;
        frows.push_back(0);
        fvals.push_back(n - 1);
        for (int64_t r : drows) {
            auto it = std::lower_bound(srows.begin(), srows.end(), r);
            if (it == srows.end() || *it != r) { rc = ctx->fail(MSG_EINVAL, "a '$' row of the BWT is not an SA sample"); goto done; }
            const int64_t v = svals[it - srows.begin()];
            if (v == 0) continue;
            frows.push_back((int64_t)frows.size());
            fvals.push_back(v - 1);
        }
        std::vector<int64_t> arows, avals;
        // start rows: the samples merged with the '$'-suffix rows, dropping
        // duplicates; false when a duplicate's values disagree
        auto merge_starts = [&]() {
            arows.clear();
            avals.clear();
            arows.reserve(ns + nd);
            avals.reserve(ns + nd);
            size_t a = 0, f = 0;
            while (a < srows.size() || f < frows.size()) {
                if (f == frows.size() || (a < srows.size() && srows[a] < frows[f])) { arows.push_back(srows[a]); avals.push_back(svals[a]); ++a; }
                else if (a == srows.size() || frows[f] < srows[a]) { arows.push_back(frows[f]); avals.push_back(fvals[f]); ++f; }
                else {
                    if (svals[a] != fvals[f]) return false;
                    arows.push_back(srows[a]); avals.push_back(svals[a]); ++a; ++f;
                }
            }
            return true;
        };
        if ((int64_t)frows.size() != nd || !merge_starts()) {
            // the '$'-suffix rows are not in whole-text order (a merged
            // database): their values by accessSA walks on the device
            int64_t* d_sr = nullptr;
            int64_t* d_sv = nullptr;
            int64_t* d_dv = nullptr;
            cudaError_t e1 = cudaMalloc(&d_sr, (ns + 1) * sizeof(int64_t));
            if (e1 == cudaSuccess) e1 = cudaMalloc(&d_sv, (ns + 1) * sizeof(int64_t));
            if (e1 == cudaSuccess) e1 = cudaMalloc(&d_dv, (nd + 1) * sizeof(int64_t));
            if (e1 == cudaSuccess) e1 = cudaMemcpyAsync(d_sr, srows.data(), ns * sizeof(int64_t), cudaMemcpyHostToDevice, st);
            if (e1 == cudaSuccess) e1 = cudaMemcpyAsync(d_sv, svals.data(), ns * sizeof(int64_t), cudaMemcpyHostToDevice, st);
            if (e1 == cudaSuccess) e1 = cudaMemsetAsync(d_bad, 0, sizeof(uint32_t), st);
            if (e1 == cudaSuccess && nd > 0) {
                k_dollar_sa<<<blocks_for(nd, 128), 128, 0, st>>>(ix, d_sr, d_sv, ns, nd, d_dv, d_bad,
                                                                 std::min<int64_t>(n + 1, (int64_t)1 << 22));
                e1 = cudaGetLastError();
            }
            fvals.assign(nd, 0);
            if (e1 == cudaSuccess && nd > 0)
                e1 = cudaMemcpyAsync(fvals.data(), d_dv, nd * sizeof(int64_t), cudaMemcpyDeviceToHost, st);
            uint32_t bad1 = 0;
            if (e1 == cudaSuccess) e1 = cudaMemcpyAsync(&bad1, d_bad, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
            if (e1 == cudaSuccess) e1 = cudaStreamSynchronize(st);
            cudaFree(d_sr);
            cudaFree(d_sv);
            cudaFree(d_dv);
            if (e1 != cudaSuccess) { rc = ctx->cuda_fail(e1); goto done; }
            if (bad1) { rc = ctx->fail(MSG_EINVAL, "a '$'-suffix row reaches no SA sample"); goto done; }
            frows.resize(nd);
            for (int64_t r = 0; r < nd; ++r) frows[r] = r;
            if (!merge_starts()) { rc = ctx->fail(MSG_EINVAL, "SA sample disagrees with the '$' rows"); goto done; }
        }
        const int64_t m = (int64_t)arows.size();
        int64_t* d_rows = nullptr;
        int64_t* d_vals = nullptr;
        uint32_t* d_bits = nullptr;
        const int64_t nwords = n / 32 + 1;
        CK(cudaMalloc(&im.sa, n * sizeof(uint32_t)));
        CK(cudaMalloc(&d_rows, m * sizeof(int64_t)));
        CK(cudaMalloc(&d_vals, m * sizeof(int64_t)));
        CK(cudaMalloc(&d_bits, nwords * sizeof(uint32_t)));
        CK(cudaMemcpyAsync(d_rows, arows.data(), m * sizeof(int64_t), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(d_vals, avals.data(), m * sizeof(int64_t), cudaMemcpyHostToDevice, st));
        CK(cudaMemsetAsync(d_bits, 0, nwords * sizeof(uint32_t), st));
        k_mark_starts<<<blocks_for(m, 256), 256, 0, st>>>(d_rows, m, d_bits);
        CK(cudaGetLastError());
        CK(cudaMemsetAsync(d_bad, 0, sizeof(uint32_t), st));
        k_recover_sa<<<blocks_for(m, 128), 128, 0, st>>>(ix, d_rows, d_vals, m, d_bits, im.sa, d_bad,
                                                          std::min<int64_t>(n + 1, (int64_t)1 << 22));
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(st));
        cudaFree(d_rows);
        cudaFree(d_vals);
        cudaFree(d_bits);
        uint32_t bad = 0;
        CK(cudaMemcpy(&bad, d_bad, sizeof(uint32_t), cudaMemcpyDeviceToHost));
        if (bad) { rc = ctx->fail(MSG_EINTERNAL, "suffix-array recovery did not terminate"); goto done; }
        ix.sa = im.sa;
        // the text and inverse suffix array the SMEM kernel's fast-forward
        // over unique matches reads
        CK(cudaMalloc(&im.text, n + 32));
        CK(cudaMalloc(&im.isa, n * sizeof(uint32_t)));
        CK(cudaMemsetAsync(im.text + n, 0, 32, st));
        k_text_isa<<<ctx->num_sms * 16, 256, 0, st>>>(d_bwt, im.sa, n, im.text, im.isa);
        CK(cudaGetLastError());
        ix.text = im.text;
        ix.isa = im.isa;
    }
    // chromosome table and targets
    {
        const int64_t nc = mtg->n_chrom;
        CK(cudaMalloc(&im.chr_tab, 4 * nc * sizeof(int64_t) + 8));
        CK(cudaMemcpyAsync(im.chr_tab, mtg->bd_start, nc * sizeof(int64_t), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(im.chr_tab + nc, mtg->bd_end, nc * sizeof(int64_t), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(im.chr_tab + 2 * nc, mtg->chr_len, nc * sizeof(int64_t), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(im.chr_tab + 3 * nc, mtg->chr_off, (nc + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st));
        const int64_t tl = mtg->chr_off[nc];
        CK(cudaMalloc(&im.chr_seq, tl + 16));
        CK(cudaMemcpyAsync(im.chr_seq, mtg->chr_seq, tl, cudaMemcpyHostToDevice, st));
        ix.bd_start = im.chr_tab;
        ix.bd_end = im.chr_tab + nc;
        ix.chr_len = im.chr_tab + 2 * nc;
        ix.chr_off = im.chr_tab + 3 * nc;
        ix.chr_seq = im.chr_seq;
        ix.n_chrom = nc;
        im.chr_len_host.assign(mtg->chr_len, mtg->chr_len + nc);
        im.bytes = nb * sizeof(Bucket) + B[0] * sizeof(int64_t) + 2 * n * sizeof(uint32_t) + n + 4 * nc * 8 + tl +
                   (B[15] > 0 ? B[15] * (int64_t)sizeof(int64_t) + nb * (int64_t)sizeof(uint32_t) : 0);
        CK(cudaStreamSynchronize(st));
    }
    // loglik table (FMDIndex::loglik, FMDIndex.h:195-197)
    {
        static const int to_basic[16] = {0, 1, 2, 2, 4, 4, 4, 4, 8, 8, 8, 8, 8, 8, 8, 15};
        for (int b = 0; b < 16; ++b) im.llk[b] = std::log((double)B[to_basic[b]]) - std::log((double)n);
    }
    if (!ctx->index_own()) {
        rc = ctx->fail(MSG_ENOMEM, "index ownership record");
        goto done;
    }
    im.loaded = true;
done:
#undef CK
    if (d_bwt) cudaFree(d_bwt);
    if (tmp) cudaFree(tmp);
    if (d_bad) cudaFree(d_bad);
    if (rc != MSG_OK) ctx->index_free();
    return rc;
}

extern "C" int msg_index_bytes(const msg_ctx* ctx, int64_t* bytes) {
    if (!ctx || !bytes) return MSG_EINVAL;
    if (!ctx->idx.loaded) return MSG_ESTATE;
    *bytes = ctx->idx.bytes;
    return MSG_OK;
}

extern "C" int msg_ctx_share_index(msg_ctx* ctx, const msg_ctx* owner) {
    if (!ctx || !owner || ctx == owner) return MSG_EINVAL;
    if (ctx->device != owner->device) return ctx->fail(MSG_EINVAL, "contexts on different devices");
    if (!owner->idx.loaded || !owner->idx.mem) return ctx->fail(MSG_ESTATE, "the owner has no index loaded");
    msg::DeviceGuard dg_(ctx->device);
    if (!dg_.ok) return ctx->fail(MSG_ECUDA, "cudaSetDevice");
    // work this context still has in flight may read its current index
    const cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return ctx->cuda_fail(e);
    try {
        msg::IndexImage im = owner->idx;  // copies the chromosome lengths: may throw
        ctx->index_free();
        ctx->idx = std::move(im);
    } catch (const std::bad_alloc&) {
        return ctx->fail(MSG_ENOMEM, "chromosome table");
    }
    return MSG_OK;
}

template <typename F>
static int run_query(msg_ctx* ctx, int64_t count, size_t bytes_in, F&& body) {
    if (!ctx) return MSG_EINVAL;
    if (!ctx->idx.loaded) return MSG_ESTATE;
    if (count <= 0) return MSG_OK;
    msg::DeviceGuard dg_(ctx->device);
    if (!dg_.ok) return ctx->fail(MSG_ECUDA, "cudaSetDevice");
    void* buf = nullptr;
    cudaError_t e = cudaMalloc(&buf, bytes_in);
    if (e != cudaSuccess) return ctx->cuda_fail(e);
    int rc = body(static_cast<char*>(buf));
    cudaFree(buf);
    return rc;
}

extern "C" int msg_occ_query(msg_ctx* ctx, int64_t count, const uint8_t* b, const int64_t* i, int64_t* out) {
    if (count > 0 && (!b || !i || !out)) return MSG_EINVAL;
    return run_query(ctx, count, count * 17 + 64, [&](char* buf) {
        uint8_t* db = reinterpret_cast<uint8_t*>(buf);
        int64_t* di = reinterpret_cast<int64_t*>(buf + ((count + 15) / 16) * 16);
        int64_t* dout = di + count;
        cudaStream_t st = ctx->stream;
        cudaMemcpyAsync(db, b, count, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(di, i, count * 8, cudaMemcpyHostToDevice, st);
        k_occ_query<<<blocks_for(count, 256), 256, 0, st>>>(ctx->idx.dev, count, db, di, dout);
        cudaMemcpyAsync(out, dout, count * 8, cudaMemcpyDeviceToHost, st);
        cudaError_t e = cudaStreamSynchronize(st);
        return e == cudaSuccess ? (int)MSG_OK : ctx->cuda_fail(e);
    });
}

extern "C" int msg_bi_ext_query(msg_ctx* ctx, int64_t count, int dir, const uint8_t* b, int64_t* p, int64_t* q,
                                int64_t* s, int64_t* ret) {
    if (count > 0 && (!b || !p || !q || !s || !ret)) return MSG_EINVAL;
    if (dir != 0 && dir != 1) return MSG_EINVAL;
    return run_query(ctx, count, count * 33 + 64, [&](char* buf) {
        uint8_t* db = reinterpret_cast<uint8_t*>(buf);
        int64_t* dp = reinterpret_cast<int64_t*>(buf + ((count + 15) / 16) * 16);
        int64_t* dq = dp + count;
        int64_t* ds = dq + count;
        int64_t* dr = ds + count;
        cudaStream_t st = ctx->stream;
        cudaMemcpyAsync(db, b, count, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(dp, p, count * 8, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(dq, q, count * 8, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(ds, s, count * 8, cudaMemcpyHostToDevice, st);
        k_ext_query<<<blocks_for(count, 256), 256, 0, st>>>(ctx->idx.dev, count, dir, db, dp, dq, ds, dr);
        cudaMemcpyAsync(p, dp, count * 8, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(q, dq, count * 8, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(s, ds, count * 8, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(ret, dr, count * 8, cudaMemcpyDeviceToHost, st);
        cudaError_t e = cudaStreamSynchronize(st);
        return e == cudaSuccess ? (int)MSG_OK : ctx->cuda_fail(e);
    });
}

extern "C" int msg_sa_query(msg_ctx* ctx, int64_t count, const int64_t* rows, int64_t* out) {
    if (count > 0 && (!rows || !out)) return MSG_EINVAL;
    for (int64_t k = 0; k < count; ++k)
        if (rows[k] < 0 || (ctx && rows[k] >= ctx->idx.dev.n)) return MSG_EINVAL;
    return run_query(ctx, count, count * 16 + 64, [&](char* buf) {
        int64_t* dr = reinterpret_cast<int64_t*>(buf);
        int64_t* dout = dr + count;
        cudaStream_t st = ctx->stream;
        cudaMemcpyAsync(dr, rows, count * 8, cudaMemcpyHostToDevice, st);
        k_sa_query<<<blocks_for(count, 256), 256, 0, st>>>(ctx->idx.dev, count, dr, dout);
        cudaMemcpyAsync(out, dout, count * 8, cudaMemcpyDeviceToHost, st);
        cudaError_t e = cudaStreamSynchronize(st);
        return e == cudaSuccess ? (int)MSG_OK : ctx->cuda_fail(e);
    });
}
