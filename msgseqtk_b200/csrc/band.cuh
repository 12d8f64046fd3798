// Learned DP band (included by map.cu after map_kernels.cuh).
//
// A chain's 5' and 3' flank rectangles hold most of the reference cell set
// when its seeds cover little of the read. A small classifier picks, per
// chain, the half-width of a diagonal band around the adjacent seed's diagonal
// (7, 15 or 31) or the whole rectangle; the DP certifies every banded result
// (see dp_chain) and recomputes uncertified chains on the whole cell set, so
// the records are the reference's whatever the classifier says.
//
// Classifier: 16 chain features -> 64 -> 64 -> 4 (ReLU), bf16 weights, fp32
// accumulation. Trained on the GPU by k_mlp_grad (forward, softmax cross
// entropy, backward, per-block weight-gradient reduction) and k_adam.
#pragma once
#include <cuda_bf16.h>

#include "map_kernels.cuh"

namespace msg {

constexpr int kFeat = MSG_BAND_FEATURES;
constexpr int kHid = MSG_BAND_HIDDEN;
constexpr int kCls = MSG_BAND_CLASSES;
// parameter vector layout (floats): feature mean, feature scale, W1 (row j:
// weights of hidden unit j), b1, W2, b2, W3, b3
constexpr int kOffMu = 0;
constexpr int kOffSd = kFeat;
constexpr int kOffW1 = 2 * kFeat;
constexpr int kOffB1 = kOffW1 + kHid * kFeat;
constexpr int kOffW2 = kOffB1 + kHid;
constexpr int kOffB2 = kOffW2 + kHid * kHid;
constexpr int kOffW3 = kOffB2 + kHid;
constexpr int kOffB3 = kOffW3 + kCls * kHid;
constexpr int kNParams = kOffB3 + kCls;
constexpr int kNTrain = kNParams - kOffW1;  // trainable part (weights and biases)
static_assert(kNParams == MSG_BAND_NPARAMS, "parameter layout");

// class -> band half-width (-1: the whole rectangle)
__host__ __device__ inline int band_width(int cls) { return cls == 0 ? 7 : cls == 1 ? 15 : cls == 2 ? 31 : -1; }

// Chain statistics for the classifier (all from the chain, the read and the
// target window):
//  0 log2(1+seeds)  1 L/256  2 seed coverage of the read  3 5' rows/L
//  4 (5' cols - rows)/L  5 3' rows/L  6 (3' cols - rows)/L  7 log2(1+diagonal spread)
//  8 largest read gap/L  9 largest target gap/L  10 log2(1+sum |gap rows - gap cols|)
//  11 log2(1+chains of the read)  12 longest seed/L  13 shortest seed/L
//  14 log2(1+flank area)  15 mismatch rate of the flanks on the seeds' diagonals
__global__ void k_chain_features(IndexDev ix, const Seed* __restrict__ seeds, const int64_t* __restrict__ chain_idx_off,
                                 const int32_t* __restrict__ chain_len, const int32_t* __restrict__ chain_read,
                                 const int64_t* __restrict__ chain_idx, const int64_t* __restrict__ roff,
                                 const uint8_t* __restrict__ rseq, const int64_t* __restrict__ read_chain_off,
                                 const int4* __restrict__ geo, int64_t n_chain, DpParams pp, float* __restrict__ feat) {
    const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= n_chain) return;
    const int64_t* idx = chain_idx + chain_idx_off[c];
    const int n = chain_len[c];
    const int64_t r = chain_read[c];
    const int64_t L = roff[r + 1] - roff[r];
    const Seed f = seeds[idx[0]], l = seeds[idx[n - 1]];
    const int4 g = geo[c];
    int64_t sum_len = 0, longest = 0, shortest = INT64_MAX, dmin = INT64_MAX, dmax = INT64_MIN, maxq = 0, maxt = 0, indel = 0;
    for (int k = 0; k < n; ++k) {
        const Seed s = seeds[idx[k]];
        const int64_t len = s.to - s.from;
        sum_len += len;
        longest = max(longest, len);
        shortest = min(shortest, len);
        const int64_t d = s.start - s.from;
        dmin = min(dmin, d);
        dmax = max(dmax, d);
        if (k + 1 < n) {
            const Seed t = seeds[idx[k + 1]];
            const int64_t R = t.from - s.to, C = t.start - s.end;
            maxq = max(maxq, R);
            maxt = max(maxt, C);
            indel += R > C ? R - C : C - R;
        }
    }
    // ungapped mismatches of the 5' flank on the first seed's diagonal and of
    // the 3' flank on the last seed's
    const uint8_t* rd = rseq + roff[r];
    const uint8_t* chr = ix.chr_seq + ix.chr_off[f.tid];
    const int64_t clen = ix.chr_len[f.tid];
    auto qbase = [&](int64_t i) { return f.strand == FWD ? (int)rd[i] : comp16(rd[L - 1 - i]); };
    auto tbase = [&](int64_t t) { return (t >= 0 && t < clen) ? (int)__ldg(chr + t) : 0; };
    auto miss = [&](int qb, int tb) { return !((qb & tb) && qb != 15 && tb != 15); };
    int64_t mm = 0;
    for (int64_t d = 1; d <= g.x; ++d) mm += miss(qbase(f.from - d), tbase(f.start - d));
    for (int64_t d = 0; d < g.z; ++d) mm += miss(qbase(l.to + d), tbase(l.end + d));
    const float iL = L > 0 ? 1.0f / (float)L : 0.0f;
    const int64_t area = (int64_t)max(g.x, 0) * max(g.y, 0) + (int64_t)max(g.z, 0) * max(g.w, 0);
    float* o = feat + c * kFeat;
    o[0] = log2f(1.0f + (float)n);
    o[1] = (float)L * (1.0f / 256.0f);
    o[2] = (float)sum_len * iL;
    o[3] = (float)g.x * iL;
    o[4] = (float)(g.y - g.x) * iL;
    o[5] = (float)g.z * iL;
    o[6] = (float)(g.w - g.z) * iL;
    o[7] = log2f(1.0f + (float)(dmax - dmin));
    o[8] = (float)maxq * iL;
    o[9] = (float)maxt * iL;
    o[10] = log2f(1.0f + (float)indel);
    o[11] = log2f(1.0f + (float)(read_chain_off[r + 1] - read_chain_off[r]));
    o[12] = (float)longest * iL;
    o[13] = (float)shortest * iL;
    o[14] = log2f(1.0f + (float)area);
    o[15] = (float)mm / (float)(g.x + g.z + 1);
    (void)pp;
}

// Forward pass of one sample on weights held in shared memory as floats.
__device__ inline int mlp_class(const float* __restrict__ xr, const float* __restrict__ W, const float* __restrict__ nrm) {
    float x[kFeat];
#pragma unroll
    for (int i = 0; i < kFeat; ++i) x[i] = (xr[i] - nrm[i]) / nrm[kFeat + i];
    const float* W1 = W;
    const float* B1 = W1 + kHid * kFeat;
    const float* W2 = B1 + kHid;
    const float* B2 = W2 + kHid * kHid;
    const float* W3 = B2 + kHid;
    const float* B3 = W3 + kCls * kHid;
    float h1[kHid];
#pragma unroll
    for (int j = 0; j < kHid; ++j) {
        float acc = B1[j];
#pragma unroll
        for (int i = 0; i < kFeat; ++i) acc = fmaf(W1[j * kFeat + i], x[i], acc);
        h1[j] = fmaxf(acc, 0.0f);
    }
    float z[kCls];
#pragma unroll
    for (int c = 0; c < kCls; ++c) z[c] = B3[c];
    for (int j = 0; j < kHid; ++j) {
        float acc = B2[j];
#pragma unroll
        for (int k = 0; k < kHid; ++k) acc = fmaf(W2[j * kHid + k], h1[k], acc);
        const float h = fmaxf(acc, 0.0f);
#pragma unroll
        for (int c = 0; c < kCls; ++c) z[c] = fmaf(W3[c * kHid + j], h, z[c]);
    }
    int best = 0;
#pragma unroll
    for (int c = 1; c < kCls; ++c) if (z[c] > z[best]) best = c;
    return best;
}

constexpr int64_t kSmallArea = 256;  // plain chains up to this many rectangle cells run one thread each

// A band of half-width w is used on an R x C flank rectangle when it covers
// less than half of it (at most R (2w+1) cells).
__host__ __device__ inline bool bandable(int R, int C, int w) {
    return R > 0 && C > 0 && w < max(R, C) - 1 && 2 * (2 * w + 1) < C;
}

// DP classes of a chain. The chains of a range are sorted by class, then by
// the sizes of their 5' and 3' flank rectangles (half powers of two, larger
// first), then by area (larger first); each class runs as one launch over its
// part of the sorted list. The threads of a warp then hold chains of similar
// shape -- their flank fills run side by side rather than one after the
// other -- and the launch ends on small chains.
enum DpClass : int {
    kDpSmall = 0,       // unbanded, area <= small_area: k_dp_small (thread, row by row)
    kDpStripe = 1,      // unbanded, up to warp_area: k_dp_stripe (thread, register stripes)
    kDpStripeBand = 2,  // banded, up to warp_area: k_dp_stripe with bands
    kDpWarp = 3,        // unbanded, larger: k_dp (warp wavefront)
    kDpWarpBand = 4,    // banded, larger: k_dp with bands
    kDpClasses = 5
};
// Counter block of the DP stage (unsigned long long words): class sizes
// [0, kDpClasses), the fallback lists of the stripe and warp kernels, the
// traceback list, then the statistics (fallback, exact, dropped, then cells
// computed per class), then per class the work counter of its launch (chains
// handed out so far).
static_assert(kDpWarp == kDpClassWarp, "DP class numbering");
constexpr int kCtrFbStripe = 5, kCtrFbWarp = 6, kCtrTrace = 7, kCtrStat = 8, kCtrQueue = 16, kCtrWords = 24;
constexpr int kKeyAreaBits = 11;
constexpr int kKeyBits = kKeyAreaBits + 5 + 5 + 3;

// size class (0..31) of a flank area: half powers of two
__device__ __forceinline__ uint32_t area_class(int64_t a) {
    if (a <= 0) return 0u;
    const int b = 63 - __clzll((unsigned long long)a);                  // floor(log2 a)
    const int half = b >= 1 && ((unsigned long long)a >> (b - 1)) >= 3;  // a >= 1.5 * 2^b
    return (uint32_t)min(31, 1 + 2 * b + half);
}

__global__ void k_iota(int64_t c0, int64_t n, int64_t* __restrict__ v) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) v[i] = c0 + i;
}

// Band half-widths per chain, its DP class and sort key.
// mode 0: no band; 1: fixed_w for every chain above kSmallArea; 2: the
// classifier's choice for chains above kSmallArea with a flank that a band of
// half-width 7 would cut. Each flank is banded only when bandable().
__global__ void __launch_bounds__(128) k_band_assign(int64_t c0, int64_t n_chain, const int4* __restrict__ geo,
                                                     const int64_t* __restrict__ area, const float* __restrict__ feat,
                                                     int mode, int fixed_w, const __nv_bfloat16* __restrict__ wts,
                                                     const float* __restrict__ nrm, int64_t small_area,
                                                     int64_t warp_area, int8_t* __restrict__ band,
                                                     unsigned long long* __restrict__ counts,
                                                     uint32_t* __restrict__ key) {
    __shared__ float sW[kNTrain];
    __shared__ float sN[2 * kFeat];
    if (mode == 2) {
        for (int k = threadIdx.x; k < kNTrain; k += blockDim.x) sW[k] = __bfloat162float(wts[k]);
        for (int k = threadIdx.x; k < 2 * kFeat; k += blockDim.x) sN[k] = nrm[k];
        __syncthreads();
    }
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;  // chains c0 .. c0 + n_chain
    int cls = -1;
    if (t < n_chain) {
        const int64_t c = c0 + t;
        const int4 g = geo[c];
        const int64_t ar = area[c];
        int w = -1;
        if (ar > kSmallArea) {  // small chains are never banded
            if (mode == 1) w = fixed_w;
            else if (mode == 2 && (bandable(g.x, g.y, band_width(0)) || bandable(g.z, g.w, band_width(0))))
                w = band_width(mlp_class(feat + c * kFeat, sW, sN));
        }
        const int w5 = (w >= 0 && bandable(g.x, g.y, w)) ? w : -1;
        const int w3 = (w >= 0 && bandable(g.z, g.w, w)) ? w : -1;
        band[2 * c] = (int8_t)w5;
        band[2 * c + 1] = (int8_t)w3;
        const bool huge = ar > warp_area;
        if (w5 >= 0 || w3 >= 0) cls = huge ? kDpWarpBand : kDpStripeBand;
        else if (ar <= small_area) cls = kDpSmall;
        else cls = huge ? kDpWarp : kDpStripe;
        const uint32_t amax = (1u << kKeyAreaBits) - 1u;
        const uint32_t q5 = 31u - area_class((int64_t)max(g.x, 0) * max(g.y, 0));
        const uint32_t q3 = 31u - area_class((int64_t)max(g.z, 0) * max(g.w, 0));
        key[t] = ((uint32_t)cls << (kKeyAreaBits + 10)) | (q5 << (kKeyAreaBits + 5)) | (q3 << kKeyAreaBits) |
                 (amax - (uint32_t)min(ar >> 5, (int64_t)amax));
    }
#pragma unroll
    for (int q = 0; q < kDpClasses; ++q) {  // one atomic per warp and class
        const unsigned b = __ballot_sync(0xffffffffu, cls == q);
        if ((threadIdx.x & 31) == 0 && b) atomicAdd(&counts[q], (unsigned long long)__popc(b));
    }
}

// ---------------------------------------------------------------------------
// Training
// ---------------------------------------------------------------------------
constexpr int kTile = 64;           // samples per block of k_mlp_grad
constexpr int kTs = kTile + 1;      // row stride of the [unit][sample] tiles (bank-conflict free)

__global__ void k_normalize(int64_t n, const float* __restrict__ raw, const float* __restrict__ nrm, float* __restrict__ out) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n * kFeat) return;
    const int i = (int)(k % kFeat);
    out[k] = (raw[k] - nrm[i]) / nrm[kFeat + i];
}

__global__ void k_to_bf16(int n, const float* __restrict__ w, __nv_bfloat16* __restrict__ wb) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) wb[k] = __float2bfloat16_rn(w[k]);
}

// Gradient of (sum over samples of the cross entropy) * inv_n for the samples
// order[lo .. hi), added to grad (kNTrain floats); the summed loss is added
// to *loss. Shared memory: weights (float), then the x, h1, h2, d2, d1, dz
// tiles.
__global__ void __launch_bounds__(kTile) k_mlp_grad(const float* __restrict__ xn, const int32_t* __restrict__ label,
                                                   const int32_t* __restrict__ order, int64_t lo, int64_t hi,
                                                   const __nv_bfloat16* __restrict__ wts, float inv_n,
                                                   float* __restrict__ grad, float* __restrict__ loss) {
    extern __shared__ float sm[];
    float* W = sm;
    float* X = W + kNTrain;
    float* H1 = X + kFeat * kTs;
    float* H2 = H1 + kHid * kTs;
    float* D2 = H2 + kHid * kTs;
    float* D1 = D2 + kHid * kTs;
    float* DZ = D1 + kHid * kTs;
    __shared__ float red[kTile];
    const float* W1 = W;
    const float* B1 = W1 + kHid * kFeat;
    const float* W2 = B1 + kHid;
    const float* B2 = W2 + kHid * kHid;
    const float* W3 = B2 + kHid;
    const float* B3 = W3 + kCls * kHid;
    const int t = threadIdx.x;
    for (int k = t; k < kNTrain; k += kTile) W[k] = __bfloat162float(wts[k]);
    const int64_t s = lo + (int64_t)blockIdx.x * kTile + t;
    const bool valid = s < hi;
    const int64_t row = valid ? (order ? (int64_t)order[s] : s) : 0;
    for (int i = 0; i < kFeat; ++i) X[i * kTs + t] = valid ? xn[row * kFeat + i] : 0.0f;
    __syncthreads();
    // forward
    for (int j = 0; j < kHid; ++j) {
        float acc = B1[j];
        for (int i = 0; i < kFeat; ++i) acc = fmaf(W1[j * kFeat + i], X[i * kTs + t], acc);
        H1[j * kTs + t] = fmaxf(acc, 0.0f);
    }
    float z[kCls];
    for (int c = 0; c < kCls; ++c) z[c] = B3[c];
    for (int j = 0; j < kHid; ++j) {
        float acc = B2[j];
        for (int k = 0; k < kHid; ++k) acc = fmaf(W2[j * kHid + k], H1[k * kTs + t], acc);
        const float h = fmaxf(acc, 0.0f);
        H2[j * kTs + t] = h;
        for (int c = 0; c < kCls; ++c) z[c] = fmaf(W3[c * kHid + j], h, z[c]);
    }
    // softmax cross entropy
    float mx = z[0];
    for (int c = 1; c < kCls; ++c) mx = fmaxf(mx, z[c]);
    float se = 0.0f;
    float p[kCls];
    for (int c = 0; c < kCls; ++c) { p[c] = expf(z[c] - mx); se += p[c]; }
    const int y = valid ? label[row] : 0;
    float zy = z[0];
    for (int c = 1; c < kCls; ++c) if (c == y) zy = z[c];
    red[t] = valid ? (logf(se) + mx - zy) : 0.0f;
    for (int c = 0; c < kCls; ++c) DZ[c * kTs + t] = valid ? (p[c] / se - (c == y ? 1.0f : 0.0f)) * inv_n : 0.0f;
    // backward through the hidden layers
    for (int j = 0; j < kHid; ++j) {
        float acc = 0.0f;
        for (int c = 0; c < kCls; ++c) acc = fmaf(W3[c * kHid + j], DZ[c * kTs + t], acc);
        D2[j * kTs + t] = H2[j * kTs + t] > 0.0f ? acc : 0.0f;
    }
    for (int k = 0; k < kHid; ++k) {
        float acc = 0.0f;
        for (int j = 0; j < kHid; ++j) acc = fmaf(W2[j * kHid + k], D2[j * kTs + t], acc);
        D1[k * kTs + t] = H1[k * kTs + t] > 0.0f ? acc : 0.0f;
    }
    __syncthreads();
    // weight gradients: sums over the tile's samples
    for (int q = t; q < kNTrain; q += kTile) {
        const float* a;
        const float* b = nullptr;
        if (q < kOffB1 - kOffW1) { a = D1 + (q / kFeat) * kTs; b = X + (q % kFeat) * kTs; }
        else if (q < kOffW2 - kOffW1) { a = D1 + (q - (kOffB1 - kOffW1)) * kTs; }
        else if (q < kOffB2 - kOffW1) { const int u = q - (kOffW2 - kOffW1); a = D2 + (u / kHid) * kTs; b = H1 + (u % kHid) * kTs; }
        else if (q < kOffW3 - kOffW1) { a = D2 + (q - (kOffB2 - kOffW1)) * kTs; }
        else if (q < kOffB3 - kOffW1) { const int u = q - (kOffW3 - kOffW1); a = DZ + (u / kHid) * kTs; b = H2 + (u % kHid) * kTs; }
        else { a = DZ + (q - (kOffB3 - kOffW1)) * kTs; }
        float acc = 0.0f;
        if (b) for (int m = 0; m < kTile; ++m) acc = fmaf(a[m], b[m], acc);
        else for (int m = 0; m < kTile; ++m) acc += a[m];
        atomicAdd(grad + q, acc);
    }
    for (int o = kTile / 2; o > 0; o >>= 1) {
        __syncthreads();
        if (t < o) red[t] += red[t + o];
    }
    if (t == 0) atomicAdd(loss, red[0]);
}

constexpr size_t kGradSmem = sizeof(float) * ((size_t)kNTrain + (size_t)(kFeat + 4 * kHid + kCls) * kTs);

// Adam step on the fp32 master weights; the bf16 copy is what the forward
// and backward passes read.
__global__ void k_adam(int n, float* __restrict__ w, __nv_bfloat16* __restrict__ wb, const float* __restrict__ g,
                       float* __restrict__ m, float* __restrict__ v, float lr, float beta1, float beta2, float eps,
                       float bc1, float bc2) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const float gk = g[k];
    const float mk = beta1 * m[k] + (1.0f - beta1) * gk;
    const float vk = beta2 * v[k] + (1.0f - beta2) * gk * gk;
    m[k] = mk;
    v[k] = vk;
    const float wk = w[k] - lr * (mk / bc1) / (sqrtf(vk / bc2) + eps);
    w[k] = wk;
    wb[k] = __float2bfloat16_rn(wk);
}

}  // namespace msg
