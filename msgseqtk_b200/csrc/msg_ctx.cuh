// Context object behind the C ABI: one CUDA stream, the device index image and
// reusable per-batch device buffers.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/msg_b200.h"
#include "msg_internal.cuh"

namespace msg {

// The device allocations of one loaded index. Held through a shared_ptr by
// the context that loaded it and by every context that shares it
// (msg_ctx_share_index); the last holder to let go frees them.
struct IndexMem {
    int device = 0;
    void* p[9] = {};
    ~IndexMem();
};

struct IndexImage {
    bool loaded = false;
    std::shared_ptr<IndexMem> mem;  // set once a load has succeeded
    Bucket* bkt = nullptr;
    int64_t* dollar_rows = nullptr;
    int64_t* n_rows = nullptr;
    uint32_t* n_before = nullptr;
    uint32_t* sa = nullptr;
    uint8_t* text = nullptr;
    uint32_t* isa = nullptr;
    int64_t* chr_tab = nullptr;
    uint8_t* chr_seq = nullptr;
    int64_t B[16] = {0};
    double llk[16] = {0};
    int64_t bytes = 0;
    std::vector<int64_t> chr_len_host;  // chromosome lengths, for host-side checks of caller arrays
    IndexDev dev{};
};

// A grow-only device buffer reused across batches.
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= cap) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        size_t want = bytes + bytes / 4 + 256;
        cudaError_t e = cudaMalloc(&p, want);
        if (e == cudaSuccess) cap = want;
        return e;
    }
    template <typename T> T* as() const { return static_cast<T*>(p); }
    void release() { if (p) cudaFree(p); p = nullptr; cap = 0; }
};

// Makes `device` current for the scope of an entry point and gives the
// caller's current device back on exit, so a call never changes which device
// the calling thread has selected.
struct DeviceGuard {
    int prev = -1;
    bool ok = false;
    explicit DeviceGuard(int device) {
        if (cudaGetDevice(&prev) != cudaSuccess) { prev = -1; return; }
        ok = prev == device || cudaSetDevice(device) == cudaSuccess;
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
    DeviceGuard(const DeviceGuard&) = delete;
    DeviceGuard& operator=(const DeviceGuard&) = delete;
};

inline IndexMem::~IndexMem() {
    DeviceGuard g(device);
    for (void* q : p)
        if (q) cudaFree(q);
}

}  // namespace msg

struct msg_ctx {
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    msg::IndexImage idx;
    std::string last_error;
    msg_map_stats stats{};
    // batch buffers
    msg::DevBuf reads, offs, smem, smem_cnt, prev, sel, seedoff, seeds, seeds2, rcount, chains, chainidx, dpinfo,
        scratch, path, alnbuf, cigbuf, misc, status, geobuf, bandbuf, alnbuf2, recoff, rlist, prevw, hsort;
    // band model (bf16 weights, fp32 feature mean/scale) and training buffers
    msg::DevBuf band_wts, band_nrm, tr_x, tr_y, tr_ord, tr_w, tr_m, tr_v, tr_g, tr_loss;
    // MEM search / read cleaning: per-unit loglik and counts, clean outputs, MEM rows, row slots
    msg::DevBuf memo, memo2, memrows, memslot;
    // msg_map_batches: a copy stream, two input slots and two result staging slots
    cudaStream_t cstream = nullptr;
    cudaEvent_t pev[6] = {};  // [0..1] upload done, [2..3] staged, [4..5] download done
    msg::DevBuf in_seq[2], in_off[2], stage[2];
    bool band_loaded = false;
    int64_t scratch_limit = 16ll << 30;  // DP rectangle storage per pass (msg_ctx_set_scratch_limit)
    // DP work split (msg_ctx_set_dp_shape): unbanded chains of at most
    // dp_small_area rectangle cells run row by row on one thread, chains of
    // at most dp_warp_area in register stripes of dp_k rows on one thread,
    // larger ones on a warp
    int dp_k = 16;
    int dp_lanes = 16;     // 16: unbanded GLOBAL stripe chains that fit use 16-bit lanes (msg_ctx_set_dp_lanes)
    int dp_stripe_blocks = 3;  // register budget of the stripe kernel: 3 or 4 resident blocks (msg_ctx_set_dp_occupancy)
    int smem_ff = 0;       // SMEM walks and single-entry passes skip unique matches by text comparison (variant 7)
    int smem_variant = 0;  // SMEM thread path (msg_ctx_set_smem_shape): 0 one read per thread, 1/2 two,
                           // 3/4 a pass's candidates extended several at a time
    int64_t smem_cap = 16;  // SMEM rows per 150 read bases the slots start with (grows after an overflow)
    int64_t dp_small_area = 64;
    int64_t dp_warp_area = 262144;
    cudaEvent_t ev[8];
    int64_t* hpin = nullptr;  // pinned host words for counts copied back without extra waits
    // DP class launches side by side: three streams forked from `stream`
    cudaStream_t dp_side[3] = {};
    cudaEvent_t dp_ev[4] = {};
    cudaError_t dp_streams_ready() {
        if (dp_side[0]) return cudaSuccess;
        for (auto& s : dp_side) {
            const cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
            if (e != cudaSuccess) return e;
        }
        for (auto& e : dp_ev) {
            const cudaError_t r = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
            if (r != cudaSuccess) return r;
        }
        return cudaSuccess;
    }
    const msg_aln* res_aln = nullptr;
    const uint32_t* res_cigar = nullptr;
    const int64_t* res_off = nullptr;

    int fail(int code, const char* why) {
        last_error = why;
        return code;
    }
    int cuda_fail(cudaError_t e) {
        last_error = cudaGetErrorString(e);
        return e == cudaErrorMemoryAllocation ? MSG_ENOMEM : MSG_ECUDA;
    }
    void buffers_free() {
        for (msg::DevBuf* b : {&reads, &offs, &smem, &smem_cnt, &prev, &sel, &seedoff, &seeds, &seeds2, &rcount,
                               &chains, &chainidx, &dpinfo, &scratch, &path, &alnbuf, &cigbuf, &misc, &status, &geobuf,
                               &bandbuf, &alnbuf2, &recoff, &rlist, &prevw, &hsort, &band_wts, &band_nrm, &tr_x, &tr_y,
                               &tr_ord, &tr_w, &tr_m, &tr_v, &tr_g, &tr_loss, &memo, &memo2, &memrows, &memslot,
                               &in_seq[0], &in_seq[1], &in_off[0], &in_off[1], &stage[0], &stage[1]})
            b->release();
        if (cstream) {
            for (cudaEvent_t& e : pev) cudaEventDestroy(e);
            cudaStreamDestroy(cstream);
            cstream = nullptr;
        }
        for (auto& s : dp_side) if (s) { cudaStreamSynchronize(s); cudaStreamDestroy(s); s = nullptr; }
        for (auto& e : dp_ev) if (e) { cudaEventDestroy(e); e = nullptr; }
    }
    // After a successful load the image's allocations move into a shared
    // IndexMem; index_free then only drops this context's hold on them.
    bool index_own() {
        try {
            auto m = std::make_shared<msg::IndexMem>();
            m->device = device;
            void* ps[9] = {idx.bkt, idx.dollar_rows, idx.n_rows, idx.n_before, idx.sa, idx.text, idx.isa,
                           idx.chr_tab, idx.chr_seq};
            for (int k = 0; k < 9; ++k) m->p[k] = ps[k];
            idx.mem = std::move(m);
        } catch (const std::bad_alloc&) {
            return false;
        }
        return true;
    }
    void index_free() {
        if (idx.mem) {
            idx = msg::IndexImage();  // frees the allocations if no other context holds them
            return;
        }
        if (idx.bkt) cudaFree(idx.bkt);
        if (idx.dollar_rows) cudaFree(idx.dollar_rows);
        if (idx.n_rows) cudaFree(idx.n_rows);
        if (idx.n_before) cudaFree(idx.n_before);
        if (idx.sa) cudaFree(idx.sa);
        if (idx.text) cudaFree(idx.text);
        if (idx.isa) cudaFree(idx.isa);
        if (idx.chr_tab) cudaFree(idx.chr_tab);
        if (idx.chr_seq) cudaFree(idx.chr_seq);
        idx = msg::IndexImage();
    }
};
