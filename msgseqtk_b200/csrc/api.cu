// Context lifetime and status strings of the C ABI.
#include <cstdio>

#include "msg_ctx.cuh"

extern "C" const char* msg_strerror(int status) {
    switch (status) {
        case MSG_OK: return "ok";
        case MSG_EINVAL: return "invalid argument";
        case MSG_ENOMEM: return "out of memory";
        case MSG_EUNSUPPORTED: return "unsupported input for the CUDA path";
        case MSG_ETIMEOUT: return "bounded device wait ran out";
        case MSG_ECUDA: return "CUDA runtime error";
        case MSG_ESTATE: return "call out of order";
        case MSG_EINTERNAL: return "device consistency check failed";
        default: return "unknown status";
    }
}

extern "C" int msg_ctx_create(int device, msg_ctx** out) {
    if (!out) return MSG_EINVAL;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return MSG_ECUDA;
    if (device < 0 || device >= n) return MSG_EINVAL;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return MSG_ECUDA;
    // the library carries sm_100a code only (no PTX): other architectures,
    // sm_103 and sm_120 included, could not launch its kernels
    if (prop.major != 10 || prop.minor != 0) return MSG_EUNSUPPORTED;
    msg::DeviceGuard dg_(device);
    if (!dg_.ok) return MSG_ECUDA;
    msg_ctx* c = new (std::nothrow) msg_ctx();
    if (!c) return MSG_ENOMEM;
    c->device = device;
    c->num_sms = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) { delete c; return MSG_ECUDA; }
    if (cudaHostAlloc(reinterpret_cast<void**>(&c->hpin), 64 * sizeof(int64_t), cudaHostAllocDefault) != cudaSuccess) {
        cudaStreamDestroy(c->stream);
        delete c;
        return MSG_ENOMEM;
    }
    for (auto& e : c->ev) cudaEventCreate(&e);
    *out = c;
    return MSG_OK;
}

extern "C" void msg_ctx_destroy(msg_ctx* c) {
    if (!c) return;
    msg::DeviceGuard dg_(c->device);
    cudaStreamSynchronize(c->stream);
    c->index_free();
    c->buffers_free();
    for (auto& e : c->ev) cudaEventDestroy(e);
    cudaStreamDestroy(c->stream);
    if (c->hpin) cudaFreeHost(c->hpin);
    delete c;
}

extern "C" const char* msg_last_error(const msg_ctx* c) { return c ? c->last_error.c_str() : ""; }
