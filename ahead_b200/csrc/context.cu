// context.cu -- ahead_ctx lifetime and bookkeeping entry points of the C ABI.
#include "context.cuh"

extern "C" {

int ahead_ctx_create(int device, void* stream, ahead_ctx** out) {
    if (!out) return AHEAD_BAD_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return AHEAD_CUDA_ERROR;
    if (device < 0 || device >= ndev) return AHEAD_BAD_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return AHEAD_CUDA_ERROR;
    ahead::noalloc_forget_device(device);
    ahead_ctx* c = new ahead_ctx();
    c->device = device;
    cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (stream) {
        c->stream = (cudaStream_t)stream;
    } else {
        if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete c;
            return AHEAD_CUDA_ERROR;
        }
        c->own_stream = true;
    }
    if (cudaMallocHost(&c->h_stage, ahead::kStageWords * sizeof(uint64_t)) != cudaSuccess) {
        if (c->own_stream) cudaStreamDestroy(c->stream);
        delete c;
        return AHEAD_NO_MEMORY;
    }
    *out = c;
    return AHEAD_OK;
}

void ahead_ctx_destroy(ahead_ctx* c) {
    if (!c) return;
    cudaStreamSynchronize(c->stream);
    if (c->arena) cudaFree(c->arena);
    if (c->h_stage) cudaFreeHost(c->h_stage);
    if (c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
}

void* ahead_ctx_stream(ahead_ctx* c) { return c ? (void*)c->stream : nullptr; }

const char* ahead_ctx_last_error(ahead_ctx* c) { return c ? c->err.c_str() : "no context"; }

uint64_t ahead_ctx_launches(ahead_ctx* c) { return c ? c->launches : 0; }

uint64_t ahead_ctx_scratch_bytes(ahead_ctx* c) { return c ? (uint64_t)c->arena_cap : 0; }

const char* ahead_status_string(int s) {
    static const char* names[] = {"OK",         "BAD_ARG",   "SIZE_MISMATCH", "CAPACITY",
                                  "TIMEOUT",    "CUDA_ERROR", "NO_MEMORY",    "UNSUPPORTED"};
    return (s >= 0 && s < 8) ? names[s] : "UNKNOWN";
}

}  // extern "C"
