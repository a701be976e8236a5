// context.cuh -- the ahead_ctx behind the C ABI and the per-call scope that
// carves device scratch out of the context's arena.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <memory>
#include <string>

#include "../../include/ahead_gpu.h"
#include "common.cuh"
#include "compact.cuh"

struct ahead_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    char* arena = nullptr;  // device scratch, reused by every call
    size_t arena_cap = 0;
    uint64_t* h_stage = nullptr;  // pinned host words for count read-back
    uint64_t launches = 0;
    int num_sms = 148;
    std::string err;
    // staging buffers of the table loader (pinned host + device text blocks),
    // kept across loads; freed with the context
    std::shared_ptr<void> loader;
};

namespace ahead {

constexpr int kStageWords = 64;

// noalloc.cu: drop the cached scratch address of a device (a new context may
// follow a device reset).
void noalloc_forget_device(int dev);

inline int fail(ahead_ctx* ctx, int status, const std::string& what) {
    if (ctx) ctx->err = what;
    return status;
}

inline int cuda_fail(ahead_ctx* ctx, cudaError_t e, const char* where) {
    return fail(ctx, AHEAD_CUDA_ERROR, std::string(where) + ": " + cudaGetErrorString(e));
}

#define AHEAD_CUDA(ctx, call)                                      \
    do {                                                           \
        cudaError_t _e = (call);                                   \
        if (_e != cudaSuccess) return ::ahead::cuda_fail((ctx), _e, #call); \
    } while (0)

// One operator call.  Layout of the arena: [status word + 63 counters][bump
// region].  reserve() must be called with the call's total scratch need
// before any pointer is handed out (it may reallocate the arena).
struct OpScope {
    ahead_ctx* ctx;
    size_t off = 0;
    uint32_t* d_status = nullptr;
    uint64_t* d_counters = nullptr;  // [kStageWords - 1]
    int rc = AHEAD_OK;

    explicit OpScope(ahead_ctx* c) : ctx(c) {}

    int reserve(size_t bytes) {
        size_t need = 512 + bytes + 256;
        if (need > ctx->arena_cap) {
            cudaError_t e = cudaStreamSynchronize(ctx->stream);
            if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamSynchronize");
            if (ctx->arena) cudaFree(ctx->arena);
            ctx->arena = nullptr;
            size_t cap = need < (64u << 20) ? (64u << 20) : need + need / 4;
            e = cudaMalloc(&ctx->arena, cap);
            if (e != cudaSuccess) {
                ctx->arena_cap = 0;
                return fail(ctx, AHEAD_NO_MEMORY, "scratch arena allocation failed");
            }
            ctx->arena_cap = cap;
        }
        d_status = (uint32_t*)ctx->arena;
        d_counters = (uint64_t*)(ctx->arena + 8);
        off = 512;
        cudaError_t e = cudaMemsetAsync(ctx->arena, 0, 512, ctx->stream);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemsetAsync");
        return AHEAD_OK;
    }

    void* alloc(size_t bytes) {
        off = (off + 255) & ~size_t(255);
        void* p = ctx->arena + off;
        off += bytes;
        return p;
    }

    // Compaction scratch for `ntiles` tiles and `nchan` streams; the stream
    // totals land in d_counters[first_counter ...].  Only the per-tile counts
    // need clearing; every other word is written before it is read.
    CompactBufs compact_bufs(uint32_t ntiles, uint32_t nchan, int first_counter) {
        CompactBufs cb;
        cb.words = (uint32_t*)alloc((size_t)ntiles * kTileWords * 4);
        cb.counts = (uint32_t*)alloc((size_t)ntiles * nchan * 4);
        cb.offsets = (uint64_t*)alloc((size_t)ntiles * nchan * 8);
        cb.gbase = (uint64_t*)alloc((size_t)scan_groups(ntiles) * nchan * 8);
        cb.totals = d_counters + first_counter;
        cb.ntiles = ntiles;
        cb.nchan = nchan;
        cudaMemsetAsync(cb.counts, 0, (size_t)ntiles * nchan * 4, ctx->stream);
        return cb;
    }

    void launched(int n = 1) { ctx->launches += n; }

    // Copy the status word and the first `ncounters` counters to the host and
    // wait for the stream.  Returns the call's status.
    int finish(int ncounters) {
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(ctx, e, "kernel launch");
        e = cudaMemcpyAsync(ctx->h_stage, ctx->arena, 8 + 8 * (size_t)ncounters, cudaMemcpyDeviceToHost,
                            ctx->stream);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemcpyAsync");
        e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamSynchronize");
        uint32_t st = (uint32_t)ctx->h_stage[0];
        if (st & kDevStatusTimeout) return fail(ctx, AHEAD_TIMEOUT, "a bounded device wait gave up");
        if (st & kDevStatusBadInput) return fail(ctx, AHEAD_UNSUPPORTED, "input outside the supported domain");
        return AHEAD_OK;
    }
    uint64_t counter(int i) const { return ctx->h_stage[1 + i]; }
};

inline DCol dcol(const ahead_col& c) {
    DCol d;
    d.data = c.data;
    d.seqbase = c.seqbase;
    d.type = c.type;
    d.width = type_width(c.type);
    d.enc = type_encoded(c.type);
    d.ainv = d.enc ? (c.Ainv & wmask(d.width)) : 0;
    d.umax = c.unenc_max & wmask(d.width);
    d.pad = 0;
    return d;
}

inline void set_meta(ahead_col* c, int type, uint64_t A, uint64_t Ainv, uint64_t umax, uint64_t seq) {
    c->type = type;
    c->A = (uint16_t)A;  // ColumnMetaData::AN_A is a 16-bit A_t
    c->Ainv = Ainv;
    c->unenc_max = umax;
    c->seqbase = seq;
}
inline void copy_meta(ahead_col* c, int type, const ahead_col* src) {
    set_meta(c, type, src->A, src->Ainv, src->unenc_max, src->seqbase);
}
// ColumnDescriptor's default metadata: A=1, Ainv=1, unencMaxU=0 and, for a
// non-void column, seqbase = sizeof(type_t) (ColumnDescriptor.hpp:39-41 picks
// the oid_t seqbase constructor of ColumnMetaData).
inline void default_meta(ahead_col* c, int type) {
    set_meta(c, type, 1, 1, 0, type == AHEAD_VOID ? 0 : (uint64_t)type_width(type));
}
inline uint64_t type_unenc_max(int t) {
    switch (t) {
        case AHEAD_RESTINY: return 0xFF;
        case AHEAD_RESSHORT: return 0xFFFF;
        case AHEAD_RESINT: return 0xFFFFFFFFull;
        default: return kRes56Max;
    }
}

inline void ev_begin(ahead_errvec* e, int present) {
    if (!e) return;
    e->present = present;
    e->count = 0;
}

// Modular inverse of odd a modulo 2^bits (Newton iteration x <- x(2 - ax)).
inline uint64_t inv_pow2(uint64_t a, int bits) {
    uint64_t x = a;  // correct to 3 bits for odd a
    for (int i = 0; i < 6; ++i) x *= 2 - a * x;
    return x & wmask(bits / 8);
}

inline uint32_t compact_tiles(uint64_t n) { return (uint32_t)((n + kTileRows - 1) / kTileRows); }

// A kernel's dynamic shared-memory limit is a function attribute of each
// device: set it once per device (the context's, current in the calling
// thread), tracked per kernel in a set of devices 0..63 (beyond that it is
// set on every call).  False when the attribute could not be set.
template <auto Kernel>
inline bool dyn_smem_ready(const ahead_ctx* ctx, int bytes) {
    static std::atomic<uint64_t> done{0};
    const int dev = ctx->device;
    const uint64_t bit = (dev >= 0 && dev < 64) ? (1ull << dev) : 0ull;
    if (bit && (done.load(std::memory_order_acquire) & bit)) return true;
    if (cudaFuncSetAttribute(Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) != cudaSuccess) {
        cudaGetLastError();  // (not sticky)
        return false;
    }
    if (bit) done.fetch_or(bit, std::memory_order_acq_rel);
    return true;
}

// Pass 1 of a compaction: the bulk-copy fed classify kernel for 16-byte
// aligned columns (when its shared memory could be granted), else the one
// that loads rows directly.
template <class Op>
inline void launch_classify(const ahead_ctx* ctx, cudaStream_t st, const Op& op, uint64_t n, const CompactBufs& cb) {
    const uint32_t nt = cb.ntiles;
    constexpr int smem = RingCfg<Op::W>::SMEM;
    if (((uintptr_t)op.base & 15) == 0 && dyn_smem_ready<classify_kernel<Op, true>>(ctx, smem)) {
        const uint32_t g2 = nt < (uint32_t)ctx->num_sms * 3 ? nt : (uint32_t)ctx->num_sms * 3;
        classify_kernel<Op, true><<<g2, kCThreads, smem, st>>>(op, n, cb);
    } else {
        const uint32_t cap = (uint32_t)ctx->num_sms * 8;
        classify_kernel<Op, false><<<nt < cap ? nt : cap, kCThreads, 0, st>>>(op, n, cb);
    }
}

// Launch one compaction over n rows (classify, scan, emit); totals land in
// counters [c0, c0+NCH).
template <class Op>
inline void run_compact(OpScope& s, const Op& op, uint64_t n, int c0) {
    if (n == 0) return;
    const uint32_t nt = compact_tiles(n);
    CompactBufs cb = s.compact_bufs(nt, Op::NCH, c0);
    const uint32_t cap = (uint32_t)s.ctx->num_sms * 8;
    const uint32_t grid = nt < cap ? nt : cap;
    launch_classify(s.ctx, s.ctx->stream, op, n, cb);
    tile_scan_kernel<<<scan_groups(nt), kScanGroup, 0, s.ctx->stream>>>(cb);
    group_scan_kernel<<<1, 1024, 0, s.ctx->stream>>>(cb);
    emit_kernel<Op><<<grid, kCThreads, 0, s.ctx->stream>>>(op, n, cb);
    s.launched(4);
}

template <class Op>
inline size_t compact_scratch(uint64_t n) {
    if (n == 0) return 0;
    return compact_bytes(compact_tiles(n), Op::NCH) + 1024;
}

}  // namespace ahead
