// noalloc.cu -- checkAN that allocates nothing: the compaction's scratch is a
// fixed, file-scope device array instead of the context's growable arena.
//
// Who needs this.  ahead_gpu_check_an may grow the context's scratch arena,
// which means cudaFree + cudaMalloc.  Two kinds of caller cannot accept that:
//   * a caller running under a fixed device-memory budget after start-up, such
//     as a query server that admits work by its memory footprint -- an
//     operator that allocates in the middle of serving breaks that accounting
//     and can fail with out-of-memory while admitted work holds the rest;
//   * a caller that shares the device with latency-critical streams --
//     cudaFree synchronizes the whole device, so an arena reallocation stalls
//     every other stream until it completes.
// This entry point does no allocation of any kind at call time: no
// cudaMalloc/cudaFree/cudaMallocHost, no arena, no library routine that
// allocates.  Limits and rules:
//   * at most kNoAllocMaxRows (16,777,216) rows per call; larger inputs are
//     rejected with AHEAD_CAPACITY before anything is launched;
//   * the first call on a device does the set-up (it resolves the scratch
//     array's device address with cudaGetSymbolAddress, with that device
//     current, and caches it); creating a context on the device drops the
//     cached address, so a device reset between contexts is safe, but a
//     context must not be used across a reset of its device;
//   * every call copies its status to the host and waits for its stream, so
//     a call blocks and is never usable inside stream capture;
//   * the scratch is one buffer per device: calls must not overlap on a device
//     (one stream, or wait for the previous call to return -- each call
//     returns only after its stream has finished); overlapping calls race;
//   * what must start at zero: the status word and the counters (first 512
//     bytes) and the per-tile counts; each call clears them with
//     cudaMemsetAsync on the context's stream before its kernels run.
// Results are those of ahead_gpu_check_an (checkAN, encdecAN_scalar.tcc:
// 69-94): the positions row * AOID of the codes whose decoded value exceeds the
// largest unencoded value.  The reference has no such entry point.
#include <mutex>

#include "ops_common.cuh"

using namespace ahead;

namespace {

constexpr uint64_t kNoAllocMaxRows = 1ull << 24;
constexpr uint32_t kNoAllocTiles = (uint32_t)(kNoAllocMaxRows / kTileRows);
constexpr size_t align256(size_t b) { return (b + 255) & ~size_t(255); }
constexpr size_t kHeadBytes = 512;  // status word (8 B) + counters
constexpr size_t kWordsBytes = align256((size_t)kNoAllocTiles * kTileWords * 4);
constexpr size_t kCountsBytes = align256((size_t)kNoAllocTiles * 4);
constexpr size_t kOffsetsBytes = align256((size_t)kNoAllocTiles * 8);
constexpr size_t kGbaseBytes = align256(((kNoAllocTiles + kScanGroup - 1) / kScanGroup) * 8);
constexpr size_t kScratchBytes = kHeadBytes + kWordsBytes + kCountsBytes + kOffsetsBytes + kGbaseBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
void* g_scratch_ptr[kMaxDevices] = {};

}  // namespace

namespace ahead {
// Called by ahead_ctx_create: the next call on `dev` resolves the address again.
void noalloc_forget_device(int dev) {
    if (dev < 0 || dev >= kMaxDevices) return;
    std::lock_guard<std::mutex> lk(g_setup_mu);
    g_scratch_ptr[dev] = nullptr;
}
}  // namespace ahead

namespace {

// The device address of the scratch array on `device` (set-up on first use).
int scratch_for(ahead_ctx* ctx, unsigned char** out) {
    const int dev = ctx->device;
    if (dev < 0 || dev >= kMaxDevices) return fail(ctx, AHEAD_BAD_ARG, "check_an_noalloc: device index");
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_ptr[dev]) {
        int cur = 0;
        cudaError_t e = cudaGetDevice(&cur);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGetDevice");
        if (cur != dev && (e = cudaSetDevice(dev)) != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (cur != dev) cudaSetDevice(cur);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGetSymbolAddress (no-alloc scratch)");
        g_scratch_ptr[dev] = p;
    }
    *out = static_cast<unsigned char*>(g_scratch_ptr[dev]);
    return AHEAD_OK;
}

template <int W>
int check_noalloc(ahead_ctx* ctx, unsigned char* scratch, const ahead_bat* in, uint64_t ainv, uint64_t unenc_max,
                  uint64_t aoid, ahead_errvec* err) {
    typedef CheckOp<W> Op;
    const uint64_t n = in->count;
    cudaStream_t st = ctx->stream;
    uint32_t* status = reinterpret_cast<uint32_t*>(scratch);
    uint64_t* counters = reinterpret_cast<uint64_t*>(scratch + 8);
    cudaError_t e = cudaMemsetAsync(scratch, 0, kHeadBytes, st);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemsetAsync");
    if (n) {
        const uint32_t nt = compact_tiles(n);
        CompactBufs cb;
        cb.words = reinterpret_cast<uint32_t*>(scratch + kHeadBytes);
        cb.counts = reinterpret_cast<uint32_t*>(scratch + kHeadBytes + kWordsBytes);
        cb.offsets = reinterpret_cast<uint64_t*>(scratch + kHeadBytes + kWordsBytes + kCountsBytes);
        cb.gbase = reinterpret_cast<uint64_t*>(scratch + kHeadBytes + kWordsBytes + kCountsBytes + kOffsetsBytes);
        cb.totals = counters;
        cb.ntiles = nt;
        cb.nchan = Op::NCH;
        e = cudaMemsetAsync(cb.counts, 0, (size_t)nt * Op::NCH * 4, st);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemsetAsync");
        Op op;
        op.base = (const char*)in->tail.data;
        op.status = status;
        op.ainv = ainv & wmask(W);
        op.umax = unenc_max & wmask(W);
        op.aoid = aoid;
        op.err = edata(err);
        op.errcap = ecap(err);
        op.acc = nullptr;
        const uint32_t cap = (uint32_t)ctx->num_sms * 8;
        const uint32_t grid = nt < cap ? nt : cap;
        launch_classify(ctx, st, op, n, cb);
        tile_scan_kernel<<<scan_groups(nt), kScanGroup, 0, st>>>(cb);
        group_scan_kernel<<<1, 1024, 0, st>>>(cb);
        emit_kernel<Op><<<grid, kCThreads, 0, st>>>(op, n, cb);
        ctx->launches += 4;
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(ctx, e, "kernel launch");
    uint64_t h[2] = {0, 0};  // status word, error count (pageable host copy: no pinned buffer)
    e = cudaMemcpyAsync(h, scratch, sizeof h, cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemcpyAsync");
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamSynchronize");
    if ((uint32_t)h[0] & kDevStatusTimeout) return fail(ctx, AHEAD_TIMEOUT, "a bounded device wait gave up");
    if (err) err->count = n ? h[1] : 0;
    return AHEAD_OK;
}

}  // namespace

extern "C" int ahead_gpu_check_an_noalloc(ahead_ctx* ctx, const ahead_bat* in, uint64_t ainv, uint64_t unenc_max,
                                          uint64_t aoid, ahead_errvec* err) {
    if (!ctx || !in) return AHEAD_BAD_ARG;
    const int t = in->tail.type;
    if (!(in->head.type == AHEAD_VOID || in->head.type == AHEAD_OID) || !type_encoded(t))
        return fail(ctx, AHEAD_BAD_ARG, "check_an_noalloc: unencoded head and AN tail required");
    if (in->count > kNoAllocMaxRows)
        return fail(ctx, AHEAD_CAPACITY,
                    "check_an_noalloc: at most 16777216 rows per call (the fixed scratch); split the column");
    unsigned char* scratch = nullptr;
    int rc = scratch_for(ctx, &scratch);
    if (rc) return rc;
    ev_begin(err, 1);
    return by_width_enc(type_width(t), [&](auto tag) -> int {
        constexpr int W = decltype(tag)::value;
        return check_noalloc<W>(ctx, scratch, in, ainv, unenc_max, aoid, err);
    });
}
