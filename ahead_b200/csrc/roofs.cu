// roofs.cu -- the measured roofs of the indexed cube scan.
//
// The cube scan streams a fact row's columns (4 foreign keys, price and the
// packed join-index word: six 8-byte columns, and the 2-byte discount; 50 B per
// row) and adds one decoded product into a random cell of the signature cube
// in L2.  Both the stream and the adds pass through L2, so the scan has two
// roofs: the device's streaming read bandwidth and its rate of L2 reductions.
// ahead_gpu_cube_roofs measures them on synthetic columns of that layout, with
// the scan's access pattern (two adjacent rows per thread, 16-byte loads that
// skip L1, persistent blocks over 512-row tiles):
//   ms[0]  the stream alone (every loaded word folded into a register);
//   ms[1]  one 64-bit reduction per row into `cells` random cells, no stream;
//   ms[2]  the stream and one reduction per row into a cell hashed from the
//          row's loaded words (the reduction waits for the loads, as the
//          scan's does).
// A scan whose time per row is close to ms[2]'s is bound by the two together.
#include <algorithm>
#include <vector>

#include "ops_common.cuh"

using namespace ahead;

namespace {

struct RoofCols {
    const unsigned long long* f[6];  // foreign keys 0..3, price, index word
    const uint16_t* disc;
    unsigned long long* cube;
    uint32_t cells;
};

__device__ __forceinline__ ulonglong2 roof_ld(const unsigned long long* p) {
    ulonglong2 v;
    asm volatile("ld.global.nc.L1::no_allocate.v2.u64 {%0, %1}, [%2];" : "=l"(v.x), "=l"(v.y) : "l"(p));
    return v;
}

__device__ __forceinline__ uint32_t roof_hash(uint64_t x) {
    x ^= x >> 31;
    x *= 0x7fb5d329728ea185ull;
    x ^= x >> 27;
    return (uint32_t)(x >> 32);
}

template <bool STREAM, bool RED>
__global__ void __launch_bounds__(256) roof_kernel(RoofCols c, uint32_t n, unsigned long long* sink) {
    constexpr uint32_t kTile = 512;
    const uint32_t ntiles = n / kTile;
    unsigned long long acc = 0;
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const uint32_t r0 = t * kTile + 2u * threadIdx.x;
        uint64_t w[2] = {r0, r0 + 1ull};
        uint32_t d = 0;
        if (STREAM) {
#pragma unroll
            for (int p = 0; p < 6; ++p) {
                const ulonglong2 v = roof_ld(c.f[p] + r0);
                w[0] ^= v.x * (2 * p + 3);
                w[1] ^= v.y * (2 * p + 3);
            }
            d = __ldg(reinterpret_cast<const uint32_t*>(c.disc + r0));
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const uint64_t v = (w[j] & 0xffffffffull) * ((j ? d >> 16 : d & 0xffffu) | 1u);
            if (RED) atomicAdd(c.cube + roof_hash(w[j]) % c.cells, (unsigned long long)v);
            else acc += v;
        }
    }
    if (acc == 0x5eed5eed5eed5eedull) sink[0] = acc;  // keeps the stream's loads
}

__global__ void roof_fill(unsigned long long* p, uint64_t n, uint64_t seed) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        p[i] = (i + seed) * 0x9e3779b97f4a7c15ull;
}

}  // namespace

extern "C" int ahead_gpu_cube_roofs(ahead_ctx* ctx, uint64_t rows, uint32_t cells, float* ms) {
    if (!ctx || !ms || !cells) return AHEAD_BAD_ARG;
    rows = rows / 512 * 512;
    if (!rows || rows >= (1ull << 32)) return fail(ctx, AHEAD_BAD_ARG, "cube roofs: 512 <= rows < 2^32");
    cudaStream_t st = ctx->stream;
    RoofCols c{};
    std::vector<void*> bufs;
    auto take = [&](size_t bytes) -> void* {
        void* p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
        bufs.push_back(p);
        return p;
    };
    auto release = [&]() {
        cudaStreamSynchronize(st);
        for (void* p : bufs) cudaFree(p);
    };
    for (int p = 0; p < 6; ++p) {
        auto* col = static_cast<unsigned long long*>(take(rows * 8));
        if (!col) {
            release();
            return fail(ctx, AHEAD_NO_MEMORY, "cube roofs: columns");
        }
        roof_fill<<<ctx->num_sms * 8, 256, 0, st>>>(col, rows, 1000003ull * (p + 1));
        c.f[p] = col;
    }
    auto* disc = static_cast<uint16_t*>(take(rows * 2));
    c.cube = static_cast<unsigned long long*>(take((size_t)cells * 8));
    auto* sink = static_cast<unsigned long long*>(take(8));
    if (!disc || !c.cube || !sink) {
        release();
        return fail(ctx, AHEAD_NO_MEMORY, "cube roofs: buffers");
    }
    cudaMemsetAsync(disc, 7, rows * 2, st);
    cudaMemsetAsync(c.cube, 0, (size_t)cells * 8, st);
    c.disc = disc;
    c.cells = cells;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int grid = ctx->num_sms * 4;
    auto time = [&](auto launch) {
        for (int i = 0; i < 2; ++i) launch();
        float t[5];
        for (float& x : t) {
            cudaEventRecord(e0, st);
            launch();
            cudaEventRecord(e1, st);
            cudaEventSynchronize(e1);
            cudaEventElapsedTime(&x, e0, e1);
        }
        std::sort(t, t + 5);
        return t[2];
    };
    const uint32_t n = (uint32_t)rows;
    ms[0] = time([&] { roof_kernel<true, false><<<grid, 256, 0, st>>>(c, n, sink); });
    ms[1] = time([&] { roof_kernel<false, true><<<grid, 256, 0, st>>>(c, n, sink); });
    ms[2] = time([&] { roof_kernel<true, true><<<grid, 256, 0, st>>>(c, n, sink); });
    const cudaError_t ce = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    release();
    return ce == cudaSuccess ? AHEAD_OK : fail(ctx, AHEAD_CUDA_ERROR, "cube roofs: launch");
}
