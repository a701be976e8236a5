// compact.cuh -- stable multi-stream compaction in three streaming passes.
//
// Every AN operator that filters rows (selectAN, checkAndDecodeAN, the
// positional matchjoinAN / fetchjoinAN ...) produces up to five output
// streams in scan order: the kept rows (stream 0, dense) and up to four
// error-position vectors (rare).  The reference builds them with push_back in
// one sequential loop (e.g. lib/column_operators/AN/selectAN_scalar.tcc:84-92).
//
//   pass 1  classify: each 4096-row tile is read once; a warp walks its
//           512 rows one row per lane per step, the per-step ballot of
//           stream 0 is stored as a 32-row bitmap word, and every stream is
//           counted per tile.  No inter-block waiting of any kind.
//   pass 2  two small scans turn the per-tile counts into offsets.
//   pass 3  emit: stream 0 is written from the bitmap words (ranks are
//           popcounts, consecutive lanes write consecutive addresses), or,
//           for a tile whose every row is in it, as a plain transform; the
//           sparse streams are recomputed only for tiles whose count is > 0.
//
// Traffic beyond the input and the outputs: one bit per row written and read
// back, plus re-reading the few tiles that hold errors.
#pragma once

#include <type_traits>

#include "common.cuh"

namespace ahead {

constexpr int kCThreads = 256;  // threads per tile block
constexpr int kCWarps = kCThreads / 32;
constexpr int kCSteps = 16;  // rows per lane per tile
constexpr int kTileRows = kCThreads * kCSteps;  // 4096
constexpr int kTileWords = kTileRows / 32;      // 128 bitmap words per tile
constexpr int kWarpWords = kTileWords / kCWarps;  // 16

template <int W>
AHEAD_DEV uint64_t gmem_ld(const char* p, uint64_t i) {
    if (W == 1) return __ldg((const uint8_t*)p + i);
    if (W == 2) return __ldg((const uint16_t*)p + i);
    if (W == 4) return __ldg((const uint32_t*)p + i);
    return __ldg((const unsigned long long*)p + i);
}

// ------------------------------------------------------------ mbarrier / TMA
AHEAD_DEV uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
AHEAD_DEV void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
AHEAD_DEV void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
AHEAD_DEV void mbar_arrive_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}
AHEAD_DEV void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
AHEAD_DEV bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, "
        "p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait (try_wait suspends for a hardware time slice per call); false
// when it gave up.
AHEAD_DEV bool mbar_wait(uint64_t* bar, uint32_t parity) {
    for (uint32_t i = 0; i < (1u << 22); ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// Bulk copy global -> shared (16-byte aligned addresses, size multiple of 16),
// completion signalled on `bar` as transaction bytes.
AHEAD_DEV void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}
template <int W>
AHEAD_DEV uint64_t smem_ld(const char* p, int i) {
    if (W == 1) return ((const uint8_t*)p)[i];
    if (W == 2) return ((const uint16_t*)p)[i];
    if (W == 4) return ((const uint32_t*)p)[i];
    return ((const unsigned long long*)p)[i];
}

// Stage ring of the TMA-fed classify pass: 64 KB per block.
template <int W>
struct RingCfg {
    static constexpr int TILE_BYTES = kTileRows * W;
    static constexpr int RAW = (64 * 1024) / TILE_BYTES;
    static constexpr int STAGES = RAW < 2 ? 2 : (RAW > 8 ? 8 : RAW);
    static constexpr int SMEM = STAGES * TILE_BYTES;
};

// Scratch of one compaction: bitmap words, per-tile counts and offsets.
struct CompactBufs {
    uint32_t* words;    // [ntiles * 128] stream-0 bitmap
    uint32_t* counts;   // [ntiles][NCH], zeroed before pass 1
    uint64_t* offsets;  // [ntiles][NCH] exclusive offset within the tile's group
    uint64_t* gbase;    // [ngroups][NCH] exclusive offset of each group of 1024 tiles
    uint64_t* totals;   // [NCH]
    uint32_t ntiles;
    uint32_t nchan;
};

constexpr int kScanGroup = 1024;  // tiles per first-level scan block

AHEAD_HD uint32_t scan_groups(uint32_t ntiles) { return (ntiles + kScanGroup - 1) / kScanGroup; }

inline size_t compact_bytes(uint32_t ntiles, uint32_t nchan) {
    return (size_t)ntiles * kTileWords * 4 + (size_t)ntiles * nchan * 12 + (size_t)scan_groups(ntiles) * nchan * 8 +
           2048;
}

// `Op` supplies
//   static constexpr int W;     width in bytes of the driving column `base`
//   static constexpr int NCH;   number of output streams (0 = kept rows)
//   static constexpr bool ACC;  sum the eval accumulator into *op.acc
//   static constexpr bool EMIT_V; stream 0 emission needs the driving value
//   static constexpr int NOUT;  output columns written per stream-0 row
//   const char* base;
//   uint32_t* status;           device status word (timeouts)
//   uint32_t eval(uint64_t v, uint64_t row, uint64_t& acc) const;  bit c = stream c
//   uint64_t out0(int k, uint64_t v, uint64_t row) const;  k-th output of a kept row
//   void put0(int k, uint64_t pos, uint64_t val) const;    store it at pos
//   void emit(int c, uint64_t pos, uint64_t v, uint64_t row) const;  streams c >= 1
//
// Row layout of a tile: warp w owns rows [512w, 512w+512); in step s each lane
// holds one 16-byte vector of VEC = 16/W consecutive rows, row =
// 512w + s*32*VEC + lane*VEC + k.  Stream 0's bitmap is kept in row order: bit
// b of the warp's word j is row 512w + 32j + b.
template <int W>
struct Vec {
    static constexpr int VEC = 16 / W;
    static constexpr int STEPS = 512 / (32 * VEC);  // steps per warp per tile
};

template <int W>
AHEAD_DEV void unpack16(const uint4 q, uint64_t (&v)[16 / W]) {
    const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int k = 0; k < 16 / W; ++k) {
        if (W == 8) v[k] = (uint64_t)w[2 * k] | ((uint64_t)w[2 * k + 1] << 32);
        else if (W == 4) v[k] = w[k];
        else if (W == 2) v[k] = (w[k / 2] >> (16 * (k & 1))) & 0xffffu;
        else v[k] = (w[k / 4] >> (8 * (k & 3))) & 0xffu;
    }
}

// Pass 1: a persistent grid walks the tiles (tile = block + k * grid).  With
// BULK, one thread streams the tiles into a ring of shared-memory stages with
// cp.async.bulk several tiles ahead, so the bytes in flight cost no
// registers; without it (unaligned column) lanes load rows directly.  Per-warp
// counts go to the tile's counters with one atomic each.
template <class Op, bool BULK>
__global__ void __launch_bounds__(kCThreads) classify_kernel(Op op, uint64_t n, CompactBufs cb) {
    constexpr int W = Op::W;
    constexpr int NCH = Op::NCH;
    constexpr int VEC = Vec<W>::VEC;
    constexpr int STEPS = Vec<W>::STEPS;
    typedef RingCfg<W> Ring;
    extern __shared__ __align__(128) char s_ring[];
    __shared__ __align__(8) uint64_t s_bar[8];
    __shared__ int s_abort;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t total_bytes = n * W;
    const uint32_t nmine = blockIdx.x < cb.ntiles ? (cb.ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;

    auto issue = [&](uint32_t k) {  // start the copy of my k-th tile
        const int st = k % Ring::STAGES;
        const uint64_t off = (uint64_t)(blockIdx.x + k * gridDim.x) * Ring::TILE_BYTES;
        const uint64_t rem = total_bytes - off;
        const uint32_t bytes = (uint32_t)((rem < (uint64_t)Ring::TILE_BYTES ? rem : Ring::TILE_BYTES) & ~15ull);
        if (bytes) {
            mbar_arrive_tx(&s_bar[st], bytes);
            bulk_g2s(s_ring + st * Ring::TILE_BYTES, op.base + off, bytes, &s_bar[st]);
        } else {
            mbar_arrive(&s_bar[st]);
        }
    };
    if (BULK) {
        if (threadIdx.x == 0) {
            s_abort = 0;
            for (int i = 0; i < Ring::STAGES; ++i) mbar_init(&s_bar[i], 1);
            mbar_fence_init();
            for (uint32_t k = 0; k < nmine && k < (uint32_t)Ring::STAGES; ++k) issue(k);
        }
        __syncthreads();
    }
    uint64_t acc = 0;
    for (uint32_t k = 0; k < nmine; ++k) {
        const uint32_t tile = blockIdx.x + k * gridDim.x;
        const uint64_t trow0 = (uint64_t)tile * kTileRows;
        const char* tb = s_ring + (k % Ring::STAGES) * Ring::TILE_BYTES;
        uint32_t in_smem = 0;  // rows of this tile that the bulk copy brought in
        if (BULK) {
            if (!mbar_wait(&s_bar[k % Ring::STAGES], (k / Ring::STAGES) & 1)) {
                atomicOr(op.status, kDevStatusTimeout);
                s_abort = 1;
            }
            const uint64_t rem = total_bytes - trow0 * W;
            in_smem = (uint32_t)(((rem < (uint64_t)Ring::TILE_BYTES ? rem : Ring::TILE_BYTES) & ~15ull) / W);
        }
        uint32_t sparse[NCH];  // this lane's rows per stream
#pragma unroll
        for (int c = 0; c < NCH; ++c) sparse[c] = 0;
        // Word j of the warp covers rows [32j, 32j+32) of its 512-row segment:
        // in step s the lanes of group g = lane / (32/VEC) contribute word
        // s*VEC + g, each its VEC bits at bit position VEC * (lane % (32/VEC)).
        constexpr int LPW = 32 / VEC;  // lanes per word
        uint32_t mine = 0;  // lane (s*VEC + g) keeps word (s, g)
        auto step = [&](auto full_tag) {
            constexpr bool FULL = decltype(full_tag)::value;
#pragma unroll
            for (int s = 0; s < STEPS; ++s) {
                const uint32_t lr = warp * 512 + s * 32 * VEC + lane * VEC;
                const uint64_t row0 = trow0 + lr;
                uint64_t v[VEC];
                if (BULK && (FULL || lr + VEC <= in_smem)) {
                    unpack16<W>(*(const uint4*)(tb + (size_t)lr * W), v);
                } else if (!BULK && (FULL || row0 + VEC <= n) && (((uintptr_t)op.base + row0 * W) & 15) == 0) {
                    unpack16<W>(__ldg((const uint4*)(op.base + row0 * W)), v);
                } else {
#pragma unroll
                    for (int q = 0; q < VEC; ++q) v[q] = (FULL || row0 + q < n) ? gmem_ld<W>(op.base, row0 + q) : 0;
                }
                uint32_t m0 = 0;
#pragma unroll
                for (int q = 0; q < VEC; ++q) {
                    const uint32_t bits = (FULL || row0 + q < n) ? op.eval(v[q], row0 + q, acc) : 0u;
                    m0 |= (bits & 1u) << q;
#pragma unroll
                    for (int c = 1; c < NCH; ++c) sparse[c] += (bits >> c) & 1u;
                }
                sparse[0] += __popc(m0);
                uint32_t word = m0 << (VEC * (lane % LPW));
#pragma unroll
                for (int d = 1; d < LPW; d <<= 1) word |= __shfl_xor_sync(kFull, word, d);
                // group g's word sits in all its lanes; lane s*VEC+g takes it
                const uint32_t g = (uint32_t)(lane - s * VEC);
                const uint32_t wv = __shfl_sync(kFull, word, (g < (uint32_t)VEC ? g : 0) * LPW);
                if (g < (uint32_t)VEC) mine = wv;
            }
        };
        const bool full = (BULK ? in_smem == (uint32_t)kTileRows : trow0 + kTileRows <= n);
        if (full) step(std::true_type());
        else step(std::false_type());
        if (lane < kWarpWords) cb.words[(size_t)tile * kTileWords + warp * kWarpWords + lane] = mine;
        const uint32_t c0 = __reduce_add_sync(kFull, sparse[0]);
        uint32_t mycnt = (lane == 0) ? c0 : 0;
#pragma unroll
        for (int c = 1; c < NCH; ++c) {
            const uint32_t t = __reduce_add_sync(kFull, sparse[c]);
            if (lane == c) mycnt = t;
        }
        if (lane < NCH && mycnt) atomicAdd(&cb.counts[(size_t)tile * NCH + lane], mycnt);
        if (BULK) {
            __syncthreads();  // every warp is done with this stage
            if (s_abort) {
                // Wait (bounded) for the copies still in flight before leaving.
                if (threadIdx.x == 0)
                    for (uint32_t q = k + 1; q < nmine && q < k + Ring::STAGES; ++q)
                        mbar_wait(&s_bar[q % Ring::STAGES], (q / Ring::STAGES) & 1);
                break;
            }
            if (threadIdx.x == 0 && k + Ring::STAGES < nmine) issue(k + Ring::STAGES);
        }
    }
    if constexpr (Op::ACC) {
        acc = warp_sum64(acc);
        if (lane == 0 && acc) atomicAdd((unsigned long long*)op.acc, (unsigned long long)acc);
    }
}

// Pass 2a: each block scans the counts of 1024 consecutive tiles per channel
// (exclusive, within the group) and writes the group totals to gbase.
static __global__ void __launch_bounds__(kScanGroup) tile_scan_kernel(CompactBufs cb) {
    __shared__ uint64_t s_part[32];
    const uint32_t nch = cb.nchan;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t t = blockIdx.x * kScanGroup + threadIdx.x;
    for (uint32_t c = 0; c < nch; ++c) {
        const uint64_t x = t < cb.ntiles ? cb.counts[(size_t)t * nch + c] : 0;
        const uint64_t incl = warp_incl_scan64(x);
        if (lane == 31) s_part[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            const uint64_t p = s_part[lane];
            const uint64_t pi = warp_incl_scan64(p);
            s_part[lane] = pi - p;
            if (lane == 31) cb.gbase[(size_t)blockIdx.x * nch + c] = pi;
        }
        __syncthreads();
        if (t < cb.ntiles) cb.offsets[(size_t)t * nch + c] = s_part[warp] + incl - x;
        __syncthreads();
    }
}

// Pass 2b: one block turns the group totals into exclusive group offsets.
static __global__ void __launch_bounds__(1024) group_scan_kernel(CompactBufs cb) {
    __shared__ uint64_t s_part[32];
    const uint32_t ng = scan_groups(cb.ntiles), nch = cb.nchan;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t c = 0; c < nch; ++c) {
        uint64_t carry = 0;
        for (uint32_t g0 = 0; g0 < ng; g0 += 1024) {
            const uint32_t g = g0 + threadIdx.x;
            const uint64_t x = g < ng ? cb.gbase[(size_t)g * nch + c] : 0;
            const uint64_t incl = warp_incl_scan64(x);
            if (lane == 31) s_part[warp] = incl;
            __syncthreads();
            if (warp == 0) {
                const uint64_t p = s_part[lane];
                s_part[lane] = warp_incl_scan64(p) - p;
            }
            __syncthreads();
            const uint64_t ex = carry + s_part[warp] + incl - x;
            __syncthreads();
            if (g < ng) cb.gbase[(size_t)g * nch + c] = ex;
            if (threadIdx.x == blockDim.x - 1) s_part[0] = ex + x;
            __syncthreads();
            carry = s_part[0];
            __syncthreads();
        }
        if (threadIdx.x == 0) cb.totals[c] = carry;
    }
}

// Pass 3: a persistent grid writes the streams.  Stream 0 comes from the
// bitmap; each warp derives its offset inside the tile from the popcounts of
// the preceding warps' words, ranks the rows of a step with one warp scan of
// the lanes' counts, stages the outputs in shared memory and writes them with
// full-width stores.  Sparse streams are recomputed only for tiles that hold
// any (block-uniform branch).
template <class Op>
__global__ void __launch_bounds__(kCThreads, 4) emit_kernel(Op op, uint64_t n, CompactBufs cb) {
    constexpr int W = Op::W;
    constexpr int NCH = Op::NCH;
    constexpr int VEC = Vec<W>::VEC;
    constexpr int STEPS = Vec<W>::STEPS;
    __shared__ uint32_t s_sc[NCH][kCWarps];
    __shared__ uint16_t s_rows[kCWarps][512];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t tile = blockIdx.x; tile < cb.ntiles; tile += gridDim.x) {
        const uint32_t* counts = cb.counts + (size_t)tile * NCH;
        const uint64_t* offs = cb.offsets + (size_t)tile * NCH;
        const uint64_t* gb = cb.gbase + (size_t)(tile / kScanGroup) * NCH;
        const uint64_t trow0 = (uint64_t)tile * kTileRows;
        // the tile's header and bitmap words in one round trip
        const uint32_t* tw = cb.words + (size_t)tile * kTileWords;
        const uint32_t cnt0 = counts[0];
        const uint64_t base0 = offs[0] + gb[0];
        uint32_t tws[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) tws[q] = tw[lane + 32 * q];
        const uint32_t hw = tw[warp * kWarpWords + (lane >> 1)];
        const uint32_t trows = trow0 + kTileRows <= n ? (uint32_t)kTileRows : (uint32_t)(n - trow0);
        if (cnt0 == trows) {
            // every row of the tile is in stream 0: output i is row i, a plain
            // coalesced transform with all of a thread's loads in flight together
            uint64_t v[kCSteps];
#pragma unroll
            for (int k = 0; k < kCSteps; ++k) {
                const uint32_t i = threadIdx.x + k * kCThreads;
                v[k] = (Op::EMIT_V && i < trows) ? gmem_ld<W>(op.base, trow0 + i) : 0;
            }
#pragma unroll
            for (int k = 0; k < kCSteps; ++k) {
                const uint32_t i = threadIdx.x + k * kCThreads;
                if (i < trows)
#pragma unroll
                    for (int o = 0; o < Op::NOUT; ++o) op.put0(o, base0 + i, op.out0(o, v[k], trow0 + i));
            }
        } else if (cnt0) {
            uint32_t before = 0;  // kept rows of the preceding warps
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int wi = lane + 32 * q;
                if (wi < warp * kWarpWords) before += __popc(tws[q]);
            }
            before = __reduce_add_sync(kFull, before);
            // Lane l owns rows [16l, 16l+16) of the warp's segment: half of word l/2.
            uint32_t h = (hw >> (16 * (lane & 1))) & 0xffffu;
            const uint32_t c = __popc(h);
            const uint32_t incl = warp_incl_scan(c);
            const uint32_t tot = __shfl_sync(kFull, incl, 31);
            uint32_t r = incl - c;
            while (h) {  // stage the kept rows' segment offsets in row order
                const uint32_t bit = __ffs(h) - 1;
                h &= h - 1;
                s_rows[warp][r++] = (uint16_t)(16 * lane + bit);
            }
            __syncwarp();
            const uint64_t base = base0 + before;
            const uint64_t srow = trow0 + (uint64_t)warp * 512;
            for (uint32_t i = lane; i < tot; i += 32) {
                const uint64_t row = srow + s_rows[warp][i];
                const uint64_t v = Op::EMIT_V ? gmem_ld<W>(op.base, row) : 0;
#pragma unroll
                for (int o = 0; o < Op::NOUT; ++o) op.put0(o, base + i, op.out0(o, v, row));
            }
            __syncwarp();
        }
        if constexpr (NCH > 1) {
            bool any = false;
#pragma unroll
            for (int c = 1; c < NCH; ++c) any |= counts[c] != 0;
            if (any) {
                // Recompute the tile; bits[s] holds, per slot q, the stream bits.
                uint32_t bits[STEPS][VEC];
                uint32_t wc[NCH];
#pragma unroll
                for (int c = 0; c < NCH; ++c) wc[c] = 0;
                uint64_t dummy = 0;
#pragma unroll
                for (int s = 0; s < STEPS; ++s) {
                    const uint64_t row0 = trow0 + warp * 512 + s * 32 * VEC + lane * VEC;
#pragma unroll
                    for (int q = 0; q < VEC; ++q) {
                        bits[s][q] = row0 + q < n ? op.eval(gmem_ld<W>(op.base, row0 + q), row0 + q, dummy) : 0u;
#pragma unroll
                        for (int c = 1; c < NCH; ++c) wc[c] += (bits[s][q] >> c) & 1u;
                    }
                }
#pragma unroll
                for (int c = 1; c < NCH; ++c) wc[c] = __reduce_add_sync(kFull, wc[c]);
                __syncthreads();
                if (lane == 0)
#pragma unroll
                    for (int c = 1; c < NCH; ++c) s_sc[c][warp] = wc[c];
                __syncthreads();
#pragma unroll
                for (int c = 1; c < NCH; ++c) {
                    if (!counts[c]) continue;
                    uint64_t pos = offs[c] + gb[c];
                    for (int k = 0; k < warp; ++k) pos += s_sc[c][k];
#pragma unroll
                    for (int s = 0; s < STEPS; ++s) {
                        uint32_t cl = 0;
#pragma unroll
                        for (int q = 0; q < VEC; ++q) cl += (bits[s][q] >> c) & 1u;
                        const uint32_t incl = warp_incl_scan(cl);
                        uint64_t p = pos + incl - cl;
                        const uint64_t row0 = trow0 + warp * 512 + s * 32 * VEC + lane * VEC;
#pragma unroll
                        for (int q = 0; q < VEC; ++q)
                            if ((bits[s][q] >> c) & 1u) op.emit(c, p++, gmem_ld<W>(op.base, row0 + q), row0 + q);
                        pos += __shfl_sync(kFull, incl, 31);
                    }
                }
            }
        }
    }
}

}  // namespace ahead
