// common.cuh -- device-side building blocks shared by all AN operator kernels.
//
// Value model: every column element is carried in a uint64_t and reduced
// modulo 2^(8*width) where the reference's C++ types wrap, so each kernel is
// bit-identical to the reference's scalar operators (include/util/
// resilience.hpp:36-276 for the types, lib/util/resilience.cpp:47-71 for the
// largest valid decoded values).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/ahead_types.h"

#define AHEAD_DEV __device__ __forceinline__
#define AHEAD_HD __host__ __device__ __forceinline__

namespace ahead {

constexpr int kWarp = 32;
constexpr unsigned kFull = 0xffffffffu;

// ----------------------------------------------------------------- types
AHEAD_HD int type_width(int t) {  // storage width in bytes
    switch (t) {
        case AHEAD_TINYINT: return 1;
        case AHEAD_SHORTINT: case AHEAD_RESTINY: return 2;
        case AHEAD_VOID: case AHEAD_INT: case AHEAD_OID: case AHEAD_RESSHORT: return 4;
        default: return 8;
    }
}
AHEAD_HD int type_base_width(int t) {  // width of TypeMap<T>::v2_base_t::type_t
    switch (t) {
        case AHEAD_TINYINT: case AHEAD_RESTINY: return 1;
        case AHEAD_SHORTINT: case AHEAD_RESSHORT: return 2;
        case AHEAD_BIGINT: case AHEAD_RESBIGINT: return 8;
        default: return 4;
    }
}
AHEAD_HD bool type_encoded(int t) { return t >= AHEAD_RESTINY && t <= AHEAD_RESOID; }
AHEAD_HD int type_encoded_of(int t) {  // TypeMap<T>::v2_encoded_t
    switch (t) {
        case AHEAD_TINYINT: case AHEAD_RESTINY: return AHEAD_RESTINY;
        case AHEAD_SHORTINT: case AHEAD_RESSHORT: return AHEAD_RESSHORT;
        case AHEAD_INT: case AHEAD_RESINT: return AHEAD_RESINT;
        case AHEAD_BIGINT: case AHEAD_RESBIGINT: return AHEAD_RESBIGINT;
        default: return AHEAD_RESOID;
    }
}
AHEAD_HD int type_select_of(int t) { return t == AHEAD_VOID ? AHEAD_OID : t; }
AHEAD_HD int type_unenc_of(int t) {
    switch (t) {
        case AHEAD_RESTINY: return AHEAD_TINYINT;
        case AHEAD_RESSHORT: return AHEAD_SHORTINT;
        case AHEAD_RESINT: return AHEAD_INT;
        case AHEAD_RESBIGINT: return AHEAD_BIGINT;
        case AHEAD_RESOID: return AHEAD_OID;
        default: return t;
    }
}
AHEAD_HD int type_larger_of(int t) {  // v2_larger_t
    switch (t) {
        case AHEAD_TINYINT: return AHEAD_SHORTINT;
        case AHEAD_SHORTINT: return AHEAD_INT;
        case AHEAD_RESTINY: return AHEAD_RESSHORT;
        case AHEAD_RESSHORT: return AHEAD_RESINT;
        case AHEAD_RESINT: case AHEAD_RESBIGINT: case AHEAD_RESOID: return AHEAD_RESBIGINT;
        default: return AHEAD_BIGINT;
    }
}
AHEAD_HD uint64_t wmask(int bytes) { return bytes >= 8 ? ~0ull : ((1ull << (8 * bytes)) - 1); }
AHEAD_HD uint64_t mulw(uint64_t a, uint64_t b, int bytes) { return (a * b) & wmask(bytes); }

// Largest resoid A and its inverse (resilience.hpp:99-105) and UNENC_MAX_U of
// the 64-bit code types (lib/util/resilience.cpp:59-71).
constexpr uint64_t kResoidAMax = 65117ull;
constexpr uint64_t kResoidAInvMax = 0x3E36D3BC8D9BC5F5ull;
constexpr uint64_t kRes56Max = 0x00FFFFFFFFFFFFFFull;

// A device view of one column: everything pre-masked to the storage width.
struct DCol {
    const void* data;
    uint64_t seqbase;
    uint64_t ainv;  // A^-1 (masked), 0 when the column is not encoded
    uint64_t umax;  // largest valid decoded value (masked)
    int type;
    int width;
    int enc;
    int pad;
};

AHEAD_DEV uint64_t load_at(const DCol& c, uint64_t i) {
    if (c.type == AHEAD_VOID) return (uint32_t)(c.seqbase + i);
    switch (c.width) {
        case 1: return __ldg((const uint8_t*)c.data + i);
        case 2: return __ldg((const uint16_t*)c.data + i);
        case 4: return __ldg((const uint32_t*)c.data + i);
        default: return __ldg((const unsigned long long*)c.data + i);
    }
}
AHEAD_DEV void store_at(void* p, int width, uint64_t i, uint64_t v) {
    switch (width) {
        case 1: ((uint8_t*)p)[i] = (uint8_t)v; break;
        case 2: ((uint16_t*)p)[i] = (uint16_t)v; break;
        case 4: ((uint32_t*)p)[i] = (uint32_t)v; break;
        default: ((uint64_t*)p)[i] = v; break;
    }
}
// ANhelper<V>::mulIfEncoded(x, f): (storage)(x*f) when encoded, else x.
AHEAD_DEV uint64_t dec_if(const DCol& c, uint64_t x, uint64_t f) { return c.enc ? mulw(x, f, c.width) : x; }

// ----------------------------------------------------------------- predicates
AHEAD_DEV bool cmp_op(int op, uint64_t a, uint64_t b) {
    switch (op) {
        case AHEAD_CMP_LT: return a < b;
        case AHEAD_CMP_LE: return a <= b;
        case AHEAD_CMP_EQ: return a == b;
        case AHEAD_CMP_NE: return a != b;
        case AHEAD_CMP_GE: return a >= b;
        case AHEAD_CMP_GT: return a > b;
        default: return false;
    }
}
struct Pred {
    uint64_t th1, th2;
    int op1, op2, comb, pad;
    AHEAD_DEV bool operator()(uint64_t v) const {
        bool a = cmp_op(op1, v, th1);
        if (op2 == AHEAD_CMP_NONE) return a;
        bool b = cmp_op(op2, v, th2);
        return comb == AHEAD_OR ? (a || b) : (a && b);
    }
};

// Branch-free predicate: every comparison of a w-bit unsigned value with a
// threshold is an interval test ((v - lo) mod 2^w <= span), possibly negated;
// two predicates combined with `and` over intervals collapse into one.
struct RangePred {
    uint64_t lo1, span1, lo2, span2, mask;
    int neg1, neg2, two, orc;
    AHEAD_HD bool operator()(uint64_t v) const {
        const bool a = (((v - lo1) & mask) <= span1) != (neg1 != 0);
        if (!two) return a;
        const bool b = (((v - lo2) & mask) <= span2) != (neg2 != 0);
        return orc ? (a || b) : (a && b);
    }
    static AHEAD_HD void interval(int op, uint64_t th, uint64_t mask, uint64_t& lo, uint64_t& span, int& neg) {
        neg = 0;
        th &= mask;
        switch (op) {
            case AHEAD_CMP_LT:
                if (th == 0) { lo = 0; span = mask; neg = 1; } else { lo = 0; span = th - 1; }
                break;
            case AHEAD_CMP_LE: lo = 0; span = th; break;
            case AHEAD_CMP_EQ: lo = th; span = 0; break;
            case AHEAD_CMP_NE: lo = th; span = 0; neg = 1; break;
            case AHEAD_CMP_GE: lo = th; span = mask - th; break;
            default:  // GT
                if (th == mask) { lo = 0; span = mask; neg = 1; } else { lo = th + 1; span = mask - th - 1; }
                break;
        }
    }
    static AHEAD_HD RangePred make(int op1, uint64_t th1, int op2, uint64_t th2, int comb, uint64_t mask) {
        RangePred p;
        p.mask = mask;
        interval(op1, th1, mask, p.lo1, p.span1, p.neg1);
        p.two = op2 != AHEAD_CMP_NONE;
        p.orc = comb == AHEAD_OR;
        p.lo2 = 0;
        p.span2 = mask;
        p.neg2 = 0;
        if (p.two) interval(op2, th2, mask, p.lo2, p.span2, p.neg2);
        if (p.two && !p.orc && !p.neg1 && !p.neg2) {  // intersect two plain intervals
            const uint64_t hi1 = p.lo1 + p.span1, hi2 = p.lo2 + p.span2;
            const uint64_t lo = p.lo1 > p.lo2 ? p.lo1 : p.lo2, hi = hi1 < hi2 ? hi1 : hi2;
            if (lo > hi) { p.lo1 = 0; p.span1 = mask; p.neg1 = 1; }
            else { p.lo1 = lo; p.span1 = hi - lo; }
            p.two = 0;
        }
        return p;
    }
};

// ----------------------------------------------------------------- memory order
AHEAD_DEV uint64_t ld_acquire(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
AHEAD_DEV void st_release(uint64_t* p, uint64_t v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
AHEAD_DEV uint32_t ld_acquire32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// ----------------------------------------------------------------- warp scans
AHEAD_DEV uint32_t warp_incl_scan(uint32_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint32_t o = __shfl_up_sync(kFull, v, d);
        if (lane >= d) v += o;
    }
    return v;
}
AHEAD_DEV uint64_t warp_incl_scan64(uint64_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint64_t o = __shfl_up_sync(kFull, v, d);
        if (lane >= d) v += o;
    }
    return v;
}
AHEAD_DEV uint64_t warp_sum64(uint64_t v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(kFull, v, d);
    return v;
}

// Device-side status word bits (written with atomicOr, read by the host).
enum : uint32_t {
    kDevStatusTimeout = 1u,      // a bounded spin gave up
    kDevStatusCapacity = 2u,     // an output did not fit
    kDevStatusDupKey = 4u,       // a build side had duplicate keys (fused paths only)
    kDevStatusBadInput = 8u,     // an input outside the supported domain
};

}  // namespace ahead
