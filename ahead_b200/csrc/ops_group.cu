// ops_group.cu -- groupbyAN (unary and binary), aggregate_sum_groupedAN, and
// their unencoded twins (groupby, aggregate_sum_grouped, aggregate_sum,
// arithmetic).
//
// Group ids are assigned in order of first occurrence, as the reference's
// dictionary loop does (lib/column_operators/AN/groupbyAN.tcc:70-91,
// 127-160).  On the GPU: every row inserts its key into the hash table of
// hash.cuh and atomicMin's its row index into the slot's first-row word; a
// stable compaction of the rows that are their key's first row ranks the
// groups by first occurrence; a last pass writes every row's encoded group id.
#include "hash.cuh"
#include "ops_common.cuh"

using namespace ahead;

namespace {

struct GbKey {
    DCol tail, grp;
    uint64_t keymask, lmask, ngroups, gainv;
    int binary;
};

AHEAD_DEV uint64_t gb_key(const GbKey& k, uint64_t row) {
    const uint64_t t = dec_if(k.tail, load_at(k.tail, row), k.tail.ainv);
    if (!k.binary) return t & k.keymask;  // unary: the unencoded base type
    // binary: hash(t) * numGroups + g in the larger tail type (groupbyAN.tcc:144)
    const uint64_t g = load_at(k.grp, row) * k.gainv;
    return ((t & k.lmask) * (k.ngroups & k.lmask) + (g & k.lmask)) & k.lmask;
}

__global__ void gb_insert_kernel(HashTab h, GbKey k, uint64_t n, uint32_t* slot_of, uint32_t* first) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t s = ht_insert(h, gb_key(k, i));
        slot_of[i] = s;
        atomicMin(&first[s], (uint32_t)i);
    }
}

// Rows that are the first row of their group, in row order; the rank of such
// a row is its group id.  The driving column is the row's slot.
struct FirstOp {
    static constexpr int W = 4;
    static constexpr int NCH = 1;
    static constexpr bool ACC = false;
    static constexpr bool EMIT_V = false;
    static constexpr int NOUT = 1;
    const char* base;
    uint32_t* status;
    const uint32_t* first;
    uint32_t* gid_of_slot;
    DCol head;
    uint64_t aoid, cap;
    uint64_t* firsts;
    uint64_t* acc;
    int decode_head;
    AHEAD_DEV uint32_t eval(uint64_t v, uint64_t row, uint64_t&) const { return first[v] == (uint32_t)row ? 1u : 0u; }
    AHEAD_DEV uint64_t out0(int, uint64_t, uint64_t row) const { return row; }
    AHEAD_DEV void put0(int, uint64_t pos, uint64_t row) const {
        const uint32_t s = ((const uint32_t*)base)[row];
        gid_of_slot[s] = (uint32_t)pos;
        if (pos < cap) {
            const uint64_t h = load_at(head, row);
            // unary: raw head (groupbyAN.tcc:87); binary: decoded head (:153)
            firsts[pos] = (decode_head ? dec_if(head, h, head.ainv) : h) * aoid;
        }
    }
    AHEAD_DEV void emit(int, uint64_t, uint64_t, uint64_t) const {}
};

// Encoded group id of every row.  The binary group-by's dictionary stores the
// encoded id in an oid_t (groupbyAN.tcc:150): the first row of a group gets
// all 64 bits, later rows the low 32.
__global__ void gb_assign_kernel(const uint32_t* slot_of, const uint32_t* first, const uint32_t* gid_of_slot,
                                 uint64_t n, uint64_t aoid, int binary, uint64_t* gids, uint64_t cap) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n && i < cap;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t s = slot_of[i];
        const uint64_t v = (uint64_t)gid_of_slot[s] * aoid;
        gids[i] = (binary && first[s] != (uint32_t)i) ? (uint64_t)(uint32_t)v : v;
    }
}

// Grouped sums: sum[gid] += t * (AResult * AT^-1) over rows with a valid
// group id (aggregateAN.tcc:92-111); privatised in shared memory when the
// groups fit.
constexpr int kPrivGroups = 2048;

__global__ void __launch_bounds__(256) grouped_sum_kernel(DCol tail, DCol grp, uint64_t n, uint64_t ginv, uint64_t gmax,
                                                          uint64_t ngroups, uint64_t enc, unsigned long long* sums) {
    __shared__ unsigned long long s_sum[kPrivGroups];
    const bool priv = ngroups <= kPrivGroups;
    if (priv) {
        for (uint32_t g = threadIdx.x; g < ngroups; g += blockDim.x) s_sum[g] = 0;
        __syncthreads();
    }
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t gid = load_at(grp, i) * ginv;
        if (gid > gmax || gid >= ngroups) continue;
        const unsigned long long x = (unsigned long long)(load_at(tail, i) * enc);
        if (priv) atomicAdd(&s_sum[gid], x);
        else atomicAdd(&sums[gid], x);
    }
    if (priv) {
        __syncthreads();
        for (uint32_t g = threadIdx.x; g < ngroups; g += blockDim.x)
            if (s_sum[g]) atomicAdd(&sums[g], s_sum[g]);
    }
}

// hash<str_t>::get (miscellaneous.hpp:99-119): the Java-style string hash of
// a slot's chars up to its NUL (at most `width`), in 64 bits; each char is
// signed, and the multiplier's update (x 31) goes through a 32-bit int.
AHEAD_DEV uint64_t str_hash(const char* s, uint64_t width) {
    uint64_t len = 0;
    while (len < width && s[len]) ++len;
    uint64_t hash = 0, mult = 1;
    for (uint64_t k = len; k-- > 0;) {
        hash += (uint64_t)(int64_t)(signed char)s[k] * mult;
        const int32_t shifted = (int32_t)(uint32_t)(mult << 5);
        mult = (uint64_t)(int64_t)shifted - mult;
    }
    return hash;
}

// The binary group-by's keys over a string tail: hash(row) * numGroups + g
// in the larger type of v2_str_t, v2_bigint_t (groupbyAN.tcc:144).
__global__ void gb_insert_str_kernel(HashTab h, const char* strs, uint64_t width, DCol grp, uint64_t gainv,
                                     uint64_t ngroups, uint64_t n, uint32_t* slot_of, uint32_t* first) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t key = str_hash(strs + i * width, width) * ngroups + load_at(grp, i) * gainv;
        const uint32_t s = ht_insert(h, key);
        slot_of[i] = s;
        atomicMin(&first[s], (uint32_t)i);
    }
}

ahead_errvec* ev(ahead_errvec* errs, int k) { return errs ? &errs[k] : nullptr; }

int run_groupby(ahead_ctx* ctx, const ahead_bat* in, const ahead_bat* grouping, uint64_t ngroups, uint64_t aoid,
                uint64_t aoidinv, ahead_bat* gids, ahead_bat* firsts, uint64_t cap, ahead_errvec* errs, bool binary) {
    const int H = in->head.type, T = in->tail.type;
    const int eH = type_encoded(H);
    const uint64_t n = in->count;
    set_meta(&gids->head, AHEAD_VOID, 1, 1, 0, 0);
    set_meta(&gids->tail, AHEAD_RESOID, aoid, aoidinv, kRes56Max, 0);
    set_meta(&firsts->head, AHEAD_VOID, 1, 1, 0, 0);
    set_meta(&firsts->tail, AHEAD_RESOID, aoid, aoidinv, kRes56Max, 0);
    if (errs) {
        ev_begin(&errs[0], eH);
        ev_begin(&errs[1], 1);
        if (binary) ev_begin(&errs[2], 1);
    }
    gids->count = n;
    firsts->count = 0;
    OpScope s(ctx);
    const uint32_t cap_slots = ht_capacity(n);
    size_t need = (size_t)(cap_slots + 1) * (8 + 4 + 4) + n * 4 + compact_scratch<FirstOp>(n) + 3 * colcheck_scratch(n) +
                  4096;
    int rc = s.reserve(need);
    if (rc) return rc;
    if (n) {
        cudaStream_t st = ctx->stream;
        HashTab h{};
        h.mask = cap_slots - 1;
        h.keys = (uint64_t*)s.alloc((size_t)(cap_slots + 1) * 8);
        uint32_t* first = (uint32_t*)s.alloc((size_t)(cap_slots + 1) * 4);
        uint32_t* gid_of_slot = (uint32_t*)s.alloc((size_t)(cap_slots + 1) * 4);
        uint32_t* slot_of = (uint32_t*)s.alloc(n * 4);
        cudaMemsetAsync(h.keys, 0xff, (size_t)(cap_slots + 1) * 8, st);
        cudaMemsetAsync(first, 0xff, (size_t)(cap_slots + 1) * 4, st);
        GbKey k;
        k.tail = dcol(in->tail);
        k.grp = binary ? dcol(grouping->tail) : dcol(in->tail);
        k.keymask = wmask(type_base_width(T));
        k.lmask = wmask(type_width(type_larger_of(T)));
        k.ngroups = ngroups;
        k.gainv = binary ? grouping->tail.Ainv : 0;
        k.binary = binary;
        gb_insert_kernel<<<grid_for(n, 256), 256, 0, st>>>(h, k, n, slot_of, first);
        FirstOp op;
        op.base = (const char*)slot_of;
        op.status = s.d_status;
        op.first = first;
        op.gid_of_slot = gid_of_slot;
        op.head = dcol(in->head);
        op.aoid = aoid;
        op.cap = firsts->tail.data ? cap : 0;
        op.firsts = (uint64_t*)firsts->tail.data;
        op.acc = nullptr;
        op.decode_head = binary;
        run_compact(s, op, n, 0);
        if (gids->tail.data)
            gb_assign_kernel<<<grid_for(n, 256), 256, 0, st>>>(slot_of, first, gid_of_slot, n, aoid, binary,
                                                                (uint64_t*)gids->tail.data, cap);
        s.launched(2);
        if (eH) {
            const DCol hc = dcol(in->head);
            run_colcheck(s, in->head, n, hc.ainv, hc.umax, hc.width, aoid, ev(errs, 0), 1);
        }
        run_colcheck(s, in->tail, n, k.tail.ainv, k.tail.umax, k.tail.width, aoid, ev(errs, 1), 2);
        if (binary) run_colcheck(s, grouping->tail, n, grouping->tail.Ainv, grouping->tail.unenc_max, 8, aoid, ev(errs, 2), 3);
    }
    rc = s.finish(4);
    if (rc) return rc;
    firsts->count = n ? s.counter(0) : 0;
    if (errs && n) {
        if (eH) errs[0].count = s.counter(1);
        errs[1].count = s.counter(2);
        if (binary) errs[2].count = s.counter(3);
    }
    return (n > cap || firsts->count > cap) ? AHEAD_CAPACITY : AHEAD_OK;
}

bool head_ok(int h) { return h == AHEAD_VOID || h == AHEAD_OID || h == AHEAD_RESOID; }

// ------------------------------------------------------------ unencoded twins
// groupby (Normal/groupby.tcc:51-150): the same first-occurrence numbering on
// the raw tail (unary) or on t * numGroups + g in the tail's larger type
// (binary); outputs are oid_t: the group id of every row and the head of
// each group's first row.
struct FirstPlainOp {
    static constexpr int W = 4;
    static constexpr int NCH = 1;
    static constexpr bool ACC = false;
    static constexpr bool EMIT_V = false;
    static constexpr int NOUT = 1;
    const char* base;
    uint32_t* status;
    const uint32_t* first;
    uint32_t* gid_of_slot;
    DCol head;
    uint64_t cap;
    uint32_t* firsts;
    uint64_t* acc;
    AHEAD_DEV uint32_t eval(uint64_t v, uint64_t row, uint64_t&) const { return first[v] == (uint32_t)row ? 1u : 0u; }
    AHEAD_DEV uint64_t out0(int, uint64_t, uint64_t row) const { return row; }
    AHEAD_DEV void put0(int, uint64_t pos, uint64_t row) const {
        const uint32_t s = ((const uint32_t*)base)[row];
        gid_of_slot[s] = (uint32_t)pos;
        if (pos < cap) firsts[pos] = (uint32_t)load_at(head, row);
    }
    AHEAD_DEV void emit(int, uint64_t, uint64_t, uint64_t) const {}
};

__global__ void gb_assign_plain_kernel(const uint32_t* slot_of, const uint32_t* gid_of_slot, uint64_t n,
                                       uint32_t* gids, uint64_t cap) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n && i < cap;
         i += (uint64_t)gridDim.x * blockDim.x)
        gids[i] = gid_of_slot[slot_of[i]];
}

bool plain_groupable(int t) {
    return t == AHEAD_OID || t == AHEAD_TINYINT || t == AHEAD_SHORTINT || t == AHEAD_INT || t == AHEAD_RESOID ||
           t == AHEAD_RESTINY || t == AHEAD_RESSHORT || t == AHEAD_RESINT;
}

int run_groupby_plain(ahead_ctx* ctx, const ahead_bat* in, const ahead_bat* grouping, uint64_t ngroups,
                      ahead_bat* gids, ahead_bat* firsts, uint64_t cap, bool binary) {
    const int T = in->tail.type;
    const uint64_t n = in->count;
    default_meta(&gids->head, AHEAD_VOID);
    default_meta(&gids->tail, AHEAD_OID);
    default_meta(&firsts->head, AHEAD_VOID);
    default_meta(&firsts->tail, AHEAD_OID);
    gids->count = n;
    firsts->count = 0;
    OpScope s(ctx);
    const uint32_t cap_slots = ht_capacity(n);
    const size_t need = (size_t)(cap_slots + 1) * (8 + 4 + 4) + n * 4 + compact_scratch<FirstPlainOp>(n) + 4096;
    int rc = s.reserve(need);
    if (rc) return rc;
    if (n) {
        cudaStream_t st = ctx->stream;
        HashTab h{};
        h.mask = cap_slots - 1;
        h.keys = (uint64_t*)s.alloc((size_t)(cap_slots + 1) * 8);
        uint32_t* first = (uint32_t*)s.alloc((size_t)(cap_slots + 1) * 4);
        uint32_t* gid_of_slot = (uint32_t*)s.alloc((size_t)(cap_slots + 1) * 4);
        uint32_t* slot_of = (uint32_t*)s.alloc(n * 4);
        cudaMemsetAsync(h.keys, 0xff, (size_t)(cap_slots + 1) * 8, st);
        cudaMemsetAsync(first, 0xff, (size_t)(cap_slots + 1) * 4, st);
        GbKey k;
        k.tail = dcol(in->tail);
        k.tail.enc = 0;  // the raw tail: an encoded tail is grouped by its codes
        k.grp = binary ? dcol(grouping->tail) : dcol(in->tail);
        k.keymask = wmask(type_width(T));
        k.lmask = wmask(type_width(type_larger_of(T)));
        k.ngroups = ngroups;
        k.gainv = 1;
        k.binary = binary;
        gb_insert_kernel<<<grid_for(n, 256), 256, 0, st>>>(h, k, n, slot_of, first);
        FirstPlainOp op;
        op.base = (const char*)slot_of;
        op.status = s.d_status;
        op.first = first;
        op.gid_of_slot = gid_of_slot;
        op.head = dcol(in->head);
        op.cap = firsts->tail.data ? cap : 0;
        op.firsts = (uint32_t*)firsts->tail.data;
        op.acc = nullptr;
        run_compact(s, op, n, 0);
        if (gids->tail.data)
            gb_assign_plain_kernel<<<grid_for(n, 256), 256, 0, st>>>(slot_of, gid_of_slot, n,
                                                                      (uint32_t*)gids->tail.data, cap);
        s.launched(2);
    }
    rc = s.finish(1);
    if (rc) return rc;
    firsts->count = n ? s.counter(0) : 0;
    return (n > cap || firsts->count > cap) ? AHEAD_CAPACITY : AHEAD_OK;
}

// aggregate_sum<Result> (Normal/aggregate_scalar.tcc:47-58): the sum of the
// tails (the result type is at least as wide as the tail), mod 2^64 here and
// narrowed on the host.
__global__ void sum_plain_kernel(DCol tail, uint64_t n, unsigned long long* out) {
    unsigned long long acc = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        acc += load_at(tail, i);
    acc = warp_sum64(acc);
    if ((threadIdx.x & 31) == 0 && acc) atomicAdd(out, acc);
}

// arithmetic<Op, Result> (Normal/arithmetic_scalar.tcc:46-82) in the tails'
// width; division by zero yields 0 (undefined in the reference).
__global__ void arith_plain_kernel(DCol a, DCol b, uint64_t n, int op, int w, void* out) {
    const uint64_t m = wmask(w);
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t x = load_at(a, i), y = load_at(b, i);
        uint64_t r;
        switch (op) {
            case AHEAD_ADD: r = x + y; break;
            case AHEAD_SUB: r = x - y; break;
            case AHEAD_MUL: r = x * y; break;
            default: r = y ? x / y : 0; break;
        }
        store_at(out, w, i, r & m);
    }
}

}  // namespace

extern "C" {

int ahead_gpu_groupby_an(ahead_ctx* ctx, const ahead_bat* in, uint64_t aoid, uint64_t aoidinv, ahead_bat* gids,
                         ahead_bat* firsts, uint64_t cap, ahead_errvec* errs) {
    if (!ctx || !in || !gids || !firsts) return AHEAD_BAD_ARG;
    if (!head_ok(in->head.type) || !type_encoded(in->tail.type))
        return fail(ctx, AHEAD_BAD_ARG, "groupbyAN: void/oid/resoid head and AN tail required");
    return run_groupby(ctx, in, nullptr, 0, aoid, aoidinv, gids, firsts, cap, errs, false);
}

int ahead_gpu_groupby2_an(ahead_ctx* ctx, const ahead_bat* in, const ahead_bat* grouping, uint64_t ngroups,
                          uint64_t aoid, uint64_t aoidinv, ahead_bat* gids, ahead_bat* firsts, uint64_t cap,
                          ahead_errvec* errs) {
    if (!ctx || !in || !grouping || !gids || !firsts) return AHEAD_BAD_ARG;
    if (!head_ok(in->head.type) || !type_encoded(in->tail.type) || grouping->head.type != AHEAD_VOID ||
        grouping->tail.type != AHEAD_RESOID)
        return fail(ctx, AHEAD_BAD_ARG, "groupbyAN: (void/oid/resoid, AN) and a (void, resoid) grouping required");
    if (in->count != grouping->count)
        return fail(ctx, AHEAD_SIZE_MISMATCH, "input BAT and existing grouping have different sizes!");
    return run_groupby(ctx, in, grouping, ngroups, aoid, aoidinv, gids, firsts, cap, errs, true);
}

int ahead_gpu_aggregate_sum_grouped_an(ahead_ctx* ctx, const ahead_bat* in, const ahead_bat* grouping,
                                       uint64_t ngroups, int result_type, uint64_t ar, uint64_t arinv, uint64_t aoid,
                                       ahead_bat* out, ahead_errvec* errs) {
    if (!ctx || !in || !grouping || !out) return AHEAD_BAD_ARG;
    const int H = in->head.type, T = in->tail.type;
    if (result_type != AHEAD_RESBIGINT) return fail(ctx, AHEAD_BAD_ARG, "aggregate_sum_groupedAN: resbigint result");
    if (!head_ok(H) || !(T == AHEAD_INT || T == AHEAD_RESINT || T == AHEAD_RESBIGINT || T == AHEAD_RESSHORT ||
                         T == AHEAD_RESTINY))
        return fail(ctx, AHEAD_BAD_ARG, "aggregate_sum_groupedAN: unsupported input types");
    if (grouping->head.type != AHEAD_VOID || grouping->tail.type != AHEAD_RESOID)
        return fail(ctx, AHEAD_BAD_ARG, "aggregate_sum_groupedAN: (void, resoid) grouping required");
    if (in->count != grouping->count) return fail(ctx, AHEAD_SIZE_MISMATCH, "bat and grouping must have the same size!");
    const int eH = type_encoded(H), eT = type_encoded(T);
    const int wh = type_width(type_encoded_of(H)), wt = type_width(type_encoded_of(T));
    const uint64_t AT = in->tail.A & wmask(wt);
    const uint64_t enc = ar * (eT ? inv_pow2(AT, 64) : 1ull);
    default_meta(&out->head, AHEAD_VOID);
    set_meta(&out->tail, AHEAD_RESBIGINT, ar, arinv, kRes56Max, 0);
    if (errs) {
        ev_begin(&errs[0], eH);
        ev_begin(&errs[1], eT);
        ev_begin(&errs[2], 1);
    }
    out->count = ngroups;
    const uint64_t n = in->count;
    OpScope s(ctx);
    int rc = s.reserve(3 * colcheck_scratch(n));
    if (rc) return rc;
    if (ngroups && out->tail.data) cudaMemsetAsync(out->tail.data, 0, ngroups * 8, ctx->stream);
    if (n && out->tail.data) {
        grouped_sum_kernel<<<grid_for(n, 256), 256, 0, ctx->stream>>>(dcol(in->tail), dcol(grouping->tail), n,
                                                                      grouping->tail.Ainv, grouping->tail.unenc_max,
                                                                      ngroups, enc,
                                                                      (unsigned long long*)out->tail.data);
        s.launched();
    }
    if (n) {
        if (eH) run_colcheck(s, in->head, n, in->head.Ainv & wmask(wh), in->head.unenc_max & wmask(wh), wh, aoid, ev(errs, 0), 0);
        if (eT) run_colcheck(s, in->tail, n, in->tail.Ainv & wmask(wt), in->tail.unenc_max & wmask(wt), wt, aoid, ev(errs, 1), 1);
        run_colcheck(s, grouping->tail, n, grouping->tail.Ainv, grouping->tail.unenc_max, 8, aoid, ev(errs, 2), 2);
    }
    rc = s.finish(3);
    if (rc) return rc;
    if (errs && n) {
        if (eH) errs[0].count = s.counter(0);
        if (eT) errs[1].count = s.counter(1);
        errs[2].count = s.counter(2);
    }
    return AHEAD_OK;
}


int ahead_gpu_groupby(ahead_ctx* ctx, const ahead_bat* in, ahead_bat* gids, ahead_bat* firsts, uint64_t cap) {
    if (!ctx || !in || !gids || !firsts) return AHEAD_BAD_ARG;
    if (!(in->head.type == AHEAD_VOID || in->head.type == AHEAD_OID) || !plain_groupable(in->tail.type))
        return fail(ctx, AHEAD_BAD_ARG, "groupby: void/oid head and an integer or code tail required");
    return run_groupby_plain(ctx, in, nullptr, 0, gids, firsts, cap, false);
}

int ahead_gpu_groupby2(ahead_ctx* ctx, const ahead_bat* in, const ahead_bat* grouping, uint64_t ngroups,
                       ahead_bat* gids, ahead_bat* firsts, uint64_t cap) {
    if (!ctx || !in || !grouping || !gids || !firsts) return AHEAD_BAD_ARG;
    if (!(in->head.type == AHEAD_VOID || in->head.type == AHEAD_OID) || !plain_groupable(in->tail.type) ||
        grouping->head.type != AHEAD_VOID || grouping->tail.type != AHEAD_OID)
        return fail(ctx, AHEAD_BAD_ARG, "groupby: (void/oid, integer) and a (void, oid) grouping required");
    if (in->count != grouping->count)
        return fail(ctx, AHEAD_SIZE_MISMATCH, "input BAT and existing grouping have different sizes!");
    return run_groupby_plain(ctx, in, grouping, ngroups, gids, firsts, cap, true);
}

int ahead_gpu_aggregate_sum_grouped(ahead_ctx* ctx, const ahead_bat* in, const ahead_bat* grouping,
                                    uint64_t ngroups, int result_type, ahead_bat* out) {
    if (!ctx || !in || !grouping || !out) return AHEAD_BAD_ARG;
    if (result_type != AHEAD_BIGINT || !(in->head.type == AHEAD_VOID || in->head.type == AHEAD_OID) ||
        in->tail.type != AHEAD_INT || grouping->head.type != AHEAD_VOID || grouping->tail.type != AHEAD_OID)
        return fail(ctx, AHEAD_BAD_ARG, "aggregate_sum_grouped: (void/oid, int), (void, oid) grouping, bigint result");
    if (in->count != grouping->count) return fail(ctx, AHEAD_SIZE_MISMATCH, "bat and grouping must have the same size!");
    default_meta(&out->head, AHEAD_VOID);
    default_meta(&out->tail, AHEAD_BIGINT);
    out->count = ngroups;
    const uint64_t n = in->count;
    OpScope s(ctx);
    int rc = s.reserve(0);
    if (rc) return rc;
    if (ngroups && out->tail.data) cudaMemsetAsync(out->tail.data, 0, ngroups * 8, ctx->stream);
    if (n && out->tail.data) {
        // group ids beyond numGroups index past the reference's vector; skipped here
        grouped_sum_kernel<<<grid_for(n, 256), 256, 0, ctx->stream>>>(dcol(in->tail), dcol(grouping->tail), n, 1,
                                                                      ~0ull, ngroups, 1,
                                                                      (unsigned long long*)out->tail.data);
        s.launched();
    }
    return s.finish(0);
}

int ahead_gpu_aggregate_sum(ahead_ctx* ctx, const ahead_bat* in, int result_type, uint64_t* total) {
    if (!ctx || !in || !total) return AHEAD_BAD_ARG;
    const int T = in->tail.type;
    const bool ints = [](int t) {
        return t == AHEAD_TINYINT || t == AHEAD_SHORTINT || t == AHEAD_INT || t == AHEAD_BIGINT;
    }(T) && (result_type == AHEAD_TINYINT || result_type == AHEAD_SHORTINT || result_type == AHEAD_INT ||
             result_type == AHEAD_BIGINT);
    if (in->head.type != AHEAD_OID || !ints || type_width(result_type) < type_width(T))
        return fail(ctx, AHEAD_BAD_ARG, "aggregate_sum: (oid, integer) input and a result at least as wide");
    OpScope s(ctx);
    int rc = s.reserve(0);
    if (rc) return rc;
    if (in->count) {
        sum_plain_kernel<<<grid_for(in->count, 256), 256, 0, ctx->stream>>>(dcol(in->tail), in->count,
                                                                             (unsigned long long*)s.d_counters);
        s.launched();
    }
    rc = s.finish(1);
    if (rc) return rc;
    *total = (in->count ? s.counter(0) : 0) & wmask(type_width(result_type));
    return AHEAD_OK;
}

int ahead_gpu_arithmetic(ahead_ctx* ctx, int op, int result_type, const ahead_bat* a, const ahead_bat* b,
                         ahead_bat* out) {
    if (!ctx || !a || !b || !out) return AHEAD_BAD_ARG;
    const int T = a->tail.type;
    if (a->head.type != AHEAD_VOID || b->head.type != AHEAD_VOID || b->tail.type != T || result_type != T ||
        !(T == AHEAD_INT || T == AHEAD_RESINT) || op < AHEAD_ADD || op > AHEAD_DIV)
        return fail(ctx, AHEAD_BAD_ARG, "arithmetic: (void, int|resint) inputs of one type and that result type");
    if (a->count != b->count) return fail(ctx, AHEAD_SIZE_MISMATCH, "arithmetic: bat1->size() != bat2->size()");
    // the result keeps the first input's metadata (skeleton, miscellaneous.hpp:122-132)
    copy_meta(&out->head, AHEAD_VOID, &a->head);
    copy_meta(&out->tail, result_type, &a->tail);
    out->count = a->count;
    OpScope s(ctx);
    int rc = s.reserve(0);
    if (rc) return rc;
    if (a->count && out->tail.data) {
        arith_plain_kernel<<<grid_for(a->count, 256), 256, 0, ctx->stream>>>(dcol(a->tail), dcol(b->tail), a->count,
                                                                              op, type_width(T), out->tail.data);
        s.launched();
    }
    return s.finish(0);
}

int ahead_gpu_groupby2_str_an(ahead_ctx* ctx, const char* strs, uint64_t width, uint64_t count, uint64_t seqbase,
                              const ahead_bat* grouping, uint64_t ngroups, uint64_t aoid, uint64_t aoidinv,
                              ahead_bat* gids, ahead_bat* firsts, uint64_t cap, ahead_errvec* errs) {
    if (!ctx || !grouping || !gids || !firsts || !width || (count && !strs)) return AHEAD_BAD_ARG;
    if (grouping->head.type != AHEAD_VOID || grouping->tail.type != AHEAD_RESOID)
        return fail(ctx, AHEAD_BAD_ARG, "groupbyAN(str): (void, resoid) grouping required");
    if (count != grouping->count) return fail(ctx, AHEAD_SIZE_MISMATCH, "groupbyAN(str): sizes differ");
    set_meta(&gids->head, AHEAD_VOID, 1, 1, 0, 0);
    set_meta(&gids->tail, AHEAD_RESOID, aoid, aoidinv, kRes56Max, 0);
    set_meta(&firsts->head, AHEAD_VOID, 1, 1, 0, 0);
    set_meta(&firsts->tail, AHEAD_RESOID, aoid, aoidinv, kRes56Max, 0);
    if (errs) {
        ev_begin(&errs[0], 0);
        ev_begin(&errs[1], 0);
        ev_begin(&errs[2], 1);
    }
    const uint64_t n = count;
    gids->count = n;
    firsts->count = 0;
    OpScope s(ctx);
    const uint32_t cap_slots = ht_capacity(n);
    int rc = s.reserve((size_t)(cap_slots + 1) * (8 + 4 + 4) + n * 4 + compact_scratch<FirstOp>(n) +
                       colcheck_scratch(n) + 4096);
    if (rc) return rc;
    if (n) {
        cudaStream_t st = ctx->stream;
        HashTab h{};
        h.mask = cap_slots - 1;
        h.keys = (uint64_t*)s.alloc((size_t)(cap_slots + 1) * 8);
        uint32_t* first = (uint32_t*)s.alloc((size_t)(cap_slots + 1) * 4);
        uint32_t* gid_of_slot = (uint32_t*)s.alloc((size_t)(cap_slots + 1) * 4);
        uint32_t* slot_of = (uint32_t*)s.alloc(n * 4);
        cudaMemsetAsync(h.keys, 0xff, (size_t)(cap_slots + 1) * 8, st);
        cudaMemsetAsync(first, 0xff, (size_t)(cap_slots + 1) * 4, st);
        gb_insert_str_kernel<<<grid_for(n, 256), 256, 0, st>>>(h, strs, width, dcol(grouping->tail),
                                                               grouping->tail.Ainv, ngroups, n, slot_of, first);
        ahead_col vh{};
        vh.type = AHEAD_VOID;
        vh.seqbase = seqbase;
        FirstOp op;
        op.base = (const char*)slot_of;
        op.status = s.d_status;
        op.first = first;
        op.gid_of_slot = gid_of_slot;
        op.head = dcol(vh);
        op.aoid = aoid;
        op.cap = firsts->tail.data ? cap : 0;
        op.firsts = (uint64_t*)firsts->tail.data;
        op.acc = nullptr;
        op.decode_head = 1;
        run_compact(s, op, n, 0);
        if (gids->tail.data)
            gb_assign_kernel<<<grid_for(n, 256), 256, 0, st>>>(slot_of, first, gid_of_slot, n, aoid, 1,
                                                                (uint64_t*)gids->tail.data, cap);
        s.launched(2);
        run_colcheck(s, grouping->tail, n, grouping->tail.Ainv, grouping->tail.unenc_max, 8, aoid, ev(errs, 2), 1);
    }
    rc = s.finish(2);
    if (rc) return rc;
    firsts->count = n ? s.counter(0) : 0;
    if (errs && n) errs[2].count = s.counter(1);
    return (n > cap || firsts->count > cap) ? AHEAD_CAPACITY : AHEAD_OK;
}

int ahead_gpu_groupby2_str(ahead_ctx* ctx, const char* strs, uint64_t width, uint64_t count, uint64_t seqbase,
                           const ahead_bat* grouping, uint64_t ngroups, ahead_bat* gids, ahead_bat* firsts,
                           uint64_t cap) {
    if (!ctx || !grouping || !gids || !firsts || !width || (count && !strs)) return AHEAD_BAD_ARG;
    if (grouping->head.type != AHEAD_VOID || grouping->tail.type != AHEAD_OID)
        return fail(ctx, AHEAD_BAD_ARG, "groupby(str): (void, oid) grouping required");
    if (count != grouping->count) return fail(ctx, AHEAD_SIZE_MISMATCH, "groupby(str): sizes differ");
    default_meta(&gids->head, AHEAD_VOID);
    default_meta(&gids->tail, AHEAD_OID);
    default_meta(&firsts->head, AHEAD_VOID);
    default_meta(&firsts->tail, AHEAD_OID);
    const uint64_t n = count;
    gids->count = n;
    firsts->count = 0;
    OpScope s(ctx);
    const uint32_t cap_slots = ht_capacity(n);
    int rc = s.reserve((size_t)(cap_slots + 1) * (8 + 4 + 4) + n * 4 + compact_scratch<FirstPlainOp>(n) + 4096);
    if (rc) return rc;
    if (n) {
        cudaStream_t st = ctx->stream;
        HashTab h{};
        h.mask = cap_slots - 1;
        h.keys = (uint64_t*)s.alloc((size_t)(cap_slots + 1) * 8);
        uint32_t* first = (uint32_t*)s.alloc((size_t)(cap_slots + 1) * 4);
        uint32_t* gid_of_slot = (uint32_t*)s.alloc((size_t)(cap_slots + 1) * 4);
        uint32_t* slot_of = (uint32_t*)s.alloc(n * 4);
        cudaMemsetAsync(h.keys, 0xff, (size_t)(cap_slots + 1) * 8, st);
        cudaMemsetAsync(first, 0xff, (size_t)(cap_slots + 1) * 4, st);
        gb_insert_str_kernel<<<grid_for(n, 256), 256, 0, st>>>(h, strs, width, dcol(grouping->tail), 1, ngroups, n,
                                                               slot_of, first);
        ahead_col vh{};
        vh.type = AHEAD_VOID;
        vh.seqbase = seqbase;
        FirstPlainOp op;
        op.base = (const char*)slot_of;
        op.status = s.d_status;
        op.first = first;
        op.gid_of_slot = gid_of_slot;
        op.head = dcol(vh);
        op.cap = firsts->tail.data ? cap : 0;
        op.firsts = (uint32_t*)firsts->tail.data;
        op.acc = nullptr;
        run_compact(s, op, n, 0);
        if (gids->tail.data)
            gb_assign_plain_kernel<<<grid_for(n, 256), 256, 0, st>>>(slot_of, gid_of_slot, n,
                                                                      (uint32_t*)gids->tail.data, cap);
        s.launched(2);
    }
    rc = s.finish(1);
    if (rc) return rc;
    firsts->count = n ? s.counter(0) : 0;
    return (n > cap || firsts->count > cap) ? AHEAD_CAPACITY : AHEAD_OK;
}

}  // extern "C"
