// ops_scan.cu -- streaming AN operators: selectAN / select, checkAN,
// decodeAN, checkAndDecodeAN, encodeAN, aggregate_mul_sum(AN), arithmeticAN.
//
// Each operator is one pass over its input columns through the compaction
// kernel of compact.cuh: the AN check is fused into the load (multiply by
// A^-1 mod 2^w, compare with the largest valid value), predicates are
// evaluated on the codes, and kept rows and error positions are written in
// scan order.
#include <cstring>

#include "ops_common.cuh"

using namespace ahead;

namespace {

// ------------------------------------------------------------ selection
// selectAN_scalar.tcc:84-92 (AN) and Normal/select_scalar.tcc:66-72 (plain).
template <int WW, bool AN>
struct SelectOp {
    static constexpr int W = WW;
    static constexpr int NCH = AN ? 2 : 1;
    static constexpr bool ACC = false;
    const char* base;
    uint32_t* status;
    uint64_t seqbase, ainv, umax, aoid, cap, errcap;
    uint64_t* out_an;
    uint32_t* out_oid;
    uint64_t* err;
    uint64_t* acc;
    static constexpr bool EMIT_V = false;
    static constexpr int NOUT = 1;
    RangePred pred;
    AHEAD_DEV uint64_t out0(int, uint64_t, uint64_t row) const {
        const uint32_t oid = (uint32_t)(seqbase + row);
        return AN ? (uint64_t)oid * kResoidAMax : (uint64_t)oid;
    }
    AHEAD_DEV void put0(int, uint64_t pos, uint64_t val) const {
        if (pos < cap) {
            if (AN) out_an[pos] = val;
            else out_oid[pos] = (uint32_t)val;
        }
    }
    AHEAD_DEV uint32_t eval(uint64_t v, uint64_t, uint64_t&) const {
        if constexpr (W <= 4) {
            // narrow codes: 32-bit arithmetic; a single plain interval is the common case
            const uint32_t x = (uint32_t)v;
            const bool keep = pred.two || pred.neg1 ? pred(v) : (x - (uint32_t)pred.lo1) <= (uint32_t)pred.span1;
            uint32_t b = keep ? 1u : 0u;
            if (AN) {
                const uint32_t d = x * (uint32_t)ainv;
                if ((W == 4 ? d : (d & (uint32_t)wmask(W))) > (uint32_t)umax) b |= 2u;
            }
            return b;
        } else {
            uint32_t b = pred(v) ? 1u : 0u;
            if (AN && v * ainv > umax) b |= 2u;
            return b;
        }
    }
    AHEAD_DEV void emit(int c, uint64_t pos, uint64_t, uint64_t row) const {
        const uint32_t oid = (uint32_t)(seqbase + row);
        if (c == 0) {
            if (pos < cap) {
                if (AN) out_an[pos] = (uint64_t)oid * kResoidAMax;
                else out_oid[pos] = oid;
            }
        } else if (pos < errcap) {
            err[pos] = row * aoid;
        }
    }
};

template <int W, bool AN>
int run_select(OpScope& s, const ahead_bat* in, const RangePred& p, uint64_t aoid, ahead_bat* out, uint64_t cap,
               ahead_errvec* err) {
    typedef SelectOp<W, AN> Op;
    int rc = s.reserve(compact_scratch<Op>(in->count));
    if (rc) return rc;
    Op op;
    op.base = (const char*)in->tail.data;
    op.status = s.d_status;
    op.seqbase = in->head.seqbase;
    op.ainv = in->tail.Ainv & wmask(W);
    op.umax = in->tail.unenc_max & wmask(W);
    op.aoid = aoid;
    op.cap = out->head.data ? cap : 0;
    op.out_an = (uint64_t*)out->head.data;
    op.out_oid = (uint32_t*)out->head.data;
    op.err = err ? err->data : nullptr;
    op.errcap = (err && err->data) ? err->capacity : 0;
    op.acc = nullptr;
    op.pred = p;
    run_compact<Op>(s, op, in->count, 0);
    rc = s.finish(Op::NCH);
    if (rc) return rc;
    out->count = s.counter(0);
    if (AN && err) err->count = s.counter(1);
    return out->count > cap ? AHEAD_CAPACITY : AHEAD_OK;
}

bool op_ok(int op) { return op >= AHEAD_CMP_LT && op <= AHEAD_CMP_GT; }

// ------------------------------------------------------ string selection
// Selection(AN)1/2<..., v2_void_t, v2_str_t>::filter (selectAN_scalar.tcc:98-131,
// 185-222; Normal/select_scalar.tcc:78-101, 137-165): keep a row when
// Op(strcmp(row, th), 0) holds.  One pass classifies every row into a byte
// flag (1 = kept), then the select compaction of the flags writes the OIDs in
// row order.  String columns live in dimension tables (at most a few million
// rows), so the flag pass is one thread per row reading its slot through L1.
struct StrPred {
    char th[2][AHEAD_STR_TH_MAX + 1];  // NUL-terminated
    int op1, op2, comb;
};

// Sign of strcmp(row, th) over unsigned bytes; the row ends at its first NUL
// or after `width` bytes, the threshold at its NUL.
AHEAD_DEV int str_sign(const unsigned char* row, uint64_t width, const char* th) {
    for (uint64_t k = 0;; ++k) {
        const unsigned a = k < width ? (unsigned)__ldg(row + k) : 0u;
        const unsigned b = (unsigned char)th[k];
        if (a != b) return a < b ? -1 : 1;
        if (a == 0) return 0;
    }
}

AHEAD_DEV bool sign_holds(int op, int c) {
    switch (op) {
        case AHEAD_CMP_LT: return c < 0;
        case AHEAD_CMP_LE: return c <= 0;
        case AHEAD_CMP_EQ: return c == 0;
        case AHEAD_CMP_NE: return c != 0;
        case AHEAD_CMP_GE: return c >= 0;
        default: return c > 0;
    }
}

__global__ void __launch_bounds__(256) str_flag_kernel(const unsigned char* strs, uint64_t width, uint64_t n,
                                                       StrPred p, uint8_t* flags) {
    __shared__ char th[2][AHEAD_STR_TH_MAX + 1];
    for (int i = threadIdx.x; i < 2 * (AHEAD_STR_TH_MAX + 1); i += blockDim.x) (&th[0][0])[i] = (&p.th[0][0])[i];
    __syncthreads();
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += stride) {
        const unsigned char* row = strs + r * width;
        bool keep = sign_holds(p.op1, str_sign(row, width, th[0]));
        if (p.op2 != AHEAD_CMP_NONE) {
            const bool b = sign_holds(p.op2, str_sign(row, width, th[1]));
            keep = p.comb == AHEAD_OR ? (keep || b) : (keep && b);
        }
        flags[r] = keep ? 1 : 0;
    }
}

template <bool AN>
int run_select_str(ahead_ctx* ctx, const char* strs, uint64_t width, uint64_t count, uint64_t seqbase,
                   const StrPred& sp, ahead_bat* out, uint64_t cap) {
    typedef SelectOp<1, AN> Op;
    OpScope s(ctx);
    int rc = s.reserve(compact_scratch<Op>(count) + count + 256);
    if (rc) return rc;
    uint8_t* flags = (uint8_t*)s.alloc(count);
    if (count) {
        const uint64_t want = (count + 255) / 256;
        const unsigned grid = (unsigned)(want < (uint64_t)ctx->num_sms * 8 ? want : (uint64_t)ctx->num_sms * 8);
        str_flag_kernel<<<grid, 256, 0, ctx->stream>>>((const unsigned char*)strs, width, count, sp, flags);
        s.launched();
    }
    Op op;  // over the flag bytes: A^-1 = 1 and maximum 0xFF, so no flag is ever reported as corrupt
    op.base = (const char*)flags;
    op.status = s.d_status;
    op.seqbase = seqbase;
    op.ainv = 1;
    op.umax = 0xFF;
    op.aoid = 0;
    op.cap = out->head.data ? cap : 0;
    op.out_an = (uint64_t*)out->head.data;
    op.out_oid = (uint32_t*)out->head.data;
    op.err = nullptr;
    op.errcap = 0;
    op.acc = nullptr;
    op.pred = RangePred::make(AHEAD_CMP_EQ, 1, AHEAD_CMP_NONE, 0, AHEAD_AND, wmask(1));
    run_compact<Op>(s, op, count, 0);
    rc = s.finish(Op::NCH);
    if (rc) return rc;
    out->count = s.counter(0);
    return out->count > cap ? AHEAD_CAPACITY : AHEAD_OK;
}

// Positions of the restiny codes whose product with A^-1, taken in 32 bits
// and compared signed, exceeds the largest value: the unreduced check of the
// string hash join's left build (hashjoinAN.tcc:290).  The flags go through
// the error stream of the select compaction (A^-1 = 1, maximum 0), which
// writes row * aoid for every flagged row in row order.
__global__ void __launch_bounds__(256) promoted_check_kernel(const uint16_t* codes, uint64_t n, uint32_t ainv,
                                                             int32_t umax, uint8_t* flags) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += stride)
        flags[r] = (int32_t)((uint32_t)codes[r] * ainv) > umax ? 1 : 0;
}

int select_str_args(ahead_ctx* ctx, const char* strs, uint64_t width, uint64_t count, int op1, const char* th1,
                    int op2, const char* th2, int comb, ahead_bat* out, StrPred* sp, const char* what) {
    if (!out || !th1 || (op2 != AHEAD_CMP_NONE && !th2)) return fail(ctx, AHEAD_BAD_ARG, what);
    if (count && (!strs || width == 0)) return fail(ctx, AHEAD_BAD_ARG, what);
    if (!op_ok(op1) || (op2 != AHEAD_CMP_NONE && !op_ok(op2))) return fail(ctx, AHEAD_BAD_ARG, what);
    if (op2 != AHEAD_CMP_NONE && comb != AHEAD_AND && comb != AHEAD_OR) return fail(ctx, AHEAD_BAD_ARG, what);
    std::memset(sp, 0, sizeof(*sp));
    const char* th[2] = {th1, op2 != AHEAD_CMP_NONE ? th2 : ""};
    for (int i = 0; i < 2; ++i) {
        const size_t len = std::strlen(th[i]);
        if (len > AHEAD_STR_TH_MAX)
            return fail(ctx, AHEAD_UNSUPPORTED, "string select: threshold longer than AHEAD_STR_TH_MAX");
        std::memcpy(sp->th[i], th[i], len);
    }
    sp->op1 = op1;
    sp->op2 = op2;
    sp->comb = comb;
    return AHEAD_OK;
}

RangePred make_pred(int op1, uint64_t th1, int op2, uint64_t th2, int comb, int w) {
    return RangePred::make(op1, th1, op2, th2, comb, wmask(w));
}

// ------------------------------------------------------------ check / decode
// checkAndDecodeAN with a void head (encdecAN_scalar.tcc:195-204): corrupt rows
// are dropped and reported; kept rows are decoded and narrowed.
template <int WW>
struct CadVoidOp {
    static constexpr int W = WW;
    static constexpr int NCH = 2;
    static constexpr bool ACC = false;
    const char* base;
    uint32_t* status;
    void* out;
    int ow;
    uint64_t ainv, umax, aoid, cap, errcap;
    uint64_t* err;
    uint64_t* acc;
    static constexpr bool EMIT_V = true;
    static constexpr int NOUT = 1;
    AHEAD_DEV uint32_t eval(uint64_t v, uint64_t, uint64_t&) const {
        return mulw(v, ainv, W) > umax ? 2u : 1u;
    }
    AHEAD_DEV uint64_t out0(int, uint64_t v, uint64_t) const { return mulw(v, ainv, W); }
    AHEAD_DEV void put0(int, uint64_t pos, uint64_t val) const {
        if (pos < cap) store_at(out, ow, pos, val);
    }
    AHEAD_DEV void emit(int c, uint64_t pos, uint64_t v, uint64_t row) const {
        if (c == 0) {
            if (pos < cap) store_at(out, ow, pos, mulw(v, ainv, W));
        } else if (pos < errcap) {
            err[pos] = row * aoid;
        }
    }
};

// checkAndDecodeAN with an oid / resoid head (encdecAN_scalar.tcc:152-170).
// Driving column: the tail; the head is read per row (consecutive lanes read
// consecutive rows).
template <int WW>
struct CadGenOp {
    static constexpr int W = WW;
    static constexpr int NCH = 3;
    static constexpr bool ACC = false;
    const char* base;
    uint32_t* status;
    DCol hc, tc;
    void *oh, *ot;
    int ohw, otw;
    uint64_t aoid, cap, ecap_h, ecap_t;
    uint64_t *err_h, *err_t;
    uint64_t* acc;
    static constexpr bool EMIT_V = true;
    static constexpr int NOUT = 2;
    AHEAD_DEV uint64_t out0(int k, uint64_t t, uint64_t row) const {
        return k == 0 ? dec_if(hc, load_at(hc, row), hc.ainv) : mulw(t, tc.ainv, W);
    }
    AHEAD_DEV void put0(int k, uint64_t pos, uint64_t val) const {
        if (pos < cap) store_at(k == 0 ? oh : ot, k == 0 ? ohw : otw, pos, val);
    }
    AHEAD_DEV uint32_t eval(uint64_t t, uint64_t row, uint64_t&) const {
        const uint64_t h = load_at(hc, row);
        const uint64_t dh = dec_if(hc, h, hc.ainv), dt = mulw(t, tc.ainv, W);
        const bool hok = !hc.enc || dh <= hc.umax, tok = dt <= tc.umax;
        return (hok && tok ? 1u : 0u) | (hok ? 0u : 2u) | (tok ? 0u : 4u);
    }
    AHEAD_DEV void emit(int c, uint64_t pos, uint64_t t, uint64_t row) const {
        if (c == 0) {
            if (pos < cap) {
                store_at(oh, ohw, pos, dec_if(hc, load_at(hc, row), hc.ainv));
                store_at(ot, otw, pos, mulw(t, tc.ainv, W));
            }
        } else if (c == 1) {
            if (pos < ecap_h) err_h[pos] = row * aoid;
        } else if (pos < ecap_t) {
            err_t[pos] = row * aoid;
        }
    }
};

// decodeAN (encdecAN_scalar.tcc:115-122): every row is decoded and kept.
template <int WW>
struct DecodeOp {
    static constexpr int W = WW;
    static constexpr int NCH = 1;
    static constexpr bool ACC = false;
    const char* base;
    uint32_t* status;
    DCol hc, tc;
    void *oh, *ot;
    int ohw, otw;
    uint64_t aoid, errcap;
    uint64_t* err;
    uint64_t* acc;
    static constexpr bool EMIT_V = false;
    static constexpr int NOUT = 1;
    AHEAD_DEV uint64_t out0(int, uint64_t, uint64_t row) const { return row * aoid; }
    AHEAD_DEV void put0(int, uint64_t pos, uint64_t val) const {
        if (pos < errcap) err[pos] = val;
    }
    AHEAD_DEV uint32_t eval(uint64_t t, uint64_t row, uint64_t&) const {
        const uint64_t d = mulw(t, tc.ainv, W);
        store_at(oh, ohw, row, load_at(hc, row));
        store_at(ot, otw, row, d);
        return d > tc.umax ? 1u : 0u;
    }
    AHEAD_DEV void emit(int, uint64_t pos, uint64_t, uint64_t row) const {
        if (pos < errcap) err[pos] = row * aoid;
    }
};

// ------------------------------------------------------------ mul-sum
// aggregate_mul_sumAN (aggregateAN_scalar.tcc:98-124): sum of the raw code
// products, then one multiplication by RA * A1^-1 * A2^-1 on the host.
template <int WW>
struct MulSumOp {
    static constexpr int W = WW;
    static constexpr int NCH = 2;
    static constexpr bool ACC = true;
    const char* base;
    uint32_t* status;
    DCol ac, bc;
    uint64_t aoid, ecap1, ecap2;
    uint64_t *e1, *e2;
    uint64_t* acc;
    static constexpr bool EMIT_V = false;
    static constexpr int NOUT = 1;
    AHEAD_DEV uint64_t out0(int, uint64_t, uint64_t row) const { return row * aoid; }
    AHEAD_DEV void put0(int, uint64_t pos, uint64_t val) const {
        if (pos < ecap1) e1[pos] = val;
    }
    AHEAD_DEV uint32_t eval(uint64_t a, uint64_t row, uint64_t& s) const {
        const uint64_t b = load_at(bc, row);
        s += a * b;
        return (mulw(a, ac.ainv, W) > ac.umax ? 1u : 0u) | (mulw(b, bc.ainv, bc.width) > bc.umax ? 2u : 0u);
    }
    AHEAD_DEV void emit(int c, uint64_t pos, uint64_t, uint64_t row) const {
        if (c == 0) {
            if (pos < ecap1) e1[pos] = row * aoid;
        } else if (pos < ecap2) {
            e2[pos] = row * aoid;
        }
    }
};

// aggregate_mul_sumAN without the compaction when errors are rare: one pass
// reads both columns with 16-byte loads (8 rows a thread a step), sums the
// code products and appends the rows of corrupt codes to two small lists
// (counts in cnt[0..1], the sum in cnt[2]); a second kernel sorts each list
// (ascending rows, as the reference's loop pushes them) into the error
// vectors.  More than kFastErrCap errors in either column: the caller runs
// the compaction instead.
constexpr uint32_t kFastErrCap = 4096;

template <int W>
AHEAD_DEV void load8(const char* p, uint64_t chunk, uint64_t (&v)[8]) {
    const uint4* q = reinterpret_cast<const uint4*>(p + chunk * 8 * W);
#pragma unroll
    for (int k = 0; k < W / 2; ++k) {
        uint64_t u[16 / W];
        unpack16<W>(__ldg(q + k), u);
#pragma unroll
        for (int j = 0; j < 16 / W; ++j) v[k * (16 / W) + j] = u[j];
    }
}

template <int W1, int W2>
__global__ void __launch_bounds__(256) mulsum_fast_kernel(const char* a, const char* b, uint64_t n, uint64_t ainv1,
                                                          uint64_t umax1, uint64_t ainv2, uint64_t umax2,
                                                          unsigned long long* cnt, uint64_t* rows1, uint64_t* rows2) {
    uint64_t s = 0;
    const uint64_t nch = n / 8, stride = (uint64_t)gridDim.x * blockDim.x;
    auto row = [&](uint64_t r, uint64_t x, uint64_t y) {
        s += x * y;
        if (mulw(x, ainv1, W1) > umax1) {
            const unsigned long long k = atomicAdd(&cnt[0], 1ull);
            if (k < kFastErrCap) rows1[k] = r;
        }
        if (mulw(y, ainv2, W2) > umax2) {
            const unsigned long long k = atomicAdd(&cnt[1], 1ull);
            if (k < kFastErrCap) rows2[k] = r;
        }
    };
    uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    for (; c + stride < nch; c += 2 * stride) {  // two chunks' loads in flight
        uint64_t x0[8], y0[8], x1[8], y1[8];
        load8<W1>(a, c, x0);
        load8<W2>(b, c, y0);
        load8<W1>(a, c + stride, x1);
        load8<W2>(b, c + stride, y1);
#pragma unroll
        for (int q = 0; q < 8; ++q) row(8 * c + q, x0[q], y0[q]);
#pragma unroll
        for (int q = 0; q < 8; ++q) row(8 * (c + stride) + q, x1[q], y1[q]);
    }
    if (c < nch) {
        uint64_t x0[8], y0[8];
        load8<W1>(a, c, x0);
        load8<W2>(b, c, y0);
#pragma unroll
        for (int q = 0; q < 8; ++q) row(8 * c + q, x0[q], y0[q]);
    }
    if (blockIdx.x == 0 && threadIdx.x < n % 8) {
        const uint64_t r = 8 * nch + threadIdx.x;
        row(r, gmem_ld<W1>(a, r), gmem_ld<W2>(b, r));
    }
    s = warp_sum64(s);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(&cnt[2], (unsigned long long)s);
}

// checkAN the same way: one pass of 16-byte loads (two in flight per
// thread), corrupt rows appended to one list (count in cnt[0]).
template <int W>
__global__ void __launch_bounds__(256) check_fast_kernel(const char* a, uint64_t n, uint64_t ainv, uint64_t umax,
                                                         unsigned long long* cnt, uint64_t* rows) {
    constexpr int R = 16 / W;  // rows per 16-byte load
    const uint64_t nv = n / R, stride = (uint64_t)gridDim.x * blockDim.x;
    const uint4* p = reinterpret_cast<const uint4*>(a);
    auto check = [&](uint64_t r, uint64_t x) {
        if (mulw(x, ainv, W) > umax) {
            const unsigned long long k = atomicAdd(&cnt[0], 1ull);
            if (k < kFastErrCap) rows[k] = r;
        }
    };
    uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    for (; c + stride < nv; c += 2 * stride) {
        uint64_t x0[R], x1[R];
        unpack16<W>(__ldg(p + c), x0);
        unpack16<W>(__ldg(p + c + stride), x1);
#pragma unroll
        for (int q = 0; q < R; ++q) check(R * c + q, x0[q]);
#pragma unroll
        for (int q = 0; q < R; ++q) check(R * (c + stride) + q, x1[q]);
    }
    if (c < nv) {
        uint64_t x0[R];
        unpack16<W>(__ldg(p + c), x0);
#pragma unroll
        for (int q = 0; q < R; ++q) check(R * c + q, x0[q]);
    }
    if (blockIdx.x == 0 && threadIdx.x < n % R) check(R * nv + threadIdx.x, gmem_ld<W>(a, R * nv + threadIdx.x));
}

// Block c sorts list c (at most kFastErrCap rows, bitonic in shared memory)
// and writes row * aoid into the error vector, up to its capacity; block 0
// also writes its sorted rows to `sorted` when given.
__global__ void __launch_bounds__(1024) sort_err_rows_kernel(const unsigned long long* cnt, const uint64_t* rows1,
                                                             const uint64_t* rows2, uint64_t* e1, uint64_t cap1,
                                                             uint64_t* e2, uint64_t cap2, uint64_t aoid,
                                                             uint64_t* sorted = nullptr) {
    __shared__ uint64_t s_r[kFastErrCap];
    const int c = blockIdx.x;
    const unsigned long long k = cnt[c];
    uint64_t* e = c == 0 ? e1 : e2;
    const uint64_t cap = c == 0 ? cap1 : cap2;
    if (k == 0 || k > kFastErrCap) return;
    const uint64_t* rows = c == 0 ? rows1 : rows2;
    uint32_t m = 1;
    while (m < k) m <<= 1;
    for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) s_r[i] = i < k ? rows[i] : ~0ull;
    __syncthreads();
    for (uint32_t size = 2; size <= m; size <<= 1)
        for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
            for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
                const uint32_t j = i ^ stride;
                if (j > i) {
                    const bool up = (i & size) == 0;
                    const uint64_t x = s_r[i], y = s_r[j];
                    if ((x > y) == up) {
                        s_r[i] = y;
                        s_r[j] = x;
                    }
                }
            }
            __syncthreads();
        }
    if (e)
        for (uint32_t i = threadIdx.x; i < k && i < cap; i += blockDim.x) e[i] = s_r[i] * aoid;
    if (sorted && c == 0)
        for (uint32_t i = threadIdx.x; i < k; i += blockDim.x) sorted[i] = s_r[i];
}

// checkAndDecodeAN of a void-head column once its corrupt rows are known:
// `err_rows` holds them in ascending order (k = *cnt of them, k <=
// kFastErrCap).  A clean row r goes to output position r - (corrupt rows
// below r).  Blocks walk chunks of U x 256 16-byte input vectors.  A chunk
// without a corrupt row (nearly all) shifts every row by the same count: its
// decoded values are staged in shared memory at the byte alignment of their
// destination and written out as aligned 16-byte stores (only the chunk's two
// edge words byte by byte).  A chunk with corrupt rows places each clean row
// by counting the few list entries inside the chunk.
template <int W>
__global__ void __launch_bounds__(256) decode_shift_kernel(const char* a, uint64_t n, uint64_t ainv, uint64_t umax,
                                                           const unsigned long long* cnt, const uint64_t* err_rows,
                                                           void* out, int ow, uint64_t cap) {
    constexpr int R = 16 / W;
    constexpr int U = W == 4 ? 8 : 4;  // (8 vectors of 2- or 8-byte codes cost registers or spills)
    __shared__ __align__(16) uint8_t s_o[U * 256 * 16 + 16];
    const unsigned long long k = *cnt;
    if (k > kFastErrCap) return;  // the caller runs the compaction instead
    auto below = [&](uint32_t lo, uint32_t hi, uint64_t r) {  // list entries < r in [lo, hi)
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (__ldg(err_rows + mid) < r) lo = mid + 1;
            else hi = mid;
        }
        return lo;
    };
    const uint4* p = reinterpret_cast<const uint4*>(a);
    char* o = reinterpret_cast<char*>(out);
    const uint64_t nv = n / R, chunk = (uint64_t)blockDim.x * U;
    for (uint64_t c0 = (uint64_t)blockIdx.x * chunk; c0 < nv; c0 += (uint64_t)gridDim.x * chunk) {
        const uint64_t c1 = min(c0 + chunk, nv);
        // the whole block searches the same entries (cached broadcast reads)
        const uint32_t lo = below(0, (uint32_t)k, c0 * R);
        const uint32_t hi = below(lo, (uint32_t)k, c1 * R);
        uint4 raw[U];  // 16-byte vectors, unpacked where used (registers)
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint64_t v = c0 + (uint64_t)u * blockDim.x + threadIdx.x;
            raw[u] = v < c1 ? __ldg(p + v) : make_uint4(0, 0, 0, 0);
        }
        if (lo == hi) {
            const uint64_t first = c0 * R - lo;                   // output position of the chunk's row 0
            const uint64_t last = min(c1 * R - lo, cap);          // one past its last stored position
            if (first >= last) continue;                          // block-uniform
            const uint64_t dst = (uint64_t)(uintptr_t)(o + first * ow);
            const uint32_t mis = (uint32_t)(dst & 15);
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const uint64_t v = c0 + (uint64_t)u * blockDim.x + threadIdx.x;
                if (v >= c1) continue;
                uint64_t x[R];
                unpack16<W>(raw[u], x);
#pragma unroll
                for (int q = 0; q < R; ++q) {
                    const uint32_t e = (uint32_t)((v - c0) * R + q);
                    store_at(s_o + mis, ow, e, mulw(x[q], ainv, W));
                }
            }
            __syncthreads();
            const uint32_t total = mis + (uint32_t)((last - first) * ow);
            const uint32_t words = (total + 15) / 16;
            char* g = reinterpret_cast<char*>(dst - mis);
            for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) {
                const uint32_t b0 = i * 16, b1 = b0 + 16;
                if (b0 >= mis && b1 <= total) {
                    *reinterpret_cast<uint4*>(g + b0) = *reinterpret_cast<const uint4*>(s_o + b0);
                } else {
                    for (uint32_t j = max(b0, mis); j < min(b1, total); ++j) g[j] = (char)s_o[j];
                }
            }
            __syncthreads();  // the next chunk reuses s_o
        } else {
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const uint64_t v = c0 + (uint64_t)u * blockDim.x + threadIdx.x;
                if (v >= c1) continue;
                uint64_t x[R];
                unpack16<W>(raw[u], x);
#pragma unroll
                for (int q = 0; q < R; ++q) {
                    const uint64_t r = v * R + q;
                    const uint64_t d = mulw(x[q], ainv, W);
                    if (d > umax) continue;
                    const uint64_t pos = r - below(lo, hi, r);
                    if (pos < cap) store_at(out, ow, pos, d);
                }
            }
        }
    }
    if (blockIdx.x == 0 && threadIdx.x < n % R) {  // rows past the last whole vector
        const uint64_t r = nv * R + threadIdx.x;
        const uint64_t d = mulw(gmem_ld<W>(a, r), ainv, W);
        if (d <= umax) {
            const uint64_t pos = r - below(0, (uint32_t)k, r);
            if (pos < cap) store_at(out, ow, pos, d);
        }
    }
}

__global__ void mul_sum_plain_kernel(DCol a, DCol b, uint64_t n, unsigned long long* out) {
    uint64_t s = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        s += load_at(a, i) * load_at(b, i);
    s = warp_sum64(s);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(out, (unsigned long long)s);
}

// ------------------------------------------------------------ arithmetic
// arithmeticAN (arithmeticAN_scalar.tcc:87-107).
template <int WW>
struct ArithOp {
    static constexpr int W = WW;
    static constexpr int NCH = 2;
    static constexpr bool ACC = false;
    const char* base;
    uint32_t* status;
    DCol ac, bc;
    uint64_t ar, aoid, ecap1, ecap2;
    uint64_t *e1, *e2;
    void* out;
    int ow, op;
    uint64_t* acc;
    static constexpr bool EMIT_V = false;
    static constexpr int NOUT = 1;
    AHEAD_DEV uint64_t out0(int, uint64_t, uint64_t row) const { return row * aoid; }
    AHEAD_DEV void put0(int, uint64_t pos, uint64_t val) const {
        if (pos < ecap1) e1[pos] = val;
    }
    AHEAD_DEV uint32_t eval(uint64_t a, uint64_t row, uint64_t&) const {
        const uint64_t t1 = mulw(a, ac.ainv, W), t2 = mulw(load_at(bc, row), bc.ainv, bc.width);
        const uint64_t x = t1 * ar, y = t2 * ar;
        uint64_t v;
        switch (op) {
            case AHEAD_ADD: v = x + y; break;
            case AHEAD_SUB: v = x - y; break;
            case AHEAD_MUL: v = x * y; break;
            default: v = y ? x / y : 0; break;
        }
        store_at(out, ow, row, v);
        return (t1 > ac.umax ? 1u : 0u) | (t2 > bc.umax ? 2u : 0u);
    }
    AHEAD_DEV void emit(int c, uint64_t pos, uint64_t, uint64_t row) const {
        if (c == 0) {
            if (pos < ecap1) e1[pos] = row * aoid;
        } else if (pos < ecap2) {
            e2[pos] = row * aoid;
        }
    }
};

__global__ void encode_kernel(DCol in, void* out, int ow, uint64_t A, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        store_at(out, ow, i, mulw(load_at(in, i), A, ow));
}

}  // namespace

namespace ahead {
int restiny_promoted_check(ahead_ctx* ctx, const uint16_t* codes, uint64_t n, uint32_t ainv, uint32_t umax,
                           uint64_t aoid, ahead_errvec* err) {
    typedef SelectOp<1, true> Op;
    ev_begin(err, 1);
    OpScope s(ctx);
    int rc = s.reserve(compact_scratch<Op>(n) + n + 256);
    if (rc) return rc;
    uint8_t* flags = (uint8_t*)s.alloc(n);
    if (n) {
        const uint64_t want = (n + 255) / 256;
        const unsigned grid = (unsigned)(want < (uint64_t)ctx->num_sms * 8 ? want : (uint64_t)ctx->num_sms * 8);
        promoted_check_kernel<<<grid, 256, 0, ctx->stream>>>(codes, n, ainv, (int32_t)umax, flags);
        s.launched();
    }
    Op op;
    op.base = (const char*)flags;
    op.status = s.d_status;
    op.seqbase = 0;
    op.ainv = 1;
    op.umax = 0;  // every set flag is an error row
    op.aoid = aoid;
    op.cap = 0;   // no selected rows are written
    op.out_an = nullptr;
    op.out_oid = nullptr;
    op.err = err ? err->data : nullptr;
    op.errcap = (err && err->data) ? err->capacity : 0;
    op.acc = nullptr;
    op.pred = RangePred::make(AHEAD_CMP_EQ, 2, AHEAD_CMP_NONE, 0, AHEAD_AND, wmask(1));  // never holds
    run_compact<Op>(s, op, n, 0);
    rc = s.finish(Op::NCH);
    if (rc) return rc;
    if (err) err->count = s.counter(1);
    return AHEAD_OK;
}
}  // namespace ahead

extern "C" {

int ahead_gpu_select_an(ahead_ctx* ctx, const ahead_bat* in, int op1, uint64_t th1, int op2, uint64_t th2, int comb,
                        uint64_t aoid, ahead_bat* out, uint64_t cap, ahead_errvec* err) {
    if (!ctx || !in || !out) return AHEAD_BAD_ARG;
    const int t = in->tail.type;
    if (in->head.type != AHEAD_VOID || !(t == AHEAD_RESTINY || t == AHEAD_RESSHORT || t == AHEAD_RESINT))
        return fail(ctx, AHEAD_BAD_ARG, "selectAN: void head and restiny/resshort/resint tail required");
    if (!op_ok(op1) || (op2 != AHEAD_CMP_NONE && !op_ok(op2))) return fail(ctx, AHEAD_BAD_ARG, "selectAN: bad predicate");
    const int w = type_width(t);
    set_meta(&out->head, AHEAD_RESOID, kResoidAMax, kResoidAInvMax, kRes56Max, 0);
    copy_meta(&out->tail, t, &in->tail);
    out->tail.data = nullptr;  // the reference fills only the head (selectAN_scalar.tcc:89-91)
    ev_begin(err, 1);
    out->count = 0;
    OpScope s(ctx);
    RangePred p = make_pred(op1, th1, op2, th2, comb, w);
    switch (w) {
        case 2: return run_select<2, true>(s, in, p, aoid, out, cap, err);
        case 4: return run_select<4, true>(s, in, p, aoid, out, cap, err);
        default: return run_select<8, true>(s, in, p, aoid, out, cap, err);
    }
}

int ahead_gpu_select_str_an(ahead_ctx* ctx, const char* strs, uint64_t width, uint64_t count, uint64_t seqbase,
                            int op1, const char* th1, int op2, const char* th2, int comb, ahead_bat* out,
                            uint64_t cap) {
    if (!ctx) return AHEAD_BAD_ARG;
    StrPred sp;
    int rc = select_str_args(ctx, strs, width, count, op1, th1, op2, th2, comb, out, &sp,
                             "selectAN(str): bad argument");
    if (rc) return rc;
    set_meta(&out->head, AHEAD_RESOID, kResoidAMax, kResoidAInvMax, kRes56Max, 0);
    set_meta(&out->tail, AHEAD_STR, 0, 0, 0, 0);
    out->tail.data = nullptr;  // only the head is filled (selectAN_scalar.tcc:124-126)
    out->count = 0;
    return run_select_str<true>(ctx, strs, width, count, seqbase, sp, out, cap);
}

int ahead_gpu_select_str(ahead_ctx* ctx, const char* strs, uint64_t width, uint64_t count, uint64_t seqbase,
                         int op1, const char* th1, int op2, const char* th2, int comb, ahead_bat* out,
                         uint64_t cap) {
    if (!ctx) return AHEAD_BAD_ARG;
    StrPred sp;
    int rc = select_str_args(ctx, strs, width, count, op1, th1, op2, th2, comb, out, &sp,
                             "select(str): bad argument");
    if (rc) return rc;
    set_meta(&out->head, AHEAD_OID, 0, 0, 0, 0);
    set_meta(&out->tail, AHEAD_STR, 0, 0, 0, 0);
    out->tail.data = nullptr;  // only the head is filled (Normal/select_scalar.tcc:93-95)
    out->count = 0;
    return run_select_str<false>(ctx, strs, width, count, seqbase, sp, out, cap);
}

int ahead_gpu_select(ahead_ctx* ctx, const ahead_bat* in, int op1, uint64_t th1, int op2, uint64_t th2, int comb,
                     ahead_bat* out, uint64_t cap) {
    if (!ctx || !in || !out) return AHEAD_BAD_ARG;
    const int t = in->tail.type;
    if (in->head.type != AHEAD_VOID || t == AHEAD_VOID || t == AHEAD_OID || t == AHEAD_RESOID)
        return fail(ctx, AHEAD_BAD_ARG, "select: void head and a value tail required");
    if (!op_ok(op1) || (op2 != AHEAD_CMP_NONE && !op_ok(op2))) return fail(ctx, AHEAD_BAD_ARG, "select: bad predicate");
    const int w = type_width(t);
    copy_meta(&out->head, AHEAD_OID, &in->head);
    copy_meta(&out->tail, t, &in->tail);
    out->tail.data = nullptr;  // only the head is filled (Normal/select_scalar.tcc:66-72)
    out->count = 0;
    OpScope s(ctx);
    RangePred p = make_pred(op1, th1, op2, th2, comb, w);
    return by_width(w, [&](auto tag) -> int {
        return run_select<decltype(tag)::value, false>(s, in, p, 0, out, cap, nullptr);
    });
}

int ahead_gpu_check_an(ahead_ctx* ctx, const ahead_bat* in, uint64_t ainv, uint64_t unenc_max, uint64_t aoid,
                       ahead_errvec* err) {
    if (!ctx || !in) return AHEAD_BAD_ARG;
    const int t = in->tail.type;
    if (!(in->head.type == AHEAD_VOID || in->head.type == AHEAD_OID) || !type_encoded(t))
        return fail(ctx, AHEAD_BAD_ARG, "checkAN: unencoded head and AN tail required");
    ev_begin(err, 1);
    OpScope s(ctx);
    // rare errors: one pass, then a sort of the few error rows
    if (((uintptr_t)in->tail.data % 16) == 0 && in->count) {
        int rc = s.reserve((size_t)kFastErrCap * 8 + 1024);
        if (rc) return rc;
        uint64_t* rows = (uint64_t*)s.alloc((size_t)kFastErrCap * 8);
        unsigned long long* cnt = (unsigned long long*)s.d_counters;
        const int w = type_width(t);
        by_width_enc(w, [&](auto tag) -> int {
            constexpr int W = decltype(tag)::value;
            check_fast_kernel<W><<<ctx->num_sms * 8, 256, 0, ctx->stream>>>(
                (const char*)in->tail.data, in->count, ainv & wmask(W), unenc_max & wmask(W), cnt, rows);
            return 0;
        });
        sort_err_rows_kernel<<<1, 1024, 0, ctx->stream>>>(cnt, rows, nullptr, edata(err), ecap(err), nullptr, 0, aoid);
        s.launched(2);
        rc = s.finish(1);
        if (rc) return rc;
        if (s.counter(0) <= kFastErrCap) {
            if (err) err->count = s.counter(0);
            return AHEAD_OK;
        }
    }
    return by_width_enc(type_width(t), [&](auto tag) -> int {
        constexpr int W = decltype(tag)::value;
        typedef CheckOp<W> Op;
        int rc = s.reserve(compact_scratch<Op>(in->count));
        if (rc) return rc;
        Op op;
        op.base = (const char*)in->tail.data;
        op.status = s.d_status;
        op.ainv = ainv & wmask(W);
        op.umax = unenc_max & wmask(W);
        op.aoid = aoid;
        op.err = edata(err);
        op.errcap = ecap(err);
        op.acc = nullptr;
        run_compact<Op>(s, op, in->count, 0);
        rc = s.finish(1);
        if (rc) return rc;
        if (err) err->count = s.counter(0);
        return AHEAD_OK;
    });
}

int ahead_gpu_decode_an(ahead_ctx* ctx, const ahead_bat* in, uint64_t aoid, ahead_bat* out, uint64_t cap,
                        ahead_errvec* err) {
    if (!ctx || !in || !out) return AHEAD_BAD_ARG;
    const int h = in->head.type, t = in->tail.type;
    if (h != AHEAD_RESOID || !type_encoded(t)) return fail(ctx, AHEAD_BAD_ARG, "decodeAN: resoid head and AN tail required");
    const int ut = type_unenc_of(t);
    copy_meta(&out->head, h, &in->head);
    default_meta(&out->tail, ut);
    ev_begin(err, 1);
    out->count = in->count;
    if (in->count > cap) return AHEAD_CAPACITY;
    OpScope s(ctx);
    return by_width_enc(type_width(t), [&](auto tag) -> int {
        constexpr int W = decltype(tag)::value;
        typedef DecodeOp<W> Op;
        int rc = s.reserve(compact_scratch<Op>(in->count));
        if (rc) return rc;
        Op op;
        op.base = (const char*)in->tail.data;
        op.status = s.d_status;
        op.hc = dcol(in->head);
        op.tc = dcol(in->tail);
        op.oh = out->head.data;
        op.ot = out->tail.data;
        op.ohw = type_width(h);
        op.otw = type_width(ut);
        op.aoid = aoid;
        op.err = edata(err);
        op.errcap = ecap(err);
        op.acc = nullptr;
        run_compact<Op>(s, op, in->count, 0);
        rc = s.finish(1);
        if (rc) return rc;
        if (err) err->count = s.counter(0);
        return AHEAD_OK;
    });
}

int ahead_gpu_check_and_decode_an(ahead_ctx* ctx, const ahead_bat* in, uint64_t aoid, ahead_bat* out, uint64_t cap,
                                  ahead_errvec* err_head, ahead_errvec* err_tail) {
    if (!ctx || !in || !out) return AHEAD_BAD_ARG;
    const int h = in->head.type, t = in->tail.type;
    if (!(h == AHEAD_VOID || h == AHEAD_OID || h == AHEAD_RESOID) || !type_encoded(t))
        return fail(ctx, AHEAD_BAD_ARG, "checkAndDecodeAN: void/oid/resoid head and AN tail required");
    const int ut = type_unenc_of(t), uh = type_unenc_of(h);
    out->count = 0;
    OpScope s(ctx);
    if (h == AHEAD_VOID) {
        ev_begin(err_head, 0);
        ev_begin(err_tail, 1);
        default_meta(&out->head, AHEAD_VOID);
        default_meta(&out->tail, ut);
        // rare errors: the corrupt rows first (one pass), then one decode pass
        // that shifts each clean row down by the corrupt rows before it
        if (((uintptr_t)in->tail.data % 16) == 0 && in->count) {
            int rc = s.reserve((size_t)kFastErrCap * 16 + 1024);
            if (rc) return rc;
            uint64_t* rows = (uint64_t*)s.alloc((size_t)kFastErrCap * 8);
            uint64_t* sorted = (uint64_t*)s.alloc((size_t)kFastErrCap * 8);
            unsigned long long* cnt = (unsigned long long*)s.d_counters;
            by_width_enc(type_width(t), [&](auto tag) -> int {
                constexpr int W = decltype(tag)::value;
                const uint64_t ainv = in->tail.Ainv & wmask(W), umax = in->tail.unenc_max & wmask(W);
                check_fast_kernel<W><<<ctx->num_sms * 8, 256, 0, ctx->stream>>>((const char*)in->tail.data,
                                                                                in->count, ainv, umax, cnt, rows);
                sort_err_rows_kernel<<<1, 1024, 0, ctx->stream>>>(cnt, rows, nullptr, edata(err_tail),
                                                                   ecap(err_tail), nullptr, 0, aoid, sorted);
                decode_shift_kernel<W><<<ctx->num_sms * 8, 256, 0, ctx->stream>>>(
                    (const char*)in->tail.data, in->count, ainv, umax, cnt, sorted, out->tail.data,
                    type_width(ut), out->tail.data ? cap : 0);
                return 0;
            });
            s.launched(3);
            rc = s.finish(1);
            if (rc) return rc;
            const uint64_t k = s.counter(0);
            if (k <= kFastErrCap) {
                out->count = in->count - k;
                if (err_tail) err_tail->count = k;
                return out->count > cap ? AHEAD_CAPACITY : AHEAD_OK;
            }
        }
        return by_width_enc(type_width(t), [&](auto tag) -> int {
            constexpr int W = decltype(tag)::value;
            typedef CadVoidOp<W> Op;
            int rc = s.reserve(compact_scratch<Op>(in->count));
            if (rc) return rc;
            Op op;
            op.base = (const char*)in->tail.data;
            op.status = s.d_status;
            op.out = out->tail.data;
            op.ow = type_width(ut);
            op.ainv = in->tail.Ainv & wmask(W);
            op.umax = in->tail.unenc_max & wmask(W);
            op.aoid = aoid;
            op.cap = out->tail.data ? cap : 0;
            op.err = edata(err_tail);
            op.errcap = ecap(err_tail);
            op.acc = nullptr;
            run_compact<Op>(s, op, in->count, 0);
            rc = s.finish(2);
            if (rc) return rc;
            out->count = s.counter(0);
            if (err_tail) err_tail->count = s.counter(1);
            return out->count > cap ? AHEAD_CAPACITY : AHEAD_OK;
        });
    }
    ev_begin(err_head, type_encoded(h));
    ev_begin(err_tail, 1);
    default_meta(&out->head, uh);
    default_meta(&out->tail, ut);
    return by_width_enc(type_width(t), [&](auto tag) -> int {
        constexpr int W = decltype(tag)::value;
        typedef CadGenOp<W> Op;
        int rc = s.reserve(compact_scratch<Op>(in->count));
        if (rc) return rc;
        Op op;
        op.base = (const char*)in->tail.data;
        op.status = s.d_status;
        op.hc = dcol(in->head);
        op.tc = dcol(in->tail);
        op.oh = out->head.data;
        op.ot = out->tail.data;
        op.ohw = type_width(uh);
        op.otw = type_width(ut);
        op.aoid = aoid;
        op.cap = (out->head.data && out->tail.data) ? cap : 0;
        op.err_h = edata(err_head);
        op.err_t = edata(err_tail);
        op.ecap_h = ecap(err_head);
        op.ecap_t = ecap(err_tail);
        op.acc = nullptr;
        run_compact<Op>(s, op, in->count, 0);
        rc = s.finish(3);
        if (rc) return rc;
        out->count = s.counter(0);
        if (err_head) err_head->count = type_encoded(h) ? s.counter(1) : 0;
        if (err_tail) err_tail->count = s.counter(2);
        return out->count > cap ? AHEAD_CAPACITY : AHEAD_OK;
    });
}

int ahead_gpu_encode_an(ahead_ctx* ctx, const ahead_bat* in, uint64_t A, ahead_bat* out, uint64_t cap) {
    if (!ctx || !in || !out) return AHEAD_BAD_ARG;
    const int t = in->tail.type;
    if (in->head.type != AHEAD_VOID || !(t == AHEAD_TINYINT || t == AHEAD_SHORTINT || t == AHEAD_INT))
        return fail(ctx, AHEAD_BAD_ARG, "encodeAN: void head and tinyint/shortint/int tail required");
    const int et = type_encoded_of(t), w = type_width(et);
    copy_meta(&out->head, AHEAD_VOID, &in->head);
    set_meta(&out->tail, et, A, inv_pow2(A, 8 * w), type_unenc_max(et), 0);
    out->count = in->count;
    if (in->count > cap) return AHEAD_CAPACITY;
    OpScope s(ctx);
    int rc = s.reserve(0);
    if (rc) return rc;
    if (in->count) {
        encode_kernel<<<grid_for(in->count, 256), 256, 0, ctx->stream>>>(dcol(in->tail), out->tail.data, w, A,
                                                                          in->count);
        s.launched();
    }
    return s.finish(0);
}

int ahead_gpu_aggregate_mul_sum_an(ahead_ctx* ctx, const ahead_bat* a, const ahead_bat* b, int result_type,
                                   uint64_t init, uint64_t ra, uint64_t rainv, uint64_t aoid, uint64_t* total,
                                   ahead_errvec* errs) {
    (void)rainv;
    if (!ctx || !a || !b || !total) return AHEAD_BAD_ARG;
    const int T1 = a->tail.type, T2 = b->tail.type;
    if (result_type != AHEAD_RESBIGINT) return fail(ctx, AHEAD_BAD_ARG, "aggregate_mul_sumAN: resbigint result only");
    if (!(a->head.type == AHEAD_VOID || a->head.type == AHEAD_RESOID) ||
        !(b->head.type == AHEAD_VOID || b->head.type == AHEAD_RESOID))
        return fail(ctx, AHEAD_BAD_ARG, "aggregate_mul_sumAN: void/resoid heads required");
    if (!(T1 == AHEAD_RESTINY || T1 == AHEAD_RESSHORT || T1 == AHEAD_RESINT) ||
        !(T2 == AHEAD_RESTINY || T2 == AHEAD_RESSHORT || T2 == AHEAD_RESINT))
        return fail(ctx, AHEAD_BAD_ARG, "aggregate_mul_sumAN: restiny/resshort/resint tails required");
    ahead_errvec *e1 = errs ? &errs[0] : nullptr, *e2 = errs ? &errs[1] : nullptr;
    ev_begin(e1, 1);
    ev_begin(e2, 1);
    const uint64_t n = a->count < b->count ? a->count : b->count;
    const uint64_t enc = ra * inv_pow2(a->tail.A & wmask(type_width(T1)), 64) *
                         inv_pow2(b->tail.A & wmask(type_width(T2)), 64);
    OpScope s(ctx);
    // rare errors: one pass, then a sort of the few error rows
    const bool aligned = ((uintptr_t)a->tail.data % 16) == 0 && ((uintptr_t)b->tail.data % 16) == 0;
    if (aligned && n >= 8) {
        int rc = s.reserve(2 * (size_t)kFastErrCap * 8 + 1024);
        if (rc) return rc;
        uint64_t* rows1 = (uint64_t*)s.alloc((size_t)kFastErrCap * 8);
        uint64_t* rows2 = (uint64_t*)s.alloc((size_t)kFastErrCap * 8);
        const DCol ac = dcol(a->tail), bc = dcol(b->tail);
        unsigned long long* cnt = (unsigned long long*)s.d_counters;
        rc = by_width_enc(ac.width, [&](auto t1) -> int {
            return by_width_enc(bc.width, [&](auto t2) -> int {
                constexpr int W1 = decltype(t1)::value, W2 = decltype(t2)::value;
                mulsum_fast_kernel<W1, W2><<<ctx->num_sms * 8, 256, 0, ctx->stream>>>(
                    (const char*)a->tail.data, (const char*)b->tail.data, n, ac.ainv, ac.umax, bc.ainv, bc.umax,
                    cnt, rows1, rows2);
                return 0;
            });
        });
        sort_err_rows_kernel<<<2, 1024, 0, ctx->stream>>>(cnt, rows1, rows2, edata(e1), ecap(e1), edata(e2), ecap(e2),
                                                          aoid);
        s.launched(2);
        rc = s.finish(3);
        if (rc) return rc;
        if (s.counter(0) <= kFastErrCap && s.counter(1) <= kFastErrCap) {
            if (e1) e1->count = s.counter(0);
            if (e2) e2->count = s.counter(1);
            *total = (init + s.counter(2)) * enc;
            return AHEAD_OK;
        }
    }
    return by_width_enc(type_width(T1), [&](auto tag) -> int {
        constexpr int W = decltype(tag)::value;
        typedef MulSumOp<W> Op;
        int rc = s.reserve(compact_scratch<Op>(n));
        if (rc) return rc;
        Op op;
        op.base = (const char*)a->tail.data;
        op.status = s.d_status;
        op.ac = dcol(a->tail);
        op.bc = dcol(b->tail);
        op.aoid = aoid;
        op.e1 = edata(e1);
        op.e2 = edata(e2);
        op.ecap1 = ecap(e1);
        op.ecap2 = ecap(e2);
        op.acc = s.d_counters + 2;
        run_compact<Op>(s, op, n, 0);
        rc = s.finish(3);
        if (rc) return rc;
        if (e1) e1->count = s.counter(0);
        if (e2) e2->count = s.counter(1);
        *total = (init + s.counter(2)) * enc;
        return AHEAD_OK;
    });
}

int ahead_gpu_aggregate_mul_sum(ahead_ctx* ctx, const ahead_bat* a, const ahead_bat* b, int result_type,
                                uint64_t init, uint64_t* total) {
    if (!ctx || !a || !b || !total) return AHEAD_BAD_ARG;
    if (result_type != AHEAD_BIGINT) return fail(ctx, AHEAD_BAD_ARG, "aggregate_mul_sum: bigint result only");
    if (a->tail.type == AHEAD_VOID || b->tail.type == AHEAD_VOID) return fail(ctx, AHEAD_BAD_ARG, "aggregate_mul_sum: value tails required");
    const uint64_t n = a->count < b->count ? a->count : b->count;
    OpScope s(ctx);
    int rc = s.reserve(0);
    if (rc) return rc;
    if (n) {
        mul_sum_plain_kernel<<<grid_for(n, 256), 256, 0, ctx->stream>>>(dcol(a->tail), dcol(b->tail), n,
                                                                        (unsigned long long*)s.d_counters);
        s.launched();
    }
    rc = s.finish(1);
    if (rc) return rc;
    *total = init + s.counter(0);
    return AHEAD_OK;
}

int ahead_gpu_arithmetic_an(ahead_ctx* ctx, int op, int result_type, const ahead_bat* a, const ahead_bat* b,
                            uint64_t ar, uint64_t arinv, uint64_t aoid, ahead_bat* out, ahead_errvec* errs) {
    if (!ctx || !a || !b || !out) return AHEAD_BAD_ARG;
    const int T1 = a->tail.type, T2 = b->tail.type;
    if (!(result_type == AHEAD_RESINT || result_type == AHEAD_RESBIGINT)) return fail(ctx, AHEAD_BAD_ARG, "arithmeticAN: resint/resbigint result");
    if (a->head.type != AHEAD_VOID || b->head.type != AHEAD_VOID) return fail(ctx, AHEAD_BAD_ARG, "arithmeticAN: void heads");
    if (!(T1 == AHEAD_RESTINY || T1 == AHEAD_RESSHORT || T1 == AHEAD_RESINT) ||
        !(T2 == AHEAD_RESTINY || T2 == AHEAD_RESSHORT || T2 == AHEAD_RESINT))
        return fail(ctx, AHEAD_BAD_ARG, "arithmeticAN: restiny/resshort/resint tails");
    if (op < AHEAD_ADD || op > AHEAD_DIV) return fail(ctx, AHEAD_BAD_ARG, "arithmeticAN: bad operator");
    if (a->count != b->count) return fail(ctx, AHEAD_SIZE_MISMATCH, "arithmetic: bat1->size() != bat2->size()");
    ahead_errvec* e = errs;
    ev_begin(e ? &e[0] : nullptr, 0);
    ev_begin(e ? &e[1] : nullptr, 1);
    ev_begin(e ? &e[2] : nullptr, 0);
    ev_begin(e ? &e[3] : nullptr, 1);
    default_meta(&out->head, AHEAD_VOID);
    set_meta(&out->tail, result_type, ar, arinv, type_unenc_max(result_type), 0);
    out->count = a->count;
    OpScope s(ctx);
    return by_width_enc(type_width(T1), [&](auto tag) -> int {
        constexpr int W = decltype(tag)::value;
        typedef ArithOp<W> Op;
        int rc = s.reserve(compact_scratch<Op>(a->count));
        if (rc) return rc;
        Op o;
        o.base = (const char*)a->tail.data;
        o.status = s.d_status;
        o.ac = dcol(a->tail);
        o.bc = dcol(b->tail);
        o.ar = ar;
        o.aoid = aoid;
        o.e1 = edata(e ? &e[1] : nullptr);
        o.e2 = edata(e ? &e[3] : nullptr);
        o.ecap1 = ecap(e ? &e[1] : nullptr);
        o.ecap2 = ecap(e ? &e[3] : nullptr);
        o.out = out->tail.data;
        o.ow = type_width(result_type);
        o.op = op;
        o.acc = nullptr;
        run_compact<Op>(s, o, a->count, 0);
        rc = s.finish(2);
        if (rc) return rc;
        if (e) {
            e[1].count = s.counter(0);
            e[3].count = s.counter(1);
        }
        return AHEAD_OK;
    });
}

}  // extern "C"
