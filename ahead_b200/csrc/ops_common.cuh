// ops_common.cuh -- pieces shared by the operator translation units: width
// dispatch, error-vector plumbing and the column check used for every
// error-position vector that is a plain "decode and compare" over a column.
#pragma once

#include <type_traits>

#include "context.cuh"

namespace ahead {

// Dispatch a functor on the storage width of a column type.
template <class F>
inline int by_width(int w, F&& f) {
    switch (w) {
        case 1: return f(std::integral_constant<int, 1>());
        case 2: return f(std::integral_constant<int, 2>());
        case 4: return f(std::integral_constant<int, 4>());
        default: return f(std::integral_constant<int, 8>());
    }
}

// Same for AN-coded columns, whose codes are 2, 4 or 8 bytes wide.
template <class F>
inline int by_width_enc(int w, F&& f) {
    switch (w) {
        case 2: return f(std::integral_constant<int, 2>());
        case 4: return f(std::integral_constant<int, 4>());
        default: return f(std::integral_constant<int, 8>());
    }
}


inline uint32_t grid_for(uint64_t n, int threads) {
    uint64_t g = (n + threads - 1) / threads;
    return (uint32_t)(g < 148 * 16 ? (g ? g : 1) : 148 * 16);
}

inline uint64_t ecap(const ahead_errvec* e) { return (e && e->data) ? e->capacity : 0; }
inline uint64_t* edata(const ahead_errvec* e) { return e ? e->data : nullptr; }


// checkAN: encdecAN_scalar.tcc:84-90.
template <int WW>
struct CheckOp {
    static constexpr int W = WW;
    static constexpr int NCH = 1;
    static constexpr bool ACC = false;
    const char* base;
    uint32_t* status;
    uint64_t ainv, umax, aoid, errcap;
    uint64_t* err;
    uint64_t* acc;
    static constexpr bool EMIT_V = false;
    static constexpr int NOUT = 1;
    AHEAD_DEV uint32_t eval(uint64_t v, uint64_t, uint64_t&) const {
        return mulw(v, ainv, W) > umax ? 1u : 0u;
    }
    AHEAD_DEV uint64_t out0(int, uint64_t, uint64_t row) const { return row * aoid; }
    AHEAD_DEV void put0(int, uint64_t pos, uint64_t val) const {
        if (pos < errcap) err[pos] = val;
    }
    AHEAD_DEV void emit(int, uint64_t pos, uint64_t, uint64_t row) const {
        if (pos < errcap) err[pos] = row * aoid;
    }
};


// Error positions of one column: rows whose code, multiplied by ainv in the
// `wenc`-byte ring, exceeds umax (the check every AN operator applies to each
// of its encoded inputs, e.g. hashjoinAN.tcc:144-149).  Rows [0, n).
template <int WW>
struct ColCheckOp {
    static constexpr int W = WW;
    static constexpr int NCH = 1;
    static constexpr bool ACC = false;
    static constexpr bool EMIT_V = false;
    static constexpr int NOUT = 1;
    const char* base;
    uint32_t* status;
    uint64_t ainv, umax, aoid, errcap, wmaskenc;
    uint64_t* err;
    uint64_t* acc;
    AHEAD_DEV uint32_t eval(uint64_t v, uint64_t, uint64_t&) const { return ((v * ainv) & wmaskenc) > umax ? 1u : 0u; }
    AHEAD_DEV uint64_t out0(int, uint64_t, uint64_t row) const { return row * aoid; }
    AHEAD_DEV void put0(int, uint64_t pos, uint64_t val) const {
        if (pos < errcap) err[pos] = val;
    }
    AHEAD_DEV void emit(int, uint64_t pos, uint64_t, uint64_t row) const {
        if (pos < errcap) err[pos] = row * aoid;
    }
};

inline size_t colcheck_scratch(uint64_t n) { return n ? compact_bytes(compact_tiles(n), 1) + 1024 : 0; }

// Launch the column check; the error count lands in counter `ci`.
inline void run_colcheck(OpScope& s, const ahead_col& c, uint64_t n, uint64_t ainv, uint64_t umax, int wenc,
                         uint64_t aoid, ahead_errvec* e, int ci) {
    if (!n || !e) return;
    by_width_enc(type_width(c.type), [&](auto tag) -> int {
        constexpr int W = decltype(tag)::value;
        ColCheckOp<W> op;
        op.base = (const char*)c.data;
        op.status = s.d_status;
        op.ainv = ainv;
        op.umax = umax;
        op.aoid = aoid;
        op.errcap = ecap(e);
        op.err = edata(e);
        op.wmaskenc = wmask(wenc);
        op.acc = nullptr;
        run_compact(s, op, n, ci);
        return 0;
    });
}

}  // namespace ahead

namespace ahead {
// ANhelper<V>::mulIfEncoded(x, f) on the host with f = the column's A^-1:
// (storage)(x * A^-1) for an encoded column, (storage)x otherwise.  Used for
// re-encoding factors A_new * A_old^-1 (hashjoinAN.tcc:95-96, matchjoinAN.tcc:80-81).
inline uint64_t dec_if_host(const DCol& c, uint64_t x) { return c.enc ? mulw(x, c.ainv, c.width) : (x & wmask(c.width)); }
}  // namespace ahead
