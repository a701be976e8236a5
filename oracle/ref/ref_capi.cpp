// ref_capi.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Exposes the reference's own scalar AN (and unencoded) operator templates
// through the oracle's C interface (an_oracle.h), so that tests can run the
// reference itself on the same inputs as the GPU library.  This file contains
// no operator logic: it converts ahead_bat descriptors into the reference's
// TempBAT objects, calls the reference template, and copies the result BATs
// and error vectors back out.  It is compiled against the reference sources
// by oracle/Makefile into oracle/_ref/libahead_ref.so.
//
// Operators wrapped (reference paths relative to the reference project):
//   selectAN               lib/column_operators/AN/selectAN.tcc:33-70
//   select (unencoded)     lib/column_operators/Normal/select_scalar.tcc:53-160
//   string selections      selectAN_scalar.tcc:98-131,185-222; Normal/select_scalar.tcc:78-165
//   hashjoinAN (str tail)  lib/column_operators/AN/hashjoinAN.tcc:225-367
//   checkAN/decodeAN       lib/column_operators/AN/encdecAN_scalar.tcc:69-127
//   checkAndDecodeAN       lib/column_operators/AN/encdecAN_scalar.tcc:129-219
//   encodeAN               lib/column_operators/AN/encdecAN_scalar.tcc:43-67
//   hashjoinAN             lib/column_operators/AN/hashjoinAN.tcc:552-585
//   hashjoin (unencoded)   lib/column_operators/Normal/hashjoin.tcc:38-90
//   matchjoinAN/fetchjoin  lib/column_operators/AN/matchjoinAN.tcc:46-354
//   matchjoin/fetchjoin    lib/column_operators/Normal/matchjoin.tcc:37-178
//   groupbyAN              lib/column_operators/AN/groupbyAN.tcc:51-211
//   aggregate_sum_grouped  lib/column_operators/AN/aggregateAN.tcc:35-120
//   aggregate_mul_sumAN    lib/column_operators/AN/aggregateAN_scalar.tcc:56-131
//   aggregate_mul_sum      lib/column_operators/Normal/aggregate_scalar.tcc:69-90
//   arithmeticAN           lib/column_operators/AN/arithmeticAN_scalar.tcc:48-111
//   groupby (unencoded)    lib/column_operators/Normal/groupby.tcc:51-150
//   aggregate_sum_grouped  lib/column_operators/Normal/aggregate.tcc:32-50
//   aggregate_sum          lib/column_operators/Normal/aggregate_scalar.tcc:47-58
//   arithmetic             lib/column_operators/Normal/arithmetic_scalar.tcc:46-82
#include <column_operators/ANbase.hpp>
#include <column_operators/functors.hpp>
#include "column_operators/AN/selectAN.tcc"
#include "column_operators/AN/encdecAN_scalar.tcc"
#include "column_operators/AN/arithmeticAN_scalar.tcc"
#include "column_operators/AN/hashjoinAN.tcc"
#include "column_operators/AN/matchjoinAN.tcc"
#include "column_operators/AN/groupbyAN.tcc"
#include "column_operators/AN/aggregateAN.tcc"
#include "column_operators/Normal/select.tcc"
#include "column_operators/Normal/hashjoin.tcc"
#include "column_operators/Normal/matchjoin.tcc"
#include "column_operators/Normal/aggregate.tcc"
#include "column_operators/Normal/groupby.tcc"
#include "column_operators/Normal/arithmetic_scalar.tcc"

#include <cstring>
#include <functional>
#include <stdexcept>
#include <tuple>
#include <utility>
#include <vector>

#include "../an_oracle.h"

using namespace ahead;
using namespace ahead::bat::ops;

namespace {

template <class V> struct TI;
template <> struct TI<v2_void_t> { static constexpr int id = AHEAD_VOID; };
template <> struct TI<v2_tinyint_t> { static constexpr int id = AHEAD_TINYINT; };
template <> struct TI<v2_shortint_t> { static constexpr int id = AHEAD_SHORTINT; };
template <> struct TI<v2_int_t> { static constexpr int id = AHEAD_INT; };
template <> struct TI<v2_bigint_t> { static constexpr int id = AHEAD_BIGINT; };
template <> struct TI<v2_oid_t> { static constexpr int id = AHEAD_OID; };
template <> struct TI<v2_restiny_t> { static constexpr int id = AHEAD_RESTINY; };
template <> struct TI<v2_resshort_t> { static constexpr int id = AHEAD_RESSHORT; };
template <> struct TI<v2_resint_t> { static constexpr int id = AHEAD_RESINT; };
template <> struct TI<v2_resbigint_t> { static constexpr int id = AHEAD_RESBIGINT; };
template <> struct TI<v2_resoid_t> { static constexpr int id = AHEAD_RESOID; };

template <class... Ts> struct tl {};

template <class F> int visit(int, tl<>, F&&) { return AHEAD_BAD_ARG; }
template <class T0, class... Ts, class F> int visit(int t, tl<T0, Ts...>, F&& f) {
    if (t == TI<T0>::id) return f(T0{});
    return visit(t, tl<Ts...>{}, std::forward<F>(f));
}

typedef tl<v2_restiny_t, v2_resshort_t, v2_resint_t> ResSmall;
typedef tl<v2_restiny_t, v2_resshort_t, v2_resint_t, v2_resbigint_t, v2_resoid_t> ResAll;
typedef tl<v2_tinyint_t, v2_shortint_t, v2_int_t, v2_bigint_t, v2_oid_t> Plain;
typedef tl<v2_void_t, v2_resoid_t, v2_oid_t> OidCols;

template <class V> ColumnMetaData md_of(const ahead_col& c) {
    ColumnMetaData m(size_bytes<typename V::type_t>, (A_t)c.A, c.Ainv, c.unenc_max, 0);
    m.seqbase = c.seqbase;
    return m;
}

template <class V> typename V::type_t load(const ahead_col& c, uint64_t i) {
    typedef typename V::type_t T;
    if constexpr (std::is_same<V, v2_void_t>::value) {
        return (T)(c.seqbase + i);
    } else {
        return ((const T*)c.data)[i];
    }
}

// Build a TempBAT<H, T> holding a copy of the descriptor's data.
template <class H, class T> TempBAT<H, T>* make_bat(const ahead_bat* b) {
    auto* bat = new TempBAT<H, T>();
    bat->head.metaData = md_of<H>(b->head);
    bat->tail.metaData = md_of<T>(b->tail);
    constexpr bool hv = std::is_same<H, v2_void_t>::value;
    constexpr bool tv = std::is_same<T, v2_void_t>::value;
    if constexpr (hv && tv) {
        bat->overwrite_size(b->count);
    } else if constexpr (hv) {
        bat->reserve(b->count);
        for (uint64_t i = 0; i < b->count; ++i) bat->append_tail(load<T>(b->tail, i));
    } else if constexpr (tv) {
        bat->reserve(b->count);
        for (uint64_t i = 0; i < b->count; ++i) bat->append_head(load<H>(b->head, i));
    } else {
        bat->reserve(b->count);
        for (uint64_t i = 0; i < b->count; ++i)
            bat->append(std::make_pair(load<H>(b->head, i), load<T>(b->tail, i)));
    }
    return bat;
}

template <class V> void set_meta(ahead_col& c, const ColumnMetaData& m) {
    c.type = TI<V>::id;
    c.A = m.AN_A;
    c.Ainv = m.AN_Ainv;
    c.unenc_max = m.AN_unencMaxU;
    c.seqbase = m.seqbase;
}

template <class V, class Desc> void export_col(Desc& d, ahead_col& c, uint64_t n, uint64_t cap) {
    set_meta<V>(c, d.metaData);
    if constexpr (!std::is_same<V, v2_void_t>::value) {
        typedef typename V::type_t E;
        auto* vec = d.container.get();
        uint64_t m = std::min<uint64_t>(n, std::min<uint64_t>(cap, vec->size()));
        if (c.data)
            for (uint64_t i = 0; i < m; ++i) ((E*)c.data)[i] = (*vec)[i];
    }
}

// Copy a result BAT out.  `count_from_head` selects which column defines the
// row count (select results fill only the head).
template <class H, class T>
int export_bat(BAT<H, T>* bat, ahead_bat* out, uint64_t cap, int count_from = 0) {
    auto* tb = dynamic_cast<TempBAT<H, T>*>(bat);
    if (!tb) return AHEAD_BAD_ARG;
    uint64_t n = tb->size();
    if constexpr (!std::is_same<H, v2_void_t>::value) {
        if (count_from == 1) n = tb->head.container->size();
    }
    out->count = n;
    export_col<H>(tb->head, out->head, n, cap);
    export_col<T>(tb->tail, out->tail, n, cap);
    if (count_from == 1) out->tail.data = nullptr;  // only the head was filled
    return n > cap ? AHEAD_CAPACITY : AHEAD_OK;
}

void export_vec(AN_indicator_vector* v, ahead_errvec* e) {
    if (!e) {
        delete v;
        return;
    }
    if (!v) {
        e->present = 0;
        e->count = 0;
        return;
    }
    e->present = 1;
    e->count = v->size();
    uint64_t m = std::min<uint64_t>(e->capacity, v->size());
    if (e->data)
        for (uint64_t i = 0; i < m; ++i) e->data[i] = (*v)[i];
    delete v;
}

template <class T> using Lt = std::less<T>;
template <class T> using Le = std::less_equal<T>;
template <class T> using Eq = std::equal_to<T>;
template <class T> using Ne = std::not_equal_to<T>;
template <class T> using Ge = std::greater_equal<T>;
template <class T> using Gt = std::greater<T>;

template <class F> int with_op(int op, F&& f) {
    switch (op) {
        case AHEAD_CMP_LT: return f.template operator()<Lt>();
        case AHEAD_CMP_LE: return f.template operator()<Le>();
        case AHEAD_CMP_EQ: return f.template operator()<Eq>();
        case AHEAD_CMP_NE: return f.template operator()<Ne>();
        case AHEAD_CMP_GE: return f.template operator()<Ge>();
        case AHEAD_CMP_GT: return f.template operator()<Gt>();
        default: return AHEAD_BAD_ARG;
    }
}

template <class F> int with_comb(int comb, F&& f) {
    if (comb == AHEAD_AND) return f.template operator()<ahead::and_is>();
    if (comb == AHEAD_OR) return f.template operator()<ahead::or_is>();
    return AHEAD_BAD_ARG;
}

int guarded(const std::function<int()>& fn) {
    try {
        return fn();
    } catch (std::runtime_error&) {
        return AHEAD_SIZE_MISMATCH;
    }
}

// String selections: the reference's Selection(AN)1/2<..., v2_void_t, v2_str_t>
// on a TempBAT whose str_t tails point at NUL-terminated copies of the rows.
template <bool AN>
int select_str_ref(const char* strs, uint64_t width, uint64_t count, uint64_t seqbase, int op1, const char* th1,
                   int op2, const char* th2, int comb, ahead_bat* out, uint64_t cap) {
    if (!th1 || (op2 != AHEAD_CMP_NONE && !th2)) return AHEAD_BAD_ARG;
    std::vector<char> rows((size_t)count * (width + 1), 0);
    auto* bat = new TempBAT<v2_void_t, v2_str_t>();
    bat->head.metaData.seqbase = seqbase;
    bat->reserve(count);
    for (uint64_t i = 0; i < count; ++i) {
        char* r = rows.data() + i * (width + 1);
        std::memcpy(r, strs + i * width, width);
        bat->append_tail(r);
    }
    std::string t1(th1), t2(th2 ? th2 : "");
    auto finish = [&](auto* res) -> int {
        auto* tb = dynamic_cast<TempBAT<typename std::remove_pointer_t<decltype(res)>::v2_head_t,
                                        v2_str_t>*>(res);
        if (!tb) return AHEAD_BAD_ARG;
        typedef typename std::remove_pointer_t<decltype(res)>::v2_head_t H;
        uint64_t n = tb->head.container->size();
        out->count = n;
        export_col<H>(tb->head, out->head, n, cap);
        out->tail.type = AHEAD_STR;
        out->tail.data = nullptr;
        out->tail.A = 0;
        out->tail.Ainv = 0;
        out->tail.unenc_max = 0;
        out->tail.seqbase = 0;
        delete res;
        return n > cap ? AHEAD_CAPACITY : AHEAD_OK;
    };
    int rc;
    if (op2 == AHEAD_CMP_NONE) {
        rc = with_op(op1, [&]<template <class> class O1>() -> int {
            if constexpr (AN) return finish(scalar::selectAN<O1>(bat, t1.data(), (resoid_t)16089).first);
            else return finish(scalar::select<O1>(bat, t1.data()));
        });
    } else {
        rc = with_op(op1, [&]<template <class> class O1>() -> int {
            return with_op(op2, [&]<template <class> class O2>() -> int {
                return with_comb(comb, [&]<template <class> class C>() -> int {
                    if constexpr (AN)
                        return finish(scalar::selectAN<O1, O2, C>(bat, t1.data(), t2.data(), (resoid_t)16089).first);
                    else return finish(scalar::select<O1, O2, C>(bat, t1.data(), t2.data()));
                });
            });
        });
    }
    delete bat;
    return rc;
}

// hashjoinAN with a string right tail: the reference's
// hashjoinANunencHashmap<..., v2_str_t, ...> on a TempBAT<H2, v2_str_t> whose
// str_t tails point at NUL-terminated copies of the right slots; the matched
// strings are copied back into `width`-byte slots.
template <class H1, class T1, class H2>
int hashjoin_str_ref(const ahead_bat* l, const ahead_bat* r, const char* r_strs, uint64_t width, int reenc_head,
                     uint64_t ah1r, uint64_t ah1invr, int side, uint64_t aoid, ahead_bat* out, uint64_t cap,
                     ahead_errvec* errs) {
    hash_side_t hs = side == AHEAD_HASH_LEFT ? hash_side_t::left : hash_side_t::right;
    std::vector<char> copies((size_t)r->count * (width + 1), 0);
    auto* b = new TempBAT<H2, v2_str_t>();
    b->head.metaData = md_of<H2>(r->head);
    b->reserve(r->count);
    for (uint64_t i = 0; i < r->count; ++i) {
        char* c = copies.data() + i * (width + 1);
        std::memcpy(c, r_strs + i * width, width);
        b->append(std::make_pair(load<H2>(r->head, i), (str_t)c));
    }
    auto* a = make_bat<H1, T1>(l);
    auto finish = [&](auto res) -> int {
        auto* tb = std::get<0>(res);
        typedef typename std::remove_pointer_t<decltype(tb)>::v2_head_t HO;
        uint64_t n = tb->size();
        out->count = n;
        export_col<HO>(tb->head, out->head, n, cap);
        char* dst = (char*)out->tail.data;
        if (dst) {
            auto* strs = tb->tail.container.get();
            for (uint64_t i = 0; i < std::min<uint64_t>(n, cap); ++i) std::memcpy(dst + i * width, (*strs)[i], width);
        }
        out->tail.type = AHEAD_STR;
        out->tail.A = 0;
        out->tail.Ainv = 0;
        out->tail.unenc_max = 0;
        out->tail.seqbase = 0;
        export_vec(std::get<1>(res), errs ? &errs[0] : nullptr);
        export_vec(std::get<2>(res), errs ? &errs[1] : nullptr);
        export_vec(std::get<3>(res), errs ? &errs[2] : nullptr);
        export_vec(std::get<4>(res), errs ? &errs[3] : nullptr);
        delete tb;
        return n > cap ? AHEAD_CAPACITY : AHEAD_OK;
    };
    typedef typename TypeMap<H1>::v2_encoded_t::type_t h1e;
    int rc = reenc_head ? finish(hashjoinAN(a, b, (h1e)ah1r, (h1e)ah1invr, hs, (resoid_t)aoid))
                        : finish(hashjoinAN(a, b, hs, (resoid_t)aoid));
    delete a;
    delete b;
    return rc;
}

// A TempBAT<v2_void_t, v2_str_t> whose str_t tails point at NUL-terminated
// copies (in `copies`) of `count` slots of `width` bytes.
TempBAT<v2_void_t, v2_str_t>* str_bat(const char* strs, uint64_t width, uint64_t count, uint64_t seqbase,
                                      std::vector<char>& copies) {
    copies.assign((size_t)count * (width + 1), 0);
    auto* bat = new TempBAT<v2_void_t, v2_str_t>();
    bat->head.metaData.seqbase = seqbase;
    bat->reserve(count);
    for (uint64_t i = 0; i < count; ++i) {
        char* c = copies.data() + i * (width + 1);
        std::memcpy(c, strs + i * width, width);
        bat->append_tail(c);
    }
    return bat;
}

}  // namespace

extern "C" {

int orc_select_an(const ahead_bat* in, int op1, uint64_t th1, int op2, uint64_t th2, int comb,
                  uint64_t aoid, ahead_bat* out, uint64_t cap, ahead_errvec* err) {
    if (in->head.type != AHEAD_VOID) return AHEAD_BAD_ARG;
    return visit(in->tail.type, ResSmall{}, [&](auto t) -> int {
        typedef decltype(t) T;
        typedef typename T::type_t tt;
        auto* bat = make_bat<v2_void_t, T>(in);
        int rc;
        if (op2 == AHEAD_CMP_NONE) {
            rc = with_op(op1, [&]<template <class> class O1>() -> int {
                auto res = scalar::selectAN<O1>(bat, (tt)th1, (resoid_t)aoid);
                int r = export_bat(res.first, out, cap, 1);
                export_vec(res.second, err);
                delete res.first;
                return r;
            });
        } else {
            rc = with_op(op1, [&]<template <class> class O1>() -> int {
                return with_op(op2, [&]<template <class> class O2>() -> int {
                    return with_comb(comb, [&]<template <class> class C>() -> int {
                        auto res = scalar::selectAN<O1, O2, C>(bat, (tt)th1, (tt)th2, (resoid_t)aoid);
                        int r = export_bat(res.first, out, cap, 1);
                        export_vec(res.second, err);
                        delete res.first;
                        return r;
                    });
                });
            });
        }
        delete bat;
        return rc;
    });
}

int orc_select(const ahead_bat* in, int op1, uint64_t th1, int op2, uint64_t th2, int comb,
               ahead_bat* out, uint64_t cap) {
    if (in->head.type != AHEAD_VOID) return AHEAD_BAD_ARG;
    typedef tl<v2_tinyint_t, v2_shortint_t, v2_int_t, v2_bigint_t, v2_restiny_t, v2_resshort_t,
               v2_resint_t, v2_resbigint_t>
        Sel;
    return visit(in->tail.type, Sel{}, [&](auto t) -> int {
        typedef decltype(t) T;
        typedef typename T::type_t tt;
        auto* bat = make_bat<v2_void_t, T>(in);
        int rc;
        if (op2 == AHEAD_CMP_NONE) {
            rc = with_op(op1, [&]<template <class> class O1>() -> int {
                auto* res = scalar::select<O1>(bat, (tt)th1);
                int r = export_bat(res, out, cap, 1);
                delete res;
                return r;
            });
        } else {
            rc = with_op(op1, [&]<template <class> class O1>() -> int {
                return with_op(op2, [&]<template <class> class O2>() -> int {
                    return with_comb(comb, [&]<template <class> class C>() -> int {
                        auto* res = scalar::select<O1, O2, C>(bat, (tt)th1, (tt)th2);
                        int r = export_bat(res, out, cap, 1);
                        delete res;
                        return r;
                    });
                });
            });
        }
        delete bat;
        return rc;
    });
}

int orc_select_str_an(const char* strs, uint64_t width, uint64_t count, uint64_t seqbase, int op1,
                      const char* th1, int op2, const char* th2, int comb, ahead_bat* out, uint64_t cap) {
    return select_str_ref<true>(strs, width, count, seqbase, op1, th1, op2, th2, comb, out, cap);
}

int orc_select_str(const char* strs, uint64_t width, uint64_t count, uint64_t seqbase, int op1,
                   const char* th1, int op2, const char* th2, int comb, ahead_bat* out, uint64_t cap) {
    return select_str_ref<false>(strs, width, count, seqbase, op1, th1, op2, th2, comb, out, cap);
}

int orc_check_an(const ahead_bat* in, uint64_t ainv, uint64_t unenc_max, uint64_t aoid,
                 ahead_errvec* err) {
    // checkAN static_asserts an unencoded head (encdecAN_scalar.tcc:80).
    return visit(in->head.type, tl<v2_void_t, v2_oid_t>{}, [&](auto h) -> int {
        typedef decltype(h) H;
        return visit(in->tail.type, ResAll{}, [&](auto t) -> int {
            typedef decltype(t) T;
            typedef typename T::type_t tt;
            auto* bat = make_bat<H, T>(in);
            export_vec(scalar::checkAN(bat, (tt)ainv, (tt)unenc_max, (resoid_t)aoid), err);
            delete bat;
            return AHEAD_OK;
        });
    });
}

int orc_decode_an(const ahead_bat* in, uint64_t aoid, ahead_bat* out, uint64_t cap,
                  ahead_errvec* err) {
    return visit(in->head.type, tl<v2_resoid_t>{}, [&](auto h) -> int {
        typedef decltype(h) H;
        return visit(in->tail.type, ResAll{}, [&](auto t) -> int {
            typedef decltype(t) T;
            auto* bat = make_bat<H, T>(in);
            auto res = scalar::decodeAN(bat, (resoid_t)aoid);
            int r = export_bat(res.first, out, cap);
            export_vec(res.second, err);
            delete res.first;
            delete bat;
            return r;
        });
    });
}

int orc_check_and_decode_an(const ahead_bat* in, uint64_t aoid, ahead_bat* out, uint64_t cap,
                            ahead_errvec* err_head, ahead_errvec* err_tail) {
    return visit(in->head.type, OidCols{}, [&](auto h) -> int {
        typedef decltype(h) H;
        return visit(in->tail.type, ResAll{}, [&](auto t) -> int {
            typedef decltype(t) T;
            auto* bat = make_bat<H, T>(in);
            auto res = scalar::checkAndDecodeAN(bat, (resoid_t)aoid);
            int r = export_bat(std::get<0>(res), out, cap);
            export_vec(std::get<1>(res), err_head);
            export_vec(std::get<2>(res), err_tail);
            delete std::get<0>(res);
            delete bat;
            return r;
        });
    });
}

// encodeAN is not wrapped: its scalar definition does not compile
// (encdecAN_scalar.tcc:59 passes size_t where ColumnMetaData expects a
// data_width_t), so the reference cannot be run for it.
int orc_encode_an(const ahead_bat*, uint64_t, ahead_bat*, uint64_t) { return AHEAD_UNSUPPORTED; }

int orc_hashjoin_an(const ahead_bat* l, const ahead_bat* r, int reenc_head, uint64_t ah1r,
                    uint64_t ah1invr, int reenc_tail, uint64_t at2r, uint64_t at2invr, int side,
                    uint64_t aoid, ahead_bat* out, uint64_t cap, ahead_errvec* errs) {
    if (reenc_tail && !reenc_head) return AHEAD_BAD_ARG;
    hash_side_t hs = side == AHEAD_HASH_LEFT ? hash_side_t::left : hash_side_t::right;
    typedef tl<v2_void_t, v2_resoid_t> HT;
    return visit(l->head.type, HT{}, [&](auto h1) -> int {
        typedef decltype(h1) H1;
        return visit(l->tail.type, ResSmall{}, [&](auto t1) -> int {
            typedef decltype(t1) T1;
            return visit(r->head.type, ResSmall{}, [&](auto h2) -> int {
                typedef decltype(h2) H2;
                return visit(r->tail.type, HT{}, [&](auto t2) -> int {
                    typedef decltype(t2) T2;
                    auto* a = make_bat<H1, T1>(l);
                    auto* b = make_bat<H2, T2>(r);
                    int rc;
                    auto finish = [&](auto res) -> int {
                        int x = export_bat(std::get<0>(res), out, cap);
                        for (int k = 0; k < 4; ++k)
                            export_vec(k == 0 ? std::get<1>(res)
                                       : k == 1 ? std::get<2>(res)
                                       : k == 2 ? std::get<3>(res)
                                                : std::get<4>(res),
                                       errs ? &errs[k] : nullptr);
                        delete std::get<0>(res);
                        return x;
                    };
                    typedef typename TypeMap<H1>::v2_encoded_t::type_t h1e;
                    typedef typename TypeMap<T2>::v2_encoded_t::type_t t2e;
                    if (!reenc_head)
                        rc = finish(hashjoinAN(a, b, hs, (resoid_t)aoid));
                    else if (!reenc_tail)
                        rc = finish(hashjoinAN(a, b, (h1e)ah1r, (h1e)ah1invr, hs, (resoid_t)aoid));
                    else
                        rc = finish(hashjoinAN(a, b, (h1e)ah1r, (h1e)ah1invr, (t2e)at2r, (t2e)at2invr,
                                               hs, (resoid_t)aoid));
                    delete a;
                    delete b;
                    return rc;
                });
            });
        });
    });
}

int orc_hashjoin_str_an(const ahead_bat* l, const ahead_bat* r, const char* r_strs, uint64_t width,
                        int reenc_head, uint64_t ah1r, uint64_t ah1invr, int side, uint64_t aoid,
                        ahead_bat* out, uint64_t cap, ahead_errvec* errs) {
    typedef tl<v2_void_t, v2_resoid_t> HT;
    return visit(l->head.type, HT{}, [&](auto h1) -> int {
        return visit(l->tail.type, ResSmall{}, [&](auto t1) -> int {
            return visit(r->head.type, ResSmall{}, [&](auto h2) -> int {
                return hashjoin_str_ref<decltype(h1), decltype(t1), decltype(h2)>(
                    l, r, r_strs, width, reenc_head, ah1r, ah1invr, side, aoid, out, cap, errs);
            });
        });
    });
}

int orc_hashjoin(const ahead_bat* l, const ahead_bat* r, int side, ahead_bat* out, uint64_t cap) {
    hash_side_t hs = side == AHEAD_HASH_LEFT ? hash_side_t::left : hash_side_t::right;
    typedef tl<v2_void_t, v2_oid_t> HT;
    typedef tl<v2_tinyint_t, v2_shortint_t, v2_int_t, v2_restiny_t, v2_resshort_t, v2_resint_t> KT;
    return visit(l->head.type, HT{}, [&](auto h1) -> int {
        typedef decltype(h1) H1;
        return visit(l->tail.type, KT{}, [&](auto t1) -> int {
            typedef decltype(t1) T1;
            return visit(r->head.type, tl<T1>{}, [&](auto h2) -> int {
                typedef decltype(h2) H2;
                return visit(r->tail.type, HT{}, [&](auto t2) -> int {
                    typedef decltype(t2) T2;
                    auto* a = make_bat<H1, T1>(l);
                    auto* b = make_bat<H2, T2>(r);
                    auto* res = hashjoin(a, b, hs);
                    int rc = export_bat(res, out, cap);
                    delete res;
                    delete a;
                    delete b;
                    return rc;
                });
            });
        });
    });
}

int orc_matchjoin_an(const ahead_bat* a, const ahead_bat* b, int reenc, uint64_t ah1r,
                     uint64_t ah1invr, uint64_t at2r, uint64_t at2invr, uint64_t aoid,
                     ahead_bat* out, uint64_t cap, ahead_errvec* errs) {
    typedef tl<v2_void_t, v2_resoid_t, v2_resint_t> H1L;
    typedef tl<v2_void_t, v2_resoid_t> T1L;
    typedef tl<v2_void_t, v2_resoid_t> H2L;
    typedef tl<v2_restiny_t, v2_resshort_t, v2_resint_t, v2_resbigint_t, v2_resoid_t, v2_void_t> T2L;
    return visit(a->head.type, H1L{}, [&](auto h1) -> int {
        typedef decltype(h1) H1;
        return visit(a->tail.type, T1L{}, [&](auto t1) -> int {
            typedef decltype(t1) T1;
            return visit(b->head.type, H2L{}, [&](auto h2) -> int {
                typedef decltype(h2) H2;
                return visit(b->tail.type, T2L{}, [&](auto t2) -> int {
                    typedef decltype(t2) T2;
                    // Only the forms the reference defines: (void tail, void head),
                    // (resoid tail, void head) and the general merge on resoid.
                    constexpr bool vv = std::is_same<T1, v2_void_t>::value && std::is_same<H2, v2_void_t>::value;
                    constexpr bool rv = std::is_same<T1, v2_resoid_t>::value && std::is_same<H2, v2_void_t>::value;
                    constexpr bool gm = std::is_same<T1, v2_resoid_t>::value && std::is_same<H2, v2_resoid_t>::value;
                    constexpr bool mv = std::is_same<T1, v2_void_t>::value && std::is_same<H2, v2_resoid_t>::value;
                    constexpr bool h1void_ok = !std::is_same<H1, v2_void_t>::value || !std::is_same<T1, v2_void_t>::value;
                    if constexpr (!(vv || rv || gm || mv) || !h1void_ok ||
                                  (std::is_same<T2, v2_void_t>::value && !gm)) {
                        return AHEAD_BAD_ARG;
                    } else {
                        auto* x = make_bat<H1, T1>(a);
                        auto* y = make_bat<H2, T2>(b);
                        typedef typename ANhelper<H1>::type_t h1t;
                        typedef typename ANhelper<T2>::type_t t2t;
                        auto finish = [&](auto res) -> int {
                            int rc = export_bat(std::get<0>(res), out, cap);
                            export_vec(std::get<1>(res), errs ? &errs[0] : nullptr);
                            export_vec(std::get<2>(res), errs ? &errs[1] : nullptr);
                            export_vec(std::get<3>(res), errs ? &errs[2] : nullptr);
                            export_vec(std::get<4>(res), errs ? &errs[3] : nullptr);
                            delete std::get<0>(res);
                            return rc;
                        };
                        int rc;
                        // The re-encoding overloads only compile in the reference when
                        // neither H1 nor T2 is void (the declared and the actual result
                        // types differ otherwise, matchjoinAN.tcc:405-414).
                        constexpr bool reenc_ok = !std::is_same<H1, v2_void_t>::value && !std::is_same<T2, v2_void_t>::value;
                        if (reenc) {
                            if constexpr (reenc_ok)
                                rc = finish(matchjoinAN(x, y, (h1t)ah1r, (h1t)ah1invr, (t2t)at2r, (t2t)at2invr, (resoid_t)aoid));
                            else
                                rc = AHEAD_UNSUPPORTED;
                        } else {
                            rc = finish(matchjoinAN(x, y, (resoid_t)aoid));
                        }
                        delete x;
                        delete y;
                        return rc;
                    }
                });
            });
        });
    });
}

int orc_matchjoin(const ahead_bat* a, const ahead_bat* b, ahead_bat* out, uint64_t cap) {
    typedef tl<v2_void_t, v2_oid_t> OL;
    typedef tl<v2_tinyint_t, v2_shortint_t, v2_int_t, v2_bigint_t, v2_restiny_t, v2_resshort_t,
               v2_resint_t, v2_resbigint_t, v2_oid_t>
        T2L;
    typedef tl<v2_void_t, v2_oid_t, v2_tinyint_t, v2_shortint_t, v2_int_t, v2_bigint_t, v2_restiny_t, v2_resshort_t,
               v2_resint_t, v2_resbigint_t>
        H1L;
    return visit(a->head.type, H1L{}, [&](auto h1) -> int {
        typedef decltype(h1) H1;
        return visit(a->tail.type, OL{}, [&](auto t1) -> int {
            typedef decltype(t1) T1;
            return visit(b->head.type, OL{}, [&](auto h2) -> int {
                typedef decltype(h2) H2;
                return visit(b->tail.type, T2L{}, [&](auto t2) -> int {
                    typedef decltype(t2) T2;
                    constexpr bool ok = !(std::is_same<H1, v2_void_t>::value && std::is_same<T1, v2_void_t>::value);
                    if constexpr (!ok) {
                        return AHEAD_BAD_ARG;
                    } else {
                        auto* x = make_bat<H1, T1>(a);
                        auto* y = make_bat<H2, T2>(b);
                        auto* res = matchjoin(x, y);
                        int rc = export_bat(res, out, cap);
                        delete res;
                        delete x;
                        delete y;
                        return rc;
                    }
                });
            });
        });
    });
}

int orc_fetchjoin_an(const ahead_bat* a, const ahead_bat* b, int reenc, uint64_t atr,
                     uint64_t atrinv, uint64_t aoid, ahead_bat* out, uint64_t cap,
                     ahead_errvec* errs) {
    if (a->head.type != AHEAD_VOID || a->tail.type != AHEAD_RESOID || b->head.type != AHEAD_VOID)
        return AHEAD_BAD_ARG;
    return visit(b->tail.type, ResAll{}, [&](auto t2) -> int {
        typedef decltype(t2) T2;
        typedef typename TypeMap<T2>::v2_encoded_t::type_t te;
        auto* x = make_bat<v2_void_t, v2_resoid_t>(a);
        auto* y = make_bat<v2_void_t, T2>(b);
        auto res = reenc ? fetchjoinAN(x, y, (te)atr, (te)atrinv, (resoid_t)aoid)
                         : fetchjoinAN(x, y, (resoid_t)aoid);
        int rc = export_bat(std::get<0>(res), out, cap);
        export_vec(std::get<1>(res), errs ? &errs[0] : nullptr);
        export_vec(std::get<2>(res), errs ? &errs[1] : nullptr);
        delete std::get<0>(res);
        delete x;
        delete y;
        return rc;
    });
}

int orc_fetchjoin(const ahead_bat* a, const ahead_bat* b, ahead_bat* out, uint64_t cap) {
    if (a->head.type != AHEAD_VOID || a->tail.type != AHEAD_OID || b->head.type != AHEAD_VOID)
        return AHEAD_BAD_ARG;
    typedef tl<v2_tinyint_t, v2_shortint_t, v2_int_t, v2_bigint_t, v2_restiny_t, v2_resshort_t,
               v2_resint_t, v2_resbigint_t, v2_oid_t>
        T2L;
    return visit(b->tail.type, T2L{}, [&](auto t2) -> int {
        typedef decltype(t2) T2;
        auto* x = make_bat<v2_void_t, v2_oid_t>(a);
        auto* y = make_bat<v2_void_t, T2>(b);
        auto* res = fetchjoin(x, y);
        int rc = export_bat(res, out, cap);
        delete res;
        delete x;
        delete y;
        return rc;
    });
}

int orc_groupby_an(const ahead_bat* in, uint64_t aoid, uint64_t aoidinv, ahead_bat* gids,
                   ahead_bat* firsts, uint64_t cap, ahead_errvec* errs) {
    return visit(in->head.type, OidCols{}, [&](auto h) -> int {
        typedef decltype(h) H;
        return visit(in->tail.type, ResAll{}, [&](auto t) -> int {
            typedef decltype(t) T;
            auto* bat = make_bat<H, T>(in);
            auto res = groupbyAN(bat, (resoid_t)aoid, (resoid_t)aoidinv);
            int r1 = export_bat(std::get<0>(res), gids, cap);
            int r2 = export_bat(std::get<1>(res), firsts, cap);
            export_vec(std::get<2>(res), errs ? &errs[0] : nullptr);
            export_vec(std::get<3>(res), errs ? &errs[1] : nullptr);
            delete std::get<0>(res);
            delete std::get<1>(res);
            delete bat;
            return r1 ? r1 : r2;
        });
    });
}

int orc_groupby2_an(const ahead_bat* in, const ahead_bat* grouping, uint64_t ngroups,
                    uint64_t aoid, uint64_t aoidinv, ahead_bat* gids, ahead_bat* firsts,
                    uint64_t cap, ahead_errvec* errs) {
    if (grouping->head.type != AHEAD_VOID || grouping->tail.type != AHEAD_RESOID) return AHEAD_BAD_ARG;
    return visit(in->head.type, OidCols{}, [&](auto h) -> int {
        typedef decltype(h) H;
        return visit(in->tail.type, ResAll{}, [&](auto t) -> int {
            typedef decltype(t) T;
            return guarded([&]() -> int {
                auto* bat = make_bat<H, T>(in);
                auto* g = make_bat<v2_void_t, v2_resoid_t>(grouping);
                int rc;
                try {
                    auto res = groupbyAN(bat, g, (size_t)ngroups, (resoid_t)aoid, (resoid_t)aoidinv);
                    int r1 = export_bat(std::get<0>(res), gids, cap);
                    int r2 = export_bat(std::get<1>(res), firsts, cap);
                    export_vec(std::get<2>(res), errs ? &errs[0] : nullptr);
                    export_vec(std::get<3>(res), errs ? &errs[1] : nullptr);
                    export_vec(std::get<4>(res), errs ? &errs[2] : nullptr);
                    delete std::get<0>(res);
                    delete std::get<1>(res);
                    rc = r1 ? r1 : r2;
                } catch (...) {
                    delete bat;
                    delete g;
                    throw;
                }
                delete bat;
                delete g;
                return rc;
            });
        });
    });
}

int orc_aggregate_sum_grouped_an(const ahead_bat* in, const ahead_bat* grouping,
                                 uint64_t ngroups, int result_type, uint64_t ar, uint64_t arinv,
                                 uint64_t aoid, ahead_bat* out, ahead_errvec* errs) {
    if (result_type != AHEAD_RESBIGINT) return AHEAD_BAD_ARG;
    if (grouping->head.type != AHEAD_VOID || grouping->tail.type != AHEAD_RESOID) return AHEAD_BAD_ARG;
    typedef tl<v2_void_t, v2_oid_t, v2_resoid_t> HL;
    typedef tl<v2_int_t, v2_resint_t, v2_resbigint_t, v2_resshort_t, v2_restiny_t> TL;
    return visit(in->head.type, HL{}, [&](auto h) -> int {
        typedef decltype(h) H;
        return visit(in->tail.type, TL{}, [&](auto t) -> int {
            typedef decltype(t) T;
            return guarded([&]() -> int {
                auto* bat = make_bat<H, T>(in);
                auto* g = make_bat<v2_void_t, v2_resoid_t>(grouping);
                int rc;
                try {
                    auto res = aggregate_sum_groupedAN<v2_resbigint_t>(bat, g, (size_t)ngroups, (resbigint_t)ar,
                                                                       (resbigint_t)arinv, (resoid_t)aoid);
                    rc = export_bat(std::get<0>(res), out, ngroups);
                    export_vec(std::get<1>(res), errs ? &errs[0] : nullptr);
                    export_vec(std::get<2>(res), errs ? &errs[1] : nullptr);
                    export_vec(std::get<3>(res), errs ? &errs[2] : nullptr);
                    delete std::get<0>(res);
                } catch (...) {
                    delete bat;
                    delete g;
                    throw;
                }
                delete bat;
                delete g;
                return rc;
            });
        });
    });
}

int orc_aggregate_mul_sum_an(const ahead_bat* a, const ahead_bat* b, int result_type,
                             uint64_t init, uint64_t ra, uint64_t rainv, uint64_t aoid,
                             uint64_t* total, ahead_errvec* errs) {
    if (result_type != AHEAD_RESBIGINT) return AHEAD_BAD_ARG;
    typedef tl<v2_void_t, v2_resoid_t> HL;
    return visit(a->head.type, HL{}, [&](auto h1) -> int {
        typedef decltype(h1) H1;
        return visit(a->tail.type, ResSmall{}, [&](auto t1) -> int {
            typedef decltype(t1) T1;
            return visit(b->head.type, HL{}, [&](auto h2) -> int {
                typedef decltype(h2) H2;
                return visit(b->tail.type, ResSmall{}, [&](auto t2) -> int {
                    typedef decltype(t2) T2;
                    auto* x = make_bat<H1, T1>(a);
                    auto* y = make_bat<H2, T2>(b);
                    auto res = scalar::aggregate_mul_sumAN<v2_resbigint_t>(x, y, (resbigint_t)init, (resbigint_t)ra,
                                                                           (resbigint_t)rainv, (resoid_t)aoid);
                    auto* rb = dynamic_cast<TempBAT<v2_void_t, v2_resbigint_t>*>(std::get<0>(res));
                    *total = (*rb->tail.container)[0];
                    export_vec(std::get<1>(res), errs ? &errs[0] : nullptr);
                    export_vec(std::get<2>(res), errs ? &errs[1] : nullptr);
                    delete std::get<0>(res);
                    delete x;
                    delete y;
                    return AHEAD_OK;
                });
            });
        });
    });
}

int orc_aggregate_mul_sum(const ahead_bat* a, const ahead_bat* b, int result_type,
                          uint64_t init, uint64_t* total) {
    if (result_type != AHEAD_BIGINT) return AHEAD_BAD_ARG;
    typedef tl<v2_void_t, v2_oid_t> HL;
    typedef tl<v2_tinyint_t, v2_shortint_t, v2_int_t, v2_bigint_t> TL;
    return visit(a->head.type, HL{}, [&](auto h1) -> int {
        typedef decltype(h1) H1;
        return visit(a->tail.type, TL{}, [&](auto t1) -> int {
            typedef decltype(t1) T1;
            return visit(b->head.type, HL{}, [&](auto h2) -> int {
                typedef decltype(h2) H2;
                return visit(b->tail.type, TL{}, [&](auto t2) -> int {
                    typedef decltype(t2) T2;
                    auto* x = make_bat<H1, T1>(a);
                    auto* y = make_bat<H2, T2>(b);
                    auto* res = scalar::aggregate_mul_sum<v2_bigint_t>(x, y, (bigint_t)init);
                    auto* rb = dynamic_cast<TempBAT<v2_void_t, v2_bigint_t>*>(res);
                    *total = (*rb->tail.container)[0];
                    delete res;
                    delete x;
                    delete y;
                    return AHEAD_OK;
                });
            });
        });
    });
}

int orc_arithmetic_an(int op, int result_type, const ahead_bat* a, const ahead_bat* b,
                      uint64_t ar, uint64_t arinv, uint64_t aoid, ahead_bat* out,
                      ahead_errvec* errs) {
    typedef tl<v2_resint_t, v2_resbigint_t> RL;
    typedef tl<v2_resint_t, v2_resshort_t, v2_restiny_t> TL;
    if (a->head.type != AHEAD_VOID || b->head.type != AHEAD_VOID) return AHEAD_BAD_ARG;
    return visit(result_type, RL{}, [&](auto rt) -> int {
        typedef decltype(rt) R;
        typedef typename R::type_t rtt;
        return visit(a->tail.type, TL{}, [&](auto t1) -> int {
            typedef decltype(t1) T1;
            return visit(b->tail.type, TL{}, [&](auto t2) -> int {
                typedef decltype(t2) T2;
                return guarded([&]() -> int {
                    auto* x = make_bat<v2_void_t, T1>(a);
                    auto* y = make_bat<v2_void_t, T2>(b);
                    int rc = AHEAD_OK;
                    try {
                        auto run = [&](auto res) {
                            rc = export_bat(std::get<0>(res), out, a->count);
                            for (int k = 0; k < 4; ++k)
                                export_vec(k == 0 ? std::get<1>(res)
                                           : k == 1 ? std::get<2>(res)
                                           : k == 2 ? std::get<3>(res)
                                                    : std::get<4>(res),
                                           errs ? &errs[k] : nullptr);
                            delete std::get<0>(res);
                        };
                        switch (op) {
                            case AHEAD_ADD: run(scalar::arithmeticAN<ahead::add, R>(x, y, (rtt)ar, (rtt)arinv, (resoid_t)aoid)); break;
                            case AHEAD_SUB: run(scalar::arithmeticAN<ahead::sub, R>(x, y, (rtt)ar, (rtt)arinv, (resoid_t)aoid)); break;
                            case AHEAD_MUL: run(scalar::arithmeticAN<ahead::mul, R>(x, y, (rtt)ar, (rtt)arinv, (resoid_t)aoid)); break;
                            case AHEAD_DIV: run(scalar::arithmeticAN<ahead::div, R>(x, y, (rtt)ar, (rtt)arinv, (resoid_t)aoid)); break;
                            default: rc = AHEAD_BAD_ARG;
                        }
                    } catch (...) {
                        delete x;
                        delete y;
                        throw;
                    }
                    delete x;
                    delete y;
                    return rc;
                });
            });
        });
    });
}

uint64_t orc_ainv(uint64_t a, int bits) {
    return v2convert<uint64_t>(ext_euclidean(uint128_t((unsigned long long)a), (size_t)bits));
}


// ---------------------------------------------------------------- unencoded twins
typedef tl<v2_void_t, v2_oid_t> VoidOid;
typedef tl<v2_oid_t, v2_tinyint_t, v2_shortint_t, v2_int_t, v2_resoid_t, v2_restiny_t, v2_resshort_t, v2_resint_t>
    GbTails;

int orc_groupby(const ahead_bat* in, ahead_bat* gids, ahead_bat* firsts, uint64_t cap) {
    return visit(in->head.type, VoidOid{}, [&](auto h) -> int {
        typedef decltype(h) H;
        return visit(in->tail.type, GbTails{}, [&](auto t) -> int {
            typedef decltype(t) T;
            auto* bat = make_bat<H, T>(in);
            auto res = groupby(bat);
            int r1 = export_bat(res.first, gids, cap);
            int r2 = export_bat(res.second, firsts, cap);
            delete res.first;
            delete res.second;
            delete bat;
            return r1 ? r1 : r2;
        });
    });
}

int orc_groupby2(const ahead_bat* in, const ahead_bat* grouping, uint64_t ngroups, ahead_bat* gids,
                 ahead_bat* firsts, uint64_t cap) {
    if (grouping->head.type != AHEAD_VOID || grouping->tail.type != AHEAD_OID) return AHEAD_BAD_ARG;
    return visit(in->head.type, VoidOid{}, [&](auto h) -> int {
        typedef decltype(h) H;
        return visit(in->tail.type, GbTails{}, [&](auto t) -> int {
            typedef decltype(t) T;
            return guarded([&]() -> int {
                auto* bat = make_bat<H, T>(in);
                auto* g = make_bat<v2_void_t, v2_oid_t>(grouping);
                int rc;
                try {
                    auto res = groupby(bat, g, (size_t)ngroups);
                    int r1 = export_bat(res.first, gids, cap);
                    int r2 = export_bat(res.second, firsts, cap);
                    delete res.first;
                    delete res.second;
                    rc = r1 ? r1 : r2;
                } catch (...) {
                    delete bat;
                    delete g;
                    throw;
                }
                delete bat;
                delete g;
                return rc;
            });
        });
    });
}

int orc_aggregate_sum_grouped(const ahead_bat* in, const ahead_bat* grouping, uint64_t ngroups,
                              int result_type, ahead_bat* out) {
    if (result_type != AHEAD_BIGINT || in->tail.type != AHEAD_INT) return AHEAD_BAD_ARG;
    if (grouping->head.type != AHEAD_VOID || grouping->tail.type != AHEAD_OID) return AHEAD_BAD_ARG;
    return visit(in->head.type, VoidOid{}, [&](auto h) -> int {
        typedef decltype(h) H;
        return guarded([&]() -> int {
            auto* bat = make_bat<H, v2_int_t>(in);
            auto* g = make_bat<v2_void_t, v2_oid_t>(grouping);
            int rc;
            try {
                auto* res = aggregate_sum_grouped<v2_bigint_t>(bat, g, (size_t)ngroups);
                rc = export_bat(res, out, ngroups);
                delete res;
            } catch (...) {
                delete bat;
                delete g;
                throw;
            }
            delete bat;
            delete g;
            return rc;
        });
    });
}

int orc_aggregate_sum(const ahead_bat* in, int result_type, uint64_t* total) {
    if (in->head.type != AHEAD_OID) return AHEAD_BAD_ARG;
    typedef tl<v2_tinyint_t, v2_shortint_t, v2_int_t, v2_bigint_t> IntTypes;
    return visit(result_type, IntTypes{}, [&](auto r) -> int {
        typedef decltype(r) R;
        return visit(in->tail.type, IntTypes{}, [&](auto t) -> int {
            typedef decltype(t) T;
            if constexpr (sizeof(typename R::type_t) < sizeof(typename T::type_t)) {
                return AHEAD_BAD_ARG;
            } else {
                auto* bat = make_bat<v2_oid_t, T>(in);
                *total = (uint64_t)scalar::aggregate_sum<R>(bat);
                delete bat;
                return AHEAD_OK;
            }
        });
    });
}

int orc_arithmetic(int op, int result_type, const ahead_bat* a, const ahead_bat* b, ahead_bat* out) {
    if (a->head.type != AHEAD_VOID || b->head.type != AHEAD_VOID) return AHEAD_BAD_ARG;
    if (a->tail.type != b->tail.type || a->tail.type != result_type) return AHEAD_BAD_ARG;
    typedef tl<v2_int_t, v2_resint_t> ArTypes;
    return visit(result_type, ArTypes{}, [&](auto r) -> int {
        typedef decltype(r) R;
        return guarded([&]() -> int {
            auto* x = make_bat<v2_void_t, R>(a);
            auto* y = make_bat<v2_void_t, R>(b);
            BAT<v2_void_t, R>* res = nullptr;
            try {
                switch (op) {
                    case AHEAD_ADD: res = scalar::arithmetic<ahead::add, R>(x, y); break;
                    case AHEAD_SUB: res = scalar::arithmetic<ahead::sub, R>(x, y); break;
                    case AHEAD_MUL: res = scalar::arithmetic<ahead::mul, R>(x, y); break;
                    case AHEAD_DIV: res = scalar::arithmetic<ahead::div, R>(x, y); break;
                    default: break;
                }
            } catch (...) {
                delete x;
                delete y;
                throw;
            }
            delete x;
            delete y;
            if (!res) return AHEAD_BAD_ARG;
            int rc = export_bat(res, out, a->count);
            delete res;
            return rc;
        });
    });
}

}  // extern "C"

extern "C" {

// fetchjoinAN with a string tail: the reference's FetchjoinAN<v2_str_t, false>
// (matchjoinAN.tcc:304-354) on a string TempBAT; the fetched strings are copied
// back into `width`-byte slots.
int orc_fetchjoin_str_an(const ahead_bat* a, const char* strs, uint64_t width, uint64_t count, uint64_t aoid,
                         char* out, uint64_t cap, uint64_t* n_out, ahead_errvec* errs) {
    if (a->head.type != AHEAD_VOID || a->tail.type != AHEAD_RESOID || !width) return AHEAD_BAD_ARG;
    std::vector<char> copies;
    auto* y = str_bat(strs, width, count, 0, copies);
    auto* x = make_bat<v2_void_t, v2_resoid_t>(a);
    auto res = fetchjoinAN(x, y, (resoid_t)aoid);
    auto* tb = std::get<0>(res);
    uint64_t n = tb->size();
    auto* got = tb->tail.container.get();
    if (out)
        for (uint64_t i = 0; i < std::min<uint64_t>(n, cap); ++i) {
            std::memset(out + i * width, 0, width);
            std::strncpy(out + i * width, (*got)[i], width);
        }
    *n_out = n;
    export_vec(std::get<1>(res), errs ? &errs[0] : nullptr);
    export_vec(std::get<2>(res), errs ? &errs[1] : nullptr);
    delete tb;
    delete x;
    delete y;
    return n > cap ? AHEAD_CAPACITY : AHEAD_OK;
}

// groupbyAN binary over a string tail: the reference's groupbyAN on a
// BAT<v2_void_t, v2_str_t> (groupbyAN.tcc:99-165, hash<str_t>).
int orc_groupby2_str_an(const char* strs, uint64_t width, uint64_t count, uint64_t seqbase,
                        const ahead_bat* grouping, uint64_t ngroups, uint64_t aoid, uint64_t aoidinv,
                        ahead_bat* gids, ahead_bat* firsts, uint64_t cap, ahead_errvec* errs) {
    if (grouping->head.type != AHEAD_VOID || grouping->tail.type != AHEAD_RESOID || !width) return AHEAD_BAD_ARG;
    return guarded([&]() -> int {
        std::vector<char> copies;
        auto* bat = str_bat(strs, width, count, seqbase, copies);
        auto* g = make_bat<v2_void_t, v2_resoid_t>(grouping);
        int rc;
        try {
            auto res = groupbyAN(bat, g, (size_t)ngroups, (resoid_t)aoid, (resoid_t)aoidinv);
            int r1 = export_bat(std::get<0>(res), gids, cap);
            int r2 = export_bat(std::get<1>(res), firsts, cap);
            export_vec(std::get<2>(res), errs ? &errs[0] : nullptr);
            export_vec(std::get<3>(res), errs ? &errs[1] : nullptr);
            export_vec(std::get<4>(res), errs ? &errs[2] : nullptr);
            delete std::get<0>(res);
            delete std::get<1>(res);
            rc = r1 ? r1 : r2;
        } catch (...) {
            delete bat;
            delete g;
            throw;
        }
        delete bat;
        delete g;
        return rc;
    });
}

// The unencoded twins: the reference's fetchjoin (Normal/matchjoin.tcc) and
// binary groupby (Normal/groupby.tcc) over string BATs.
int orc_fetchjoin_str(const ahead_bat* a, const char* strs, uint64_t width, uint64_t count, char* out, uint64_t cap,
                      uint64_t* n_out) {
    if (a->head.type != AHEAD_VOID || a->tail.type != AHEAD_OID || !width) return AHEAD_BAD_ARG;
    std::vector<char> copies;
    auto* y = str_bat(strs, width, count, 0, copies);
    auto* x = make_bat<v2_void_t, v2_oid_t>(a);
    auto* res = fetchjoin(x, y);
    uint64_t n = res->size();
    auto* tb = dynamic_cast<TempBAT<v2_void_t, v2_str_t>*>(res);
    if (out && tb) {
        auto* got = tb->tail.container.get();
        for (uint64_t i = 0; i < std::min<uint64_t>(n, cap); ++i) {
            std::memset(out + i * width, 0, width);
            std::strncpy(out + i * width, (*got)[i], width);
        }
    }
    *n_out = n;
    delete res;
    delete x;
    delete y;
    return n > cap ? AHEAD_CAPACITY : AHEAD_OK;
}

int orc_groupby2_str(const char* strs, uint64_t width, uint64_t count, uint64_t seqbase, const ahead_bat* grouping,
                     uint64_t ngroups, ahead_bat* gids, ahead_bat* firsts, uint64_t cap) {
    if (grouping->head.type != AHEAD_VOID || grouping->tail.type != AHEAD_OID || !width) return AHEAD_BAD_ARG;
    return guarded([&]() -> int {
        std::vector<char> copies;
        auto* bat = str_bat(strs, width, count, seqbase, copies);
        auto* g = make_bat<v2_void_t, v2_oid_t>(grouping);
        int rc;
        try {
            auto res = groupby(bat, g, (size_t)ngroups);
            int r1 = export_bat(res.first, gids, cap);
            int r2 = export_bat(res.second, firsts, cap);
            delete res.first;
            delete res.second;
            rc = r1 ? r1 : r2;
        } catch (...) {
            delete bat;
            delete g;
            throw;
        }
        delete bat;
        delete g;
        return rc;
    });
}

}  // extern "C"
