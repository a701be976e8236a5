/*
 * an_oracle.c -- TEST INFRASTRUCTURE ONLY (see an_oracle.h).
 *
 * Plain-C restatement of the reference's scalar AN operators and their
 * unencoded twins.  Every value is carried in a uint64_t and reduced modulo
 * 2^(8*width) exactly where the reference's C++ types wrap, so results
 * (including error-position vectors) are bit-identical to the reference's
 * scalar build.  Reference paths are relative to the reference project.
 *
 * Where the reference has undefined behaviour this file makes one documented
 * choice (the GPU library makes the same one):
 *   - positional fetches whose decoded position equals the column size read
 *     one past the end in the reference (matchjoinAN.tcc:283,337); here such a
 *     position counts as out of range;
 *   - unchecked positional fetches of the unencoded matchjoin/fetchjoin
 *     (Normal/matchjoin.tcc:150,168) out of range produce no row;
 *   - grouped sums whose group id is >= numGroups (aggregateAN.tcc:109 writes
 *     out of bounds) are skipped;
 *   - arithmetic division by zero yields 0.
 */
#include "an_oracle.h"

#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* Type model (include/util/v2types.hpp:242-455, resilience.hpp:36-276).     */

static int tw(int t) { /* storage width in bytes */
    static const int w[AHEAD_NTYPES] = {4, 1, 2, 4, 8, 4, 2, 4, 8, 8, 8};
    return (t >= 0 && t < AHEAD_NTYPES) ? w[t] : 0;
}
static int tbase(int t) { /* width of TypeMap<T>::v2_base_t::type_t */
    static const int w[AHEAD_NTYPES] = {4, 1, 2, 4, 8, 4, 1, 2, 4, 8, 4};
    return w[t];
}
static int tenc(int t) { return t >= AHEAD_RESTINY && t <= AHEAD_RESOID; }
static int tenctype(int t) { /* TypeMap<T>::v2_encoded_t */
    static const int e[AHEAD_NTYPES] = {AHEAD_RESOID,   AHEAD_RESTINY, AHEAD_RESSHORT, AHEAD_RESINT,
                                        AHEAD_RESBIGINT, AHEAD_RESOID,  AHEAD_RESTINY,  AHEAD_RESSHORT,
                                        AHEAD_RESINT,    AHEAD_RESBIGINT, AHEAD_RESOID};
    return e[t];
}
static int tsel(int t) { return t == AHEAD_VOID ? AHEAD_OID : t; } /* v2_select_t */
static int tunenc(int t) { /* v2_unenc_t */
    switch (t) {
        case AHEAD_RESTINY: return AHEAD_TINYINT;
        case AHEAD_RESSHORT: return AHEAD_SHORTINT;
        case AHEAD_RESINT: return AHEAD_INT;
        case AHEAD_RESBIGINT: return AHEAD_BIGINT;
        case AHEAD_RESOID: return AHEAD_OID;
        default: return t;
    }
}
static int tlarger(int t) { /* v2_larger_t */
    switch (t) {
        case AHEAD_TINYINT: return AHEAD_SHORTINT;
        case AHEAD_SHORTINT: return AHEAD_INT;
        case AHEAD_RESTINY: return AHEAD_RESSHORT;
        case AHEAD_RESSHORT: return AHEAD_RESINT;
        case AHEAD_RESINT: case AHEAD_RESBIGINT: case AHEAD_RESOID: return AHEAD_RESBIGINT;
        default: return AHEAD_BIGINT;
    }
}
static uint64_t msk(int bytes) { return bytes >= 8 ? ~0ull : ((1ull << (8 * bytes)) - 1); }
static uint64_t mulw(uint64_t a, uint64_t b, int bytes) { return (a * b) & msk(bytes); }

static uint64_t ld(const ahead_col* c, uint64_t i) {
    switch (c->type) {
        case AHEAD_VOID: return (uint32_t)(c->seqbase + i);
        default: break;
    }
    switch (tw(c->type)) {
        case 1: return ((const uint8_t*)c->data)[i];
        case 2: return ((const uint16_t*)c->data)[i];
        case 4: return ((const uint32_t*)c->data)[i];
        default: return ((const uint64_t*)c->data)[i];
    }
}
static void st(ahead_col* c, uint64_t i, uint64_t v) {
    if (c->type == AHEAD_VOID || !c->data) return;
    switch (tw(c->type)) {
        case 1: ((uint8_t*)c->data)[i] = (uint8_t)v; break;
        case 2: ((uint16_t*)c->data)[i] = (uint16_t)v; break;
        case 4: ((uint32_t*)c->data)[i] = (uint32_t)v; break;
        default: ((uint64_t*)c->data)[i] = v; break;
    }
}
static void setmeta(ahead_col* c, int type, uint64_t A, uint64_t Ainv, uint64_t umax, uint64_t seq) {
    c->type = type;
    c->A = (uint16_t)A; /* ColumnMetaData::AN_A is a 16-bit A_t */
    c->Ainv = Ainv;
    c->unenc_max = umax;
    c->seqbase = seq;
}
static void copymeta(ahead_col* c, int type, const ahead_col* src) {
    setmeta(c, type, src->A, src->Ainv, src->unenc_max, src->seqbase);
}
/* Default column metadata.  ColumnDescriptor's default constructor passes
 * sizeof(type_t) to ColumnMetaData, which resolves to the oid_t seqbase
 * constructor (include/column_storage/ColumnDescriptor.hpp:39-41,
 * ColumnMetaData.hpp:178-186): A=1, Ainv=1, unencMaxU=0, seqbase=sizeof.
 * A void column's default metadata has seqbase 0. */
static void defmeta(ahead_col* c, int type) { setmeta(c, type, 1, 1, 0, type == AHEAD_VOID ? 0 : (uint64_t)tw(type)); }

/* Largest A of the resint/resoid tables and its inverse (resilience.hpp:99-105)
 * and UNENC_MAX_U of the 64-bit code types (lib/util/resilience.cpp:59-71). */
#define RESOID_A_MAX 65117ull
#define RESOID_AINV_MAX 0x3E36D3BC8D9BC5F5ull
#define RES56_MAX 0x00FFFFFFFFFFFFFFull
static uint64_t type_unenc_max(int t) {
    switch (t) {
        case AHEAD_RESTINY: return 0xFF;
        case AHEAD_RESSHORT: return 0xFFFF;
        case AHEAD_RESINT: return 0xFFFFFFFFull;
        default: return RES56_MAX;
    }
}

/* error vectors */
static void ev_init(ahead_errvec* e, int present) {
    if (!e) return;
    e->count = 0;
    e->present = present;
}
static void ev_push(ahead_errvec* e, uint64_t v) {
    if (!e || !e->present) return;
    if (e->count < e->capacity && e->data) e->data[e->count] = v;
    e->count++;
}

/* ext_euclidean over 2^bits (resilience.hpp:481-516), for odd a. */
uint64_t orc_ainv(uint64_t a, int bits) {
    unsigned __int128 m = (unsigned __int128)1 << bits;
    unsigned __int128 q[130], ra = m, rb = a;
    int n = 0;
    while (rb > 0) {
        q[n++] = ra / rb;
        unsigned __int128 r = ra % rb;
        ra = rb;
        rb = r;
    }
    unsigned __int128 s = 1, t = 0; /* back-substitution, wrapping mod 2^128 */
    for (int j = n; j > 0; --j) {
        unsigned __int128 ns = t;
        unsigned __int128 nt = s - q[j - 1] * t;
        s = ns;
        t = nt;
    }
    unsigned __int128 chk = ((unsigned __int128)a * t) % m;
    if (chk != 1) return 0;
    return (uint64_t)t;
}

/* ------------------------------------------------------------------------ */
/* Predicates (std::less ... std::greater).                                  */
static int cmp(int op, uint64_t a, uint64_t b) {
    switch (op) {
        case AHEAD_CMP_LT: return a < b;
        case AHEAD_CMP_LE: return a <= b;
        case AHEAD_CMP_EQ: return a == b;
        case AHEAD_CMP_NE: return a != b;
        case AHEAD_CMP_GE: return a >= b;
        case AHEAD_CMP_GT: return a > b;
        default: return 0;
    }
}
static int pred(int op1, uint64_t th1, int op2, uint64_t th2, int comb, uint64_t t) {
    if (op2 == AHEAD_CMP_NONE) return cmp(op1, t, th1);
    int a = cmp(op1, t, th1), b = cmp(op2, t, th2);
    return comb == AHEAD_OR ? (a || b) : (a && b);
}
static int op_ok(int op) { return op >= AHEAD_CMP_LT && op <= AHEAD_CMP_GT; }
/* Op<int>(c, 0) of the string selections: c is strcmp's result. */
static int cmp_sign(int op, int c) {
    switch (op) {
        case AHEAD_CMP_LT: return c < 0;
        case AHEAD_CMP_LE: return c <= 0;
        case AHEAD_CMP_EQ: return c == 0;
        case AHEAD_CMP_NE: return c != 0;
        case AHEAD_CMP_GE: return c >= 0;
        case AHEAD_CMP_GT: return c > 0;
        default: return 0;
    }
}

/* selectAN: lib/column_operators/AN/selectAN_scalar.tcc:54-98 (one predicate)
 * and :137-184 (two predicates); the reencoding overloads ignore ATR/ATInvR
 * (selectAN.tcc:51-70). */
int orc_select_an(const ahead_bat* in, int op1, uint64_t th1, int op2, uint64_t th2, int comb,
                  uint64_t aoid, ahead_bat* out, uint64_t cap, ahead_errvec* err) {
    int t = in->tail.type;
    if (in->head.type != AHEAD_VOID || !(t == AHEAD_RESTINY || t == AHEAD_RESSHORT || t == AHEAD_RESINT))
        return AHEAD_BAD_ARG;
    if (!op_ok(op1) || (op2 != AHEAD_CMP_NONE && !op_ok(op2))) return AHEAD_BAD_ARG;
    int w = tw(t);
    uint64_t ainv = in->tail.Ainv & msk(w), umax = in->tail.unenc_max & msk(w);
    th1 &= msk(w);
    th2 &= msk(w);
    ev_init(err, 1);
    uint64_t n = 0;
    for (uint64_t pos = 0; pos < in->count; ++pos) {
        uint64_t v = ld(&in->tail, pos);
        if (mulw(v, ainv, w) > umax) ev_push(err, pos * aoid);
        if (pred(op1, th1, op2, th2, comb, v)) {
            uint64_t oid = (uint32_t)(in->head.seqbase + pos);
            if (n < cap && out->head.data) ((uint64_t*)out->head.data)[n] = oid * RESOID_A_MAX;
            ++n;
        }
    }
    setmeta(&out->head, AHEAD_RESOID, RESOID_A_MAX, RESOID_AINV_MAX, RES56_MAX, 0);
    copymeta(&out->tail, t, &in->tail);
    out->tail.data = NULL; /* only the head is filled (selectAN_scalar.tcc:89-91) */
    out->count = n;
    return n > cap ? AHEAD_CAPACITY : AHEAD_OK;
}

/* String selection: Selection(AN)1/2<..., v2_void_t, v2_str_t>::filter
 * (selectAN_scalar.tcc:98-131, 185-222; Normal/select_scalar.tcc:78-101,
 * 137-165).  Each row is copied into a NUL-terminated buffer and compared with
 * libc strcmp, as the reference does on its str_t tails. */
static int select_str(const char* strs, uint64_t width, uint64_t count, uint64_t seqbase, int op1,
                      const char* th1, int op2, const char* th2, int comb, ahead_bat* out, uint64_t cap,
                      int an) {
    if (!th1 || (op2 != AHEAD_CMP_NONE && !th2)) return AHEAD_BAD_ARG;
    if (!op_ok(op1) || (op2 != AHEAD_CMP_NONE && !op_ok(op2))) return AHEAD_BAD_ARG;
    if (count && (!strs || width == 0)) return AHEAD_BAD_ARG;
    char* row = (char*)calloc((size_t)width + 1, 1);
    if (!row) return AHEAD_NO_MEMORY;
    uint64_t n = 0;
    for (uint64_t pos = 0; pos < count; ++pos) {
        memcpy(row, strs + pos * width, (size_t)width);
        int keep = cmp_sign(op1, strcmp(row, th1));
        if (op2 != AHEAD_CMP_NONE) {
            int b = cmp_sign(op2, strcmp(row, th2));
            keep = comb == AHEAD_OR ? (keep || b) : (keep && b);
        }
        if (keep) {
            uint32_t oid = (uint32_t)(seqbase + pos);
            if (n < cap && out->head.data) {
                if (an) ((uint64_t*)out->head.data)[n] = (uint64_t)oid * RESOID_A_MAX;
                else ((uint32_t*)out->head.data)[n] = oid;
            }
            ++n;
        }
    }
    free(row);
    if (an) setmeta(&out->head, AHEAD_RESOID, RESOID_A_MAX, RESOID_AINV_MAX, RES56_MAX, 0);
    else setmeta(&out->head, AHEAD_OID, 0, 0, 0, 0);
    setmeta(&out->tail, AHEAD_STR, 0, 0, 0, 0);
    out->tail.data = NULL; /* only the head is filled */
    out->count = n;
    return n > cap ? AHEAD_CAPACITY : AHEAD_OK;
}

int orc_select_str_an(const char* strs, uint64_t width, uint64_t count, uint64_t seqbase, int op1,
                      const char* th1, int op2, const char* th2, int comb, ahead_bat* out, uint64_t cap) {
    return select_str(strs, width, count, seqbase, op1, th1, op2, th2, comb, out, cap, 1);
}

int orc_select_str(const char* strs, uint64_t width, uint64_t count, uint64_t seqbase, int op1,
                   const char* th1, int op2, const char* th2, int comb, ahead_bat* out, uint64_t cap) {
    return select_str(strs, width, count, seqbase, op1, th1, op2, th2, comb, out, cap, 0);
}

/* select (unencoded): lib/column_operators/Normal/select_scalar.tcc:53-76,
 * :104-131.  Head: the void head's oid_t; metadata copied by skeleton(). */
int orc_select(const ahead_bat* in, int op1, uint64_t th1, int op2, uint64_t th2, int comb,
               ahead_bat* out, uint64_t cap) {
    int t = in->tail.type;
    if (in->head.type != AHEAD_VOID || t == AHEAD_VOID || t == AHEAD_OID || t == AHEAD_RESOID) return AHEAD_BAD_ARG;
    if (!op_ok(op1) || (op2 != AHEAD_CMP_NONE && !op_ok(op2))) return AHEAD_BAD_ARG;
    int w = tw(t);
    th1 &= msk(w);
    th2 &= msk(w);
    uint64_t n = 0;
    for (uint64_t pos = 0; pos < in->count; ++pos) {
        uint64_t v = ld(&in->tail, pos);
        if (pred(op1, th1, op2, th2, comb, v)) {
            if (n < cap && out->head.data) ((uint32_t*)out->head.data)[n] = (uint32_t)(in->head.seqbase + pos);
            ++n;
        }
    }
    copymeta(&out->head, AHEAD_OID, &in->head);
    copymeta(&out->tail, t, &in->tail);
    out->tail.data = NULL; /* only the head is filled */
    out->count = n;
    return n > cap ? AHEAD_CAPACITY : AHEAD_OK;
}

/* checkAN: lib/column_operators/AN/encdecAN_scalar.tcc:69-94. */
int orc_check_an(const ahead_bat* in, uint64_t ainv, uint64_t unenc_max, uint64_t aoid,
                 ahead_errvec* err) {
    int t = in->tail.type;
    if (!(in->head.type == AHEAD_VOID || in->head.type == AHEAD_OID) || !tenc(t)) return AHEAD_BAD_ARG;
    int w = tw(t);
    ainv &= msk(w);
    unenc_max &= msk(w);
    ev_init(err, 1);
    for (uint64_t i = 0; i < in->count; ++i)
        if (mulw(ld(&in->tail, i), ainv, w) > unenc_max) ev_push(err, i * aoid);
    return AHEAD_OK;
}

/* decodeAN: lib/column_operators/AN/encdecAN_scalar.tcc:96-127 (encoded head
 * only: the template static_asserts it). */
int orc_decode_an(const ahead_bat* in, uint64_t aoid, ahead_bat* out, uint64_t cap,
                  ahead_errvec* err) {
    int h = in->head.type, t = in->tail.type;
    if (h != AHEAD_RESOID || !tenc(t)) return AHEAD_BAD_ARG;
    int w = tw(t);
    uint64_t ainv = in->tail.Ainv & msk(w), umax = in->tail.unenc_max & msk(w);
    int ut = tunenc(t);
    copymeta(&out->head, h, &in->head);
    defmeta(&out->tail, ut);
    ev_init(err, 1);
    out->count = in->count;
    if (in->count > cap) return AHEAD_CAPACITY;
    for (uint64_t pos = 0; pos < in->count; ++pos) {
        uint64_t d = mulw(ld(&in->tail, pos), ainv, w);
        st(&out->head, pos, ld(&in->head, pos));
        st(&out->tail, pos, d & msk(tw(ut)));
        if (d > umax) ev_push(err, pos * aoid);
    }
    return AHEAD_OK;
}

/* checkAndDecodeAN: lib/column_operators/AN/encdecAN_scalar.tcc:178-211 (void
 * head: erroneous rows dropped, vec1 = nullptr) and :129-176 (general head). */
int orc_check_and_decode_an(const ahead_bat* in, uint64_t aoid, ahead_bat* out, uint64_t cap,
                            ahead_errvec* err_head, ahead_errvec* err_tail) {
    int h = in->head.type, t = in->tail.type;
    if (!(h == AHEAD_VOID || h == AHEAD_OID || h == AHEAD_RESOID) || !tenc(t)) return AHEAD_BAD_ARG;
    int wt = tw(t), wh = tw(h);
    uint64_t tainv = in->tail.Ainv & msk(wt), tmax = in->tail.unenc_max & msk(wt);
    uint64_t hainv = in->head.Ainv & msk(wh), hmax = in->head.unenc_max & msk(wh);
    int hence = tenc(h);
    int ut = tunenc(t), uh = tunenc(h);
    uint64_t n = 0;
    if (h == AHEAD_VOID) {
        ev_init(err_head, 0);
        ev_init(err_tail, 1);
        defmeta(&out->head, AHEAD_VOID);
        defmeta(&out->tail, ut);
        for (uint64_t i = 0; i < in->count; ++i) {
            uint64_t d = mulw(ld(&in->tail, i), tainv, wt);
            if (d > tmax) {
                ev_push(err_tail, i * aoid);
            } else {
                if (n < cap) st(&out->tail, n, d);
                ++n;
            }
        }
    } else {
        ev_init(err_head, hence);
        ev_init(err_tail, 1);
        defmeta(&out->head, uh);
        defmeta(&out->tail, ut);
        for (uint64_t pos = 0; pos < in->count; ++pos) {
            uint64_t dh = hence ? mulw(ld(&in->head, pos), hainv, wh) : ld(&in->head, pos);
            uint64_t dt = mulw(ld(&in->tail, pos), tainv, wt);
            int hok = !hence || dh <= hmax;
            if (!hok) ev_push(err_head, pos * aoid);
            int tok = dt <= tmax;
            if (!tok) ev_push(err_tail, pos * aoid);
            if (hok && tok) {
                if (n < cap) {
                    st(&out->head, n, dh);
                    st(&out->tail, n, dt);
                }
                ++n;
            }
        }
    }
    out->count = n;
    return n > cap ? AHEAD_CAPACITY : AHEAD_OK;
}

/* encodeAN (encdecAN_scalar.tcc:43-67): tail * A in the encoded width.  The
 * reference's definition does not compile; this follows its loop. */
int orc_encode_an(const ahead_bat* in, uint64_t A, ahead_bat* out, uint64_t cap) {
    int t = in->tail.type;
    if (in->head.type != AHEAD_VOID || !(t == AHEAD_TINYINT || t == AHEAD_SHORTINT || t == AHEAD_INT)) return AHEAD_BAD_ARG;
    int et = tenctype(t);
    int w = tw(et);
    copymeta(&out->head, AHEAD_VOID, &in->head);
    setmeta(&out->tail, et, A, orc_ainv(A, 8 * w) & msk(w), type_unenc_max(et), 0);
    out->count = in->count;
    if (in->count > cap) return AHEAD_CAPACITY;
    for (uint64_t i = 0; i < in->count; ++i) st(&out->tail, i, mulw(ld(&in->tail, i), A, w));
    return AHEAD_OK;
}

/* ------------------------------------------------------------------------ */
/* A multimap u64 -> u64 keeping insertion order per key (the reference's
 * dense_hash_map<key, std::vector<payload>>).                              */
typedef struct {
    uint64_t* keys;
    int64_t* first; /* entry index of first payload, -1 = empty slot */
    int64_t* last;
    uint64_t cap;   /* slots, power of two */
    uint64_t* pay;
    int64_t* next;
    uint64_t n;
} mmap_t;

static uint64_t mix(uint64_t k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    return k;
}
static int mm_init(mmap_t* m, uint64_t n) {
    uint64_t c = 16;
    while (c < 2 * n + 2) c <<= 1;
    m->cap = c;
    m->keys = (uint64_t*)calloc(c, 8);
    m->first = (int64_t*)malloc(c * 8);
    m->last = (int64_t*)malloc(c * 8);
    m->pay = (uint64_t*)malloc((n + 1) * 8);
    m->next = (int64_t*)malloc((n + 1) * 8);
    m->n = 0;
    if (!m->keys || !m->first || !m->last || !m->pay || !m->next) return -1;
    for (uint64_t i = 0; i < c; ++i) m->first[i] = -1;
    return 0;
}
static void mm_free(mmap_t* m) {
    free(m->keys);
    free(m->first);
    free(m->last);
    free(m->pay);
    free(m->next);
}
static uint64_t mm_slot(const mmap_t* m, uint64_t k) {
    uint64_t s = mix(k) & (m->cap - 1);
    while (m->first[s] >= 0 && m->keys[s] != k) s = (s + 1) & (m->cap - 1);
    return s;
}
static void mm_add(mmap_t* m, uint64_t k, uint64_t p) {
    uint64_t s = mm_slot(m, k);
    int64_t e = (int64_t)m->n++;
    m->pay[e] = p;
    m->next[e] = -1;
    if (m->first[s] < 0) {
        m->keys[s] = k;
        m->first[s] = e;
    } else {
        m->next[m->last[s]] = e;
    }
    m->last[s] = e;
}
static int64_t mm_find(const mmap_t* m, uint64_t k) {
    uint64_t s = mm_slot(m, k);
    return m->first[s];
}

/* Output writer for join results with capacity handling. */
typedef struct {
    ahead_bat* out;
    uint64_t cap, n;
} jw_t;
static void jw_put(jw_t* j, uint64_t h, uint64_t t) {
    if (j->n < j->cap) {
        st(&j->out->head, j->n, h);
        st(&j->out->tail, j->n, t);
    }
    j->n++;
}

/* hashjoinAN: lib/column_operators/AN/hashjoinAN.tcc:54-223; API :552-585.
 * Keys are decoded and cast to the unencoded base type; rows with detected
 * errors are still built/probed. */
int orc_hashjoin_an(const ahead_bat* l, const ahead_bat* r, int reenc_head, uint64_t ah1r,
                    uint64_t ah1invr, int reenc_tail, uint64_t at2r, uint64_t at2invr, int side,
                    uint64_t aoid, ahead_bat* out, uint64_t cap, ahead_errvec* errs) {
    int H1 = l->head.type, T1 = l->tail.type, H2 = r->head.type, T2 = r->tail.type;
    if (!(H1 == AHEAD_VOID || H1 == AHEAD_RESOID) || !(T2 == AHEAD_VOID || T2 == AHEAD_RESOID)) return AHEAD_BAD_ARG;
    if (!(T1 == AHEAD_RESTINY || T1 == AHEAD_RESSHORT || T1 == AHEAD_RESINT)) return AHEAD_BAD_ARG;
    if (!(H2 == AHEAD_RESTINY || H2 == AHEAD_RESSHORT || H2 == AHEAD_RESINT)) return AHEAD_BAD_ARG;
    if (reenc_tail && !reenc_head) return AHEAD_BAD_ARG;
    int eH1 = tenc(H1), eT2 = tenc(T2);
    int wh1e = tw(tenctype(H1)), wt1e = tw(tenctype(T1)), wh2e = tw(tenctype(H2)), wt2e = tw(tenctype(T2));
    int bt1 = tbase(T1), bh2 = tbase(H2);
    int blarger = bt1 >= bh2 ? bt1 : bh2;
    /* getIfEncoded: unencoded columns give 0 */
    uint64_t AH1Inv = eH1 ? l->head.Ainv & msk(wh1e) : 0, AH1Max = l->head.unenc_max & msk(wh1e);
    uint64_t AT1Inv = l->tail.Ainv & msk(wt1e), AT1Max = l->tail.unenc_max & msk(wt1e);
    uint64_t AH2Inv = r->head.Ainv & msk(wh2e), AH2Max = r->head.unenc_max & msk(wh2e);
    uint64_t AT2Inv = eT2 ? r->tail.Ainv & msk(wt2e) : 0, AT2Max = r->tail.unenc_max & msk(wt2e);
    /* mulIfEncoded(AR, AInv): encoded -> (T)(AR*AInv) in the storage type;
     * unencoded -> (T)AR with T = oid_t */
    uint64_t fH1 = eH1 ? mulw(ah1r, AH1Inv, tw(H1)) : (ah1r & 0xFFFFFFFFull);
    uint64_t fT2 = eT2 ? mulw(at2r, AT2Inv, tw(T2)) : (at2r & 0xFFFFFFFFull);
    /* output types and metadata */
    int oH = reenc_head ? tenctype(H1) : tsel(H1);
    int oT = reenc_tail ? tenctype(T2) : tsel(T2);
    if (reenc_head) {
        setmeta(&out->head, oH, ah1r, ah1invr, l->head.unenc_max, 0);
        if (reenc_tail) setmeta(&out->tail, oT, at2r, at2invr, r->tail.unenc_max, 0);
        else setmeta(&out->tail, oT, r->tail.A, r->tail.Ainv, r->tail.unenc_max, 0);
    } else {
        copymeta(&out->head, oH, &l->head);
        copymeta(&out->tail, oT, &r->tail);
    }
    for (int k = 0; k < 4; ++k) ev_init(errs ? &errs[k] : NULL, k == 0 ? eH1 : k == 3 ? eT2 : 1);
    ahead_errvec *v1 = errs ? &errs[0] : NULL, *v2 = errs ? &errs[1] : NULL, *v3 = errs ? &errs[2] : NULL,
                 *v4 = errs ? &errs[3] : NULL;
    jw_t j = {out, cap, 0};
    if (l->count > 0 && r->count > 0) {
        mmap_t m;
        if (side == AHEAD_HASH_LEFT) {
            /* build on the left (:138-170) */
            uint64_t t1max = msk(bt1) & msk(blarger);
            if (mm_init(&m, l->count)) return AHEAD_NO_MEMORY;
            for (uint64_t pos = 0; pos < l->count; ++pos) {
                uint64_t h1 = ld(&l->head, pos);
                if (eH1 && mulw(h1, AH1Inv, wh1e) > AH1Max) ev_push(v1, pos * aoid);
                uint64_t t1 = mulw(ld(&l->tail, pos), AT1Inv, tw(T1));
                if (t1 > AT1Max) ev_push(v2, pos * aoid);
                mm_add(&m, t1 & msk(bt1), h1);
            }
            for (uint64_t pos = 0; pos < r->count; ++pos) {
                uint64_t h2 = mulw(ld(&r->head, pos), AH2Inv, tw(H2));
                if (h2 > AH2Max) ev_push(v3, pos * aoid);
                uint64_t t2 = ld(&r->tail, pos);
                if (eT2 && t2 * AT2Inv > AT2Max) ev_push(v4, pos * aoid);
                if ((h2 & msk(blarger)) <= t1max) {
                    for (int64_t e = mm_find(&m, h2 & msk(bt1)); e >= 0; e = m.next[e]) {
                        uint64_t mh = m.pay[e];
                        jw_put(&j, reenc_head ? mh * fH1 : mh, reenc_tail ? t2 * fT2 : t2);
                    }
                }
            }
        } else {
            /* build on the right (:172-216) */
            uint64_t h2max = msk(bh2) & msk(blarger);
            if (mm_init(&m, r->count)) return AHEAD_NO_MEMORY;
            for (uint64_t pos = 0; pos < r->count; ++pos) {
                uint64_t h2 = mulw(ld(&r->head, pos), AH2Inv, tw(H2));
                if (h2 > AH2Max) ev_push(v3, pos * aoid);
                uint64_t t2 = ld(&r->tail, pos);
                if (eT2 && mulw(t2, AT2Inv, wt2e) > AT2Max) ev_push(v4, pos * aoid);
                mm_add(&m, h2 & msk(bh2), t2);
            }
            for (uint64_t pos = 0; pos < l->count; ++pos) {
                uint64_t h1 = ld(&l->head, pos);
                if (eH1 && mulw(h1, AH1Inv, wh1e) > AH1Max) ev_push(v1, pos * aoid);
                uint64_t t1 = mulw(ld(&l->tail, pos), AT1Inv, tw(T1));
                if (t1 > AT1Max) ev_push(v2, pos * aoid);
                if ((t1 & msk(blarger)) <= h2max) {
                    for (int64_t e = mm_find(&m, t1 & msk(bh2)); e >= 0; e = m.next[e]) {
                        uint64_t mt = m.pay[e];
                        jw_put(&j, reenc_head ? h1 * fH1 : h1, reenc_tail ? mt * fT2 : mt);
                    }
                }
            }
        }
        mm_free(&m);
    }
    out->count = j.n;
    return j.n > cap ? AHEAD_CAPACITY : AHEAD_OK;
}

/* hashjoin (unencoded): lib/column_operators/Normal/hashjoin.tcc:38-90.  Keys
 * are the raw stored values. */
int orc_hashjoin(const ahead_bat* l, const ahead_bat* r, int side, ahead_bat* out, uint64_t cap) {
    int H1 = l->head.type, T1 = l->tail.type, H2 = r->head.type, T2 = r->tail.type;
    if (!(H1 == AHEAD_VOID || H1 == AHEAD_OID) || !(T2 == AHEAD_VOID || T2 == AHEAD_OID)) return AHEAD_BAD_ARG;
    if (T1 != H2 || T1 == AHEAD_VOID || T1 == AHEAD_OID || T1 == AHEAD_BIGINT || T1 == AHEAD_RESBIGINT || T1 == AHEAD_RESOID)
        return AHEAD_BAD_ARG;
    int w = tw(T1);
    copymeta(&out->head, tsel(H1), &l->head);
    copymeta(&out->tail, tsel(T2), &r->tail);
    jw_t j = {out, cap, 0};
    if (l->count > 0 && r->count > 0) {
        mmap_t m;
        if (side == AHEAD_HASH_LEFT) {
            if (mm_init(&m, l->count)) return AHEAD_NO_MEMORY;
            for (uint64_t i = 0; i < l->count; ++i) mm_add(&m, ld(&l->tail, i), ld(&l->head, i));
            for (uint64_t i = 0; i < r->count; ++i) {
                uint64_t h2 = ld(&r->head, i);
                if (h2 <= msk(w))
                    for (int64_t e = mm_find(&m, h2); e >= 0; e = m.next[e]) jw_put(&j, m.pay[e], ld(&r->tail, i));
            }
        } else {
            if (mm_init(&m, r->count)) return AHEAD_NO_MEMORY;
            for (uint64_t i = 0; i < r->count; ++i) mm_add(&m, ld(&r->head, i), ld(&r->tail, i));
            for (uint64_t i = 0; i < l->count; ++i) {
                uint64_t t1 = ld(&l->tail, i);
                if (t1 <= msk(w))
                    for (int64_t e = mm_find(&m, t1); e >= 0; e = m.next[e]) jw_put(&j, ld(&l->head, i), m.pay[e]);
            }
        }
        mm_free(&m);
    }
    out->count = j.n;
    return j.n > cap ? AHEAD_CAPACITY : AHEAD_OK;
}

/* ------------------------------------------------------------------------ */
/* matchjoinAN: lib/column_operators/AN/matchjoinAN.tcc.
 *   general merge                 :46-144
 *   <H1, void, void, T2>          :146-224
 *   <H1, resoid, void, T2>        :226-302                                   */

/* ANhelper<V>::mulIfEncoded(x, f): (storage)(x*f) when encoded, else x. */
static uint64_t dec_if(int type, uint64_t x, uint64_t f) {
    return tenc(type) ? mulw(x, f, tw(type)) : x;
}
/* ANhelper<V>::getIfEncoded(meta): the value in the select storage type, or 0 */
static uint64_t get_if(int type, uint64_t v) { return tenc(type) ? v & msk(tw(type)) : 0; }

int orc_matchjoin_an(const ahead_bat* a, const ahead_bat* b, int reenc, uint64_t ah1r,
                     uint64_t ah1invr, uint64_t at2r, uint64_t at2invr, uint64_t aoid,
                     ahead_bat* out, uint64_t cap, ahead_errvec* errs) {
    int H1 = a->head.type, T1 = a->tail.type, H2 = b->head.type, T2 = b->tail.type;
    int vv = T1 == AHEAD_VOID && H2 == AHEAD_VOID;
    int rv = T1 == AHEAD_RESOID && H2 == AHEAD_VOID;
    int gm = T1 == AHEAD_RESOID && H2 == AHEAD_RESOID;
    int mv = T1 == AHEAD_VOID && H2 == AHEAD_RESOID;
    if (!(H1 == AHEAD_VOID || H1 == AHEAD_RESOID || H1 == AHEAD_RESINT)) return AHEAD_BAD_ARG;
    if (!(vv || rv || gm || mv)) return AHEAD_BAD_ARG;
    if (H1 == AHEAD_VOID && T1 == AHEAD_VOID) return AHEAD_BAD_ARG;
    if (T2 == AHEAD_VOID && !gm) return AHEAD_BAD_ARG;
    if (!(T2 == AHEAD_VOID || tenc(T2))) return AHEAD_BAD_ARG;
    if (reenc && (H1 == AHEAD_VOID || T2 == AHEAD_VOID)) return AHEAD_UNSUPPORTED;
    uint64_t AH1Inv = get_if(H1, a->head.Ainv), AH1Max = get_if(H1, a->head.unenc_max);
    uint64_t AT1Inv = get_if(T1, a->tail.Ainv), AT1Max = get_if(T1, a->tail.unenc_max);
    uint64_t AH2Inv = get_if(H2, b->head.Ainv), AH2Max = get_if(H2, b->head.unenc_max);
    uint64_t AT2Inv = get_if(T2, b->tail.Ainv), AT2Max = get_if(T2, b->tail.unenc_max);
    uint64_t fH1 = dec_if(H1, ah1r, AH1Inv), fT2 = dec_if(T2, at2r, AT2Inv);
    int oH = reenc ? tenctype(H1) : tsel(H1);
    int oT = reenc ? tenctype(T2) : tsel(T2);
    if (reenc) {
        setmeta(&out->head, oH, ah1r, ah1invr, a->head.unenc_max, 0);
        /* the positional form stores (uint16_t)AT2R (:261-263); same value */
        setmeta(&out->tail, oT, at2r, at2invr, b->tail.unenc_max, 0);
    } else {
        copymeta(&out->head, oH, &a->head);
        copymeta(&out->tail, oT, &b->tail);
    }
    ahead_errvec *v1 = errs ? &errs[0] : NULL, *v2 = errs ? &errs[1] : NULL, *v3 = errs ? &errs[2] : NULL,
                 *v4 = errs ? &errs[3] : NULL;
    jw_t j = {out, cap, 0};
#define EMIT(h, t) jw_put(&j, reenc ? dec_if(H1, (h), fH1) : (h), reenc ? dec_if(T2, (t), fT2) : (t))
    if (gm || mv) {
        ev_init(v1, tenc(H1));
        ev_init(v2, tenc(T1));
        ev_init(v3, tenc(H2));
        ev_init(v4, tenc(T2));
        uint64_t p1 = 0, p2 = 0, n1 = a->count, n2 = b->count;
        while (p1 < n1 && p2 < n2) {
            uint64_t h2 = dec_if(H2, ld(&b->head, p2), AH2Inv);
            if (tenc(H2) && h2 > AH2Max) ev_push(v3, p2 * aoid);
            if (tenc(T2) && dec_if(T2, ld(&b->tail, p2), AT2Inv) > AT2Max) ev_push(v4, p2 * aoid);
            uint64_t t1 = dec_if(T1, ld(&a->tail, p1), AT1Inv);
            int valid;
            while ((valid = p1 < n1) && t1 < h2) {
                if (tenc(H1) && dec_if(H1, ld(&a->head, p1), AH1Inv) > AH1Max) ev_push(v1, p1 * aoid);
                if (tenc(T1) && t1 > AT1Max) ev_push(v2, p1 * aoid);
                ++p1;
                if (p1 < n1) t1 = dec_if(T1, ld(&a->tail, p1), AT1Inv);
            }
            if (valid) {
                while ((valid = p2 < n2) && t1 > h2) {
                    if (tenc(H2) && h2 > AH2Max) ev_push(v3, p2 * aoid);
                    if (tenc(T2) && dec_if(T2, ld(&b->tail, p2), AT2Inv) > AT2Max) ev_push(v4, p2 * aoid);
                    ++p2;
                    if (p2 < n2) h2 = dec_if(H2, ld(&b->head, p2), AH2Inv);
                }
                if (valid && t1 == h2) {
                    EMIT(ld(&a->head, p1), ld(&b->tail, p2));
                    ++p1;
                    ++p2;
                }
            }
        }
    } else if (vv) {
        ev_init(v1, tenc(H1));
        ev_init(v2, 0);
        ev_init(v3, 0);
        ev_init(v4, tenc(T2));
        uint64_t p1 = 0, p2 = 0, n1 = a->count, n2 = b->count;
        if (n1 > 0 && n2 > 0) {
            if (a->tail.seqbase < b->head.seqbase) {
                uint64_t x = b->head.seqbase;
                for (; p1 < n1 && p2 < n2 && (uint64_t)(uint32_t)(a->tail.seqbase + p1) < x; ++p1)
                    if (tenc(H1) && mulw(ld(&a->head, p1), AH1Inv, tw(H1)) > AH1Max) ev_push(v1, p1 * aoid);
            } else if (a->tail.seqbase > b->head.seqbase) {
                uint64_t x = a->tail.seqbase;
                for (; p1 < n1 && p2 < n2 && (uint64_t)(uint32_t)(b->head.seqbase + p2) < x; ++p2)
                    if (tenc(T2) && mulw(ld(&b->tail, p2), AT2Inv, tw(T2)) > AT2Max) ev_push(v4, p2 * aoid);
            }
            for (; p1 < n1 && p2 < n2; ++p1, ++p2) {
                if (tenc(H1) && mulw(ld(&a->head, p1), AH1Inv, tw(H1)) > AH1Max) ev_push(v1, p1 * aoid);
                if (tenc(T2) && mulw(ld(&b->tail, p2), AT2Inv, tw(T2)) > AT2Max) ev_push(v4, p2 * aoid);
                EMIT(ld(&a->head, p1), ld(&b->tail, p2));
            }
        }
    } else { /* rv: positional fetch through a resoid tail */
        ev_init(v1, tenc(H1));
        ev_init(v2, 1);
        ev_init(v3, 0);
        ev_init(v4, tenc(T2));
        uint64_t sz = (uint32_t)b->count; /* BAT::size() is an oid_t */
        for (uint64_t p1 = 0; p1 < a->count; ++p1) {
            uint64_t h1 = ld(&a->head, p1);
            if (tenc(H1) && h1 * AH1Inv > AH1Max) ev_push(v1, p1 * aoid);
            uint64_t pos2 = ld(&a->tail, p1) * AT1Inv;
            if (pos2 >= sz) {
                ev_push(v2, p1 * aoid);
            } else {
                uint64_t t2 = ld(&b->tail, pos2);
                if (tenc(T2) && dec_if(T2, t2, AT2Inv) > AT2Max) ev_push(v4, pos2 * aoid);
                else EMIT(h1, t2);
            }
        }
    }
#undef EMIT
    out->count = j.n;
    return j.n > cap ? AHEAD_CAPACITY : AHEAD_OK;
}

/* matchjoin (unencoded): lib/column_operators/Normal/matchjoin.tcc:37-157. */
int orc_matchjoin(const ahead_bat* a, const ahead_bat* b, ahead_bat* out, uint64_t cap) {
    int H1 = a->head.type, T1 = a->tail.type, H2 = b->head.type, T2 = b->tail.type;
    /* heads instantiated in lib/column_operators/Normal/matchjoin.hpp:36-50 (strings aside) */
    if (H1 == AHEAD_RESOID || !(T1 == AHEAD_VOID || T1 == AHEAD_OID) ||
        !(H2 == AHEAD_VOID || H2 == AHEAD_OID) || T2 == AHEAD_VOID || T2 == AHEAD_RESOID)
        return AHEAD_BAD_ARG;
    if (H1 == AHEAD_VOID && T1 == AHEAD_VOID) return AHEAD_BAD_ARG;
    copymeta(&out->head, tsel(H1), &a->head);
    copymeta(&out->tail, tsel(T2), &b->tail);
    jw_t j = {out, cap, 0};
    uint64_t n1 = a->count, n2 = b->count;
    if (T1 == AHEAD_VOID && H2 == AHEAD_VOID) {
        uint64_t p1 = 0, p2 = 0;
        if (n1 > 0 && n2 > 0) {
            if (a->tail.seqbase < b->head.seqbase) {
                for (; p1 < n1 && p2 < n2 && (uint64_t)(uint32_t)(a->tail.seqbase + p1) < b->head.seqbase; ++p1) {}
            } else if (a->tail.seqbase > b->head.seqbase) {
                for (; p1 < n1 && p2 < n2 && (uint64_t)(uint32_t)(b->head.seqbase + p2) < a->tail.seqbase; ++p2) {}
            }
            for (; p1 < n1 && p2 < n2; ++p1, ++p2) jw_put(&j, ld(&a->head, p1), ld(&b->tail, p2));
        }
    } else if (T1 == AHEAD_OID && H2 == AHEAD_VOID) {
        for (uint64_t p1 = 0; p1 < n1; ++p1) {
            uint64_t pos = ld(&a->tail, p1);
            if (pos < n2) jw_put(&j, ld(&a->head, p1), ld(&b->tail, pos));
        }
    } else {
        uint64_t p1 = 0, p2 = 0;
        while (p1 < n1 && p2 < n2) {
            uint64_t h2 = ld(&b->head, p2), t1 = ld(&a->tail, p1);
            int valid;
            while ((valid = p1 < n1) && t1 < h2) {
                ++p1;
                if (p1 < n1) t1 = ld(&a->tail, p1);
            }
            if (valid) {
                while ((valid = p2 < n2) && t1 > h2) {
                    ++p2;
                    if (p2 < n2) h2 = ld(&b->head, p2);
                }
                if (valid && t1 == h2) {
                    jw_put(&j, ld(&a->head, p1), ld(&b->tail, p2));
                    ++p1;
                    ++p2;
                }
            }
        }
    }
    out->count = j.n;
    return j.n > cap ? AHEAD_CAPACITY : AHEAD_OK;
}

/* fetchjoinAN: lib/column_operators/AN/matchjoinAN.tcc:304-354.  The check
 * `(t2 * AT2inv) > AT2unencMaxU` (:342) has no cast: for 16-bit codes the
 * product is formed in a 32-bit int and compared signed. */
int orc_fetchjoin_an(const ahead_bat* a, const ahead_bat* b, int reenc, uint64_t atr,
                     uint64_t atrinv, uint64_t aoid, ahead_bat* out, uint64_t cap,
                     ahead_errvec* errs) {
    int T2 = b->tail.type;
    if (a->head.type != AHEAD_VOID || a->tail.type != AHEAD_RESOID || b->head.type != AHEAD_VOID || !tenc(T2))
        return AHEAD_BAD_ARG;
    int w = tw(T2);
    uint64_t AT1inv = a->tail.Ainv, AT2inv = b->tail.Ainv & msk(w), AT2max = b->tail.unenc_max & msk(w);
    uint64_t fac = 1;
    copymeta(&out->head, AHEAD_VOID, &a->head);
    copymeta(&out->tail, T2, &b->tail);
    if (reenc) {
        out->tail.A = (uint16_t)atr;
        out->tail.Ainv = atrinv;
        uint64_t inv = orc_ainv(b->tail.A, 8 * w);
        fac = mulw(atr, inv, w);
    }
    ahead_errvec *v1 = errs ? &errs[0] : NULL, *v2 = errs ? &errs[1] : NULL;
    ev_init(v1, 1);
    ev_init(v2, 1);
    uint64_t vsz = b->count, n = 0;
    for (uint64_t i = 0; i < a->count; ++i) {
        uint64_t t1 = ld(&a->tail, i) * AT1inv;
        if (t1 >= vsz) {
            ev_push(v1, i * aoid);
            continue;
        }
        uint64_t t2 = ld(&b->tail, t1) & msk(w);
        int bad;
        if (w == 2) bad = (int32_t)(uint32_t)(t2 * AT2inv) > (int32_t)AT2max;
        else bad = mulw(t2, AT2inv, w) > AT2max;
        if (bad) {
            ev_push(v2, t1 * aoid);
        } else {
            if (n < cap) st(&out->tail, n, reenc ? mulw(t2, fac, w) : t2);
            ++n;
        }
    }
    out->count = n;
    return n > cap ? AHEAD_CAPACITY : AHEAD_OK;
}

/* fetchjoin (unencoded): lib/column_operators/Normal/matchjoin.tcc:159-178. */
int orc_fetchjoin(const ahead_bat* a, const ahead_bat* b, ahead_bat* out, uint64_t cap) {
    int T2 = b->tail.type;
    if (a->head.type != AHEAD_VOID || a->tail.type != AHEAD_OID || b->head.type != AHEAD_VOID || T2 == AHEAD_VOID ||
        T2 == AHEAD_RESOID)
        return AHEAD_BAD_ARG;
    copymeta(&out->head, AHEAD_VOID, &a->head);
    copymeta(&out->tail, T2, &b->tail);
    uint64_t n = 0;
    for (uint64_t i = 0; i < a->count; ++i) {
        uint64_t pos = ld(&a->tail, i);
        if (pos >= b->count) continue;
        if (n < cap) st(&out->tail, n, ld(&b->tail, pos));
        ++n;
    }
    out->count = n;
    return n > cap ? AHEAD_CAPACITY : AHEAD_OK;
}

/* ------------------------------------------------------------------------ */
/* A map u64 -> u64 (the reference's dense_hash_map dictionaries).          */
typedef struct {
    uint64_t *keys, *vals;
    uint8_t* used;
    uint64_t cap;
} dmap_t;
static int dm_init(dmap_t* m, uint64_t n) {
    uint64_t c = 16;
    while (c < 2 * n + 2) c <<= 1;
    m->cap = c;
    m->keys = (uint64_t*)malloc(c * 8);
    m->vals = (uint64_t*)malloc(c * 8);
    m->used = (uint8_t*)calloc(c, 1);
    return (m->keys && m->vals && m->used) ? 0 : -1;
}
static void dm_free(dmap_t* m) {
    free(m->keys);
    free(m->vals);
    free(m->used);
}
static int dm_find(const dmap_t* m, uint64_t k, uint64_t* s_out) {
    uint64_t s = mix(k) & (m->cap - 1);
    while (m->used[s] && m->keys[s] != k) s = (s + 1) & (m->cap - 1);
    *s_out = s;
    return m->used[s];
}

/* groupbyAN unary: lib/column_operators/AN/groupbyAN.tcc:51-94. */
int orc_groupby_an(const ahead_bat* in, uint64_t aoid, uint64_t aoidinv, ahead_bat* gids,
                   ahead_bat* firsts, uint64_t cap, ahead_errvec* errs) {
    int H = in->head.type, T = in->tail.type;
    if (!(H == AHEAD_VOID || H == AHEAD_OID || H == AHEAD_RESOID) || !tenc(T)) return AHEAD_BAD_ARG;
    int eH = tenc(H);
    uint64_t HAInv = get_if(H, in->head.Ainv), HMax = get_if(H, in->head.unenc_max);
    uint64_t TAInv = get_if(T, in->tail.Ainv), TMax = get_if(T, in->tail.unenc_max);
    ahead_errvec *v1 = errs ? &errs[0] : NULL, *v2 = errs ? &errs[1] : NULL;
    ev_init(v1, eH);
    ev_init(v2, 1);
    setmeta(&gids->head, AHEAD_VOID, 1, 1, 0, 0);
    setmeta(&gids->tail, AHEAD_RESOID, aoid, aoidinv, RES56_MAX, 0);
    setmeta(&firsts->head, AHEAD_VOID, 1, 1, 0, 0);
    setmeta(&firsts->tail, AHEAD_RESOID, aoid, aoidinv, RES56_MAX, 0);
    dmap_t m;
    if (dm_init(&m, in->count)) return AHEAD_NO_MEMORY;
    uint64_t ng = 0;
    for (uint64_t i = 0; i < in->count; ++i) {
        uint64_t hraw = ld(&in->head, i);
        uint64_t h = dec_if(H, hraw, HAInv);
        if (eH && h > HMax) ev_push(v1, i * aoid);
        uint64_t t1 = dec_if(T, ld(&in->tail, i), TAInv);
        if (t1 > TMax) ev_push(v2, i * aoid);
        uint64_t key = t1 & msk(tbase(T)), s;
        uint64_t g;
        if (dm_find(&m, key, &s)) {
            g = m.vals[s];
        } else {
            g = ng;
            if (ng < cap) st(&firsts->tail, ng, hraw * aoid);
            ++ng;
            m.used[s] = 1;
            m.keys[s] = key;
            m.vals[s] = (uint32_t)g; /* stored as oid_t */
        }
        if (i < cap) st(&gids->tail, i, g * aoid);
    }
    dm_free(&m);
    gids->count = in->count;
    firsts->count = ng;
    return (in->count > cap || ng > cap) ? AHEAD_CAPACITY : AHEAD_OK;
}

/* groupbyAN binary: lib/column_operators/AN/groupbyAN.tcc:99-165.  The
 * dictionary stores the encoded GID in an oid_t (:150), so repeated rows get
 * its low 32 bits while the first row of a group gets all 64. */
int orc_groupby2_an(const ahead_bat* in, const ahead_bat* grouping, uint64_t ngroups,
                    uint64_t aoid, uint64_t aoidinv, ahead_bat* gids, ahead_bat* firsts,
                    uint64_t cap, ahead_errvec* errs) {
    int H = in->head.type, T = in->tail.type;
    if (!(H == AHEAD_VOID || H == AHEAD_OID || H == AHEAD_RESOID) || !tenc(T)) return AHEAD_BAD_ARG;
    if (grouping->head.type != AHEAD_VOID || grouping->tail.type != AHEAD_RESOID) return AHEAD_BAD_ARG;
    if (in->count != grouping->count) return AHEAD_SIZE_MISMATCH;
    int eH = tenc(H);
    uint64_t HAInv = get_if(H, in->head.Ainv), HMax = get_if(H, in->head.unenc_max);
    uint64_t TAInv = get_if(T, in->tail.Ainv), TMax = get_if(T, in->tail.unenc_max);
    uint64_t GAInv = grouping->tail.Ainv, GMax = grouping->tail.unenc_max;
    int wl = tw(tlarger(T));
    ahead_errvec *v1 = errs ? &errs[0] : NULL, *v2 = errs ? &errs[1] : NULL, *v3 = errs ? &errs[2] : NULL;
    ev_init(v1, eH);
    ev_init(v2, 1);
    ev_init(v3, 1);
    setmeta(&gids->head, AHEAD_VOID, 1, 1, 0, 0);
    setmeta(&gids->tail, AHEAD_RESOID, aoid, aoidinv, RES56_MAX, 0);
    setmeta(&firsts->head, AHEAD_VOID, 1, 1, 0, 0);
    setmeta(&firsts->tail, AHEAD_RESOID, aoid, aoidinv, RES56_MAX, 0);
    dmap_t m;
    if (dm_init(&m, in->count)) return AHEAD_NO_MEMORY;
    uint64_t ng = 0;
    for (uint64_t i = 0; i < in->count; ++i) {
        uint64_t h = dec_if(H, ld(&in->head, i), HAInv);
        if (eH && h > HMax) ev_push(v1, i * aoid);
        uint64_t t = dec_if(T, ld(&in->tail, i), TAInv);
        if (t > TMax) ev_push(v2, i * aoid);
        uint64_t g = ld(&grouping->tail, i) * GAInv;
        if (g > GMax) ev_push(v3, i * aoid);
        uint64_t key = ((t & msk(wl)) * (ngroups & msk(wl)) + (g & msk(wl))) & msk(wl), s;
        uint64_t val;
        if (dm_find(&m, key, &s)) {
            val = m.vals[s];
        } else {
            val = ng * aoid;
            if (ng < cap) st(&firsts->tail, ng, h * aoid);
            ++ng;
            m.used[s] = 1;
            m.keys[s] = key;
            m.vals[s] = (uint32_t)val;
        }
        if (i < cap) st(&gids->tail, i, val);
    }
    dm_free(&m);
    gids->count = in->count;
    firsts->count = ng;
    return (in->count > cap || ng > cap) ? AHEAD_CAPACITY : AHEAD_OK;
}

/* aggregate_sum_groupedAN: lib/column_operators/AN/aggregateAN.tcc:35-120. */
int orc_aggregate_sum_grouped_an(const ahead_bat* in, const ahead_bat* grouping,
                                 uint64_t ngroups, int result_type, uint64_t ar, uint64_t arinv,
                                 uint64_t aoid, ahead_bat* out, ahead_errvec* errs) {
    int H = in->head.type, T = in->tail.type;
    if (result_type != AHEAD_RESBIGINT) return AHEAD_BAD_ARG;
    if (!(H == AHEAD_VOID || H == AHEAD_OID || H == AHEAD_RESOID)) return AHEAD_BAD_ARG;
    if (!(T == AHEAD_INT || T == AHEAD_RESINT || T == AHEAD_RESBIGINT || T == AHEAD_RESSHORT || T == AHEAD_RESTINY))
        return AHEAD_BAD_ARG;
    if (grouping->head.type != AHEAD_VOID || grouping->tail.type != AHEAD_RESOID) return AHEAD_BAD_ARG;
    if (in->count != grouping->count) return AHEAD_SIZE_MISMATCH;
    int eH = tenc(H), eT = tenc(T);
    int wh = tw(tenctype(H)), wt = tw(tenctype(T));
    uint64_t AHinv = in->head.Ainv & msk(wh), AHmax = in->head.unenc_max & msk(wh);
    uint64_t AT = in->tail.A & msk(wt), ATinv = in->tail.Ainv & msk(wt), ATmax = in->tail.unenc_max & msk(wt);
    uint64_t AGinv = grouping->tail.Ainv, AGmax = grouping->tail.unenc_max;
    uint64_t enc = ar * (eT ? orc_ainv(AT, 64) : 1ull);
    ahead_errvec *vh = errs ? &errs[0] : NULL, *vt = errs ? &errs[1] : NULL, *vg = errs ? &errs[2] : NULL;
    ev_init(vh, eH);
    ev_init(vt, eT);
    ev_init(vg, 1);
    defmeta(&out->head, AHEAD_VOID);
    setmeta(&out->tail, AHEAD_RESBIGINT, ar, arinv, RES56_MAX, 0);
    uint64_t* sums = (uint64_t*)out->tail.data;
    for (uint64_t g = 0; g < ngroups; ++g) sums[g] = 0;
    for (uint64_t i = 0; i < in->count; ++i) {
        if (eH && mulw(ld(&in->head, i), AHinv, wh) > AHmax) ev_push(vh, i * aoid);
        uint64_t t = ld(&in->tail, i);
        if (eT && mulw(t, ATinv, wt) > ATmax) ev_push(vt, i * aoid);
        uint64_t gid = ld(&grouping->tail, i) * AGinv;
        if (gid > AGmax) ev_push(vg, i * aoid);
        else if (gid < ngroups) sums[gid] += t * enc;
    }
    out->count = ngroups;
    return AHEAD_OK;
}

/* aggregate_mul_sumAN: lib/column_operators/AN/aggregateAN_scalar.tcc:56-131. */
int orc_aggregate_mul_sum_an(const ahead_bat* a, const ahead_bat* b, int result_type,
                             uint64_t init, uint64_t ra, uint64_t rainv, uint64_t aoid,
                             uint64_t* total, ahead_errvec* errs) {
    (void)rainv;
    int T1 = a->tail.type, T2 = b->tail.type;
    if (result_type != AHEAD_RESBIGINT) return AHEAD_BAD_ARG;
    if (!(a->head.type == AHEAD_VOID || a->head.type == AHEAD_RESOID) ||
        !(b->head.type == AHEAD_VOID || b->head.type == AHEAD_RESOID))
        return AHEAD_BAD_ARG;
    if (!(T1 == AHEAD_RESTINY || T1 == AHEAD_RESSHORT || T1 == AHEAD_RESINT)) return AHEAD_BAD_ARG;
    if (!(T2 == AHEAD_RESTINY || T2 == AHEAD_RESSHORT || T2 == AHEAD_RESINT)) return AHEAD_BAD_ARG;
    int w1 = tw(T1), w2 = tw(T2);
    uint64_t AT1 = a->tail.A & msk(w1), AT1inv = a->tail.Ainv & msk(w1), AT1max = a->tail.unenc_max & msk(w1);
    uint64_t AT2 = b->tail.A & msk(w2), AT2inv = b->tail.Ainv & msk(w2), AT2max = b->tail.unenc_max & msk(w2);
    uint64_t enc = ra * orc_ainv(AT1, 64) * orc_ainv(AT2, 64);
    ahead_errvec *v1 = errs ? &errs[0] : NULL, *v2 = errs ? &errs[1] : NULL;
    ev_init(v1, 1);
    ev_init(v2, 1);
    uint64_t tot = init, n = a->count < b->count ? a->count : b->count;
    for (uint64_t i = 0; i < n; ++i) {
        uint64_t t1 = ld(&a->tail, i), t2 = ld(&b->tail, i);
        if (mulw(t1, AT1inv, w1) > AT1max) ev_push(v1, i * aoid);
        if (mulw(t2, AT2inv, w2) > AT2max) ev_push(v2, i * aoid);
        tot += t1 * t2;
    }
    *total = tot * enc;
    return AHEAD_OK;
}

/* aggregate_mul_sum (unencoded): lib/column_operators/Normal/aggregate_scalar.tcc:69-90. */
int orc_aggregate_mul_sum(const ahead_bat* a, const ahead_bat* b, int result_type,
                          uint64_t init, uint64_t* total) {
    if (result_type != AHEAD_BIGINT) return AHEAD_BAD_ARG;
    uint64_t tot = init, n = a->count < b->count ? a->count : b->count;
    for (uint64_t i = 0; i < n; ++i) tot += ld(&a->tail, i) * ld(&b->tail, i);
    *total = tot;
    return AHEAD_OK;
}

/* Tail types the unencoded groupby is instantiated for
 * (lib/column_operators/Normal/groupby.cpp:36-48, strings aside). */
static int plain_groupable(int t) {
    return t == AHEAD_OID || t == AHEAD_TINYINT || t == AHEAD_SHORTINT || t == AHEAD_INT || t == AHEAD_RESOID ||
           t == AHEAD_RESTINY || t == AHEAD_RESSHORT || t == AHEAD_RESINT;
}

/* groupby unary: lib/column_operators/Normal/groupby.tcc:51-76.  A dictionary
 * from the tail value (hash<T> is the identity, miscellaneous.hpp:81-93) to the
 * group id; a new id is the number of groups so far, and the group's first
 * row contributes its head to the second output. */
int orc_groupby(const ahead_bat* in, ahead_bat* gids, ahead_bat* firsts, uint64_t cap) {
    int H = in->head.type, T = in->tail.type;
    if (!(H == AHEAD_VOID || H == AHEAD_OID) || !plain_groupable(T)) return AHEAD_BAD_ARG;
    defmeta(&gids->head, AHEAD_VOID);
    defmeta(&gids->tail, AHEAD_OID);
    defmeta(&firsts->head, AHEAD_VOID);
    defmeta(&firsts->tail, AHEAD_OID);
    dmap_t m;
    if (dm_init(&m, in->count)) return AHEAD_NO_MEMORY;
    uint64_t ng = 0;
    for (uint64_t i = 0; i < in->count; ++i) {
        uint64_t key = ld(&in->tail, i), s, g;
        if (dm_find(&m, key, &s)) {
            g = m.vals[s];
        } else {
            g = ng;
            if (ng < cap) st(&firsts->tail, ng, (uint32_t)ld(&in->head, i));
            ++ng;
            m.used[s] = 1;
            m.keys[s] = key;
            m.vals[s] = (uint32_t)g;
        }
        if (i < cap) st(&gids->tail, i, g);
    }
    dm_free(&m);
    gids->count = in->count;
    firsts->count = ng;
    return (in->count > cap || ng > cap) ? AHEAD_CAPACITY : AHEAD_OK;
}

/* groupby binary: lib/column_operators/Normal/groupby.tcc:81-119.  The key is
 * t * numGroups + g in the tail's larger type (v2_larger_t), so it wraps in
 * that width. */
int orc_groupby2(const ahead_bat* in, const ahead_bat* grouping, uint64_t ngroups, ahead_bat* gids,
                 ahead_bat* firsts, uint64_t cap) {
    int H = in->head.type, T = in->tail.type;
    if (!(H == AHEAD_VOID || H == AHEAD_OID) || !plain_groupable(T)) return AHEAD_BAD_ARG;
    if (grouping->head.type != AHEAD_VOID || grouping->tail.type != AHEAD_OID) return AHEAD_BAD_ARG;
    if (in->count != grouping->count) return AHEAD_SIZE_MISMATCH;
    int wl = tw(tlarger(T));
    defmeta(&gids->head, AHEAD_VOID);
    defmeta(&gids->tail, AHEAD_OID);
    defmeta(&firsts->head, AHEAD_VOID);
    defmeta(&firsts->tail, AHEAD_OID);
    dmap_t m;
    if (dm_init(&m, in->count)) return AHEAD_NO_MEMORY;
    uint64_t ng = 0;
    for (uint64_t i = 0; i < in->count; ++i) {
        uint64_t t = ld(&in->tail, i) & msk(wl), g = ld(&grouping->tail, i) & msk(wl);
        uint64_t key = (t * (ngroups & msk(wl)) + g) & msk(wl), s, gid;
        if (dm_find(&m, key, &s)) {
            gid = m.vals[s];
        } else {
            gid = ng;
            if (ng < cap) st(&firsts->tail, ng, (uint32_t)ld(&in->head, i));
            ++ng;
            m.used[s] = 1;
            m.keys[s] = key;
            m.vals[s] = (uint32_t)gid;
        }
        if (i < cap) st(&gids->tail, i, gid);
    }
    dm_free(&m);
    gids->count = in->count;
    firsts->count = ng;
    return (in->count > cap || ng > cap) ? AHEAD_CAPACITY : AHEAD_OK;
}

/* aggregate_sum_grouped<bigint>: lib/column_operators/Normal/aggregate.tcc:
 * 32-50 (instantiated for int tails with void or oid heads,
 * aggregate.cpp:62-66).  A group id outside [0, numGroups) indexes past the
 * reference's vector; such rows are skipped here. */
int orc_aggregate_sum_grouped(const ahead_bat* in, const ahead_bat* grouping, uint64_t ngroups,
                              int result_type, ahead_bat* out) {
    int H = in->head.type, T = in->tail.type;
    if (result_type != AHEAD_BIGINT || !(H == AHEAD_VOID || H == AHEAD_OID) || T != AHEAD_INT) return AHEAD_BAD_ARG;
    if (grouping->head.type != AHEAD_VOID || grouping->tail.type != AHEAD_OID) return AHEAD_BAD_ARG;
    if (in->count != grouping->count) return AHEAD_SIZE_MISMATCH;
    defmeta(&out->head, AHEAD_VOID);
    defmeta(&out->tail, AHEAD_BIGINT);
    for (uint64_t g = 0; g < ngroups; ++g) st(&out->tail, g, 0);
    for (uint64_t i = 0; i < in->count; ++i) {
        uint64_t g = ld(&grouping->tail, i);
        if (g < ngroups) st(&out->tail, g, ld(&out->tail, g) + ld(&in->tail, i));
    }
    out->count = ngroups;
    return AHEAD_OK;
}

/* aggregate_sum<Result>: lib/column_operators/Normal/aggregate_scalar.tcc:
 * 47-58, instantiated for oid heads (aggregate.cpp:28-41). */
int orc_aggregate_sum(const ahead_bat* in, int result_type, uint64_t* total) {
    int T = in->tail.type;
    if (in->head.type != AHEAD_OID) return AHEAD_BAD_ARG;
    if (!(T == AHEAD_TINYINT || T == AHEAD_SHORTINT || T == AHEAD_INT || T == AHEAD_BIGINT)) return AHEAD_BAD_ARG;
    if (!(result_type == AHEAD_TINYINT || result_type == AHEAD_SHORTINT || result_type == AHEAD_INT ||
          result_type == AHEAD_BIGINT) || tw(result_type) < tw(T))
        return AHEAD_BAD_ARG;
    uint64_t sum = 0;
    for (uint64_t i = 0; i < in->count; ++i) sum = (sum + (ld(&in->tail, i) & msk(tw(result_type)))) & msk(tw(result_type));
    *total = sum;
    return AHEAD_OK;
}

/* arithmetic<Op, Result>: lib/column_operators/Normal/arithmetic_scalar.tcc:
 * 46-67, instantiated for (int, int) -> int and (resint, resint) -> resint
 * (arithmetic.cpp:45-46).  Op(t1, t2) in the tails' type; the result keeps
 * the first input's metadata (skeleton, miscellaneous.hpp:122-132).
 * Division by zero is undefined in the reference; here it yields 0. */
int orc_arithmetic(int op, int result_type, const ahead_bat* a, const ahead_bat* b, ahead_bat* out) {
    int T1 = a->tail.type, T2 = b->tail.type;
    if (a->head.type != AHEAD_VOID || b->head.type != AHEAD_VOID) return AHEAD_BAD_ARG;
    if (!((T1 == AHEAD_INT && T2 == AHEAD_INT && result_type == AHEAD_INT) ||
          (T1 == AHEAD_RESINT && T2 == AHEAD_RESINT && result_type == AHEAD_RESINT)))
        return AHEAD_BAD_ARG;
    if (op < AHEAD_ADD || op > AHEAD_DIV) return AHEAD_BAD_ARG;
    if (a->count != b->count) return AHEAD_SIZE_MISMATCH;
    copymeta(&out->head, AHEAD_VOID, &a->head);
    copymeta(&out->tail, result_type, &a->tail);
    const uint64_t m = msk(tw(T1));
    for (uint64_t i = 0; i < a->count; ++i) {
        uint64_t x = ld(&a->tail, i), y = ld(&b->tail, i), r;
        switch (op) {
            case AHEAD_ADD: r = x + y; break;
            case AHEAD_SUB: r = x - y; break;
            case AHEAD_MUL: r = x * y; break;
            default: r = y ? x / y : 0; break;
        }
        st(&out->tail, i, r & m);
    }
    out->count = a->count;
    return AHEAD_OK;
}

/* arithmeticAN: lib/column_operators/AN/arithmeticAN_scalar.tcc:48-111. */
int orc_arithmetic_an(int op, int result_type, const ahead_bat* a, const ahead_bat* b,
                      uint64_t ar, uint64_t arinv, uint64_t aoid, ahead_bat* out,
                      ahead_errvec* errs) {
    int T1 = a->tail.type, T2 = b->tail.type;
    if (!(result_type == AHEAD_RESINT || result_type == AHEAD_RESBIGINT)) return AHEAD_BAD_ARG;
    if (a->head.type != AHEAD_VOID || b->head.type != AHEAD_VOID) return AHEAD_BAD_ARG;
    if (!(T1 == AHEAD_RESTINY || T1 == AHEAD_RESSHORT || T1 == AHEAD_RESINT)) return AHEAD_BAD_ARG;
    if (!(T2 == AHEAD_RESTINY || T2 == AHEAD_RESSHORT || T2 == AHEAD_RESINT)) return AHEAD_BAD_ARG;
    if (op < AHEAD_ADD || op > AHEAD_DIV) return AHEAD_BAD_ARG;
    if (a->count != b->count) return AHEAD_SIZE_MISMATCH;
    int w1 = tw(T1), w2 = tw(T2);
    uint64_t AT1inv = a->tail.Ainv & msk(w1), T1max = a->tail.unenc_max & msk(w1);
    uint64_t AT2inv = b->tail.Ainv & msk(w2), T2max = b->tail.unenc_max & msk(w2);
    ahead_errvec* v = errs;
    ev_init(v ? &v[0] : NULL, 0);
    ev_init(v ? &v[1] : NULL, 1);
    ev_init(v ? &v[2] : NULL, 0);
    ev_init(v ? &v[3] : NULL, 1);
    defmeta(&out->head, AHEAD_VOID);
    setmeta(&out->tail, result_type, ar, arinv, type_unenc_max(result_type), 0);
    for (uint64_t pos = 0; pos < a->count; ++pos) {
        uint64_t t1 = mulw(ld(&a->tail, pos), AT1inv, w1);
        if (t1 > T1max) ev_push(v ? &v[1] : NULL, pos * aoid);
        uint64_t t2 = mulw(ld(&b->tail, pos), AT2inv, w2);
        if (t2 > T2max) ev_push(v ? &v[3] : NULL, pos * aoid);
        uint64_t x = t1 * ar, y = t2 * ar, r;
        switch (op) {
            case AHEAD_ADD: r = x + y; break;
            case AHEAD_SUB: r = x - y; break;
            case AHEAD_MUL: r = x * y; break;
            default: r = y ? x / y : 0; break;
        }
        st(&out->tail, pos, r);
    }
    out->count = a->count;
    return AHEAD_OK;
}

/* hashjoinAN with a string right tail: hashjoinAN.tcc:225-367.  Its steps are
 * those of the general join (:54-223) with the right tail's strings as the
 * payload, except that with the right side hashed the left head is decoded
 * before it is emitted (:339, :352: h1 * A^-1, times the re-encoding factor).
 * Restated as the general join over the right rows' ids, then the payload
 * strings and the decoded head. */
int orc_hashjoin_str_an(const ahead_bat* l, const ahead_bat* r, const char* r_strs, uint64_t width,
                        int reenc_head, uint64_t ah1r, uint64_t ah1invr, int side, uint64_t aoid,
                        ahead_bat* out, uint64_t cap, ahead_errvec* errs) {
    if (r->count && (!r_strs || width == 0)) return AHEAD_BAD_ARG;
    ahead_bat rr = *r;
    memset(&rr.tail, 0, sizeof(rr.tail));
    rr.tail.type = AHEAD_VOID;
    uint64_t rcap = (out->head.data && out->tail.data) ? cap : 0;
    uint32_t* rows = (uint32_t*)malloc((size_t)(rcap ? rcap : 1) * 4);
    if (!rows) return AHEAD_NO_MEMORY;
    ahead_bat o = *out;
    o.tail.data = rows;
    int rc = orc_hashjoin_an(l, &rr, reenc_head, ah1r, ah1invr, 0, 1, 1, side, aoid, &o, rcap, errs);
    if (rc == AHEAD_OK) {
        int decode = side == AHEAD_HASH_RIGHT && tenc(l->head.type);
        int hw = tw(o.head.type);
        for (uint64_t i = 0; i < o.count; ++i) {
            memcpy((char*)out->tail.data + i * width, r_strs + (uint64_t)rows[i] * width, (size_t)width);
            if (decode) {
                if (hw == 8) ((uint64_t*)o.head.data)[i] *= l->head.Ainv;
                else ((uint32_t*)o.head.data)[i] *= (uint32_t)l->head.Ainv;
            }
        }
    }
    if (rc == AHEAD_OK && side == AHEAD_HASH_LEFT && l->tail.type == AHEAD_RESTINY && errs && l->count && r->count) {
        /* The string join's left build checks `(t1 * AT1Inv) > AT1UnencMaxU`
         * on the restiny code without a cast (hashjoinAN.tcc:290): both u16
         * operands are promoted to int, so the product is not reduced mod 2^16;
         * the compiled reference wraps it to 32 bits and compares signed. */
        uint32_t ainv = (uint32_t)(l->tail.Ainv & 0xFFFF);
        uint32_t umax = (uint32_t)(l->tail.unenc_max & 0xFFFF);
        ev_init(&errs[1], 1);
        for (uint64_t pos = 0; pos < l->count; ++pos) {
            uint32_t t = ((const uint16_t*)l->tail.data)[pos];
            if ((int32_t)(t * ainv) > (int32_t)umax) ev_push(&errs[1], pos * aoid);
        }
    }
    free(rows);
    void* tdata = out->tail.data;
    out->head = o.head;
    out->count = o.count;
    setmeta(&out->tail, AHEAD_STR, 0, 0, 0, 0);
    out->tail.data = tdata;
    if (errs) {
        errs[3].present = 0;
        errs[3].count = 0;
    }
    return rc;
}

/* fetchjoinAN with a string tail: FetchjoinAN<v2_str_t, false>::run,
 * matchjoinAN.tcc:304-354.  The string tail is not encoded, so there is no
 * tail check and vec2 is not present; an OID at or past the column's end is
 * reported in vec1 (the reference's `>` reads one past the end: the single
 * intended divergence); every other row's slot is copied as it is. */
int orc_fetchjoin_str_an(const ahead_bat* a, const char* strs, uint64_t width, uint64_t count, uint64_t aoid,
                         char* out, uint64_t cap, uint64_t* n_out, ahead_errvec* errs) {
    if (a->head.type != AHEAD_VOID || a->tail.type != AHEAD_RESOID || !width || (count && !strs))
        return AHEAD_BAD_ARG;
    ahead_errvec *v1 = errs ? &errs[0] : NULL, *v2 = errs ? &errs[1] : NULL;
    ev_init(v1, 1);
    ev_init(v2, 0);
    uint64_t n = 0;
    for (uint64_t i = 0; i < a->count; ++i) {
        uint64_t t1 = ld(&a->tail, i) * a->tail.Ainv;
        if (t1 >= count) {
            ev_push(v1, i * aoid);
            continue;
        }
        if (out && n < cap) memcpy(out + n * width, strs + t1 * width, (size_t)width);
        ++n;
    }
    *n_out = n;
    return n > cap ? AHEAD_CAPACITY : AHEAD_OK;
}

/* hash<str_t>::get (miscellaneous.hpp:99-119): the Java string hash of the
 * row's chars up to its NUL (at most `width`), in size_t; each char is a
 * signed char promoted to int, and the multiplier's update (x31) goes through
 * an int: (int)(m << 5) - m. */
static uint64_t str_hash(const char* s, uint64_t width) {
    size_t len = 0;
    while (len < width && s[len]) ++len;
    uint64_t hash = 0, mult = 1;
    for (int64_t i = (int64_t)len - 1; i >= 0; --i) {
        hash += (uint64_t)(int64_t)(signed char)s[i] * mult;
        int32_t shifted = (int32_t)(uint32_t)(mult << 5);
        mult = (uint64_t)(int64_t)shifted - mult;
    }
    return hash;
}

/* groupbyAN binary over a string tail: groupbyAN.tcc:99-165 with hash<str_t>
 * and the larger type v2_bigint_t, so the dictionary key is hash(row) *
 * numGroups + g in 64 bits (strings with equal hashes share groups, as in the
 * reference).  The head is void: a group's first OID is (seqbase + row) *
 * AOID; vec1 (head) and vec2 (tail) are not present, vec3 reports grouping
 * codes that fail their check. */
int orc_groupby2_str_an(const char* strs, uint64_t width, uint64_t count, uint64_t seqbase,
                        const ahead_bat* grouping, uint64_t ngroups, uint64_t aoid, uint64_t aoidinv,
                        ahead_bat* gids, ahead_bat* firsts, uint64_t cap, ahead_errvec* errs) {
    if (!width || (count && !strs)) return AHEAD_BAD_ARG;
    if (grouping->head.type != AHEAD_VOID || grouping->tail.type != AHEAD_RESOID) return AHEAD_BAD_ARG;
    if (count != grouping->count) return AHEAD_SIZE_MISMATCH;
    uint64_t GAInv = grouping->tail.Ainv, GMax = grouping->tail.unenc_max;
    ahead_errvec *v1 = errs ? &errs[0] : NULL, *v2 = errs ? &errs[1] : NULL, *v3 = errs ? &errs[2] : NULL;
    ev_init(v1, 0);
    ev_init(v2, 0);
    ev_init(v3, 1);
    setmeta(&gids->head, AHEAD_VOID, 1, 1, 0, 0);
    setmeta(&gids->tail, AHEAD_RESOID, aoid, aoidinv, RES56_MAX, 0);
    setmeta(&firsts->head, AHEAD_VOID, 1, 1, 0, 0);
    setmeta(&firsts->tail, AHEAD_RESOID, aoid, aoidinv, RES56_MAX, 0);
    dmap_t m;
    if (dm_init(&m, count)) return AHEAD_NO_MEMORY;
    uint64_t ng = 0;
    for (uint64_t i = 0; i < count; ++i) {
        uint64_t g = ld(&grouping->tail, i) * GAInv;
        if (g > GMax) ev_push(v3, i * aoid);
        uint64_t key = str_hash(strs + i * width, width) * ngroups + g, s;
        uint64_t val;
        if (dm_find(&m, key, &s)) {
            val = m.vals[s];
        } else {
            val = ng * aoid;
            if (ng < cap) st(&firsts->tail, ng, (seqbase + i) * aoid);
            ++ng;
            m.used[s] = 1;
            m.keys[s] = key;
            m.vals[s] = (uint32_t)val;
        }
        if (i < cap) st(&gids->tail, i, val);
    }
    dm_free(&m);
    gids->count = count;
    firsts->count = ng;
    return (count > cap || ng > cap) ? AHEAD_CAPACITY : AHEAD_OK;
}

/* fetchjoin over a string tail: Normal/matchjoin.tcc:144-160 (Fetchjoin<T2>
 * with T2 = v2_str_t): the slot of every listed OID, no checks; an OID past
 * the column's end is skipped (the reference reads past its vector). */
int orc_fetchjoin_str(const ahead_bat* a, const char* strs, uint64_t width, uint64_t count, char* out, uint64_t cap,
                      uint64_t* n_out) {
    if (a->head.type != AHEAD_VOID || a->tail.type != AHEAD_OID || !width || (count && !strs)) return AHEAD_BAD_ARG;
    uint64_t n = 0;
    for (uint64_t i = 0; i < a->count; ++i) {
        uint64_t pos = ld(&a->tail, i);
        if (pos >= count) continue;
        if (out && n < cap) memcpy(out + n * width, strs + pos * width, (size_t)width);
        ++n;
    }
    *n_out = n;
    return n > cap ? AHEAD_CAPACITY : AHEAD_OK;
}

/* groupby binary over a string BAT: Normal/groupby.tcc:85-121 with hash<str_t>
 * and the larger type v2_bigint_t: key = hash(row) * numGroups + g; group ids
 * and first heads (seqbase + row) as oid_t. */
int orc_groupby2_str(const char* strs, uint64_t width, uint64_t count, uint64_t seqbase, const ahead_bat* grouping,
                     uint64_t ngroups, ahead_bat* gids, ahead_bat* firsts, uint64_t cap) {
    if (!width || (count && !strs)) return AHEAD_BAD_ARG;
    if (grouping->head.type != AHEAD_VOID || grouping->tail.type != AHEAD_OID) return AHEAD_BAD_ARG;
    if (count != grouping->count) return AHEAD_SIZE_MISMATCH;
    defmeta(&gids->head, AHEAD_VOID);
    defmeta(&gids->tail, AHEAD_OID);
    defmeta(&firsts->head, AHEAD_VOID);
    defmeta(&firsts->tail, AHEAD_OID);
    dmap_t m;
    if (dm_init(&m, count)) return AHEAD_NO_MEMORY;
    uint64_t ng = 0;
    for (uint64_t i = 0; i < count; ++i) {
        uint64_t key = str_hash(strs + i * width, width) * ngroups + ld(&grouping->tail, i), s, gid;
        if (dm_find(&m, key, &s)) {
            gid = m.vals[s];
        } else {
            gid = ng;
            if (ng < cap) st(&firsts->tail, ng, (uint32_t)(seqbase + i));
            ++ng;
            m.used[s] = 1;
            m.keys[s] = key;
            m.vals[s] = (uint32_t)gid;
        }
        if (i < cap) st(&gids->tail, i, gid);
    }
    dm_free(&m);
    gids->count = count;
    firsts->count = ng;
    return (count > cap || ng > cap) ? AHEAD_CAPACITY : AHEAD_OK;
}
