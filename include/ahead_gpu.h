/*
 * ahead_gpu.h -- C ABI of the B200 AN-hardened operator library
 * (libahead_b200.so).
 *
 * Each entry point replaces one operator of the reference's operator API
 * (include/column_operators/OperatorsAN.hpp and Operators.hpp in the
 * reference project; the citation on each declaration names the template it
 * stands in for).  Template parameters of the reference become runtime
 * arguments: column types travel in ahead_bat, predicates as ahead_cmp codes.
 *
 * Conventions
 *   - All data pointers inside ahead_bat / ahead_errvec are DEVICE pointers.
 *   - Output BATs: the caller passes head.data / tail.data buffers of `cap`
 *     rows (8 bytes per row is always enough); the library fills in the
 *     output column types and AN metadata, writes the rows at the output
 *     type's width and sets `count`.  If `count` > `cap` the call returns
 *     AHEAD_CAPACITY and only the first `cap` rows are written.
 *   - Error-position vectors are written in the reference's scan order
 *     (row * A_OID, ascending scan position); `count` is always exact, at most
 *     `capacity` entries are stored, `present` = 0 marks the reference's
 *     nullptr vector of an unencoded column.
 *   - Every call is stream-ordered on the context's stream and returns after
 *     the output counts are known on the host (the reference's operators are
 *     synchronous and return materialised BATs).
 *   - Corrupted data is never an error status: detected AN errors are data.
 */
#ifndef AHEAD_GPU_H
#define AHEAD_GPU_H

#include <stddef.h>
#include <stdint.h>

#include "ahead_types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ahead_ctx ahead_ctx;

/* ---------------------------------------------------------------- context */
/* Create a context on `device` issuing work on `stream` (a cudaStream_t; NULL
 * creates a private non-blocking stream).  The context owns a growable device
 * scratch arena and a pinned host staging area.  No reference counterpart:
 * the reference runs on the host and allocates per call. */
int ahead_ctx_create(int device, void* stream, ahead_ctx** out);
void ahead_ctx_destroy(ahead_ctx* ctx);
void* ahead_ctx_stream(ahead_ctx* ctx);
/* Human-readable detail of the last failing call on this context. */
const char* ahead_ctx_last_error(ahead_ctx* ctx);
/* Number of kernels this context has launched (for launch accounting). */
uint64_t ahead_ctx_launches(ahead_ctx* ctx);
/* Bytes of device scratch the context holds (its growable arena; 0 before
 * the first operator that needed scratch). */
uint64_t ahead_ctx_scratch_bytes(ahead_ctx* ctx);
const char* ahead_status_string(int status);

/* ------------------------------------------------------------- selection */
/* selectAN<Op>(arg, th, AOID) and selectAN<Op1,Op2,Comb>(arg, th1, th2, AOID)
 * (OperatorsAN.hpp:164-195; lib/column_operators/AN/selectAN_scalar.tcc:54-184).
 * Input: void head, restiny/resshort/resint tail.  Thresholds compare against
 * the codes.  Output head: resoid codes oid*65117 (tail left empty). */
int ahead_gpu_select_an(ahead_ctx* ctx, const ahead_bat* in, int op1, uint64_t th1, int op2,
                        uint64_t th2, int comb, uint64_t aoid, ahead_bat* out, uint64_t cap,
                        ahead_errvec* err);
/* select<Op>(arg, th) / select<Op1,Op2,Comb> (Operators.hpp:104-118;
 * lib/column_operators/Normal/select_scalar.tcc:53-131).  Output head: oid_t. */
int ahead_gpu_select(ahead_ctx* ctx, const ahead_bat* in, int op1, uint64_t th1, int op2,
                     uint64_t th2, int comb, ahead_bat* out, uint64_t cap);

/* selectAN<Op>(BAT<void, str>, threshold, AOID) and selectAN<Op1,Op2,Comb>
 * over a string tail (lib/column_operators/AN/selectAN_scalar.tcc:98-131,
 * 185-222; instantiated at lib/column_operators/AN/selectAN.cpp:140,151):
 * a row is kept when Op(strcmp(row, threshold), 0) holds.  `strs` holds
 * `count` rows of `width` bytes each (device memory); a row's string ends at
 * its first NUL or after `width` bytes.  The thresholds are NUL-terminated
 * host strings of at most AHEAD_STR_TH_MAX bytes (AHEAD_UNSUPPORTED beyond).
 * Output head: resoid codes (seqbase + i) * 65117.  No error vector: a string
 * column carries no AN code (the reference returns a nullptr vector). */
#define AHEAD_STR_TH_MAX 255
int ahead_gpu_select_str_an(ahead_ctx* ctx, const char* strs, uint64_t width, uint64_t count,
                            uint64_t seqbase, int op1, const char* th1, int op2, const char* th2,
                            int comb, ahead_bat* out, uint64_t cap);
/* select<Op>(BAT<void, str>, threshold) / select<Op1,Op2,Comb>
 * (lib/column_operators/Normal/select_scalar.tcc:78-101, 137-165).  Output
 * head: oid_t seqbase + i. */
int ahead_gpu_select_str(ahead_ctx* ctx, const char* strs, uint64_t width, uint64_t count,
                         uint64_t seqbase, int op1, const char* th1, int op2, const char* th2,
                         int comb, ahead_bat* out, uint64_t cap);

/* ------------------------------------------------------ check and decode */
/* checkAN (OperatorsAN.hpp:145-150; encdecAN_scalar.tcc:69-94). */
int ahead_gpu_check_an(ahead_ctx* ctx, const ahead_bat* in, uint64_t ainv, uint64_t unenc_max,
                       uint64_t aoid, ahead_errvec* err);
/* checkAN without any allocation: the same results as ahead_gpu_check_an, with
 * its scratch in a fixed per-device array instead of the context's growable
 * arena (for callers under a fixed device-memory budget, or that must not
 * trigger the device-wide synchronisation of cudaFree).  At most 16,777,216
 * rows per call (AHEAD_CAPACITY beyond, nothing launched); the first call on a
 * device after a context is created there resolves the array's address; a
 * call waits for its stream before it returns, so it cannot run inside stream
 * capture; calls must not overlap on one device (the scratch is shared).  No
 * counterpart in the reference. */
int ahead_gpu_check_an_noalloc(ahead_ctx* ctx, const ahead_bat* in, uint64_t ainv, uint64_t unenc_max,
                               uint64_t aoid, ahead_errvec* err);
/* decodeAN (OperatorsAN.hpp:152-155; encdecAN_scalar.tcc:96-127). */
int ahead_gpu_decode_an(ahead_ctx* ctx, const ahead_bat* in, uint64_t aoid, ahead_bat* out,
                        uint64_t cap, ahead_errvec* err);
/* checkAndDecodeAN (OperatorsAN.hpp:157-161; encdecAN_scalar.tcc:129-219). */
int ahead_gpu_check_and_decode_an(ahead_ctx* ctx, const ahead_bat* in, uint64_t aoid,
                                  ahead_bat* out, uint64_t cap, ahead_errvec* err_head,
                                  ahead_errvec* err_tail);
/* encodeAN (OperatorsAN.hpp:139-143; encdecAN_scalar.tcc:43-67). */
int ahead_gpu_encode_an(ahead_ctx* ctx, const ahead_bat* in, uint64_t A, ahead_bat* out,
                        uint64_t cap);

/* ------------------------------------------------------------------ joins */
/* hashjoinAN, plain / re-encoded head / re-encoded head and tail
 * (OperatorsAN.hpp:60-90; lib/column_operators/AN/hashjoinAN.tcc:54-223,
 * 552-585).  errs[0..3] = head1, tail1, head2, tail2. */
int ahead_gpu_hashjoin_an(ahead_ctx* ctx, const ahead_bat* l, const ahead_bat* r, int reenc_head,
                          uint64_t ah1r, uint64_t ah1invr, int reenc_tail, uint64_t at2r,
                          uint64_t at2invr, int side, uint64_t aoid, ahead_bat* out, uint64_t cap,
                          ahead_errvec* errs);
/* hashjoinAN with a string right tail, plain / re-encoded head
 * (hashjoinAN.tcc:225-367; the same three overloads at :552-585).  `r` gives
 * the right head (its tail is not read); the right tail is `r_strs`, r->count
 * slots of `width` bytes (device memory).  out->head.data receives the heads,
 * out->tail.data `cap` slots of `width` bytes: the matched row's slot, copied
 * whole.  With the right side hashed (the default) the reference emits the
 * DECODED left head (h1 * A^-1, times the re-encoding factor when re-encoding,
 * hashjoinAN.tcc:339,352); hashing the left side emits the left head as it is.
 * Hashing the left side with a restiny left tail, the tail check there is the
 * reference's unreduced one (hashjoinAN.tcc:290: the u16 product promoted to
 * int, wrapped to 32 bits, compared signed), so it reports more rows than
 * the general join does.
 * errs[0..2] = head1, tail1, head2; errs[3] is never present. */
int ahead_gpu_hashjoin_str_an(ahead_ctx* ctx, const ahead_bat* l, const ahead_bat* r, const char* r_strs,
                              uint64_t width, int reenc_head, uint64_t ah1r, uint64_t ah1invr, int side,
                              uint64_t aoid, ahead_bat* out, uint64_t cap, ahead_errvec* errs);
/* fetchjoinAN with a string tail (FetchjoinAN<v2_str_t, false>,
 * matchjoinAN.tcc:304-354): `a` is a (void, resoid) OID list into `count`
 * string slots of `width` bytes (device).  The fetched slots go to `out`
 * (`cap` slots, device), their number to *n_out.  errs[0] = OIDs at or past
 * the column's end (row * aoid); errs[1] is never present (strings are not
 * encoded). */
int ahead_gpu_fetchjoin_str_an(ahead_ctx* ctx, const ahead_bat* a, const char* strs, uint64_t width, uint64_t count,
                               uint64_t aoid, char* out, uint64_t cap, uint64_t* n_out, ahead_errvec* errs);
/* groupbyAN binary over a string tail (groupbyAN.tcc:99-165 with hash<str_t>,
 * lib/column_operators/miscellaneous.hpp:99-119): a row's key is the
 * Java-style hash of its string (chars up to its NUL) times `ngroups` plus its
 * decoded group id, in 64 bits; groups are numbered by first occurrence.  The
 * head is void (`seqbase`): a group's first OID is (seqbase + row) * aoid.
 * errs[0], errs[1] are never present; errs[2] = grouping codes that fail their
 * check. */
int ahead_gpu_groupby2_str_an(ahead_ctx* ctx, const char* strs, uint64_t width, uint64_t count, uint64_t seqbase,
                              const ahead_bat* grouping, uint64_t ngroups, uint64_t aoid, uint64_t aoidinv,
                              ahead_bat* gids, ahead_bat* firsts, uint64_t cap, ahead_errvec* errs);
/* The unencoded twins: fetchjoin over a string tail (Normal/matchjoin.tcc:
 * 144-160; a (void, oid) list, no checks, an OID past the column skipped) and
 * the binary groupby over a string BAT (Normal/groupby.tcc:85-121, the same
 * string hash; oid_t group ids and first heads). */
int ahead_gpu_fetchjoin_str(ahead_ctx* ctx, const ahead_bat* a, const char* strs, uint64_t width, uint64_t count,
                            char* out, uint64_t cap, uint64_t* n_out);
int ahead_gpu_groupby2_str(ahead_ctx* ctx, const char* strs, uint64_t width, uint64_t count, uint64_t seqbase,
                           const ahead_bat* grouping, uint64_t ngroups, ahead_bat* gids, ahead_bat* firsts,
                           uint64_t cap);
/* hashjoin (Operators.hpp:66-71; lib/column_operators/Normal/hashjoin.tcc:38-90). */
int ahead_gpu_hashjoin(ahead_ctx* ctx, const ahead_bat* l, const ahead_bat* r, int side,
                       ahead_bat* out, uint64_t cap);
/* matchjoinAN (OperatorsAN.hpp:33-58; lib/column_operators/AN/matchjoinAN.tcc:46-302):
 * the general merge, the (void tail, void head) and the (resoid tail, void
 * head) positional forms.  errs[0..3] = head1, tail1, head2, tail2. */
int ahead_gpu_matchjoin_an(ahead_ctx* ctx, const ahead_bat* a, const ahead_bat* b, int reenc,
                           uint64_t ah1r, uint64_t ah1invr, uint64_t at2r, uint64_t at2invr,
                           uint64_t aoid, ahead_bat* out, uint64_t cap, ahead_errvec* errs);
/* matchjoin (Operators.hpp:53-57; lib/column_operators/Normal/matchjoin.tcc:37-157). */
int ahead_gpu_matchjoin(ahead_ctx* ctx, const ahead_bat* a, const ahead_bat* b, ahead_bat* out,
                        uint64_t cap);
/* fetchjoinAN, plain / re-encoded (OperatorsAN.hpp:92-106;
 * lib/column_operators/AN/matchjoinAN.tcc:304-354).  errs[0] = bad OID,
 * errs[1] = corrupt fetched value. */
int ahead_gpu_fetchjoin_an(ahead_ctx* ctx, const ahead_bat* a, const ahead_bat* b, int reenc,
                           uint64_t atr, uint64_t atrinv, uint64_t aoid, ahead_bat* out,
                           uint64_t cap, ahead_errvec* errs);
/* fetchjoin (Operators.hpp:59-63; lib/column_operators/Normal/matchjoin.tcc:159-178). */
int ahead_gpu_fetchjoin(ahead_ctx* ctx, const ahead_bat* a, const ahead_bat* b, ahead_bat* out,
                        uint64_t cap);

/* ------------------------------------------------- grouping / aggregation */
/* groupbyAN unary (OperatorsAN.hpp:108-112; groupbyAN.tcc:51-94, 181-189).
 * gids: void -> encoded GID per row; firsts: void -> encoded first OID per group. */
int ahead_gpu_groupby_an(ahead_ctx* ctx, const ahead_bat* in, uint64_t aoid, uint64_t aoidinv,
                         ahead_bat* gids, ahead_bat* firsts, uint64_t cap, ahead_errvec* errs);
/* groupbyAN binary (OperatorsAN.hpp:114-121; groupbyAN.tcc:99-165, 204-211). */
int ahead_gpu_groupby2_an(ahead_ctx* ctx, const ahead_bat* in, const ahead_bat* grouping,
                          uint64_t ngroups, uint64_t aoid, uint64_t aoidinv, ahead_bat* gids,
                          ahead_bat* firsts, uint64_t cap, ahead_errvec* errs);
/* aggregate_sum_groupedAN<Result> (OperatorsAN.hpp:123-131; aggregateAN.tcc:35-120).
 * out->tail receives ngroups AN-coded sums.  errs = head, tail, grouping. */
int ahead_gpu_aggregate_sum_grouped_an(ahead_ctx* ctx, const ahead_bat* in,
                                       const ahead_bat* grouping, uint64_t ngroups,
                                       int result_type, uint64_t ar, uint64_t arinv, uint64_t aoid,
                                       ahead_bat* out, ahead_errvec* errs);
/* aggregate_mul_sumAN<Result> (OperatorsAN.hpp:205-214; aggregateAN_scalar.tcc:56-131). */
int ahead_gpu_aggregate_mul_sum_an(ahead_ctx* ctx, const ahead_bat* a, const ahead_bat* b,
                                   int result_type, uint64_t init, uint64_t ra, uint64_t rainv,
                                   uint64_t aoid, uint64_t* total, ahead_errvec* errs);
/* aggregate_mul_sum<Result> (Operators.hpp:133-138; Normal/aggregate_scalar.tcc:69-90). */
int ahead_gpu_aggregate_mul_sum(ahead_ctx* ctx, const ahead_bat* a, const ahead_bat* b,
                                int result_type, uint64_t init, uint64_t* total);
/* groupby unary / binary (Operators.hpp:75-84; Normal/groupby.tcc:51-150):
 * gids (void, oid) numbered by first occurrence, firsts (void, oid) = the head
 * of each group's first row; binary keys are t * numGroups + g in the tail's
 * larger type. */
int ahead_gpu_groupby(ahead_ctx* ctx, const ahead_bat* in, ahead_bat* gids, ahead_bat* firsts, uint64_t cap);
int ahead_gpu_groupby2(ahead_ctx* ctx, const ahead_bat* in, const ahead_bat* grouping, uint64_t ngroups,
                       ahead_bat* gids, ahead_bat* firsts, uint64_t cap);
/* aggregate_sum_grouped<bigint> (Operators.hpp:86-91; Normal/aggregate.tcc:32-50):
 * out->tail holds ngroups sums (caller capacity >= ngroups). */
int ahead_gpu_aggregate_sum_grouped(ahead_ctx* ctx, const ahead_bat* in, const ahead_bat* grouping,
                                    uint64_t ngroups, int result_type, ahead_bat* out);
/* aggregate_sum<Result> (Operators.hpp:115-119; Normal/aggregate_scalar.tcc:47-58). */
int ahead_gpu_aggregate_sum(ahead_ctx* ctx, const ahead_bat* in, int result_type, uint64_t* total);
/* arithmetic<Op,Result> (Operators.hpp:108-113; Normal/arithmetic_scalar.tcc:46-82):
 * (int, int) -> int and (resint, resint) -> resint on the raw values. */
int ahead_gpu_arithmetic(ahead_ctx* ctx, int op, int result_type, const ahead_bat* a, const ahead_bat* b,
                         ahead_bat* out);

/* arithmeticAN<Op,Result> (OperatorsAN.hpp:196-203; arithmeticAN_scalar.tcc:48-111).
 * errs = head1, tail1, head2, tail2. */
int ahead_gpu_arithmetic_an(ahead_ctx* ctx, int op, int result_type, const ahead_bat* a,
                            const ahead_bat* b, uint64_t ar, uint64_t arinv, uint64_t aoid,
                            ahead_bat* out, ahead_errvec* errs);

/* ------------------------------------------------------ fused star joins */
/* A star join over the SSB-shaped schema, fused into one scan of the fact
 * table for a batch of up to 64 queries.  It computes exactly what the
 * operator-at-a-time composition of the reference's AN operators computes
 * (the SSB query programs, e.g. tools/ssbm/ssbm-q41_continuous.cpp:97-216):
 * dimension predicates on codes, the first join probing the whole foreign-key
 * column with hashjoinAN semantics (corrupt keys are decoded, truncated to 32
 * bits and probed), later foreign keys and the measures fetched positionally
 * (rows with a corrupt value are dropped), price*discount via
 * arithmeticAN<mul>, groups numbered by first occurrence (groupbyAN) and
 * AN-coded 64-bit sums (aggregate_sum_groupedAN), or aggregate_mul_sumAN for
 * ungrouped queries.  No reference counterpart exists as one call.
 *
 * The SSB programs' own shapes (ssbm-q11_continuous.cpp:70-127,
 * ssbm-q21_continuous.cpp, ssbm-q41_continuous.cpp:99-215):
 *   - fact predicates (Q1.x): selectAN on lo_quantity and/or lo_discount over
 *     the query's whole prefix, on the codes (thresholds times A), before any
 *     join; a corrupt code is reported, and selected when the code itself
 *     passes, as selectAN does; every foreign key of such a query is then
 *     fetched positionally;
 *   - two predicates on one dimension's attributes, combined with AND (Q1.3:
 *     d_year and d_weeknuminyear, intersected with matchjoinAN);
 *   - the measure: extendedprice * discount (Q1.x), revenue (Q2.x, Q3.x) or
 *     revenue - supplycost (arithmeticAN<sub>, Q4.x); the measure columns are
 *     fetched positionally one after the other, a corrupt value dropping the
 *     row from all of them.  Ungrouped queries take the first measure only.
 * Queries with fact predicates or another measure than price * discount run
 * the per-row strategy. */
#define AHEAD_SJ_DATE 0
#define AHEAD_SJ_CUSTOMER 1
#define AHEAD_SJ_PART 2
#define AHEAD_SJ_SUPPLIER 3
#define AHEAD_SJ_MAXQ 64
#define AHEAD_SJ_MAXATTR 4
/* fact columns of the error vectors (the foreign keys are 0-3, AHEAD_SJ_*) */
#define AHEAD_SJ_COL_PRICE 4
#define AHEAD_SJ_COL_DISCOUNT 5
#define AHEAD_SJ_COL_QUANTITY 6
#define AHEAD_SJ_COL_REVENUE 7
#define AHEAD_SJ_COL_SUPPLYCOST 8
#define AHEAD_SJ_NCOL 9
/* measures */
#define AHEAD_SJ_MEASURE_PRICE_DISCOUNT 0 /* sum(lo_extendedprice * lo_discount) */
#define AHEAD_SJ_MEASURE_REVENUE 1        /* sum(lo_revenue) */
#define AHEAD_SJ_MEASURE_PROFIT 2         /* sum(lo_revenue - lo_supplycost) */

typedef struct ahead_sj_dim {
    ahead_col key;                     /* resint key column (device) */
    ahead_col attr[AHEAD_SJ_MAXATTR];  /* AN-coded attribute columns */
    uint64_t rows;
    int32_t nattr;
    int32_t _pad;
} ahead_sj_dim;

typedef struct ahead_sj_schema {
    ahead_col fk[4];        /* lineorder foreign keys, indexed by AHEAD_SJ_* (resint) */
    ahead_col price;        /* resint */
    ahead_col discount;     /* restiny */
    uint64_t fact_rows;
    ahead_sj_dim dim[4];
    /* the programs' further fact columns; data NULL when absent (queries
     * that read one are then AHEAD_BAD_ARG) */
    ahead_col quantity;     /* restiny */
    ahead_col revenue;      /* resint */
    ahead_col supplycost;   /* resint */
} ahead_sj_schema;

typedef struct ahead_sj_pred {
    int32_t dim, attr, op1, op2, comb, _pad;
    uint64_t th1, th2;      /* thresholds on the codes */
} ahead_sj_pred;

/* selectAN<op1[, op2, comb]> on a fact column (AHEAD_SJ_COL_QUANTITY or
 * AHEAD_SJ_COL_DISCOUNT), thresholds on the codes */
typedef struct ahead_sj_fpred {
    int32_t col, op1, op2, comb;
    uint64_t th1, th2;
} ahead_sj_fpred;

typedef struct ahead_sj_query {
    uint64_t fact_rows;     /* prefix of lineorder the query reads */
    int32_t npred, ngroup;
    ahead_sj_pred pred[4];  /* at most two per dimension, on different attributes */
    int32_t gdim[3], gattr[3];
    int32_t measure;        /* AHEAD_SJ_MEASURE_* */
    int32_t nfpred;         /* 0..2, at most one per fact column */
    ahead_sj_fpred fpred[2];
} ahead_sj_query;

/* Per-query result in HOST memory: groups in first-occurrence order with the
 * codes of their group attributes and their AN-coded sums, or the total of an
 * ungrouped query; error positions (row * A_OID) per fact column: the four
 * foreign keys (AHEAD_SJ_* index), then AHEAD_SJ_COL_PRICE ... SUPPLYCOST.
 * status: AHEAD_OK; AHEAD_UNSUPPORTED when the inputs leave the fused
 * path's domain (duplicate or corrupt dimension keys, a filtered or grouped
 * attribute that is corrupt or not packed into the key records, a dense
 * group domain above 2^23, more than 65536 detected errors in the batch, more
 * group output than the batch's packed area holds), and the caller then runs
 * the operator-at-a-time path, which handles every input; AHEAD_CAPACITY when
 * `capacity` or an error vector's capacity is too small (ngroups and the
 * error counts hold the sizes needed; ahead_sj_fetch returns them). */
typedef struct ahead_sj_result {
    uint64_t ngroups;
    uint64_t capacity;      /* entries of keys[j] / sums */
    uint64_t* keys[3];
    uint64_t* sums;
    uint64_t total;
    int32_t status;
    int32_t _pad;
    ahead_errvec fact_err[AHEAD_SJ_NCOL];
} ahead_sj_result;

typedef struct ahead_sj_engine ahead_sj_engine;

/* The same star join operator at a time (no engine): one query composed in C++
 * from the AN operators above, as the reference's programs compose theirs
 * (ssbm-q11_continuous.cpp, ssbm-q21_continuous.cpp, ssbm-q41_continuous.cpp;
 * its Python twin is ahead_b200/pipelines.py::starjoin_continuous).  Per
 * joined dimension its predicates are selectAN chains on the attribute codes
 * and the key -> OID map is a matchjoinAN.  The first join probes the whole
 * foreign-key column (hashjoinAN), unless fact predicates (selectAN on
 * quantity / discount) select the rows first.  The later joins fetch
 * positionally (matchjoinAN) and probe.  The measures are fetched one after
 * the other.  Then aggregate_mul_sumAN, or the group attributes, arithmeticAN,
 * groupbyAN / binary groupbyAN and aggregate_sum_groupedAN.  It fills `res`
 * as ahead_sj_wait does for the fused engine (AHEAD_CAPACITY when the groups
 * or an error vector exceed `res`'s capacities; ngroups and the counts give the
 * sizes needed).  Synchronous.  Its device buffers come from a memory pool of
 * its own per device (the stream-ordered allocator on the context's stream),
 * which keeps the memory it frees for later calls: the footprint of the
 * largest query so far stays reserved until the process ends. */
int ahead_plain_starjoin(ahead_ctx* ctx, const ahead_sj_schema* schema, const ahead_sj_query* q,
                         ahead_sj_result* res);

/* Prepare a schema resident in device memory (key maps of the dimensions,
 * checks of the dimension columns).  The schema's buffers must outlive the
 * engine.  fact_rows must not exceed 2^32 - 2^16 (AHEAD_UNSUPPORTED). */
int ahead_sj_create(ahead_ctx* ctx, const ahead_sj_schema* schema, ahead_sj_engine** out);
void ahead_sj_destroy(ahead_sj_engine* eng);
/* Run a batch of nq (1..64) queries in one fused pass; results in host memory. */
int ahead_sj_run(ahead_sj_engine* eng, const ahead_sj_query* qs, int nq, ahead_sj_result* res);
/* Same, replaying a CUDA graph captured for this batch shape (captured on the
 * first call with a new shape). */
int ahead_sj_run_graph(ahead_sj_engine* eng, const ahead_sj_query* qs, int nq, ahead_sj_result* res);
/* Asynchronous form.  submit plans the batch, uploads its descriptors and
 * enqueues its kernels (use_graph: replay the slot's captured CUDA graph) and
 * returns a ticket; wait blocks until that batch is done and fills `res`.
 * Two batches may be in flight: while one runs, the host prepares or reads
 * back the other.  A third submit before a wait returns AHEAD_CAPACITY. */
int ahead_sj_submit(ahead_sj_engine* eng, const ahead_sj_query* qs, int nq, int use_graph, uint64_t* ticket);
int ahead_sj_wait(ahead_sj_engine* eng, uint64_t ticket, ahead_sj_result* res);
/* Device time in ms of the last waited batch's kernels (CUDA events). */
float ahead_sj_last_ms(ahead_sj_engine* eng);

/* ------------------------------------------------ fact-sharded batches
 * The engine's fact columns may be one contiguous row range of a larger
 * lineorder, the rest held by other engines (one per GPU):
 * ahead_sj_set_shard declares them rows [first_row, first_row + fact_rows)
 * of a table of table_rows rows (below 2^32).  Queries then name prefixes of
 * the whole table, and every row the engine reports (error positions, group
 * first rows) is a row of the whole table.  A batch runs in two halves around
 * one exchange between the engines:
 *   submit_local  plans the batch and runs its scan over the local rows up to
 *                 the per-query dense group tables, which it exports into the
 *                 slot's exchange area (*x);
 *   (caller)      combines every engine's area, on the device: all-reduce
 *                 SUM of x->sums (int64 adds wrap mod 2^64 as the reference's
 *                 u64 sums do), MIN of x->firsts, MAX of x->flags, and an
 *                 all-gather of x->log (1 + log_cap words each), after the
 *                 context's stream has reached submit_local's work and before
 *                 submit_final's;
 *   submit_final  takes the combined tables back from the exchange area and
 *                 the gathered logs (world areas of 1 + log_cap words,
 *                 contiguous), orders the groups and errors of the whole
 *                 table and packs the results; ahead_sj_wait collects them.
 * Exact because every step of the composition is local to one fact row.
 * No reference counterpart: the reference runs on one host. */
typedef struct ahead_sj_xchg {
    int64_t* sums;    /* [groups] AN-coded group sums over this engine's rows */
    int64_t* firsts;  /* [groups] first row (of the table) of each group; INT64_MAX: none */
    int64_t* flags;   /* [4] status flags, 0/1 */
    uint64_t* log;    /* [1 + log_cap] entry count, then (query, column, row) error entries */
    uint64_t groups, log_cap;
} ahead_sj_xchg;
int ahead_sj_set_shard(ahead_sj_engine* eng, uint64_t first_row, uint64_t table_rows);
int ahead_sj_submit_local(ahead_sj_engine* eng, const ahead_sj_query* qs, int nq, int use_graph, uint64_t* ticket,
                          ahead_sj_xchg* x);
int ahead_sj_submit_final(ahead_sj_engine* eng, uint64_t ticket, const uint64_t* gathered_logs, int world);

/* Fact-kernel shape (rows per thread x blocks per SM), chosen among a few
 * compiled variants.  tune times every variant on the given batch (median of
 * three runs, outside any graph) and keeps the fastest; set_variant sets one.
 * Both drop the slots' captured graphs, which are captured again. */
int ahead_sj_tune(ahead_sj_engine* eng, const ahead_sj_query* qs, int nq, int* variant);
int ahead_sj_set_variant(ahead_sj_engine* eng, int variant);
/* Shape of the cube strategy's scan kernel (tune chooses it as well), one of
 * ahead_sj_cube_variant_count() compiled shapes.  The indexed shapes need the
 * fact columns 16-byte aligned (discount 4-byte) and return AHEAD_UNSUPPORTED
 * otherwise; tune skips them then. */
int ahead_sj_set_cube_variant(ahead_sj_engine* eng, int variant);
int ahead_sj_cube_variant_count(void);
/* 1 when cube shape `variant` reads the engine's join index, 0 when it looks
 * every dimension code up, -1 when there is no such shape. */
int ahead_sj_cube_variant_is_indexed(int variant);
/* Index arrays cube shape `variant` reads (0, 1: the largest dimension's, 2:
 * both; 3: both dimensions from the packed index), -1 when there is no such
 * shape.  A shape reads only its own index format; with the other format it
 * looks every dimension code up (tune skips it then). */
int ahead_sj_cube_variant_slots(int variant);
/* The engine's join index, built by ahead_sj_create: per fact row, for the
 * two dimensions with the largest key ranges, the decoded foreign key's offset
 * (the 32-bit difference key - smallest key) and that key's packed attributes
 * (0: no dimension row has the key).  Two formats:
 *  - two words (16 bytes per row): one 64-bit word per dimension holding
 *    offset | attributes << 32 AN-coded with A = 65117, the largest
 *    dimension's [rows] words, then the second's;
 *  - packed (8 bytes per row, built by default when it fits): one 64-bit
 *    word id1 | id2 << bits(n1) | (o1 + (range1 + 1) * o2) << (bits(n1) +
 *    bits(n2)), where a key's id is the dense number of its attribute record
 *    among the dimension's n records (0: no dimension row has the key) and o
 *    its offset clamped to the key range, AN-coded with the A that
 *    ahead_sj_index_packing reports.
 * An indexed cube scan uses a row's entry only while the row's foreign keys,
 * decoded and checked in every batch, still have those offsets and the word
 * passes its AN check; any other row takes the exact per-row path, so results
 * never depend on the index.  *data = device address of the words (NULL: the
 * engine has no index, e.g. the device memory was short), *bytes_per_row =
 * 16 or 8 (the format), *rows = fact rows; *dims = bit d set when dimension d
 * (AHEAD_SJ_*) is indexed.  No reference counterpart: the reference probes a
 * hash table per query. */
int ahead_sj_index_info(ahead_sj_engine* eng, const void** data, uint64_t* bytes_per_row, uint64_t* rows,
                        uint32_t* dims);
/* Rebuilds the join index in a format: -1 packed when it fits, else two
 * words (what ahead_sj_create builds); 0 none; 1 two words; 2 packed
 * (AHEAD_UNSUPPORTED when its fields and AN code do not fit 64 bits; the
 * engine then has no index).  Waits for the device; no batch may be in
 * flight.  The cube shape changes to the format's default when the current
 * one reads the other format. */
int ahead_sj_set_index(ahead_sj_engine* eng, int format);
/* The packed index's layout for two dimensions with key ranges krange[0],
 * krange[1] and nrec[0], nrec[1] distinct attribute records: *payload_bits =
 * the fields' total width, *A = the first A of the AN code lists (65117,
 * 16089, 7785, 881, 463, 233, 125, 61, 29), else the largest odd A below
 * 2^16, with payload_bits + bits of A <= 64 under which every flip of one or
 * two bits of the word is detected.  AHEAD_UNSUPPORTED when none fits.  Host
 * arithmetic only (no device). */
int ahead_sj_index_packing(const uint64_t krange[2], const uint64_t nrec[2], uint64_t* A, uint32_t* payload_bits);
/* The measured roofs of the indexed cube scan on the context's device, on
 * `rows` (rounded down to 512, below 2^32) synthetic rows of its column layout
 * (six 8-byte columns and a 2-byte one: 50 B per row), median of five timed
 * launches in milliseconds: ms[0] the columns streamed alone, ms[1] one 64-bit
 * L2 reduction per row into `cells` random cells alone, ms[2] both, each
 * reduction's cell hashed from its row's loaded words.  Allocates and frees
 * its buffers (about 50 B per row).  No reference counterpart. */
int ahead_gpu_cube_roofs(ahead_ctx* ctx, uint64_t rows, uint32_t cells, float* ms);
/* Rows of the cube scan's first phase (0, the default: 16 per signature of the
 * batch, rounded up to 8192; UINT64_MAX: one phase).  The second phase reads a
 * signature's first row only for signatures the first phase did not see;
 * results do not depend on the split.  tune chooses it with the shape. */
int ahead_sj_set_cube_split(ahead_sj_engine* eng, uint64_t rows);
/* How a batch is evaluated.  Per-row (0): each fact row walks the dimensions
 * for every query alive on it.  Signature cube (1): one scan aggregates the
 * decoded price x discount of clean rows per prefix segment and per code of
 * the dimension attributes the batch references; each query then takes the
 * codes it accepts; rows with a detected error run the per-row semantics.
 * -1 (default): the cube for batches of at least 4 queries when it fits. */
int ahead_sj_set_strategy(ahead_sj_engine* eng, int strategy);

/* One query's result again, from the last batch collected in that ticket's
 * slot (valid until the slot's next submit): for a result that returned
 * AHEAD_CAPACITY, with buffers of the sizes it reported. */
int ahead_sj_fetch(ahead_sj_engine* eng, uint64_t ticket, int query, ahead_sj_result* res);
/* 1 when a submitted batch's results can be collected without waiting, 0 when
 * it is still running, a negative status on error. */
int ahead_sj_ready(ahead_sj_engine* eng, uint64_t ticket);
/* Device memory a query holds while its batch runs (dense group slots and its
 * share of the result areas), for admission control. */
int ahead_sj_footprint(ahead_sj_engine* eng, const ahead_sj_query* q, uint64_t* bytes);

/* Measurements of the last waited batch. */
typedef struct ahead_sj_stats {
    float batch_ms;          /* all kernels of the batch (CUDA events) */
    float fact_ms;           /* the fact-table kernel alone */
    uint64_t fact_rows;      /* rows the fact kernel scanned (longest prefix) */
    uint64_t h2d_bytes;      /* descriptors uploaded */
    uint64_t d2h_bytes;      /* header + packed results read back */
    uint64_t errors_logged;  /* (query, column, row) error entries */
    uint32_t strategy;       /* 0: per-row pass, 1: signature cube */
    uint32_t unseen_sigs;    /* cube: signatures the scan's first phase did not see */
    uint64_t exception_rows; /* rows the cube pass sent to the exact per-row path */
    int32_t cube_variant;    /* cube: the scan shape that ran (ahead_sj_set_cube_variant) */
    uint32_t pad;
} ahead_sj_stats;
int ahead_sj_last_stats(ahead_sj_engine* eng, ahead_sj_stats* out);

/* ------------------------------------------------------------------ serving
 * A request loop over one engine, on its own host thread.  Requests arrive
 * (submit, or an open-loop replay of scheduled arrivals), wait at most
 * `window_ms` for companions, and start as one fused batch when an engine
 * slot is free: while one batch runs on the device the next is formed from the
 * requests that arrived meanwhile and queued behind it (continuous batching).
 * A request is admitted into a batch only while the device memory of all
 * admitted, unfinished requests (ahead_sj_footprint) stays within
 * `hbm_budget`.  The fact and dimension columns stay resident.  No reference
 * counterpart: the reference runs one query program per process. */
typedef struct ahead_sj_server ahead_sj_server;

typedef struct ahead_sj_server_cfg {
    double window_ms;     /* batching window */
    int32_t max_batch;    /* requests per batch, 1..64 */
    int32_t use_graph;    /* replay the slots' CUDA graphs */
    uint64_t hbm_budget;  /* bytes */
    uint64_t max_groups;  /* per-request result capacity */
    uint64_t max_errors;  /* per-request, per-column error-position capacity */
} ahead_sj_server_cfg;

/* A finished request.  Times in microseconds on the server's steady clock:
 * arrival (the scheduled arrival for a replay), start of its batch, results on
 * the host.  `result` points into server-owned memory that stays valid until
 * ahead_sj_server_release(id). */
typedef struct ahead_sj_done {
    uint64_t id;
    double arrival_us, start_us, done_us;
    uint32_t batch_size;
    int32_t _pad;
    ahead_sj_result result;
} ahead_sj_done;

typedef struct ahead_sj_server_stats {
    uint64_t batches, requests, completed;
    double busy_ms;        /* summed device time of the batches' kernels */
    double mean_batch;
    uint32_t max_inflight_bytes_frac_pct;  /* peak admitted footprint, % of the budget */
    uint32_t _pad;
} ahead_sj_server_stats;

int ahead_sj_server_create(ahead_sj_engine* eng, const ahead_sj_server_cfg* cfg, ahead_sj_server** out);
/* Stops the loop after the admitted requests finished; releases everything. */
void ahead_sj_server_destroy(ahead_sj_server* srv);
/* Thread-safe.  The request arrives now. */
int ahead_sj_server_submit(ahead_sj_server* srv, const ahead_sj_query* q, uint64_t* id);
/* Open-loop arrivals: request i arrives arrival_us[i] microseconds after this
 * call (non-decreasing); ids are first_id, first_id + 1, ... */
int ahead_sj_server_replay(ahead_sj_server* srv, const ahead_sj_query* qs, const double* arrival_us, int n,
                           uint64_t* first_id);
/* Up to `max` finished requests; waits up to wait_ms for the first. */
int ahead_sj_server_poll(ahead_sj_server* srv, ahead_sj_done* out, int max, int wait_ms, int* n);
int ahead_sj_server_release(ahead_sj_server* srv, uint64_t id);
int ahead_sj_server_stats_get(ahead_sj_server* srv, ahead_sj_server_stats* out);
/* The server's clock now, in microseconds. */
double ahead_sj_server_now_us(ahead_sj_server* srv);

#ifdef __cplusplus
}
#endif

#endif /* AHEAD_GPU_H */
