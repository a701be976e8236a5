/*
 * an_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU oracle for the AN-hardened operator path.  Two libraries implement this
 * one interface:
 *   - liban_oracle.so       (an_oracle.c): a plain-C restatement of the
 *                            reference's scalar operators, each function citing
 *                            the reference file:line it follows;
 *   - _ref/libahead_ref.so  (ref/ref_capi.cpp): the reference's own scalar
 *                            operator templates, compiled from the reference
 *                            sources with small header stand-ins.
 * Only tests, the smoke check and the CPU-baseline leg of bench.py load them,
 * and only as the checker.  The GPU library never calls into either.
 *
 * All pointers are host pointers.  Output BATs: the caller passes head.data /
 * tail.data buffers of `cap` elements of 8 bytes each; the oracle fills in the
 * output column types, metadata and count and writes elements at the output
 * type's storage width.  If an output needs more than `cap` rows the function
 * returns AHEAD_CAPACITY with out->count holding the need.  Error vectors
 * follow ahead_errvec (count is always exact; at most capacity entries).
 */
#ifndef AHEAD_AN_ORACLE_H
#define AHEAD_AN_ORACLE_H

#include "../include/ahead_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* selectAN<Op> / selectAN<Op1,Op2,Comb> (scalar): void head, AN tail.
 * out->head receives resoid codes (oid * 65117); out->tail stays empty. */
int orc_select_an(const ahead_bat* in, int op1, uint64_t th1, int op2, uint64_t th2, int comb,
                  uint64_t aoid, ahead_bat* out, uint64_t cap, ahead_errvec* err);

/* selectAN / select over a string tail (selectAN_scalar.tcc:98-131, 185-222;
 * Normal/select_scalar.tcc:78-101, 137-165): keep a row when
 * Op(strcmp(row, th), 0).  `strs` holds `count` rows of `width` bytes; a row
 * ends at its first NUL or after `width` bytes.  The AN form writes resoid
 * codes (seqbase + i) * 65117, the plain form oid_t. */
int orc_select_str_an(const char* strs, uint64_t width, uint64_t count, uint64_t seqbase, int op1,
                      const char* th1, int op2, const char* th2, int comb, ahead_bat* out, uint64_t cap);
int orc_select_str(const char* strs, uint64_t width, uint64_t count, uint64_t seqbase, int op1,
                   const char* th1, int op2, const char* th2, int comb, ahead_bat* out, uint64_t cap);

/* Unencoded select (Normal/select_scalar.tcc): out->head receives oid_t. */
int orc_select(const ahead_bat* in, int op1, uint64_t th1, int op2, uint64_t th2, int comb,
               ahead_bat* out, uint64_t cap);

/* checkAN / decodeAN / checkAndDecodeAN (encdecAN_scalar.tcc). */
int orc_check_an(const ahead_bat* in, uint64_t ainv, uint64_t unenc_max, uint64_t aoid,
                 ahead_errvec* err);
int orc_decode_an(const ahead_bat* in, uint64_t aoid, ahead_bat* out, uint64_t cap,
                  ahead_errvec* err);
int orc_check_and_decode_an(const ahead_bat* in, uint64_t aoid, ahead_bat* out, uint64_t cap,
                            ahead_errvec* err_head, ahead_errvec* err_tail);
/* encodeAN: tail * A into the encoded type of the tail. */
int orc_encode_an(const ahead_bat* in, uint64_t A, ahead_bat* out, uint64_t cap);

/* hashjoinAN (hashjoinAN.tcc): errs[0..3] = H1, T1, H2, T2. */
int orc_hashjoin_an(const ahead_bat* l, const ahead_bat* r, int reenc_head, uint64_t ah1r,
                    uint64_t ah1invr, int reenc_tail, uint64_t at2r, uint64_t at2invr, int side,
                    uint64_t aoid, ahead_bat* out, uint64_t cap, ahead_errvec* errs);
int orc_hashjoin(const ahead_bat* l, const ahead_bat* r, int side, ahead_bat* out, uint64_t cap);
/* hashjoinAN with a string right tail (hashjoinAN.tcc:225-367): the right
 * tail is r_strs (r->count slots of `width` bytes); out->tail.data receives
 * `cap` slots.  errs[0..2] = head1, tail1, head2; errs[3] is never present. */
int orc_hashjoin_str_an(const ahead_bat* l, const ahead_bat* r, const char* r_strs, uint64_t width,
                        int reenc_head, uint64_t ah1r, uint64_t ah1invr, int side, uint64_t aoid,
                        ahead_bat* out, uint64_t cap, ahead_errvec* errs);
/* fetchjoinAN with a string tail (matchjoinAN.tcc:304-354, T2 = v2_str_t):
 * `count` slots of `width` bytes; the fetched slots go to `out` (n_out of
 * them); errs[0] = OIDs past the column, errs[1] not present. */
int orc_fetchjoin_str_an(const ahead_bat* a, const char* strs, uint64_t width, uint64_t count, uint64_t aoid,
                         char* out, uint64_t cap, uint64_t* n_out, ahead_errvec* errs);
/* groupbyAN binary over a string tail (groupbyAN.tcc:99-165 with hash<str_t>,
 * miscellaneous.hpp:99-119): a void head (seqbase) and `count` slots. */
int orc_groupby2_str_an(const char* strs, uint64_t width, uint64_t count, uint64_t seqbase,
                        const ahead_bat* grouping, uint64_t ngroups, uint64_t aoid, uint64_t aoidinv,
                        ahead_bat* gids, ahead_bat* firsts, uint64_t cap, ahead_errvec* errs);
/* The unencoded twins: fetchjoin over a string tail (Normal/matchjoin.tcc:
 * 144-160; a (void, oid) list) and the binary groupby over a string BAT
 * (Normal/groupby.tcc:85-121, the same string hash). */
int orc_fetchjoin_str(const ahead_bat* a, const char* strs, uint64_t width, uint64_t count, char* out, uint64_t cap,
                      uint64_t* n_out);
int orc_groupby2_str(const char* strs, uint64_t width, uint64_t count, uint64_t seqbase, const ahead_bat* grouping,
                     uint64_t ngroups, ahead_bat* gids, ahead_bat* firsts, uint64_t cap);

/* matchjoinAN (matchjoinAN.tcc): general merge, void-void and resoid-void
 * positional forms.  errs[0..3] = H1, T1, H2, T2 (absent ones present=0). */
int orc_matchjoin_an(const ahead_bat* a, const ahead_bat* b, int reenc, uint64_t ah1r,
                     uint64_t ah1invr, uint64_t at2r, uint64_t at2invr, uint64_t aoid,
                     ahead_bat* out, uint64_t cap, ahead_errvec* errs);
int orc_matchjoin(const ahead_bat* a, const ahead_bat* b, ahead_bat* out, uint64_t cap);

/* fetchjoinAN (matchjoinAN.tcc FetchjoinAN): errs[0] = bad OID, errs[1] = bad value. */
int orc_fetchjoin_an(const ahead_bat* a, const ahead_bat* b, int reenc, uint64_t atr,
                     uint64_t atrinv, uint64_t aoid, ahead_bat* out, uint64_t cap,
                     ahead_errvec* errs);
int orc_fetchjoin(const ahead_bat* a, const ahead_bat* b, ahead_bat* out, uint64_t cap);

/* groupbyAN unary / binary (groupbyAN.tcc).  gids: void -> resoid GID codes;
 * firsts: void -> resoid OID codes of each group's first row. */
int orc_groupby_an(const ahead_bat* in, uint64_t aoid, uint64_t aoidinv, ahead_bat* gids,
                   ahead_bat* firsts, uint64_t cap, ahead_errvec* errs);
int orc_groupby2_an(const ahead_bat* in, const ahead_bat* grouping, uint64_t ngroups,
                    uint64_t aoid, uint64_t aoidinv, ahead_bat* gids, ahead_bat* firsts,
                    uint64_t cap, ahead_errvec* errs);

/* aggregate_sum_groupedAN (aggregateAN.tcc): out->tail = ngroups sums. */
int orc_aggregate_sum_grouped_an(const ahead_bat* in, const ahead_bat* grouping,
                                 uint64_t ngroups, int result_type, uint64_t ar, uint64_t arinv,
                                 uint64_t aoid, ahead_bat* out, ahead_errvec* errs);

/* aggregate_mul_sumAN (aggregateAN_scalar.tcc). */
int orc_aggregate_mul_sum_an(const ahead_bat* a, const ahead_bat* b, int result_type,
                             uint64_t init, uint64_t ra, uint64_t rainv, uint64_t aoid,
                             uint64_t* total, ahead_errvec* errs);
/* Unencoded aggregate_mul_sum (Normal/aggregate_scalar.tcc). */
int orc_aggregate_mul_sum(const ahead_bat* a, const ahead_bat* b, int result_type,
                          uint64_t init, uint64_t* total);

/* arithmeticAN<Op,Result> (arithmeticAN_scalar.tcc): errs = H1, T1, H2, T2. */
int orc_arithmetic_an(int op, int result_type, const ahead_bat* a, const ahead_bat* b,
                      uint64_t ar, uint64_t arinv, uint64_t aoid, ahead_bat* out,
                      ahead_errvec* errs);

/* Unencoded groupby, unary and binary (Normal/groupby.tcc): gids (void, oid)
 * in first-occurrence order, firsts (void, oid) = head of each group's first row. */
int orc_groupby(const ahead_bat* in, ahead_bat* gids, ahead_bat* firsts, uint64_t cap);
int orc_groupby2(const ahead_bat* in, const ahead_bat* grouping, uint64_t ngroups, ahead_bat* gids,
                 ahead_bat* firsts, uint64_t cap);
/* Unencoded aggregate_sum_grouped<bigint> (Normal/aggregate.tcc): out->tail = ngroups sums. */
int orc_aggregate_sum_grouped(const ahead_bat* in, const ahead_bat* grouping, uint64_t ngroups,
                              int result_type, ahead_bat* out);
/* Unencoded aggregate_sum<Result> (Normal/aggregate_scalar.tcc). */
int orc_aggregate_sum(const ahead_bat* in, int result_type, uint64_t* total);
/* Unencoded arithmetic<Op, Result> (Normal/arithmetic_scalar.tcc). */
int orc_arithmetic(int op, int result_type, const ahead_bat* a, const ahead_bat* b, ahead_bat* out);

/* ext_euclidean(A, bits): modular inverse of odd A mod 2^bits
 * (include/util/resilience.hpp:481-516). */
uint64_t orc_ainv(uint64_t a, int bits);

#ifdef __cplusplus
}
#endif

#endif
