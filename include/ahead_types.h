/*
 * ahead_types.h -- plain-C data model shared by the GPU operator library
 * (ahead_gpu.h) and the CPU oracle.
 *
 * A BAT ("binary association table") is a pair of equally long columns,
 * head and tail.  Each column has one of the AHEAD value types below and the
 * AN-coding metadata of the reference's ColumnMetaData
 * (include/column_storage/ColumnMetaData.hpp:150-200): A, A^-1 mod 2^w and the
 * largest valid decoded value.  A VOID column is virtual: value(i) is the
 * dense object id (oid_t, 32 bit) seqbase + i, exactly what the reference's
 * TempBATIterator<v2_void_t, Tail>::head() yields
 * (include/column_storage/TempBatIterator.h:436-452).
 *
 * No torch or CUDA types appear here; pointers are plain addresses (device
 * addresses for the GPU library, host addresses for the oracle).
 */
#ifndef AHEAD_TYPES_H
#define AHEAD_TYPES_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Value types: one per v2_*_t tag type of the reference
 * (include/util/v2types.hpp:242-455, include/util/resilience.hpp:36-276). */
typedef enum ahead_type {
    AHEAD_VOID = 0,      /* virtual dense oid_t (u32)                         */
    AHEAD_TINYINT = 1,   /* u8                                                */
    AHEAD_SHORTINT = 2,  /* u16                                               */
    AHEAD_INT = 3,       /* u32                                               */
    AHEAD_BIGINT = 4,    /* u64                                               */
    AHEAD_OID = 5,       /* u32 object id                                     */
    AHEAD_RESTINY = 6,   /* u16 AN code of a u8   (v2_restiny_t)              */
    AHEAD_RESSHORT = 7,  /* u32 AN code of a u16  (v2_resshort_t)             */
    AHEAD_RESINT = 8,    /* u64 AN code of a u32  (v2_resint_t)               */
    AHEAD_RESBIGINT = 9, /* u64 AN code of a u64 < 2^56 (v2_resbigint_t)      */
    AHEAD_RESOID = 10,   /* u64 AN code of an oid_t (v2_resoid_t)             */
    AHEAD_NTYPES = 11,
    /* Fixed-width string slots (v2_str_t): a row is `width` bytes holding the
     * string and NUL padding, as the table loader stores STRING columns.  Only
     * the string entry points take or return it. */
    AHEAD_STR = 16
} ahead_type;

/* Comparison predicates (std::less ... std::greater of the reference's
 * selectAN<Op> template argument). */
typedef enum ahead_cmp {
    AHEAD_CMP_NONE = 0, /* no second predicate: the one-predicate selectAN */
    AHEAD_CMP_LT = 1,
    AHEAD_CMP_LE = 2,
    AHEAD_CMP_EQ = 3,
    AHEAD_CMP_NE = 4,
    AHEAD_CMP_GE = 5,
    AHEAD_CMP_GT = 6
} ahead_cmp;

/* Predicate combiners (ahead::and_is / ahead::or_is,
 * include/column_operators/functors.hpp:224,272). */
typedef enum ahead_comb { AHEAD_AND = 0, AHEAD_OR = 1 } ahead_comb;

/* Hash side of a hash join (hash_side_t, include/ColumnStore.h:80-83). */
typedef enum ahead_hash_side { AHEAD_HASH_LEFT = 0, AHEAD_HASH_RIGHT = 1 } ahead_hash_side;

/* Arithmetic operators of arithmeticAN (functors.hpp add/sub/mul/div). */
typedef enum ahead_arith { AHEAD_ADD = 0, AHEAD_SUB = 1, AHEAD_MUL = 2, AHEAD_DIV = 3 } ahead_arith;

/* Status codes.  Data corruption is never a status: detected AN errors are
 * data, reported in the error-position vectors. */
typedef enum ahead_status {
    AHEAD_OK = 0,
    AHEAD_BAD_ARG = 1,        /* unsupported type combination or bad pointer        */
    AHEAD_SIZE_MISMATCH = 2,  /* the reference throws std::runtime_error here        */
    AHEAD_CAPACITY = 3,       /* an output buffer is too small; counts hold the need */
    AHEAD_TIMEOUT = 4,        /* a bounded device wait gave up                        */
    AHEAD_CUDA_ERROR = 5,     /* a CUDA runtime call failed                           */
    AHEAD_NO_MEMORY = 6,      /* device memory could not be obtained                  */
    AHEAD_UNSUPPORTED = 7     /* input outside what this entry point handles          */
} ahead_status;

/* One column.  `data` is NULL for AHEAD_VOID.  A / Ainv / unenc_max are the
 * reference's AN_A / AN_Ainv / AN_unencMaxU; for unencoded types they are
 * carried but never used for checking. */
typedef struct ahead_col {
    void* data;
    int32_t type;       /* ahead_type */
    uint32_t A;         /* AN_A (the reference stores it as a 16-bit A_t) */
    uint64_t Ainv;      /* AN_Ainv */
    uint64_t unenc_max; /* AN_unencMaxU */
    uint64_t seqbase;   /* dense start OID of a VOID column */
} ahead_col;

typedef struct ahead_bat {
    ahead_col head;
    ahead_col tail;
    uint64_t count;
} ahead_bat;

/* An error-position vector (AN_indicator_vector, ANbase.hpp:32): positions
 * i * A_OID in ascending scan order.  `present` = 0 stands for the reference's
 * nullptr vector of an unencoded column.  The library writes at most
 * `capacity` entries and always the full `count`. */
typedef struct ahead_errvec {
    uint64_t* data;
    uint64_t capacity;
    uint64_t count;
    int32_t present;
    int32_t _pad;
} ahead_errvec;

#ifdef __cplusplus
}
#endif

#endif /* AHEAD_TYPES_H */
