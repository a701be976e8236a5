/*
 * ahead_ingest.h -- C ABI of the table loader in libahead_b200.so: `.tbl`
 * text and `.ahead` binary column files into device memory.
 *
 * Replaces TransactionManager::Transaction::load (reference:
 * include/column_storage/TransactionManager.h:129-135,
 * lib/column_storage/Transaction.cpp:66-648) and the column-file reader and
 * writer it calls (lib/column_storage/ColumnManager.cpp:268-391).
 *
 * What the reference does, and what this library does in its place:
 *   - `<path>_header.csv`: line 1 holds the column names, line 2 their types
 *     (Transaction.cpp:167-283).  Parsed on the host, same rules.
 *   - `<path>.tbl`: one row per line, fields split with strtok on the
 *     delimiter set; integers through atoi/atol/atoll, AN columns multiplied
 *     by the load A (restiny 233, resshort 63877, resint 65117;
 *     Transaction.cpp:357-376, 485-590).  Here the text is streamed into
 *     device memory in blocks and every line is parsed by a CUDA kernel.
 *   - `<path>_<column>.ahead`: the raw column values (width bytes each) of an
 *     earlier load (Transaction.cpp:594-610, ColumnManager.cpp:381-391).
 *     Read back whenever present (Transaction.cpp:416-479); with a minimum
 *     bit-flip weight (AN.minbfw) AN columns are re-encoded on read to
 *     AsBFW[min(|AsBFW|, minbfw)] (ColumnManager.cpp:283-371).  Here the
 *     values are streamed into device memory and re-encoded there by a bulk
 *     kernel.
 *
 * Deliberate differences (the reference's behaviour there is undefined or a
 * crash): a line longer than 1022 characters, a line with fewer fields than
 * columns, a header whose type count differs from its name count, and a
 * `.tbl` that is needed but missing are errors; a last line without '\n' is
 * a line.
 */
#ifndef AHEAD_INGEST_H
#define AHEAD_INGEST_H

#include <stddef.h>
#include <stdint.h>

#include "ahead_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Column types of a header file (column_type_t of the reference,
 * Transaction.cpp:236-276): INTEGER/INT, TINYINT, SHORTINT, LARGEINT,
 * STRING[:n] (n + 1 bytes, n = 64 by default), FIXED (double), CHAR and the
 * AN types.  RESBIGINT parses but cannot be loaded (Transaction.cpp:377-381). */
typedef enum ahead_tbl_type {
    AHEAD_TBL_TINYINT = 0,
    AHEAD_TBL_SHORTINT = 1,
    AHEAD_TBL_INT = 2,
    AHEAD_TBL_LARGEINT = 3,
    AHEAD_TBL_STRING = 4,
    AHEAD_TBL_FIXED = 5,
    AHEAD_TBL_CHAR = 6,
    AHEAD_TBL_RESTINY = 7,
    AHEAD_TBL_RESSHORT = 8,
    AHEAD_TBL_RESINT = 9,
    AHEAD_TBL_RESBIGINT = 10
} ahead_tbl_type;

/* How the parse kernel stores one field (Transaction.cpp:519-571). */
typedef enum ahead_tbl_kind {
    AHEAD_TBLK_SKIP = 0,   /* column read from its .ahead file: field consumed, nothing stored */
    AHEAD_TBLK_INT = 1,    /* strtol semantics, low `width` bytes stored                        */
    AHEAD_TBLK_RES = 2,    /* strtol semantics, value * A modulo 2^(8 * width)                  */
    AHEAD_TBLK_STRING = 3, /* strncpy(dst, field, width)                                        */
    AHEAD_TBLK_FIXED = 4,  /* atof; 8-byte double                                               */
    AHEAD_TBLK_CHAR = 5    /* the field's first byte                                            */
} ahead_tbl_kind;

/* One output column of ahead_gpu_tbl_parse. */
typedef struct ahead_tbl_col {
    int32_t kind;   /* ahead_tbl_kind */
    uint32_t width; /* bytes per value: 1/2/4/8 (INT), 2/4/8 (RES), 8 (FIXED), 1 (CHAR), any (STRING) */
    uint64_t A;     /* AN multiplier of a RES column */
    void* data;     /* device column, room for `cap` rows */
} ahead_tbl_col;

/* Parse `len` bytes of `.tbl` text held in device memory into rows
 * [row0, row0 + n) of `cols` (the loop of Transaction.cpp:485-590).
 * `text` must be 16-byte aligned and end with '\n' (whole lines only).
 * `delim` is the strtok delimiter set (NULL: "|"); `ignore_more_data` drops
 * fields past the last column (else they are an error).  Only the first
 * `max_lines` lines are stored (the reference's `size` argument): n =
 * min(lines, max_lines).  On return `*lines` holds the number of lines in
 * the text.  Errors: AHEAD_CAPACITY (row0 + n > cap, nothing written),
 * AHEAD_BAD_ARG (line longer than 1022 characters or extra fields),
 * AHEAD_SIZE_MISMATCH (fewer fields than columns), AHEAD_UNSUPPORTED (a FIXED
 * field outside the exact decimal fast path); `*bad_line` is then the line's
 * index in the text (0-based). */
int ahead_gpu_tbl_parse(ahead_ctx* ctx, const void* text, uint64_t len, const char* delim,
                        int ignore_more_data, const ahead_tbl_col* cols, int ncols, uint64_t row0,
                        uint64_t cap, uint64_t max_lines, uint64_t* lines, uint64_t* bad_line);

/* Bulk re-encode of an AN column in device memory, in place: every code c
 * becomes c * (A_old^-1 * A_new) modulo 2^(8 * width) (ColumnManager.cpp:
 * 320-343).  width 2, 4 or 8; A_old and A_new odd. */
int ahead_gpu_reencode(ahead_ctx* ctx, void* data, uint64_t n, int width, uint64_t a_old, uint64_t a_new);

/* ------------------------------------------------------------ header file */
typedef struct ahead_tbl_header_col {
    char name[256];   /* prefix + name (at most 255 characters, Transaction.cpp:186-192) */
    int32_t tbl_type; /* ahead_tbl_type */
    uint32_t width;   /* bytes per value */
} ahead_tbl_header_col;

/* Read `<path>_header.csv` (Transaction.cpp:167-283).  Needs no GPU.  Writes
 * at most `cap` columns and sets `*ncols` to the number in the header.  On an
 * error the message goes to `err` (`errlen` bytes). */
int ahead_tbl_read_header(const char* path, const char* prefix, const char* delim,
                          ahead_tbl_header_col* cols, int cap, int* ncols, char* err, size_t errlen);

/* AN parameters the loader uses (resilience.hpp:56-109, Transaction.cpp:
 * 357-376, 424-456): the A of a freshly loaded AN column of `tbl_type`, and
 * the A that `min_bfw` re-encodes it to.  Returns 0 for a type without AN
 * coding, for min_bfw == 0, and when the type has no A for that weight (the
 * reference throws there). */
uint64_t ahead_tbl_load_a(int tbl_type);
uint64_t ahead_tbl_minbfw_a(int tbl_type, uint32_t min_bfw);

/* ------------------------------------------------------------ table load */
typedef struct ahead_load_opts {
    const char* prefix;           /* prepended to every column name (NULL: none)           */
    uint64_t size;                /* at most this many .tbl lines (UINT64_MAX: all)          */
    const char* delim;            /* strtok delimiter set (NULL: "|")                        */
    int32_t ignore_more_data;     /* extra fields are dropped (the reference's default: 1)   */
    uint32_t min_bfw;             /* AN.minbfw (default 0: no re-encode)                     */
    int32_t convert_table_files;  /* --convert-table-files (default 1)                       */
    uint32_t block_mb;            /* text/binary streaming block in MiB (0: 64)              */
} ahead_load_opts;

typedef struct ahead_table ahead_table;

typedef struct ahead_table_col {
    const char* name;   /* owned by the table */
    int32_t tbl_type;   /* ahead_tbl_type */
    int32_t type;       /* ahead_type of the column as a BAT tail; -1 for STRING/FIXED/CHAR */
    uint32_t width;     /* bytes per value */
    int32_t from_file;  /* 1: read from its .ahead file, 0: parsed from the .tbl */
    uint64_t A, Ainv, unenc_max; /* AN metadata (A = 1, Ainv = 1, unenc_max = 0 if unencoded) */
    void* data;         /* device memory, count * width bytes, owned by the table */
    uint64_t count;
} ahead_table_col;

typedef struct ahead_load_stats {
    uint64_t text_bytes;    /* .tbl bytes streamed to the device        */
    uint64_t binary_bytes;  /* .ahead bytes read                        */
    uint64_t written_bytes; /* .ahead bytes written                     */
    uint64_t blocks;        /* text blocks parsed                       */
    uint64_t reencoded;     /* AN values re-encoded on the device       */
    double total_ms;        /* wall time of ahead_table_load            */
    double file_ms;         /* host time in file reads and writes       */
    double parse_ms;        /* device time of the line count and parse kernels */
    double reencode_ms;     /* device time of the re-encode kernel      */
} ahead_load_stats;

/* Load table `path` into device memory on the context's device
 * (Transaction.cpp:66-648 minus the catalog entries).  `opts` NULL takes the
 * reference's defaults.  Returns the table handle in `*out`. */
int ahead_table_load(ahead_ctx* ctx, const char* path, const ahead_load_opts* opts, ahead_table** out);
int ahead_table_ncols(const ahead_table* t);
uint64_t ahead_table_rows(const ahead_table* t);
int ahead_table_column(const ahead_table* t, int i, ahead_table_col* out);
int ahead_table_stats(const ahead_table* t, ahead_load_stats* out);
void ahead_table_destroy(ahead_table* t);

#ifdef __cplusplus
}
#endif

#endif /* AHEAD_INGEST_H */
