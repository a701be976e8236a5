/*
 * tbl_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference's table-load conversions, the checker of
 * the GPU loader (libahead_b200.so, include/ahead_ingest.h):
 *   - orc_tbl_parse: the line loop of TransactionManager::Transaction::load
 *     (lib/column_storage/Transaction.cpp:485-590 in the reference), on an
 *     in-memory text, with the same C library calls the reference makes
 *     (fgets-style line reads of at most 1023 characters, strtok, atoi, atol,
 *     atoll, strncpy, atof);
 *   - orc_reencode: the min-BFW re-encode of ColumnIterator::read0<true>
 *     (lib/column_storage/ColumnManager.cpp:320-343).
 *
 * Parity is pinned against the reference's own loader, compiled from its
 * sources by `make refload` (oracle/ref/ref_load.cpp, one boost predicate
 * stood in for): tests/test_ingest.py compares both on seeded texts of every
 * column type and on its .ahead files, min-BFW re-encodes and row limits.  Where the reference is undefined (a line without
 * '\n' after fgets: a line longer than 1022 characters or one holding a NUL
 * byte) this restatement reports the error code AHEAD_BAD_ARG; a line with
 * fewer fields than columns, which the reference leaves as a short column,
 * is AHEAD_SIZE_MISMATCH.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/ahead_types.h"

/* kinds: 0 skip, 1 integer, 2 AN integer, 3 string, 4 fixed, 5 char
 * (the ahead_tbl_kind values of include/ahead_ingest.h) */
int orc_tbl_parse(const char* text, uint64_t len, const char* delim, int ignore_more_data, int ncols,
                  const int32_t* kinds, const uint32_t* widths, const uint64_t* As, void** outs,
                  uint64_t max_lines, uint64_t* lines, uint64_t* bad_line) {
    const char* actDelim = delim ? delim : "|";
    char line[1024];
    uint64_t pos = 0, numValues = 0, total = 0;
    for (uint64_t i = 0; i < len; ++i) total += text[i] == '\n';
    if (len && text[len - 1] != '\n') ++total;
    *lines = total;
    *bad_line = 0;
    /* while (fgets(line, LEN_LINE, valuesFile) != 0 && numValues < size) */
    while (pos < len && numValues < max_lines) {
        uint64_t n = 0;
        while (n < sizeof line - 1 && pos + n < len) {
            char c = text[pos + n++];
            if (c == '\n') break;
        }
        memcpy(line, text + pos, n);
        line[n] = 0;
        pos += n;
        char* pPos = strchr(line, '\n');
        if (!pPos) { /* the reference dereferences a null pointer here */
            *bad_line = numValues;
            return AHEAD_BAD_ARG;
        }
        *pPos = 0;
        if (pPos > line && *(pPos - 1) == '\r') *(pPos - 1) = 0;
        const uint64_t row = numValues++;
        char* buffer = strtok(line, actDelim);
        int colIdx = 0;
        while (buffer != NULL) {
            if (colIdx >= ncols) {
                if (ignore_more_data) break;
                *bad_line = row;
                return AHEAD_BAD_ARG;
            }
            char* o = (char*)outs[colIdx];
            const uint32_t w = widths[colIdx];
            switch (kinds[colIdx]) {
                case 1: /* Transaction.cpp:522-537 */
                    if (w == 1) ((int8_t*)o)[row] = (int8_t)atoi(buffer);
                    else if (w == 2) ((int16_t*)o)[row] = (int16_t)atoi(buffer);
                    else if (w == 4) ((int32_t*)o)[row] = (int32_t)atol(buffer);
                    else ((int64_t*)o)[row] = (int64_t)atoll(buffer);
                    break;
                case 2: /* Transaction.cpp:550-561 */
                    if (w == 2) ((uint16_t*)o)[row] = (uint16_t)((uint16_t)atol(buffer) * (uint16_t)As[colIdx]);
                    else if (w == 4) ((uint32_t*)o)[row] = (uint32_t)atol(buffer) * (uint32_t)As[colIdx];
                    else ((uint64_t*)o)[row] = (uint64_t)atoll(buffer) * (uint64_t)As[colIdx];
                    break;
                case 3: /* Transaction.cpp:538-540 */
                    strncpy(o + row * w, buffer, w);
                    break;
                case 4: /* Transaction.cpp:542-544 */
                    ((double*)o)[row] = atof(buffer);
                    break;
                case 5: /* Transaction.cpp:546-548 */
                    o[row] = buffer[0];
                    break;
                default:
                    break;
            }
            ++colIdx;
            buffer = strtok(NULL, actDelim);
        }
        if (colIdx < ncols) {
            *bad_line = row;
            return AHEAD_SIZE_MISMATCH;
        }
    }
    return AHEAD_OK;
}

/* Inverse of odd a modulo 2^64 (Newton's iteration). */
static uint64_t inv64(uint64_t a) {
    uint64_t x = a;
    for (int i = 0; i < 5; ++i) x *= 2 - a * x;
    return x;
}

/* ColumnManager.cpp:324-342: reencFactor = ext_euclidean(A_old, bits) * newA
 * in the column's width, every value multiplied by it. */
void orc_reencode(void* data, uint64_t n, int width, uint64_t a_old, uint64_t a_new) {
    if (width == 2) {
        uint16_t f = (uint16_t)((uint16_t)inv64(a_old) * (uint16_t)a_new);
        uint16_t* p = (uint16_t*)data;
        for (uint64_t i = 0; i < n; ++i) p[i] = (uint16_t)(p[i] * f);
    } else if (width == 4) {
        uint32_t f = (uint32_t)inv64(a_old) * (uint32_t)a_new;
        uint32_t* p = (uint32_t*)data;
        for (uint64_t i = 0; i < n; ++i) p[i] *= f;
    } else {
        uint64_t f = inv64(a_old) * a_new;
        uint64_t* p = (uint64_t*)data;
        for (uint64_t i = 0; i < n; ++i) p[i] *= f;
    }
}
