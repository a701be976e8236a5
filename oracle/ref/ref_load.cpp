// TEST INFRASTRUCTURE ONLY: a C entry to the reference's own table loader
// (lib/column_storage/Transaction.cpp, TransactionManager::Transaction::load,
// through the AHEAD facade, lib/AHEAD.cpp:96-128), compiled from the reference
// sources by `make refload` in oracle/Makefile.  It is the checker that pins
// the loader restatement (oracle/tbl_oracle.c) and the GPU loader on the same
// header and `.tbl` / `.ahead` files; nothing on the product path uses it.
//
//   refl_load     creates the AHEAD instance with the reference's own options
//                 (--dbpath, --AN-minbfw, --convert-table-files) and loads
//                 `<dbpath>/<table>` (its _header.csv, .tbl and .ahead files);
//   refl_column   copies one loaded column out, `width` bytes per row in the
//                 column's own type (strings: the slot's bytes up to the first
//                 NUL, NUL-padded to `width`);
//   refl_reset    destroys the instance (and with it every loaded column).
// Errors the reference raises (std::exception) come back as -1 and their text.
#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include <AHEAD.hpp>
#include <column_storage/ColumnBat.h>

using namespace ahead;

namespace {

void put_err(const char* msg, char* err, size_t errlen) {
    if (err && errlen) {
        std::strncpy(err, msg, errlen - 1);
        err[errlen - 1] = 0;
    }
}

template <typename V2>
int copy_column(const char* table, const char* attr, uint32_t width, unsigned char* out, uint64_t cap,
                uint64_t* count) {
    ColumnBAT<V2> bat(table, attr);
    auto* it = bat.begin();
    uint64_t n = 0;
    for (; it->hasNext(); ++*it) {  // (the iterator starts on the first row, as the reference's copy() uses it)
        if (n < cap) {
            auto v = it->tail();
            unsigned char* dst = out + n * width;
            if constexpr (std::is_pointer_v<decltype(v)>) {
                std::memset(dst, 0, width);
                const size_t len = v ? strnlen(v, width) : 0;
                std::memcpy(dst, v, len);
            } else {
                std::memset(dst, 0, width);
                std::memcpy(dst, &v, sizeof v < width ? sizeof v : width);
            }
        }
        ++n;
    }
    delete it;
    *count = n;
    return 0;
}

}  // namespace

extern "C" {

int refl_load(const char* dbpath, const char* table, int minbfw, int convert, uint64_t size, const char* delim,
              int ignore_more, uint64_t* rows, char* err, size_t errlen) {
    try {
        std::string bfw = std::to_string(minbfw);
        std::vector<const char*> argv = {"refload", "--dbpath", dbpath, "--AN-minbfw", bfw.c_str()};
        if (!convert) argv.push_back("--no-convert-table-files");
        AHEAD::createInstance((int)argv.size(), argv.data());
        *rows = AHEAD::getInstance()->loadTable(table, nullptr, size == UINT64_MAX ? static_cast<size_t>(-1) : size,
                                                delim, ignore_more != 0);
        return 0;
    } catch (const std::exception& ex) {
        put_err(ex.what(), err, errlen);
        return -1;
    }
}

// tbl_type: the codes of include/ahead_ingest.h (TINYINT 0, SHORTINT 1,
// INTEGER 2, LARGEINT 3, STRING 4, FIXED 5, CHAR 6, RESTINY 7, RESSHORT 8,
// RESINT 9, RESBIGINT 10).
int refl_column(const char* table, const char* attr, int tbl_type, uint32_t width, void* out, uint64_t cap,
                uint64_t* count, char* err, size_t errlen) {
    auto* o = static_cast<unsigned char*>(out);
    try {
        switch (tbl_type) {
            case 0: return copy_column<v2_tinyint_t>(table, attr, width, o, cap, count);
            case 1: return copy_column<v2_shortint_t>(table, attr, width, o, cap, count);
            case 2: return copy_column<v2_int_t>(table, attr, width, o, cap, count);
            case 3: return copy_column<v2_bigint_t>(table, attr, width, o, cap, count);
            case 4: return copy_column<v2_str_t>(table, attr, width, o, cap, count);
            case 5: return copy_column<v2_fixed_t>(table, attr, width, o, cap, count);
            case 6: return copy_column<v2_char_t>(table, attr, width, o, cap, count);
            case 7: return copy_column<v2_restiny_t>(table, attr, width, o, cap, count);
            case 8: return copy_column<v2_resshort_t>(table, attr, width, o, cap, count);
            case 9: return copy_column<v2_resint_t>(table, attr, width, o, cap, count);
            case 10: return copy_column<v2_resbigint_t>(table, attr, width, o, cap, count);
            default: put_err("unknown column type", err, errlen); return -1;
        }
    } catch (const std::exception& ex) {
        put_err(ex.what(), err, errlen);
        return -1;
    }
}

void refl_reset(void) { AHEAD::destroyInstance(); }

}  // extern "C"
