// ingest.cu -- the table loader: `.tbl` text parsed line by line on the
// device, `.ahead` binary column files streamed in and re-encoded to another
// A on the device, header files read on the host.
//
// Reference: lib/column_storage/Transaction.cpp:66-648 (load) and
// lib/column_storage/ColumnManager.cpp:268-391 (column file read / write).
//
// Text path.  The host streams the `.tbl` file in blocks of whole lines
// (pinned buffer -> device) and per block launches
//   tbl_count_kernel  one CTA per 8 KiB tile counts the '\n' bytes in it;
//   tbl_scan_kernel   one CTA turns the tile counts into each tile's first
//                     line index and the block's line total;
//   tbl_parse_kernel  one CTA per tile stages the tile plus the 1 KiB before
//                     it in shared memory, lists the tile's line ends, and
//                     parses each line that ENDS in the tile with one thread:
//                     strtok-style fields, strtol/strncpy/atof conversions,
//                     AN columns multiplied by A, stores at row = first row +
//                     line index (rows stay in file order).
// A line is at most 1022 characters (fgets(line, 1024) in the reference keeps
// no longer line whole), so the start of a tile's first line is always
// inside the staged 1 KiB window or the line is too long.
//
// Binary path.  `.ahead` files are raw values; they are streamed to the
// device in blocks and, with a minimum bit-flip weight, every AN value is
// multiplied by A_old^-1 * A_new by reencode_kernel (HBM-bound: 2 x width
// bytes per value).
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/ahead_ingest.h"
#include "context.cuh"

namespace ahead {
namespace {

constexpr int kTblTile = 8192;      // text bytes per count / parse CTA
constexpr int kTblBack = 1024;      // bytes staged before a tile
constexpr int kTblThreads = 256;
constexpr int kTblLineMax = 1022;   // longest line content (without '\n')
constexpr int kTblMaxCols = 128;
constexpr int kScanThreads = 1024;

// error word: (global row << 3) | code, the smallest one wins
enum : uint32_t { kTblErrLong = 1, kTblErrMore = 2, kTblErrFewer = 3, kTblErrFixed = 4 };

struct TblColDev {
    uint32_t kind;
    uint32_t width;
    uint64_t A;
    char* data;
};

struct TblParams {
    const uint8_t* text;
    uint64_t len;
    uint64_t row0;       // row of the block's line 0
    uint64_t max_lines;  // lines at or past this index are not stored
    const uint64_t* tile_base;
    unsigned long long* err;
    uint32_t delim[8];   // 256-bit delimiter set
    int32_t single;      // the delimiter when the set has one byte, else -1
    int32_t ncols;
    int32_t ignore_more;
    TblColDev cols[kTblMaxCols];
};

// ------------------------------------------------------------ line counting
AHEAD_DEV uint32_t nl_count4(uint32_t w) { return __popc(__vcmpeq4(w, 0x0a0a0a0au)) >> 3; }

__global__ void __launch_bounds__(kTblThreads) tbl_count_kernel(const uint8_t* __restrict__ text, uint64_t len,
                                                                uint32_t* __restrict__ tile_cnt) {
    const uint64_t beg = (uint64_t)blockIdx.x * kTblTile;
    const uint64_t end = min(beg + (uint64_t)kTblTile, len);
    uint32_t c = 0;
    for (uint64_t p = beg + (uint64_t)threadIdx.x * 16; p < end; p += (uint64_t)kTblThreads * 16) {
        if (p + 16 <= end) {
            uint4 w = *reinterpret_cast<const uint4*>(text + p);
            c += nl_count4(w.x) + nl_count4(w.y) + nl_count4(w.z) + nl_count4(w.w);
        } else {
            for (uint64_t q = p; q < end; ++q) c += text[q] == '\n';
        }
    }
    __shared__ uint32_t ws[kTblThreads / 32];
    for (int d = 16; d > 0; d >>= 1) c += __shfl_xor_sync(kFull, c, d);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t s = 0;
        for (int i = 0; i < kTblThreads / 32; ++i) s += ws[i];
        tile_cnt[blockIdx.x] = s;
    }
}

// Exclusive prefix of the tile counts; total -> *total.  Also checks that
// the text ends with '\n' (flag 1 in *bad otherwise).
__global__ void __launch_bounds__(kScanThreads) tbl_scan_kernel(const uint32_t* __restrict__ tile_cnt,
                                                                uint32_t ntiles, uint64_t* __restrict__ tile_base,
                                                                uint64_t* total, const uint8_t* text, uint64_t len,
                                                                uint32_t* bad) {
    __shared__ uint64_t ws[kScanThreads / 32];
    const uint32_t per = (ntiles + kScanThreads - 1) / kScanThreads;
    const uint32_t b = threadIdx.x * per, e = min(b + per, ntiles);
    uint64_t s = 0;
    for (uint32_t i = b; i < e; ++i) s += tile_cnt[i];
    uint64_t inc = warp_incl_scan64(s);
    if ((threadIdx.x & 31) == 31) ws[threadIdx.x >> 5] = inc;
    __syncthreads();
    if (threadIdx.x < 32) {
        uint64_t v = ws[threadIdx.x];
        uint64_t vi = warp_incl_scan64(v);
        ws[threadIdx.x] = vi - v;
        if (threadIdx.x == 31) *total = vi;
    }
    __syncthreads();
    uint64_t run = ws[threadIdx.x >> 5] + inc - s;
    for (uint32_t i = b; i < e; ++i) {
        tile_base[i] = run;
        run += tile_cnt[i];
    }
    if (threadIdx.x == 0 && len > 0 && text[len - 1] != '\n') *bad = 1;
}

// ------------------------------------------------------------ conversions
AHEAD_DEV bool c_isspace(uint32_t c) { return c == ' ' || (c >= '\t' && c <= '\r'); }

// strtol(s, nullptr, 10) on the field [b, e) (glibc semantics: leading
// white space, optional sign, decimal digits up to the first non-digit,
// saturation at the long range).  atoi = (int)strtol on LP64 and every
// store keeps only the low bytes, so one routine serves atoi/atol/atoll.
AHEAD_DEV int64_t parse_long(const uint8_t* s, int b, int e) {
    int i = b;
    while (i < e && c_isspace(s[i])) ++i;
    bool neg = false;
    if (i < e && (s[i] == '-' || s[i] == '+')) {
        neg = s[i] == '-';
        ++i;
    }
    uint64_t mag = 0;
    bool ovf = false;
    for (; i < e; ++i) {
        uint32_t d = (uint32_t)s[i] - '0';
        if (d > 9) break;
        if (mag > (~0ull - d) / 10) ovf = true;
        else mag = mag * 10 + d;
    }
    const uint64_t lim = neg ? (1ull << 63) : (1ull << 63) - 1;
    if (ovf || mag > lim) return neg ? INT64_MIN : INT64_MAX;
    return neg ? (int64_t)(0 - mag) : (int64_t)mag;
}

// atof on [b, e): Clinger's exact fast path (W. D. Clinger, "How to read
// floating point numbers accurately", PLDI 1990): a decimal significand M <
// 2^53 and a power of ten |k| <= 22 are both exact doubles, so one IEEE
// multiply or divide is the correctly rounded result strtod returns.
// Anything else (more digits, larger exponents, inf/nan, hex) returns false.
__constant__ double kP10[23] = {1e0,  1e1,  1e2,  1e3,  1e4,  1e5,  1e6,  1e7,  1e8,  1e9,  1e10, 1e11,
                                1e12, 1e13, 1e14, 1e15, 1e16, 1e17, 1e18, 1e19, 1e20, 1e21, 1e22};

AHEAD_DEV bool parse_fixed(const uint8_t* s, int b, int e, double* out) {
    const double* p10 = kP10;
    int i = b;
    while (i < e && c_isspace(s[i])) ++i;
    bool neg = false;
    if (i < e && (s[i] == '-' || s[i] == '+')) {
        neg = s[i] == '-';
        ++i;
    }
    // strtod also reads "inf", "infinity", "nan" and hexadecimal forms
    auto lower = [&](int j) { return j < e ? (s[j] | 0x20u) : 0u; };
    auto hexd = [&](int j) {
        const uint32_t c = lower(j);
        return (c >= '0' && c <= '9') || (c >= 'a' && c <= 'f');
    };
    if ((lower(i) == 'i' && lower(i + 1) == 'n' && lower(i + 2) == 'f') ||
        (lower(i) == 'n' && lower(i + 1) == 'a' && lower(i + 2) == 'n'))
        return false;
    if (i < e && s[i] == '0' && lower(i + 1) == 'x' && (hexd(i + 2) || (lower(i + 2) == '.' && hexd(i + 3))))
        return false;
    uint64_t m = 0;
    int k = 0, ndig = 0;
    bool exact = true, frac = false;
    for (; i < e; ++i) {
        uint32_t c = s[i];
        if (c == '.' && !frac) {
            frac = true;
            continue;
        }
        uint32_t d = c - '0';
        if (d > 9) break;
        ++ndig;
        if (m < (1ull << 53) / 10 + 1 && m * 10 + d <= (1ull << 53)) {
            m = m * 10 + d;
            if (frac) --k;
        } else if (d != 0) {
            exact = false;
        } else if (!frac) {
            ++k;  // a trailing integer zero that no longer fits: scale instead
        }
    }
    if (ndig == 0) {  // no conversion: strtod returns +0.0
        *out = 0.0;
        return true;
    }
    if (i < e && (s[i] | 0x20u) == 'e') {
        int j = i + 1;
        bool eneg = false;
        if (j < e && (s[j] == '-' || s[j] == '+')) {
            eneg = s[j] == '-';
            ++j;
        }
        if (j < e && (uint32_t)(s[j] - '0') <= 9) {
            int x = 0;
            for (; j < e && (uint32_t)(s[j] - '0') <= 9; ++j) x = min(x * 10 + (s[j] - '0'), 100000);
            k += eneg ? -x : x;
        }
    }
    if (!exact) return false;
    double v;
    if (m == 0) v = 0.0;
    else if (k == 0) v = (double)m;
    else if (k > 0 && k <= 22) v = (double)m * p10[k];
    else if (k < 0 && k >= -22) v = (double)m / p10[-k];
    else return false;
    *out = neg ? -v : v;
    return true;
}

AHEAD_DEV void store_int(char* p, uint32_t width, uint64_t row, uint64_t v) {
    switch (width) {
        case 1: reinterpret_cast<uint8_t*>(p)[row] = (uint8_t)v; break;
        case 2: reinterpret_cast<uint16_t*>(p)[row] = (uint16_t)v; break;
        case 4: reinterpret_cast<uint32_t*>(p)[row] = (uint32_t)v; break;
        default: reinterpret_cast<uint64_t*>(p)[row] = v; break;
    }
}

AHEAD_DEV void tbl_error(const TblParams& p, uint64_t row, uint32_t code) {
    atomicMin(p.err, (unsigned long long)((row << 3) | code));
}

// One line [b, e) of the staged window (e is the '\n').  Transaction.cpp:
// 487-581: a trailing '\r' is dropped, fields are the maximal runs of
// non-delimiter bytes (strtok), each converted by its column's type.
template <bool ONE>
AHEAD_DEV void parse_line(const TblParams& p, const uint8_t* w, const uint32_t* dm, uint32_t d1,
                          const TblColDev* cols, int b, int e, uint64_t row) {
    auto isd = [&](uint32_t c) { return ONE ? c == d1 : ((dm[c >> 5] >> (c & 31)) & 1u) != 0; };
    if (e > b && w[e - 1] == '\r') --e;
    int pos = b, col = 0;
    for (;;) {
        // strtok stops at a NUL byte as at the end of the line
        uint32_t c = 0;
        while (pos < e && (c = w[pos]) != 0 && isd(c)) ++pos;
        if (pos >= e || c == 0) break;
        const int ts = pos;
        while (pos < e && (c = w[pos]) != 0 && !isd(c)) ++pos;
        if (col >= p.ncols) {
            if (p.ignore_more) break;
            tbl_error(p, row, kTblErrMore);
            return;
        }
        const TblColDev cd = cols[col];
        switch (cd.kind) {
            case AHEAD_TBLK_INT:
                store_int(cd.data, cd.width, row, (uint64_t)parse_long(w, ts, pos));
                break;
            case AHEAD_TBLK_RES:
                store_int(cd.data, cd.width, row, (uint64_t)parse_long(w, ts, pos) * cd.A);
                break;
            case AHEAD_TBLK_STRING: {
                char* d = cd.data + row * cd.width;
                const uint32_t n = min((uint32_t)(pos - ts), cd.width);
                for (uint32_t k = 0; k < n; ++k) d[k] = (char)w[ts + k];
                for (uint32_t k = n; k < cd.width; ++k) d[k] = 0;
                break;
            }
            case AHEAD_TBLK_FIXED: {
                double v = 0.0;
                if (!parse_fixed(w, ts, pos, &v)) tbl_error(p, row, kTblErrFixed);
                reinterpret_cast<double*>(cd.data)[row] = v;
                break;
            }
            case AHEAD_TBLK_CHAR:
                cd.data[row] = (char)w[ts];
                break;
            default:
                break;
        }
        ++col;
    }
    if (col < p.ncols) tbl_error(p, row, kTblErrFewer);
}

__global__ void __launch_bounds__(kTblThreads) tbl_parse_kernel(const __grid_constant__ TblParams p) {
    __shared__ __align__(16) uint8_t win[kTblBack + kTblTile];
    __shared__ uint16_t nl[kTblTile];
    __shared__ uint32_t dm[8];
    __shared__ uint32_t wsum[kTblThreads / 32];
    __shared__ int first_start;
    __shared__ TblColDev cols[kTblMaxCols];

    const uint64_t tbeg = (uint64_t)blockIdx.x * kTblTile;
    const uint64_t tend = min(tbeg + (uint64_t)kTblTile, p.len);
    const uint64_t wbeg = tbeg >= (uint64_t)kTblBack ? tbeg - kTblBack : 0;
    const uint32_t wlen = (uint32_t)(tend - wbeg);
    const uint32_t toff = (uint32_t)(tbeg - wbeg);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

    if (threadIdx.x < 8) dm[threadIdx.x] = p.delim[threadIdx.x];
    for (int i = threadIdx.x; i < p.ncols; i += kTblThreads) cols[i] = p.cols[i];
    // stage [wbeg, tend): wbeg is a multiple of 16 and text is 16-byte aligned
    for (uint32_t i = threadIdx.x * 16; i < wlen; i += kTblThreads * 16) {
        if (i + 16 <= wlen) {
            *reinterpret_cast<uint4*>(win + i) = *reinterpret_cast<const uint4*>(p.text + wbeg + i);
        } else {
            for (uint32_t j = i; j < wlen; ++j) win[j] = p.text[wbeg + j];
        }
    }
    __syncthreads();

    // line ends inside the tile: thread t owns tile bytes [32t, 32t + 32)
    uint32_t mask = 0;
    const uint32_t mb = toff + threadIdx.x * 32;
    if (mb < wlen) {
        const uint4* q = reinterpret_cast<const uint4*>(win + mb);
        const uint4 a = q[0], c = q[1];
        const uint32_t wd[8] = {a.x, a.y, a.z, a.w, c.x, c.y, c.z, c.w};
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const uint32_t x = __vcmpeq4(wd[i], 0x0a0a0a0au) & 0x01010101u;
            mask |= ((x | (x >> 7) | (x >> 14) | (x >> 21)) & 0xFu) << (4 * i);
        }
        if (wlen - mb < 32) mask &= (1u << (wlen - mb)) - 1;
    }
    const uint32_t cnt = __popc(mask);
    const uint32_t inc = warp_incl_scan(cnt);
    if (lane == 31) wsum[warp] = inc;
    // start of the tile's first line: one past the last '\n' before the tile
    if (warp == 0) {
        int found = -1;
        for (int base = (int)toff - 1; base >= 0; base -= 32) {
            const int i = base - lane;
            const unsigned m = __ballot_sync(kFull, i >= 0 && win[i] == '\n');
            if (m) {
                found = base - (__ffs(m) - 1);
                break;
            }
        }
        if (lane == 0) first_start = found >= 0 ? found + 1 : (wbeg == 0 ? 0 : -1);
    }
    __syncthreads();
    uint32_t before = 0, total = 0;
    for (int i = 0; i < kTblThreads / 32; ++i) {
        before += i < warp ? wsum[i] : 0;
        total += wsum[i];
    }
    uint32_t o = before + inc - cnt;
    while (mask) {
        const int k = __ffs(mask) - 1;
        mask &= mask - 1;
        nl[o++] = (uint16_t)(threadIdx.x * 32 + k);
    }
    __syncthreads();

    const uint64_t line0 = p.tile_base[blockIdx.x];
    for (uint32_t j = threadIdx.x; j < total; j += kTblThreads) {
        const uint64_t line = line0 + j;
        if (line >= p.max_lines) break;
        const uint64_t row = p.row0 + line;
        const int e = (int)toff + nl[j];
        const int b = j == 0 ? first_start : (int)toff + nl[j - 1] + 1;
        if (b < 0 || e - b > kTblLineMax) {
            tbl_error(p, row, kTblErrLong);
            continue;
        }
        if (p.single >= 0) parse_line<true>(p, win, dm, (uint32_t)p.single, cols, b, e, row);
        else parse_line<false>(p, win, dm, 0, cols, b, e, row);
    }
}

// ------------------------------------------------------------ re-encode
template <typename T>
AHEAD_DEV uint4 mul_vec(uint4 v, T f) {
    T* t = reinterpret_cast<T*>(&v);
#pragma unroll
    for (int i = 0; i < (int)(16 / sizeof(T)); ++i) t[i] = (T)(t[i] * f);
    return v;
}

// In place: data[i] *= f (mod 2^(8 sizeof T)), 16-byte vectors, 4 in flight
// per thread.  `head` scalar elements come first so the vectors are aligned.
template <typename T>
__global__ void __launch_bounds__(256) reencode_kernel(T* __restrict__ data, uint64_t n, uint64_t head, T f) {
    constexpr uint64_t kPer = 16 / sizeof(T);
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    if (tid < head) data[tid] = (T)(data[tid] * f);
    const uint64_t nv = (n - head) / kPer;
    uint4* v = reinterpret_cast<uint4*>(data + head);
    uint64_t i = tid;
    for (; i + 3 * nth < nv; i += 4 * nth) {
        uint4 a = v[i], b = v[i + nth], c = v[i + 2 * nth], d = v[i + 3 * nth];
        v[i] = mul_vec<T>(a, f);
        v[i + nth] = mul_vec<T>(b, f);
        v[i + 2 * nth] = mul_vec<T>(c, f);
        v[i + 3 * nth] = mul_vec<T>(d, f);
    }
    for (; i < nv; i += nth) v[i] = mul_vec<T>(v[i], f);
    const uint64_t t0 = head + nv * kPer;
    if (tid < n - t0) data[t0 + tid] = (T)(data[t0 + tid] * f);
}

// ------------------------------------------------------------ host helpers
// Inverse of odd a modulo 2^64 by Newton's iteration x <- x (2 - a x); each
// step doubles the correct low bits (a x = 1 mod 8 holds for x = a).
uint64_t inv64(uint64_t a) {
    uint64_t x = a;
    for (int i = 0; i < 5; ++i) x *= 2 - a * x;
    return x;
}

// A tables of the AN types the loader creates (resilience.hpp:56-109 in the
// reference): the load A is the largest (As[7] / As[15] / As[15],
// Transaction.cpp:357-376), the min-BFW As are AsBFW.
const uint64_t kBfwTiny[] = {1, 3, 29, 233};
const uint64_t kBfwShort[] = {1, 3, 61, 463, 7785, 63877};
const uint64_t kBfwInt[] = {1, 3, 125, 881, 16089};

int tbl_width_of(int t) {
    switch (t) {
        case AHEAD_TBL_TINYINT: case AHEAD_TBL_CHAR: return 1;
        case AHEAD_TBL_SHORTINT: case AHEAD_TBL_RESTINY: return 2;
        case AHEAD_TBL_INT: case AHEAD_TBL_RESSHORT: return 4;
        default: return 8;
    }
}

int tbl_bat_type(int t) {
    switch (t) {
        case AHEAD_TBL_TINYINT: return AHEAD_TINYINT;
        case AHEAD_TBL_SHORTINT: return AHEAD_SHORTINT;
        case AHEAD_TBL_INT: return AHEAD_INT;
        case AHEAD_TBL_LARGEINT: return AHEAD_BIGINT;
        case AHEAD_TBL_RESTINY: return AHEAD_RESTINY;
        case AHEAD_TBL_RESSHORT: return AHEAD_RESSHORT;
        case AHEAD_TBL_RESINT: return AHEAD_RESINT;
        case AHEAD_TBL_RESBIGINT: return AHEAD_RESBIGINT;
        default: return -1;
    }
}

bool tbl_is_res(int t) { return t >= AHEAD_TBL_RESTINY && t <= AHEAD_TBL_RESBIGINT; }

uint64_t umax_of(int t) {
    switch (t) {
        case AHEAD_TBL_RESTINY: return 0xFFull;
        case AHEAD_TBL_RESSHORT: return 0xFFFFull;
        case AHEAD_TBL_RESINT: return 0xFFFFFFFFull;
        default: return 0;
    }
}

uint64_t wmask_bytes(int w) { return w >= 8 ? ~0ull : ((1ull << (8 * w)) - 1); }

// strtok-style split on a delimiter set: maximal runs of non-delimiters
std::vector<std::string> split_fields(const std::string& s, const std::string& delim) {
    std::vector<std::string> out;
    size_t i = 0;
    while (i < s.size()) {
        while (i < s.size() && delim.find(s[i]) != std::string::npos) ++i;
        if (i >= s.size()) break;
        size_t j = i;
        while (j < s.size() && delim.find(s[j]) == std::string::npos) ++j;
        out.push_back(s.substr(i, j - i));
        i = j;
    }
    return out;
}

// One line as fgets(line, 1024) + the '\n' / '\r' strip of Transaction.cpp:
// 167-181; strtok stops at a NUL.
bool read_header_line(FILE* f, std::string& out) {
    char line[1024];
    std::memset(line, 0, sizeof line);
    if (std::fgets(line, sizeof line, f) != line) return false;
    size_t n = std::strlen(line);
    if (n && line[n - 1] == '\n') line[--n] = 0;
    if (n && line[n - 1] == '\r') line[--n] = 0;
    out.assign(line, n);
    return true;
}

// Type name -> type and width, in the order of Transaction.cpp:236-276
// (prefix comparisons: "INT" also matches "INTEGER").
bool tbl_type_of(const std::string& s, int* type, uint32_t* width, std::string* err) {
    auto pre = [&](const char* p) { return s.compare(0, std::strlen(p), p) == 0; };
    if (pre("INTEGER") || pre("INT")) *type = AHEAD_TBL_INT;
    else if (pre("TINYINT")) *type = AHEAD_TBL_TINYINT;
    else if (pre("SHORTINT")) *type = AHEAD_TBL_SHORTINT;
    else if (pre("LARGEINT")) *type = AHEAD_TBL_LARGEINT;
    else if (pre("STRING")) {
        *type = AHEAD_TBL_STRING;
        long maxlen = 64;  // MAXLEN_STRING (MetaRepositoryManager.cpp:41)
        if (s.size() > 6 && s[6] == ':') maxlen = std::atoi(s.c_str() + 7);
        if (maxlen < 0) {
            *err = "data type " + s + " in header has a negative length";
            return false;
        }
        *width = (uint32_t)maxlen + 1;
        return true;
    } else if (pre("FIXED")) *type = AHEAD_TBL_FIXED;
    else if (pre("CHAR")) *type = AHEAD_TBL_CHAR;
    else if (pre("RESTINY")) *type = AHEAD_TBL_RESTINY;
    else if (pre("RESSHORT")) *type = AHEAD_TBL_RESSHORT;
    else if (pre("RESINT")) *type = AHEAD_TBL_RESINT;
    else if (pre("RESBIGINT")) *type = AHEAD_TBL_RESBIGINT;
    else {
        *err = "data type " + s + " in header unknown";
        return false;
    }
    *width = (uint32_t)tbl_width_of(*type);
    return true;
}

struct HeaderCol {
    std::string name;
    int type;
    uint32_t width;
};

int read_header(const std::string& path, const char* prefix, const std::string& delim, std::vector<HeaderCol>& cols,
                std::string* err) {
    const std::string hp = path + "_header.csv";
    FILE* f = std::fopen(hp.c_str(), "r");
    if (!f) {
        *err = "header file cannot be opened (" + hp + ")";
        return AHEAD_BAD_ARG;
    }
    std::string l1, l2;
    bool ok1 = read_header_line(f, l1), ok2 = ok1 && read_header_line(f, l2);
    std::fclose(f);
    if (!ok1 || !ok2) {
        *err = "error reading line of " + hp;
        return AHEAD_BAD_ARG;
    }
    const std::string pfx = prefix ? prefix : "";
    std::vector<std::string> names = split_fields(l1, delim), types = split_fields(l2, delim);
    if (names.empty()) {
        *err = "header " + hp + " names no column";
        return AHEAD_BAD_ARG;
    }
    if (names.size() != types.size()) {
        *err = "header " + hp + " has " + std::to_string(names.size()) + " names but " +
               std::to_string(types.size()) + " types";
        return AHEAD_BAD_ARG;
    }
    cols.clear();
    for (size_t i = 0; i < names.size(); ++i) {
        if (pfx.size() + names[i].size() > 255) {
            *err = "name of column is too long (>255)";
            return AHEAD_BAD_ARG;
        }
        HeaderCol c;
        c.name = pfx + names[i];
        if (!tbl_type_of(types[i], &c.type, &c.width, err)) return AHEAD_BAD_ARG;
        cols.push_back(c);
    }
    return AHEAD_OK;
}

bool build_delim(const char* delim, uint32_t dm[8], std::string* set) {
    const char* d = delim ? delim : "|";
    std::memset(dm, 0, 8 * sizeof(uint32_t));
    if (!*d) return false;
    for (const unsigned char* q = (const unsigned char*)d; *q; ++q) dm[*q >> 5] |= 1u << (*q & 31);
    if (set) *set = d;
    return true;
}

double ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// pread / pwrite of [off, off + n) of fd with up to 16 threads (slices of at
// least 4 MiB): copies out of the page cache scale with the threads
bool pio_all(int fd, char* buf, uint64_t off, uint64_t n, bool write) {
    const uint64_t kSlice = 4ull << 20;
    const uint64_t hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    int nt = (int)std::min<uint64_t>(hw, (n + kSlice - 1) / kSlice);
    auto work = [&](int t, bool* ok) {
        const uint64_t per = (n + nt - 1) / nt;
        uint64_t b = per * t, e = std::min(n, b + per);
        while (b < e) {
            ssize_t r = write ? ::pwrite(fd, buf + b, e - b, (off_t)(off + b))
                              : ::pread(fd, buf + b, e - b, (off_t)(off + b));
            if (r <= 0) {
                *ok = false;
                return;
            }
            b += (uint64_t)r;
        }
        *ok = true;
    };
    if (nt <= 1) {
        bool ok = true;
        if (n) work(0, &ok);
        return ok;
    }
    std::vector<std::thread> th;
    bool oks[16];
    for (int t = 0; t < nt; ++t) th.emplace_back(work, t, &oks[t]);
    for (auto& x : th) x.join();
    for (int t = 0; t < nt; ++t)
        if (!oks[t]) return false;
    return true;
}

bool pread_all(int fd, char* dst, uint64_t off, uint64_t n) { return pio_all(fd, dst, off, n, false); }

struct EvPair {
    cudaEvent_t a = nullptr, b = nullptr;
    double* sink = nullptr;
};

}  // namespace
}  // namespace ahead

using namespace ahead;

struct TblColHost {
    std::string name;
    int tbl_type = 0;
    uint32_t width = 1;
    bool from_file = false;
    uint64_t A = 1, Ainv = 1, umax = 0;
    char* data = nullptr;
    uint64_t count = 0;
    uint64_t cap = 0;
};

struct ahead_table {
    int device = 0;
    std::vector<TblColHost> cols;
    uint64_t rows = 0;
    ahead_load_stats stats{};
    ~ahead_table() {
        for (auto& c : cols)
            if (c.data) cudaFree(c.data);
    }
};

namespace {

// Device scratch of the text path: two text blocks, tile counts / bases and
// a small result area ([0] line total, [1] error word, [2] "no trailing
// newline" flag).
struct TblScratch {
    uint8_t* text[2] = {nullptr, nullptr};
    uint32_t* tile_cnt = nullptr;
    uint64_t* tile_base = nullptr;
    uint64_t* words = nullptr;
    uint64_t text_cap = 0;
    uint32_t tile_cap = 0;
    void release() {
        for (auto*& t : text) {
            if (t) cudaFree(t);
            t = nullptr;
        }
        if (tile_cnt) cudaFree(tile_cnt);
        if (tile_base) cudaFree(tile_base);
        if (words) cudaFree(words);
        tile_cnt = nullptr;
        tile_base = nullptr;
        words = nullptr;
        text_cap = 0;
        tile_cap = 0;
    }
    ~TblScratch() { release(); }
    int init(uint64_t cap, int nbuf) {
        if (text_cap >= cap && (nbuf < 2 || text[1])) return AHEAD_OK;
        release();
        text_cap = (cap + 15) & ~15ull;
        tile_cap = (uint32_t)((text_cap + kTblTile - 1) / kTblTile);
        for (int i = 0; i < nbuf; ++i)
            if (cudaMalloc(&text[i], text_cap + 16) != cudaSuccess) return AHEAD_NO_MEMORY;
        if (cudaMalloc(&tile_cnt, (size_t)tile_cap * 4) != cudaSuccess) return AHEAD_NO_MEMORY;
        if (cudaMalloc(&tile_base, (size_t)tile_cap * 8) != cudaSuccess) return AHEAD_NO_MEMORY;
        if (cudaMalloc(&words, 64) != cudaSuccess) return AHEAD_NO_MEMORY;
        return AHEAD_OK;
    }
};

// count + scan of one text block; the line total and the trailing-newline
// flag land in words[0] / words[2] (copied to h[0] / h[2] asynchronously)
void launch_count(ahead_ctx* ctx, const TblScratch& s, const uint8_t* text, uint64_t len, uint64_t* h) {
    const uint32_t ntiles = (uint32_t)((len + kTblTile - 1) / kTblTile);
    cudaMemsetAsync(s.words, 0, 8, ctx->stream);
    cudaMemsetAsync(s.words + 2, 0, 8, ctx->stream);
    tbl_count_kernel<<<ntiles, kTblThreads, 0, ctx->stream>>>(text, len, s.tile_cnt);
    tbl_scan_kernel<<<1, kScanThreads, 0, ctx->stream>>>(s.tile_cnt, ntiles, s.tile_base, s.words, text, len,
                                                         reinterpret_cast<uint32_t*>(s.words + 2));
    ctx->launches += 2;
    cudaMemcpyAsync(h, s.words, 24, cudaMemcpyDeviceToHost, ctx->stream);
}

int fill_params(TblParams& p, const ahead_tbl_col* cols, int ncols, const char* delim, int ignore_more,
                std::string* err) {
    std::memset(&p, 0, sizeof p);
    if (ncols <= 0 || ncols > kTblMaxCols) {
        *err = "between 1 and 128 columns";
        return AHEAD_BAD_ARG;
    }
    std::string dset;
    if (!build_delim(delim, p.delim, &dset)) {
        *err = "empty delimiter set";
        return AHEAD_BAD_ARG;
    }
    p.single = dset.size() == 1 ? (int32_t)(unsigned char)dset[0] : -1;
    p.ncols = ncols;
    p.ignore_more = ignore_more ? 1 : 0;
    for (int i = 0; i < ncols; ++i) {
        const ahead_tbl_col& c = cols[i];
        bool ok = true;
        switch (c.kind) {
            case AHEAD_TBLK_SKIP: break;
            case AHEAD_TBLK_INT: ok = c.width == 1 || c.width == 2 || c.width == 4 || c.width == 8; break;
            case AHEAD_TBLK_RES: ok = c.width == 2 || c.width == 4 || c.width == 8; break;
            case AHEAD_TBLK_STRING: ok = c.width >= 1; break;
            case AHEAD_TBLK_FIXED: ok = c.width == 8; break;
            case AHEAD_TBLK_CHAR: ok = c.width == 1; break;
            default: ok = false;
        }
        if (!ok || (c.kind != AHEAD_TBLK_SKIP && !c.data)) {
            *err = "column " + std::to_string(i) + ": bad kind, width or data pointer";
            return AHEAD_BAD_ARG;
        }
        p.cols[i].kind = (uint32_t)c.kind;
        p.cols[i].width = c.width;
        p.cols[i].A = c.A & wmask_bytes((int)std::min<uint32_t>(c.width, 8));
        p.cols[i].data = (char*)c.data;
    }
    return AHEAD_OK;
}

void launch_parse(ahead_ctx* ctx, TblParams& p, const TblScratch& s, const uint8_t* text, uint64_t len) {
    const uint32_t ntiles = (uint32_t)((len + kTblTile - 1) / kTblTile);
    p.text = text;
    p.len = len;
    p.tile_base = s.tile_base;
    p.err = reinterpret_cast<unsigned long long*>(s.words + 1);
    tbl_parse_kernel<<<ntiles, kTblThreads, 0, ctx->stream>>>(p);
    ctx->launches += 1;
}

int tbl_status(uint64_t errw, uint64_t* bad_row, std::string* msg) {
    if (errw == ~0ull) return AHEAD_OK;
    *bad_row = errw >> 3;
    const uint32_t code = (uint32_t)(errw & 7);
    const std::string at = "line " + std::to_string(*bad_row + 1);
    switch (code) {
        case kTblErrLong: *msg = at + ": longer than 1022 characters"; return AHEAD_BAD_ARG;
        case kTblErrMore: *msg = at + ": more values than types registered"; return AHEAD_BAD_ARG;
        case kTblErrFewer: *msg = at + ": fewer values than columns"; return AHEAD_SIZE_MISMATCH;
        default: *msg = at + ": FIXED value outside the exact decimal fast path"; return AHEAD_UNSUPPORTED;
    }
}

template <typename T>
void launch_reencode_t(ahead_ctx* ctx, void* data, uint64_t n, uint64_t f) {
    const uint64_t addr = (uint64_t)data;
    uint64_t head = ((16 - (addr & 15)) & 15) / sizeof(T);
    head = std::min(head, n);
    const int grid = std::max(1, ctx->num_sms * 8);
    reencode_kernel<T><<<grid, 256, 0, ctx->stream>>>((T*)data, n, head, (T)f);
    ctx->launches += 1;
}

void launch_reencode(ahead_ctx* ctx, void* data, uint64_t n, int width, uint64_t f) {
    if (n == 0) return;
    if (width == 2) launch_reencode_t<uint16_t>(ctx, data, n, f);
    else if (width == 4) launch_reencode_t<uint32_t>(ctx, data, n, f);
    else launch_reencode_t<uint64_t>(ctx, data, n, f);
}

uint64_t reenc_factor(uint64_t a_old, uint64_t a_new, int width) {
    return (inv64(a_old) * a_new) & wmask_bytes(width);
}

}  // namespace

extern "C" {

uint64_t ahead_tbl_load_a(int t) {
    switch (t) {
        case AHEAD_TBL_RESTINY: return 233;
        case AHEAD_TBL_RESSHORT: return 63877;
        case AHEAD_TBL_RESINT: return 65117;
        default: return 0;
    }
}

uint64_t ahead_tbl_minbfw_a(int t, uint32_t bfw) {
    if (bfw == 0) return 0;
    const uint64_t* tab;
    uint32_t n;
    switch (t) {
        case AHEAD_TBL_RESTINY: tab = kBfwTiny; n = 4; break;
        case AHEAD_TBL_RESSHORT: tab = kBfwShort; n = 6; break;
        case AHEAD_TBL_RESINT: tab = kBfwInt; n = 5; break;
        default: return 0;
    }
    // AsBFW->at(min(AsBFW->size(), minBFW)): out of range at the size itself
    const uint32_t idx = std::min(n, bfw);
    return idx < n ? tab[idx] : 0;
}

int ahead_tbl_read_header(const char* path, const char* prefix, const char* delim, ahead_tbl_header_col* cols,
                          int cap, int* ncols, char* err, size_t errlen) {
    std::string msg;
    int rc = AHEAD_OK;
    std::string dset;
    uint32_t dm[8];
    std::vector<HeaderCol> hc;
    if (!path || !ncols) {
        msg = "path and ncols are required";
        rc = AHEAD_BAD_ARG;
    } else if (!build_delim(delim, dm, &dset)) {
        msg = "empty delimiter set";
        rc = AHEAD_BAD_ARG;
    } else {
        rc = read_header(path, prefix, dset, hc, &msg);
    }
    if (rc == AHEAD_OK) {
        *ncols = (int)hc.size();
        for (int i = 0; i < (int)hc.size() && i < cap; ++i) {
            std::memset(cols[i].name, 0, sizeof cols[i].name);
            std::memcpy(cols[i].name, hc[i].name.data(), hc[i].name.size());
            cols[i].tbl_type = hc[i].type;
            cols[i].width = hc[i].width;
        }
    }
    if (err && errlen) {
        std::snprintf(err, errlen, "%s", msg.c_str());
    }
    return rc;
}

int ahead_gpu_tbl_parse(ahead_ctx* ctx, const void* text, uint64_t len, const char* delim, int ignore_more_data,
                        const ahead_tbl_col* cols, int ncols, uint64_t row0, uint64_t cap, uint64_t max_lines,
                        uint64_t* lines, uint64_t* bad_line) {
    if (!ctx || !lines || !cols || (!text && len)) return fail(ctx, AHEAD_BAD_ARG, "null argument");
    if (((uint64_t)text & 15) != 0) return fail(ctx, AHEAD_BAD_ARG, "text must be 16-byte aligned");
    *lines = 0;
    if (bad_line) *bad_line = 0;
    TblParams p;
    std::string msg;
    int rc = fill_params(p, cols, ncols, delim, ignore_more_data, &msg);
    if (rc != AHEAD_OK) return fail(ctx, rc, msg);
    if (len == 0) return AHEAD_OK;
    TblScratch s;
    // only the tile arrays and the result words: the text stays where it is
    s.tile_cap = (uint32_t)((len + kTblTile - 1) / kTblTile);
    if (cudaMalloc(&s.tile_cnt, (size_t)s.tile_cap * 4) != cudaSuccess ||
        cudaMalloc(&s.tile_base, (size_t)s.tile_cap * 8) != cudaSuccess || cudaMalloc(&s.words, 64) != cudaSuccess)
        return fail(ctx, AHEAD_NO_MEMORY, "parse scratch");
    uint64_t* h = ctx->h_stage;
    launch_count(ctx, s, (const uint8_t*)text, len, h);
    AHEAD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    AHEAD_CUDA(ctx, cudaGetLastError());
    if (h[2]) return fail(ctx, AHEAD_BAD_ARG, "text does not end with a newline");
    *lines = h[0];
    const uint64_t n = std::min(h[0], max_lines);
    if (row0 + n > cap) return fail(ctx, AHEAD_CAPACITY, "columns too small for the lines");
    p.row0 = row0;
    p.max_lines = max_lines;
    AHEAD_CUDA(ctx, cudaMemsetAsync(s.words + 1, 0xff, 8, ctx->stream));
    launch_parse(ctx, p, s, (const uint8_t*)text, len);
    AHEAD_CUDA(ctx, cudaGetLastError());
    AHEAD_CUDA(ctx, cudaMemcpyAsync(h + 1, s.words + 1, 8, cudaMemcpyDeviceToHost, ctx->stream));
    AHEAD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    uint64_t bad = 0;
    rc = tbl_status(h[1], &bad, &msg);
    if (rc != AHEAD_OK) {
        if (bad_line) *bad_line = bad - row0;
        return fail(ctx, rc, "line " + std::to_string(bad - row0 + 1) + msg.substr(msg.find(':')));
    }
    return AHEAD_OK;
}

int ahead_gpu_reencode(ahead_ctx* ctx, void* data, uint64_t n, int width, uint64_t a_old, uint64_t a_new) {
    if (!ctx || (!data && n)) return fail(ctx, AHEAD_BAD_ARG, "null argument");
    if (width != 2 && width != 4 && width != 8) return fail(ctx, AHEAD_BAD_ARG, "width must be 2, 4 or 8");
    if (!(a_old & 1) || !(a_new & 1)) return fail(ctx, AHEAD_BAD_ARG, "A must be odd");
    if ((uint64_t)data % (uint64_t)width) return fail(ctx, AHEAD_BAD_ARG, "data not aligned to its width");
    launch_reencode(ctx, data, n, width, reenc_factor(a_old, a_new, width));
    AHEAD_CUDA(ctx, cudaGetLastError());
    AHEAD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return AHEAD_OK;
}

int ahead_table_ncols(const ahead_table* t) { return t ? (int)t->cols.size() : 0; }
uint64_t ahead_table_rows(const ahead_table* t) { return t ? t->rows : 0; }

int ahead_table_column(const ahead_table* t, int i, ahead_table_col* out) {
    if (!t || !out || i < 0 || i >= (int)t->cols.size()) return AHEAD_BAD_ARG;
    const TblColHost& c = t->cols[i];
    out->name = c.name.c_str();
    out->tbl_type = c.tbl_type;
    out->type = tbl_bat_type(c.tbl_type);
    out->width = c.width;
    out->from_file = c.from_file ? 1 : 0;
    out->A = c.A;
    out->Ainv = c.Ainv;
    out->unenc_max = c.umax;
    out->data = c.data;
    out->count = c.count;
    return AHEAD_OK;
}

int ahead_table_stats(const ahead_table* t, ahead_load_stats* out) {
    if (!t || !out) return AHEAD_BAD_ARG;
    *out = t->stats;
    return AHEAD_OK;
}

void ahead_table_destroy(ahead_table* t) { delete t; }

}  // extern "C"

namespace {

// Pinned double buffer of the loader.  It lives in the context (pinning
// hundreds of MB costs tenths of a second) and only grows.
struct Pinned {
    char* p[2] = {nullptr, nullptr};
    uint64_t cap = 0;
    void release() {
        for (auto*& x : p) {
            if (x) cudaFreeHost(x);
            x = nullptr;
        }
        cap = 0;
    }
    ~Pinned() { release(); }
    int init(uint64_t c) {
        if (cap >= c) return AHEAD_OK;
        release();
        for (auto*& x : p)
            if (cudaMallocHost(&x, c) != cudaSuccess) {
                release();
                return AHEAD_NO_MEMORY;
            }
        cap = c;
        return AHEAD_OK;
    }
};

struct LoadStaging {
    Pinned pin;
    TblScratch dev;
};

LoadStaging* staging_of(ahead_ctx* ctx) {
    if (!ctx->loader) ctx->loader = std::shared_ptr<void>(new LoadStaging(), [](void* p) { delete (LoadStaging*)p; });
    return static_cast<LoadStaging*>(ctx->loader.get());
}

struct Fd {
    int fd = -1;
    ~Fd() {
        if (fd >= 0) ::close(fd);
    }
};

uint64_t file_size(int fd) {
    struct stat st;
    return fstat(fd, &st) == 0 ? (uint64_t)st.st_size : 0;
}

bool file_exists(const std::string& p) {
    Fd f;
    f.fd = ::open(p.c_str(), O_RDONLY);
    return f.fd >= 0;
}

struct Loader {
    ahead_ctx* ctx;
    ahead_table* t;
    std::string path;
    ahead_load_opts o;
    uint64_t block;
    uint64_t stage = 0;  // bytes of each staging buffer this load uses
    std::vector<EvPair> evs;
    std::string msg;

    void ev_begin(EvPair& e, double* sink) {
        cudaEventCreate(&e.a);
        cudaEventCreate(&e.b);
        e.sink = sink;
        cudaEventRecord(e.a, ctx->stream);
    }
    void ev_end(EvPair& e) {
        cudaEventRecord(e.b, ctx->stream);
        evs.push_back(e);
    }
    void ev_collect() {
        for (auto& e : evs) {
            float ms = 0;
            if (cudaEventElapsedTime(&ms, e.a, e.b) == cudaSuccess) *e.sink += ms;
            cudaEventDestroy(e.a);
            cudaEventDestroy(e.b);
        }
        evs.clear();
    }
    ~Loader() {
        ev_collect();
        for (auto& ev : bdone)
            if (ev) cudaEventDestroy(ev);
    }

    // Transaction.cpp:416-479 and ColumnManager.cpp:283-371: the whole file,
    // then (min BFW) the re-encode of every value on the device.
    // pinned-buffer turns of the binary reads, shared by every file of the
    // load, so one file's copies overlap the next file's reads
    cudaEvent_t bdone[2] = {nullptr, nullptr};
    bool bused[2] = {false, false};
    int bk = 0;

    int read_binary(TblColHost& c, const std::string& fp, Pinned& pin, uint64_t new_a) {
        Fd f;
        f.fd = ::open(fp.c_str(), O_RDONLY);
        if (f.fd < 0) {
            msg = "error loading binary data from file \"" + fp + "\"";
            return AHEAD_BAD_ARG;
        }
        const uint64_t n = file_size(f.fd) / c.width;
        const uint64_t bytes = n * c.width;
        c.count = n;
        c.cap = n;
        if (bytes && cudaMalloc(&c.data, bytes) != cudaSuccess) {
            msg = "device memory for column " + c.name;
            return AHEAD_NO_MEMORY;
        }
        if (!bdone[0]) {
            cudaEventCreateWithFlags(&bdone[0], cudaEventDisableTiming);
            cudaEventCreateWithFlags(&bdone[1], cudaEventDisableTiming);
        }
        const uint64_t step = (stage / c.width) * c.width;
        uint64_t off = 0;
        while (off < bytes) {
            const uint64_t m = std::min(step, bytes - off);
            const int q = bk & 1;
            char* hb = pin.p[q];
            if (bused[q]) cudaEventSynchronize(bdone[q]);
            auto t0 = std::chrono::steady_clock::now();
            if (!pread_all(f.fd, hb, off, m)) {
                msg = "error loading binary data from file \"" + fp + "\"";
                return AHEAD_BAD_ARG;
            }
            t->stats.file_ms += ms_since(t0);
            cudaMemcpyAsync(c.data + off, hb, m, cudaMemcpyHostToDevice, ctx->stream);
            cudaEventRecord(bdone[q], ctx->stream);
            bused[q] = true;
            off += m;
            ++bk;
        }
        t->stats.binary_bytes += bytes;
        if (new_a) {
            EvPair e;
            ev_begin(e, &t->stats.reencode_ms);
            launch_reencode(ctx, c.data, n, (int)c.width, reenc_factor(c.A, new_a, (int)c.width));
            ev_end(e);
            t->stats.reencoded += n;
            c.A = new_a;
            c.Ainv = inv64(new_a) & wmask_bytes((int)c.width);
        }
        return AHEAD_OK;
    }

    int grow(std::vector<int>& parsed, uint64_t need, uint64_t rows) {
        for (int i : parsed) {
            TblColHost& c = t->cols[i];
            if (c.cap >= need) continue;
            char* nd = nullptr;
            if (cudaMalloc(&nd, need * c.width) != cudaSuccess) {
                msg = "device memory for column " + c.name;
                return AHEAD_NO_MEMORY;
            }
            if (c.data) {
                if (rows) cudaMemcpyAsync(nd, c.data, rows * c.width, cudaMemcpyDeviceToDevice, ctx->stream);
                cudaStreamSynchronize(ctx->stream);
                cudaFree(c.data);
            }
            c.data = nd;
            c.cap = need;
        }
        return AHEAD_OK;
    }

    // Transaction.cpp:481-590, one text block at a time.
    int parse_text(std::vector<int>& parsed, Pinned& pin, TblScratch& s, const std::string& tp, uint64_t* rows_out) {
        Fd f;
        f.fd = ::open(tp.c_str(), O_RDONLY);
        if (f.fd < 0) {
            msg = "content file cannot be opened (" + tp + ")";
            return AHEAD_BAD_ARG;
        }
        const uint64_t fsize = file_size(f.fd);
        TblParams p;
        std::vector<ahead_tbl_col> tc(t->cols.size());
        for (size_t i = 0; i < t->cols.size(); ++i) {
            const TblColHost& c = t->cols[i];
            tc[i].kind = AHEAD_TBLK_SKIP;
            tc[i].width = c.width;
            tc[i].A = c.A;
            tc[i].data = nullptr;
        }
        for (int i : parsed) {
            const TblColHost& c = t->cols[i];
            switch (c.tbl_type) {
                case AHEAD_TBL_STRING: tc[i].kind = AHEAD_TBLK_STRING; break;
                case AHEAD_TBL_FIXED: tc[i].kind = AHEAD_TBLK_FIXED; break;
                case AHEAD_TBL_CHAR: tc[i].kind = AHEAD_TBLK_CHAR; break;
                case AHEAD_TBL_RESTINY: case AHEAD_TBL_RESSHORT: case AHEAD_TBL_RESINT: tc[i].kind = AHEAD_TBLK_RES; break;
                default: tc[i].kind = AHEAD_TBLK_INT; break;
            }
            tc[i].data = (void*)16;  // placeholder; the real pointer is set per block
        }
        int rc = fill_params(p, tc.data(), (int)tc.size(), o.delim, o.ignore_more_data, &msg);
        if (rc != AHEAD_OK) return rc;
        uint64_t* h = ctx->h_stage;
        uint64_t rows = 0, off = 0, carry = 0;
        const uint64_t limit = o.size;
        int k = 0;
        bool eof = fsize == 0;
        uint64_t have = 0;  // bytes of the current block in pin.p[k & 1]
        // first block
        if (!eof) {
            const uint64_t m = std::min(stage - 1, fsize);
            auto t0 = std::chrono::steady_clock::now();
            if (!pread_all(f.fd, pin.p[0], 0, m)) {
                msg = "error reading " + tp;
                return AHEAD_BAD_ARG;
            }
            t->stats.file_ms += ms_since(t0);
            off = m;
            have = m;
            eof = off >= fsize;
        }
        bool any_parse = false, carry_long = false;
        while (have > 0 && rows < limit) {
            char* hb = pin.p[k & 1];
            if (eof && hb[have - 1] != '\n') hb[have++] = '\n';  // a last line without '\n' is a line
            uint64_t L = have;
            while (L > 0 && hb[L - 1] != '\n') --L;
            if (L == 0 || carry_long) {
                msg = "line " + std::to_string(rows + 1) + ": longer than 1022 characters";
                return AHEAD_BAD_ARG;
            }
            carry = have - L;
            // a partial line already longer than a line may be: an error once
            // the next block reaches it (it may lie past `size`)
            carry_long = carry > (uint64_t)kTblLineMax;
            char* nb = pin.p[(k + 1) & 1];
            if (carry) std::memcpy(nb, hb + L, carry);
            uint8_t* dt = s.text[k & 1];
            cudaMemcpyAsync(dt, hb, L, cudaMemcpyHostToDevice, ctx->stream);
            t->stats.text_bytes += L;
            EvPair ec;
            ev_begin(ec, &t->stats.parse_ms);
            launch_count(ctx, s, dt, L, h);
            ev_end(ec);
            // read the next block while the device counts this one
            uint64_t next = carry;
            if (!eof) {
                const uint64_t m = std::min(stage - 1 - carry, fsize - off);
                auto t0 = std::chrono::steady_clock::now();
                if (!pread_all(f.fd, nb + carry, off, m)) {
                    msg = "error reading " + tp;
                    return AHEAD_BAD_ARG;
                }
                t->stats.file_ms += ms_since(t0);
                off += m;
                next += m;
                eof = off >= fsize;
            }
            cudaError_t ce = cudaStreamSynchronize(ctx->stream);
            if (ce != cudaSuccess) {
                msg = std::string("text block: ") + cudaGetErrorString(ce);
                return AHEAD_CUDA_ERROR;
            }
            if (any_parse && h[1] != ~0ull) break;  // the previous block failed
            const uint64_t lines = h[0];
            const uint64_t take = std::min(lines, limit - rows);
            if (k == 0) {
                // capacity: exact for a one-block file, else from the first
                // block's line density
                uint64_t est = lines;
                if (fsize > L) est = (uint64_t)((double)lines / (double)L * (double)fsize * 1.02) + 1024;
                rc = grow(parsed, std::max(std::min(est, limit), take), rows);
                if (rc != AHEAD_OK) return rc;
            }
            const uint64_t need = rows + take;
            bool short_cap = false;
            for (int i : parsed) short_cap |= t->cols[i].cap < need;
            if (short_cap) {
                rc = grow(parsed, std::min(need + need / 4, limit), rows);
                if (rc != AHEAD_OK) return rc;
            }
            for (int i : parsed) p.cols[i].data = t->cols[i].data;
            p.row0 = rows;
            p.max_lines = take;
            cudaMemsetAsync(s.words + 1, 0xff, 8, ctx->stream);
            EvPair ep;
            ev_begin(ep, &t->stats.parse_ms);
            if (take) launch_parse(ctx, p, s, dt, L);
            ev_end(ep);
            cudaMemcpyAsync(h + 1, s.words + 1, 8, cudaMemcpyDeviceToHost, ctx->stream);
            any_parse = true;
            rows += take;
            t->stats.blocks += 1;
            have = next;
            ++k;
        }
        cudaError_t ce = cudaStreamSynchronize(ctx->stream);
        if (ce != cudaSuccess) {
            msg = std::string("text parse: ") + cudaGetErrorString(ce);
            return AHEAD_CUDA_ERROR;
        }
        if (any_parse) {
            uint64_t bad = 0;
            rc = tbl_status(h[1], &bad, &msg);
            if (rc != AHEAD_OK) return rc;
        }
        *rows_out = rows;
        return AHEAD_OK;
    }

    // Transaction.cpp:594-610: raw values of each newly parsed column
    int write_binary(const TblColHost& c, const std::string& fp, Pinned& pin) {
        Fd f;
        f.fd = ::open(fp.c_str(), O_WRONLY | O_CREAT | O_TRUNC, 0644);
        if (f.fd < 0) {
            msg = "cannot write " + fp;
            return AHEAD_BAD_ARG;
        }
        // device -> pinned block k+1 is in flight while block k is written
        const uint64_t bytes = c.count * c.width;
        cudaEvent_t done[2];
        cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming);
        cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming);
        auto issue = [&](uint64_t off, int k) {
            const uint64_t m = std::min(stage, bytes - off);
            cudaMemcpyAsync(pin.p[k & 1], c.data + off, m, cudaMemcpyDeviceToHost, ctx->stream);
            cudaEventRecord(done[k & 1], ctx->stream);
        };
        int rc = AHEAD_OK;
        uint64_t off = 0;
        int k = 0;
        if (bytes) issue(0, 0);
        while (off < bytes) {
            const uint64_t m = std::min(stage, bytes - off);
            if (cudaEventSynchronize(done[k & 1]) != cudaSuccess) {
                msg = "device read of column " + c.name;
                rc = AHEAD_CUDA_ERROR;
                break;
            }
            if (off + m < bytes) issue(off + m, k + 1);
            auto t0 = std::chrono::steady_clock::now();
            const bool ok = pio_all(f.fd, pin.p[k & 1], off, m, true);
            t->stats.file_ms += ms_since(t0);
            if (!ok) {
                msg = "cannot write " + fp;
                rc = AHEAD_BAD_ARG;
                break;
            }
            off += m;
            ++k;
        }
        cudaStreamSynchronize(ctx->stream);
        cudaEventDestroy(done[0]);
        cudaEventDestroy(done[1]);
        if (rc == AHEAD_OK) t->stats.written_bytes += bytes;
        return rc;
    }

    int run() {
        std::string dset;
        uint32_t dm[8];
        if (!build_delim(o.delim, dm, &dset)) {
            msg = "empty delimiter set";
            return AHEAD_BAD_ARG;
        }
        std::vector<HeaderCol> hc;
        int rc = read_header(path, o.prefix, dset, hc, &msg);
        if (rc != AHEAD_OK) return rc;
        const size_t nc = hc.size();
        t->cols.resize(nc);
        for (size_t i = 0; i < nc; ++i) {
            TblColHost& c = t->cols[i];
            c.name = hc[i].name;
            c.tbl_type = hc[i].type;
            c.width = hc[i].width;
            if (c.tbl_type == AHEAD_TBL_RESBIGINT) {
                msg = "data type RESBIGINT in header currently unsupported for load";
                return AHEAD_UNSUPPORTED;
            }
            if (tbl_is_res(c.tbl_type)) {
                c.A = ahead_tbl_load_a(c.tbl_type);
                c.Ainv = inv64(c.A) & wmask_bytes((int)c.width);
                c.umax = umax_of(c.tbl_type);
            }
        }
        // column files (Transaction.cpp:286-313, 411-479)
        std::vector<std::string> cpath(nc);
        std::vector<bool> present(nc);
        bool all_present = true;
        for (size_t i = 0; i < nc; ++i) {
            cpath[i] = path + "_" + t->cols[i].name + ".ahead";
            present[i] = file_exists(cpath[i]);
            all_present = all_present && present[i];
        }
        const std::string tp = path + ".tbl";
        const bool all_converted = o.convert_table_files && all_present;
        bool need_text = false;
        for (size_t i = 0; i < nc; ++i) need_text = need_text || !present[i];
        if (need_text && !file_exists(tp)) {
            msg = "content file cannot be opened (" + tp + "). Missing columns are:";
            for (size_t i = 0; i < nc; ++i)
                if (!present[i]) msg += " " + t->cols[i].name;
            return AHEAD_BAD_ARG;
        }
        // a minimum bit-flip weight the AN types of the table cannot meet
        if (o.min_bfw) {
            for (size_t i = 0; i < nc; ++i) {
                const TblColHost& c = t->cols[i];
                if (present[i] && tbl_is_res(c.tbl_type) && !ahead_tbl_minbfw_a(c.tbl_type, o.min_bfw)) {
                    msg = "data type of column " + c.name + " currently does not support a minimum bit flip weight of " +
                          std::to_string(o.min_bfw);
                    return AHEAD_UNSUPPORTED;
                }
            }
        }
        LoadStaging* st = staging_of(ctx);
        Pinned& pin = st->pin;
        uint64_t pin_cap = block;
        {
            uint64_t biggest = 0;
            for (size_t i = 0; i < nc; ++i) {
                Fd f;
                f.fd = ::open(present[i] ? cpath[i].c_str() : tp.c_str(), O_RDONLY);
                if (f.fd >= 0) biggest = std::max(biggest, file_size(f.fd));
            }
            pin_cap = std::max<uint64_t>(std::min(block, biggest + 2 * kTblBack + 64), 4 * kTblBack);
            pin_cap = (pin_cap + 15) & ~15ull;
        }
        rc = pin.init(pin_cap);
        if (rc != AHEAD_OK) {
            msg = "pinned staging buffers";
            return rc;
        }
        stage = pin_cap;
        for (size_t i = 0; i < nc; ++i) {
            if (!present[i]) continue;
            TblColHost& c = t->cols[i];
            c.from_file = true;
            const uint64_t na = (o.min_bfw && tbl_is_res(c.tbl_type)) ? ahead_tbl_minbfw_a(c.tbl_type, o.min_bfw) : 0;
            rc = read_binary(c, cpath[i], pin, na);
            if (rc != AHEAD_OK) return rc;
        }
        {
            const cudaError_t ce = cudaStreamSynchronize(ctx->stream);
            if (ce != cudaSuccess) {
                msg = std::string("binary column read: ") + cudaGetErrorString(ce);
                return AHEAD_CUDA_ERROR;
            }
        }
        std::vector<int> parsed;
        for (size_t i = 0; i < nc; ++i)
            if (!present[i]) parsed.push_back((int)i);
        if (!all_converted && !parsed.empty()) {
            TblScratch& s = st->dev;
            if (s.init(stage, 2) != AHEAD_OK) {
                msg = "device text buffers";
                return AHEAD_NO_MEMORY;
            }
            uint64_t rows = 0;
            rc = parse_text(parsed, pin, s, tp, &rows);
            if (rc != AHEAD_OK) return rc;
            for (int i : parsed) t->cols[i].count = rows;
        }
        // Transaction.cpp:636-645
        for (size_t i = 1; i < nc; ++i) {
            if (t->cols[i].count != t->cols[i - 1].count) {
                msg = "column sizes don't match! previous (" + std::to_string(i - 1) + ", " + t->cols[i - 1].name +
                      ") = " + std::to_string(t->cols[i - 1].count) + ", current (" + std::to_string(i) + ", " +
                      t->cols[i].name + ") = " + std::to_string(t->cols[i].count);
                return AHEAD_SIZE_MISMATCH;
            }
        }
        t->rows = nc ? t->cols[0].count : 0;
        if (o.convert_table_files && !all_converted) {
            for (int i : parsed) {
                rc = write_binary(t->cols[i], cpath[i], pin);
                if (rc != AHEAD_OK) return rc;
            }
        }
        return AHEAD_OK;
    }
};

}  // namespace

extern "C" int ahead_table_load(ahead_ctx* ctx, const char* path, const ahead_load_opts* opts, ahead_table** out) {
    if (!ctx || !out) return fail(ctx, AHEAD_BAD_ARG, "null argument");
    *out = nullptr;
    if (!path || !*path || std::strlen(path) > 1024) return fail(ctx, AHEAD_BAD_ARG, "path missing or too long (>1024)");
    auto t0 = std::chrono::steady_clock::now();
    ahead_load_opts o;
    if (opts) {
        o = *opts;
    } else {
        std::memset(&o, 0, sizeof o);
        o.size = ~0ull;
        o.ignore_more_data = 1;
        o.convert_table_files = 1;
    }
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, AHEAD_CUDA_ERROR, "cudaSetDevice");
    ahead_table* t = new ahead_table();
    t->device = ctx->device;
    Loader L{ctx, t, path, o, (uint64_t)(o.block_mb ? o.block_mb : 64) << 20, 0, {}, {}};
    int rc = L.run();
    cudaError_t ce = cudaStreamSynchronize(ctx->stream);
    L.ev_collect();
    if (rc == AHEAD_OK && ce != cudaSuccess) {
        rc = AHEAD_CUDA_ERROR;
        L.msg = std::string("table load: ") + cudaGetErrorString(ce);
    }
    if (rc != AHEAD_OK) {
        delete t;
        return fail(ctx, rc, L.msg);
    }
    t->stats.total_ms = ms_since(t0);
    *out = t;
    return AHEAD_OK;
}
