// starjoin.cu -- fused star joins: one scan of the fact table answers a batch
// of up to 64 star-join queries.
//
// What it computes is the operator-at-a-time composition of the reference's
// AN operators (the SSB query programs, tools/ssbm/ssbm-q41_continuous.cpp:
// 97-216, and ahead_b200/pipelines.py): per fact row and query, the joined
// dimensions are visited in the fixed order customer, supplier, part, date.
//   * the first joined dimension's foreign key is probed for every row with
//     hashjoinAN semantics (hashjoinAN.tcc:189-215): decoded, checked (an
//     error is reported, the row is still probed), truncated to the 32-bit
//     key type;
//   * every later foreign key and the measures are fetched with positional
//     matchjoinAN semantics (matchjoinAN.tcc:276-297): a corrupt value is
//     reported and drops the row for that query;
//   * price*discount is arithmeticAN<mul, resbigint> of the decoded values
//     times AR (arithmeticAN_scalar.tcc:107), summed per group
//     (aggregate_sum_groupedAN, aggregateAN.tcc:109) with groups numbered by
//     first occurrence (groupbyAN.tcc:83-90, 148-159); an ungrouped query is
//     aggregate_mul_sumAN (aggregateAN_scalar.tcc:98-124).
//
// GPU structure:
//   - schema preparation (once per engine): each dimension's decoded keys
//     are placed into a direct-mapped key -> row array;
//   - per batch, one CUDA graph (or the same launches directly): a clear
//     kernel, one pass over each dimension building per dimension row a
//     64-bit mask of the queries that accept it (predicates on codes), the
//     fact kernel, a finalize kernel (per query the non-empty groups sorted
//     by first row) and a pack kernel (sorts the error log and packs errors
//     and groups into one contiguous result area).  Every launch reads the
//     batch descriptor from device memory, so one captured graph per slot
//     serves every batch;
//   - the fact kernel: a persistent grid; each thread owns 8 rows of a
//     2048-row tile and walks the dimensions in stages (all 8 rows' loads of
//     a stage are in flight together); a foreign key is loaded only while some
//     query that joins it is still alive for the row, so a selective query
//     reads the later columns sparsely; surviving (row, query) pairs add
//     their product to the query's dense group table and atomicMin their row
//     into the group's first-row word;
//   - two slots (descriptor staging, result areas, events) let the host
//     prepare and read back one batch while the other runs.
// Detected errors are appended to a log (query, column, row) that the pack
// kernel sorts; every wait in here is a kernel boundary, none spins.
#include <algorithm>
#include <climits>
#include <cstring>
#include <vector>

#include "ops_common.cuh"

using namespace ahead;

namespace {

constexpr int kSjThreads = 256;
// fact-kernel shapes the tuner chooses from (rows per thread 2, 4, 8): blocks per SM
constexpr int kSjVariants = 3;
constexpr int kSjVarBlocks[kSjVariants] = {4, 3, 2};
constexpr uint32_t kNoRow = 0xffffffffu;
constexpr uint64_t kMaxDense = 1u << 23;  // dense group-index domain per query
constexpr int kErrLogCap = 1 << 16;       // (query, column, row) entries per batch
constexpr int kLogColShift = 54;          // log word: query << 58 | column << 54 | row (rows < 2^32)
constexpr int kSlots = 2;
constexpr int kMaxQ = AHEAD_SJ_MAXQ;
constexpr int kSmemGroups = 4096;         // block-shared group slots (8 B sum + 4 B first row)
constexpr size_t kFactSmem = (size_t)kSmemGroups * 12;
// signature cube: prefix segments, signatures, rows routed to the exact path
constexpr int kMaxSeg = 8;
constexpr uint32_t kMaxSig = 1u << 24;
// fact rows per engine: row numbers, and a tile's end past the last row, stay in 32 bits
constexpr uint64_t kMaxFactRows = (1ull << 32) - (1ull << 16);
constexpr uint32_t kExcCap = 1u << 20;
constexpr int kCubeMinQueries = 4;  // fewer queries: the per-row strategy
enum : uint32_t { kStratRows = 0, kStratCube = 1 };
// cube scan: the set of signatures its first phase did not see
constexpr uint32_t kUnseenLog = 11;
constexpr uint32_t kUnseenSlots = 1u << kUnseenLog;  // open-addressing set of signatures phase 0 did not see
constexpr uint32_t kUnseenCap = kUnseenSlots / 2;
constexpr uint32_t kUnseenEmpty = 0xffffffffu;  // (signatures are below kMaxSig)
constexpr uint64_t kR0PerSig = 16;
constexpr uint64_t kR0Align = 8192;

// join order of the dimensions: customer, supplier, part, date
AHEAD_HD int join_dim(int k) {
    return k == 0 ? AHEAD_SJ_CUSTOMER : k == 1 ? AHEAD_SJ_SUPPLIER : k == 2 ? AHEAD_SJ_PART : AHEAD_SJ_DATE;
}

// One 32-bit record per key of a dimension, at (decoded key - smallest key):
// 0 for a key no row has, else 1 + the row's attributes packed at fixed bit
// offsets (decoded value - the attribute's smallest value), at most
// kAccBits bits.  A row's accept mask depends only on those attributes, so
// each batch tabulates it once per packed value: acc[record] holds the batch
// queries accepting a row with that record (acc[0] = 0).
constexpr int kAccBits = 12;
constexpr uint32_t kAccEntries = (1u << kAccBits) + 1;

struct SjDimDev {
    const unsigned long long* fk;   // fact foreign-key codes
    const uint32_t* rec;            // [krange] key records
    void* code;                     // [krange] the batch's dimension code of each key (cube strategy)
    uint32_t cw, pad;               // code width in bytes: 1 when the codes fit, else 2
    // packed code table (cbits != 0): `per` codes of cbits bits in each 64-bit
    // word, none straddling; word = key * cmagic >> 40 (exact division by per)
    uint32_t cbits, per;
    uint64_t cmagic;
    const unsigned long long* acc;  // [kAccEntries] accept masks by record
    uint64_t fk_ainv, kmin, krange;
    unsigned long long joins, first;  // queries joining / joining first
    // join index slot of this dimension (1 or 2: the first or second word of
    // a fact row's entry; 0: not indexed), read by the indexed cube scans
    uint32_t ixslot, pad_ix;
    // row mode (per-row strategy, a batch that filters or groups on an
    // attribute the records do not pack): the batch's accept masks by key
    // offset, and a row's `at` for this dimension is its key offset
    const unsigned long long* accr;
};

// A joined dimension in the order the indexed scan's fast path takes them
// (the two index slots first, then the two looked-up dimensions): the
// signature is the sum of code x stride, stride = the product of the radices
// of the dimensions after it in AHEAD_SJ_* order, so any order gives it.
struct SjPos {
    const unsigned long long* fk;
    const void* code;      // looked-up positions: the batch's code table (bytes, or packed with cbits/per/cmagic)
    const uint16_t* rank;  // index positions: record -> the batch's code
    const unsigned long long* acode;  // the batch's accept masks by this dimension's code
    uint64_t ainv, cmagic;
    uint32_t kmin, krange, stride, cbits, per, pad;
};

struct SjQDev {
    uint64_t nrows, gsize;  // fact prefix; dense group domain (1 for an ungrouped query)
    uint64_t glo[3], gstride[3], gA[3], gwm[3];
    uint32_t gdim[3], gshift[3], gpmask[3];
    uint32_t ngroup, gbase;  // gbase: first dense index; indices below nsm live in shared memory
    uint32_t segs;           // cube segments the prefix covers
    uint32_t pad_q;
    // row-mode group attributes: (value - smallest value) by key offset
    const uint32_t* gtab[3];
};

// Counters the kernels fill and the layout of the packed result.
struct SjHdr {
    unsigned long long raw[kMaxQ];      // ungrouped queries: sum of code products
    unsigned long long nonempty[4];     // per dimension: queries accepting >= 1 row
    unsigned long long errcnt, status, exccnt, unseen;
    unsigned long long fkept;  // rows the fact-predicate prefilter kept
    // groups per query (counted by the compact kernel); ~0: the packed area
    // could not take them  (zeroed by the clear kernel up to here)
    unsigned long long ngroups[kMaxQ];
    unsigned long long off[kMaxQ];      // offset of each query's groups in packed
    unsigned long long nerr, packed_len;  // sorted errors at packed[0, nerr); words used
};
constexpr int kHdrClearWords = kMaxQ + 4 + 5 + kMaxQ;

struct SjBatch {
    SjDimDev dim[4];
    const unsigned long long* price;
    const uint16_t* disc;
    uint64_t price_ainv, disc_ainv;
    const SjQDev* q;
    unsigned long long* sums;  // dense group tables
    uint32_t* firsts;
    SjHdr* hdr;
    unsigned long long* errlog;
    unsigned long long* lists;      // per dense slot: present groups, sorted by first row (finalize)
    unsigned long long* lists_tmp;  // radix-sort scratch of the same size
    unsigned long long* packed;
    uint64_t packed_cap;            // words
    uint64_t nmax, gtotal;
    uint32_t nq, nsm;
    // signature cube (strategy kStratCube): per prefix segment and signature
    // (the codes of the row's dimension attributes the batch references), the
    // sum of decoded price x discount over clean rows, and each signature's
    // first clean row; rows with a detected error go to `exc`
    unsigned long long* cube;
    uint32_t* cfirst;
    uint32_t* exc;
    const uint16_t* rank[4];  // record -> dimension code
    const uint16_t* rep[4];   // dimension code -> a record with that code
    // [4][kAccEntries] per dimension code: the batch queries that accept it
    // (those not joining the dimension included); a row whose codes' masks
    // have no query in common adds nothing any query reads
    unsigned long long* acode;
    unsigned long long qmask;  // the batch's queries
    uint64_t seg_end[kMaxSeg];
    // per segment: the queries whose prefix covers it (segments [0, segs))
    unsigned long long segq[kMaxSeg];
    uint32_t radix[4];
    uint32_t nseg, nsig, strategy;
    uint32_t pad2;
    // the cube scan runs in two phases: rows [0, r0) and [r0, nmax); the second
    // reads a signature's first row only if the first phase did not see it
    // (the signatures in `unseen`, a hash set of kUnseenSlots)
    uint64_t r0;
    uint32_t* unseen;
    // join index: per fact row one AN-coded word (kIxA) per index slot, one
    // array per slot; idx_on: the batch's cube scan reads it, slots [1, nslot]
    const unsigned long long* fidx1;
    const unsigned long long* fidx2;
    uint32_t idx_on, nslot;
    // the packed index (ixpack; fidx1 only): one word per row for both slots,
    // payload = id 1 | id 2 << ixp_s1 | (o1 + ixp_r0 * o2) << ixp_ib, AN-coded
    // (a clean word decodes below ixp_lim); o = a slot's key offset, clamped
    // to ixp_kr (its key range); an id is the dense number of the key's
    // record among the dimension's records
    uint64_t ixp_ainv, ixp_lim;
    uint32_t ixpack, ixp_ib, ixp_m0, ixp_s1, ixp_m1, ixp_r0, ixp_kr[2];
    // per index slot: the entry's record (two-word index) or id (packed) -> the batch's code
    const uint16_t* ixrank[2];
    // fast: all four dimensions joined, the shape's index slots present and
    // the looked-up dimensions' code tables bytes (or packed): the indexed
    // scan runs its straight-line body over pos[] (indexed positions first)
    uint32_t fast, pad5;
    SjPos pos[4];
    // the SSB programs' shapes (per-row strategy only): fact predicates on
    // quantity (c = 0) and discount (c = 1) -- fq[c]: the queries with one;
    // facc[c * 256 + v]: the queries whose predicate holds on a clean code of
    // value v -- and the measures (mrev: revenue, mprof: revenue -
    // supplycost; every other query price x discount)
    const uint16_t* qty;
    const unsigned long long* rev;
    const unsigned long long* cost;
    uint64_t qty_ainv, rev_ainv, cost_ainv, rev_umax, cost_umax;
    const unsigned long long* facc;
    const RangePred* fpr;  // [query * 2 + c] the predicates themselves, for corrupt codes
    unsigned long long fq[2], mrev, mprof;
    // the prefilter (per-row strategy): flist_on 1 -- every query has a fact
    // predicate: the rows a query's predicates can keep, or whose fact codes
    // are corrupt; 2 -- no query has one and every query joins dimension
    // flist_dim first: the rows that dimension accepts for a query, or whose
    // foreign key is corrupt.  In flist[0, fkept) when they fit flist_cap.
    uint32_t* flist;
    uint64_t flist_cap;
    uint32_t flist_on, flist_dim;
    // flist_on 2: bit k set when some query of the batch accepts key offset k
    // of dimension flist_dim (null: the prefilter reads the masks themselves)
    uint32_t* pfmap;
};
static_assert(sizeof(SjBatch) % 8 == 0, "SjBatch is copied in 8-byte words");
static_assert(sizeof(SjQDev) % 8 == 0, "SjQDev is copied in 8-byte words");

// (not inlined: a rare path whose copies would crowd the fact kernel's registers)
__device__ __noinline__ void log_err(const SjBatch& b, unsigned long long qs, uint32_t col, uint64_t row) {
    while (qs) {
        const int q = __ffsll(qs) - 1;
        qs &= qs - 1;
        const unsigned long long i = atomicAdd(&b.hdr->errcnt, 1ull);
        if (i < (unsigned long long)kErrLogCap)
            b.errlog[i] = ((unsigned long long)q << 58) | ((unsigned long long)col << kLogColShift) | row;
        else
            atomicOr(&b.hdr->status, (unsigned long long)kDevStatusCapacity);
    }
}

__device__ __forceinline__ uint32_t pick4(uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t d) {
    return d == 0 ? a0 : d == 1 ? a1 : d == 2 ? a2 : a3;
}

// The prefilter of a per-row batch (SjBatch::flist_on), appending to flist --
// in no particular order: the per-row pass adds sums, lowers first rows and
// logs errors, none of which depends on row order -- the rows that pass:
//  1: every query has a fact predicate: the rows that some query's selectAN on
//     quantity / discount keeps, or whose code of such a column is corrupt (the
//     per-row pass reports it, and selects the row when the code itself passes);
//  2: no query has one, and every query joins dimension flist_dim first: the
//     rows whose foreign key that dimension accepts for some query (the accept
//     masks of the batch's accept pass), or whose foreign key is corrupt (the
//     first join reports it).
// Any other row is rejected by every query before anything is reported, so it
// joins nothing and reports nothing.  Its cost is a column or two per row,
// instead of the per-row pass's ~110 instructions for a rejected row.
constexpr int kPfRows = 16;  // rows per thread and tile
constexpr uint64_t kFlistMaxRows = 1ull << 28;  // the row list's capacity (1 GiB); more kept rows: every row is scanned
// the first-join prefilter runs when the rows its dimension accepts are
// expected (uniform attribute values) to be at most this share of the rows
constexpr double kPrefilterMaxShare = 0.25;

// Each thread takes a run of kPfRows consecutive rows of a tile: one 16-byte
// load per 8 two-byte codes or 2 foreign-key codes, all of a run's loads (and
// then all of its record and mask gathers) in flight together.  One row per
// thread and step had kept a few bytes per thread in flight and ran at a
// fifth of the copy bandwidth.
__device__ __forceinline__ void pf_load16(const uint16_t* __restrict__ col, uint64_t r0, uint64_t nmax, bool vec,
                                          uint32_t (&w)[kPfRows / 2]) {
    static_assert(kPfRows % 8 == 0, "runs of whole 16-byte words");
    if (vec && r0 + kPfRows <= nmax) {
        const uint4* p = reinterpret_cast<const uint4*>(col + r0);
#pragma unroll
        for (int k = 0; k < kPfRows / 8; ++k) {
            const uint4 x = __ldg(p + k);
            w[4 * k] = x.x;
            w[4 * k + 1] = x.y;
            w[4 * k + 2] = x.z;
            w[4 * k + 3] = x.w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < kPfRows / 2; ++k) {
            const uint64_t r = r0 + 2 * k;
            const uint32_t lo = r < nmax ? __ldg(col + r) : 0u, hi = r + 1 < nmax ? __ldg(col + r + 1) : 0u;
            w[k] = lo | hi << 16;
        }
    }
}

// The first-join prefilter's accepted keys (flist_on 2): bit k of pfmap set
// when the batch's accept mask of key offset k of dimension flist_dim is not
// empty -- by key offset in row mode, else through the key's record.  One bit
// a key keeps the table in L1 (supplier: 25 KB at 2M rows; customer: 375 KB
// at 3M), where the masks themselves (8 bytes a key or record, behind a 4-byte
// record) made the prefilter one L2 request per row.
__global__ void sj_pfmap_kernel(const SjBatch* __restrict__ bp) {
    if (bp->strategy != kStratRows || bp->flist_on != 2 || !bp->pfmap) return;
    const SjDimDev& D = bp->dim[bp->flist_dim & 3];
    const uint64_t krange = D.krange, words = krange / 32 + 1;
    uint32_t* map = bp->pfmap;
    const int lane = threadIdx.x & 31;
    const uint64_t w0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t wstride = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t w = w0; w < words; w += wstride) {  // (warp-uniform)
        const uint64_t k = w * 32 + lane;
        unsigned long long m = 0;
        if (k < krange) m = D.accr ? __ldg(D.accr + k) : __ldg(D.acc + __ldg(D.rec + k));
        const unsigned bits = __ballot_sync(0xffffffffu, m != 0);
        if (lane == 0) map[w] = bits;
    }
}

// 8 warps a block, at most 80 registers a thread: three blocks an SM
__global__ void __launch_bounds__(kSjThreads, 3) sj_prefilter_kernel(const SjBatch* __restrict__ bp) {
    __shared__ unsigned long long s_acc[512];
    __shared__ uint64_t s_n[kMaxQ];
    // a tile's kept rows are staged here and appended with one global atomic
    // per tile (one per warp and row slot had serialised on the counter)
    __shared__ uint32_t s_rows[kPfRows * kSjThreads];
    __shared__ uint32_t s_cnt;
    __shared__ unsigned long long s_base;
    // fact predicates, every query alive: bit vd of word vq * 8 + vd / 32 set
    // when a row with decoded quantity vq and discount vd passes some query
    __shared__ uint32_t s_T[256 * 256 / 32];
    if (__ldg(&bp->strategy) != kStratRows || !__ldg(&bp->flist_on)) return;  // (block-uniform)
    const uint32_t nq = bp->nq;
    for (int i = threadIdx.x; i < 512; i += blockDim.x) s_acc[i] = __ldg(bp->facc + i);
    if (threadIdx.x < nq) s_n[threadIdx.x] = bp->q[threadIdx.x].nrows;
    __syncthreads();
    const unsigned long long fq0 = bp->fq[0], fq1 = bp->fq[1];
    unsigned long long fall = 0;  // the queries with rows
    for (uint32_t q = 0; q < nq; ++q)
        if (s_n[q]) fall |= 1ull << q;
    const unsigned long long A0 = fall & fq0, A1 = fall & fq1;
    if (bp->flist_on == 1) {  // (block-uniform)
        for (int w = threadIdx.x; w < 256 * 256 / 32; w += blockDim.x) {
            const unsigned long long mq = fall & (s_acc[w >> 3] | ~A0);
            uint32_t bits = 0;
            for (int k = 0; k < 32; ++k)
                if (mq & (s_acc[256 + (w & 7) * 32 + k] | ~A1)) bits |= 1u << k;
            s_T[w] = bits;
        }
        __syncthreads();
    }
    const uint16_t* qty = bp->qty;
    const uint16_t* disc = bp->disc;
    const uint32_t qa = (uint32_t)bp->qty_ainv, da = (uint32_t)bp->disc_ainv;
    const uint64_t nmax = bp->nmax, cap = bp->flist_cap;
    uint32_t* list = bp->flist;
    const bool by_dim = bp->flist_on == 2;
    const SjDimDev& D = bp->dim[bp->flist_dim & 3];
    const unsigned long long* fk = D.fk;
    const uint32_t* rec = D.rec;
    const unsigned long long *dacc = D.acc, *accr = D.accr;
    const uint64_t fk_ainv = D.fk_ainv, kmin = D.kmin, krange = D.krange;
    const uint32_t* pfmap = bp->pfmap;
    unsigned long long* kept = &bp->hdr->fkept;
    const int lane = threadIdx.x & 31;
    // 16-byte loads need 16-byte aligned columns (a run starts at a multiple of
    // kPfRows rows); any other column is read code by code
    const bool vec_fk = (reinterpret_cast<uintptr_t>(fk) & 15) == 0;
    const bool vec_q = (reinterpret_cast<uintptr_t>(qty) & 15) == 0;
    const bool vec_d = (reinterpret_cast<uintptr_t>(disc) & 15) == 0;
    constexpr uint64_t kTile = (uint64_t)kPfRows * kSjThreads;
    const uint64_t ntiles = (nmax + kTile - 1) / kTile;
    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint64_t t0 = tile * kTile;
        if (threadIdx.x == 0) s_cnt = 0;
        __syncthreads();
        unsigned long long full = 0, part = 0;  // queries alive for the whole tile / ending inside it
        for (uint32_t q = 0; q < nq; ++q) {
            if (s_n[q] >= t0 + kTile) full |= 1ull << q;
            else if (s_n[q] > t0) part |= 1ull << q;
        }
        const uint64_t r0 = t0 + (uint64_t)threadIdx.x * kPfRows;  // this thread's run
        // the queries a row of the run is alive for (recomputed where used: a
        // run's sixteen masks would hold 32 registers)
        auto alive = [&](int j) -> unsigned long long {
            const uint64_t row = r0 + j;
            if (row >= nmax) return 0ull;
            unsigned long long m = full;
            for (unsigned long long p = part; p; p &= p - 1) {
                const int q = __ffsll(p) - 1;
                if (row < s_n[q]) m |= 1ull << q;
            }
            return m;
        };
        uint32_t km = 0;  // bit j: row r0 + j is kept
        if (by_dim) {
            // the first join, as the per-row pass takes it: the truncated key
            // probes even when corrupt, and a corrupt key is reported; the run
            // in two halves of 8 keys (64 bytes of loads in flight a thread)
            constexpr int kH = kPfRows / 2;
#pragma unroll 1
            for (int h = 0; h < 2; ++h) {
                const uint64_t rh = r0 + (uint64_t)h * kH;
                unsigned long long c[kH];
                if (vec_fk && rh + kH <= nmax) {
                    const ulonglong2* p = reinterpret_cast<const ulonglong2*>(fk + rh);
#pragma unroll
                    for (int k = 0; k < kH / 2; ++k) {
                        const ulonglong2 x = __ldg(p + k);
                        c[2 * k] = x.x;
                        c[2 * k + 1] = x.y;
                    }
                } else {
#pragma unroll
                    for (int j = 0; j < kH; ++j) c[j] = rh + j < nmax ? __ldg(fk + rh + j) : 0ull;
                }
                uint32_t rv[kH];
                uint32_t bad = 0;  // bit j: row rh + j's key is corrupt
                if (pfmap) {
                    // a key some query accepts: the row is kept for every query
                    // alive on it (one not accepting it drops it again in the
                    // per-row pass, which reports nothing before its first join)
                    uint32_t sh[kH / 4] = {};  // each key's bit in its word, a byte a row
#pragma unroll
                    for (int j = 0; j < kH; ++j) {
                        const uint64_t dec = c[j] * fk_ainv;
                        const uint64_t idx = (dec & 0xffffffffull) - kmin;
                        if (dec > 0xffffffffull) bad |= 1u << j;
                        rv[j] = rh + j < nmax && idx < krange ? __ldg(pfmap + (idx >> 5)) : 0u;
                        sh[j >> 2] |= (uint32_t)(idx & 31) << ((j & 3) * 8);
                    }
#pragma unroll
                    for (int j = 0; j < kH; ++j)
                        if (((rv[j] >> ((sh[j >> 2] >> ((j & 3) * 8)) & 31u)) & 1u) || ((bad >> j) & 1u))
                            if (alive(h * kH + j)) km |= 1u << (h * kH + j);
                } else {
#pragma unroll
                    for (int j = 0; j < kH; ++j) {
                        const uint64_t dec = c[j] * fk_ainv;
                        const uint64_t idx = (dec & 0xffffffffull) - kmin;
                        if (dec > 0xffffffffull) bad |= 1u << j;
                        rv[j] = rh + j < nmax && idx < krange ? (accr ? (uint32_t)idx + 1u : __ldg(rec + idx)) : 0u;
                    }
#pragma unroll
                    for (int j = 0; j < kH; ++j) {
                        const unsigned long long a = alive(h * kH + j);
                        if (!a) continue;
                        const unsigned long long acc =
                            accr ? (rv[j] ? __ldg(accr + rv[j] - 1u) : 0ull) : __ldg(dacc + rv[j]);
                        if ((a & acc) != 0 || ((bad >> j) & 1u)) km |= 1u << (h * kH + j);
                    }
                }
            }
        } else {
            // (a column no alive query selects on is not read)
            const unsigned long long live = r0 < nmax ? full | part : 0ull;
            uint32_t qw[kPfRows / 2], dw[kPfRows / 2];
            if (live & fq0) pf_load16(qty, r0, nmax, vec_q, qw);
            if (live & fq1) pf_load16(disc, r0, nmax, vec_d, dw);
            if (part == 0 && full == fall && r0 + kPfRows <= nmax) {
                // every query alive on the whole run: one table bit a row (a
                // corrupt code, above 255 decoded, is kept and never looked up)
#pragma unroll
                for (int j = 0; j < kPfRows; ++j) {
                    const uint32_t vq = A0 ? (((qw[j >> 1] >> ((j & 1) * 16)) & 0xffffu) * qa) & 0xffffu : 0u;
                    const uint32_t vd = A1 ? (((dw[j >> 1] >> ((j & 1) * 16)) & 0xffffu) * da) & 0xffffu : 0u;
                    if ((vq | vd) > 0xffu || ((s_T[(vq << 3) | (vd >> 5)] >> (vd & 31)) & 1u)) km |= 1u << j;
                }
            } else
#pragma unroll
            for (int j = 0; j < kPfRows; ++j) {
                const unsigned long long a = alive(j);
                if (!a) continue;
                unsigned long long m = a;
                bool bad = false;
                if (a & fq0) {
                    const uint32_t v = (((qw[j >> 1] >> ((j & 1) * 16)) & 0xffffu) * qa) & 0xffffu;
                    if (v > 0xffu) bad = true;
                    else m &= s_acc[v] | ~(a & fq0);
                }
                if (a & fq1) {
                    const uint32_t v = (((dw[j >> 1] >> ((j & 1) * 16)) & 0xffffu) * da) & 0xffffu;
                    if (v > 0xffu) bad = true;
                    else m &= s_acc[256 + v] | ~(a & fq1);
                }
                if (bad || m != 0) km |= 1u << j;
            }
        }
        // the warp's kept rows, one shared atomic per warp: exclusive offsets
        // by an inclusive scan of the threads' counts
        const uint32_t cnt = (uint32_t)__popc(km);
        uint32_t incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        uint32_t wbase = 0;
        if (lane == 31 && incl) wbase = atomicAdd(&s_cnt, incl);
        wbase = __shfl_sync(0xffffffffu, wbase, 31);
        uint32_t pos = wbase + incl - cnt;
        for (uint32_t m = km; m; m &= m - 1) s_rows[pos++] = (uint32_t)(r0 + (uint64_t)(__ffs(m) - 1));
        __syncthreads();
        const uint32_t nt = s_cnt;
        if (threadIdx.x == 0 && nt) s_base = atomicAdd(kept, (unsigned long long)nt);
        __syncthreads();
        for (uint32_t j = threadIdx.x; j < nt; j += blockDim.x)
            if (s_base + j < cap) list[s_base + j] = s_rows[j];
        __syncthreads();  // (s_rows and s_cnt are reused by the next tile)
    }
}

template <int kSjRows, int kSjBlocksPerSm>
__global__ void __launch_bounds__(kSjThreads, kSjBlocksPerSm) sj_fact_kernel(const SjBatch* __restrict__ bp) {
    constexpr int kSjTile = kSjRows * kSjThreads;
    extern __shared__ unsigned long long s_dyn[];  // [kSmemGroups] sums, then [kSmemGroups] first rows
    __shared__ SjBatch b;
    __shared__ SjQDev s_q[kMaxQ];
    __shared__ uint64_t s_n[kMaxQ];
    if (__ldg(&bp->strategy) != kStratRows) return;  // (block-uniform) a cube batch: nothing to do here
    for (int i = threadIdx.x; i < (int)(sizeof(SjBatch) / 8); i += blockDim.x)
        reinterpret_cast<unsigned long long*>(&b)[i] = reinterpret_cast<const unsigned long long*>(bp)[i];
    __syncthreads();
    for (int i = threadIdx.x; i < (int)(b.nq * sizeof(SjQDev) / 8); i += blockDim.x)
        reinterpret_cast<unsigned long long*>(s_q)[i] = reinterpret_cast<const unsigned long long*>(b.q)[i];
    unsigned long long* s_sum = s_dyn;
    uint32_t* s_first = reinterpret_cast<uint32_t*>(s_dyn + kSmemGroups);
    for (uint32_t i = threadIdx.x; i < b.nsm; i += blockDim.x) {
        s_sum[i] = 0;
        s_first[i] = kNoRow;
    }
    __syncthreads();
    if (threadIdx.x < b.nq) s_n[threadIdx.x] = s_q[threadIdx.x].nrows;
    __syncthreads();
    const uint32_t nsm = b.nsm;
    // over the prefilter's row list when it ran and its rows fit the list,
    // else over the rows themselves (block-uniform)
    const unsigned long long nkept = b.flist_on ? b.hdr->fkept : 0ull;
    const bool listed = b.flist_on && nkept <= b.flist_cap;
    const uint64_t nitems = listed ? nkept : b.nmax;
    const uint32_t ntiles = (uint32_t)((nitems + kSjTile - 1) / kSjTile);
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint64_t t0 = (uint64_t)tile * kSjTile;
        // queries alive for the whole tile, and those whose prefix ends inside it
        // (listed rows: every query is tested row by row)
        unsigned long long full = 0, part = 0;
        for (uint32_t q = 0; q < b.nq; ++q) {
            if (listed) {
                if (s_n[q]) part |= 1ull << q;
            } else if (s_n[q] >= t0 + kSjTile) {
                full |= 1ull << q;
            } else if (s_n[q] > t0) {
                part |= 1ull << q;
            }
        }
        // this thread's rows (a listed slot past the list's end: row nmax, never alive)
        uint64_t rowv[kSjRows];
#pragma unroll
        for (int i = 0; i < kSjRows; ++i) {
            const uint64_t idx = t0 + (uint64_t)i * kSjThreads + threadIdx.x;
            rowv[i] = !listed ? idx : idx < nitems ? (uint64_t)__ldg(b.flist + idx) : b.nmax;
        }
        unsigned long long alive[kSjRows];
        uint32_t at[kSjRows][4];
#pragma unroll
        for (int i = 0; i < kSjRows; ++i) {
            const uint64_t row = rowv[i];
            unsigned long long a = full;
            unsigned long long p = part;
            while (p) {
                const int q = __ffsll(p) - 1;
                p &= p - 1;
                if (row < s_n[q]) a |= 1ull << q;
            }
            alive[i] = row < b.nmax ? a : 0ull;
#pragma unroll
            for (int d = 0; d < 4; ++d) at[i][d] = 0;
        }
        // fact predicates: selectAN over each such query's whole prefix, quantity
        // and discount independently (a corrupt code is reported by each
        // selection that reads it and never selected), before any join
        if (b.fq[0] | b.fq[1]) {
#pragma unroll
            for (int i = 0; i < kSjRows; ++i) {
                const uint64_t row = rowv[i];
                const unsigned long long a0 = alive[i];
                unsigned long long keep = a0;
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    const unsigned long long fq = a0 & b.fq[c];
                    if (!fq) continue;
                    const uint32_t code = __ldg((c ? b.disc : b.qty) + row);
                    const uint32_t v = (code * (uint32_t)(c ? b.disc_ainv : b.qty_ainv)) & 0xffffu;
                    if (v > 0xffu) {  // reported, and selected when the code itself passes (selectAN_scalar.tcc:84-92)
                        log_err(b, fq, c ? AHEAD_SJ_COL_DISCOUNT : AHEAD_SJ_COL_QUANTITY, row);
                        unsigned long long sel = 0, m = fq;
                        while (m) {
                            const int q = __ffsll(m) - 1;
                            m &= m - 1;
                            if (b.fpr[q * 2 + c](code)) sel |= 1ull << q;
                        }
                        keep &= sel | ~fq;
                    } else {
                        keep &= __ldg(b.facc + c * 256 + v) | ~fq;
                    }
                }
                alive[i] = keep;
            }
        }
        // dimensions, in the pipeline's join order
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int d = join_dim(k);
            const SjDimDev& D = b.dim[d];
            if (!D.joins) continue;
            unsigned long long code[kSjRows];
#pragma unroll
            for (int i = 0; i < kSjRows; ++i)
                code[i] = (alive[i] & D.joins) ? __ldg(D.fk + rowv[i]) : 0ull;
            uint32_t rv[kSjRows];
#pragma unroll
            for (int i = 0; i < kSjRows; ++i) {
                rv[i] = 0;
                if (alive[i] & D.joins) {
                    const uint64_t key = (code[i] * D.fk_ainv) & 0xffffffffull;  // truncated to the key type
                    const uint64_t idx = key - D.kmin;
                    // row mode: the key offset + 1 (its row's accept mask is 0 when no row has the key)
                    if (idx < D.krange) rv[i] = D.accr ? (uint32_t)idx + 1u : __ldg(D.rec + idx);
                }
            }
#pragma unroll
            for (int i = 0; i < kSjRows; ++i) {
                const unsigned long long jq = alive[i] & D.joins;
                if (!jq) continue;
                const unsigned long long acc =
                    D.accr ? (rv[i] ? __ldg(D.accr + rv[i] - 1u) : 0ull) : __ldg(D.acc + rv[i]);
                at[i][d] = rv[i] - 1u;
                if ((code[i] * D.fk_ainv) > 0xffffffffull) {
                    log_err(b, jq, d, rowv[i]);
                    alive[i] &= ~(jq & ~D.first);  // positional fetch drops the row
                }
                alive[i] &= acc | ~D.joins;
            }
        }
        // measures for surviving rows, each fetched positionally after the
        // previous one: price then discount, or revenue then supplycost
        const unsigned long long mother = b.mrev | b.mprof;
#pragma unroll
        for (int i = 0; i < kSjRows; ++i) {
            if (!alive[i]) continue;
            const uint64_t row = rowv[i];
            unsigned long long am = alive[i] & ~mother, ar = alive[i] & mother;
            unsigned long long vm = 0, vr = 0, vp = 0;
            if (am) {
                const uint64_t pdec = __ldg(b.price + row) * b.price_ainv;
                const uint32_t ddec = ((uint32_t)__ldg(b.disc + row) * (uint32_t)b.disc_ainv) & 0xffffu;
                if (pdec > 0xffffffffull) {
                    log_err(b, am, AHEAD_SJ_COL_PRICE, row);
                    am = 0;
                } else if (ddec > 0xffu) {
                    log_err(b, am, AHEAD_SJ_COL_DISCOUNT, row);
                    am = 0;
                }
                vm = pdec * ddec;  // scaled by the result's A at the end
            }
            if (ar) {
                const uint64_t rdec = __ldg(b.rev + row) * b.rev_ainv;
                if (rdec > b.rev_umax) {
                    log_err(b, ar, AHEAD_SJ_COL_REVENUE, row);
                    ar = 0;
                } else if (ar & b.mprof) {
                    const unsigned long long ap = ar & b.mprof;
                    const uint64_t cdec = __ldg(b.cost + row) * b.cost_ainv;
                    if (cdec > b.cost_umax) {
                        log_err(b, ap, AHEAD_SJ_COL_SUPPLYCOST, row);
                        ar &= ~ap;
                    }
                    vp = rdec - cdec;  // arithmeticAN<sub>, mod 2^64
                }
                vr = rdec;
            }
            unsigned long long qs = am | ar;
            while (qs) {
                const int q = __ffsll(qs) - 1;
                qs &= qs - 1;
                const unsigned long long v = ((b.mprof >> q) & 1ull) ? vp : ((b.mrev >> q) & 1ull) ? vr : vm;
                const SjQDev& Q = s_q[q];
                uint64_t g = 0;
                for (uint32_t j = 0; j < Q.ngroup; ++j) {
                    const uint32_t a = pick4(at[i][0], at[i][1], at[i][2], at[i][3], Q.gdim[j]);
                    const uint32_t gv = Q.gtab[j] ? __ldg(Q.gtab[j] + a) : ((a >> Q.gshift[j]) & Q.gpmask[j]);
                    g += (uint64_t)gv * Q.gstride[j];
                }
                const uint64_t slot = Q.gbase + g;
                if (slot < nsm) {
                    atomicAdd(&s_sum[slot], v);
                    if (s_first[slot] > (uint32_t)row) atomicMin(&s_first[slot], (uint32_t)row);
                } else {
                    atomicAdd(&b.sums[slot], v);
                    if (b.firsts[slot] > (uint32_t)row) atomicMin(&b.firsts[slot], (uint32_t)row);
                }
            }
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < nsm; i += blockDim.x) {
        if (s_first[i] != kNoRow) {
            atomicAdd(&b.sums[i], s_sum[i]);
            atomicMin(&b.firsts[i], s_first[i]);
        }
    }
}

using SjFactFn = void (*)(const SjBatch*);
const SjFactFn kSjFact[kSjVariants] = {sj_fact_kernel<2, 4>, sj_fact_kernel<4, 3>, sj_fact_kernel<8, 2>};

// Zero the group tables and the header counters of a batch.
__global__ void sj_clear_kernel(const SjBatch* __restrict__ bp) {
    const uint64_t n = bp->gtotal;
    unsigned long long* sums = bp->sums;
    uint32_t* firsts = bp->firsts;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        sums[i] = 0;
        firsts[i] = kNoRow;
    }
    if (bp->strategy == kStratCube) {
        const uint64_t nc = (uint64_t)bp->nseg * bp->nsig;
        for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nc; i += (uint64_t)gridDim.x * blockDim.x)
            bp->cube[i] = 0;
        for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < bp->nsig;
             i += (uint64_t)gridDim.x * blockDim.x)
            bp->cfirst[i] = kNoRow;
        if (blockIdx.x == 1)
            for (uint32_t i = threadIdx.x; i < kUnseenSlots; i += blockDim.x) bp->unseen[i] = kUnseenEmpty;
    }
    if (blockIdx.x == 0)
        for (int i = threadIdx.x; i < kHdrClearWords; i += blockDim.x)
            reinterpret_cast<unsigned long long*>(bp->hdr)[i] = 0;
}

// ---------------------------------------------------------------- cube
// Pass 1: one scan of the fact prefix for the whole batch.  A clean row adds
// its decoded price x discount to cube[segment][signature] and lowers the
// signature's first row; a row with a corrupt foreign key (of a dimension
// the batch joins) or measure goes to the exact per-row path.
//
// The batch descriptor is a __grid_constant__ parameter: its fields are
// constant-bank operands, not shared-memory loads competing with the row
// gathers for the load/store pipe.  The kernel holds nothing in shared
// memory, so the whole L1 caches code-table lines: the per-row code lookups
// are the scan's bound, and every shared-memory carve-out that shrinks L1
// (staging the small tables there included) made the scan slower.  Besides
// its streamed bytes the scan makes random requests per row (a dimension code
// per joined dimension, the cube add, the first-row check).  It can run in two
// phases to drop the last of
// them: once rows [0, r0) are done (r0 ~ kR0PerSig rows per signature) nearly
// every signature that occurs has been seen, and a row of [r0, nmax) whose
// signature was seen cannot lower its first row: the second phase reads
// cfirst only for the signatures of the (small) set of those not seen, or for
// every row when that set overflows kUnseenCap.  A signature with a missing
// key (code 0) is always checked.  Two more options per shape: packed code
// tables (cbits-bit codes, `per` to a 64-bit word: smaller tables, more L1
// hits, a multiply-shift per lookup) and the acceptance skip (a row whose
// codes no batch query accepts makes no cube add and no first-row check).
// The tuner picks the shape and whether to split.
__device__ __forceinline__ uint32_t unseen_slot(uint32_t s) { return (s * 2654435761u) >> (32 - kUnseenLog); }

__device__ __forceinline__ bool unseen_has(const uint32_t* __restrict__ t, uint32_t s) {
    uint32_t h = unseen_slot(s);
    for (uint32_t n = 0; n < kUnseenSlots; ++n) {
        const uint32_t v = __ldg(t + h);
        if (v == s) return true;
        if (v == kUnseenEmpty) return false;
        h = (h + 1) & (kUnseenSlots - 1);
    }
    return false;
}

// The batch's dimension code of every key (cube strategy): code[k] =
// rank[rec[k]]; one pass over each dimension the batch joins.
__global__ void sj_code_kernel(const SjBatch* __restrict__ bp) {
    const int d = blockIdx.y;
    if (bp->strategy != kStratCube || !bp->dim[d].joins) return;
    const SjDimDev& D = bp->dim[d];
    const uint16_t* rank = bp->rank[d];
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    if (blockIdx.x == 0)
        for (uint32_t c = threadIdx.x; c < bp->radix[d]; c += blockDim.x)
            bp->acode[(size_t)d * kAccEntries + c] = __ldg(D.acc + bp->rep[d][c]) | ~D.joins;
    if (bp->idx_on && D.ixslot && D.ixslot <= bp->nslot) return;  // the scan reads this dimension's records from the index
    // every table also holds entry krange = code 0 (the fast path clamps keys to it)
    if (D.cbits) {
        const uint64_t words = D.krange / D.per + 1;
        for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < words; w += stride) {
            unsigned long long v = 0;
            for (uint32_t j = 0; j < D.per; ++j) {
                const uint64_t k = w * D.per + j;
                if (k >= D.krange) break;
                v |= (unsigned long long)__ldg(rank + __ldg(D.rec + k)) << (j * D.cbits);
            }
            static_cast<unsigned long long*>(D.code)[w] = v;
        }
        return;
    }
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k <= D.krange; k += stride) {
        const uint16_t c = k < D.krange ? __ldg(rank + __ldg(D.rec + k)) : (uint16_t)0;
        if (D.cw == 1) static_cast<uint8_t*>(D.code)[k] = (uint8_t)c;
        else static_cast<uint16_t*>(D.code)[k] = c;
    }
}

// One phase of the cube scan (phase 0: rows [0, r0); phase 1: rows [r0, nmax)).
template <int ROWS, int BPS, bool PACK, bool ACC>
__global__ void __launch_bounds__(kSjThreads, BPS) sj_cube_kernel(const __grid_constant__ SjBatch b, int phase) {
    constexpr int THREADS = kSjThreads;
    constexpr int kTile = ROWS * THREADS;
    if (b.strategy != kStratCube) return;
    const uint64_t lo = phase ? b.r0 : 0, hi = phase ? b.nmax : b.r0;
    if (lo >= hi) return;
    // 0: every row checks its signature's first row; 1: only signatures of
    // the unseen set; 2: none (the set is empty)
    int filter = 0;
    if (phase) {
        const unsigned long long nun = __ldg(&b.hdr->unseen);
        if (nun <= kUnseenCap) filter = nun ? 1 : 2;
    }
    const uint32_t ntiles = (uint32_t)((hi - lo + kTile - 1) / kTile);
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint64_t t0 = lo + (uint64_t)tile * kTile;
        uint32_t seg0 = 0;
        while (seg0 + 1 < b.nseg && t0 >= b.seg_end[seg0]) ++seg0;
        const bool one_seg = seg0 + 1 >= b.nseg || t0 + kTile <= b.seg_end[seg0];
        // every streaming load of the tile's rows first, all in flight together
        unsigned long long code[4][ROWS];
        unsigned long long pc[ROWS];
        uint32_t dc[ROWS];
#pragma unroll
        for (int i = 0; i < ROWS; ++i) {
            const uint64_t row = t0 + (uint64_t)i * THREADS + threadIdx.x;
            const bool in = row < hi;
#pragma unroll
#pragma unroll
            for (int d = 0; d < 4; ++d) code[d][i] = (in && b.dim[d].joins) ? __ldg(b.dim[d].fk + row) : 0ull;
            pc[i] = in ? __ldg(b.price + row) : 0ull;
            dc[i] = in ? (uint32_t)__ldg(b.disc + row) : 0u;
        }
        // dimension codes (independent lookups), then the signature
        uint32_t cv[4][ROWS];
        bool exc[ROWS];
#pragma unroll
        for (int i = 0; i < ROWS; ++i) exc[i] = false;
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            const SjDimDev& D = b.dim[d];
#pragma unroll
            for (int i = 0; i < ROWS; ++i) {
                cv[d][i] = 0;
                if (D.joins) {
                    const uint64_t dec = code[d][i] * D.fk_ainv;
                    exc[i] |= dec > 0xffffffffull;
                    const uint64_t idx = (dec & 0xffffffffull) - D.kmin;
                    if (idx < D.krange) {
                        if (PACK) {
                            const uint32_t q = (uint32_t)((idx * D.cmagic) >> 40);
                            const uint32_t r = (uint32_t)idx - q * D.per;
                            const unsigned long long w = __ldg(static_cast<const unsigned long long*>(D.code) + q);
                            cv[d][i] = (uint32_t)(w >> (r * D.cbits)) & ((1u << D.cbits) - 1u);
                        } else {
                            cv[d][i] = D.cw == 1 ? __ldg(static_cast<const uint8_t*>(D.code) + idx)
                                                 : __ldg(static_cast<const uint16_t*>(D.code) + idx);
                        }
                    }
                }
            }
        }
#pragma unroll
        for (int i = 0; i < ROWS; ++i) {
            const uint64_t row = t0 + (uint64_t)i * THREADS + threadIdx.x;
            if (row >= hi) continue;
            uint32_t sig = 0;
            bool nz = true;
            unsigned long long m = b.qmask;
#pragma unroll
            for (int d = 0; d < 4; ++d)
                if (b.dim[d].joins) {
                    sig = sig * b.radix[d] + cv[d][i];
                    nz &= cv[d][i] != 0;
                    if (ACC) m &= __ldg(b.acode + (size_t)d * kAccEntries + cv[d][i]);
                }
            const uint64_t pdec = pc[i] * b.price_ainv;
            const uint32_t ddec = (dc[i] * (uint32_t)b.disc_ainv) & 0xffffu;
            if (exc[i] || pdec > 0xffffffffull || ddec > 0xffu) {
                const unsigned long long k = atomicAdd(&b.hdr->exccnt, 1ull);
                if (k < kExcCap) b.exc[k] = (uint32_t)row;
                else atomicOr(&b.hdr->status, (unsigned long long)kDevStatusCapacity);
                continue;
            }
            if (ACC && !m) continue;  // no query accepts the row
            uint32_t seg = seg0;
            if (!one_seg)
                while (seg + 1 < b.nseg && row >= b.seg_end[seg]) ++seg;
            atomicAdd(&b.cube[(uint64_t)seg * b.nsig + sig], (unsigned long long)(pdec * ddec));
            bool chk = filter == 0 || !nz;
            if (!chk && filter == 1) chk = unseen_has(b.unseen, sig);
            if (chk && b.cfirst[sig] > (uint32_t)row) atomicMin(&b.cfirst[sig], (uint32_t)row);
        }
    }
}


// Between the phases: the signatures without a missing key that phase 0 did
// not see go into the unseen set (their count into hdr->unseen; only the
// first kUnseenCap are inserted, and a larger count turns the filter off).
__global__ void sj_unseen_kernel(const SjBatch* __restrict__ bp) {
    if (bp->strategy != kStratCube || bp->r0 >= bp->nmax) return;
    const uint32_t nsig = bp->nsig;
    uint32_t radix[4];
    bool joins[4];
    for (int d = 0; d < 4; ++d) {
        radix[d] = bp->radix[d];
        joins[d] = bp->dim[d].joins != 0;
    }
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < nsig; s += gridDim.x * blockDim.x) {
        if (bp->cfirst[s] != kNoRow) continue;
        uint32_t rem = s;
        bool nz = true;
        unsigned long long m = bp->qmask;
        for (int d = 3; d >= 0; --d) {
            const uint32_t c = rem % radix[d];
            rem /= radix[d];
            if (!joins[d]) continue;
            if (c == 0) nz = false;
            m &= bp->acode[(size_t)d * kAccEntries + c];
        }
        if (!nz || !m) continue;  // always checked, or read by no query
        const unsigned long long k = atomicAdd(&bp->hdr->unseen, 1ull);
        if (k >= kUnseenCap) continue;
        uint32_t h = unseen_slot(s);
        for (uint32_t n = 0; n < kUnseenSlots; ++n) {
            if (atomicCAS(&bp->unseen[h], kUnseenEmpty, s) == kUnseenEmpty) break;
            h = (h + 1) & (kUnseenSlots - 1);
        }
    }
}

// The join index: per fact row, for the two dimensions with the largest key
// ranges, the decoded foreign key's offset (key - kmin) and that key's record,
// built once per engine.  An indexed cube scan takes those two dimensions'
// records from the index instead of random code-table lookups, and uses a
// row's entry only while the row's foreign key, decoded and checked as
// always, still has the offset the entry holds; any other row (its foreign
// key changed since the index was built, or the index word is corrupt) is
// sent to the exact per-row path, so results never depend on the index
// being current.  Entry of index slot s (one 64-bit word each): payload =
// offset | record << 32, the offset the 32-bit difference (decoded key -
// kmin) and the record below 2^13, AN-coded with kIxA -- a corrupt word
// decodes above 2^48 - 1, the same check as the fact columns'.
//
// The packed form holds both slots in ONE word per row (8 bytes instead of
// 16): each key's dense record id (id 0: no dimension row has the key) in
// fields just as wide as the record counts need, and both key offsets as one
// mixed-radix number o1 + (range 1 + 1) * o2, an offset outside its key range
// stored as the range itself.  It is built when those fields and an AN code
// that detects every one- and two-bit flip of the word fit 64 bits (SSB at
// SF100: 6 + 8 id bits and 42 key bits, A = 253).
constexpr uint64_t kIxA = kResoidAMax;
constexpr uint64_t kIxAinv = kResoidAInvMax;
constexpr int kIxSlots = 2;
constexpr int kIxPacked = 3;  // a cube shape's slot count when it reads the packed index

// One row's index entry: the two slots' records (ids), whether the word is
// corrupt, and what the row's current key offsets are checked against (the
// two-word index: each slot's offset; packed: the joint key field).
struct IxEntry {
    uint32_t k0, k1, r0, r1, bad;
    uint64_t kj;
};

// Decodes the entry of a row from its index word(s): w0 (slot 1, or the
// packed word) and w1 (slot 2 of the two-word index).
template <bool PACKED>
__device__ __forceinline__ IxEntry ix_entry(const SjBatch& b, uint64_t w0, uint64_t w1) {
    IxEntry x;
    if (PACKED) {
        const uint64_t p = w0 * b.ixp_ainv;
        x.bad = p >= b.ixp_lim;
        x.r0 = (uint32_t)p & b.ixp_m0;
        x.r1 = ((uint32_t)p >> b.ixp_s1) & b.ixp_m1;
        x.kj = p >> b.ixp_ib;
        x.k0 = x.k1 = 0;
    } else {
        const uint64_t q0 = w0 * kIxAinv, q1 = w1 * kIxAinv;
        x.bad = (uint32_t)((q0 | q1) >> 48);
        x.k0 = (uint32_t)q0;
        x.k1 = (uint32_t)q1;
        x.r0 = (uint32_t)(q0 >> 32) & 0x1fffu;
        x.r1 = (uint32_t)(q1 >> 32) & 0x1fffu;
        x.kj = 0;
    }
    return x;
}

// Nonzero when the entry was not built from the row's current key offsets
// o0 (slot 1) and o1 (slot 2; read only with NSLOT > 1): the row then takes
// the exact path.  A packed entry stores an offset outside the key range as
// the range itself, so any two such offsets match (both mean "no row").
template <bool PACKED, int NSLOT>
__device__ __forceinline__ uint32_t ix_key_differs(const SjBatch& b, const IxEntry& x, uint32_t o0, uint32_t o1) {
    if (PACKED)
        return (uint64_t)min(o0, b.ixp_kr[0]) + (uint64_t)b.ixp_r0 * min(o1, b.ixp_kr[1]) != x.kj;
    return (o0 ^ x.k0) | (NSLOT > 1 ? (o1 ^ x.k1) : 0u);
}

// Streaming loads that leave L1 to the code tables.
template <bool NA>
__device__ __forceinline__ unsigned long long ld_stream(const unsigned long long* p) {
    if (!NA) return __ldg(p);
    unsigned long long v;
    asm("ld.global.nc.L1::no_allocate.u64 %0, [%1];" : "=l"(v) : "l"(p));
    return v;
}
template <bool NA>
__device__ __forceinline__ uint32_t ld_stream(const uint16_t* p) {
    if (!NA) return __ldg(p);
    unsigned short v;
    asm("ld.global.nc.L1::no_allocate.u16 %0, [%1];" : "=h"(v) : "l"(p));
    return v;
}
template <bool NA>
__device__ __forceinline__ uint32_t ld_stream(const uint32_t* p) {
    if (!NA) return __ldg(p);
    uint32_t v;
    asm("ld.global.nc.L1::no_allocate.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}
template <bool NA>
__device__ __forceinline__ ulonglong2 ld_stream(const ulonglong2* p) {
    if (!NA) return __ldg(p);
    ulonglong2 v;
    asm("ld.global.nc.L1::no_allocate.v2.u64 {%0, %1}, [%2];" : "=l"(v.x), "=l"(v.y) : "l"(p));
    return v;
}

// A looked-up dimension's code in the fast path: the code table read at k
// when k is inside the key range, else code 0 (the load then reads entry 0,
// so no branch).
template <bool PACK>
__device__ __forceinline__ uint32_t pos_code(const SjPos& P, uint32_t k) {
    const bool in = k < P.krange;
    const uint32_t kk = in ? k : 0u;
    uint32_t c;
    if (PACK) {
        const uint32_t q = (uint32_t)(((uint64_t)kk * P.cmagic) >> 40);
        const uint32_t r = kk - q * P.per;
        const unsigned long long w = __ldg(static_cast<const unsigned long long*>(P.code) + q);
        c = (uint32_t)(w >> (r * P.cbits)) & ((1u << P.cbits) - 1u);
    } else {
        c = __ldg(static_cast<const uint8_t*>(P.code) + kk);
    }
    return in ? c : 0u;
}

// The same with the key clamped to the range instead of tested: the entry
// at krange is code 0 (the tables keep it zero), so an out-of-range key reads
// code 0 as above, in one instruction instead of three.
template <bool PACK>
__device__ __forceinline__ uint32_t pos_code_clamped(const SjPos& P, uint32_t k) {
    const uint32_t kk = min(k, P.krange);
    if (PACK) {
        const uint32_t q = (uint32_t)(((uint64_t)kk * P.cmagic) >> 40);
        const uint32_t r = kk - q * P.per;
        const unsigned long long w = __ldg(static_cast<const unsigned long long*>(P.code) + q);
        return (uint32_t)(w >> (r * P.cbits)) & ((1u << P.cbits) - 1u);
    }
    return __ldg(static_cast<const uint8_t*>(P.code) + kk);
}

// The streamed columns of a thread's two adjacent rows (fast path).
struct PairCols {
    ulonglong2 f[4], pc, w0, w1;  // w0: index slot 1 of the two rows, w1: slot 2
    uint32_t dc;
};

// w0: index slot 1 (or the packed words) of rows r0, r0 + 1; w1: slot 2
// (NSLOT 2 only).
template <bool NA, int NSLOT>
__device__ __forceinline__ void load_pair(const SjBatch& b, uint32_t r0, uint32_t hi, PairCols& c) {
    if (r0 + 1 < hi) {
#pragma unroll
        for (int p = 0; p < 4; ++p) c.f[p] = ld_stream<NA>(reinterpret_cast<const ulonglong2*>(b.pos[p].fk + r0));
        c.pc = ld_stream<NA>(reinterpret_cast<const ulonglong2*>(b.price + r0));
        c.dc = ld_stream<NA>(reinterpret_cast<const uint32_t*>(b.disc + r0));
        c.w0 = ld_stream<NA>(reinterpret_cast<const ulonglong2*>(b.fidx1 + r0));
        c.w1 = NSLOT == 2 ? ld_stream<NA>(reinterpret_cast<const ulonglong2*>(b.fidx2 + r0))
                          : make_ulonglong2(0ull, 0ull);
    } else {  // the last row of an odd range (or none)
        const bool in = r0 < hi;
#pragma unroll
        for (int p = 0; p < 4; ++p) c.f[p] = make_ulonglong2(in ? __ldg(b.pos[p].fk + r0) : 0ull, 0ull);
        c.pc = make_ulonglong2(in ? __ldg(b.price + r0) : 0ull, 0ull);
        c.dc = in ? (uint32_t)__ldg(b.disc + r0) : 0u;
        c.w0 = make_ulonglong2(in ? __ldg(b.fidx1 + r0) : 0ull, 0ull);
        c.w1 = make_ulonglong2((NSLOT == 2 && in) ? __ldg(b.fidx2 + r0) : 0ull, 0ull);
    }
}

// The indexed scan's straight-line body for batches joining all four
// dimensions with both index slots present (SjBatch::fast): the dimensions
// in pos[] order, a row's badness one OR of the decoded words' high halves,
// the index offsets' differences and the discount's high byte.  With PF the
// next tile's columns are loaded before this tile's rows are processed, so a
// thread always has a pair of rows in flight.
template <bool PACK, bool NA, bool PF, int NSLOT, bool ACC>
__device__ __forceinline__ void cube_ix_fast(const SjBatch& b, uint64_t lo64, uint64_t hi64, int filter) {
    constexpr int kTile = 2 * kSjThreads;
    // row arithmetic in 32 bits: the engine keeps fact_rows <= kMaxFactRows
    const uint32_t lo = (uint32_t)lo64, hi = (uint32_t)hi64;
    const int lane = threadIdx.x & 31;
    const uint32_t base = lo & ~1u;
    const uint32_t ntiles = (hi - base + kTile - 1) / kTile;
    PairCols cur, nxt;
    uint32_t tile = blockIdx.x;
    if (PF && tile < ntiles) load_pair<NA, NSLOT>(b, base + tile * kTile + 2u * threadIdx.x, hi, cur);
    uint32_t seg0 = 0;  // a block's tiles come in row order: its segment only moves forward
    for (; tile < ntiles; tile += gridDim.x) {
        const uint32_t t0 = base + tile * kTile;
        const uint32_t r0 = t0 + 2u * threadIdx.x;  // this thread's rows r0, r0 + 1
        if (PF) {
            const uint32_t nt = tile + gridDim.x;
            if (nt < ntiles) load_pair<NA, NSLOT>(b, base + nt * kTile + 2u * threadIdx.x, hi, nxt);
        } else {
            load_pair<NA, NSLOT>(b, r0, hi, cur);
        }
        while (seg0 + 1 < b.nseg && t0 >= b.seg_end[seg0]) ++seg0;
        const bool one_seg = seg0 + 1 >= b.nseg || t0 + kTile <= b.seg_end[seg0];
        const uint32_t segbase = seg0 * b.nsig;
        const unsigned long long segm = b.segq[seg0];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const uint32_t row = r0 + j;
            const bool live = row - lo < hi - lo;  // lo <= row < hi
            const IxEntry ix = ix_entry<NSLOT == kIxPacked>(b, j ? cur.w0.y : cur.w0.x,
                                                            NSLOT == 2 ? (j ? cur.w1.y : cur.w1.x) : 0ull);
            uint64_t dd[4];
            uint32_t k[4];
#pragma unroll
            for (int p = 0; p < 4; ++p) {
                dd[p] = (j ? cur.f[p].y : cur.f[p].x) * b.pos[p].ainv;
                k[p] = (uint32_t)dd[p] - b.pos[p].kmin;
            }
            const uint64_t pdec = (j ? cur.pc.y : cur.pc.x) * b.price_ainv;
            const uint32_t ddec = ((j ? cur.dc >> 16 : cur.dc & 0xffffu) * (uint32_t)b.disc_ainv) & 0xffffu;
            // a corrupt foreign key, measure or index word, or a row indexed with another key
            // (a corrupt packed word never matches the row's keys: ix_key_differs covers its check)
            const uint32_t badw = (uint32_t)(dd[0] >> 32) | (uint32_t)(dd[1] >> 32) | (uint32_t)(dd[2] >> 32) |
                                  (uint32_t)(dd[3] >> 32) | (uint32_t)(pdec >> 32) |
                                  (NSLOT == kIxPacked ? 0u : ix.bad) |
                                  ix_key_differs<NSLOT == kIxPacked, NSLOT>(b, ix, k[0], k[1]) | (ddec >> 8);
            const uint32_t c0 = __ldg(b.pos[0].rank + ix.r0);
            const uint32_t c1 = NSLOT > 1 ? __ldg(b.pos[1].rank + ix.r1) : pos_code<PACK>(b.pos[1], k[1]);
            const uint32_t c2 = pos_code_clamped<PACK>(b.pos[2], k[2]);
            const uint32_t c3 = pos_code_clamped<PACK>(b.pos[3], k[3]);
            const uint32_t sig = c0 * b.pos[0].stride + c1 * b.pos[1].stride + c2 * b.pos[2].stride + c3 * b.pos[3].stride;
            const bool nz = c0 != 0 && c1 != 0 && c2 != 0 && c3 != 0;
            const bool ex = live && badw != 0;
            const unsigned em = __ballot_sync(0xffffffffu, ex);
            if (em) {
                const int lead = __ffs(em) - 1;
                unsigned long long e0 = 0;
                if (lane == lead) e0 = atomicAdd(&b.hdr->exccnt, (unsigned long long)__popc(em));
                e0 = __shfl_sync(0xffffffffu, e0, lead);
                if (ex) {
                    const unsigned long long x = e0 + __popc(em & ((1u << lane) - 1u));
                    if (x < kExcCap) b.exc[x] = row;
                    else atomicOr(&b.hdr->status, (unsigned long long)kDevStatusCapacity);
                }
            }
            uint32_t cell = segbase + sig;
            unsigned long long qs = segm;
            if (!one_seg) {
                uint32_t seg = seg0;
                while (seg + 1 < b.nseg && row >= b.seg_end[seg]) ++seg;
                cell = seg * b.nsig + sig;
                qs = b.segq[seg];
            }
            // with ACC a clean row that no query reads (none whose prefix covers
            // it accepts its codes) neither adds nor sets a first row: every
            // (query, signature) pair the contraction reads keeps its sum, and
            // its first row (the first row of the signature that the query
            // covers and accepts, which is never skipped)
            if (ACC)
                qs &= __ldg(b.pos[0].acode + c0) & __ldg(b.pos[1].acode + c1) & __ldg(b.pos[2].acode + c2) &
                      __ldg(b.pos[3].acode + c3);
            const bool ok = live && badw == 0 && (!ACC || qs != 0);
            if (ok) atomicAdd(&b.cube[cell], (unsigned long long)(uint32_t)pdec * ddec);
            bool chk = filter == 0 || !nz;
            if (filter == 1 && ok && !chk) chk = unseen_has(b.unseen, sig);
            if (ok && chk && b.cfirst[sig] > row) atomicMin(&b.cfirst[sig], row);
        }
        if (PF) cur = nxt;
    }
}

// One phase of the cube scan over the join index.  Each thread takes two
// adjacent rows per tile, so every streamed column (joined foreign keys,
// price, the index words: 16 bytes per pair; discount: 4 bytes) is one
// vector load per pair -- the fact columns must be 16-byte aligned (the
// engine checks; an odd lo starts the tiles one row early and skips that
// row).  Per row: each joined foreign key decoded and checked (32-bit offset
// arithmetic: keys are below 2^32), an indexed dimension's code from the
// batch's rank table of the entry's record when the entry holds this very
// offset, another dimension's from its code table; then the signature, and
// either the exception list (appended once per warp) or a predicated cube add
// and first-row check, the same steps as sj_cube_kernel.  Without an index
// (idx_on = 0) every dimension is looked up.  Batches of the common shape
// (SjBatch::fast) run cube_ix_fast instead.
template <int BPS, bool PACK, bool NA, bool PF, int NSLOT = 2, bool ACC = false>
__global__ void __launch_bounds__(kSjThreads, BPS) sj_cube_ix_kernel(const __grid_constant__ SjBatch b, int phase) {
    constexpr int kTile = 2 * kSjThreads;
    if (b.strategy != kStratCube) return;
    const uint64_t lo = phase ? b.r0 : 0, hi = phase ? b.nmax : b.r0;
    if (lo >= hi) return;
    int filter = 0;  // as in sj_cube_kernel
    if (phase) {
        const unsigned long long nun = __ldg(&b.hdr->unseen);
        if (nun <= kUnseenCap) filter = nun ? 1 : 2;
    }
    if (b.fast) {  // (block-uniform)
        cube_ix_fast<PACK, NA, PF, NSLOT, ACC>(b, lo, hi, filter);
        return;
    }
    const bool use_idx = b.idx_on != 0;
    const int lane = threadIdx.x & 31;
    const uint64_t base = lo & ~1ull;
    const uint32_t ntiles = (uint32_t)((hi - base + kTile - 1) / kTile);
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint64_t t0 = base + (uint64_t)tile * kTile;
        uint32_t seg0 = 0;
        while (seg0 + 1 < b.nseg && t0 >= b.seg_end[seg0]) ++seg0;
        const bool one_seg = seg0 + 1 >= b.nseg || t0 + kTile <= b.seg_end[seg0];
        const uint64_t r0 = t0 + 2u * threadIdx.x;  // this thread's rows r0, r0 + 1
        ulonglong2 fk[4], pc, iw[2];
        uint32_t dc;
        if (r0 + 1 < hi) {
#pragma unroll
            for (int d = 0; d < 4; ++d)
                fk[d] = b.dim[d].joins ? ld_stream<NA>(reinterpret_cast<const ulonglong2*>(b.dim[d].fk + r0))
                                       : make_ulonglong2(0ull, 0ull);
            pc = ld_stream<NA>(reinterpret_cast<const ulonglong2*>(b.price + r0));
            dc = ld_stream<NA>(reinterpret_cast<const uint32_t*>(b.disc + r0));
            if (use_idx) {  // iw[0]: slot 1 (or the packed words) of the two rows, iw[1]: slot 2
                iw[0] = ld_stream<NA>(reinterpret_cast<const ulonglong2*>(b.fidx1 + r0));
                iw[1] = (b.nslot > 1 && !b.ixpack) ? ld_stream<NA>(reinterpret_cast<const ulonglong2*>(b.fidx2 + r0))
                                                   : make_ulonglong2(0ull, 0ull);
            }
        } else {  // the last row of an odd range (or none)
            const bool in = r0 < hi;
#pragma unroll
            for (int d = 0; d < 4; ++d)
                fk[d] = make_ulonglong2((in && b.dim[d].joins) ? __ldg(b.dim[d].fk + r0) : 0ull, 0ull);
            pc = make_ulonglong2(in ? __ldg(b.price + r0) : 0ull, 0ull);
            dc = in ? (uint32_t)__ldg(b.disc + r0) : 0u;
            if (use_idx) {
                iw[0] = make_ulonglong2(in ? __ldg(b.fidx1 + r0) : 0ull, 0ull);
                iw[1] = make_ulonglong2((in && b.nslot > 1 && !b.ixpack) ? __ldg(b.fidx2 + r0) : 0ull, 0ull);
            }
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const uint64_t row = r0 + j;
            const bool live = row >= lo && row < hi;
            IxEntry ix{0u, 0u, 0u, 0u, 0u, 0ull};
            if (use_idx) {  // (block-uniform)
                const uint64_t w0 = j ? iw[0].y : iw[0].x, w1 = j ? iw[1].y : iw[1].x;
                ix = b.ixpack ? ix_entry<true>(b, w0, w1) : ix_entry<false>(b, w0, w1);
            }
            bool bad = ix.bad != 0;  // a corrupt index word
            uint32_t ko[2] = {0u, 0u}, kseen = 0;  // the indexed dimensions' current key offsets
            uint32_t sig = 0;
            bool nz = true;
#pragma unroll
            for (int d = 0; d < 4; ++d) {
                const SjDimDev& D = b.dim[d];
                if (!D.joins) continue;
                const uint64_t dec = (j ? fk[d].y : fk[d].x) * D.fk_ainv;
                bad |= (dec >> 32) != 0;
                const uint32_t k = (uint32_t)dec - (uint32_t)D.kmin;
                uint32_t cv = 0;
                if (use_idx && D.ixslot && D.ixslot <= b.nslot) {
                    ko[D.ixslot - 1] = k;
                    kseen |= 1u << (D.ixslot - 1);
                    cv = __ldg(b.ixrank[D.ixslot - 1] + (D.ixslot == 1 ? ix.r0 : ix.r1));
                } else if (k < (uint32_t)D.krange) {
                    if (PACK) {
                        const uint32_t q = (uint32_t)(((uint64_t)k * D.cmagic) >> 40);
                        const uint32_t r = k - q * D.per;
                        const unsigned long long w = __ldg(static_cast<const unsigned long long*>(D.code) + q);
                        cv = (uint32_t)(w >> (r * D.cbits)) & ((1u << D.cbits) - 1u);
                    } else {
                        cv = D.cw == 1 ? __ldg(static_cast<const uint8_t*>(D.code) + k)
                                       : __ldg(static_cast<const uint16_t*>(D.code) + k);
                    }
                }
                sig = sig * b.radix[d] + cv;
                nz &= cv != 0;
            }
            // not the keys the row was indexed with (a packed batch joins both indexed dimensions)
            if (use_idx) {
                if (b.ixpack) bad |= ix_key_differs<true, 2>(b, ix, ko[0], ko[1]) != 0;
                else bad |= ((kseen & 1u) && ko[0] != ix.k0) || ((kseen & 2u) && ko[1] != ix.k1);
            }
            const uint64_t pdec = (j ? pc.y : pc.x) * b.price_ainv;
            const uint32_t ddec = ((j ? dc >> 16 : dc & 0xffffu) * (uint32_t)b.disc_ainv) & 0xffffu;
            bad |= (pdec >> 32) != 0 || ddec > 0xffu;
            // rows with a detected error (or an index entry of another key): the exact path
            const bool ex = live && bad;
            const unsigned em = __ballot_sync(0xffffffffu, ex);
            if (em) {
                const int lead = __ffs(em) - 1;
                unsigned long long k0 = 0;
                if (lane == lead) k0 = atomicAdd(&b.hdr->exccnt, (unsigned long long)__popc(em));
                k0 = __shfl_sync(0xffffffffu, k0, lead);
                if (ex) {
                    const unsigned long long k = k0 + __popc(em & ((1u << lane) - 1u));
                    if (k < kExcCap) b.exc[k] = (uint32_t)row;
                    else atomicOr(&b.hdr->status, (unsigned long long)kDevStatusCapacity);
                }
            }
            const bool ok = live && !bad;
            uint32_t seg = seg0;
            if (!one_seg)
                while (seg + 1 < b.nseg && row >= b.seg_end[seg]) ++seg;
            if (ok) atomicAdd(&b.cube[(uint64_t)seg * b.nsig + sig], (unsigned long long)(uint32_t)pdec * ddec);
            bool chk = filter == 0 || !nz;
            if (filter == 1 && ok && !chk) chk = unseen_has(b.unseen, sig);
            if (ok && chk && b.cfirst[sig] > (uint32_t)row) atomicMin(&b.cfirst[sig], (uint32_t)row);
        }
    }
}

using SjCubeFn = void (*)(SjBatch, int);
// Cube-scan shapes the tuner chooses from: rows per thread, blocks per SM,
// packed code tables, acceptance skip (each of the last two helps some shapes
// and costs others); the indexed shapes read the join index (and stream
// without L1 allocation, or not).
struct CubeShape {
    SjCubeFn fn;
    int blocks_per_sm;
    bool pack, idx;
    int nslot;  // index slots the shape reads (0: none; kIxPacked: both, from the packed index)
};
const CubeShape kCubeShapes[] = {
    {sj_cube_kernel<2, 4, true, false>, 4, true, false, 0},
    {sj_cube_kernel<2, 4, false, true>, 4, false, false, 0},
    {sj_cube_kernel<4, 3, false, true>, 3, false, false, 0},
    {sj_cube_kernel<4, 3, true, false>, 3, true, false, 0},
    {sj_cube_ix_kernel<3, true, true, true>, 3, true, true, 2},  // the default when the engine has an index
    {sj_cube_ix_kernel<4, true, true, true>, 4, true, true, 2},
    {sj_cube_ix_kernel<4, true, true, false>, 4, true, true, 2},
    {sj_cube_ix_kernel<6, true, true, false>, 6, true, true, 2},
    {sj_cube_ix_kernel<4, false, true, true>, 4, false, true, 2},
    {sj_cube_ix_kernel<4, true, false, true>, 4, true, true, 2},
    // one index slot (8 B per row less; the second dimension's code is looked
    // up again): 8.8 ms against 6.7 ms per 600M-row batch on SSB at SF100,
    // where the second slot's dimension (part) has 1.4M keys
    {sj_cube_ix_kernel<3, true, true, true, 1>, 3, true, true, 1},
    // the packed index (one word per row for both slots)
    {sj_cube_ix_kernel<3, true, true, true, kIxPacked>, 3, true, true, kIxPacked},
    {sj_cube_ix_kernel<4, true, true, false, kIxPacked>, 4, true, true, kIxPacked},
    // the same and the acceptance skip: a row no query reads makes no cube add
    // (at SF100 the default: 6.0 ms per 600M-row batch against 6.2 without the
    // skip and 6.5 with the two-word index)
    {sj_cube_ix_kernel<4, true, true, false, kIxPacked, true>, 4, true, true, kIxPacked},
    {sj_cube_ix_kernel<6, true, true, false, kIxPacked, true>, 6, true, true, kIxPacked},
};
constexpr int kCubeIndexedDefault = 4;
constexpr int kCubePackedDefault = 13;
constexpr int kCubeVariants = (int)(sizeof(kCubeShapes) / sizeof(kCubeShapes[0]));

// The exact per-query semantics of one fact row (the operator composition's
// drops and error reports), for rows the cube scan routed here.
__global__ void __launch_bounds__(kSjThreads) sj_exc_kernel(const SjBatch* __restrict__ bp) {
    __shared__ SjBatch b;
    __shared__ SjQDev s_q[kMaxQ];
    for (int i = threadIdx.x; i < (int)(sizeof(SjBatch) / 8); i += blockDim.x)
        reinterpret_cast<unsigned long long*>(&b)[i] = reinterpret_cast<const unsigned long long*>(bp)[i];
    __syncthreads();
    if (b.strategy != kStratCube) return;
    for (int i = threadIdx.x; i < (int)(b.nq * sizeof(SjQDev) / 8); i += blockDim.x)
        reinterpret_cast<unsigned long long*>(s_q)[i] = reinterpret_cast<const unsigned long long*>(b.q)[i];
    __syncthreads();
    const unsigned long long cnt = b.hdr->exccnt;
    const uint32_t n = cnt < kExcCap ? (uint32_t)cnt : kExcCap;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint64_t row = b.exc[k];
        unsigned long long alive = 0;
        for (uint32_t q = 0; q < b.nq; ++q)
            if (row < s_q[q].nrows) alive |= 1ull << q;
        // every load first (foreign keys, then records, then accept masks, and the
        // measures), so a row costs three dependent round trips instead of twelve;
        // the drops and reports then follow the join order as before
        unsigned long long code[4], accm[4];
        uint32_t rv[4];
#pragma unroll
        for (int d = 0; d < 4; ++d) code[d] = (alive & b.dim[d].joins) ? __ldg(b.dim[d].fk + row) : 0ull;
        const unsigned long long pcode = __ldg(b.price + row);
        const uint32_t dcode = __ldg(b.disc + row);
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            const SjDimDev& D = b.dim[d];
            const uint64_t idx = ((code[d] * D.fk_ainv) & 0xffffffffull) - D.kmin;  // truncated to the key type
            rv[d] = ((alive & D.joins) && idx < D.krange) ? __ldg(D.rec + idx) : 0u;
        }
#pragma unroll
        for (int d = 0; d < 4; ++d) accm[d] = (alive & b.dim[d].joins) ? __ldg(b.dim[d].acc + rv[d]) : ~0ull;
        uint32_t at[4] = {0, 0, 0, 0};
        for (int kk = 0; kk < 4; ++kk) {
            const int d = join_dim(kk);
            const SjDimDev& D = b.dim[d];
            const unsigned long long jq = alive & D.joins;
            if (!jq) continue;
            at[d] = rv[d] - 1u;
            if ((code[d] * D.fk_ainv) > 0xffffffffull) {
                log_err(b, jq, d, row);
                alive &= ~(jq & ~D.first);  // positional fetch drops the row
            }
            alive &= accm[d] | ~D.joins;
        }
        if (!alive) continue;
        const uint64_t pdec = pcode * b.price_ainv;
        if (pdec > 0xffffffffull) {
            log_err(b, alive, 4, row);
            continue;
        }
        const uint32_t ddec = (dcode * (uint32_t)b.disc_ainv) & 0xffffu;
        if (ddec > 0xffu) {
            log_err(b, alive, 5, row);
            continue;
        }
        const unsigned long long v = pdec * ddec;
        while (alive) {
            const int q = __ffsll(alive) - 1;
            alive &= alive - 1;
            const SjQDev& Q = s_q[q];
            uint64_t g = 0;
            for (uint32_t j = 0; j < Q.ngroup; ++j)
                g += (uint64_t)((at[Q.gdim[j]] >> Q.gshift[j]) & Q.gpmask[j]) * Q.gstride[j];
            atomicAdd(&b.sums[Q.gbase + g], v);
            atomicMin(&b.firsts[Q.gbase + g], (uint32_t)row);
        }
    }
}

// Pass 2: per signature present in the cube, the batch queries accepting it
// (from the accept tables of its dimension codes) take its segment sums up to
// their prefix and its first row into their group.
__global__ void __launch_bounds__(kSjThreads) sj_contract_kernel(const SjBatch* __restrict__ bp) {
    extern __shared__ unsigned long long s_dyn[];  // [kSmemGroups] sums, then [kSmemGroups] first rows
    __shared__ SjBatch b;
    __shared__ SjQDev s_q[kMaxQ];
    __shared__ uint64_t s_n[kMaxQ];
    for (int i = threadIdx.x; i < (int)(sizeof(SjBatch) / 8); i += blockDim.x)
        reinterpret_cast<unsigned long long*>(&b)[i] = reinterpret_cast<const unsigned long long*>(bp)[i];
    __syncthreads();
    if (b.strategy != kStratCube) return;
    for (int i = threadIdx.x; i < (int)(b.nq * sizeof(SjQDev) / 8); i += blockDim.x)
        reinterpret_cast<unsigned long long*>(s_q)[i] = reinterpret_cast<const unsigned long long*>(b.q)[i];
    unsigned long long* s_sum = s_dyn;
    uint32_t* s_first = reinterpret_cast<uint32_t*>(s_dyn + kSmemGroups);
    for (uint32_t i = threadIdx.x; i < b.nsm; i += blockDim.x) {
        s_sum[i] = 0;
        s_first[i] = kNoRow;
    }
    __syncthreads();
    if (threadIdx.x < b.nq) s_n[threadIdx.x] = s_q[threadIdx.x].nrows;
    __syncthreads();
    unsigned long long okm = 0;
    for (uint32_t q = 0; q < b.nq; ++q)
        if (s_n[q]) okm |= 1ull << q;
    const uint32_t nsm = b.nsm;
    for (uint32_t sg = blockIdx.x * blockDim.x + threadIdx.x; sg < b.nsig; sg += gridDim.x * blockDim.x) {
        const uint32_t f = b.cfirst[sg];
        if (f == kNoRow) continue;
        uint32_t c[4];
        uint32_t rem = sg;
#pragma unroll
        for (int d = 3; d >= 0; --d) {
            c[d] = rem % b.radix[d];
            rem /= b.radix[d];
        }
        unsigned long long m = okm;
        uint32_t rp[4] = {0, 0, 0, 0};
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            const SjDimDev& D = b.dim[d];
            if (!D.joins) continue;
            rp[d] = b.rep[d][c[d]];
            m &= __ldg(D.acc + rp[d]) | ~D.joins;
        }
        if (!m) continue;
        unsigned long long cum[kMaxSeg];
        unsigned long long run = 0;
#pragma unroll
        for (int k = 0; k < kMaxSeg; ++k) {
            if (k < (int)b.nseg) run += b.cube[(uint64_t)k * b.nsig + sg];
            cum[k] = run;
        }
        while (m) {
            const int q = __ffsll(m) - 1;
            m &= m - 1;
            if (f >= s_n[q]) continue;
            const SjQDev& Q = s_q[q];
            unsigned long long v = 0;
#pragma unroll
            for (int k = 0; k < kMaxSeg; ++k)
                if (k + 1 == (int)Q.segs) v = cum[k];
            uint64_t g = 0;
            for (uint32_t j = 0; j < Q.ngroup; ++j) {
                const uint32_t a = pick4(rp[0], rp[1], rp[2], rp[3], Q.gdim[j]) - 1u;
                g += (uint64_t)((a >> Q.gshift[j]) & Q.gpmask[j]) * Q.gstride[j];
            }
            const uint64_t slot = Q.gbase + g;
            if (slot < nsm) {
                atomicAdd(&s_sum[slot], v);
                atomicMin(&s_first[slot], f);
            } else {
                atomicAdd(&b.sums[slot], v);
                atomicMin(&b.firsts[slot], f);
            }
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < nsm; i += blockDim.x) {
        if (s_first[i] != kNoRow) {
            atomicAdd(&b.sums[i], s_sum[i]);
            atomicMin(&b.firsts[i], s_first[i]);
        }
    }
}

// Accept tables of a batch: per dimension and packed attribute value, the
// batch queries joining the dimension whose predicate (if any) holds on the
// attribute's code -- the code a clean row with that value has.
struct AcceptQ {
    RangePred pred, pred2;  // pred2: a second predicate on another attribute (AND)
    int attr, has_pred, attr2, has_pred2;
};

struct SjDimPack {
    uint32_t bits;                   // packed bits (<= kAccBits); 0: no record table
    uint32_t shift[AHEAD_SJ_MAXATTR], pmask[AHEAD_SJ_MAXATTR];
    uint64_t amin[AHEAD_SJ_MAXATTR], A[AHEAD_SJ_MAXATTR], wm[AHEAD_SJ_MAXATTR];
    int packed[AHEAD_SJ_MAXATTR];
    const uint8_t* present;          // [2^bits] packed values some row has
    // row mode: (value - amin) of every clean attribute by key offset, and the
    // key records (0: no row has the key)
    const uint32_t* aval[AHEAD_SJ_MAXATTR];
    const uint32_t* rec;
    uint64_t krange;
};

struct SjPackAll {
    SjDimPack d[4];
};

// `nonempty` collects the queries that accept at least one row: hashjoinAN
// probes nothing when its build side is empty (hashjoinAN.tcc:128), so such a
// query reports no errors for its first foreign key.
__global__ void sj_accept_kernel(const SjBatch* __restrict__ bp, const AcceptQ* __restrict__ aq, SjPackAll pk,
                                 unsigned long long* acc_all) {
    const int d = blockIdx.y;
    const SjDimPack& P = pk.d[d];
    const unsigned long long joins = bp->dim[d].joins;
    const uint32_t n = 1u << P.bits;
    unsigned long long* acc = acc_all + (size_t)d * kAccEntries;
    const int nq = (int)bp->nq;
    unsigned long long any = 0;
    unsigned long long* accr = const_cast<unsigned long long*>(bp->dim[d].accr);
    if (accr) {  // row mode: the masks by key offset, from the attribute values
        for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < P.krange;
             k += (uint64_t)gridDim.x * blockDim.x) {
            unsigned long long m = 0;
            if (joins && P.rec[k]) {
                for (int q = 0; q < nq; ++q) {
                    if (!((joins >> q) & 1ull)) continue;
                    const AcceptQ& x = aq[d * kMaxQ + q];
                    bool ok = true;
                    if (x.has_pred) {
                        const int a = x.attr;
                        ok = x.pred(((P.aval[a][k] + P.amin[a]) * P.A[a]) & P.wm[a]);
                    }
                    if (ok && x.has_pred2) {
                        const int a = x.attr2;
                        ok = x.pred2(((P.aval[a][k] + P.amin[a]) * P.A[a]) & P.wm[a]);
                    }
                    if (ok) m |= 1ull << q;
                }
            }
            any |= m;
            accr[k] = m;
        }
        const uint32_t lo = __reduce_or_sync(0xffffffffu, (uint32_t)any);
        const uint32_t hi = __reduce_or_sync(0xffffffffu, (uint32_t)(any >> 32));
        if ((threadIdx.x & 31) == 0 && (lo | hi))
            atomicOr(&bp->hdr->nonempty[d], ((unsigned long long)hi << 32) | lo);
        return;
    }
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e <= n; e += gridDim.x * blockDim.x) {
        unsigned long long m = 0;
        if (e > 0 && joins) {  // joins != 0 only for usable dimensions, which have `present`
            const uint32_t p = e - 1;
            for (int q = 0; q < nq; ++q) {
                if (!((joins >> q) & 1ull)) continue;
                const AcceptQ& x = aq[d * kMaxQ + q];
                bool ok = true;
                if (x.has_pred) {
                    const int a = x.attr;
                    const uint64_t v = ((p >> P.shift[a]) & P.pmask[a]) + P.amin[a];
                    ok = x.pred((v * P.A[a]) & P.wm[a]);
                }
                if (ok && x.has_pred2) {
                    const int a = x.attr2;
                    const uint64_t v = ((p >> P.shift[a]) & P.pmask[a]) + P.amin[a];
                    ok = x.pred2((v * P.A[a]) & P.wm[a]);
                }
                if (ok) m |= 1ull << q;
            }
            if (P.present[p]) any |= m;
        }
        acc[e] = m;
    }
    const uint32_t lo = __reduce_or_sync(0xffffffffu, (uint32_t)any);
    const uint32_t hi = __reduce_or_sync(0xffffffffu, (uint32_t)(any >> 32));
    if ((threadIdx.x & 31) == 0 && (lo | hi)) atomicOr(&bp->hdr->nonempty[d], ((unsigned long long)hi << 32) | lo);
}

// The code of row r of a dimension attribute column of w bytes (2, 4 or 8).
__device__ __forceinline__ uint64_t attr_code(const void* col, int w, uint64_t r) {
    return w == 2 ? (uint64_t)((const uint16_t*)col)[r]
                  : w == 4 ? (uint64_t)((const uint32_t*)col)[r] : (uint64_t)((const unsigned long long*)col)[r];
}

struct SjDimStatic {
    const unsigned long long* key;
    const void* attr[AHEAD_SJ_MAXATTR];
    int w[AHEAD_SJ_MAXATTR];
    int nattr;
    uint64_t key_ainv, kmin;
    uint32_t* rec;
    uint8_t* present;
};

// Records of every dimension row and the packed values present (once per engine).
__global__ void sj_pack_attrs_kernel(SjDimStatic ds, SjDimPack pk, uint64_t rows, uint64_t ainv0, uint64_t ainv1,
                                     uint64_t ainv2, uint64_t ainv3) {
    const uint64_t ainv[4] = {ainv0, ainv1, ainv2, ainv3};
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < rows; r += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t packed = 0;
        for (int a = 0; a < ds.nattr; ++a) {
            if (!pk.packed[a]) continue;
            const uint64_t c = attr_code(ds.attr[a], ds.w[a], r);
            const uint64_t v = mulw(c, ainv[a], ds.w[a]);
            packed |= (uint32_t)(v - pk.amin[a]) << pk.shift[a];
        }
        const uint64_t idx = ds.key[r] * ds.key_ainv - ds.kmin;
        ds.rec[idx] = packed + 1u;
        ds.present[packed] = 1;
    }
}

// Row mode's attribute tables: (decoded value - amin) by key offset, for
// every clean attribute (once per engine).
__global__ void sj_aval_kernel(SjDimStatic ds, uint64_t rows, int a, uint64_t ainv, uint64_t amin, uint32_t* out) {
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < rows; r += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t c = attr_code(ds.attr[a], ds.w[a], r);
        const uint64_t idx = ds.key[r] * ds.key_ainv - ds.kmin;
        out[idx] = (uint32_t)(mulw(c, ainv, ds.w[a]) - amin);
    }
}

// Key map: decoded keys (all valid) minus kmin index the dimension rows.
__global__ void sj_keyrange_kernel(const unsigned long long* codes, uint64_t n, uint64_t ainv,
                                   unsigned long long* mm /* [0]=min [1]=max [2]=bad */) {
    unsigned long long lo = ~0ull, hi = 0, bad = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = codes[i] * ainv;
        if (k > 0xffffffffull) {
            ++bad;
            continue;
        }
        lo = k < lo ? k : lo;
        hi = k > hi ? k : hi;
    }
    atomicMin(&mm[0], lo);
    atomicMax(&mm[1], hi);
    if (bad) atomicAdd(&mm[2], bad);
}

__global__ void sj_kmap_kernel(const unsigned long long* codes, uint64_t n, uint64_t ainv, uint64_t kmin,
                               uint32_t* kmap, unsigned long long* dup) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = codes[i] * ainv;
        if (atomicCAS(&kmap[k - kmin], 0u, (uint32_t)(i + 1)) != 0u) atomicAdd(dup, 1ull);
    }
}

// The join index of every fact row (once per engine): per index slot, the
// decoded foreign key's 32-bit offset (key - kmin, wrapping) and that key's
// record (0 outside [0, krange)), AN-coded.  A corrupt foreign key is indexed by its truncated key,
// as the scan reads it (the row takes the exact path in every batch anyway).
struct SjIdxBuild {
    const unsigned long long* fk[kIxSlots];
    const uint32_t* rec[kIxSlots];
    uint64_t ainv[kIxSlots], kmin[kIxSlots], krange[kIxSlots];
    int nslots;
    // packed: one word per row (the layout of SjBatch::ixp_*), and per slot
    // record -> id ([kAccEntries])
    int packed;
    uint64_t A;
    uint32_t ib, s1, r0, kr[kIxSlots];
    const uint16_t* idmap[kIxSlots];
};

__global__ void sj_index_kernel(const SjIdxBuild ib, uint64_t n, unsigned long long* __restrict__ out1,
                                unsigned long long* __restrict__ out2) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t row = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; row < n; row += stride) {
        uint64_t w[kIxSlots] = {0, 0};
        uint32_t o[kIxSlots] = {0, 0}, id[kIxSlots] = {0, 0};
#pragma unroll
        for (int s = 0; s < kIxSlots; ++s) {
            if (s >= ib.nslots) break;
            const uint64_t dec = __ldg(ib.fk[s] + row) * ib.ainv[s];
            const uint32_t k = (uint32_t)dec - (uint32_t)ib.kmin[s];
            const bool in = k < (uint32_t)ib.krange[s];
            const uint32_t rec = in ? __ldg(ib.rec[s] + k) : 0u;
            w[s] = ((uint64_t)k | (uint64_t)rec << 32) * kIxA;
            if (ib.packed) {  // (the record is below kAccEntries: packed bits + 1)
                o[s] = in ? k : ib.kr[s];
                id[s] = __ldg(ib.idmap[s] + rec);
            }
        }
        if (ib.packed) {
            const uint64_t kj = (uint64_t)o[0] + (uint64_t)ib.r0 * o[1];
            out1[row] = ((uint64_t)id[0] | (uint64_t)id[1] << ib.s1 | kj << ib.ib) * ib.A;
        } else {
            out1[row] = w[0];
            out2[row] = w[1];
        }
    }
}

// Decoded range and corrupt count of an attribute column.
__global__ void sj_attr_kernel(const void* col, int w, uint64_t n, uint64_t ainv, uint64_t umax,
                               unsigned long long* mm) {
    unsigned long long lo = ~0ull, hi = 0, bad = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t c = attr_code(col, w, i);
        const uint64_t v = mulw(c, ainv, w);
        if (v > umax) {
            ++bad;
            continue;
        }
        lo = v < lo ? v : lo;
        hi = v > hi ? v : hi;
    }
    atomicMin(&mm[0], lo);
    atomicMax(&mm[1], hi);
    if (bad) atomicAdd(&mm[2], bad);
}

// All queries' present groups (first row set) into their lists, in any order,
// as (first row << 32 | dense index) at lists[gbase, ...); ngroups[q] counts
// them (the clear kernel zeroed it).  One pass over every query's dense slots
// with the whole grid; the finalize kernel then orders each list.  (One block
// a query, compacting inside the finalize kernel, took 2.2 ms over the 1.75M
// dense slots of one SSB program.)
__global__ void sj_compact_kernel(const SjBatch* __restrict__ bp) {
    __shared__ uint64_t s_lo[kMaxQ], s_hi[kMaxQ];
    const uint32_t nq = bp->nq;
    if (threadIdx.x < kMaxQ) {
        uint64_t lo = 0, hi = 0;
        if (threadIdx.x < nq) {
            const SjQDev& Q = bp->q[threadIdx.x];
            if (Q.ngroup) {  // (an ungrouped query's total is read from its slot by the finalize kernel)
                lo = Q.gbase;
                hi = Q.gbase + Q.gsize;
            }
        }
        s_lo[threadIdx.x] = lo;
        s_hi[threadIdx.x] = hi;
    }
    __syncthreads();
    const uint64_t n = bp->gtotal;
    const uint32_t* firsts = bp->firsts;
    unsigned long long* lists = bp->lists;
    unsigned long long* cnt = bp->hdr->ngroups;
    const int lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t g0 = (uint64_t)blockIdx.x * blockDim.x; g0 < n; g0 += stride) {  // (block-uniform)
        const uint64_t g = g0 + threadIdx.x;
        const uint32_t f = g < n ? firsts[g] : kNoRow;
        int q = -1;
        if (f != kNoRow)
            for (uint32_t k = 0; k < nq; ++k)
                if (g >= s_lo[k] && g < s_hi[k]) {
                    q = (int)k;
                    break;
                }
        if (!__any_sync(0xffffffffu, q >= 0)) continue;
        const unsigned peers = __match_any_sync(0xffffffffu, q);  // the lanes of the same query
        if (q >= 0) {
            const int lead = __ffs(peers) - 1;
            unsigned long long base = 0;
            if (lane == lead) base = atomicAdd(&cnt[q], (unsigned long long)__popc(peers));
            base = __shfl_sync(peers, base, lead);
            lists[s_lo[q] + base + __popc(peers & ((1u << lane) - 1u))] =
                ((unsigned long long)f << 32) | (g - s_lo[q]);
        }
    }
}

// Per query (one block): the present groups the compact kernel listed, ordered
// by first row -- groupbyAN numbers groups by first occurrence -- in
// lists[gbase, gbase + n), n = ngroups[q].  Up to
// kSortSmem groups sort in shared memory (bitonic); more sort in global
// memory by a least-significant-digit radix sort on the first row (first rows
// of a query's groups are distinct, one row belongs to one group).
constexpr uint32_t kSortSmem = 4096;  // (a larger bitonic sort lost to the radix sort: O(n log^2 n))

// Stable LSD radix sort of a[0, n) by one block of 1024 threads over the
// npass 8-bit digits at bits shift0, shift0 + 8, ..., ping-ponging between a
// and t (an even npass leaves the result in a).  Per 1024-key chunk a digit's
// keys are ranked by __match_any_sync within each warp and offset by the
// counts of the warps before; shared scratch: per-warp digit counts [32][256]
// and the digit bases and chunk totals [256].
__device__ void radix_block(unsigned long long* a, unsigned long long* t, uint32_t n, int shift0, int npass,
                            uint32_t (*s_wcnt)[256], uint32_t* s_base, uint32_t* s_tot) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int pass = 0; pass < npass; ++pass) {
        const unsigned long long* src = (pass & 1) ? t : a;
        unsigned long long* dst = (pass & 1) ? a : t;
        const int shift = shift0 + 8 * pass;
        for (int i = threadIdx.x; i < 256; i += blockDim.x) s_base[i] = 0;
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) atomicAdd(&s_base[(src[i] >> shift) & 0xff], 1u);
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t run = 0;
            for (int d = 0; d < 256; ++d) {
                const uint32_t c = s_base[d];
                s_base[d] = run;
                run += c;
            }
        }
        __syncthreads();
        for (uint32_t c0 = 0; c0 < n; c0 += blockDim.x) {
            for (int i = threadIdx.x; i < 32 * 256; i += blockDim.x) (&s_wcnt[0][0])[i] = 0;
            __syncthreads();
            const uint32_t i = c0 + threadIdx.x;
            const bool valid = i < n;
            const unsigned long long key = valid ? src[i] : 0ull;
            const uint32_t dg = valid ? (uint32_t)((key >> shift) & 0xff) : 256u;
            const uint32_t peers = __match_any_sync(0xffffffffu, dg);
            const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
            if (valid && rank == 0) s_wcnt[warp][dg] = __popc(peers);
            __syncthreads();
            if (threadIdx.x < 256) {  // exclusive offsets of each digit over the warps
                uint32_t run = 0;
                for (int w = 0; w < 32; ++w) {
                    const uint32_t c = s_wcnt[w][threadIdx.x];
                    s_wcnt[w][threadIdx.x] = run;
                    run += c;
                }
                s_tot[threadIdx.x] = run;
            }
            __syncthreads();
            if (valid) dst[s_base[dg] + s_wcnt[warp][dg] + rank] = key;
            __syncthreads();
            if (threadIdx.x < 256) s_base[threadIdx.x] += s_tot[threadIdx.x];
            __syncthreads();
        }
    }
}

// Ascending bitonic sort of k[0, p) by one block (p a power of two).
__device__ __forceinline__ void bitonic_block(unsigned long long* k, uint32_t p) {
    for (uint32_t w = 2; w <= p; w <<= 1) {
        for (uint32_t j = w >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < p; i += blockDim.x) {
                const uint32_t l = i ^ j;
                if (l > i) {
                    const unsigned long long a = k[i], c = k[l];
                    if ((a > c) == ((i & w) == 0)) {
                        k[i] = c;
                        k[l] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
}


__global__ void __launch_bounds__(1024) sj_finalize_kernel(const SjBatch* __restrict__ bp) {
    // the bitonic keys and the radix sort's per-warp digit counts share one buffer
    __shared__ unsigned long long s_buf[kSortSmem];
    static_assert(sizeof(s_buf) >= 32 * 256 * 4, "radix counts fit the sort buffer");
    unsigned long long* s_k = s_buf;
    uint32_t (*s_wcnt)[256] = reinterpret_cast<uint32_t (*)[256]>(s_buf);
    __shared__ uint32_t s_base[256], s_tot[256];
    const uint32_t q = blockIdx.x;
    if (q >= bp->nq) return;
    const SjQDev& Q = bp->q[q];
    SjHdr* h = bp->hdr;
    if (Q.ngroup == 0) {  // the ungrouped total sits in the query's one dense slot
        if (threadIdx.x == 0) {
            h->ngroups[q] = 0;
            h->raw[q] = Q.gsize ? bp->sums[Q.gbase] : 0ull;
        }
        return;
    }
    unsigned long long* L = bp->lists + Q.gbase;
    unsigned long long* T = bp->lists_tmp + Q.gbase;
    const uint32_t n = (uint32_t)h->ngroups[q];
    if (n <= kSortSmem) {
        uint32_t p = 1;
        while (p < n) p <<= 1;
        for (uint32_t i = threadIdx.x; i < p; i += blockDim.x) s_k[i] = i < n ? L[i] : ~0ull;
        __syncthreads();
        bitonic_block(s_k, p);
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) L[i] = s_k[i];
    } else {
        // four stable 8-bit passes over the first row (bits 32..63); L -> T -> L -> T -> L
        radix_block(L, T, n, 32, 4, s_wcnt, s_base, s_tot);
    }
    if (threadIdx.x == 0) h->ngroups[q] = n;
}

// One block per query: the query's entries of the error log, sorted ascending
// (by column, then row), at its place in the packed area -- after the entries
// of the queries before it, so the area's front is the whole log sorted by
// (query, column, row) -- gathered into shared memory and sorted there
// (bitonic) up to kPackBitonic entries, else gathered into the packed area and
// sorted in place by a radix sort in global memory.  Block 0 also lays out
// the groups after the log: per query keys[0..G) (n each), then sums (n); a
// query whose groups do not fit the packed area is marked (ngroups = ~0) and
// left to the caller's fallback.
constexpr uint32_t kPackSmem = 8192;     // 64 KB of dynamic shared memory (bitonic keys; radix counts)
constexpr uint32_t kPackBitonic = 2048;  // more entries for one query: the radix sort (bitonic is O(n log^2 n))
static_assert(kPackSmem * 8 >= 32 * 256 * 4 && kPackBitonic <= kPackSmem, "pack kernel shared memory");

__global__ void __launch_bounds__(1024) sj_pack_kernel(const SjBatch* __restrict__ bp) {
    extern __shared__ unsigned long long s_log[];  // [kPackSmem]
    __shared__ uint32_t s_cnt[2], s_fill;
    SjHdr* h = bp->hdr;
    const unsigned long long* log = bp->errlog;
    unsigned long long* out = bp->packed;
    const unsigned long long cnt = h->errcnt;
    const uint32_t n = cnt < (unsigned long long)kErrLogCap ? (uint32_t)cnt : (uint32_t)kErrLogCap;
    const uint32_t q = blockIdx.x;
    if (q == 0 && threadIdx.x == 0) {
        unsigned long long off = n;
        for (uint32_t k = 0; k < bp->nq; ++k) {
            h->off[k] = off;
            const uint32_t G = bp->q[k].ngroup;
            const unsigned long long ng = h->ngroups[k];
            if (!G || ng == ~0ull) continue;
            if (off + ng * (G + 1) > bp->packed_cap) {
                h->ngroups[k] = ~0ull;
                continue;
            }
            off += ng * (G + 1);
        }
        h->nerr = n;
        h->packed_len = off;
    }
    if (q >= bp->nq) return;
    // this query's entries and those of the queries before it
    if (threadIdx.x < 2) s_cnt[threadIdx.x] = 0;
    if (threadIdx.x == 0) s_fill = 0;
    __syncthreads();
    uint32_t lt = 0, eq = 0;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const uint32_t k = (uint32_t)(log[i] >> 58);
        lt += k < q;
        eq += k == q;
    }
    for (int o = 16; o > 0; o >>= 1) {
        lt += __shfl_down_sync(0xffffffffu, lt, o);
        eq += __shfl_down_sync(0xffffffffu, eq, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&s_cnt[0], lt);
        atomicAdd(&s_cnt[1], eq);
    }
    __syncthreads();
    const uint32_t off = s_cnt[0], m = s_cnt[1];
    if (!m) return;
    const bool in_smem = m <= kPackBitonic;
    unsigned long long* dst = in_smem ? s_log : out + off;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const unsigned long long e = log[i];
        if ((uint32_t)(e >> 58) == q) dst[atomicAdd(&s_fill, 1u)] = e;
    }
    __syncthreads();
    if (in_smem) {
        uint32_t p = 1;
        while (p < m) p <<= 1;
        for (uint32_t i = m + threadIdx.x; i < p; i += blockDim.x) s_log[i] = ~0ull;
        __syncthreads();
        bitonic_block(s_log, p);
        for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) out[off + i] = s_log[i];
    } else {
        // (column, row) as column << 32 | row (rows are below 2^32): six stable
        // 8-bit passes over bits 0..47 ping-pong through the scratch and back
        __shared__ uint32_t s_base[256], s_tot[256];
        uint32_t (*s_wcnt)[256] = reinterpret_cast<uint32_t (*)[256]>(s_log);
        for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
            const unsigned long long k = dst[i];
            dst[i] = (((k >> kLogColShift) & 15ull) << 32) | (k & 0xffffffffull);
        }
        __syncthreads();
        radix_block(dst, bp->lists_tmp + off, m, 0, 6, s_wcnt, s_base, s_tot);
        for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
            const unsigned long long k = dst[i];
            dst[i] = ((unsigned long long)q << 58) | (((k >> 32) & 15ull) << kLogColShift) | (k & 0xffffffffull);
        }
    }
}

// The groups of each query into the packed area: the group attributes' codes
// from the dense index, and the sums AN-coded as aggregate_sum_groupedAN
// leaves them: price * discount with A^2 (arithmeticAN<mul> multiplies two
// codes of A), revenue and revenue - supplycost with A.
__global__ void sj_emit_kernel(const SjBatch* __restrict__ bp) {
    const uint32_t q = blockIdx.y;
    if (q >= bp->nq) return;
    const SjQDev& Q = bp->q[q];
    const SjHdr* h = bp->hdr;
    const uint32_t G = Q.ngroup;
    const unsigned long long ng = h->ngroups[q];
    if (!G || ng == ~0ull) return;
    const unsigned long long* L = bp->lists + Q.gbase;
    const unsigned long long* sums = bp->sums + Q.gbase;
    unsigned long long* o = bp->packed + h->off[q];
    const uint64_t scale = (((bp->mrev | bp->mprof) >> q) & 1ull) ? kResoidAMax : kResoidAMax * kResoidAMax;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < ng; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t g = L[i] & 0xffffffffull;
        o[(size_t)G * ng + i] = sums[g] * scale;
        uint64_t rem = g;
        for (int j = (int)G - 1; j >= 0; --j) {
            const uint64_t vj = rem / Q.gstride[j];
            rem -= vj * Q.gstride[j];
            o[(size_t)j * ng + i] = ((vj + Q.glo[j]) * Q.gA[j]) & Q.gwm[j];
        }
    }
}

constexpr size_t kPackedWords = (size_t)1 << 22;  // packed result words per batch (errors + groups)

// ------------------------------------------------ fact-sharded batches
// Export (end of a batch's local half): the dense group tables and the error
// log with rows of the whole table (local row + the shard's first row), the
// status flags one word each, for the caller's all-reduces and all-gather.
__global__ void sj_export_kernel(const SjBatch* __restrict__ bp, long long* xsum, long long* xfirst,
                                 long long* xflag, unsigned long long* xlog, uint64_t shard_lo) {
    const uint64_t n = bp->gtotal;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    for (uint64_t i = t; i < n; i += stride) {
        xsum[i] = (long long)bp->sums[i];
        const uint32_t f = bp->firsts[i];
        xfirst[i] = f == kNoRow ? LLONG_MAX : (long long)(f + shard_lo);
    }
    const unsigned long long cnt = bp->hdr->errcnt;
    const uint64_t ne = cnt < (unsigned long long)kErrLogCap ? cnt : (uint64_t)kErrLogCap;
    for (uint64_t i = t; i < ne; i += stride) xlog[1 + i] = bp->errlog[i] + shard_lo;  // (row field, below 2^32)
    if (t == 0) {
        xlog[0] = ne;
        const unsigned long long st = bp->hdr->status | (cnt > (unsigned long long)kErrLogCap ? kDevStatusCapacity : 0);
        for (int k = 0; k < 4; ++k) xflag[k] = (long long)((st >> k) & 1ull);
    }
}

// Import (start of a batch's final half): the combined group tables, the
// status flags, and the gathered error logs of `world` engines (areas of
// 1 + kErrLogCap words: count, entries) concatenated in rank order -- which
// is row order, the pack kernel sorts them anyway.
__global__ void sj_import_kernel(const SjBatch* __restrict__ bp, const long long* xsum, const long long* xfirst,
                                 const long long* xflag, const unsigned long long* glog, int world) {
    __shared__ uint64_t s_off[65];
    const uint64_t n = bp->gtotal;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    for (uint64_t i = t; i < n; i += stride) {
        bp->sums[i] = (unsigned long long)xsum[i];
        const long long f = xfirst[i];
        bp->firsts[i] = f == LLONG_MAX ? kNoRow : (uint32_t)f;
    }
    const uint64_t area = 1 + (uint64_t)kErrLogCap;
    if (threadIdx.x == 0) {
        uint64_t run = 0;
        for (int r = 0; r < world; ++r) {
            s_off[r] = run;
            run += glog[(uint64_t)r * area];
        }
        s_off[world] = run;
    }
    __syncthreads();
    const uint64_t total = s_off[world];
    for (int r = 0; r < world; ++r) {
        const uint64_t c = glog[(uint64_t)r * area];
        for (uint64_t j = t; j < c; j += stride) {
            const uint64_t at = s_off[r] + j;
            if (at < (uint64_t)kErrLogCap) bp->errlog[at] = glog[(uint64_t)r * area + 1 + j];
        }
    }
    if (t == 0) {
        unsigned long long st = 0;
        for (int k = 0; k < 4; ++k)
            if (xflag[k]) st |= 1ull << k;
        if (total > (uint64_t)kErrLogCap) st |= kDevStatusCapacity;
        bp->hdr->status |= st;
        bp->hdr->errcnt = total < (uint64_t)kErrLogCap ? total : (uint64_t)kErrLogCap;
    }
}

// Per-batch device area of a slot: [batch | queries | accept descriptors] is
// uploaded from the slot's pinned staging; the rest is written on the device.
struct SjLayout {
    size_t batch, q, aq, rank, rep, facc, fpr, ixrank, upload, hdr, acc, acode, errlog, packed, total;
};

inline uint32_t bit_length(uint64_t v) {
    uint32_t b = 0;
    while (b < 64 && (v >> b)) ++b;
    return b;
}

// Layout and AN code of the packed join index for two slots whose key
// ranges are krange[s] and whose dimensions have nrec[s] distinct records:
// payload = id 1 | id 2 << s1 | (o1 + r0 * o2) << ib, ids bit_length(nrec)
// wide (ids 1..nrec, 0: no row has the key), o = the key offset clamped to
// its range, r0 = range 1 + 1; bits = the payload's width.  A: the first of
// the reference's AN code As (resint, resshort, restiny lists), else the
// largest odd A, with bits + bits of A <= 64 under which every flip of one or
// two bits of the word is detected.  A word w = p * A (p < 2^bits) with bits
// i and j flipped differs from w by +-2^i +- 2^j, a multiple of A only when
// 2^|i - j| = +-1 mod A (A is odd); and a word that is no multiple of A
// decodes to w * A^-1 mod 2^64 >= 2^bits, since A * 2^bits <= 2^64.
struct SjIxPacking {
    uint64_t A = 0, ainv = 0, lim = 0;
    uint32_t ib = 0, m0 = 0, s1 = 0, m1 = 0, r0 = 0, kr[2] = {}, bits = 0;
};

// Whether A detects every flip of one or two bits of a w-bit word.
inline bool ix_detects_two_flips(uint64_t A, uint32_t w) {
    if (A < 3 || !(A & 1)) return false;
    uint64_t r = 1;
    for (uint32_t j = 1; j < w; ++j) {
        r = r * 2 % A;
        if (r == 1 || r == A - 1) return false;
    }
    return true;
}

bool sj_ix_packing(const uint64_t krange[2], const uint64_t nrec[2], SjIxPacking* out) {
    uint32_t ib[2];
    for (int s = 0; s < 2; ++s) {
        if (!krange[s] || krange[s] >= 0xffffffffull) return false;  // offsets are 32-bit differences
        ib[s] = bit_length(nrec[s]) ? bit_length(nrec[s]) : 1u;
        if (ib[s] > (uint32_t)kAccBits) return false;  // ids index a [kAccEntries] table
    }
    SjIxPacking P;
    P.m0 = (1u << ib[0]) - 1u;
    P.s1 = ib[0];
    P.m1 = (1u << ib[1]) - 1u;
    P.ib = ib[0] + ib[1];
    P.r0 = (uint32_t)(krange[0] + 1);
    P.kr[0] = (uint32_t)krange[0];
    P.kr[1] = (uint32_t)krange[1];
    const uint64_t kmax = (uint64_t)krange[0] + (uint64_t)P.r0 * krange[1];  // both offsets clamped
    P.bits = P.ib + bit_length(kmax);
    if (P.bits > 61) return false;
    P.lim = 1ull << P.bits;
    uint64_t pick = 0;
    static const uint64_t kAs[] = {65117, 16089, 7785, 881, 463, 233, 125, 61, 29};
    for (const uint64_t A : kAs)
        if (!pick && P.bits + bit_length(A) <= 64 && ix_detects_two_flips(A, P.bits + bit_length(A))) pick = A;
    const uint32_t abits = 64 - P.bits < 16 ? 64 - P.bits : 16;
    for (uint64_t A = (1ull << abits) - 1; !pick && A >= 3; A -= 2)
        if (ix_detects_two_flips(A, P.bits + bit_length(A))) pick = A;
    if (!pick) return false;
    P.A = pick;
    P.ainv = inv_pow2(pick, 64);
    *out = P;
    return true;
}

SjLayout sj_layout() {
    SjLayout L;
    size_t off = 0;
    auto take = [&](size_t b) {
        size_t o = off;
        off = (off + b + 255) & ~size_t(255);
        return o;
    };
    L.batch = take(sizeof(SjBatch));
    L.q = take(sizeof(SjQDev) * kMaxQ);
    L.aq = take(sizeof(AcceptQ) * kMaxQ * 4);
    L.rank = take(2ull * 4 * kAccEntries);
    L.rep = take(2ull * 4 * kAccEntries);
    L.facc = take(8ull * 2 * 256);
    L.fpr = take(sizeof(RangePred) * 2 * kMaxQ);
    L.ixrank = take(2ull * 2 * kAccEntries);
    L.upload = off;
    L.hdr = take(sizeof(SjHdr));
    L.acc = take(8ull * 4 * kAccEntries);
    L.acode = take(8ull * 4 * kAccEntries);
    L.errlog = take(8ull * kErrLogCap);
    L.packed = take(8ull * kPackedWords);
    L.total = off;
    return L;
}

}  // namespace

// ------------------------------------------------------------------ engine
struct SjSlot {
    char* dev = nullptr;                     // device area (SjLayout)
    char* h_up = nullptr;                    // pinned upload staging [0, L.upload)
    SjHdr* h_hdr = nullptr;                  // pinned header copy
    unsigned long long* h_packed = nullptr;  // pinned packed result copy
    cudaEvent_t e0 = nullptr, e1 = nullptr;  // around the batch's kernels
    cudaEvent_t f0 = nullptr, f1 = nullptr;  // around the fact kernel (graph event nodes)
    cudaEvent_t hdr_done = nullptr;          // the header read-back finished (copy stream)
    cudaStream_t copy = nullptr;             // this slot's result read-back, overlapping the other slot's batch
    cudaGraphExec_t graph = nullptr;
    cudaGraph_t gsrc = nullptr;                   // the captured graph `graph` was made from
    cudaGraphNode_t cube_node[2] = {};            // its cube-scan nodes (phase 0, 1)
    cudaKernelNodeParams cube_kp[2] = {};
    bool busy = false;
    uint64_t ticket = 0;
    // what collection needs from the plan
    int nq = 0;
    int ok[kMaxQ] = {};
    int ngroup[kMaxQ] = {};
    unsigned long long first[4] = {};
    uint64_t nmax = 0;
    uint32_t strategy = 0;
    int cube_variant = 0;
    // fact-sharded batches: the exchange area and whether the final half is still to come
    long long* xsum = nullptr;
    long long* xfirst = nullptr;
    long long* xflag = nullptr;
    unsigned long long* xlog = nullptr;
    size_t xcap = 0;  // groups the area holds
    bool local_pending = false;
    bool graph_local = false;  // the captured graph is a local half (up to the export)
};

// Release a slot's captured graph (it is captured again on its next use).
inline void sj_drop_graph(SjSlot& S) {
    if (S.graph) cudaGraphExecDestroy(S.graph);
    if (S.gsrc) cudaGraphDestroy(S.gsrc);
    S.graph = nullptr;
    S.gsrc = nullptr;
    S.cube_node[0] = S.cube_node[1] = nullptr;
}

struct ahead_sj_engine {
    ahead_ctx* ctx = nullptr;
    ahead_sj_schema sch{};
    struct Dim {
        uint64_t kmin = 0, krange = 0;
        bool usable = false;  // keys clean, unique, mappable
        uint32_t* rec = nullptr;     // [krange] key records
        void* code = nullptr;        // [krange] per-batch dimension codes (cube strategy), 1 or 2 bytes each
        uint8_t* present = nullptr;  // [2^bits] packed values some row has
        std::vector<uint32_t> present_vals;  // the same, on the host (for the cube's dimension codes)
        uint64_t amin[AHEAD_SJ_MAXATTR] = {}, amax[AHEAD_SJ_MAXATTR] = {}, abad[AHEAD_SJ_MAXATTR] = {};
        SjDimPack pack{};  // which attributes are packed (clean, within kAccBits), and where
        uint32_t ixslot = 0;  // join index slot (1, 2; 0: not indexed)
        uint32_t* aval[AHEAD_SJ_MAXATTR] = {};  // row mode: clean attributes by key offset
        unsigned long long* accr = nullptr;      // row mode: a batch's accept masks by key offset
    } dim[4];
    // join index (null: none): ixfmt 1: slot 1 [fact_rows], then slot 2
    // [fact_rows]; ixfmt 2: one packed word per row (layout ixp)
    // the prefilter's row list (per-row batches; allocated with the engine for
    // fact tables of at least 2^20 rows, shared by the slots)
    uint32_t* flist = nullptr;
    uint64_t flist_cap = 0;
    uint32_t* pfmap = nullptr;  // the first-join prefilter's accepted keys, one bit a key (the largest dimension)
    unsigned long long* fidx = nullptr;
    int ixfmt = 0;
    SjIxPacking ixp{};
    // fact-sharded: the columns are rows [shard_lo, shard_lo + fact_rows) of a table of table_rows rows
    bool sharded = false;
    uint64_t shard_lo = 0, table_rows = 0;
    bool vec_ok = false;  // fact columns aligned for the indexed scans' pair loads (16 B; discount 4 B)
    unsigned long long* sums = nullptr;  // dense group tables, shared by the slots (stream-ordered)
    uint32_t* firsts = nullptr;
    unsigned long long* lists = nullptr;      // finalize: present groups per dense slot range
    unsigned long long* lists_tmp = nullptr;  // radix-sort scratch
    size_t gcap = 0;
    SjSlot slot[kSlots];
    uint64_t next_ticket = 0;
    float last_ms = 0.f;
    ahead_sj_stats stats{};
    int variant = 1;  // fact-kernel shape (kSjFact / kSjVarBlocks)
    int strategy = -1;  // -1: chosen per batch; else kStratRows / kStratCube when the batch allows it
    int cube_variant = 0;  // cube-scan shape (kCubeShapes)
    uint64_t cube_split = 0;  // rows of the cube scan's first phase; 0: kR0PerSig per signature
    unsigned long long* cube = nullptr;  // signature cube, shared by the slots (stream-ordered)
    uint32_t* cfirst = nullptr;
    uint32_t* exc = nullptr;
    uint32_t* unseen = nullptr;  // [kUnseenSlots]
    size_t cube_cap = 0, sig_cap = 0;
};

namespace {

// The buffers the batches share (stream-ordered).  Growing one waits for the
// device and frees, which stalls a pipelined caller, so sj_prepare sizes them
// for every batch the schema allows and these only grow past unusual bounds.
int sj_reserve_groups(ahead_sj_engine* e, uint64_t gtotal) {
    if (e->sums && gtotal <= e->gcap) return AHEAD_OK;
    cudaStreamSynchronize(e->ctx->stream);
    for (unsigned long long** p : {&e->sums, &e->lists, &e->lists_tmp})
        if (*p) cudaFree(*p), *p = nullptr;
    if (e->firsts) cudaFree(e->firsts), e->firsts = nullptr;
    static_assert((1u << 16) >= (unsigned)kErrLogCap, "lists_tmp is the error-log sort's scratch too");
    const size_t cap = gtotal < (1u << 16) ? (1u << 16) : gtotal + gtotal / 4;
    if (cudaMalloc(&e->sums, cap * 8) != cudaSuccess) return AHEAD_NO_MEMORY;
    if (cudaMalloc(&e->firsts, cap * 4) != cudaSuccess) return AHEAD_NO_MEMORY;
    if (cudaMalloc(&e->lists, cap * 8) != cudaSuccess) return AHEAD_NO_MEMORY;
    if (cudaMalloc(&e->lists_tmp, cap * 8) != cudaSuccess) return AHEAD_NO_MEMORY;
    e->gcap = cap;
    return AHEAD_OK;
}

int sj_reserve_cube(ahead_sj_engine* e, size_t cube_words, size_t nsig) {
    if (e->cube && cube_words <= e->cube_cap && nsig <= e->sig_cap) return AHEAD_OK;
    cudaStreamSynchronize(e->ctx->stream);
    if (e->cube) cudaFree(e->cube), e->cube = nullptr;
    if (e->cfirst) cudaFree(e->cfirst), e->cfirst = nullptr;
    const size_t cc = cube_words + cube_words / 4 + 1024, sc = nsig + nsig / 4 + 1024;
    if (cudaMalloc(&e->cube, cc * 8) != cudaSuccess) return AHEAD_NO_MEMORY;
    if (cudaMalloc(&e->cfirst, sc * 4) != cudaSuccess) return AHEAD_NO_MEMORY;
    e->cube_cap = cc;
    e->sig_cap = sc;
    return AHEAD_OK;
}

// The join index: the two usable dimensions with the largest key ranges
// (records are below 2^13: kAccBits packed bits + 1).  format: -1 the packed
// word when its fields fit (else two words), 0 none, 1 two words per row, 2
// packed (AHEAD_UNSUPPORTED when its fields do not fit).  Without the device
// memory for it (8 or 16 bytes per fact row) the engine runs without one.
int sj_build_index(ahead_sj_engine* e, int format) {
    const uint64_t n = e->sch.fact_rows;
    if (e->fidx) {
        cudaStreamSynchronize(e->ctx->stream);
        cudaFree(e->fidx);
        e->fidx = nullptr;
    }
    e->ixfmt = 0;
    e->ixp = SjIxPacking{};
    for (auto& X : e->dim) X.ixslot = 0;
    if (format == 0) return AHEAD_OK;
    int order[4] = {0, 1, 2, 3};
    std::stable_sort(order, order + 4, [&](int x, int y) { return e->dim[x].krange > e->dim[y].krange; });
    SjIdxBuild ib{};
    int sdim[kIxSlots] = {-1, -1};
    for (int d : order) {
        auto& X = e->dim[d];
        if (ib.nslots == kIxSlots || !X.usable || !e->sch.fk[d].data) continue;
        X.ixslot = (uint32_t)(ib.nslots + 1);
        sdim[ib.nslots] = d;
        ib.fk[ib.nslots] = (const unsigned long long*)e->sch.fk[d].data;
        ib.rec[ib.nslots] = X.rec;
        ib.ainv[ib.nslots] = e->sch.fk[d].Ainv;
        ib.kmin[ib.nslots] = X.kmin;
        ib.krange[ib.nslots] = X.krange;
        ib.nslots++;
    }
    SjIxPacking P;
    bool packed = false;
    if (format != 1 && ib.nslots == kIxSlots) {
        const uint64_t nrec[2] = {e->dim[sdim[0]].present_vals.size(), e->dim[sdim[1]].present_vals.size()};
        packed = sj_ix_packing(ib.krange, nrec, &P);
    }
    if (format == 2 && !packed) {
        for (auto& X : e->dim) X.ixslot = 0;
        return fail(e->ctx, AHEAD_UNSUPPORTED, "star join: the packed join index does not fit 64 bits");
    }
    if (!ib.nslots || !n) return AHEAD_OK;
    const uint64_t words = packed ? n : n * 2;
    if (cudaMalloc(&e->fidx, words * sizeof(unsigned long long)) != cudaSuccess) {
        cudaGetLastError();  // (not sticky) the engine runs without the index
        e->fidx = nullptr;
        for (auto& X : e->dim) X.ixslot = 0;
        return AHEAD_OK;
    }
    uint16_t* idmap = nullptr;
    if (packed) {
        // record -> dense id: the i-th present packed value v (record v + 1) is id i + 1
        std::vector<uint16_t> h((size_t)kIxSlots * kAccEntries, 0);
        for (int s = 0; s < kIxSlots; ++s) {
            const auto& pv = e->dim[sdim[s]].present_vals;
            for (size_t i = 0; i < pv.size(); ++i) h[(size_t)s * kAccEntries + pv[i] + 1] = (uint16_t)(i + 1);
        }
        if (cudaMalloc(&idmap, h.size() * 2) != cudaSuccess) {
            cudaGetLastError();
            cudaFree(e->fidx);
            e->fidx = nullptr;
            for (auto& X : e->dim) X.ixslot = 0;
            return AHEAD_OK;
        }
        cudaMemcpyAsync(idmap, h.data(), h.size() * 2, cudaMemcpyHostToDevice, e->ctx->stream);
        ib.packed = 1;
        ib.A = P.A;
        ib.ib = P.ib;
        ib.s1 = P.s1;
        ib.r0 = P.r0;
        ib.kr[0] = P.kr[0];
        ib.kr[1] = P.kr[1];
        ib.idmap[0] = idmap;
        ib.idmap[1] = idmap + kAccEntries;
    }
    sj_index_kernel<<<e->ctx->num_sms * 8, 256, 0, e->ctx->stream>>>(ib, n, e->fidx, packed ? nullptr : e->fidx + n);
    e->ctx->launches++;
    const cudaError_t ce = cudaStreamSynchronize(e->ctx->stream);
    if (idmap) cudaFree(idmap);
    e->ixfmt = packed ? 2 : 1;
    e->ixp = P;
    return ce == cudaSuccess ? AHEAD_OK : AHEAD_CUDA_ERROR;
}

// Whether cube shape cs can read the engine's index format (a shape reading
// the other format runs its lookups instead).
inline bool sj_shape_fits(const CubeShape& cs, int ixfmt) {
    return !cs.idx || cs.nslot == 0 || (cs.nslot == kIxPacked) == (ixfmt == 2);
}

int sj_prepare(ahead_sj_engine* e) {
    ahead_ctx* ctx = e->ctx;
    cudaStream_t st = ctx->stream;
    unsigned long long* mm = nullptr;
    if (cudaMalloc(&mm, 64 * sizeof(unsigned long long)) != cudaSuccess) return AHEAD_NO_MEMORY;
    for (int d = 0; d < 4; ++d) {
        const ahead_sj_dim& D = e->sch.dim[d];
        if (!D.rows || !D.key.data) continue;
        auto& X = e->dim[d];
        unsigned long long h[3] = {~0ull, 0, 0};
        cudaMemcpyAsync(mm, h, sizeof h, cudaMemcpyHostToDevice, st);
        sj_keyrange_kernel<<<grid_for(D.rows, 256), 256, 0, st>>>((const unsigned long long*)D.key.data, D.rows,
                                                                  D.key.Ainv, mm);
        cudaMemcpyAsync(h, mm, sizeof h, cudaMemcpyDeviceToHost, st);
        cudaStreamSynchronize(st);
        ctx->launches++;
        X.usable = false;
        if (!(h[2] == 0 && h[0] <= h[1] && (h[1] - h[0]) < (1ull << 28))) continue;
        X.kmin = h[0];
        X.krange = h[1] - h[0] + 1;
        // duplicate keys: a key map built once, then dropped
        uint32_t* kmap = nullptr;
        if (cudaMalloc(&kmap, X.krange * 4) != cudaSuccess) return AHEAD_NO_MEMORY;
        cudaMemsetAsync(kmap, 0, X.krange * 4, st);
        cudaMemsetAsync(mm, 0, 8, st);
        sj_kmap_kernel<<<grid_for(D.rows, 256), 256, 0, st>>>((const unsigned long long*)D.key.data, D.rows,
                                                              D.key.Ainv, X.kmin, kmap, mm);
        unsigned long long dup = 0;
        cudaMemcpyAsync(&dup, mm, 8, cudaMemcpyDeviceToHost, st);
        cudaStreamSynchronize(st);
        cudaFree(kmap);
        ctx->launches++;
        if (dup) continue;
        // attribute ranges; clean attributes are packed into the records
        uint64_t ainv[4] = {0, 0, 0, 0};
        SjDimPack& P = X.pack;
        P = SjDimPack{};
        uint32_t used_bits = 0;
        for (int a = 0; a < D.nattr; ++a) {
            const ahead_col& c = D.attr[a];
            const int w = type_width(c.type);
            unsigned long long g[3] = {~0ull, 0, 0};
            cudaMemcpyAsync(mm, g, sizeof g, cudaMemcpyHostToDevice, st);
            sj_attr_kernel<<<grid_for(D.rows, 256), 256, 0, st>>>(c.data, w, D.rows, c.Ainv & wmask(w),
                                                                  c.unenc_max & wmask(w), mm);
            cudaMemcpyAsync(g, mm, sizeof g, cudaMemcpyDeviceToHost, st);
            cudaStreamSynchronize(st);
            ctx->launches++;
            X.amin[a] = g[0];
            X.amax[a] = g[1];
            X.abad[a] = g[2];
            ainv[a] = c.Ainv & wmask(w);
            P.A[a] = c.A;
            P.wm[a] = wmask(w);
            P.amin[a] = g[0];
            if (g[2] || g[0] > g[1]) continue;
            uint32_t bits = 1;
            while (bits < 32 && ((g[1] - g[0]) >> bits)) ++bits;
            if (used_bits + bits > (uint32_t)kAccBits) continue;
            P.shift[a] = used_bits;
            P.pmask[a] = (1u << bits) - 1u;
            P.packed[a] = 1;
            used_bits += bits;
        }
        P.bits = used_bits;
        if (cudaMalloc(&X.rec, X.krange * 4) != cudaSuccess) return AHEAD_NO_MEMORY;
        // 2 bytes per key (either code width) and a word of slack for the 8-byte copy into shared memory
        if (cudaMalloc(&X.code, X.krange * 2 + 16) != cudaSuccess) return AHEAD_NO_MEMORY;
        if (cudaMalloc(&X.present, (size_t)1 << used_bits) != cudaSuccess) return AHEAD_NO_MEMORY;
        cudaMemsetAsync(X.rec, 0, X.krange * 4, st);
        cudaMemsetAsync(X.present, 0, (size_t)1 << used_bits, st);
        P.present = X.present;
        SjDimStatic S{};
        S.key = (const unsigned long long*)D.key.data;
        S.nattr = D.nattr;
        for (int a = 0; a < D.nattr; ++a) {
            S.attr[a] = D.attr[a].data;
            S.w[a] = type_width(D.attr[a].type);
        }
        S.key_ainv = D.key.Ainv;
        S.kmin = X.kmin;
        S.rec = X.rec;
        S.present = X.present;
        sj_pack_attrs_kernel<<<grid_for(D.rows, 256), 256, 0, st>>>(S, P, D.rows, ainv[0], ainv[1], ainv[2], ainv[3]);
        ctx->launches++;
        // row mode: every clean attribute by key offset, and the accept masks' buffer
        for (int a = 0; a < D.nattr; ++a) {
            if (X.abad[a] || X.amin[a] > X.amax[a]) continue;
            if (cudaMalloc(&X.aval[a], X.krange * 4) != cudaSuccess) return AHEAD_NO_MEMORY;
            cudaMemsetAsync(X.aval[a], 0, X.krange * 4, st);
            sj_aval_kernel<<<grid_for(D.rows, 256), 256, 0, st>>>(S, D.rows, a, ainv[a], X.amin[a], X.aval[a]);
            ctx->launches++;
            P.aval[a] = X.aval[a];
        }
        if (cudaMalloc(&X.accr, X.krange * 8) != cudaSuccess) return AHEAD_NO_MEMORY;
        P.rec = X.rec;
        P.krange = X.krange;
        std::vector<uint8_t> pres((size_t)1 << used_bits);
        cudaMemcpyAsync(pres.data(), X.present, pres.size(), cudaMemcpyDeviceToHost, st);
        cudaStreamSynchronize(st);
        X.present_vals.clear();
        for (uint32_t v = 0; v < pres.size(); ++v)
            if (pres[v]) X.present_vals.push_back(v);
        X.usable = true;
    }
    cudaStreamSynchronize(st);
    cudaFree(mm);
    const SjLayout L = sj_layout();
    for (auto& S : e->slot) {
        if (cudaMalloc(&S.dev, L.total) != cudaSuccess) return AHEAD_NO_MEMORY;
        if (cudaMallocHost(&S.h_up, L.upload) != cudaSuccess) return AHEAD_NO_MEMORY;
        if (cudaMallocHost(&S.h_hdr, sizeof(SjHdr)) != cudaSuccess) return AHEAD_NO_MEMORY;
        if (cudaMallocHost(&S.h_packed, kPackedWords * 8) != cudaSuccess) return AHEAD_NO_MEMORY;
        cudaEventCreate(&S.e0);
        cudaEventCreate(&S.e1);
        cudaEventCreate(&S.f0);
        cudaEventCreate(&S.f1);
        cudaEventCreateWithFlags(&S.hdr_done, cudaEventDisableTiming);
    }
    for (int v = 0; v < kSjVariants; ++v)
        if (cudaFuncSetAttribute(kSjFact[v], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFactSmem) !=
            cudaSuccess)
            return AHEAD_CUDA_ERROR;
    if (cudaFuncSetAttribute(sj_contract_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFactSmem) !=
        cudaSuccess)
        return AHEAD_CUDA_ERROR;
    if (cudaFuncSetAttribute(sj_pack_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(kPackSmem * 8)) !=
        cudaSuccess)
        return AHEAD_CUDA_ERROR;
    if (cudaMalloc(&e->exc, (size_t)kExcCap * 4) != cudaSuccess) return AHEAD_NO_MEMORY;
    if (cudaMalloc(&e->unseen, (size_t)kUnseenSlots * 4) != cudaSuccess) return AHEAD_NO_MEMORY;
    // the shared batch buffers at the sizes the schema bounds: signatures are
    // at most the product of (1 + distinct records) over the dimensions, a
    // query's dense group domain at most the product of the three largest
    // attribute domains (64 queries a batch; up to 4M slots reserved now)
    {
        uint64_t nsig = 1;
        std::vector<uint64_t> doms;
        for (int d = 0; d < 4; ++d) {
            const auto& X = e->dim[d];
            if (!X.usable) continue;
            nsig *= 1 + X.present_vals.size();
            if (nsig > kMaxSig) nsig = kMaxSig;
            for (int a = 0; a < e->sch.dim[d].nattr; ++a)
                if (X.amax[a] >= X.amin[a]) doms.push_back(X.amax[a] - X.amin[a] + 1);
        }
        std::sort(doms.rbegin(), doms.rend());
        uint64_t g = 1;
        for (size_t k = 0; k < doms.size() && k < 3; ++k) g = g * doms[k] > kMaxDense ? kMaxDense : g * doms[k];
        const uint64_t gtot = (uint64_t)kMaxQ * g < (4ull << 20) ? (uint64_t)kMaxQ * g : (4ull << 20);
        int rc = sj_reserve_cube(e, (size_t)kMaxSeg * nsig, nsig);
        if (!rc) rc = sj_reserve_groups(e, gtot);
        if (rc) return rc;
    }
    for (auto& S : e->slot)
        if (cudaStreamCreateWithFlags(&S.copy, cudaStreamNonBlocking) != cudaSuccess) return AHEAD_CUDA_ERROR;
    if (cudaGetLastError() != cudaSuccess) return AHEAD_CUDA_ERROR;
    {
        bool al = ((uintptr_t)e->sch.price.data & 15) == 0 && ((uintptr_t)e->sch.discount.data & 3) == 0;
        for (int d = 0; d < 4; ++d) al = al && ((uintptr_t)e->sch.fk[d].data & 15) == 0;
        e->vec_ok = al;
    }
    // the prefilter's row list (when the device memory is short, no prefilter)
    if (e->sch.fact_rows >= (1ull << 20)) {
        const uint64_t cap = std::min<uint64_t>(e->sch.fact_rows, kFlistMaxRows);
        if (cudaMalloc(&e->flist, cap * 4) == cudaSuccess) e->flist_cap = cap;
        else cudaGetLastError(), e->flist = nullptr;  // (not sticky)
        uint64_t words = 0;
        for (int d = 0; d < 4; ++d) words = std::max<uint64_t>(words, e->dim[d].krange / 32 + 1);
        if (e->flist && cudaMalloc(&e->pfmap, words * 4) != cudaSuccess) cudaGetLastError(), e->pfmap = nullptr;
    }
    const int rc = sj_build_index(e, -1);
    if (rc == AHEAD_OK && e->fidx && e->vec_ok)
        e->cube_variant = e->ixfmt == 2 ? kCubePackedDefault : kCubeIndexedDefault;
    return rc;
}

// The fused path needs the dimension's keys clean and unique and every
// attribute the query filters or groups on clean; an attribute outside the
// packed records sets *rowmode (the batch then joins the dimension in row
// mode, on the per-row strategy).
bool dim_usable_for(const ahead_sj_engine* e, const ahead_sj_query& q, int d, bool* rowmode) {
    const auto& X = e->dim[d];
    if (!X.usable) return false;
    auto attr_ok = [&](int a) {
        if (X.pack.packed[a]) return true;
        if (!X.aval[a]) return false;
        *rowmode = true;
        return true;
    };
    for (int j = 0; j < q.ngroup; ++j)
        if (q.gdim[j] == d && !attr_ok(q.gattr[j])) return false;
    for (int k = 0; k < q.npred; ++k)
        if (q.pred[k].dim == d && !attr_ok(q.pred[k].attr)) return false;
    return true;
}

// Build the batch descriptors in the slot's pinned staging.  Dense group
// slots go first to the queries with the smallest group domains (ungrouped
// queries take one slot), as many as the fact kernel keeps in shared memory.
int sj_plan(ahead_sj_engine* e, const ahead_sj_query* qs, int nq, SjSlot& S) {
    const ahead_sj_schema& sch = e->sch;
    const SjLayout L = sj_layout();
    std::memset(S.h_up, 0, L.upload);
    SjBatch& B = *reinterpret_cast<SjBatch*>(S.h_up + L.batch);
    SjQDev* QD = reinterpret_cast<SjQDev*>(S.h_up + L.q);
    AcceptQ* AQ = reinterpret_cast<AcceptQ*>(S.h_up + L.aq);
    unsigned long long joins[4] = {0, 0, 0, 0}, first[4] = {0, 0, 0, 0};
    unsigned long long fq[2] = {0, 0}, mrev = 0, mprof = 0;
    unsigned long long* facc = reinterpret_cast<unsigned long long*>(S.h_up + L.facc);
    RangePred* fpr = reinterpret_cast<RangePred*>(S.h_up + L.fpr);
    uint64_t nmax = 0;
    bool rows_only = false;  // a program shape: the per-row strategy
    bool rowmode[4] = {false, false, false, false};
    S.nq = nq;
    for (int qi = 0; qi < nq; ++qi) {
        const ahead_sj_query& Q = qs[qi];
        if (Q.npred < 0 || Q.npred > 4 || Q.ngroup < 0 || Q.ngroup > 3) return AHEAD_BAD_ARG;
        int npd[4] = {0, 0, 0, 0};
        for (int k = 0; k < Q.npred; ++k) {
            const ahead_sj_pred& p = Q.pred[k];
            if (p.dim < 0 || p.dim > 3 || p.attr < 0 || p.attr >= sch.dim[p.dim].nattr) return AHEAD_BAD_ARG;
            if (++npd[p.dim] > 2) return AHEAD_BAD_ARG;
            for (int k2 = 0; k2 < k; ++k2)
                if (Q.pred[k2].dim == p.dim && Q.pred[k2].attr == p.attr) return AHEAD_BAD_ARG;
        }
        if (Q.measure < AHEAD_SJ_MEASURE_PRICE_DISCOUNT || Q.measure > AHEAD_SJ_MEASURE_PROFIT) return AHEAD_BAD_ARG;
        if (Q.measure != AHEAD_SJ_MEASURE_PRICE_DISCOUNT && (!Q.ngroup || !sch.revenue.data ||
                                                            (Q.measure == AHEAD_SJ_MEASURE_PROFIT && !sch.supplycost.data)))
            return AHEAD_BAD_ARG;
        if (Q.nfpred < 0 || Q.nfpred > 2) return AHEAD_BAD_ARG;
        for (int k = 0; k < Q.nfpred; ++k) {
            const int c = Q.fpred[k].col;
            if (!(c == AHEAD_SJ_COL_QUANTITY || c == AHEAD_SJ_COL_DISCOUNT)) return AHEAD_BAD_ARG;
            if (c == AHEAD_SJ_COL_QUANTITY && !sch.quantity.data) return AHEAD_BAD_ARG;
            if (k && Q.fpred[0].col == c) return AHEAD_BAD_ARG;
        }
        for (int j = 0; j < Q.ngroup; ++j)
            if (Q.gdim[j] < 0 || Q.gdim[j] > 3 || Q.gattr[j] < 0 || Q.gattr[j] >= sch.dim[Q.gdim[j]].nattr)
                return AHEAD_BAD_ARG;
        bool used[4] = {false, false, false, false};
        for (int k = 0; k < Q.npred; ++k) used[Q.pred[k].dim] = true;
        for (int j = 0; j < Q.ngroup; ++j) used[Q.gdim[j]] = true;
        if (!(used[0] || used[1] || used[2] || used[3])) return AHEAD_BAD_ARG;
        int ok = 1;
        bool rm[4] = {false, false, false, false};
        for (int d = 0; d < 4; ++d)
            if (used[d] && !dim_usable_for(e, Q, d, &rm[d])) ok = 0;
        for (int d = 0; ok && d < 4; ++d)
            if (rm[d]) rowmode[d] = rows_only = true;
        SjQDev& D = QD[qi];
        D.ngroup = Q.ngroup;
        uint64_t G = 1;
        for (int j = 0; ok && j < Q.ngroup; ++j) {
            const int d = Q.gdim[j], at = Q.gattr[j];
            const ahead_col& c = sch.dim[d].attr[at];
            const auto& X = e->dim[d];
            D.gdim[j] = d;
            D.gshift[j] = X.pack.shift[at];
            D.gpmask[j] = X.pack.pmask[at];
            D.glo[j] = X.amin[at];
            D.gstride[j] = G;
            G *= X.amax[at] - X.amin[at] + 1;
            D.gA[j] = c.A;
            D.gwm[j] = wmask(type_width(c.type));
            if (G > kMaxDense) ok = 0;
        }
        S.ok[qi] = ok;
        S.ngroup[qi] = Q.ngroup;
        if (!ok) continue;  // not evaluated here (nrows 0, no group slots); the caller falls back
        if (e->sharded) {  // the query's prefix of the whole table, within this engine's rows
            const uint64_t p = Q.fact_rows < e->table_rows ? Q.fact_rows : e->table_rows;
            const uint64_t loc = p > e->shard_lo ? p - e->shard_lo : 0;
            D.nrows = loc < sch.fact_rows ? loc : sch.fact_rows;
        } else {
            D.nrows = Q.fact_rows < sch.fact_rows ? Q.fact_rows : sch.fact_rows;
        }
        nmax = D.nrows > nmax ? D.nrows : nmax;
        D.gsize = Q.ngroup ? G : 1;
        if (Q.measure == AHEAD_SJ_MEASURE_REVENUE) mrev |= 1ull << qi;
        if (Q.measure == AHEAD_SJ_MEASURE_PROFIT) mprof |= 1ull << qi;
        for (int k = 0; k < Q.nfpred; ++k) {
            // accept masks by decoded value: selectAN compares the codes, and a
            // clean code of value v is v * A in the code width
            const ahead_sj_fpred& f = Q.fpred[k];
            const int c = f.col == AHEAD_SJ_COL_QUANTITY ? 0 : 1;
            const ahead_col& col = c ? sch.discount : sch.quantity;
            const RangePred rp = RangePred::make(f.op1, f.th1, f.op2, f.th2, f.comb, 0xffffull);
            fq[c] |= 1ull << qi;
            fpr[qi * 2 + c] = rp;
            for (uint64_t v = 0; v < 256; ++v)
                if (rp((v * col.A) & 0xffffull)) facc[c * 256 + v] |= 1ull << qi;
        }
        if (Q.nfpred || Q.measure != AHEAD_SJ_MEASURE_PRICE_DISCOUNT) rows_only = true;
        // a query with fact predicates fetches every foreign key positionally
        bool first_done = Q.nfpred > 0;
        for (int k = 0; k < 4; ++k) {
            const int d = join_dim(k);
            if (!used[d]) continue;
            joins[d] |= 1ull << qi;
            if (!first_done) {
                first[d] |= 1ull << qi;
                first_done = true;
            }
        }
        for (int k = 0; k < Q.npred; ++k) {
            const ahead_sj_pred& p = Q.pred[k];
            const ahead_col& c = sch.dim[p.dim].attr[p.attr];
            AcceptQ& a = AQ[p.dim * kMaxQ + qi];
            const RangePred rp = RangePred::make(p.op1, p.th1, p.op2, p.th2, p.comb, wmask(type_width(c.type)));
            if (!a.has_pred) {
                a.has_pred = 1;
                a.attr = p.attr;
                a.pred = rp;
            } else {  // a second predicate on the dimension: selections intersected
                a.has_pred2 = 1;
                a.attr2 = p.attr;
                a.pred2 = rp;
            }
        }
    }
    // row-mode dimensions: every query's group attributes there from the value tables
    for (int qi = 0; qi < nq; ++qi) {
        if (!S.ok[qi]) continue;
        for (int j = 0; j < qs[qi].ngroup; ++j)
            if (rowmode[qs[qi].gdim[j]]) QD[qi].gtab[j] = e->dim[qs[qi].gdim[j]].aval[qs[qi].gattr[j]];
    }
    // dense slots: smallest domains first, the leading ones in shared memory
    std::vector<int> order;
    for (int qi = 0; qi < nq; ++qi)
        if (S.ok[qi]) order.push_back(qi);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return QD[x].gsize < QD[y].gsize; });
    uint64_t gtotal = 0, nsm = 0;
    bool in_smem = true;
    for (int qi : order) {
        QD[qi].gbase = (uint32_t)gtotal;
        gtotal += QD[qi].gsize;
        if (in_smem && gtotal <= (uint64_t)kSmemGroups) nsm = gtotal;
        else in_smem = false;
    }
    for (int d = 0; d < 4; ++d) {
        B.dim[d].fk = (const unsigned long long*)sch.fk[d].data;
        B.dim[d].rec = e->dim[d].rec;
        B.dim[d].code = e->dim[d].code;
        B.dim[d].acc = reinterpret_cast<const unsigned long long*>(S.dev + L.acc) + (size_t)d * kAccEntries;
        B.dim[d].fk_ainv = sch.fk[d].Ainv;
        B.dim[d].kmin = e->dim[d].kmin;
        B.dim[d].krange = e->dim[d].krange;
        B.dim[d].joins = joins[d];
        B.dim[d].first = first[d];
        B.dim[d].ixslot = e->fidx ? e->dim[d].ixslot : 0;
        B.dim[d].accr = rowmode[d] ? e->dim[d].accr : nullptr;
        S.first[d] = first[d];
    }
    B.fidx1 = e->fidx;
    B.fidx2 = (e->fidx && e->ixfmt == 1) ? e->fidx + sch.fact_rows : nullptr;
    {
        const CubeShape& cs = kCubeShapes[e->cube_variant];
        B.idx_on = (e->fidx && cs.idx && sj_shape_fits(cs, e->ixfmt)) ? 1u : 0u;
        // a packed entry is checked against both indexed keys: the batch must read both
        if (cs.nslot == kIxPacked)
            for (int d = 0; d < 4; ++d)
                if (e->dim[d].ixslot && !joins[d]) B.idx_on = 0;
        B.ixpack = (B.idx_on && cs.nslot == kIxPacked) ? 1u : 0u;
        B.nslot = B.idx_on ? (B.ixpack ? (uint32_t)kIxSlots : (uint32_t)cs.nslot) : 0u;
        B.ixp_ainv = e->ixp.ainv;
        B.ixp_lim = e->ixp.lim;
        B.ixp_ib = e->ixp.ib;
        B.ixp_m0 = e->ixp.m0;
        B.ixp_s1 = e->ixp.s1;
        B.ixp_m1 = e->ixp.m1;
        B.ixp_r0 = e->ixp.r0;
        B.ixp_kr[0] = e->ixp.kr[0];
        B.ixp_kr[1] = e->ixp.kr[1];
    }
    B.price = (const unsigned long long*)sch.price.data;
    B.disc = (const uint16_t*)sch.discount.data;
    B.price_ainv = sch.price.Ainv;
    B.disc_ainv = sch.discount.Ainv & 0xffffull;
    B.qty = (const uint16_t*)sch.quantity.data;
    B.rev = (const unsigned long long*)sch.revenue.data;
    B.cost = (const unsigned long long*)sch.supplycost.data;
    B.qty_ainv = sch.quantity.Ainv & 0xffffull;
    B.rev_ainv = sch.revenue.Ainv;
    B.cost_ainv = sch.supplycost.Ainv;
    B.rev_umax = sch.revenue.unenc_max;
    B.cost_umax = sch.supplycost.unenc_max;
    B.facc = reinterpret_cast<const unsigned long long*>(S.dev + L.facc);
    B.fpr = reinterpret_cast<const RangePred*>(S.dev + L.fpr);
    B.fq[0] = fq[0];
    B.fq[1] = fq[1];
    B.mrev = mrev;
    B.mprof = mprof;
    B.nmax = nmax;
    B.gtotal = gtotal;
    B.nq = nq;
    B.nsm = (uint32_t)nsm;
    S.nmax = nmax;
    // strategy: the signature cube when the batch has enough queries, at
    // most kMaxSeg distinct prefixes and at most kMaxSig signatures
    B.strategy = kStratRows;
    B.nseg = 0;
    B.nsig = 0;
    B.r0 = 0;
    for (int d = 0; d < 4; ++d) B.radix[d] = 1;
    if (e->strategy != kStratRows && nmax && !rows_only &&
        (e->strategy == kStratCube || (int)order.size() >= kCubeMinQueries)) {
        std::vector<uint64_t> ends;
        for (int qi : order) ends.push_back(QD[qi].nrows);
        std::sort(ends.begin(), ends.end());
        ends.erase(std::unique(ends.begin(), ends.end()), ends.end());
        uint64_t nsig = 1;
        uint16_t* rank = reinterpret_cast<uint16_t*>(S.h_up + L.rank);
        uint16_t* rep = reinterpret_cast<uint16_t*>(S.h_up + L.rep);
        bool fits = ends.size() <= (size_t)kMaxSeg;
        for (int d = 0; d < 4 && fits; ++d) {
            if (!joins[d]) continue;
            // the attributes the batch filters or groups on in this dimension
            uint32_t pm = 0;
            const auto& X = e->dim[d];
            for (int qi : order) {
                const ahead_sj_query& Q = qs[qi];
                for (int k = 0; k < Q.npred; ++k)
                    if (Q.pred[k].dim == d) pm |= X.pack.pmask[Q.pred[k].attr] << X.pack.shift[Q.pred[k].attr];
                for (int j = 0; j < Q.ngroup; ++j)
                    if (Q.gdim[j] == d) pm |= X.pack.pmask[Q.gattr[j]] << X.pack.shift[Q.gattr[j]];
            }
            // dense codes of the distinct projections of the present records
            std::vector<uint32_t> proj;
            for (uint32_t v : X.present_vals) proj.push_back(v & pm);
            std::sort(proj.begin(), proj.end());
            proj.erase(std::unique(proj.begin(), proj.end()), proj.end());
            uint16_t* rk = rank + (size_t)d * kAccEntries;
            uint16_t* rp = rep + (size_t)d * kAccEntries;
            rk[0] = 0;  // record 0 (no row has the key): code 0, whose representative is record 0
            rp[0] = 0;
            for (uint32_t v : X.present_vals) {
                const uint32_t c = 1 + (uint32_t)(std::lower_bound(proj.begin(), proj.end(), v & pm) - proj.begin());
                rk[v + 1] = (uint16_t)c;
                rp[c] = (uint16_t)(v + 1);
            }
            if (B.ixpack && X.ixslot) {  // the packed index's ids: id i + 1 is present value i
                const uint32_t s = X.ixslot - 1;
                uint16_t* ir = reinterpret_cast<uint16_t*>(S.h_up + L.ixrank) + (size_t)s * kAccEntries;
                std::memset(ir, 0, ((size_t)(s ? B.ixp_m1 : B.ixp_m0) + 1) * 2);
                for (size_t i = 0; i < X.present_vals.size(); ++i) ir[i + 1] = rk[X.present_vals[i] + 1];
            }
            B.radix[d] = 1 + (uint32_t)proj.size();
            nsig *= B.radix[d];
            if (nsig > kMaxSig) fits = false;
        }
        if (fits) {
            // 1-byte codes where they fit; packed tables for the shapes that read them
            for (int d = 0; d < 4; ++d) {
                B.dim[d].cw = B.radix[d] <= 256 ? 1 : 2;
                B.dim[d].cbits = 0;
                B.dim[d].per = 1;
                B.dim[d].cmagic = 0;
                if (!kCubeShapes[e->cube_variant].pack || !joins[d]) continue;
                uint32_t cb = 1;
                while ((1u << cb) < B.radix[d]) ++cb;
                const uint32_t per = 64 / cb;
                B.dim[d].cbits = cb;
                B.dim[d].per = per;
                B.dim[d].cmagic = ((1ull << 40) + per - 1) / per;  // exact below 2^28 keys
            }
            B.strategy = kStratCube;
            B.nseg = (uint32_t)ends.size();
            B.nsig = (uint32_t)nsig;
            const uint64_t r0 = e->cube_split ? e->cube_split
                                              : (kR0PerSig * nsig + kR0Align - 1) / kR0Align * kR0Align;
            B.r0 = r0 < nmax ? r0 : nmax;
            for (size_t k = 0; k < ends.size(); ++k) B.seg_end[k] = ends[k];
            for (int k = 0; k < kMaxSeg; ++k) B.segq[k] = 0;
            for (int qi : order) {
                QD[qi].segs = 1 + (uint32_t)(std::lower_bound(ends.begin(), ends.end(), QD[qi].nrows) - ends.begin());
                for (uint32_t k = 0; k < QD[qi].segs && k < (uint32_t)kMaxSeg; ++k) B.segq[k] |= 1ull << qi;
            }
            const size_t need = (size_t)B.nseg * nsig;
            const int rc = sj_reserve_cube(e, need, nsig);
            if (rc) return rc;
        } else {
            for (int d = 0; d < 4; ++d) B.radix[d] = 1;
        }
    }
    B.cube = e->cube;
    B.cfirst = e->cfirst;
    B.exc = e->exc;
    B.unseen = e->unseen;
    B.acode = reinterpret_cast<unsigned long long*>(S.dev + L.acode);
    B.qmask = nq == 64 ? ~0ull : ((1ull << nq) - 1);
    for (int d = 0; d < 4; ++d) {
        B.rank[d] = reinterpret_cast<const uint16_t*>(S.dev + L.rank) + (size_t)d * kAccEntries;
        B.rep[d] = reinterpret_cast<const uint16_t*>(S.dev + L.rep) + (size_t)d * kAccEntries;
    }
    for (int s = 0; s < kIxSlots; ++s) {
        B.ixrank[s] = B.rank[0];
        if (B.ixpack) B.ixrank[s] = reinterpret_cast<const uint16_t*>(S.dev + L.ixrank) + (size_t)s * kAccEntries;
        else
            for (int d = 0; d < 4; ++d)
                if (e->dim[d].ixslot == (uint32_t)s + 1) B.ixrank[s] = B.rank[d];
    }
    // the indexed scan's fast path: every dimension joined, both index slots
    // built, byte (or packed) code tables for the dimensions the shape looks up
    // (positions nslot..3; the indexed ones first)
    B.fast = 0;
    if (B.strategy == kStratCube && B.idx_on) {
        int order[4], n = 0;
        for (uint32_t sl = 1; sl <= (uint32_t)kIxSlots; ++sl)
            for (int d = 0; d < 4; ++d)
                if (e->dim[d].ixslot == sl) order[n++] = d;
        bool ok = n == kIxSlots;
        for (int d = 0; d < 4; ++d)
            if (!e->dim[d].ixslot) order[n++] = d;
        for (int d = 0; d < 4; ++d) ok = ok && joins[d];
        const bool pack = kCubeShapes[e->cube_variant].pack;
        for (int p = (int)B.nslot; p < 4; ++p) ok = ok && (pack || B.dim[order[p]].cw == 1);  // looked up
        if (ok) {
            uint32_t stride[4], st = 1;
            for (int d = 3; d >= 0; --d) {
                stride[d] = st;
                st *= B.radix[d];
            }
            for (int p = 0; p < 4; ++p) {
                const int d = order[p];
                SjPos& P = B.pos[p];
                P.fk = B.dim[d].fk;
                P.code = B.dim[d].code;
                P.rank = p < (int)B.nslot ? B.ixrank[p] : B.rank[d];
                P.acode = reinterpret_cast<const unsigned long long*>(S.dev + L.acode) + (size_t)d * kAccEntries;
                P.ainv = B.dim[d].fk_ainv;
                P.cmagic = B.dim[d].cmagic;
                P.kmin = (uint32_t)B.dim[d].kmin;
                P.krange = (uint32_t)B.dim[d].krange;
                P.stride = stride[d];
                P.cbits = B.dim[d].cbits;
                P.per = B.dim[d].per;
            }
            B.fast = 1;
        }
    }
    // the prefilter: a per-row batch over at least 2^20 rows whose every query
    // selects on quantity or discount (1), or whose queries have no fact
    // predicate and all join one dimension first (2)
    B.flist = nullptr;
    B.flist_cap = 0;
    B.flist_on = 0;
    B.flist_dim = 0;
    B.pfmap = nullptr;
    if (B.strategy == kStratRows && nmax >= (1ull << 20) && !order.empty()) {
        bool all_fact = true, no_fact = true;
        unsigned long long om = 0;
        for (int qi : order) {
            const bool f = ((fq[0] | fq[1]) >> qi) & 1ull;
            all_fact = all_fact && f;
            no_fact = no_fact && !f;
            om |= 1ull << qi;
        }
        int mode = all_fact ? 1 : 0;
        for (int d = 0; d < 4 && !mode; ++d)
            if (no_fact && (first[d] & om) == om) {
                // the share of rows the first join keeps, summed over the queries:
                // per query the product over its predicates on d of the share of
                // the attribute's values (min..max, sampled beyond 2^16) it accepts
                double share = 0.0;
                for (int qi : order) {
                    double q = 1.0;
                    for (int k = 0; k < qs[qi].npred; ++k) {
                        const ahead_sj_pred& p = qs[qi].pred[k];
                        if (p.dim != d) continue;
                        const ahead_col& c = sch.dim[d].attr[p.attr];
                        const uint64_t wm = wmask(type_width(c.type));
                        const RangePred rp = RangePred::make(p.op1, p.th1, p.op2, p.th2, p.comb, wm);
                        const uint64_t lo = e->dim[d].amin[p.attr], hi = e->dim[d].amax[p.attr];
                        if (hi < lo) continue;
                        const uint64_t n = hi - lo + 1, step = n > (1u << 16) ? n / (1u << 16) : 1;
                        uint64_t hit = 0, seen = 0;
                        for (uint64_t v = lo; v <= hi && seen < (1u << 16); v += step, ++seen)
                            hit += rp((v * c.A) & wm) ? 1 : 0;
                        q *= seen ? (double)hit / (double)seen : 1.0;
                    }
                    share += q;
                }
                if (share <= kPrefilterMaxShare) {
                    mode = 2;
                    B.flist_dim = (uint32_t)d;
                }
                break;  // (one dimension is every query's first)
            }
        if (mode) {
            if (e->flist) {  // (allocated with the engine; without it every row is scanned)
                B.flist = e->flist;
                B.flist_cap = e->flist_cap;
                B.flist_on = (uint32_t)mode;
                if (mode == 2) B.pfmap = e->pfmap;
            }
        }
    }
    S.strategy = B.strategy;
    S.cube_variant = e->cube_variant;
    // group tables: shared by the slots (sized at set-up; growing waits for the device)
    {
        const int rc = sj_reserve_groups(e, gtotal);
        if (rc) return rc;
    }
    B.q = reinterpret_cast<const SjQDev*>(S.dev + L.q);
    B.sums = e->sums;
    B.firsts = e->firsts;
    B.hdr = reinterpret_cast<SjHdr*>(S.dev + L.hdr);
    B.errlog = reinterpret_cast<unsigned long long*>(S.dev + L.errlog);
    B.lists = e->lists;
    B.lists_tmp = e->lists_tmp;
    B.packed_cap = kPackedWords;
    B.packed = reinterpret_cast<unsigned long long*>(S.dev + L.packed);
    return AHEAD_OK;
}

// The kernels of one batch (captured once per slot, or launched directly);
// `local`: the local half of a fact-sharded batch, up to the export.
void sj_launch(ahead_sj_engine* e, SjSlot& S, bool capturing, bool local) {
    cudaStream_t st = e->ctx->stream;
    const SjLayout L = sj_layout();
    const SjBatch* bp = reinterpret_cast<const SjBatch*>(S.dev + L.batch);
    const AcceptQ* aq = reinterpret_cast<const AcceptQ*>(S.dev + L.aq);
    const int sms = e->ctx->num_sms;
    sj_clear_kernel<<<sms * 2, 256, 0, st>>>(bp);
    SjPackAll pk;
    for (int d = 0; d < 4; ++d) pk.d[d] = e->dim[d].pack;
    // (two blocks an SM for each dimension: a row-mode dimension's masks cover
    // its key range, millions of keys; 64 blocks a dimension took 0.1-0.6 ms)
    sj_accept_kernel<<<dim3(sms * 2, 4), 256, 0, st>>>(
        bp, aq, pk, reinterpret_cast<unsigned long long*>(S.dev + L.acc));
    int n = 2;
    // inside a capture the records become event nodes of the graph
    const unsigned int rf = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
    cudaEventRecordWithFlags(S.f0, st, rf);
    const int v = e->variant;
    sj_pfmap_kernel<<<sms * 2, 256, 0, st>>>(bp);
    sj_prefilter_kernel<<<sms * 3, kSjThreads, 0, st>>>(bp);  // (its launch bounds: three blocks an SM)
    kSjFact[v]<<<sms * kSjVarBlocks[v], kSjThreads, kFactSmem, st>>>(bp);
    // (wide grids: both kernels are chains of dependent loads per element)
    sj_code_kernel<<<dim3(sms * 8, 4), 256, 0, st>>>(bp);
    const int cv = e->cube_variant;
    // the cube scan takes the descriptor by value (a graph's copy is updated per batch)
    const SjBatch& hb = *reinterpret_cast<const SjBatch*>(S.h_up + L.batch);
    const CubeShape& cs = kCubeShapes[cv];
    cs.fn<<<sms * cs.blocks_per_sm, kSjThreads, 0, st>>>(hb, 0);
    sj_unseen_kernel<<<sms * 16, 256, 0, st>>>(bp);
    cs.fn<<<sms * cs.blocks_per_sm, kSjThreads, 0, st>>>(hb, 1);
    cudaEventRecordWithFlags(S.f1, st, rf);
    sj_exc_kernel<<<64, kSjThreads, 0, st>>>(bp);
    sj_contract_kernel<<<sms * 3, kSjThreads, kFactSmem, st>>>(bp);  // (3 blocks fit an SM: 62 KB of shared memory each)
    n += 9;
    if (local) {
        sj_export_kernel<<<sms * 2, 256, 0, st>>>(bp, S.xsum, S.xfirst, S.xflag, S.xlog, e->shard_lo);
        e->ctx->launches += n + 1;
        return;
    }
    sj_compact_kernel<<<sms * 2, 256, 0, st>>>(bp);
    sj_finalize_kernel<<<kMaxQ, 1024, 0, st>>>(bp);
    sj_pack_kernel<<<kMaxQ, 1024, kPackSmem * 8, st>>>(bp);
    sj_emit_kernel<<<dim3(8, kMaxQ), 256, 0, st>>>(bp);
    e->ctx->launches += n + 4;
}

int sj_finish_submit(ahead_sj_engine* e, SjSlot& S, uint64_t* ticket);

// The exchange area of a slot, for `groups` dense group slots (growing it
// waits for the device and drops the slot's graph, whose export node holds
// the old pointers).
int sj_reserve_xchg(ahead_sj_engine* e, SjSlot& S, uint64_t groups) {
    if (S.xlog && groups <= S.xcap) return AHEAD_OK;
    cudaStreamSynchronize(e->ctx->stream);
    sj_drop_graph(S);
    if (S.xsum) cudaFree(S.xsum), S.xsum = nullptr;
    if (S.xfirst) cudaFree(S.xfirst), S.xfirst = nullptr;
    const size_t cap = groups < e->gcap ? e->gcap : groups;
    if (cudaMalloc(&S.xsum, cap * 8) != cudaSuccess) return AHEAD_NO_MEMORY;
    if (cudaMalloc(&S.xfirst, cap * 8) != cudaSuccess) return AHEAD_NO_MEMORY;
    if (!S.xflag && cudaMalloc(&S.xflag, 4 * 8) != cudaSuccess) return AHEAD_NO_MEMORY;
    if (!S.xlog && cudaMalloc(&S.xlog, (1 + (size_t)kErrLogCap) * 8) != cudaSuccess) return AHEAD_NO_MEMORY;
    S.xcap = cap;
    return AHEAD_OK;
}

int sj_submit(ahead_sj_engine* e, const ahead_sj_query* qs, int nq, int use_graph, uint64_t* ticket,
              bool local = false) {
    if (!e || !qs || nq < 1 || nq > kMaxQ) return AHEAD_BAD_ARG;
    SjSlot& S = e->slot[e->next_ticket % kSlots];
    if (S.busy) return fail(e->ctx, AHEAD_CAPACITY, "star join: both slots hold unread batches");
    int rc = sj_plan(e, qs, nq, S);
    if (rc) return fail(e->ctx, rc, rc == AHEAD_NO_MEMORY ? "star join: device memory" : "star join: bad query");
    if (local) {
        rc = sj_reserve_xchg(e, S, reinterpret_cast<const SjBatch*>(S.h_up + sj_layout().batch)->gtotal);
        if (rc) return fail(e->ctx, rc, "star join: exchange area");
    }
    cudaStream_t st = e->ctx->stream;
    const SjLayout L = sj_layout();
    cudaMemcpyAsync(S.dev, S.h_up, L.upload, cudaMemcpyHostToDevice, st);
    if (use_graph && S.graph && S.graph_local != local) sj_drop_graph(S);  // captured for the other form
    if (use_graph && !S.graph) {
        S.graph_local = local;
        cudaGraph_t g;
        if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            return fail(e->ctx, AHEAD_CUDA_ERROR, "graph capture");
        sj_launch(e, S, true, local);
        if (cudaStreamEndCapture(st, &g) != cudaSuccess) return fail(e->ctx, AHEAD_CUDA_ERROR, "graph capture");
        // the cube-scan nodes, whose by-value descriptor each batch replaces
        size_t nn = 0;
        cudaGraphGetNodes(g, nullptr, &nn);
        std::vector<cudaGraphNode_t> nodes(nn);
        cudaGraphGetNodes(g, nodes.data(), &nn);
        int found = 0;
        for (cudaGraphNode_t nd : nodes) {
            cudaGraphNodeType t;
            cudaKernelNodeParams kp;
            if (cudaGraphNodeGetType(nd, &t) != cudaSuccess || t != cudaGraphNodeTypeKernel) continue;
            if (cudaGraphKernelNodeGetParams(nd, &kp) != cudaSuccess) continue;
            if (kp.func != reinterpret_cast<void*>(kCubeShapes[e->cube_variant].fn)) continue;
            const int ph = *static_cast<const int*>(kp.kernelParams[1]);
            if (ph < 0 || ph > 1 || S.cube_node[ph]) continue;
            S.cube_node[ph] = nd;
            S.cube_kp[ph] = kp;
            ++found;
        }
        const cudaError_t ie = found == 2 ? cudaGraphInstantiate(&S.graph, g, 0) : cudaErrorInvalidValue;
        if (ie != cudaSuccess) {
            cudaGraphDestroy(g);
            S.graph = nullptr;
            S.cube_node[0] = S.cube_node[1] = nullptr;
            return fail(e->ctx, AHEAD_CUDA_ERROR, "graph instantiate");
        }
        S.gsrc = g;
    }
    cudaEventRecord(S.e0, st);
    if (use_graph) {
        SjBatch* hb = reinterpret_cast<SjBatch*>(S.h_up + L.batch);
        for (int ph = 0; ph < 2; ++ph) {
            int phase = ph;
            void* args[2] = {hb, &phase};
            cudaKernelNodeParams kp = S.cube_kp[ph];
            kp.kernelParams = args;
            kp.extra = nullptr;
            const cudaError_t pe = cudaGraphExecKernelNodeSetParams(S.graph, S.cube_node[ph], &kp);
            if (pe != cudaSuccess) return cuda_fail(e->ctx, pe, "star join graph update");
        }
        cudaGraphLaunch(S.graph, st);
        e->ctx->launches += local ? 12 : 15;
    } else {
        sj_launch(e, S, false, local);
    }
    if (local) {  // the final half follows the exchange (sj_submit_final)
        const cudaError_t le = cudaGetLastError();
        if (le != cudaSuccess) return cuda_fail(e->ctx, le, "star join launch");
        S.busy = true;
        S.local_pending = true;
        S.ticket = e->next_ticket++;
        *ticket = S.ticket;
        return AHEAD_OK;
    }
    return sj_finish_submit(e, S, ticket);
}

// The tail of a batch's submission: the end event and the header read-back.
int sj_finish_submit(ahead_sj_engine* e, SjSlot& S, uint64_t* ticket) {
    cudaStream_t st = e->ctx->stream;
    const SjLayout L = sj_layout();
    cudaEventRecord(S.e1, st);
    // the header read-back overlaps the next batch on the copy stream
    cudaStreamWaitEvent(S.copy, S.e1, 0);
    cudaMemcpyAsync(S.h_hdr, S.dev + L.hdr, sizeof(SjHdr), cudaMemcpyDeviceToHost, S.copy);
    cudaEventRecord(S.hdr_done, S.copy);
    const cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) return cuda_fail(e->ctx, le, "star join launch");
    S.busy = true;
    if (S.local_pending) {
        S.local_pending = false;  // (ticket assigned by the local half)
    } else {
        S.ticket = e->next_ticket++;
    }
    *ticket = S.ticket;
    return AHEAD_OK;
}

// The final half of a fact-sharded batch, after the caller's exchange.
int sj_submit_final(ahead_sj_engine* e, uint64_t ticket, const uint64_t* glog, int world) {
    if (!e || !glog || world < 1 || world > 64) return AHEAD_BAD_ARG;
    SjSlot& S = e->slot[ticket % kSlots];
    if (!S.busy || S.ticket != ticket || !S.local_pending)
        return fail(e->ctx, AHEAD_BAD_ARG, "star join: no local half awaits this ticket");
    cudaStream_t st = e->ctx->stream;
    const SjLayout L = sj_layout();
    const SjBatch* bp = reinterpret_cast<const SjBatch*>(S.dev + L.batch);
    const int sms = e->ctx->num_sms;
    sj_import_kernel<<<sms * 2, 256, 0, st>>>(bp, S.xsum, S.xfirst, S.xflag,
                                               reinterpret_cast<const unsigned long long*>(glog), world);
    sj_compact_kernel<<<sms * 2, 256, 0, st>>>(bp);
    sj_finalize_kernel<<<kMaxQ, 1024, 0, st>>>(bp);
    sj_pack_kernel<<<kMaxQ, 1024, kPackSmem * 8, st>>>(bp);
    sj_emit_kernel<<<dim3(8, kMaxQ), 256, 0, st>>>(bp);
    e->ctx->launches += 5;
    uint64_t t = ticket;
    return sj_finish_submit(e, S, &t);
}

// One query's result from a collected slot (header and packed area on the host).
void sj_fill(const SjSlot& S, int qi, ahead_sj_result& R) {
    const SjHdr& H = *S.h_hdr;
    for (int c = 0; c < AHEAD_SJ_NCOL; ++c) {
        R.fact_err[c].count = 0;
        R.fact_err[c].present = 1;
    }
    R.ngroups = 0;
    R.total = 0;
    const int G = S.ngroup[qi];
    R.status = (!S.ok[qi] || (H.status & kDevStatusCapacity)) ? AHEAD_UNSUPPORTED : AHEAD_OK;
    if (G && H.ngroups[qi] == ~0ull) R.status = AHEAD_UNSUPPORTED;
    if (R.status != AHEAD_OK) return;
    // the first join probed nothing if its build side was empty
    int skip = -1;
    for (int d = 0; d < 4; ++d)
        if (((S.first[d] >> qi) & 1ull) && !((H.nonempty[d] >> qi) & 1ull)) skip = d;
    // errors: sorted by (query, column, row); this query's run starts at its key prefix
    const unsigned long long* P = S.h_packed;
    const unsigned long long lo = (unsigned long long)qi << 58;
    uint64_t i = std::lower_bound(P, P + H.nerr, lo) - P;
    for (; i < H.nerr && (int)(P[i] >> 58) == qi; ++i) {
        const int c = (int)((P[i] >> kLogColShift) & 15);
        if (c == skip || c >= AHEAD_SJ_NCOL) continue;
        ahead_errvec& E = R.fact_err[c];
        if (E.count < E.capacity && E.data) E.data[E.count] = (P[i] & ((1ull << kLogColShift) - 1)) * 16089ull;
        E.count++;
    }
    for (int c = 0; c < AHEAD_SJ_NCOL; ++c)
        if (R.fact_err[c].count > R.fact_err[c].capacity) R.status = AHEAD_CAPACITY;
    if (!G) {
        R.total = H.raw[qi] * kResoidAMax;  // sum of decoded products, AN-coded with the result's A
        return;
    }
    const uint64_t n = H.ngroups[qi];
    R.ngroups = n;
    if (n > R.capacity) {
        R.status = AHEAD_CAPACITY;
        return;
    }
    const unsigned long long* o = P + H.off[qi];
    for (int j = 0; j < G; ++j)
        if (R.keys[j]) std::memcpy(R.keys[j], o + (size_t)j * n, n * 8);
    if (R.sums) std::memcpy(R.sums, o + (size_t)G * n, n * 8);
}

int sj_wait(ahead_sj_engine* e, uint64_t ticket, ahead_sj_result* res) {
    if (!e || !res) return AHEAD_BAD_ARG;
    SjSlot& S = e->slot[ticket % kSlots];
    if (!S.busy || S.ticket != ticket) return fail(e->ctx, AHEAD_BAD_ARG, "star join: unknown ticket");
    if (S.local_pending) return fail(e->ctx, AHEAD_BAD_ARG, "star join: the batch's final half was not submitted");
    S.busy = false;
    cudaError_t ce = cudaStreamSynchronize(S.copy);
    if (ce != cudaSuccess) return cuda_fail(e->ctx, ce, "star join");
    const SjHdr& H = *S.h_hdr;
    const SjLayout L = sj_layout();
    if (H.packed_len > kPackedWords) return fail(e->ctx, AHEAD_CUDA_ERROR, "star join: bad packed length");
    if (H.packed_len) {
        cudaMemcpyAsync(S.h_packed, S.dev + L.packed, H.packed_len * 8, cudaMemcpyDeviceToHost, S.copy);
        ce = cudaStreamSynchronize(S.copy);
        if (ce != cudaSuccess) return cuda_fail(e->ctx, ce, "star join");
    }
    cudaEventElapsedTime(&e->last_ms, S.e0, S.e1);
    e->stats.batch_ms = e->last_ms;
    cudaEventElapsedTime(&e->stats.fact_ms, S.f0, S.f1);
    e->stats.fact_rows = S.nmax;
    e->stats.h2d_bytes = L.upload;
    e->stats.d2h_bytes = sizeof(SjHdr) + H.packed_len * 8;
    e->stats.errors_logged = H.errcnt;
    e->stats.strategy = S.strategy;
    e->stats.exception_rows = H.exccnt;
    e->stats.unseen_sigs = (uint32_t)(H.unseen < 0xffffffffull ? H.unseen : 0xffffffffull);
    e->stats.cube_variant = S.cube_variant;
    for (int qi = 0; qi < S.nq; ++qi) sj_fill(S, qi, res[qi]);
    return AHEAD_OK;
}

}  // namespace

extern "C" {

int ahead_sj_create(ahead_ctx* ctx, const ahead_sj_schema* schema, ahead_sj_engine** out) {
    if (!ctx || !schema || !out) return AHEAD_BAD_ARG;
    for (int d = 0; d < 4; ++d)
        if (schema->fk[d].type != AHEAD_RESINT || schema->dim[d].key.type != AHEAD_RESINT)
            return fail(ctx, AHEAD_BAD_ARG, "star join: resint keys and foreign keys required");
    if (schema->price.type != AHEAD_RESINT || schema->discount.type != AHEAD_RESTINY)
        return fail(ctx, AHEAD_BAD_ARG, "star join: resint price and restiny discount required");
    if ((schema->quantity.data && schema->quantity.type != AHEAD_RESTINY) ||
        (schema->revenue.data && schema->revenue.type != AHEAD_RESINT) ||
        (schema->supplycost.data && schema->supplycost.type != AHEAD_RESINT))
        return fail(ctx, AHEAD_BAD_ARG, "star join: restiny quantity, resint revenue and supplycost required");
    for (int d = 0; d < 4; ++d)
        for (int a = 0; a < schema->dim[d].nattr; ++a) {
            const int t = schema->dim[d].attr[a].type;
            if (t != AHEAD_RESTINY && t != AHEAD_RESSHORT && t != AHEAD_RESINT)
                return fail(ctx, AHEAD_BAD_ARG, "star join: restiny, resshort or resint attributes required");
        }
    if (schema->fact_rows > kMaxFactRows) return fail(ctx, AHEAD_UNSUPPORTED, "star join: fact rows <= 2^32 - 2^16");
    auto* e = new ahead_sj_engine();
    e->ctx = ctx;
    e->sch = *schema;
    int rc = sj_prepare(e);
    if (rc) {
        ahead_sj_destroy(e);
        return fail(ctx, rc, "star join: schema preparation failed");
    }
    *out = e;
    return AHEAD_OK;
}

void ahead_sj_destroy(ahead_sj_engine* e) {
    if (!e) return;
    cudaStreamSynchronize(e->ctx->stream);
    for (auto& S : e->slot)
        if (S.copy) {
            cudaStreamSynchronize(S.copy);
            cudaStreamDestroy(S.copy);
        }
    for (auto& S : e->slot) {
        sj_drop_graph(S);
        if (S.dev) cudaFree(S.dev);
        if (S.h_up) cudaFreeHost(S.h_up);
        if (S.h_hdr) cudaFreeHost(S.h_hdr);
        if (S.h_packed) cudaFreeHost(S.h_packed);
        if (S.e0) cudaEventDestroy(S.e0);
        if (S.e1) cudaEventDestroy(S.e1);
        if (S.f0) cudaEventDestroy(S.f0);
        if (S.f1) cudaEventDestroy(S.f1);
        if (S.hdr_done) cudaEventDestroy(S.hdr_done);
        for (void* x : {(void*)S.xsum, (void*)S.xfirst, (void*)S.xflag, (void*)S.xlog})
            if (x) cudaFree(x);
    }
    for (int d = 0; d < 4; ++d) {
        for (uint32_t* t : e->dim[d].aval)
            if (t) cudaFree(t);
        if (e->dim[d].accr) cudaFree(e->dim[d].accr);
        if (e->dim[d].rec) cudaFree(e->dim[d].rec);
        if (e->dim[d].code) cudaFree(e->dim[d].code);
        if (e->dim[d].present) cudaFree(e->dim[d].present);
    }
    if (e->sums) cudaFree(e->sums);
    if (e->firsts) cudaFree(e->firsts);
    if (e->lists) cudaFree(e->lists);
    if (e->lists_tmp) cudaFree(e->lists_tmp);
    if (e->cube) cudaFree(e->cube);
    if (e->cfirst) cudaFree(e->cfirst);
    if (e->exc) cudaFree(e->exc);
    if (e->unseen) cudaFree(e->unseen);
    if (e->fidx) cudaFree(e->fidx);
    if (e->flist) cudaFree(e->flist);
    if (e->pfmap) cudaFree(e->pfmap);
    delete e;
}

// A sharded engine answers whole-table queries only with the exchange; alone
// it may run them when it holds the whole table.
bool sj_whole(const ahead_sj_engine* e) { return !e->sharded || (e->shard_lo == 0 && e->table_rows == e->sch.fact_rows); }

int ahead_sj_submit(ahead_sj_engine* e, const ahead_sj_query* qs, int nq, int use_graph, uint64_t* ticket) {
    if (!ticket) return AHEAD_BAD_ARG;
    if (e && !sj_whole(e)) return fail(e->ctx, AHEAD_BAD_ARG, "star join: a shard answers through submit_local/final");
    return sj_submit(e, qs, nq, use_graph, ticket);
}

int ahead_sj_wait(ahead_sj_engine* e, uint64_t ticket, ahead_sj_result* res) { return sj_wait(e, ticket, res); }

int ahead_sj_set_shard(ahead_sj_engine* e, uint64_t first_row, uint64_t table_rows) {
    if (!e || table_rows >= (1ull << 32) || first_row > table_rows || e->sch.fact_rows > table_rows - first_row)
        return AHEAD_BAD_ARG;
    if (e->slot[0].busy || e->slot[1].busy) return fail(e->ctx, AHEAD_CAPACITY, "star join: batches in flight");
    cudaStreamSynchronize(e->ctx->stream);
    for (auto& S : e->slot) sj_drop_graph(S);  // the launch sequence differs
    e->sharded = true;
    e->shard_lo = first_row;
    e->table_rows = table_rows;
    return AHEAD_OK;
}

int ahead_sj_submit_local(ahead_sj_engine* e, const ahead_sj_query* qs, int nq, int use_graph, uint64_t* ticket,
                          ahead_sj_xchg* x) {
    if (!e || !ticket || !x) return AHEAD_BAD_ARG;
    if (!e->sharded) return fail(e->ctx, AHEAD_BAD_ARG, "star join: submit_local needs ahead_sj_set_shard");
    const int rc = sj_submit(e, qs, nq, use_graph, ticket, true);
    if (rc) return rc;
    const SjSlot& S = e->slot[*ticket % kSlots];
    x->sums = reinterpret_cast<int64_t*>(S.xsum);
    x->firsts = reinterpret_cast<int64_t*>(S.xfirst);
    x->flags = reinterpret_cast<int64_t*>(S.xflag);
    x->log = reinterpret_cast<uint64_t*>(S.xlog);
    x->groups = reinterpret_cast<const SjBatch*>(S.h_up + sj_layout().batch)->gtotal;
    x->log_cap = kErrLogCap;
    return AHEAD_OK;
}

int ahead_sj_submit_final(ahead_sj_engine* e, uint64_t ticket, const uint64_t* gathered_logs, int world) {
    return sj_submit_final(e, ticket, gathered_logs, world);
}

int ahead_sj_run(ahead_sj_engine* e, const ahead_sj_query* qs, int nq, ahead_sj_result* res) {
    if (e && !sj_whole(e)) return fail(e->ctx, AHEAD_BAD_ARG, "star join: a shard answers through submit_local/final");
    uint64_t t = 0;
    const int rc = sj_submit(e, qs, nq, 0, &t);
    return rc ? rc : sj_wait(e, t, res);
}

int ahead_sj_run_graph(ahead_sj_engine* e, const ahead_sj_query* qs, int nq, ahead_sj_result* res) {
    if (e && !sj_whole(e)) return fail(e->ctx, AHEAD_BAD_ARG, "star join: a shard answers through submit_local/final");
    uint64_t t = 0;
    const int rc = sj_submit(e, qs, nq, 1, &t);
    return rc ? rc : sj_wait(e, t, res);
}

float ahead_sj_last_ms(ahead_sj_engine* e) { return e ? e->last_ms : 0.f; }

int ahead_sj_last_stats(ahead_sj_engine* e, ahead_sj_stats* out) {
    if (!e || !out) return AHEAD_BAD_ARG;
    *out = e->stats;
    return AHEAD_OK;
}

int ahead_sj_set_variant(ahead_sj_engine* e, int variant) {
    if (!e || variant < 0 || variant >= kSjVariants) return AHEAD_BAD_ARG;
    if (e->slot[0].busy || e->slot[1].busy) return fail(e->ctx, AHEAD_CAPACITY, "star join: batches in flight");
    if (variant == e->variant) return AHEAD_OK;
    cudaStreamSynchronize(e->ctx->stream);
    for (auto& S : e->slot) sj_drop_graph(S);  // captured with the previous kernel
    e->variant = variant;
    return AHEAD_OK;
}

int ahead_sj_fetch(ahead_sj_engine* e, uint64_t ticket, int qi, ahead_sj_result* res) {
    if (!e || !res) return AHEAD_BAD_ARG;
    const SjSlot& S = e->slot[ticket % kSlots];
    if (S.busy || S.ticket != ticket || qi < 0 || qi >= S.nq)
        return fail(e->ctx, AHEAD_BAD_ARG, "star join: the batch is not the slot's last collected one");
    sj_fill(S, qi, *res);
    return AHEAD_OK;
}

int ahead_sj_ready(ahead_sj_engine* e, uint64_t ticket) {
    if (!e) return AHEAD_BAD_ARG;
    const SjSlot& S = e->slot[ticket % kSlots];
    if (!S.busy || S.ticket != ticket) return AHEAD_BAD_ARG;
    const cudaError_t r = cudaEventQuery(S.hdr_done);
    return r == cudaSuccess ? 1 : r == cudaErrorNotReady ? 0 : -AHEAD_CUDA_ERROR;
}

int ahead_sj_footprint(ahead_sj_engine* e, const ahead_sj_query* q, uint64_t* bytes) {
    if (!e || !q || !bytes || q->ngroup < 0 || q->ngroup > 3) return AHEAD_BAD_ARG;
    uint64_t G = 1;
    for (int j = 0; j < q->ngroup; ++j) {
        const int d = q->gdim[j], a = q->gattr[j];
        if (d < 0 || d > 3 || a < 0 || a >= AHEAD_SJ_MAXATTR) return AHEAD_BAD_ARG;
        const auto& X = e->dim[d];
        G *= X.amax[a] >= X.amin[a] ? X.amax[a] - X.amin[a] + 1 : 1;
    }
    // dense group slots (sum, first row, two sort-list words) and descriptors
    *bytes = G * (12 + 16) + 4096;
    return AHEAD_OK;
}

int ahead_sj_set_cube_variant(ahead_sj_engine* e, int variant) {
    if (!e || variant < 0 || variant >= kCubeVariants) return AHEAD_BAD_ARG;
    if (kCubeShapes[variant].idx && !e->vec_ok)
        return fail(e->ctx, AHEAD_UNSUPPORTED, "star join: the indexed cube scans need 16-byte aligned fact columns");
    if (e->slot[0].busy || e->slot[1].busy) return fail(e->ctx, AHEAD_CAPACITY, "star join: batches in flight");
    if (variant == e->cube_variant) return AHEAD_OK;
    cudaStreamSynchronize(e->ctx->stream);
    for (auto& S : e->slot) sj_drop_graph(S);  // captured with the previous kernel
    e->cube_variant = variant;
    return AHEAD_OK;
}

int ahead_sj_cube_variant_count(void) { return kCubeVariants; }

int ahead_sj_cube_variant_is_indexed(int variant) {
    return variant < 0 || variant >= kCubeVariants ? -1 : kCubeShapes[variant].idx ? 1 : 0;
}

int ahead_sj_cube_variant_slots(int variant) {
    return variant < 0 || variant >= kCubeVariants ? -1 : kCubeShapes[variant].nslot;
}

int ahead_sj_index_info(ahead_sj_engine* e, const void** data, uint64_t* bytes_per_row, uint64_t* rows,
                        uint32_t* dims) {
    if (!e || !data || !bytes_per_row || !rows || !dims) return AHEAD_BAD_ARG;
    *data = e->fidx;
    *bytes_per_row = e->ixfmt == 2 ? sizeof(unsigned long long) : sizeof(ulonglong2);
    *rows = e->fidx ? e->sch.fact_rows : 0;
    *dims = 0;
    for (int d = 0; d < 4; ++d)
        if (e->fidx && e->dim[d].ixslot) *dims |= 1u << d;
    return AHEAD_OK;
}

int ahead_sj_set_index(ahead_sj_engine* e, int format) {
    if (!e || format < -1 || format > 2) return AHEAD_BAD_ARG;
    if (e->slot[0].busy || e->slot[1].busy) return fail(e->ctx, AHEAD_CAPACITY, "star join: batches in flight");
    cudaStreamSynchronize(e->ctx->stream);
    for (auto& S : e->slot) sj_drop_graph(S);  // captured with the previous index
    const int rc = sj_build_index(e, format);
    // a shape that reads the other index format would run its lookups: take the format's default
    if (e->fidx && e->vec_ok && !sj_shape_fits(kCubeShapes[e->cube_variant], e->ixfmt))
        e->cube_variant = e->ixfmt == 2 ? kCubePackedDefault : kCubeIndexedDefault;
    return rc;
}

int ahead_sj_index_packing(const uint64_t krange[2], const uint64_t nrec[2], uint64_t* A, uint32_t* payload_bits) {
    if (!krange || !nrec || !A || !payload_bits) return AHEAD_BAD_ARG;
    SjIxPacking P;
    if (!sj_ix_packing(krange, nrec, &P)) return AHEAD_UNSUPPORTED;
    *A = P.A;
    *payload_bits = P.bits;
    return AHEAD_OK;
}

int ahead_sj_set_cube_split(ahead_sj_engine* e, uint64_t rows) {
    if (!e) return AHEAD_BAD_ARG;
    e->cube_split = rows;
    return AHEAD_OK;
}

int ahead_sj_set_strategy(ahead_sj_engine* e, int strategy) {
    if (!e || strategy < -1 || strategy > 1) return AHEAD_BAD_ARG;
    e->strategy = strategy;
    return AHEAD_OK;
}

int ahead_sj_tune(ahead_sj_engine* e, const ahead_sj_query* qs, int nq, int* variant) {
    if (!e || !qs || nq < 1 || nq > kMaxQ) return AHEAD_BAD_ARG;
    if (e->slot[0].busy || e->slot[1].busy) return fail(e->ctx, AHEAD_CAPACITY, "star join: batches in flight");
    std::vector<ahead_sj_result> res(nq);
    std::memset(res.data(), 0, sizeof(ahead_sj_result) * nq);
    const int keep_strategy = e->strategy;
    // median of three timings of the batch's first-pass kernel
    auto time_it = [&](float* out) -> int {
        float t[3];
        for (int r = 0; r < 3; ++r) {
            uint64_t tk = 0;
            int rc = sj_submit(e, qs, nq, 0, &tk);
            if (rc) return rc;
            rc = sj_wait(e, tk, res.data());
            if (rc) return rc;
            t[r] = e->stats.fact_ms;
        }
        std::sort(t, t + 3);
        *out = t[1];
        return AHEAD_OK;
    };
    // per-row pass shapes
    e->strategy = kStratRows;
    int best = e->variant;
    float best_ms = 0.f;
    for (int v = 0; v < kSjVariants; ++v) {
        int rc = ahead_sj_set_variant(e, v);
        if (rc) return rc;
        float ms;
        rc = time_it(&ms);
        if (rc) return rc;
        if (v == 0 || ms < best_ms) {
            best = v;
            best_ms = ms;
        }
    }
    int rc = ahead_sj_set_variant(e, best);
    if (rc) return rc;
    // cube-scan shapes, each in one phase and split in two, when the batch fits the cube
    e->strategy = kStratCube;
    int cbest = e->cube_variant;
    uint64_t sbest = e->cube_split;
    float cbest_ms = 0.f;
    bool timed = false;
    for (int v = 0; v < kCubeVariants; ++v) {
        if (kCubeShapes[v].idx && (!e->vec_ok || (e->fidx && !sj_shape_fits(kCubeShapes[v], e->ixfmt)))) continue;
        for (const uint64_t split : {(uint64_t)0, ~(uint64_t)0}) {
            e->cube_variant = v;
            e->cube_split = split;
            float ms;
            rc = time_it(&ms);
            if (rc) return rc;
            if (e->stats.strategy != kStratCube) break;
            if (!timed || ms < cbest_ms) {
                cbest = v;
                sbest = split;
                cbest_ms = ms;
                timed = true;
            }
        }
    }
    e->cube_variant = cbest;
    e->cube_split = sbest;
    e->strategy = keep_strategy;
    for (auto& S : e->slot) sj_drop_graph(S);  // captured with other kernels
    if (variant) *variant = best;
    return AHEAD_OK;
}

}  // extern "C"
