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
//   - per batch: one pass over each dimension builds, per dimension row, a
//     64-bit mask of the queries that accept it (predicates on codes);
//   - the fact kernel: a persistent grid; each thread owns 8 rows of a
//     2048-row tile and walks the dimensions in stages (all 8 rows' loads of
//     a stage are in flight together); a foreign key is loaded only while some
//     query that joins it is still alive for the row, so a selective query
//     reads the later columns sparsely;
//   - surviving (row, query) pairs add their product to the query's dense
//     group table and atomicMin their row into the group's first-row word;
//   - finalize: per query the non-empty groups are sorted by first row.
// Detected errors are appended to a log (query, column, row) that one block
// sorts afterwards; every wait in here is a kernel boundary, none spins.
#include <algorithm>
#include <map>
#include <vector>

#include "ops_common.cuh"

using namespace ahead;

namespace {

constexpr int kSjRows = 8;  // rows per thread per tile
constexpr int kSjThreads = 256;
constexpr int kSjTile = kSjRows * kSjThreads;
constexpr uint32_t kNoRow = 0xffffffffu;
constexpr int kMaxGroupsOut = 4096;      // per query, fused path
constexpr uint64_t kMaxDense = 1u << 20;  // dense group-index domain per query
constexpr int kErrLogCap = 1 << 16;
// join order of the dimensions: customer, supplier, part, date
AHEAD_HD int join_dim(int k) {
    return k == 0 ? AHEAD_SJ_CUSTOMER : k == 1 ? AHEAD_SJ_SUPPLIER : k == 2 ? AHEAD_SJ_PART : AHEAD_SJ_DATE;
}

struct SjDimDev {
    const unsigned long long* fk;  // fact foreign-key codes
    const uint32_t* kmap;           // kmap[key - kmin] = dim row + 1
    const unsigned long long* accept;  // per dimension row: queries accepting it
    uint64_t fk_ainv, kmin, krange;
    unsigned long long joins, first;  // queries joining / joining first
};

struct SjQDev {
    uint64_t nrows;
    const void* gcol[3];
    uint64_t gainv[3], gmask[3], glo[3], gstride[3], gA[3], gwm[3];
    uint32_t gdim[3], gw[3];
    uint32_t ngroup, gbase;
};

struct SjBatch {
    SjDimDev dim[4];
    const unsigned long long* price;
    const uint16_t* disc;
    uint64_t price_ainv, disc_ainv;
    const SjQDev* q;
    unsigned long long* sums;  // dense group tables
    uint32_t* firsts;
    unsigned long long* raw;   // [64] ungrouped code-product sums
    unsigned long long* errlog;
    uint32_t* errcnt;
    uint32_t* status;
    uint64_t nmax;
    uint32_t ntiles, nq;
    unsigned long long used;  // queries in the batch
};

__device__ __forceinline__ void log_err(const SjBatch& b, unsigned long long qs, uint32_t col, uint64_t row) {
    while (qs) {
        const int q = __ffsll(qs) - 1;
        qs &= qs - 1;
        const uint32_t i = atomicAdd(b.errcnt, 1u);
        if (i < kErrLogCap) b.errlog[i] = ((unsigned long long)q << 58) | ((unsigned long long)col << 55) | row;
        else atomicOr(b.status, kDevStatusCapacity);
    }
}

__global__ void __launch_bounds__(kSjThreads) sj_fact_kernel(SjBatch b) {
    __shared__ uint64_t s_n[AHEAD_SJ_MAXQ];
    if (threadIdx.x < b.nq) s_n[threadIdx.x] = b.q[threadIdx.x].nrows;
    __syncthreads();
    for (uint32_t tile = blockIdx.x; tile < b.ntiles; tile += gridDim.x) {
        const uint64_t t0 = (uint64_t)tile * kSjTile;
        // queries alive for the whole tile, and those whose prefix ends inside it
        unsigned long long full = 0, part = 0;
        for (uint32_t q = 0; q < b.nq; ++q) {
            if (s_n[q] >= t0 + kSjTile) full |= 1ull << q;
            else if (s_n[q] > t0) part |= 1ull << q;
        }
        uint64_t row[kSjRows];
        unsigned long long alive[kSjRows];
        uint32_t drow[kSjRows][4];
#pragma unroll
        for (int i = 0; i < kSjRows; ++i) {
            row[i] = t0 + (uint64_t)i * kSjThreads + threadIdx.x;
            unsigned long long a = full;
            unsigned long long p = part;
            while (p) {
                const int q = __ffsll(p) - 1;
                p &= p - 1;
                if (row[i] < s_n[q]) a |= 1ull << q;
            }
            alive[i] = row[i] < b.nmax ? a : 0ull;
#pragma unroll
            for (int d = 0; d < 4; ++d) drow[i][d] = kNoRow;
        }
        // dimensions, in the pipeline's join order
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int d = join_dim(k);
            const SjDimDev& D = b.dim[d];
            if (!D.joins) continue;
            unsigned long long code[kSjRows];
#pragma unroll
            for (int i = 0; i < kSjRows; ++i) code[i] = (alive[i] & D.joins) ? __ldg(D.fk + row[i]) : 0ull;
            uint32_t mv[kSjRows];
#pragma unroll
            for (int i = 0; i < kSjRows; ++i) {
                mv[i] = 0;
                if (alive[i] & D.joins) {
                    const uint64_t key = (code[i] * D.fk_ainv) & 0xffffffffull;  // truncated to the key type
                    const uint64_t idx = key - D.kmin;
                    if (idx < D.krange) mv[i] = __ldg(D.kmap + idx);
                }
            }
#pragma unroll
            for (int i = 0; i < kSjRows; ++i) {
                const unsigned long long jq = alive[i] & D.joins;
                if (!jq) continue;
                const unsigned long long acc = mv[i] ? __ldg(D.accept + (mv[i] - 1)) : 0ull;
                if (mv[i]) drow[i][d] = mv[i] - 1;
                const bool corrupt = (code[i] * D.fk_ainv) > 0xffffffffull;
                if (corrupt) {
                    log_err(b, jq, d, row[i]);
                    alive[i] &= ~(jq & ~D.first);  // positional fetch drops the row
                }
                alive[i] &= acc | ~D.joins;
            }
        }
        // measures for surviving rows: price, then discount
#pragma unroll
        for (int i = 0; i < kSjRows; ++i) {
            if (!alive[i]) continue;
            const unsigned long long pc = __ldg(b.price + row[i]);
            const uint64_t pdec = pc * b.price_ainv;
            if (pdec > 0xffffffffull) {
                log_err(b, alive[i], 4, row[i]);
                continue;
            }
            const uint32_t dc = __ldg(b.disc + row[i]);
            const uint32_t ddec = (dc * (uint32_t)b.disc_ainv) & 0xffffu;
            if (ddec > 0xffu) {
                log_err(b, alive[i], 5, row[i]);
                continue;
            }
            const uint64_t prod = (pdec * kResoidAMax) * ((uint64_t)ddec * kResoidAMax);
            const uint64_t rawp = pc * (uint64_t)dc;
            unsigned long long qs = alive[i];
            while (qs) {
                const int q = __ffsll(qs) - 1;
                qs &= qs - 1;
                const SjQDev& Q = b.q[q];
                if (Q.ngroup == 0) {
                    atomicAdd(&b.raw[q], (unsigned long long)rawp);
                    continue;
                }
                uint64_t g = 0;
                for (uint32_t j = 0; j < Q.ngroup; ++j) {
                    const uint32_t r = drow[i][Q.gdim[j]];
                    const uint64_t c = Q.gw[j] == 2 ? (uint64_t)__ldg((const uint16_t*)Q.gcol[j] + r)
                                                    : (uint64_t)__ldg((const uint32_t*)Q.gcol[j] + r);
                    const uint64_t v = (c * Q.gainv[j]) & Q.gmask[j];
                    g += (v - Q.glo[j]) * Q.gstride[j];
                }
                atomicAdd(&b.sums[Q.gbase + g], (unsigned long long)prod);
                if (b.firsts[Q.gbase + g] > (uint32_t)row[i]) atomicMin(&b.firsts[Q.gbase + g], (uint32_t)row[i]);
            }
        }
    }
}

// Per dimension row: the mask of batch queries that accept it (no predicate
// on this dimension, or the predicate holds on the attribute's code).
struct AcceptQ {
    RangePred pred;
    const void* col;
    int has_pred, w;
};

// `nonempty` collects the queries that accept at least one row: hashjoinAN
// probes nothing when its build side is empty (hashjoinAN.tcc:128), so such a
// query reports no errors for its first foreign key.
__global__ void sj_accept_kernel(const AcceptQ* aq, int nq, unsigned long long joins, uint64_t rows,
                                 unsigned long long* accept, unsigned long long* nonempty) {
    unsigned long long any = 0;
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < rows; r += (uint64_t)gridDim.x * blockDim.x) {
        unsigned long long m = 0;
        for (int q = 0; q < nq; ++q) {
            if (!((joins >> q) & 1ull)) continue;
            const AcceptQ& a = aq[q];
            bool ok = true;
            if (a.has_pred) {
                const uint64_t v = a.w == 2 ? (uint64_t)((const uint16_t*)a.col)[r] : (uint64_t)((const uint32_t*)a.col)[r];
                ok = a.pred(v);
            }
            if (ok) m |= 1ull << q;
        }
        accept[r] = m;
        any |= m;
    }
    const uint32_t lo = __reduce_or_sync(0xffffffffu, (uint32_t)any);
    const uint32_t hi = __reduce_or_sync(0xffffffffu, (uint32_t)(any >> 32));
    if ((threadIdx.x & 31) == 0 && (lo | hi)) atomicOr(nonempty, ((unsigned long long)hi << 32) | lo);
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

// Decoded range and corrupt count of an attribute column.
__global__ void sj_attr_kernel(const void* col, int w, uint64_t n, uint64_t ainv, uint64_t umax,
                               unsigned long long* mm) {
    unsigned long long lo = ~0ull, hi = 0, bad = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t c = w == 2 ? (uint64_t)((const uint16_t*)col)[i] : (uint64_t)((const uint32_t*)col)[i];
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

// One block sorts the error log ascending (bitonic, in global memory).
__global__ void __launch_bounds__(1024) sj_errsort_kernel(unsigned long long* log, const uint32_t* cnt) {
    const uint32_t n = *cnt < (uint32_t)kErrLogCap ? *cnt : (uint32_t)kErrLogCap;
    uint32_t p = 1;
    while (p < n) p <<= 1;
    for (uint32_t i = n + threadIdx.x; i < p; i += blockDim.x) log[i] = ~0ull;
    __syncthreads();
    for (uint32_t k = 2; k <= p; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < p; i += blockDim.x) {
                const uint32_t l = i ^ j;
                if (l > i) {
                    const unsigned long long a = log[i], c = log[l];
                    const bool up = (i & k) == 0;
                    if ((a > c) == up) {
                        log[i] = c;
                        log[l] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
}

// Per query (one block): non-empty groups sorted by first row; keys are the
// group attributes' codes, sums the AN-coded totals.
struct SjOutDev {
    unsigned long long* keys;  // [nq][3][kMaxGroupsOut]
    unsigned long long* sums;  // [nq][kMaxGroupsOut]
    unsigned long long* ngroups;  // [nq]
};

__global__ void __launch_bounds__(1024) sj_finalize_kernel(SjBatch b, SjOutDev o) {
    __shared__ unsigned long long s_k[kMaxGroupsOut];  // (first row << 32) | dense index
    __shared__ uint32_t s_n;
    const uint32_t q = blockIdx.x;
    const SjQDev& Q = b.q[q];
    if (Q.ngroup == 0) return;
    if (threadIdx.x == 0) s_n = 0;
    __syncthreads();
    // the dense group domain [gbase, gbase + gsize); gsize arrives in ngroups[q]
    const uint64_t gsize = o.ngroups[q];
    __syncthreads();
    for (uint64_t g = threadIdx.x; g < gsize; g += blockDim.x) {
        const uint32_t f = b.firsts[Q.gbase + g];
        if (f != kNoRow) {
            const uint32_t i = atomicAdd(&s_n, 1u);
            if (i < kMaxGroupsOut) s_k[i] = ((unsigned long long)f << 32) | g;
        }
    }
    __syncthreads();
    const uint32_t n = s_n;
    if (n > (uint32_t)kMaxGroupsOut) {
        if (threadIdx.x == 0) {
            atomicOr(b.status, kDevStatusCapacity);
            o.ngroups[q] = ~0ull;
        }
        return;
    }
    uint32_t p = 1;
    while (p < n) p <<= 1;
    for (uint32_t i = n + threadIdx.x; i < p; i += blockDim.x) s_k[i] = ~0ull;
    __syncthreads();
    for (uint32_t k = 2; k <= p; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < p; i += blockDim.x) {
                const uint32_t l = i ^ j;
                if (l > i) {
                    const unsigned long long a = s_k[i], c = s_k[l];
                    if ((a > c) == ((i & k) == 0)) {
                        s_k[i] = c;
                        s_k[l] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const uint64_t g = s_k[i] & 0xffffffffull;
        o.sums[(size_t)q * kMaxGroupsOut + i] = b.sums[Q.gbase + g];
        uint64_t rem = g;
        for (int j = (int)Q.ngroup - 1; j >= 0; --j) {
            const uint64_t vj = rem / Q.gstride[j];
            rem -= vj * Q.gstride[j];
            o.keys[((size_t)q * 3 + j) * kMaxGroupsOut + i] = ((vj + Q.glo[j]) * Q.gA[j]) & Q.gwm[j];
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) o.ngroups[q] = n;
}


}  // namespace

// ------------------------------------------------------------------ engine
struct ahead_sj_engine {
    ahead_ctx* ctx = nullptr;
    ahead_sj_schema sch{};
    struct Dim {
        uint32_t* kmap = nullptr;
        uint64_t kmin = 0, krange = 0;
        bool usable = false;  // keys clean, unique, mappable
        unsigned long long* accept = nullptr;
        uint64_t amin[AHEAD_SJ_MAXATTR] = {}, amax[AHEAD_SJ_MAXATTR] = {}, abad[AHEAD_SJ_MAXATTR] = {};
    } dim[4];
    // batch buffers
    char* dev = nullptr;  // one allocation: descriptors, logs, outputs
    size_t dev_cap = 0;
    unsigned long long* sums = nullptr;
    uint32_t* firsts = nullptr;
    size_t gcap = 0;
    unsigned long long* h_out = nullptr;  // pinned staging of the outputs
    size_t h_cap = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    float last_ms = 0.f;
    std::map<std::vector<uint64_t>, cudaGraphExec_t> graphs;
};

namespace {

int sj_prepare(ahead_sj_engine* e) {
    ahead_ctx* ctx = e->ctx;
    cudaStream_t st = ctx->stream;
    unsigned long long* mm = nullptr;
    if (cudaMalloc(&mm, 64 * sizeof(unsigned long long)) != cudaSuccess) return AHEAD_NO_MEMORY;
    for (int d = 0; d < 4; ++d) {
        const ahead_sj_dim& D = e->sch.dim[d];
        if (!D.rows || !D.key.data) continue;
        unsigned long long h[3] = {~0ull, 0, 0};
        cudaMemcpyAsync(mm, h, sizeof h, cudaMemcpyHostToDevice, st);
        sj_keyrange_kernel<<<grid_for(D.rows, 256), 256, 0, st>>>((const unsigned long long*)D.key.data, D.rows,
                                                                  D.key.Ainv, mm);
        cudaMemcpyAsync(h, mm, sizeof h, cudaMemcpyDeviceToHost, st);
        cudaStreamSynchronize(st);
        auto& X = e->dim[d];
        X.usable = false;
        if (h[2] == 0 && h[0] <= h[1] && (h[1] - h[0]) < (1ull << 28)) {
            X.kmin = h[0];
            X.krange = h[1] - h[0] + 1;
            if (cudaMalloc(&X.kmap, X.krange * 4) != cudaSuccess) return AHEAD_NO_MEMORY;
            cudaMemsetAsync(X.kmap, 0, X.krange * 4, st);
            cudaMemsetAsync(mm, 0, 8, st);
            sj_kmap_kernel<<<grid_for(D.rows, 256), 256, 0, st>>>((const unsigned long long*)D.key.data, D.rows,
                                                                  D.key.Ainv, X.kmin, X.kmap, mm);
            unsigned long long dup = 0;
            cudaMemcpyAsync(&dup, mm, 8, cudaMemcpyDeviceToHost, st);
            cudaStreamSynchronize(st);
            X.usable = dup == 0;
        }
        if (cudaMalloc(&X.accept, D.rows * 8) != cudaSuccess) return AHEAD_NO_MEMORY;
        for (int a = 0; a < D.nattr; ++a) {
            const ahead_col& c = D.attr[a];
            const int w = type_width(c.type);
            unsigned long long g[3] = {~0ull, 0, 0};
            cudaMemcpyAsync(mm, g, sizeof g, cudaMemcpyHostToDevice, st);
            sj_attr_kernel<<<grid_for(D.rows, 256), 256, 0, st>>>(c.data, w, D.rows, c.Ainv & wmask(w),
                                                                  c.unenc_max & wmask(w), mm);
            cudaMemcpyAsync(g, mm, sizeof g, cudaMemcpyDeviceToHost, st);
            cudaStreamSynchronize(st);
            X.amin[a] = g[0];
            X.amax[a] = g[1];
            X.abad[a] = g[2];
        }
        ctx->launches += 2 + D.nattr;
    }
    cudaFree(mm);
    return cudaGetLastError() == cudaSuccess ? AHEAD_OK : AHEAD_CUDA_ERROR;
}

// Layout of the per-batch device area.
struct SjLayout {
    size_t q, aq, raw, nonempty, errlog, errcnt, status, okeys, osums, ongroups, total;
};

SjLayout sj_layout() {
    SjLayout L;
    size_t off = 0;
    auto take = [&](size_t b) {
        size_t o = off;
        off = (off + b + 255) & ~size_t(255);
        return o;
    };
    L.q = take(sizeof(SjQDev) * AHEAD_SJ_MAXQ);
    L.aq = take(sizeof(AcceptQ) * AHEAD_SJ_MAXQ * 4);
    L.raw = take(8 * AHEAD_SJ_MAXQ);
    L.nonempty = take(8 * 4);
    L.errlog = take(8ull * kErrLogCap);
    L.errcnt = take(8);
    L.status = take(8);
    L.okeys = take(8ull * AHEAD_SJ_MAXQ * 3 * kMaxGroupsOut);
    L.osums = take(8ull * AHEAD_SJ_MAXQ * kMaxGroupsOut);
    L.ongroups = take(8 * AHEAD_SJ_MAXQ);
    L.total = off;
    return L;
}

bool dim_usable_for(const ahead_sj_engine* e, const ahead_sj_query& q, int d) {
    if (!e->dim[d].usable) return false;
    for (int j = 0; j < q.ngroup; ++j)
        if (q.gdim[j] == d && e->dim[d].abad[q.gattr[j]]) return false;
    return true;
}

// Build the batch descriptors on the host.  Returns per query whether the
// fused path can answer it.
struct Plan {
    SjBatch b;
    SjOutDev o;
    std::vector<SjQDev> q;
    std::vector<AcceptQ> aq;  // [4][64]
    unsigned long long joins[4] = {0, 0, 0, 0}, first[4] = {0, 0, 0, 0};
    std::vector<int> ok;
    std::vector<uint64_t> gsize;
    uint64_t gtotal = 0;
};

int sj_plan(ahead_sj_engine* e, const ahead_sj_query* qs, int nq, Plan& P) {
    const ahead_sj_schema& S = e->sch;
    P.q.assign(AHEAD_SJ_MAXQ, SjQDev{});
    P.aq.assign(4 * AHEAD_SJ_MAXQ, AcceptQ{});
    P.ok.assign(nq, 1);
    P.gsize.assign(nq, 0);
    P.gtotal = 0;
    uint64_t nmax = 0;
    for (int qi = 0; qi < nq; ++qi) {
        const ahead_sj_query& Q = qs[qi];
        bool used[4] = {false, false, false, false};
        for (int k = 0; k < Q.npred; ++k) used[Q.pred[k].dim] = true;
        for (int j = 0; j < Q.ngroup; ++j) used[Q.gdim[j]] = true;
        bool any = false;
        for (int d = 0; d < 4; ++d) any |= used[d];
        if (!any || Q.npred > 4 || Q.ngroup > 3) return AHEAD_BAD_ARG;
        bool first_done = false;
        for (int k = 0; k < 4; ++k) {
            const int d = join_dim(k);
            if (!used[d]) continue;
            if (!dim_usable_for(e, Q, d)) P.ok[qi] = 0;
            P.joins[d] |= 1ull << qi;
            if (!first_done) {
                P.first[d] |= 1ull << qi;
                first_done = true;
            }
        }
        for (int k = 0; k < Q.npred; ++k) {
            const ahead_sj_pred& p = Q.pred[k];
            if (p.dim < 0 || p.dim > 3 || p.attr < 0 || p.attr >= S.dim[p.dim].nattr) return AHEAD_BAD_ARG;
            const ahead_col& c = S.dim[p.dim].attr[p.attr];
            AcceptQ& a = P.aq[p.dim * AHEAD_SJ_MAXQ + qi];
            a.has_pred = 1;
            a.col = c.data;
            a.w = type_width(c.type);
            a.pred = RangePred::make(p.op1, p.th1, p.op2, p.th2, p.comb, wmask(a.w));
        }
        SjQDev& D = P.q[qi];
        D.nrows = Q.fact_rows < S.fact_rows ? Q.fact_rows : S.fact_rows;
        nmax = D.nrows > nmax ? D.nrows : nmax;
        D.ngroup = Q.ngroup;
        uint64_t G = 1;
        for (int j = 0; j < Q.ngroup; ++j) {
            const int d = Q.gdim[j], at = Q.gattr[j];
            if (d < 0 || d > 3 || at < 0 || at >= S.dim[d].nattr) return AHEAD_BAD_ARG;
            const ahead_col& c = S.dim[d].attr[at];
            const int w = type_width(c.type);
            D.gcol[j] = c.data;
            D.gw[j] = w;
            D.gdim[j] = d;
            D.gainv[j] = c.Ainv & wmask(w);
            D.gmask[j] = wmask(type_base_width(c.type));
            D.glo[j] = e->dim[d].amin[at];
            D.gstride[j] = G;
            const uint64_t range = e->dim[d].amax[at] >= e->dim[d].amin[at] ? e->dim[d].amax[at] - e->dim[d].amin[at] + 1 : 1;
            G *= range;
            D.gA[j] = c.A;
            D.gwm[j] = wmask(w);
            if (G > kMaxDense) P.ok[qi] = 0;
        }
        if (!P.ok[qi]) D.nrows = 0;  // not evaluated here; the caller falls back
        D.gbase = (uint32_t)P.gtotal;
        P.gsize[qi] = Q.ngroup && P.ok[qi] ? G : 0;
        P.gtotal += P.gsize[qi];
    }
    for (int d = 0; d < 4; ++d) {
        P.b.dim[d].fk = (const unsigned long long*)S.fk[d].data;
        P.b.dim[d].kmap = e->dim[d].kmap;
        P.b.dim[d].accept = e->dim[d].accept;
        P.b.dim[d].fk_ainv = S.fk[d].Ainv;
        P.b.dim[d].kmin = e->dim[d].kmin;
        P.b.dim[d].krange = e->dim[d].krange;
        // queries that fall back do not take part
        unsigned long long okm = 0;
        for (int qi = 0; qi < nq; ++qi)
            if (P.ok[qi]) okm |= 1ull << qi;
        P.joins[d] &= okm;
        P.first[d] &= okm;
        P.b.dim[d].joins = P.joins[d];
        P.b.dim[d].first = P.first[d];
    }
    P.b.price = (const unsigned long long*)S.price.data;
    P.b.disc = (const uint16_t*)S.discount.data;
    P.b.price_ainv = S.price.Ainv;
    P.b.disc_ainv = S.discount.Ainv & 0xffffull;
    P.b.nmax = nmax;
    P.b.nq = nq;
    P.b.ntiles = (uint32_t)((nmax + kSjTile - 1) / kSjTile);
    return AHEAD_OK;
}

int sj_ensure(ahead_sj_engine* e, uint64_t gtotal) {
    const SjLayout L = sj_layout();
    if (!e->dev) {
        if (cudaMalloc(&e->dev, L.total) != cudaSuccess) return AHEAD_NO_MEMORY;
        e->dev_cap = L.total;
        if (cudaMallocHost(&e->h_out, L.total) != cudaSuccess) return AHEAD_NO_MEMORY;
        e->h_cap = L.total;
    }
    if (!e->sums || gtotal > e->gcap) {  // the first batch allocates even when no query groups
        cudaStreamSynchronize(e->ctx->stream);
        for (auto& kv : e->graphs) cudaGraphExecDestroy(kv.second);  // they captured the old tables
        e->graphs.clear();
        if (e->sums) cudaFree(e->sums);
        if (e->firsts) cudaFree(e->firsts);
        const size_t cap = gtotal < (1u << 16) ? (1u << 16) : gtotal + gtotal / 4;
        if (cudaMalloc(&e->sums, cap * 8) != cudaSuccess) return AHEAD_NO_MEMORY;
        if (cudaMalloc(&e->firsts, cap * 4) != cudaSuccess) return AHEAD_NO_MEMORY;
        e->gcap = cap;
    }
    return AHEAD_OK;
}

// Enqueue one batch on the stream (no host synchronisation).
void sj_enqueue(ahead_sj_engine* e, Plan& P, int nq) {
    cudaStream_t st = e->ctx->stream;
    const SjLayout L = sj_layout();
    char* dev = e->dev;
    const size_t gt = P.gtotal ? P.gtotal : 1;
    cudaMemsetAsync(e->sums, 0, gt * 8, st);
    cudaMemsetAsync(e->firsts, 0xff, gt * 4, st);
    cudaMemsetAsync(dev + L.raw, 0, L.errlog - L.raw, st);
    cudaMemsetAsync(dev + L.errcnt, 0, 16, st);
    for (int d = 0; d < 4; ++d) {
        if (!P.joins[d]) continue;
        sj_accept_kernel<<<grid_for(e->sch.dim[d].rows, 256), 256, 0, st>>>(
            (const AcceptQ*)(dev + L.aq) + d * AHEAD_SJ_MAXQ, nq, P.joins[d], e->sch.dim[d].rows, e->dim[d].accept,
            (unsigned long long*)(dev + L.nonempty) + d);
        e->ctx->launches++;
    }
    const uint32_t grid = P.b.ntiles < (uint32_t)e->ctx->num_sms * 8 ? P.b.ntiles : (uint32_t)e->ctx->num_sms * 8;
    if (grid) {
        sj_fact_kernel<<<grid, kSjThreads, 0, st>>>(P.b);
        e->ctx->launches++;
    }
    sj_errsort_kernel<<<1, 1024, 0, st>>>(P.b.errlog, P.b.errcnt);
    sj_finalize_kernel<<<nq, 1024, 0, st>>>(P.b, P.o);
    e->ctx->launches += 2;
}

int sj_collect(ahead_sj_engine* e, const ahead_sj_query* qs, int nq, const Plan& P, ahead_sj_result* res) {
    const SjLayout L = sj_layout();
    unsigned long long* h = e->h_out;
    // everything after the descriptors in one copy
    cudaMemcpyAsync((char*)h + L.raw, e->dev + L.raw, L.total - L.raw, cudaMemcpyDeviceToHost, e->ctx->stream);
    if (cudaStreamSynchronize(e->ctx->stream) != cudaSuccess) return fail(e->ctx, AHEAD_CUDA_ERROR, "star join");
    const unsigned long long* raw = (const unsigned long long*)((char*)h + L.raw);
    const unsigned long long* nonempty = (const unsigned long long*)((char*)h + L.nonempty);
    const unsigned long long* log = (const unsigned long long*)((char*)h + L.errlog);
    const uint32_t nerr = (uint32_t) * (const unsigned long long*)((char*)h + L.errcnt);
    const uint32_t st = (uint32_t) * (const unsigned long long*)((char*)h + L.status);
    const unsigned long long* okeys = (const unsigned long long*)((char*)h + L.okeys);
    const unsigned long long* osums = (const unsigned long long*)((char*)h + L.osums);
    const unsigned long long* ong = (const unsigned long long*)((char*)h + L.ongroups);
    const uint32_t ne = nerr < (uint32_t)kErrLogCap ? nerr : (uint32_t)kErrLogCap;
    for (int qi = 0; qi < nq; ++qi) {
        ahead_sj_result& R = res[qi];
        for (int c = 0; c < 6; ++c) {
            R.fact_err[c].count = 0;
            R.fact_err[c].present = 1;
        }
        if (!P.ok[qi] || (st & kDevStatusCapacity)) {
            R.status = AHEAD_UNSUPPORTED;
            R.ngroups = 0;
            continue;
        }
        R.status = AHEAD_OK;
        // the first join probed nothing if its build side was empty
        int skip = -1;
        for (int d = 0; d < 4; ++d)
            if (((P.first[d] >> qi) & 1ull) && !((nonempty[d] >> qi) & 1ull)) skip = d;
        // errors: the log is sorted by (query, column, row)
        for (uint32_t i = 0; i < ne; ++i) {
            const unsigned long long x = log[i];
            if ((int)(x >> 58) != qi) continue;
            const int c = (int)((x >> 55) & 7);
            if (c == skip) continue;
            ahead_errvec& E = R.fact_err[c];
            if (E.count < E.capacity && E.data) E.data[E.count] = (x & ((1ull << 55) - 1)) * 16089ull;
            E.count++;
        }
        if (qs[qi].ngroup == 0) {
            const uint64_t enc = kResoidAMax * inv_pow2(e->sch.price.A, 64) * inv_pow2(e->sch.discount.A & 0xffff, 64);
            R.total = raw[qi] * enc;
            R.ngroups = 0;
            continue;
        }
        const uint64_t n = ong[qi];
        if (n == ~0ull) {
            R.status = AHEAD_UNSUPPORTED;
            R.ngroups = 0;
            continue;
        }
        R.ngroups = n;
        const uint64_t m = n < R.capacity ? n : R.capacity;
        for (uint64_t i = 0; i < m; ++i) {
            if (R.sums) R.sums[i] = osums[(size_t)qi * kMaxGroupsOut + i];
            for (int j = 0; j < qs[qi].ngroup; ++j)
                if (R.keys[j]) R.keys[j][i] = okeys[((size_t)qi * 3 + j) * kMaxGroupsOut + i];
        }
    }
    return AHEAD_OK;
}

int sj_setup(ahead_sj_engine* e, const ahead_sj_query* qs, int nq, Plan& P) {
    if (!e || !qs || nq < 1 || nq > AHEAD_SJ_MAXQ) return AHEAD_BAD_ARG;
    int rc = sj_plan(e, qs, nq, P);
    if (rc) return fail(e->ctx, rc, "star join: bad query");
    rc = sj_ensure(e, P.gtotal);
    if (rc) return fail(e->ctx, rc, "star join: device memory");
    const SjLayout L = sj_layout();
    P.b.q = (const SjQDev*)(e->dev + L.q);
    P.b.sums = e->sums;
    P.b.firsts = e->firsts;
    P.b.raw = (unsigned long long*)(e->dev + L.raw);
    P.b.errlog = (unsigned long long*)(e->dev + L.errlog);
    P.b.errcnt = (uint32_t*)(e->dev + L.errcnt);
    P.b.status = (uint32_t*)(e->dev + L.status);
    P.b.used = 0;
    P.o.keys = (unsigned long long*)(e->dev + L.okeys);
    P.o.sums = (unsigned long long*)(e->dev + L.osums);
    P.o.ngroups = (unsigned long long*)(e->dev + L.ongroups);
    // the finalize kernel reads each query's dense group count from ngroups
    std::vector<unsigned long long> ng(AHEAD_SJ_MAXQ, 0);
    for (int qi = 0; qi < nq; ++qi) ng[qi] = P.gsize[qi];
    cudaStream_t st = e->ctx->stream;
    cudaMemcpyAsync(e->dev + L.q, P.q.data(), sizeof(SjQDev) * AHEAD_SJ_MAXQ, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(e->dev + L.aq, P.aq.data(), sizeof(AcceptQ) * AHEAD_SJ_MAXQ * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(e->dev + L.ongroups, ng.data(), 8 * AHEAD_SJ_MAXQ, cudaMemcpyHostToDevice, st);
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
    if (schema->fact_rows >= (1ull << 32)) return fail(ctx, AHEAD_UNSUPPORTED, "star join: fact rows < 2^32");
    auto* e = new ahead_sj_engine();
    e->ctx = ctx;
    e->sch = *schema;
    cudaEventCreate(&e->e0);
    cudaEventCreate(&e->e1);
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
    for (auto& kv : e->graphs) cudaGraphExecDestroy(kv.second);
    for (int d = 0; d < 4; ++d) {
        if (e->dim[d].kmap) cudaFree(e->dim[d].kmap);
        if (e->dim[d].accept) cudaFree(e->dim[d].accept);
    }
    if (e->dev) cudaFree(e->dev);
    if (e->sums) cudaFree(e->sums);
    if (e->firsts) cudaFree(e->firsts);
    if (e->h_out) cudaFreeHost(e->h_out);
    if (e->e0) cudaEventDestroy(e->e0);
    if (e->e1) cudaEventDestroy(e->e1);
    delete e;
}

int ahead_sj_run(ahead_sj_engine* e, const ahead_sj_query* qs, int nq, ahead_sj_result* res) {
    Plan P;
    int rc = sj_setup(e, qs, nq, P);
    if (rc) return rc;
    cudaEventRecord(e->e0, e->ctx->stream);
    sj_enqueue(e, P, nq);
    cudaEventRecord(e->e1, e->ctx->stream);
    rc = sj_collect(e, qs, nq, P, res);
    cudaEventElapsedTime(&e->last_ms, e->e0, e->e1);
    if (cudaGetLastError() != cudaSuccess) return fail(e->ctx, AHEAD_CUDA_ERROR, "star join launch");
    return rc;
}

int ahead_sj_run_graph(ahead_sj_engine* e, const ahead_sj_query* qs, int nq, ahead_sj_result* res) {
    Plan P;
    int rc = sj_setup(e, qs, nq, P);
    if (rc) return rc;
    // the graph depends on the launch shapes and the scalar kernel arguments
    std::vector<uint64_t> sig = {(uint64_t)nq, P.gtotal, P.b.nmax};
    for (int d = 0; d < 4; ++d) {
        sig.push_back(P.joins[d]);
        sig.push_back(P.first[d]);
    }
    auto it = e->graphs.find(sig);
    cudaStream_t st = e->ctx->stream;
    if (it == e->graphs.end()) {
        cudaGraph_t g;
        if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            return fail(e->ctx, AHEAD_CUDA_ERROR, "graph capture");
        sj_enqueue(e, P, nq);
        if (cudaStreamEndCapture(st, &g) != cudaSuccess) return fail(e->ctx, AHEAD_CUDA_ERROR, "graph capture");
        cudaGraphExec_t ex;
        if (cudaGraphInstantiate(&ex, g, 0) != cudaSuccess) {
            cudaGraphDestroy(g);
            return fail(e->ctx, AHEAD_CUDA_ERROR, "graph instantiate");
        }
        cudaGraphDestroy(g);
        it = e->graphs.emplace(sig, ex).first;
    }
    cudaEventRecord(e->e0, st);
    cudaGraphLaunch(it->second, st);
    cudaEventRecord(e->e1, st);
    e->ctx->launches += 3;
    rc = sj_collect(e, qs, nq, P, res);
    cudaEventElapsedTime(&e->last_ms, e->e0, e->e1);
    if (cudaGetLastError() != cudaSuccess) return fail(e->ctx, AHEAD_CUDA_ERROR, "star join graph");
    return rc;
}

float ahead_sj_last_ms(ahead_sj_engine* e) { return e ? e->last_ms : 0.f; }

}  // extern "C"
