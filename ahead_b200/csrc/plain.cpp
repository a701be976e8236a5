// plain.cpp -- the operator-at-a-time star join in C++ host code: one query
// composed from the library's own AN operators through the C ABI
// (include/ahead_gpu.h), the way the reference's programs compose theirs
// (tools/ssbm/ssbm-q11_continuous.cpp, ssbm-q21_continuous.cpp,
// ssbm-q41_continuous.cpp), with continuous detection.  It computes what the
// fused engine computes for the same ahead_sj_query, operator by operator,
// and fills the same ahead_sj_result: the comparison path the fused engine is
// measured against, and the exact semantics it reproduces.
//
// The steps (one operator call each, its outputs in device buffers of its own):
//   per joined dimension, in join order (customer, supplier, part, date):
//     its predicates as selectAN on the attribute codes, intersected in
//     order with matchjoinAN; the key -> OID map = matchjoinAN(key.reverse(),
//     selection), or key.reverse() without predicates;
//   fact predicates (Q1.x): selectAN on quantity / discount over the prefix,
//     intersected the same way, then every foreign key fetched positionally;
//   else the first join probes the whole foreign-key column (hashjoinAN,
//     OIDs re-encoded with the largest resoid A), the others fetch positionally
//     (matchjoinAN of the surviving rows onto the column, then hashjoinAN);
//   the measures fetched one after the other (price then discount, or revenue
//     then supplycost), each dropping the rows it finds corrupt;
//   ungrouped: aggregate_mul_sumAN; grouped: the group attributes fetched
//     through each dimension's join result, arithmeticAN (mul or sub) of the
//     measures, groupbyAN / binary groupbyAN, aggregate_sum_groupedAN, and
//     each group's attribute codes at its first row.
// Error vectors of the fact columns are kept per column in row order (a
// column read twice -- a fact predicate, then a positional fetch -- reports
// the rows of both).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "../../include/ahead_gpu.h"

namespace {

constexpr uint64_t kAoid = 16089;
constexpr uint64_t kAr = 65117;                     // re-encoded OIDs and AN-coded results
constexpr uint64_t kArInv = 0x3E36D3BC8D9BC5F5ull;  // its inverse mod 2^64
constexpr uint64_t kGroupAoid = 65117;              // groupbyAN's OID A and inverse, as the programs call it
constexpr uint64_t kGroupAoidInv = 0x3E36D3BC8D9BC5F5ull;

int width_of(int type) {
    switch (type) {
        case AHEAD_TINYINT: return 1;
        case AHEAD_SHORTINT: case AHEAD_RESTINY: return 2;
        case AHEAD_INT: case AHEAD_OID: case AHEAD_RESSHORT: case AHEAD_VOID: return 4;
        default: return 8;
    }
}

// Device buffers come from a per-device memory pool through the stream-ordered
// allocator (cudaMallocFromPoolAsync / cudaFreeAsync on the library's stream):
// one query makes 20-30 operator calls, each with outputs sized by its inputs
// (up to the fact prefix), and a cudaMalloc / cudaFree pair per buffer --
// cudaFree waits for the whole device -- would cost more than the operators.
// The pool keeps the memory it frees for the next calls (the footprint of the
// largest query so far), as a caching allocator does: returning memory to the
// device at every synchronisation point made each query map it again.
constexpr uint64_t kPoolKeepBytes = ~uint64_t(0);

cudaMemPool_t device_pool(int dev) {
    static std::mutex mu;
    static std::map<int, cudaMemPool_t>* pools = new std::map<int, cudaMemPool_t>();  // (kept until exit)
    std::lock_guard<std::mutex> lk(mu);
    auto it = pools->find(dev);
    if (it != pools->end()) return it->second;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    uint64_t keep = kPoolKeepBytes;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    (*pools)[dev] = pool;
    return pool;
}

// Device buffers of one query, freed together (or one by one, earlier).
struct Arena {
    cudaStream_t st = nullptr;
    cudaMemPool_t pool = nullptr;
    std::vector<void*> bufs;
    void init(ahead_ctx* ctx) {
        int dev = 0;
        cudaGetDevice(&dev);
        st = static_cast<cudaStream_t>(ahead_ctx_stream(ctx));
        pool = device_pool(dev);
    }
    void* take(size_t bytes) {
        void* p = nullptr;
        if (!pool || cudaMallocFromPoolAsync(&p, bytes ? bytes : 8, pool, st) != cudaSuccess) {
            cudaGetLastError();
            // (the device's own pool, e.g. when this one could not be created)
            if (cudaMallocAsync(&p, bytes ? bytes : 8, st) != cudaSuccess) {
                cudaGetLastError();
                return nullptr;
            }
        }
        bufs.push_back(p);
        return p;
    }
    // hands one block back before the query ends
    void give_back(void* p) {
        for (size_t i = 0; i < bufs.size(); ++i)
            if (bufs[i] == p) {
                cudaFreeAsync(p, st);
                bufs.erase(bufs.begin() + (long)i);
                return;
            }
    }
    ~Arena() {
        for (void* p : bufs) cudaFreeAsync(p, st);
    }
};

struct Errs {
    std::vector<ahead_errvec> v;
    uint64_t need() const {
        uint64_t m = 0;
        for (const auto& e : v) m = std::max(m, e.count);
        return m;
    }
};

struct Plain {
    ahead_ctx* ctx;
    Arena arena;
    int rc = AHEAD_OK;
    // fact-column error positions, host, by AHEAD_SJ_COL_* index
    std::vector<uint64_t> ferr[AHEAD_SJ_NCOL];

    static ahead_bat view(const ahead_col& head, const ahead_col& tail, uint64_t count) {
        ahead_bat b{};
        b.head = head;
        b.tail = tail;
        b.count = count;
        return b;
    }
    static ahead_bat reverse(const ahead_bat& b) { return view(b.tail, b.head, b.count); }
    static ahead_bat mirror_head(const ahead_bat& b) { return view(b.head, b.head, b.count); }
    static ahead_bat clear_head(const ahead_bat& b) {
        ahead_col h{};
        h.type = AHEAD_VOID;
        return view(h, b.tail, b.count);
    }

    // One operator call with outputs of `cap` rows and error vectors of a small
    // first capacity; on AHEAD_CAPACITY (or counts above the capacities) the
    // call runs again with the sizes it reported.
    template <typename F>
    bool run(F call, uint64_t cap, int nerr, int nout, ahead_bat* outs, Errs* errs) {
        if (rc) return false;
        uint64_t ecap = std::min<uint64_t>(std::max<uint64_t>(cap, 1), 1u << 16);
        cap = std::max<uint64_t>(cap, 1);
        for (;;) {
            for (int o = 0; o < nout; ++o) {
                outs[o] = ahead_bat{};
                outs[o].head.data = arena.take(cap * 8);
                outs[o].tail.data = arena.take(cap * 8);
                if (!outs[o].head.data || !outs[o].tail.data) return fail(AHEAD_NO_MEMORY);
            }
            if (errs) {
                errs->v.assign(nerr, ahead_errvec{});
                for (auto& e : errs->v) {
                    e.data = static_cast<uint64_t*>(arena.take(ecap * 8));
                    e.capacity = ecap;
                    if (!e.data) return fail(AHEAD_NO_MEMORY);
                }
            }
            const int r = call(cap);
            uint64_t need_o = 0;
            for (int o = 0; o < nout; ++o) need_o = std::max(need_o, outs[o].count);
            const uint64_t need_e = errs ? errs->need() : 0;
            if (r == AHEAD_CAPACITY || need_o > cap || need_e > ecap) {
                if (need_o <= cap && need_e <= ecap) return fail(r);
                cap = std::max(cap, need_o);
                ecap = std::max(ecap, need_e);
                for (int o = 0; o < nout; ++o) {
                    arena.give_back(outs[o].head.data);
                    arena.give_back(outs[o].tail.data);
                }
                if (errs)
                    for (auto& e : errs->v) arena.give_back(e.data);
                continue;
            }
            if (r) return fail(r);
            // an output far below its capacity moves into a block of its size, so
            // the next operators of the query can reuse the large one
            // (a virtual-OID column holds no data: its block goes back at once)
            for (int o = 0; o < nout; ++o) {
                for (ahead_col* c : {&outs[o].head, &outs[o].tail}) {
                    void* big = c->data;
                    if (!big) continue;
                    if (c->type == AHEAD_VOID) {
                        arena.give_back(big);
                        c->data = nullptr;
                        continue;
                    }
                    if (outs[o].count * 4 >= cap) continue;
                    const size_t bytes = outs[o].count * (size_t)width_of(c->type);
                    void* small = arena.take(bytes);
                    if (!small) return fail(AHEAD_NO_MEMORY);
                    if (!copy(small, big, bytes, cudaMemcpyDeviceToDevice)) return false;
                    c->data = small;
                    arena.give_back(big);
                }
            }
            return true;
        }
    }
    bool fail(int r) {
        rc = r;
        return false;
    }
    // a copy on the library's stream, after the operators' work on it
    bool copy(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind) {
        if (!bytes) return true;
        cudaStream_t st = static_cast<cudaStream_t>(ahead_ctx_stream(ctx));
        if (cudaMemcpyAsync(dst, src, bytes, kind, st) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
            return fail(AHEAD_CUDA_ERROR);
        return true;
    }

    std::vector<uint64_t> host_errs(const ahead_errvec& e) {
        std::vector<uint64_t> h(e.present ? e.count : 0);
        copy(h.data(), e.data, h.size() * 8, cudaMemcpyDeviceToHost);
        return h;
    }
    void add_errs(int col, const ahead_errvec& e) {
        std::vector<uint64_t> h = host_errs(e);
        ferr[col].insert(ferr[col].end(), h.begin(), h.end());
        std::sort(ferr[col].begin(), ferr[col].end());
    }
    void set_errs(int col, const ahead_errvec& e) { ferr[col] = host_errs(e); }

    ahead_bat select_an(const ahead_bat& in, int op1, uint64_t th1, int op2, uint64_t th2, int comb,
                        ahead_errvec* err_out) {
        ahead_bat out{};
        Errs errs;
        run([&](uint64_t cap) {
                return ahead_gpu_select_an(ctx, &in, op1, th1, op2, th2, comb, kAoid, &out, cap, &errs.v[0]);
            },
            in.count, 1, 1, &out, &errs);
        if (!rc && err_out) *err_out = errs.v[0];
        return out;
    }
    ahead_bat matchjoin_an(const ahead_bat& a, const ahead_bat& b, ahead_errvec* errs_out = nullptr) {
        ahead_bat out{};
        Errs errs;
        run([&](uint64_t cap) {
                return ahead_gpu_matchjoin_an(ctx, &a, &b, 0, 0, 0, 0, 0, kAoid, &out, cap, errs.v.data());
            },
            std::max<uint64_t>(std::min(a.count, b.count), 1), 4, 1, &out, &errs);
        if (!rc && errs_out) std::copy(errs.v.begin(), errs.v.end(), errs_out);
        return out;
    }
    ahead_bat hashjoin_an(const ahead_bat& l, const ahead_bat& r, int reenc_head, int reenc_tail,
                          ahead_errvec* errs_out = nullptr) {
        ahead_bat out{};
        Errs errs;
        run([&](uint64_t cap) {
                return ahead_gpu_hashjoin_an(ctx, &l, &r, reenc_head, kAr, kArInv, reenc_tail, kAr, kArInv,
                                             AHEAD_HASH_RIGHT, kAoid, &out, cap, errs.v.data());
            },
            std::max(l.count, r.count), 4, 1, &out, &errs);
        if (!rc && errs_out) std::copy(errs.v.begin(), errs.v.end(), errs_out);
        return out;
    }

    // selectAN per predicate on col_of(p), intersected in order with matchjoinAN
    // (ssbm-q11_continuous.cpp:71-79, ssbm-q13_continuous.cpp); the mirrored
    // OID list, and each selection's errors in *errs
    template <typename ColOf, typename Pred>
    ahead_bat select_chain(int n, ColOf col_of, const Pred* preds, std::vector<ahead_errvec>* errs) {
        ahead_bat sel{};
        for (int i = 0; i < n && !rc; ++i) {
            const Pred& p = preds[i];
            ahead_errvec e{};
            ahead_bat s = select_an(col_of(p), p.op1, p.th1, p.op2, p.th2, p.comb, &e);
            if (rc) break;
            if (errs) errs->push_back(e);
            sel = i == 0 ? mirror_head(s) : mirror_head(matchjoin_an(sel, mirror_head(s)));
        }
        return sel;
    }
};

// the dimensions a query joins, in the pipelines' join order
std::vector<int> query_dims(const ahead_sj_query& q) {
    bool used[4] = {false, false, false, false};
    for (int k = 0; k < q.npred; ++k) used[q.pred[k].dim] = true;
    for (int j = 0; j < q.ngroup; ++j) used[q.gdim[j]] = true;
    std::vector<int> out;
    for (int d : {AHEAD_SJ_CUSTOMER, AHEAD_SJ_SUPPLIER, AHEAD_SJ_PART, AHEAD_SJ_DATE})
        if (used[d]) out.push_back(d);
    return out;
}

int copy_tail_u64(Plain& P, const ahead_bat& b, uint64_t* dst) {
    if (!dst || !b.count) return AHEAD_OK;
    const int w = width_of(b.tail.type);
    std::vector<unsigned char> h(b.count * w);
    if (!P.copy(h.data(), b.tail.data, h.size(), cudaMemcpyDeviceToHost)) return AHEAD_CUDA_ERROR;
    for (uint64_t i = 0; i < b.count; ++i) {
        uint64_t v = 0;
        std::memcpy(&v, h.data() + i * w, w);
        dst[i] = v;
    }
    return AHEAD_OK;
}

}  // namespace

extern "C" int ahead_plain_starjoin(ahead_ctx* ctx, const ahead_sj_schema* sch, const ahead_sj_query* q,
                                    ahead_sj_result* res) {
    if (!ctx || !sch || !q || !res) return AHEAD_BAD_ARG;
    const std::vector<int> dims = query_dims(*q);
    if (dims.empty() || q->npred > 4 || q->ngroup > 3 || q->nfpred > 2) return AHEAD_BAD_ARG;
    if (q->measure != AHEAD_SJ_MEASURE_PRICE_DISCOUNT && !q->ngroup) return AHEAD_BAD_ARG;
    if (cudaStreamSynchronize(static_cast<cudaStream_t>(ahead_ctx_stream(ctx))) != cudaSuccess)
        return AHEAD_CUDA_ERROR;
    Plain P{ctx};
    P.arena.init(ctx);
    const uint64_t n = std::min<uint64_t>(q->fact_rows ? q->fact_rows : sch->fact_rows, sch->fact_rows);
    ahead_col vh{};
    vh.type = AHEAD_VOID;
    // the lineorder prefix, by AHEAD_SJ_COL_* index
    const ahead_col* fcol[AHEAD_SJ_NCOL] = {&sch->fk[0], &sch->fk[1], &sch->fk[2], &sch->fk[3], &sch->price,
                                            &sch->discount, &sch->quantity, &sch->revenue, &sch->supplycost};
    auto lo = [&](int c) { return Plain::view(vh, *fcol[c], n); };
    auto dim_bat = [&](int d, const ahead_col& c) { return Plain::view(vh, c, sch->dim[d].rows); };

    // key -> OID maps
    ahead_bat km[4]{};
    for (int d : dims) {
        ahead_bat key = dim_bat(d, sch->dim[d].key);
        std::vector<ahead_sj_pred> preds;
        for (int k = 0; k < q->npred; ++k)
            if (q->pred[k].dim == d) preds.push_back(q->pred[k]);
        if (preds.empty()) {
            km[d] = Plain::reverse(key);
        } else {
            ahead_bat sel = P.select_chain(
                (int)preds.size(), [&](const ahead_sj_pred& p) { return dim_bat(d, sch->dim[d].attr[p.attr]); },
                preds.data(), nullptr);
            km[d] = P.matchjoin_an(Plain::reverse(key), sel);
        }
    }
    ahead_bat joined[4]{}, s{};
    size_t first_todo = 0;
    if (q->nfpred) {
        std::vector<ahead_errvec> errs;
        s = P.select_chain(q->nfpred, [&](const ahead_sj_fpred& p) { return lo(p.col); }, q->fpred, &errs);
        for (int k = 0; k < q->nfpred && !P.rc && k < (int)errs.size(); ++k) P.add_errs(q->fpred[k].col, errs[k]);
    } else {
        const int d0 = dims[0];
        const int void_tail = km[d0].tail.type == AHEAD_VOID;
        ahead_errvec errs[4]{};
        ahead_bat j = P.hashjoin_an(lo(d0), km[d0], 1, void_tail, errs);
        if (!P.rc) P.set_errs(d0, errs[1]);
        joined[d0] = j;
        s = Plain::mirror_head(j);
        first_todo = 1;
    }
    for (size_t i = first_todo; i < dims.size() && !P.rc; ++i) {
        const int d = dims[i];
        ahead_errvec errs[4]{};
        ahead_bat f = P.matchjoin_an(s, lo(d), errs);
        if (P.rc) break;
        P.set_errs(d, errs[3]);
        const int void_tail = km[d].tail.type == AHEAD_VOID;
        joined[d] = P.hashjoin_an(f, km[d], void_tail, void_tail);
        s = Plain::mirror_head(joined[d]);
    }
    // measures, dropped row-consistently
    const int first = q->measure == AHEAD_SJ_MEASURE_PRICE_DISCOUNT ? AHEAD_SJ_COL_PRICE : AHEAD_SJ_COL_REVENUE;
    const int second = q->measure == AHEAD_SJ_MEASURE_PRICE_DISCOUNT ? AHEAD_SJ_COL_DISCOUNT
                       : q->measure == AHEAD_SJ_MEASURE_PROFIT      ? AHEAD_SJ_COL_SUPPLYCOST
                                                                    : -1;
    ahead_errvec e4[4]{};
    ahead_bat m1 = P.matchjoin_an(s, lo(first), e4);
    if (!P.rc) P.add_errs(first, e4[3]);
    ahead_bat s6 = Plain::mirror_head(m1), m2{}, mp = m1;
    if (second >= 0 && !P.rc) {
        m2 = P.matchjoin_an(s6, lo(second), e4);
        if (!P.rc) P.add_errs(second, e4[3]);
        s6 = Plain::mirror_head(m2);
        mp = P.matchjoin_an(s6, m1);
    }
    res->total = 0;
    res->ngroups = 0;
    int status = AHEAD_OK;
    if (!q->ngroup) {
        uint64_t total = 0;
        Errs errs;
        P.run([&](uint64_t) {
                  return ahead_gpu_aggregate_mul_sum_an(ctx, &mp, &m2, AHEAD_RESBIGINT, 0, kAr, kArInv, kAoid, &total,
                                                        errs.v.data());
              },
              std::max(mp.count, m2.count), 2, 0, nullptr, &errs);
        res->total = total;
    } else if (!P.rc) {
        ahead_bat attrs[3]{};
        for (int j = 0; j < q->ngroup && !P.rc; ++j) {
            const int d = q->gdim[j];
            ahead_bat g = P.matchjoin_an(s6, joined[d]);
            attrs[j] = P.matchjoin_an(g, dim_bat(d, sch->dim[d].attr[q->gattr[j]]));
        }
        ahead_bat vals = Plain::clear_head(mp);
        if (q->measure != AHEAD_SJ_MEASURE_REVENUE && !P.rc) {
            const ahead_bat a = Plain::clear_head(mp), b = Plain::clear_head(m2);
            const int op = q->measure == AHEAD_SJ_MEASURE_PROFIT ? AHEAD_SUB : AHEAD_MUL;
            Errs errs;
            P.run([&](uint64_t) {
                      return ahead_gpu_arithmetic_an(ctx, op, AHEAD_RESBIGINT, &a, &b, kAr, kArInv, kAoid, &vals,
                                                     errs.v.data());
                  },
                  a.count, 4, 1, &vals, &errs);
        }
        ahead_bat gids{}, firsts{};
        ahead_bat gb[2]{};
        if (!P.rc) {
            const ahead_bat in = Plain::clear_head(attrs[0]);
            Errs errs;
            P.run([&](uint64_t cap) {
                      return ahead_gpu_groupby_an(ctx, &in, kGroupAoid, kGroupAoidInv, &gb[0], &gb[1], cap,
                                                  errs.v.data());
                  },
                  in.count, 2, 2, gb, &errs);
            gids = gb[0];
            firsts = gb[1];
        }
        for (int j = 1; j < q->ngroup && !P.rc; ++j) {
            const ahead_bat in = Plain::clear_head(attrs[j]), grouping = gids;
            const uint64_t ng = firsts.count;
            Errs errs;
            P.run([&](uint64_t cap) {
                      return ahead_gpu_groupby2_an(ctx, &in, &grouping, ng, kGroupAoid, kGroupAoidInv, &gb[0], &gb[1],
                                                   cap, errs.v.data());
                  },
                  in.count, 3, 2, gb, &errs);
            gids = gb[0];
            firsts = gb[1];
        }
        ahead_bat sums{};
        if (!P.rc) {
            const uint64_t ng = firsts.count;
            Errs errs;
            P.run([&](uint64_t) {
                      return ahead_gpu_aggregate_sum_grouped_an(ctx, &vals, &gids, ng, AHEAD_RESBIGINT, kAr, kArInv,
                                                                kGroupAoid, &sums, errs.v.data());
                  },
                  std::max<uint64_t>(std::max(vals.count, ng), 1), 3, 1, &sums, &errs);
        }
        if (!P.rc) {
            const uint64_t ng = firsts.count;
            res->ngroups = ng;
            if (ng > res->capacity) {
                status = AHEAD_CAPACITY;
            } else {
                for (int j = 0; j < q->ngroup && !P.rc; ++j) {
                    ahead_bat kv = P.matchjoin_an(firsts, Plain::clear_head(attrs[j]));
                    if (!P.rc && copy_tail_u64(P, kv, res->keys[j])) P.fail(AHEAD_CUDA_ERROR);
                }
                if (!P.rc && copy_tail_u64(P, sums, res->sums)) P.fail(AHEAD_CUDA_ERROR);
            }
        }
    }
    if (P.rc) {
        res->status = P.rc;
        return P.rc;
    }
    for (int c = 0; c < AHEAD_SJ_NCOL; ++c) {
        ahead_errvec& E = res->fact_err[c];
        E.present = 1;
        E.count = P.ferr[c].size();
        if (E.data) std::memcpy(E.data, P.ferr[c].data(), std::min(E.count, E.capacity) * 8);
        if (E.count > E.capacity) status = AHEAD_CAPACITY;
    }
    res->status = status;
    return status;
}
