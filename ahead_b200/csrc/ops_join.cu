// ops_join.cu -- hashjoinAN / hashjoin, matchjoinAN / matchjoin and
// fetchjoinAN / fetchjoin.
//
// Hash joins build the table of hash.cuh on the build side (the right BAT by
// default) with keys decoded and cast to the unencoded base type, probe in
// probe-row order and emit every match in build order
// (lib/column_operators/AN/hashjoinAN.tcc:54-223).  Rows with detected errors
// are still built and probed, exactly as in the reference; the four error
// vectors are column checks of the four inputs.
//
// Positional match/fetch joins are compactions over the OID list with a gather
// (matchjoinAN.tcc:226-354).  The merge matchjoin (matchjoinAN.tcc:46-144) is
// an intersection when both inputs are strictly increasing and clean (the
// common case: two selection vectors); otherwise the reference's merge loop is
// replayed step by step on the device so that every error push (including its
// repeated checks of the same row) is reproduced.
#include "hash.cuh"
#include "ops_common.cuh"

using namespace ahead;

namespace {

// --------------------------------------------------------------- hash join
struct KeyCfg {
    DCol col;
    uint64_t ainv, keymask, largermask, condmax;
    int dec, width;
};

AHEAD_DEV bool key_of(const KeyCfg& k, uint64_t row, uint64_t& key) {
    const uint64_t v = load_at(k.col, row);
    const uint64_t d = k.dec ? mulw(v, k.ainv, k.width) : v;
    if ((d & k.largermask) > k.condmax) return false;
    key = d & k.keymask;
    return true;
}

__global__ void ht_build_kernel(HashTab h, KeyCfg kc, uint64_t n, uint32_t* slot_of) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t key = 0;
        key_of(kc, i, key);
        const uint32_t s = ht_insert(h, key);
        slot_of[i] = s;
        atomicAdd(&h.cnt[s], 1u);
    }
}

__global__ void ht_offsets_kernel(HashTab h, CompactBufs cb) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < cb.ntiles; s += gridDim.x * blockDim.x)
        h.off[s] = (uint32_t)(cb.offsets[s] + cb.gbase[s / kScanGroup]);
}

__global__ void ht_fill_kernel(HashTab h, const uint32_t* slot_of, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t s = slot_of[i];
        h.rows[h.off[s] + atomicAdd(&h.cur[s], 1u)] = (uint32_t)i;
    }
}

// Restore build order inside the (rare) segments with several rows.
__global__ void ht_order_kernel(HashTab h, uint32_t nslots) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < nslots; s += gridDim.x * blockDim.x) {
        const uint32_t c = h.cnt[s];
        if (c < 2) continue;
        uint32_t* r = h.rows + h.off[s];
        for (uint32_t i = 1; i < c; ++i) {
            const uint32_t x = r[i];
            uint32_t j = i;
            while (j > 0 && r[j - 1] > x) {
                r[j] = r[j - 1];
                --j;
            }
            r[j] = x;
        }
    }
}

struct JoinOut {
    DCol pcol, bcol;  // probe-side and build-side output columns
    uint64_t fh, ft, cap;
    void *oh, *ot;
    int probe_is_head, rh, rt, ohw, otw;
};

AHEAD_DEV void join_emit(const JoinOut& o, uint64_t pos, uint64_t prow, uint64_t brow) {
    if (pos >= o.cap) return;
    uint64_t hv = o.probe_is_head ? load_at(o.pcol, prow) : load_at(o.bcol, brow);
    uint64_t tv = o.probe_is_head ? load_at(o.bcol, brow) : load_at(o.pcol, prow);
    if (o.rh) hv *= o.fh;
    if (o.rt) tv *= o.ft;
    store_at(o.oh, o.ohw, pos, hv);
    store_at(o.ot, o.otw, pos, tv);
}

constexpr int kProbeRowsPerThread = 16;
// a probe row's entry: kNoSlot, the single matching build row | kDirect, or
// the slot of a key with several build rows
constexpr uint32_t kDirect = 0x80000000u;

// the packed probe table (after the build's order step)
__global__ void ht_pack_kernel(HashTab h, ProbeSlot* t, uint32_t nslots, bool direct) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < nslots; s += gridDim.x * blockDim.x) {
        ProbeSlot e;
        e.key = h.keys[s];
        e.cnt = h.cnt[s];
        e.first = (direct && e.cnt == 1) ? h.rows[h.off[s]] : h.off[s];
        t[s] = e;
    }
}

// Pass A: find every probe row's slot and count its matches per tile.
__global__ void __launch_bounds__(256) probe_count_kernel(const ProbeSlot* __restrict__ pt, uint32_t mask, bool direct,
                                                          KeyCfg pk, uint64_t n, uint32_t* pslot, CompactBufs cb) {
    __shared__ uint32_t s_w[8];
    for (uint32_t tile = blockIdx.x; tile < cb.ntiles; tile += gridDim.x) {
        uint32_t c = 0;
#pragma unroll 4
        for (int k = 0; k < kProbeRowsPerThread; ++k) {
            const uint64_t row = (uint64_t)tile * kTileRows + k * 256 + threadIdx.x;
            if (row >= n) break;
            uint64_t key = 0;
            uint32_t s = kNoSlot;
            ProbeSlot e;
            if (key_of(pk, row, key)) s = ps_find(pt, mask, key, e);
            if (s != kNoSlot) {
                c += e.cnt;
                if (direct && e.cnt == 1) s = e.first | kDirect;
            }
            pslot[row] = s;
        }
        c = __reduce_add_sync(kFull, c);
        if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = c;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t t = 0;
            for (int w = 0; w < 8; ++w) t += s_w[w];
            cb.counts[tile] = t;
        }
        __syncthreads();
    }
}

// Pass C: each thread owns 16 consecutive probe rows; a block scan of their
// match counts gives every row its output position.
__global__ void __launch_bounds__(256) probe_emit_kernel(const ProbeSlot* __restrict__ pt, const uint32_t* rows,
                                                         uint64_t n, const uint32_t* pslot, CompactBufs cb, JoinOut o) {
    __shared__ uint32_t s_w[8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t tile = blockIdx.x; tile < cb.ntiles; tile += gridDim.x) {
        const uint64_t r0 = (uint64_t)tile * kTileRows + (uint64_t)threadIdx.x * kProbeRowsPerThread;
        uint32_t c = 0;
        for (int k = 0; k < kProbeRowsPerThread; ++k) {
            const uint64_t row = r0 + k;
            if (row >= n) break;
            const uint32_t s = pslot[row];
            if (s != kNoSlot) c += (s & kDirect) ? 1u : pt[s].cnt;
        }
        const uint32_t incl = warp_incl_scan(c);
        if (lane == 31) s_w[warp] = incl;
        __syncthreads();
        uint64_t pos = cb.offsets[tile] + cb.gbase[tile / kScanGroup] + incl - c;
        for (int w = 0; w < warp; ++w) pos += s_w[w];
        __syncthreads();
        if (!c) continue;
        for (int k = 0; k < kProbeRowsPerThread; ++k) {
            const uint64_t row = r0 + k;
            if (row >= n) break;
            const uint32_t s = pslot[row];
            if (s == kNoSlot) continue;
            if (s & kDirect) {
                join_emit(o, pos++, row, s & ~kDirect);
                continue;
            }
            const ProbeSlot e = pt[s];
            for (uint32_t j = 0; j < e.cnt; ++j) join_emit(o, pos++, row, rows[e.first + j]);
        }
    }
}

size_t join_scratch(uint64_t nb, uint64_t np) {
    const uint64_t cap = ht_capacity(nb) + 1;
    return cap * (8 + 4 + 4 + 4 + 8 + 16) + 256 + nb * 8 + np * 4 + compact_bytes(compact_tiles(cap), 1) +
           compact_bytes(compact_tiles(np), 1) + 8 * 1024;
}

// Build on `bk` (nb rows), probe with `pk` (np rows); the output total lands
// in counter `ci`.
void run_hash_join(OpScope& s, const KeyCfg& bk, uint64_t nb, const KeyCfg& pk, uint64_t np, const JoinOut& o,
                   int ci) {
    cudaStream_t st = s.ctx->stream;
    const uint32_t cap = ht_capacity(nb);
    HashTab h;
    h.mask = cap - 1;
    h.keys = (uint64_t*)s.alloc((size_t)(cap + 1) * 8);
    h.cnt = (uint32_t*)s.alloc((size_t)(cap + 1) * 4);
    h.off = (uint32_t*)s.alloc((size_t)(cap + 1) * 4);
    h.cur = (uint32_t*)s.alloc((size_t)(cap + 1) * 4);
    h.rows = (uint32_t*)s.alloc(nb * 4 + 4);
    uint32_t* slot_of = (uint32_t*)s.alloc(nb * 4 + 4);
    uint32_t* pslot = (uint32_t*)s.alloc(np * 4 + 4);
    cudaMemsetAsync(h.keys, 0xff, (size_t)(cap + 1) * 8, st);
    cudaMemsetAsync(h.cnt, 0, (size_t)(cap + 1) * 4, st);
    cudaMemsetAsync(h.cur, 0, (size_t)(cap + 1) * 4, st);
    const int g = s.ctx->num_sms * 8;
    ht_build_kernel<<<grid_for(nb, 256), 256, 0, st>>>(h, bk, nb, slot_of);
    // segment starts: scan of the slot counts (the compaction's two-level scan)
    CompactBufs sb;
    sb.words = nullptr;
    sb.counts = h.cnt;
    sb.offsets = (uint64_t*)s.alloc((size_t)(cap + 1) * 8);
    sb.gbase = (uint64_t*)s.alloc((size_t)scan_groups(cap + 1) * 8);
    sb.totals = s.d_counters + 60;
    sb.ntiles = cap + 1;
    sb.nchan = 1;
    tile_scan_kernel<<<scan_groups(cap + 1), kScanGroup, 0, st>>>(sb);
    group_scan_kernel<<<1, 1024, 0, st>>>(sb);
    ht_offsets_kernel<<<grid_for(cap + 1, 256), 256, 0, st>>>(h, sb);
    ht_fill_kernel<<<grid_for(nb, 256), 256, 0, st>>>(h, slot_of, nb);
    ht_order_kernel<<<grid_for(cap + 1, 256), 256, 0, st>>>(h, cap + 1);
    // single build rows go straight into the probe entries while rows fit 31 bits
    const bool direct = nb < (uint64_t)(kDirect - 1);
    ProbeSlot* pt = (ProbeSlot*)s.alloc((size_t)(cap + 1) * sizeof(ProbeSlot));
    ht_pack_kernel<<<grid_for(cap + 1, 256), 256, 0, st>>>(h, pt, cap + 1, direct);
    s.launched(7);
    if (!np) return;
    const uint32_t nt = compact_tiles(np);
    CompactBufs pb;
    pb.words = nullptr;
    pb.counts = (uint32_t*)s.alloc((size_t)nt * 4);
    pb.offsets = (uint64_t*)s.alloc((size_t)nt * 8);
    pb.gbase = (uint64_t*)s.alloc((size_t)scan_groups(nt) * 8);
    pb.totals = s.d_counters + ci;
    pb.ntiles = nt;
    pb.nchan = 1;
    const uint32_t pg = nt < (uint32_t)g ? nt : (uint32_t)g;
    probe_count_kernel<<<pg, 256, 0, st>>>(pt, h.mask, direct, pk, np, pslot, pb);
    tile_scan_kernel<<<scan_groups(nt), kScanGroup, 0, st>>>(pb);
    group_scan_kernel<<<1, 1024, 0, st>>>(pb);
    probe_emit_kernel<<<pg, 256, 0, st>>>(pt, h.rows, np, pslot, pb, o);
    s.launched(4);
}

bool small_res(int t) { return t == AHEAD_RESTINY || t == AHEAD_RESSHORT || t == AHEAD_RESINT; }

KeyCfg key_cfg(const ahead_col& c, int dec, int keybase, int largerbase, bool cond) {
    KeyCfg k;
    k.col = dcol(c);
    k.width = type_width(c.type);
    k.dec = dec;
    k.ainv = c.Ainv & wmask(k.width);
    k.keymask = wmask(keybase);
    k.largermask = wmask(largerbase);
    k.condmax = cond ? wmask(keybase) : ~0ull;
    return k;
}

// ------------------------------------------------------ positional joins
// matchjoinAN<H1, resoid, void, T2> (matchjoinAN.tcc:271-298) and, with
// CHECKED = false, the unencoded matchjoin<H1, oid, void, T2>
// (Normal/matchjoin.tcc:140-157).  Streams: 0 kept, 1 bad head, 2 bad
// position, 3 corrupt fetched value.
template <bool CHECKED>
struct MjPosOp {
    static constexpr int W = CHECKED ? 8 : 4;
    static constexpr int NCH = CHECKED ? 4 : 1;
    static constexpr bool ACC = false;
    static constexpr bool EMIT_V = true;
    static constexpr int NOUT = 2;
    const char* base;
    uint32_t* status;
    DCol h1c, t2c;
    uint64_t at1inv, ah1inv, ah1max, sz, fh, ft, cap, aoid, ec1, ec2, ec4;
    uint64_t *e1, *e2, *e4, *acc;
    void *oh, *ot;
    int ohw, otw, reenc, h1enc, t2enc;
    AHEAD_DEV uint64_t pos2(uint64_t v) const { return CHECKED ? v * at1inv : v; }
    AHEAD_DEV uint32_t eval(uint64_t v, uint64_t row, uint64_t&) const {
        uint32_t bits = 0;
        if (CHECKED && h1enc && load_at(h1c, row) * ah1inv > ah1max) bits |= 2u;
        const uint64_t p = pos2(v);
        if (p >= sz) return bits | (CHECKED ? 4u : 0u);
        if (CHECKED && t2enc && dec_if(t2c, load_at(t2c, p), t2c.ainv) > t2c.umax) return bits | 8u;
        return bits | 1u;
    }
    AHEAD_DEV uint64_t out0(int k, uint64_t v, uint64_t row) const {
        if (k == 0) {
            const uint64_t h = load_at(h1c, row);
            return reenc ? dec_if(h1c, h, fh) : h;
        }
        const uint64_t t = load_at(t2c, pos2(v));
        return reenc ? dec_if(t2c, t, ft) : t;
    }
    AHEAD_DEV void put0(int k, uint64_t pos, uint64_t val) const {
        if (pos < cap) store_at(k == 0 ? oh : ot, k == 0 ? ohw : otw, pos, val);
    }
    AHEAD_DEV void emit(int c, uint64_t pos, uint64_t v, uint64_t row) const {
        if (c == 1) {
            if (pos < ec1) e1[pos] = row * aoid;
        } else if (c == 2) {
            if (pos < ec2) e2[pos] = row * aoid;
        } else if (c == 3) {
            if (pos < ec4) e4[pos] = pos2(v) * aoid;
        }
    }
};

// fetchjoinAN (matchjoinAN.tcc:330-351) and, with CHECKED = false, fetchjoin
// (Normal/matchjoin.tcc:159-178).  Streams: 0 kept, 1 bad OID, 2 corrupt value.
template <bool CHECKED>
struct FetchOp {
    static constexpr int W = CHECKED ? 8 : 4;
    static constexpr int NCH = CHECKED ? 3 : 1;
    static constexpr bool ACC = false;
    static constexpr bool EMIT_V = true;
    static constexpr int NOUT = 1;
    const char* base;
    uint32_t* status;
    DCol t2c;
    uint64_t at1inv, at2inv, at2max, vsz, fac, cap, aoid, ec1, ec2;
    uint64_t *e1, *e2, *acc;
    void* ot;
    int otw, reenc, w2;
    AHEAD_DEV uint64_t pos(uint64_t v) const { return CHECKED ? v * at1inv : v; }
    AHEAD_DEV bool bad(uint64_t t2) const {
        // the check has no cast: 16-bit codes are multiplied as 32-bit ints
        if (w2 == 2) return (int32_t)(uint32_t)(t2 * at2inv) > (int32_t)at2max;
        return mulw(t2, at2inv, w2) > at2max;
    }
    AHEAD_DEV uint32_t eval(uint64_t v, uint64_t, uint64_t&) const {
        const uint64_t p = pos(v);
        if (p >= vsz) return CHECKED ? 2u : 0u;
        if (CHECKED && bad(load_at(t2c, p))) return 4u;
        return 1u;
    }
    AHEAD_DEV uint64_t out0(int, uint64_t v, uint64_t) const {
        const uint64_t t = load_at(t2c, pos(v));
        return reenc ? mulw(t, fac, w2) : t;
    }
    AHEAD_DEV void put0(int, uint64_t p, uint64_t val) const {
        if (p < cap) store_at(ot, otw, p, val);
    }
    AHEAD_DEV void emit(int c, uint64_t p, uint64_t v, uint64_t row) const {
        if (c == 1) {
            if (p < ec1) e1[p] = row * aoid;
        } else if (c == 2) {
            if (p < ec2) e2[p] = pos(v) * aoid;
        }
    }
};

// ------------------------------------------------------------ merge joins
struct MergeSide {
    DCol key, other;  // key column (decoded when encoded) and the other column
    int key_enc, other_enc;
};

AHEAD_DEV uint64_t key_val(const DCol& c, uint64_t row) { return dec_if(c, load_at(c, row), c.ainv); }

// Flags (bit 0) a key that does not strictly increase -- the parallel merge
// is exact only without one -- and (bit 1) any corrupt value in either column,
// which decides whether error positions must be produced.
__global__ void merge_check_kernel(MergeSide m, uint64_t n, uint32_t* flag) {
    uint32_t f = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = key_val(m.key, i);
        if ((m.key_enc && k > m.key.umax) ||
            (m.other_enc && dec_if(m.other, load_at(m.other, i), m.other.ainv) > m.other.umax))
            f |= 2u;
        if (i > 0 && key_val(m.key, i - 1) >= k) f |= 1u;
    }
    if (f) atomicOr(flag, f);
}

// Error positions of the reference's merge loop (matchjoinAN.tcc:101-136) for
// two strictly increasing key sequences, derived per row instead of by running
// the loop.  Walking the loop over the merged order of the keys shows:
//  - a first-input row is checked once, when the inner p1 loop passes it:
//    exactly when it is unmatched and some second-input key is larger
//    (matched rows are emitted unchecked);
//  - a second-input row j is checked at the top of an outer iteration when
//    j == 0, row j-1 matched, or a first-input key lies strictly between keys
//    j-1 and j; an unmatched row is checked again when the inner p2 loop
//    passes it, which happens when a larger first-input key exists; without
//    one, only the first unmatched row after the last first-input key is
//    checked (once), and only when that last key is itself unmatched (a match
//    of the last first-input key ends the loop).
// Each check pushes `row * AOID` into the vector of each corrupt column.
struct MergeErrs {
    DCol h1, t1, h2, t2;
    uint64_t n1, n2, aoid;
    int eh1, et1, eh2, et2;
    uint64_t last2;           // key of the last second-input row
    const uint64_t* l1m;      // device word: the last first-input key occurs in the second input
    AHEAD_DEV uint64_t lb1(uint64_t x) const {  // first-input keys below x
        uint64_t lo = 0, hi = n1;
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if (key_val(t1, mid) < x) lo = mid + 1;
            else hi = mid;
        }
        return lo;
    }
    AHEAD_DEV bool in2(uint64_t k) const {
        uint64_t lo = 0, hi = n2;
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if (key_val(h2, mid) < k) lo = mid + 1;
            else hi = mid;
        }
        return lo < n2 && key_val(h2, lo) == k;
    }
    // checks of row r of `side` (0: first input, 1: second) and which of its
    // two columns are corrupt
    AHEAD_DEV uint32_t checks(int side, uint64_t r, bool& bad_a, bool& bad_b) const {
        if (side == 0) {
            const uint64_t k = key_val(t1, r);
            bad_a = eh1 && key_val(h1, r) > h1.umax;
            bad_b = et1 && k > t1.umax;
            if (!(bad_a || bad_b)) return 0;
            return (k < last2 && !in2(k)) ? 1u : 0u;
        }
        const uint64_t K = key_val(h2, r);
        bad_a = eh2 && K > h2.umax;
        bad_b = et2 && key_val(t2, r) > t2.umax;
        if (!(bad_a || bad_b)) return 0;
        const uint64_t L = lb1(K);
        const bool matched = L < n1 && key_val(t1, L) == K;
        bool top = r == 0;
        uint64_t upto_prev = 0;  // first-input keys <= key r-1
        if (r > 0) {
            const uint64_t Kp = key_val(h2, r - 1);
            const uint64_t Lp = lb1(Kp);
            const bool mp = Lp < n1 && key_val(t1, Lp) == Kp;
            upto_prev = Lp + (mp ? 1 : 0);
            top = mp || L > upto_prev;
        }
        if (matched) return top ? 1u : 0u;
        if (L < n1) return (top ? 1u : 0u) + 1u;
        return ((r == 0 || upto_prev < n1) && !*l1m) ? 1u : 0u;
    }
};

constexpr int kMeRows = 16;
constexpr int kMeThreads = 256;
constexpr int kMeTile = kMeRows * kMeThreads;

__global__ void merge_last_kernel(MergeErrs m, uint64_t* out) { out[0] = m.in2(key_val(m.t1, m.n1 - 1)) ? 1 : 0; }

// Exclusive scan of two counters over a block of kMeThreads threads.
AHEAD_DEV void block_scan2(uint32_t& a, uint32_t& b, uint32_t* tot_a, uint32_t* tot_b) {
    __shared__ uint32_t s_a[kMeThreads / 32], s_b[kMeThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint32_t ia = warp_incl_scan(a), ib = warp_incl_scan(b);
    if (lane == 31) {
        s_a[wid] = ia;
        s_b[wid] = ib;
    }
    __syncthreads();
    uint32_t pa = 0, pb = 0, ta = 0, tb = 0;
    for (int w = 0; w < kMeThreads / 32; ++w) {
        if (w < wid) {
            pa += s_a[w];
            pb += s_b[w];
        }
        ta += s_a[w];
        tb += s_b[w];
    }
    a = pa + ia - a;
    b = pb + ib - b;
    *tot_a = ta;
    *tot_b = tb;
    __syncthreads();
}

__global__ void __launch_bounds__(kMeThreads) merge_err_count_kernel(MergeErrs m, int side, uint64_t n,
                                                                     uint32_t* tcount) {
    const uint64_t t0 = (uint64_t)blockIdx.x * kMeTile;
    uint32_t ca = 0, cb = 0;
    for (int k = 0; k < kMeRows; ++k) {
        const uint64_t r = t0 + (uint64_t)threadIdx.x * kMeRows + k;
        if (r >= n) break;
        bool ba, bb;
        const uint32_t c = m.checks(side, r, ba, bb);
        ca += ba ? c : 0;
        cb += bb ? c : 0;
    }
    uint32_t ta, tb;
    block_scan2(ca, cb, &ta, &tb);
    if (threadIdx.x == 0) {
        tcount[2 * blockIdx.x] = ta;
        tcount[2 * blockIdx.x + 1] = tb;
    }
}

// One block: exclusive offsets of the tile counts; totals into tot[0], tot[1].
__global__ void __launch_bounds__(kMeThreads) merge_err_scan_kernel(const uint32_t* tcount, uint64_t* toff,
                                                                    uint32_t ntiles, uint64_t* tot) {
    __shared__ uint64_t s_base[2];
    if (threadIdx.x == 0) s_base[0] = s_base[1] = 0;
    __syncthreads();
    for (uint32_t c0 = 0; c0 < ntiles; c0 += kMeThreads) {
        const uint32_t t = c0 + threadIdx.x;
        uint32_t a = t < ntiles ? tcount[2 * t] : 0, b = t < ntiles ? tcount[2 * t + 1] : 0;
        uint32_t ta, tb;
        block_scan2(a, b, &ta, &tb);
        if (t < ntiles) {
            toff[2 * t] = s_base[0] + a;
            toff[2 * t + 1] = s_base[1] + b;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            s_base[0] += ta;
            s_base[1] += tb;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        tot[0] = s_base[0];
        tot[1] = s_base[1];
    }
}

__global__ void __launch_bounds__(kMeThreads) merge_err_write_kernel(MergeErrs m, int side, uint64_t n,
                                                                     const uint64_t* toff, uint64_t* ea,
                                                                     uint64_t capa, uint64_t* eb, uint64_t capb) {
    const uint64_t t0 = (uint64_t)blockIdx.x * kMeTile;
    uint32_t ca = 0, cb = 0;
    uint32_t mult[kMeRows];
    uint32_t bad[kMeRows];
    for (int k = 0; k < kMeRows; ++k) {
        const uint64_t r = t0 + (uint64_t)threadIdx.x * kMeRows + k;
        mult[k] = 0;
        bad[k] = 0;
        if (r < n) {
            bool ba, bb;
            mult[k] = m.checks(side, r, ba, bb);
            bad[k] = (ba ? 1u : 0u) | (bb ? 2u : 0u);
            ca += ba ? mult[k] : 0;
            cb += bb ? mult[k] : 0;
        }
    }
    uint32_t ta, tb;
    block_scan2(ca, cb, &ta, &tb);
    uint64_t pa = toff[2 * blockIdx.x] + ca, pb = toff[2 * blockIdx.x + 1] + cb;
    for (int k = 0; k < kMeRows; ++k) {
        const uint64_t r = t0 + (uint64_t)threadIdx.x * kMeRows + k;
        for (uint32_t c = 0; c < mult[k]; ++c) {
            if (bad[k] & 1u) {
                if (ea && pa < capa) ea[pa] = r * m.aoid;
                ++pa;
            }
            if (bad[k] & 2u) {
                if (eb && pb < capb) eb[pb] = r * m.aoid;
                ++pb;
            }
        }
    }
}

// Bounds of a strictly increasing key sequence: [0] first key, [1] last key.
__global__ void isect_bounds_kernel(DCol h2, uint64_t n2, uint64_t* out) {
    out[0] = key_val(h2, 0);
    out[1] = key_val(h2, n2 - 1);
}

// Rank structure of a strictly increasing clean key sequence over
// [kmin, kmin + 64 * words): bit (k - kmin) is set for each key, and first[w]
// is the index of the first key in 64-bit word w (set only for non-empty
// words, the only ones a lookup reads).
__global__ void isect_mark_kernel(DCol h2, uint64_t n2, uint64_t kmin, unsigned long long* bits, uint32_t* first) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n2; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t d = key_val(h2, i) - kmin;
        const uint64_t w = d >> 6;
        atomicOr(&bits[w], 1ull << (d & 63));
        if (i == 0 || ((key_val(h2, i - 1) - kmin) >> 6) != w) first[w] = (uint32_t)i;
    }
}

// Intersection of two strictly increasing clean key sequences: each row of the
// first input looks its key up in the second, through the rank structure when
// the second's key range is dense enough, else by binary search.
struct IsectOp {
    static constexpr int W = 8;
    static constexpr int NCH = 1;
    static constexpr bool ACC = false;
    static constexpr bool EMIT_V = false;
    static constexpr int NOUT = 2;
    const char* base;
    uint32_t* status;
    DCol t1c, h1c, h2c, t2c;
    uint64_t n2, fh, ft, cap;
    uint64_t* acc;
    void *oh, *ot;
    int ohw, otw, reenc;
    const unsigned long long* bits;  // rank structure, or nullptr
    const uint32_t* first;
    uint64_t kmin, krange;
    AHEAD_DEV uint64_t find(uint64_t row) const {
        const uint64_t k = key_val(t1c, row);
        if (bits) {
            const uint64_t d = k - kmin;
            if (k < kmin || d >= krange) return ~0ull;
            const unsigned long long wv = bits[d >> 6];
            if (!((wv >> (d & 63)) & 1ull)) return ~0ull;
            return first[d >> 6] + __popcll(wv & ((1ull << (d & 63)) - 1ull));
        }
        uint64_t lo = 0, hi = n2;
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if (key_val(h2c, mid) < k) lo = mid + 1;
            else hi = mid;
        }
        return (lo < n2 && key_val(h2c, lo) == k) ? lo : ~0ull;
    }
    AHEAD_DEV uint32_t eval(uint64_t, uint64_t row, uint64_t&) const { return find(row) != ~0ull ? 1u : 0u; }
    AHEAD_DEV uint64_t out0(int k, uint64_t, uint64_t row) const {
        if (k == 0) {
            const uint64_t h = load_at(h1c, row);
            return reenc ? dec_if(h1c, h, fh) : h;
        }
        const uint64_t t = load_at(t2c, find(row));
        return reenc ? dec_if(t2c, t, ft) : t;
    }
    AHEAD_DEV void put0(int k, uint64_t pos, uint64_t val) const {
        if (pos < cap) store_at(k == 0 ? oh : ot, k == 0 ? ohw : otw, pos, val);
    }
    AHEAD_DEV void emit(int, uint64_t, uint64_t, uint64_t) const {}
};

// Intersection of two strictly increasing plain key sequences (binary search
// in the second); the driving column (the first input's keys, or its head when
// the tail is void) is W bytes wide.
template <int WW>
struct IsectPlainOp {
    static constexpr int W = WW;
    static constexpr int NCH = 1;
    static constexpr bool ACC = false;
    static constexpr bool EMIT_V = false;
    static constexpr int NOUT = 2;
    const char* base;
    uint32_t* status;
    DCol t1c, h1c, h2c, t2c;
    uint64_t n2, cap;
    uint64_t* acc;
    void *oh, *ot;
    int ohw, otw;
    AHEAD_DEV uint64_t find(uint64_t row) const {
        const uint64_t k = key_val(t1c, row);
        uint64_t lo = 0, hi = n2;
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if (key_val(h2c, mid) < k) lo = mid + 1;
            else hi = mid;
        }
        return (lo < n2 && key_val(h2c, lo) == k) ? lo : ~0ull;
    }
    AHEAD_DEV uint32_t eval(uint64_t, uint64_t row, uint64_t&) const { return find(row) != ~0ull ? 1u : 0u; }
    AHEAD_DEV uint64_t out0(int k, uint64_t, uint64_t row) const {
        return k == 0 ? load_at(h1c, row) : load_at(t2c, find(row));
    }
    AHEAD_DEV void put0(int k, uint64_t pos, uint64_t val) const {
        if (pos < cap) store_at(k == 0 ? oh : ot, k == 0 ? ohw : otw, pos, val);
    }
    AHEAD_DEV void emit(int, uint64_t, uint64_t, uint64_t) const {}
};

struct MergeSeq {
    DCol h1, t1, h2, t2;
    uint64_t n1, n2, fh, ft, aoid, cap;
    uint64_t ecap[4];
    uint64_t* e[4];
    void *oh, *ot;
    int ohw, otw, reenc, checked;
};

// The reference's merge loop (matchjoinAN.tcc:101-136, Normal/matchjoin.tcc:
// 49-72), one thread, for inputs that are not strictly increasing and clean.
// Counters: [0] output rows, [1..4] error counts.
__global__ void merge_seq_kernel(MergeSeq m, uint64_t* counters) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    uint64_t nout = 0, ne[4] = {0, 0, 0, 0};
    auto push = [&](int v, uint64_t pos) {
        if (!m.checked || !m.e[v]) {
            ++ne[v];
            return;
        }
        if (ne[v] < m.ecap[v]) m.e[v][ne[v]] = pos * m.aoid;
        ++ne[v];
    };
    const bool eh1 = m.checked && m.h1.enc, et1 = m.checked && m.t1.enc, eh2 = m.checked && m.h2.enc,
               et2 = m.checked && m.t2.enc;
    uint64_t p1 = 0, p2 = 0;
    while (p1 < m.n1 && p2 < m.n2) {
        uint64_t h2 = key_val(m.h2, p2);
        if (eh2 && h2 > m.h2.umax) push(2, p2);
        if (et2 && key_val(m.t2, p2) > m.t2.umax) push(3, p2);
        uint64_t t1 = key_val(m.t1, p1);
        bool valid;
        while ((valid = p1 < m.n1) && t1 < h2) {
            if (eh1 && key_val(m.h1, p1) > m.h1.umax) push(0, p1);
            if (et1 && t1 > m.t1.umax) push(1, p1);
            ++p1;
            if (p1 < m.n1) t1 = key_val(m.t1, p1);
        }
        if (valid) {
            while ((valid = p2 < m.n2) && t1 > h2) {
                if (eh2 && h2 > m.h2.umax) push(2, p2);
                if (et2 && key_val(m.t2, p2) > m.t2.umax) push(3, p2);
                ++p2;
                if (p2 < m.n2) h2 = key_val(m.h2, p2);
            }
            if (valid && t1 == h2) {
                if (nout < m.cap) {
                    uint64_t hv = load_at(m.h1, p1), tv = load_at(m.t2, p2);
                    if (m.reenc) {
                        hv = dec_if(m.h1, hv, m.fh);
                        tv = dec_if(m.t2, tv, m.ft);
                    }
                    store_at(m.oh, m.ohw, nout, hv);
                    store_at(m.ot, m.otw, nout, tv);
                }
                ++nout;
                ++p1;
                ++p2;
            }
        }
    }
    counters[0] = nout;
    for (int v = 0; v < 4; ++v) counters[1 + v] = ne[v];
}

__global__ void zip_kernel(DCol h1, DCol t2, uint64_t p1, uint64_t p2, uint64_t m, int reenc, uint64_t fh, uint64_t ft,
                           void* oh, int ohw, void* ot, int otw, uint64_t cap) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m && i < cap;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t hv = load_at(h1, p1 + i), tv = load_at(t2, p2 + i);
        if (reenc) {
            hv = dec_if(h1, hv, fh);
            tv = dec_if(t2, tv, ft);
        }
        store_at(oh, ohw, i, hv);
        store_at(ot, otw, i, tv);
    }
}

// Leading rows skipped before the zip of a void-void positional join
// (matchjoinAN.tcc:185-196): rows whose dense OID (mod 2^32) lies below the
// other side's seqbase.
uint64_t vv_skip(uint64_t my_seq, uint64_t other_seq, uint64_t n) {
    if (other_seq >= (1ull << 32)) return n;
    const uint64_t s0 = my_seq & 0xffffffffull;
    if (s0 >= other_seq) return 0;
    const uint64_t k = other_seq - s0;
    return k < n ? k : n;
}

struct CommonMj {
    int H1, T1, H2, T2;
};

void set_errs_present(ahead_errvec* errs, int p0, int p1, int p2, int p3) {
    if (!errs) return;
    ev_begin(&errs[0], p0);
    ev_begin(&errs[1], p1);
    ev_begin(&errs[2], p2);
    ev_begin(&errs[3], p3);
}

ahead_errvec* ev(ahead_errvec* errs, int k) { return errs ? &errs[k] : nullptr; }

// The string hash join's second step: copy each emitted row's matched
// right slot, and decode the left head where the reference emits it decoded.
__global__ void __launch_bounds__(256) str_gather_kernel(const uint32_t* rows, uint64_t n, const char* strs,
                                                         uint64_t width, char* out, bool decode, uint64_t ainv,
                                                         void* head, int hw) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const char* src = strs + (uint64_t)rows[i] * width;
        char* dst = out + i * width;
        for (uint64_t k = 0; k < width; ++k) dst[k] = src[k];
        if (decode) {
            if (hw == 8) ((uint64_t*)head)[i] *= ainv;
            else ((uint32_t*)head)[i] *= (uint32_t)ainv;
        }
    }
}

// fetchjoinAN with a string tail (FetchjoinAN<v2_str_t, false>,
// matchjoinAN.tcc:304-354): stream 0 = the rows whose OID is inside the
// column, written as their source row (the slots are gathered afterwards);
// stream 1 = the rest, reported as row * AOID.  The string tail is not
// encoded, so nothing else is checked.
struct FetchStrOp {
    static constexpr int W = 8;
    static constexpr int NCH = 2;
    static constexpr bool ACC = false;
    static constexpr bool EMIT_V = true;
    static constexpr int NOUT = 1;
    const char* base;
    uint32_t* status;
    uint64_t ainv, count, aoid, cap, errcap;
    uint32_t* rows;
    uint64_t* err;
    uint64_t* acc;
    AHEAD_DEV uint32_t eval(uint64_t v, uint64_t, uint64_t&) const { return v * ainv < count ? 1u : 2u; }
    AHEAD_DEV uint64_t out0(int, uint64_t v, uint64_t) const { return v * ainv; }
    AHEAD_DEV void put0(int, uint64_t pos, uint64_t val) const {
        if (pos < cap) rows[pos] = (uint32_t)val;
    }
    AHEAD_DEV void emit(int c, uint64_t pos, uint64_t v, uint64_t row) const {
        if (c == 0) put0(0, pos, out0(0, v, row));
        else if (pos < errcap) err[pos] = row * aoid;
    }
};

// fetchjoin over a string tail (Normal/matchjoin.tcc:144-160): the rows whose
// oid_t is inside the column, as their source row; no checks.
struct FetchStrPlainOp {
    static constexpr int W = 4;
    static constexpr int NCH = 1;
    static constexpr bool ACC = false;
    static constexpr bool EMIT_V = true;
    static constexpr int NOUT = 1;
    const char* base;
    uint32_t* status;
    uint64_t count, cap;
    uint32_t* rows;
    uint64_t* acc;
    AHEAD_DEV uint32_t eval(uint64_t v, uint64_t, uint64_t&) const { return v < count ? 1u : 0u; }
    AHEAD_DEV uint64_t out0(int, uint64_t v, uint64_t) const { return v; }
    AHEAD_DEV void put0(int, uint64_t pos, uint64_t val) const {
        if (pos < cap) rows[pos] = (uint32_t)val;
    }
    AHEAD_DEV void emit(int, uint64_t pos, uint64_t v, uint64_t) const { put0(0, pos, v); }
};

// The slots of a compacted row list, into `out` (the second step of both string fetch-joins).
int gather_str_rows(ahead_ctx* ctx, const uint32_t* rows, uint64_t n, const char* strs, uint64_t width, char* out) {
    if (!n || !out) return AHEAD_OK;
    str_gather_kernel<<<grid_for(n, 256), 256, 0, ctx->stream>>>(rows, n, strs, width, out, false, 0, nullptr, 8);
    ctx->launches += 1;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(ctx, e, "kernel launch");
    e = cudaStreamSynchronize(ctx->stream);
    return e == cudaSuccess ? AHEAD_OK : cuda_fail(ctx, e, "cudaStreamSynchronize");
}

}  // namespace

namespace ahead {
int restiny_promoted_check(ahead_ctx* ctx, const uint16_t* codes, uint64_t n, uint32_t ainv, uint32_t umax,
                           uint64_t aoid, ahead_errvec* err);
}

extern "C" {

int ahead_gpu_hashjoin_str_an(ahead_ctx* ctx, const ahead_bat* l, const ahead_bat* r, const char* r_strs,
                              uint64_t width, int reenc_head, uint64_t ah1r, uint64_t ah1invr, int side,
                              uint64_t aoid, ahead_bat* out, uint64_t cap, ahead_errvec* errs) {
    if (!ctx || !l || !r || !out) return AHEAD_BAD_ARG;
    if (r->count && (!r_strs || width == 0))
        return fail(ctx, AHEAD_BAD_ARG, "hashjoinAN(str): right string slots required");
    // The join itself, with the right tail as the void row ids 0..n-1: its
    // tail output is the matched right row, in the reference's emit order.
    ahead_bat rr = *r;
    rr.tail = ahead_col{};
    rr.tail.type = AHEAD_VOID;
    uint32_t* rows = nullptr;
    const uint64_t rcap = (out->head.data && out->tail.data) ? cap : 0;
    if (rcap) AHEAD_CUDA(ctx, cudaMallocAsync((void**)&rows, rcap * 4, ctx->stream));
    ahead_bat o = *out;
    o.tail.data = rows;
    int rc = ahead_gpu_hashjoin_an(ctx, l, &rr, reenc_head, ah1r, ah1invr, 0, 1, 1, side, aoid, &o, rcap, errs);
    if (rc == AHEAD_OK && o.count) {
        // right side hashed: the reference decodes the left head before it
        // emits it (hashjoinAN.tcc:339,352)
        const bool decode = side == AHEAD_HASH_RIGHT && type_encoded(l->head.type);
        const uint64_t ainv = decode ? l->head.Ainv : 1;
        const int hw = type_width(o.head.type);
        const uint64_t n = o.count;
        const uint64_t want = (n + 255) / 256;
        const unsigned grid = (unsigned)(want < (uint64_t)ctx->num_sms * 8 ? want : (uint64_t)ctx->num_sms * 8);
        str_gather_kernel<<<grid, 256, 0, ctx->stream>>>(rows, n, r_strs, width, (char*)out->tail.data, decode,
                                                         ainv, out->head.data, hw);
        ctx->launches += 1;
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "hashjoinAN(str) gather");
    }
    if (rc == AHEAD_OK && side == AHEAD_HASH_LEFT && l->tail.type == AHEAD_RESTINY && errs && l->count && r->count) {
        // The string join's left build checks the restiny code without a cast
        // (hashjoinAN.tcc:290): the u16 product is promoted to int, not reduced
        // mod 2^16, and the compiled reference wraps it to 32 bits.
        rc = restiny_promoted_check(ctx, (const uint16_t*)l->tail.data, l->count,
                                    (uint32_t)(l->tail.Ainv & 0xFFFF), (uint32_t)(l->tail.unenc_max & 0xFFFF), aoid,
                                    &errs[1]);
    }
    if (rows) cudaFreeAsync(rows, ctx->stream);
    out->head = o.head;
    out->head.data = o.head.data;
    out->count = o.count;
    const void* tdata = out->tail.data;
    set_meta(&out->tail, AHEAD_STR, 0, 0, 0, 0);
    out->tail.data = const_cast<void*>(tdata);
    if (errs) {
        errs[3].present = 0;
        errs[3].count = 0;
    }
    return rc;
}

int ahead_gpu_hashjoin_an(ahead_ctx* ctx, const ahead_bat* l, const ahead_bat* r, int reenc_head, uint64_t ah1r,
                          uint64_t ah1invr, int reenc_tail, uint64_t at2r, uint64_t at2invr, int side, uint64_t aoid,
                          ahead_bat* out, uint64_t cap, ahead_errvec* errs) {
    if (!ctx || !l || !r || !out) return AHEAD_BAD_ARG;
    const int H1 = l->head.type, T1 = l->tail.type, H2 = r->head.type, T2 = r->tail.type;
    if (!(H1 == AHEAD_VOID || H1 == AHEAD_RESOID) || !(T2 == AHEAD_VOID || T2 == AHEAD_RESOID) || !small_res(T1) ||
        !small_res(H2))
        return fail(ctx, AHEAD_BAD_ARG, "hashjoinAN: (void|resoid, restiny|resshort|resint) x (res*, void|resoid)");
    if (reenc_tail && !reenc_head) return fail(ctx, AHEAD_BAD_ARG, "hashjoinAN: tail re-encoding needs head re-encoding");
    const int eH1 = type_encoded(H1), eT2 = type_encoded(T2);
    const int wh1e = type_width(type_encoded_of(H1)), wt2e = type_width(type_encoded_of(T2));
    const uint64_t AH1Inv = eH1 ? l->head.Ainv & wmask(wh1e) : 0, AT2Inv = eT2 ? r->tail.Ainv & wmask(wt2e) : 0;
    const uint64_t fH1 = eH1 ? mulw(ah1r, AH1Inv, type_width(H1)) : (ah1r & 0xffffffffull);
    const uint64_t fT2 = eT2 ? mulw(at2r, AT2Inv, type_width(T2)) : (at2r & 0xffffffffull);
    const int oH = reenc_head ? type_encoded_of(H1) : type_select_of(H1);
    const int oT = reenc_tail ? type_encoded_of(T2) : type_select_of(T2);
    if (reenc_head) {
        set_meta(&out->head, oH, ah1r, ah1invr, l->head.unenc_max, 0);
        if (reenc_tail) set_meta(&out->tail, oT, at2r, at2invr, r->tail.unenc_max, 0);
        else set_meta(&out->tail, oT, r->tail.A, r->tail.Ainv, r->tail.unenc_max, 0);
    } else {
        copy_meta(&out->head, oH, &l->head);
        copy_meta(&out->tail, oT, &r->tail);
    }
    set_errs_present(errs, eH1, 1, 1, eT2);
    out->count = 0;
    OpScope s(ctx);
    const uint64_t nl = l->count, nr = r->count;
    const bool both = nl > 0 && nr > 0;
    const uint64_t nb = side == AHEAD_HASH_LEFT ? nl : nr, np = side == AHEAD_HASH_LEFT ? nr : nl;
    int rc = s.reserve((both ? join_scratch(nb, np) : 0) +
                       (both ? colcheck_scratch(nl) * 2 + colcheck_scratch(nr) * 2 : 0));
    if (rc) return rc;
    if (both) {
        const int bt1 = type_base_width(T1), bh2 = type_base_width(H2);
        const int larger = bt1 > bh2 ? bt1 : bh2;
        JoinOut o;
        o.fh = fH1;
        o.ft = fT2;
        o.cap = (out->head.data && out->tail.data) ? cap : 0;
        o.oh = out->head.data;
        o.ot = out->tail.data;
        o.rh = reenc_head;
        o.rt = reenc_tail;
        o.ohw = type_width(oH);
        o.otw = type_width(oT);
        if (side == AHEAD_HASH_LEFT) {
            KeyCfg bk = key_cfg(l->tail, 1, bt1, bt1, false);
            KeyCfg pk = key_cfg(r->head, 1, bt1, larger, true);
            o.probe_is_head = 0;
            o.pcol = dcol(r->tail);
            o.bcol = dcol(l->head);
            run_hash_join(s, bk, nl, pk, nr, o, 0);
        } else {
            KeyCfg bk = key_cfg(r->head, 1, bh2, bh2, false);
            KeyCfg pk = key_cfg(l->tail, 1, bh2, larger, true);
            o.probe_is_head = 1;
            o.pcol = dcol(l->head);
            o.bcol = dcol(r->tail);
            run_hash_join(s, bk, nr, pk, nl, o, 0);
        }
        if (eH1) run_colcheck(s, l->head, nl, AH1Inv, l->head.unenc_max & wmask(wh1e), wh1e, aoid, ev(errs, 0), 1);
        run_colcheck(s, l->tail, nl, l->tail.Ainv & wmask(type_width(T1)), l->tail.unenc_max & wmask(type_width(T1)),
                     type_width(T1), aoid, ev(errs, 1), 2);
        run_colcheck(s, r->head, nr, r->head.Ainv & wmask(type_width(H2)), r->head.unenc_max & wmask(type_width(H2)),
                     type_width(H2), aoid, ev(errs, 2), 3);
        if (eT2) run_colcheck(s, r->tail, nr, AT2Inv, r->tail.unenc_max & wmask(wt2e), wt2e, aoid, ev(errs, 3), 4);
    }
    rc = s.finish(5);
    if (rc) return rc;
    out->count = both ? s.counter(0) : 0;
    if (both && errs)
        for (int k = 0; k < 4; ++k)
            if (errs[k].present) errs[k].count = s.counter(1 + k);
    return out->count > cap ? AHEAD_CAPACITY : AHEAD_OK;
}

int ahead_gpu_hashjoin(ahead_ctx* ctx, const ahead_bat* l, const ahead_bat* r, int side, ahead_bat* out,
                       uint64_t cap) {
    if (!ctx || !l || !r || !out) return AHEAD_BAD_ARG;
    const int H1 = l->head.type, T1 = l->tail.type, H2 = r->head.type, T2 = r->tail.type;
    if (!(H1 == AHEAD_VOID || H1 == AHEAD_OID) || !(T2 == AHEAD_VOID || T2 == AHEAD_OID) || T1 != H2 ||
        T1 == AHEAD_VOID || T1 == AHEAD_OID || T1 == AHEAD_BIGINT || T1 == AHEAD_RESBIGINT || T1 == AHEAD_RESOID)
        return fail(ctx, AHEAD_BAD_ARG, "hashjoin: (void|oid, K) x (K, void|oid) with a 1/2/4-byte or res key K");
    copy_meta(&out->head, type_select_of(H1), &l->head);
    copy_meta(&out->tail, type_select_of(T2), &r->tail);
    out->count = 0;
    OpScope s(ctx);
    const uint64_t nl = l->count, nr = r->count;
    const bool both = nl > 0 && nr > 0;
    const uint64_t nb = side == AHEAD_HASH_LEFT ? nl : nr, np = side == AHEAD_HASH_LEFT ? nr : nl;
    int rc = s.reserve(both ? join_scratch(nb, np) : 0);
    if (rc) return rc;
    if (both) {
        const int w = type_width(T1);
        JoinOut o;
        o.fh = o.ft = 1;
        o.cap = (out->head.data && out->tail.data) ? cap : 0;
        o.oh = out->head.data;
        o.ot = out->tail.data;
        o.rh = o.rt = 0;
        o.ohw = type_width(type_select_of(H1));
        o.otw = type_width(type_select_of(T2));
        KeyCfg bk = key_cfg(side == AHEAD_HASH_LEFT ? l->tail : r->head, 0, w, w, false);
        KeyCfg pk = key_cfg(side == AHEAD_HASH_LEFT ? r->head : l->tail, 0, w, w, false);
        o.probe_is_head = side != AHEAD_HASH_LEFT;
        o.pcol = dcol(side == AHEAD_HASH_LEFT ? r->tail : l->head);
        o.bcol = dcol(side == AHEAD_HASH_LEFT ? l->head : r->tail);
        run_hash_join(s, bk, nb, pk, np, o, 0);
    }
    rc = s.finish(1);
    if (rc) return rc;
    out->count = both ? s.counter(0) : 0;
    return out->count > cap ? AHEAD_CAPACITY : AHEAD_OK;
}

int ahead_gpu_matchjoin_an(ahead_ctx* ctx, const ahead_bat* a, const ahead_bat* b, int reenc, uint64_t ah1r,
                           uint64_t ah1invr, uint64_t at2r, uint64_t at2invr, uint64_t aoid, ahead_bat* out,
                           uint64_t cap, ahead_errvec* errs) {
    if (!ctx || !a || !b || !out) return AHEAD_BAD_ARG;
    const int H1 = a->head.type, T1 = a->tail.type, H2 = b->head.type, T2 = b->tail.type;
    const bool vv = T1 == AHEAD_VOID && H2 == AHEAD_VOID, rv = T1 == AHEAD_RESOID && H2 == AHEAD_VOID;
    const bool gm = T1 == AHEAD_RESOID && H2 == AHEAD_RESOID, mv = T1 == AHEAD_VOID && H2 == AHEAD_RESOID;
    if (!(H1 == AHEAD_VOID || H1 == AHEAD_RESOID || H1 == AHEAD_RESINT) || !(vv || rv || gm || mv) ||
        (H1 == AHEAD_VOID && T1 == AHEAD_VOID) || (T2 == AHEAD_VOID && !gm) ||
        !(T2 == AHEAD_VOID || type_encoded(T2)))
        return fail(ctx, AHEAD_BAD_ARG, "matchjoinAN: unsupported type combination");
    if (reenc && (H1 == AHEAD_VOID || T2 == AHEAD_VOID))
        return fail(ctx, AHEAD_UNSUPPORTED, "matchjoinAN: re-encoding with a void head or tail");
    DCol h1 = dcol(a->head), t1 = dcol(a->tail), h2 = dcol(b->head), t2 = dcol(b->tail);
    const uint64_t fH1 = dec_if_host(h1, ah1r), fT2 = dec_if_host(t2, at2r);
    const int oH = reenc ? type_encoded_of(H1) : type_select_of(H1);
    const int oT = reenc ? type_encoded_of(T2) : type_select_of(T2);
    if (reenc) {
        set_meta(&out->head, oH, ah1r, ah1invr, a->head.unenc_max, 0);
        set_meta(&out->tail, oT, at2r, at2invr, b->tail.unenc_max, 0);
    } else {
        copy_meta(&out->head, oH, &a->head);
        copy_meta(&out->tail, oT, &b->tail);
    }
    out->count = 0;
    const uint64_t n1 = a->count, n2 = b->count;
    const uint64_t ocap = (out->head.data && out->tail.data) ? cap : 0;
    OpScope s(ctx);
    if (rv) {
        set_errs_present(errs, type_encoded(H1), 1, 0, type_encoded(T2));
        int rc = s.reserve(compact_scratch<MjPosOp<true>>(n1));
        if (rc) return rc;
        MjPosOp<true> op;
        op.base = (const char*)a->tail.data;
        op.status = s.d_status;
        op.h1c = h1;
        op.t2c = t2;
        op.at1inv = a->tail.Ainv;
        op.ah1inv = type_encoded(H1) ? a->head.Ainv : 0;
        op.ah1max = a->head.unenc_max;
        op.sz = (uint32_t)b->count;  // BAT::size() is an oid_t
        op.fh = fH1;
        op.ft = fT2;
        op.cap = ocap;
        op.aoid = aoid;
        op.e1 = edata(ev(errs, 0));
        op.e2 = edata(ev(errs, 1));
        op.e4 = edata(ev(errs, 3));
        op.ec1 = ecap(ev(errs, 0));
        op.ec2 = ecap(ev(errs, 1));
        op.ec4 = ecap(ev(errs, 3));
        op.acc = nullptr;
        op.oh = out->head.data;
        op.ot = out->tail.data;
        op.ohw = type_width(oH);
        op.otw = type_width(oT);
        op.reenc = reenc;
        op.h1enc = type_encoded(H1);
        op.t2enc = type_encoded(T2);
        run_compact(s, op, n1, 0);
        rc = s.finish(4);
        if (rc) return rc;
        out->count = s.counter(0);
        if (errs) {
            if (errs[0].present) errs[0].count = s.counter(1);
            errs[1].count = s.counter(2);
            if (errs[3].present) errs[3].count = s.counter(3);
        }
        return out->count > cap ? AHEAD_CAPACITY : AHEAD_OK;
    }
    if (vv) {
        set_errs_present(errs, type_encoded(H1), 0, 0, type_encoded(T2));
        uint64_t p1 = 0, p2 = 0, m = 0;
        if (n1 && n2) {
            if (a->tail.seqbase < b->head.seqbase) p1 = vv_skip(a->tail.seqbase, b->head.seqbase, n1);
            else if (a->tail.seqbase > b->head.seqbase) p2 = vv_skip(b->head.seqbase, a->tail.seqbase, n2);
            m = (n1 - p1) < (n2 - p2) ? (n1 - p1) : (n2 - p2);
        }
        int rc = s.reserve(colcheck_scratch(p1 + m) + colcheck_scratch(p2 + m));
        if (rc) return rc;
        if (m && ocap)
            zip_kernel<<<grid_for(m, 256), 256, 0, ctx->stream>>>(h1, t2, p1, p2, m, reenc, fH1, fT2, out->head.data,
                                                                   type_width(oH), out->tail.data, type_width(oT),
                                                                   ocap);
        if (n1 && n2) {
            if (type_encoded(H1))
                run_colcheck(s, a->head, p1 + m, h1.ainv, h1.umax, type_width(H1), aoid, ev(errs, 0), 0);
            if (type_encoded(T2))
                run_colcheck(s, b->tail, p2 + m, t2.ainv, t2.umax, type_width(T2), aoid, ev(errs, 3), 1);
        }
        rc = s.finish(2);
        if (rc) return rc;
        out->count = m;
        if (errs) {
            if (errs[0].present) errs[0].count = (n1 && n2) ? s.counter(0) : 0;
            if (errs[3].present) errs[3].count = (n1 && n2) ? s.counter(1) : 0;
        }
        return m > cap ? AHEAD_CAPACITY : AHEAD_OK;
    }
    // general merge (gm) or (void tail, resoid head) merge (mv)
    set_errs_present(errs, type_encoded(H1), type_encoded(T1), type_encoded(H2), type_encoded(T2));
    int rc = s.reserve(compact_scratch<IsectOp>(n1) + 256);
    if (rc) return rc;
    uint32_t* flag = (uint32_t*)(s.d_counters + 50);
    if (n1 && n2) {
        MergeSide ma{t1, h1, type_encoded(T1), type_encoded(H1)};
        MergeSide mb{h2, t2, type_encoded(H2), type_encoded(T2)};
        merge_check_kernel<<<grid_for(n1, 256), 256, 0, ctx->stream>>>(ma, n1, flag);
        merge_check_kernel<<<grid_for(n2, 256), 256, 0, ctx->stream>>>(mb, n2, flag);
        s.launched(2);
    }
    uint64_t hb[3] = {0, 0, 0};  // flag word, first and last key of the second input
    if (n2) {
        isect_bounds_kernel<<<1, 1, 0, ctx->stream>>>(h2, n2, s.d_counters + 51);
        s.launched();
    }
    cudaMemcpyAsync(hb, s.d_counters + 50, 24, cudaMemcpyDeviceToHost, ctx->stream);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return fail(ctx, AHEAD_CUDA_ERROR, "merge check");
    const uint32_t hflag = (uint32_t)hb[0];
    if (!(hflag & 1u)) {
        if (n1 && n2) {
            // the rank structure when the key range is at most 64 words per key
            const uint64_t krange = hb[2] - hb[1] + 1;
            const uint64_t words = (krange + 63) / 64;
            const bool use_bits = n2 < (1ull << 32) && words <= 64 * n2 + 1024;
            const uint64_t nt1 = (n1 + kMeTile - 1) / kMeTile, nt2 = (n2 + kMeTile - 1) / kMeTile;
            const size_t err_scratch = (hflag & 2u) ? (nt1 + nt2) * 24 + 2048 : 0;
            rc = s.reserve(compact_scratch<IsectOp>(n1) + (use_bits ? words * 12 + 512 : 0) + err_scratch);
            if (rc) return rc;
            IsectOp op;
            op.bits = nullptr;
            op.first = nullptr;
            op.kmin = hb[1];
            op.krange = krange;
            if (use_bits) {
                auto* bits = (unsigned long long*)s.alloc(words * 8);
                auto* first = (uint32_t*)s.alloc(words * 4);
                cudaMemsetAsync(bits, 0, words * 8, ctx->stream);
                isect_mark_kernel<<<grid_for(n2, 256), 256, 0, ctx->stream>>>(h2, n2, hb[1], bits, first);
                s.launched();
                op.bits = bits;
                op.first = first;
            }
            // the driving column must hold data: the tail, or the head when the tail is void
            op.base = (const char*)(T1 == AHEAD_VOID ? a->head.data : a->tail.data);
            op.status = s.d_status;
            op.t1c = t1;
            op.h1c = h1;
            op.h2c = h2;
            op.t2c = t2;
            op.n2 = n2;
            op.fh = fH1;
            op.ft = fT2;
            op.cap = ocap;
            op.acc = nullptr;
            op.oh = out->head.data;
            op.ot = out->tail.data;
            op.ohw = type_width(oH);
            op.otw = type_width(oT);
            op.reenc = reenc;
            if (type_width(T1 == AHEAD_VOID ? H1 : T1) != 8) return fail(ctx, AHEAD_UNSUPPORTED, "merge driving width");
            run_compact(s, op, n1, 0);
            if (hflag & 2u) {
                // corrupt values in ordered inputs: the loop's error positions, per row
                MergeErrs me;
                me.h1 = h1;
                me.t1 = t1;
                me.h2 = h2;
                me.t2 = t2;
                me.n1 = n1;
                me.n2 = n2;
                me.aoid = aoid;
                me.eh1 = type_encoded(H1);
                me.et1 = type_encoded(T1);
                me.eh2 = type_encoded(H2);
                me.et2 = type_encoded(T2);
                me.last2 = hb[2];
                uint64_t* l1m = (uint64_t*)s.alloc(8);
                me.l1m = l1m;
                merge_last_kernel<<<1, 1, 0, ctx->stream>>>(me, l1m);
                s.launched();
                for (int side = 0; side < 2; ++side) {
                    const uint64_t n = side ? n2 : n1;
                    const uint64_t nt = side ? nt2 : nt1;
                    auto* tcount = (uint32_t*)s.alloc(nt * 8);
                    auto* toff = (uint64_t*)s.alloc(nt * 16);
                    merge_err_count_kernel<<<(uint32_t)nt, kMeThreads, 0, ctx->stream>>>(me, side, n, tcount);
                    merge_err_scan_kernel<<<1, kMeThreads, 0, ctx->stream>>>(tcount, toff, (uint32_t)nt,
                                                                             s.d_counters + 1 + 2 * side);
                    const ahead_errvec* va = ev(errs, 2 * side);
                    const ahead_errvec* vb = ev(errs, 2 * side + 1);
                    merge_err_write_kernel<<<(uint32_t)nt, kMeThreads, 0, ctx->stream>>>(
                        me, side, n, toff, edata(va), ecap(va), edata(vb), ecap(vb));
                    s.launched(3);
                }
            }
        }
        rc = s.finish(5);
        if (rc) return rc;
        out->count = (n1 && n2) ? s.counter(0) : 0;
        if (errs && (hflag & 2u) && n1 && n2)
            for (int k = 0; k < 4; ++k)
                if (errs[k].present) errs[k].count = s.counter(1 + k);
        return out->count > cap ? AHEAD_CAPACITY : AHEAD_OK;
    }
    MergeSeq m;
    m.h1 = h1;
    m.t1 = t1;
    m.h2 = h2;
    m.t2 = t2;
    m.n1 = n1;
    m.n2 = n2;
    m.fh = fH1;
    m.ft = fT2;
    m.aoid = aoid;
    m.cap = ocap;
    for (int k = 0; k < 4; ++k) {
        m.e[k] = edata(ev(errs, k));
        m.ecap[k] = ecap(ev(errs, k));
    }
    m.oh = out->head.data;
    m.ot = out->tail.data;
    m.ohw = type_width(oH);
    m.otw = type_width(oT);
    m.reenc = reenc;
    m.checked = 1;
    merge_seq_kernel<<<1, 32, 0, ctx->stream>>>(m, s.d_counters);
    s.launched();
    rc = s.finish(5);
    if (rc) return rc;
    out->count = s.counter(0);
    if (errs)
        for (int k = 0; k < 4; ++k)
            if (errs[k].present) errs[k].count = s.counter(1 + k);
    return out->count > cap ? AHEAD_CAPACITY : AHEAD_OK;
}

int ahead_gpu_matchjoin(ahead_ctx* ctx, const ahead_bat* a, const ahead_bat* b, ahead_bat* out, uint64_t cap) {
    if (!ctx || !a || !b || !out) return AHEAD_BAD_ARG;
    const int H1 = a->head.type, T1 = a->tail.type, H2 = b->head.type, T2 = b->tail.type;
    auto oidish = [](int t) { return t == AHEAD_VOID || t == AHEAD_OID; };
    // heads instantiated in Normal/matchjoin.hpp:36-50 (strings aside)
    if (H1 == AHEAD_RESOID || !oidish(T1) || !oidish(H2) || T2 == AHEAD_VOID || T2 == AHEAD_RESOID ||
        (H1 == AHEAD_VOID && T1 == AHEAD_VOID))
        return fail(ctx, AHEAD_BAD_ARG, "matchjoin: unsupported type combination");
    copy_meta(&out->head, type_select_of(H1), &a->head);
    copy_meta(&out->tail, type_select_of(T2), &b->tail);
    out->count = 0;
    const uint64_t n1 = a->count, n2 = b->count;
    const uint64_t ocap = (out->head.data && out->tail.data) ? cap : 0;
    DCol h1 = dcol(a->head), t1 = dcol(a->tail), h2 = dcol(b->head), t2 = dcol(b->tail);
    OpScope s(ctx);
    if (T1 == AHEAD_VOID && H2 == AHEAD_VOID) {
        uint64_t p1 = 0, p2 = 0, m = 0;
        if (n1 && n2) {
            if (a->tail.seqbase < b->head.seqbase) p1 = vv_skip(a->tail.seqbase, b->head.seqbase, n1);
            else if (a->tail.seqbase > b->head.seqbase) p2 = vv_skip(b->head.seqbase, a->tail.seqbase, n2);
            m = (n1 - p1) < (n2 - p2) ? (n1 - p1) : (n2 - p2);
        }
        int rc = s.reserve(0);
        if (rc) return rc;
        if (m && ocap) {
            zip_kernel<<<grid_for(m, 256), 256, 0, ctx->stream>>>(h1, t2, p1, p2, m, 0, 1, 1, out->head.data,
                                                                   type_width(type_select_of(H1)), out->tail.data,
                                                                   type_width(type_select_of(T2)), ocap);
            s.launched();
        }
        rc = s.finish(0);
        if (rc) return rc;
        out->count = m;
        return m > cap ? AHEAD_CAPACITY : AHEAD_OK;
    }
    if (T1 == AHEAD_OID && H2 == AHEAD_VOID) {
        int rc = s.reserve(compact_scratch<MjPosOp<false>>(n1));
        if (rc) return rc;
        MjPosOp<false> op{};
        op.base = (const char*)a->tail.data;
        op.status = s.d_status;
        op.h1c = h1;
        op.t2c = t2;
        op.sz = n2;
        op.cap = ocap;
        op.acc = nullptr;
        op.oh = out->head.data;
        op.ot = out->tail.data;
        op.ohw = type_width(type_select_of(H1));
        op.otw = type_width(type_select_of(T2));
        run_compact(s, op, n1, 0);
        rc = s.finish(1);
        if (rc) return rc;
        out->count = n1 ? s.counter(0) : 0;
        return out->count > cap ? AHEAD_CAPACITY : AHEAD_OK;
    }
    // merge on plain oid values: strictly increasing keys intersect in parallel
    // (driving column of 2, 4 or 8 bytes); anything else replays the loop
    const int dw = type_width(T1 == AHEAD_VOID ? H1 : T1);
    if (n1 && n2 && dw >= 2) {
        int rc = s.reserve(compact_scratch<IsectPlainOp<8>>(n1) + 256);
        if (rc) return rc;
        uint32_t* flag = (uint32_t*)(s.d_counters + 50);
        MergeSide ma{t1, h1, 0, 0};
        MergeSide mb{h2, t2, 0, 0};
        merge_check_kernel<<<grid_for(n1, 256), 256, 0, ctx->stream>>>(ma, n1, flag);
        merge_check_kernel<<<grid_for(n2, 256), 256, 0, ctx->stream>>>(mb, n2, flag);
        s.launched(2);
        uint32_t hflag = 0;
        cudaMemcpyAsync(&hflag, flag, 4, cudaMemcpyDeviceToHost, ctx->stream);
        if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return fail(ctx, AHEAD_CUDA_ERROR, "merge check");
        if (!(hflag & 1u)) {
            rc = s.reserve(compact_scratch<IsectPlainOp<8>>(n1) + 256);
            if (rc) return rc;
            rc = by_width_enc(dw, [&](auto tag) -> int {
                constexpr int W = decltype(tag)::value;
                IsectPlainOp<W> op{};
                op.base = (const char*)(T1 == AHEAD_VOID ? a->head.data : a->tail.data);
                op.status = s.d_status;
                op.t1c = t1;
                op.h1c = h1;
                op.h2c = h2;
                op.t2c = t2;
                op.n2 = n2;
                op.cap = ocap;
                op.acc = nullptr;
                op.oh = out->head.data;
                op.ot = out->tail.data;
                op.ohw = type_width(type_select_of(H1));
                op.otw = type_width(type_select_of(T2));
                run_compact(s, op, n1, 0);
                return 0;
            });
            rc = s.finish(1);
            if (rc) return rc;
            out->count = s.counter(0);
            return out->count > cap ? AHEAD_CAPACITY : AHEAD_OK;
        }
    }
    int rc = s.reserve(0);
    if (rc) return rc;
    MergeSeq m{};
    m.h1 = h1;
    m.t1 = t1;
    m.h2 = h2;
    m.t2 = t2;
    m.n1 = n1;
    m.n2 = n2;
    m.cap = ocap;
    m.oh = out->head.data;
    m.ot = out->tail.data;
    m.ohw = type_width(type_select_of(H1));
    m.otw = type_width(type_select_of(T2));
    m.checked = 0;
    merge_seq_kernel<<<1, 32, 0, ctx->stream>>>(m, s.d_counters);
    s.launched();
    rc = s.finish(1);
    if (rc) return rc;
    out->count = s.counter(0);
    return out->count > cap ? AHEAD_CAPACITY : AHEAD_OK;
}

int ahead_gpu_fetchjoin_an(ahead_ctx* ctx, const ahead_bat* a, const ahead_bat* b, int reenc, uint64_t atr,
                           uint64_t atrinv, uint64_t aoid, ahead_bat* out, uint64_t cap, ahead_errvec* errs) {
    if (!ctx || !a || !b || !out) return AHEAD_BAD_ARG;
    const int T2 = b->tail.type;
    if (a->head.type != AHEAD_VOID || a->tail.type != AHEAD_RESOID || b->head.type != AHEAD_VOID || !type_encoded(T2))
        return fail(ctx, AHEAD_BAD_ARG, "fetchjoinAN: (void, resoid) x (void, AN tail) required");
    const int w = type_width(T2);
    copy_meta(&out->head, AHEAD_VOID, &a->head);
    copy_meta(&out->tail, T2, &b->tail);
    uint64_t fac = 1;
    if (reenc) {
        out->tail.A = (uint16_t)atr;
        out->tail.Ainv = atrinv;
        fac = mulw(atr, inv_pow2(b->tail.A, 8 * w), w);
    }
    if (errs) {
        ev_begin(&errs[0], 1);
        ev_begin(&errs[1], 1);
    }
    out->count = 0;
    OpScope s(ctx);
    int rc = s.reserve(compact_scratch<FetchOp<true>>(a->count));
    if (rc) return rc;
    FetchOp<true> op;
    op.base = (const char*)a->tail.data;
    op.status = s.d_status;
    op.t2c = dcol(b->tail);
    op.at1inv = a->tail.Ainv;
    op.at2inv = b->tail.Ainv & wmask(w);
    op.at2max = b->tail.unenc_max & wmask(w);
    op.vsz = b->count;
    op.fac = fac;
    op.cap = out->tail.data ? cap : 0;
    op.aoid = aoid;
    op.e1 = edata(ev(errs, 0));
    op.e2 = edata(ev(errs, 1));
    op.ec1 = ecap(ev(errs, 0));
    op.ec2 = ecap(ev(errs, 1));
    op.acc = nullptr;
    op.ot = out->tail.data;
    op.otw = w;
    op.reenc = reenc;
    op.w2 = w;
    run_compact(s, op, a->count, 0);
    rc = s.finish(3);
    if (rc) return rc;
    out->count = a->count ? s.counter(0) : 0;
    if (errs) {
        errs[0].count = a->count ? s.counter(1) : 0;
        errs[1].count = a->count ? s.counter(2) : 0;
    }
    return out->count > cap ? AHEAD_CAPACITY : AHEAD_OK;
}

int ahead_gpu_fetchjoin(ahead_ctx* ctx, const ahead_bat* a, const ahead_bat* b, ahead_bat* out, uint64_t cap) {
    if (!ctx || !a || !b || !out) return AHEAD_BAD_ARG;
    const int T2 = b->tail.type;
    if (a->head.type != AHEAD_VOID || a->tail.type != AHEAD_OID || b->head.type != AHEAD_VOID || T2 == AHEAD_VOID ||
        T2 == AHEAD_RESOID)
        return fail(ctx, AHEAD_BAD_ARG, "fetchjoin: (void, oid) x (void, value) required");
    copy_meta(&out->head, AHEAD_VOID, &a->head);
    copy_meta(&out->tail, T2, &b->tail);
    out->count = 0;
    OpScope s(ctx);
    int rc = s.reserve(compact_scratch<FetchOp<false>>(a->count));
    if (rc) return rc;
    FetchOp<false> op{};
    op.base = (const char*)a->tail.data;
    op.status = s.d_status;
    op.t2c = dcol(b->tail);
    op.vsz = b->count;
    op.fac = 1;
    op.cap = out->tail.data ? cap : 0;
    op.acc = nullptr;
    op.ot = out->tail.data;
    op.otw = type_width(T2);
    op.w2 = type_width(T2);
    run_compact(s, op, a->count, 0);
    rc = s.finish(1);
    if (rc) return rc;
    out->count = a->count ? s.counter(0) : 0;
    return out->count > cap ? AHEAD_CAPACITY : AHEAD_OK;
}

int ahead_gpu_fetchjoin_str_an(ahead_ctx* ctx, const ahead_bat* a, const char* strs, uint64_t width, uint64_t count,
                               uint64_t aoid, char* out, uint64_t cap, uint64_t* n_out, ahead_errvec* errs) {
    if (!ctx || !a || !n_out || !width) return AHEAD_BAD_ARG;
    if (a->head.type != AHEAD_VOID || a->tail.type != AHEAD_RESOID || (count && !strs) || count >= (1ull << 32))
        return fail(ctx, AHEAD_BAD_ARG, "fetchjoinAN(str): (void, resoid) OIDs and string slots required");
    if (errs) {
        ev_begin(&errs[0], 1);
        ev_begin(&errs[1], 0);
    }
    *n_out = 0;
    const uint64_t n = a->count;
    OpScope s(ctx);
    int rc = s.reserve(compact_scratch<FetchStrOp>(n) + n * 4 + 4096);
    if (rc) return rc;
    uint32_t* rows = (uint32_t*)s.alloc((n ? n : 1) * 4);
    FetchStrOp op;
    op.base = (const char*)a->tail.data;
    op.status = s.d_status;
    op.ainv = a->tail.Ainv;
    op.count = count;
    op.aoid = aoid;
    op.cap = n;
    op.rows = rows;
    op.err = edata(errs);
    op.errcap = ecap(errs);
    op.acc = nullptr;
    run_compact(s, op, n, 0);
    rc = s.finish(2);
    if (rc) return rc;
    const uint64_t kept = s.counter(0);
    *n_out = kept;
    if (errs) errs[0].count = s.counter(1);
    if (kept > cap) return AHEAD_CAPACITY;
    return gather_str_rows(ctx, rows, kept, strs, width, out);
}

int ahead_gpu_fetchjoin_str(ahead_ctx* ctx, const ahead_bat* a, const char* strs, uint64_t width, uint64_t count,
                            char* out, uint64_t cap, uint64_t* n_out) {
    if (!ctx || !a || !n_out || !width) return AHEAD_BAD_ARG;
    if (a->head.type != AHEAD_VOID || a->tail.type != AHEAD_OID || (count && !strs))
        return fail(ctx, AHEAD_BAD_ARG, "fetchjoin(str): (void, oid) OIDs and string slots required");
    *n_out = 0;
    const uint64_t n = a->count;
    OpScope s(ctx);
    int rc = s.reserve(compact_scratch<FetchStrPlainOp>(n) + n * 4 + 4096);
    if (rc) return rc;
    uint32_t* rows = (uint32_t*)s.alloc((n ? n : 1) * 4);
    FetchStrPlainOp op;
    op.base = (const char*)a->tail.data;
    op.status = s.d_status;
    op.count = count;
    op.cap = n;
    op.rows = rows;
    op.acc = nullptr;
    run_compact(s, op, n, 0);
    rc = s.finish(1);
    if (rc) return rc;
    const uint64_t kept = s.counter(0);
    *n_out = kept;
    if (kept > cap) return AHEAD_CAPACITY;
    return gather_str_rows(ctx, rows, kept, strs, width, out);
}

}  // extern "C"
