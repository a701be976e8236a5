// hash.cuh -- open-addressing hash table with build-order duplicate chains.
//
// The reference keys its joins and group-bys with
// google::dense_hash_map<key, std::vector<payload>> (hashjoinAN.tcc:132-187,
// groupbyAN.tcc:62-91): every key keeps its payloads in build order and
// probes see them in that order.  On the GPU the table is built in four
// data-parallel steps:
//   1. insert: every build row claims (or finds) its key's slot with a CAS on
//      the 64-bit key array and counts itself in the slot;
//   2. the slot counts are scanned into segment starts;
//   3. fill: every build row drops its row index into its slot's segment;
//   4. order: segments with more than one row are sorted ascending, which
//      restores build order (duplicate keys are rare: primary keys, or a
//      bit flip that made two keys collide).
// The key value ~0 cannot live in the key array (it marks empty slots); it
// gets a dedicated extra slot at index `cap`.
#pragma once

#include "compact.cuh"

namespace ahead {

constexpr uint64_t kEmptyKey = ~0ull;
constexpr uint32_t kNoSlot = 0xffffffffu;

struct HashTab {
    uint64_t* keys;  // [cap + 1], kEmptyKey = free
    uint32_t* cnt;   // [cap + 1] rows per slot
    uint32_t* off;   // [cap + 1] segment start in `rows`
    uint32_t* cur;   // [cap + 1] fill cursor
    uint32_t* rows;  // [nbuild] build row indices grouped by slot
    uint32_t mask;   // cap - 1 (cap a power of two)
};

AHEAD_HD uint32_t ht_mix(uint64_t k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return (uint32_t)k;
}

AHEAD_DEV uint32_t ht_insert(const HashTab& h, uint64_t k) {
    if (k == kEmptyKey) return h.mask + 1;
    uint32_t s = ht_mix(k) & h.mask;
    for (uint32_t i = 0; i <= h.mask; ++i) {
        const uint64_t prev = atomicCAS((unsigned long long*)&h.keys[s], (unsigned long long)kEmptyKey,
                                        (unsigned long long)k);
        if (prev == kEmptyKey || prev == k) return s;
        s = (s + 1) & h.mask;
    }
    return kNoSlot;  // unreachable: the table is at most half full
}

AHEAD_DEV uint32_t ht_find(const HashTab& h, uint64_t k) {
    if (k == kEmptyKey) return h.cnt[h.mask + 1] ? h.mask + 1 : kNoSlot;
    uint32_t s = ht_mix(k) & h.mask;
    for (uint32_t i = 0; i <= h.mask; ++i) {
        const uint64_t kk = h.keys[s];
        if (kk == k) return s;
        if (kk == kEmptyKey) return kNoSlot;
        s = (s + 1) & h.mask;
    }
    return kNoSlot;
}

// The probe side's view of a built join table: key, row count and either the
// single build row (count 1, the primary-key case) or the segment start, in
// one 16-byte slot, so a probe reads one sector per step.
struct alignas(16) ProbeSlot {
    uint64_t key;
    uint32_t cnt;
    uint32_t first;  // cnt == 1: the build row; cnt > 1: the segment start in `rows`
};

AHEAD_DEV uint32_t ps_find(const ProbeSlot* t, uint32_t mask, uint64_t k, ProbeSlot& out) {
    if (k == kEmptyKey) {
        out = t[mask + 1];
        return out.cnt ? mask + 1 : kNoSlot;
    }
    uint32_t s = ht_mix(k) & mask;
    for (uint32_t i = 0; i <= mask; ++i) {
        const ProbeSlot e = t[s];
        if (e.key == k) {
            out = e;
            return s;
        }
        if (e.key == kEmptyKey) return kNoSlot;
        s = (s + 1) & mask;
    }
    return kNoSlot;
}

inline uint32_t ht_capacity(uint64_t n) {
    uint64_t c = 64;
    while (c < 2 * n) c <<= 1;
    return (uint32_t)c;
}

}  // namespace ahead
