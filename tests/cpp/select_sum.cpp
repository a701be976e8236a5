// select_sum.cpp -- a C++ host program over the C ABI (include/ahead_gpu.h),
// the way a reference program (tools/ssbm/ssbm-q11_continuous.cpp) would
// call the GPU operators: selectAN<ge, lt, and> of [lo, hi) on the codes of a
// (void, resshort) column, a positional matchjoinAN of the selection onto the
// column, checkAndDecodeAN, the unencoded sum and its AN code (A = 65117).
//
//   select_sum <codes.u32> <A> <lo> <hi>
//
// prints the result count, the AN-coded sum and every error vector, one per
// line, for tests/test_cpp_host.py to compare with the oracle.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "ahead_gpu.h"

static uint64_t inv_mod(uint64_t a, int bits) {  // Newton's iteration, then the width's mask
    uint64_t x = a;
    for (int i = 0; i < 5; ++i) x *= 2 - a * x;
    return bits >= 64 ? x : (x & ((1ull << bits) - 1));
}

static void check(int rc, ahead_ctx* ctx, const char* what) {
    if (rc != AHEAD_OK) {
        std::fprintf(stderr, "%s: %s (%s)\n", what, ahead_status_string(rc), ahead_ctx_last_error(ctx));
        std::exit(2);
    }
}

struct DevErr {
    ahead_errvec v{};
    explicit DevErr(uint64_t cap) {
        cudaMalloc(&v.data, cap * 8);
        v.capacity = cap;
    }
    ~DevErr() { cudaFree(v.data); }
    void print(const char* name) const {
        std::vector<uint64_t> h(v.count < v.capacity ? v.count : v.capacity);
        if (!h.empty()) cudaMemcpy(h.data(), v.data, h.size() * 8, cudaMemcpyDeviceToHost);
        std::printf("%s %d", name, v.present);
        for (uint64_t x : h) std::printf(" %llu", (unsigned long long)x);
        std::printf("\n");
    }
};

int main(int argc, char** argv) {
    if (argc != 5) {
        std::fprintf(stderr, "usage: select_sum <codes.u32> <A> <lo> <hi>\n");
        return 1;
    }
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 1;
    std::fseek(f, 0, SEEK_END);
    const uint64_t n = (uint64_t)std::ftell(f) / 4;
    std::fseek(f, 0, SEEK_SET);
    std::vector<uint32_t> codes(n);
    if (std::fread(codes.data(), 4, n, f) != n) return 1;
    std::fclose(f);
    const uint64_t A = std::strtoull(argv[2], nullptr, 10), lo = std::strtoull(argv[3], nullptr, 10),
                   hi = std::strtoull(argv[4], nullptr, 10), aoid = 16089;

    ahead_ctx* ctx = nullptr;
    check(ahead_ctx_create(0, nullptr, &ctx), ctx, "ahead_ctx_create");
    void *d_codes, *sel_h, *f_h, *f_t, *d_h, *d_t;
    cudaMalloc(&d_codes, n * 4);
    cudaMemcpy(d_codes, codes.data(), n * 4, cudaMemcpyHostToDevice);
    for (void** p : {&sel_h, &f_h, &f_t, &d_h, &d_t}) cudaMalloc(p, (n + 1) * 8);

    ahead_bat col{};
    col.head.type = AHEAD_VOID;
    col.tail.data = d_codes;
    col.tail.type = AHEAD_RESSHORT;
    col.tail.A = (uint32_t)A;
    col.tail.Ainv = inv_mod(A, 32);
    col.tail.unenc_max = 0xFFFF;
    col.count = n;

    // selectAN<ge, lt, and>(col, lo * A, hi * A)   (thresholds on codes, ssbm-q11_continuous.cpp:71-73)
    ahead_bat sel{};
    sel.head.data = sel_h;
    DevErr e_sel(1 << 16);
    check(ahead_gpu_select_an(ctx, &col, AHEAD_CMP_GE, lo * A, AHEAD_CMP_LT, hi * A, AHEAD_AND, aoid, &sel, n,
                              &e_sel.v),
          ctx, "selectAN");
    // matchjoinAN(sel->mirror_head(), col): the selected rows' values
    ahead_bat mirror{};
    mirror.head = sel.head;
    mirror.tail = sel.head;
    mirror.count = sel.count;
    ahead_bat fetched{};
    fetched.head.data = f_h;
    fetched.tail.data = f_t;
    DevErr ef0(1 << 16), ef1(1 << 16), ef2(1 << 16), ef3(1 << 16);
    ahead_errvec ef[4] = {ef0.v, ef1.v, ef2.v, ef3.v};
    check(ahead_gpu_matchjoin_an(ctx, &mirror, &col, 0, 0, 0, 0, 0, aoid, &fetched, n, ef), ctx, "matchjoinAN");
    ef0.v = ef[0];
    ef1.v = ef[1];
    ef2.v = ef[2];
    ef3.v = ef[3];
    // checkAndDecodeAN(fetched)
    ahead_bat dec{};
    dec.head.data = d_h;
    dec.tail.data = d_t;
    DevErr eh(1 << 16), et(1 << 16);
    check(ahead_gpu_check_and_decode_an(ctx, &fetched, aoid, &dec, n, &eh.v, &et.v), ctx, "checkAndDecodeAN");
    // the unencoded sum, AN-coded with the largest resint A
    uint64_t total = 0;
    check(ahead_gpu_aggregate_sum(ctx, &dec, AHEAD_BIGINT, &total), ctx, "aggregate_sum");
    std::printf("selected %llu\n", (unsigned long long)sel.count);
    std::printf("decoded %llu\n", (unsigned long long)dec.count);
    std::printf("total %llu\n", (unsigned long long)(total * 65117ull));
    e_sel.print("select_errors");
    ef0.print("fetch_errors0");
    ef1.print("fetch_errors1");
    ef2.print("fetch_errors2");
    ef3.print("fetch_errors3");
    eh.print("decode_errors0");
    et.print("decode_errors1");
    std::printf("launches %llu\n", (unsigned long long)ahead_ctx_launches(ctx));
    ahead_ctx_destroy(ctx);
    for (void* p : {d_codes, sel_h, f_h, f_t, d_h, d_t}) cudaFree(p);
    return 0;
}
