// Queries served from resident tables (cf_tables_query): N_bad(n, M) mod p for primes whose whole
// V (packed triangle) and pair tables fact, ifact, inv were kept by a serving build
// (KParams::keep).  The arithmetic is that of the build's own query and finish phases
// (PrimeRun::query_row and PrimeRun::finish): the per-row sums of fast/cuckoo_fast.cu:306-323,
// 595-622 and the Horner finish of :877-890, read from the resident triangle instead of from the
// row the build is about to consume.
#pragma once
#include <cuda_runtime.h>

#include "suffix_engine.cuh"

namespace cfb {

// Queries per launch: their sizes travel in the kernel parameters (no staging buffer, so launches
// on several streams never share one).
constexpr int TQ_MAXJ = 256;
struct TQParams {
    const u64* primes;  // [B]
    int B, n, F, d, d0, model, J;
    const u64* keep;    // [B][keep_words]
    size_t keep_words;
    u64* out;           // residue of prime b, query jq at out[b * out_stride + jq]
    size_t out_stride;
    int qn[TQ_MAXJ];    // each <= n
    int qM[TQ_MAXJ];    // each <= F
};

// One CTA per (prime, query).  Dynamic shared memory: the row sums ps[0..n] and a reduction area.
template <int T>
__global__ void __launch_bounds__(T) k_table_query(TQParams tp) {
    constexpr int NW = T / 32;
    extern __shared__ __align__(16) u64 sq[];
    const int b = blockIdx.x / tp.J, jq = blockIdx.x % tp.J;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int nj = tp.qn[jq], Mj = tp.qM[jq], d0 = tp.d0;
    u64* ps = sq;             // [n + 1] row sums
    u64* red = sq + tp.n + 1;  // [NW + 1]
    __shared__ Mod smod;
    __shared__ u64 soneq;
    const u64 P = tp.primes[b];
    if (t == 0) {
        smod = make_mod(P);
        soneq = shoup_companion(1, P);
    }
    const KeepLayout kl = make_keep_layout(tp.n, tp.F);
    const u64* base = tp.keep + (size_t)b * tp.keep_words;
    const u64* tri = base + kl.tri;
    const u64* fact = base + kl.fact;
    const u64* ifact = base + kl.ifact;
    const u64* inv = base + kl.inv;
    auto sh = [&](u64 a, const u64* pairs, int k) { return shoup_mul_lazy(a, pairs[2 * k], pairs[2 * k + 1], P); };
    for (int q = t; q <= nj; q += T) ps[q] = 0;
    __syncthreads();
    const u64 oneq = soneq;
    // ps[q] = sum_{d0 <= w < q} Vs[q][w] / (M - w): one warp per row, lanes along the row
    for (int q = d0 + 1 + warp; q <= nj; q += NW) {
        const u64* row = tri + tri_off(q);
        u64 acc = 0;  // each term < 4p < 2^52, at most 512 terms per lane
        for (int w = d0 + lane; w < q; w += 32) acc += sh(row[w], inv, Mj - w);
        u64 v = shoup_mul_lazy(acc, 1, oneq, P);
        v = v >= 2 * P ? v - 2 * P : v;
        v = v >= P ? v - P : v;
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) v = madd(v, __shfl_xor_sync(0xffffffffu, v, o), P);
        if (lane == 0) ps[q] = v;
    }
    __syncthreads();
    // N_bad = M! n! sum_k inv[k] ifact[n-k] ifact[M-k] Q^(n-k) ps[k]
    const Mod m = smod;
    u64 Qm;
    if (tp.model == MODEL_REPLACEMENT) Qm = mont_pow(to_mont((u64)Mj, m), (u64)tp.d, m);
    else {
        const u64 c = sh(sh(fact[2 * Mj], ifact, tp.d), ifact, Mj - tp.d);
        Qm = to_mont(red2(red2(c, 2 * P), P), m);
    }
    u64 acc = 0;
    for (int k = t + 1; k <= nj; k += T) {
        u64 y = sh(ps[k], inv, k);
        y = sh(y, ifact, nj - k);
        y = sh(y, ifact, Mj - k);
        y = mont_mul(y, mont_pow(Qm, (u64)(nj - k), m), m);
        acc = madd(acc, y, P);
    }
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) acc = madd(acc, __shfl_xor_sync(0xffffffffu, acc, o), P);
    if (lane == 0) red[warp] = acc;
    __syncthreads();
    if (t == 0) {
        u64 s = 0;
        for (int w = 0; w < NW; ++w) s = madd(s, red[w], P);
        u64 r = sh(s, fact, nj);
        r = red2(red2(r, 2 * P), P);
        r = sh(r, fact, Mj);
        tp.out[(size_t)b * tp.out_stride + jq] = red2(red2(r, 2 * P), P);
    }
}

constexpr int TQ_THREADS = 256;
inline size_t tq_smem_bytes(int n) { return 8 * ((size_t)n + 1 + TQ_THREADS / 32 + 1); }

}  // namespace cfb
