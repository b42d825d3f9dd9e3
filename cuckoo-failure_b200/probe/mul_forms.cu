// Measurement probe (not part of the engine): issue rate of the 32-bit multiply forms and of the
// modular-product variants of csrc/modarith.cuh on the device, as independent chains over 4 CTAs
// of 256 threads per SM.  It is what showed that mul.hi.u32 issues at under half the rate of
// mul.wide.u32 on sm_100a, which is why the lazy Shoup product takes its quotient from wide
// products.
//   nvcc -gencode arch=compute_100a,code=sm_100a -O3 -Icuckoo-failure_b200/csrc \
//        cuckoo-failure_b200/probe/mul_forms.cu -o /tmp/mul_forms && /tmp/mul_forms
#include <cstdio>
#include <cstdint>
#include <cuda_runtime.h>
#include "modarith.cuh"
using namespace cfb;

template <int MODE>
__global__ void k_op(uint64_t* out, int iters, uint32_t m, uint64_t w, uint64_t wq, uint64_t p, uint32_t c) {
    uint32_t x[8];
    uint64_t y[8];
    for (int i = 0; i < 8; ++i) { x[i] = threadIdx.x * 7 + i; y[i] = (threadIdx.x * 131 + i) % p; }
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            if (MODE == 0) asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(x[i]) : "r"(m), "r"(it));
            if (MODE == 1) asm volatile("mad.hi.u32 %0, %0, %1, %2;" : "+r"(x[i]) : "r"(m), "r"(it));
            if (MODE == 2) asm volatile("mad.wide.u32 %0, %1, %2, %0;" : "+l"(y[i]) : "r"(x[i]), "r"(m));
            if (MODE == 3) asm volatile("mul.lo.u64 %0, %0, %1;" : "+l"(y[i]) : "l"(w));
            if (MODE == 4) asm volatile("add.u64 %0, %0, %1;" : "+l"(y[i]) : "l"(w));
            if (MODE == 5) { y[i] = shoup_mul_lazy(y[i], w, wq, p); asm volatile("" : "+l"(y[i])); }
            if (MODE == 6) { y[i] = shoup_mul_special(y[i], w, wq, Mod{p, 0, 0, 0}, c); asm volatile("" : "+l"(y[i])); }
            if (MODE == 7) {  // lazy Shoup, a*w via lo/hi 32-bit pieces, q*p special
                const uint64_t a = y[i];
                const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32), q0 = (uint32_t)wq, q1 = (uint32_t)(wq >> 32);
                const uint64_t q = (uint64_t)a1 * q1 + (uint64_t)__umulhi(a0, q1) + (uint64_t)__umulhi(a1, q0);
                const uint64_t qc = (uint64_t)(uint32_t)q * c + ((uint64_t)((uint32_t)(q >> 32) * c) << 32);
                y[i] = a * w - (q + (qc << 20));
                asm volatile("" : "+l"(y[i]));
            }
            if (MODE == 8) { y[i] = mont_mul(y[i], w, Mod{p, wq, 0, 0}); asm volatile("" : "+l"(y[i])); }
            if (MODE == 9) {  // fwd butterfly pair (a, c) -> lazy
                const uint64_t P4 = 4 * p;
                const uint64_t a = y[i], cc = y[(i + 1) & 7];
                const uint64_t s = a + cc;
                y[i] = s >= P4 ? s - P4 : s;
                y[(i + 1) & 7] = shoup_mul_lazy(a - cc + P4, w, wq, p);
                asm volatile("" : "+l"(y[i]), "+l"(y[(i + 1) & 7]));
            }

            if (MODE == 10) {  // lazy Shoup, quotient from wide products only (the engine's form)
                const uint64_t a = y[i];
                const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32), q0 = (uint32_t)wq, q1 = (uint32_t)(wq >> 32);
                uint64_t t1, t2, q;
                asm("mul.wide.u32 %0, %1, %2;" : "=l"(t1) : "r"(a0), "r"(q1));
                asm("mul.wide.u32 %0, %1, %2;" : "=l"(t2) : "r"(a1), "r"(q0));
                const uint64_t cc = (t1 >> 32) + (t2 >> 32);
                asm("mad.wide.u32 %0, %1, %2, %3;" : "=l"(q) : "r"(a1), "r"(q1), "l"(cc));
                y[i] = a * w - q * p;
                asm volatile("" : "+l"(y[i]));
            }
            if (MODE == 11) {  // MODE 10 with q p = q + (q c) 2^20
                const uint64_t a = y[i];
                const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32), q0 = (uint32_t)wq, q1 = (uint32_t)(wq >> 32);
                uint64_t t1, t2, q;
                asm("mul.wide.u32 %0, %1, %2;" : "=l"(t1) : "r"(a0), "r"(q1));
                asm("mul.wide.u32 %0, %1, %2;" : "=l"(t2) : "r"(a1), "r"(q0));
                const uint64_t cc = (t1 >> 32) + (t2 >> 32);
                asm("mad.wide.u32 %0, %1, %2, %3;" : "=l"(q) : "r"(a1), "r"(q1), "l"(cc));
                const uint64_t qc = (uint64_t)(uint32_t)q * c + ((uint64_t)((uint32_t)(q >> 32) * c) << 32);
                y[i] = a * w - (q + (qc << 20));
                asm volatile("" : "+l"(y[i]));
            }
            if (MODE == 12) {  // MODE 10, a w and q p low words from explicit wide + lo pieces
                const uint64_t a = y[i];
                const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32), q0 = (uint32_t)wq, q1 = (uint32_t)(wq >> 32);
                const uint32_t w0 = (uint32_t)w, w1 = (uint32_t)(w >> 32), p0 = (uint32_t)p, p1 = (uint32_t)(p >> 32);
                uint64_t t1, t2, q, aw, qp;
                asm("mul.wide.u32 %0, %1, %2;" : "=l"(t1) : "r"(a0), "r"(q1));
                asm("mul.wide.u32 %0, %1, %2;" : "=l"(t2) : "r"(a1), "r"(q0));
                const uint64_t cc = (t1 >> 32) + (t2 >> 32);
                asm("mad.wide.u32 %0, %1, %2, %3;" : "=l"(q) : "r"(a1), "r"(q1), "l"(cc));
                const uint32_t qa = (uint32_t)q, qb = (uint32_t)(q >> 32);
                asm("mul.wide.u32 %0, %1, %2;" : "=l"(aw) : "r"(a0), "r"(w0));
                asm("mul.wide.u32 %0, %1, %2;" : "=l"(qp) : "r"(qa), "r"(p0));
                const uint32_t awh = (uint32_t)(aw >> 32) + a0 * w1 + a1 * w0;
                const uint32_t qph = (uint32_t)(qp >> 32) + qa * p1 + qb * p0;
                y[i] = (((uint64_t)awh << 32) | (uint32_t)aw) - (((uint64_t)qph << 32) | (uint32_t)qp);
                asm volatile("" : "+l"(y[i]));
            }
            if (MODE == 13) { y[i] = mont_mul_special(y[i], w, Mod{p, wq, 0, 0}, c); asm volatile("" : "+l"(y[i])); }
            if (MODE == 14) {  // fwd butterfly with MODE 10 product
                const uint64_t P4 = 4 * p;
                const uint64_t a = y[i], cc0 = y[(i + 1) & 7];
                const uint64_t s = a + cc0;
                y[i] = s >= P4 ? s - P4 : s;
                const uint64_t dd = a - cc0 + P4;
                const uint32_t a0 = (uint32_t)dd, a1 = (uint32_t)(dd >> 32), q0 = (uint32_t)wq, q1 = (uint32_t)(wq >> 32);
                uint64_t t1, t2, q;
                asm("mul.wide.u32 %0, %1, %2;" : "=l"(t1) : "r"(a0), "r"(q1));
                asm("mul.wide.u32 %0, %1, %2;" : "=l"(t2) : "r"(a1), "r"(q0));
                const uint64_t cc = (t1 >> 32) + (t2 >> 32);
                asm("mad.wide.u32 %0, %1, %2, %3;" : "=l"(q) : "r"(a1), "r"(q1), "l"(cc));
                y[(i + 1) & 7] = dd * w - q * p;
                asm volatile("" : "+l"(y[i]), "+l"(y[(i + 1) & 7]));
            }
        }
    }
    uint64_t s = 0;
    for (int i = 0; i < 8; ++i) s ^= x[i] ^ y[i];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

template <int MODE>
double run(const char* name, int blocks, int threads, int iters, uint64_t* d, uint64_t p, uint32_t c) {
    const uint64_t w = 123456789012345ull % p;
    const uint64_t wq = (uint64_t)((((unsigned __int128)w) << 64) / p);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    k_op<MODE><<<blocks, threads>>>(d, iters, 12345u, w, wq, p, c);
    double best = 0;
    for (int r = 0; r < 3; ++r) {
        cudaEventRecord(a);
        k_op<MODE><<<blocks, threads>>>(d, iters, 12345u, w, wq, p, c);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        const double ops = (double)blocks * threads * 8.0 * iters;
        if (ms > 0 && ops / (ms * 1e-3) > best) best = ops / (ms * 1e-3);
    }
    cudaError_t e = cudaGetLastError();
    printf("%-28s %8.3f Gop/s  %6.2f per SM per clk(1965)%s\n", name, best / 1e9, best / 148 / 1965e6,
           e == cudaSuccess ? "" : cudaGetErrorString(e));
    return best;
}

int main() {
    const int blocks = 148 * 4, threads = 256, iters = 4096;
    uint64_t* d = nullptr;
    if (cudaMalloc(&d, sizeof(uint64_t) * blocks * threads) != cudaSuccess) return 1;
    const uint64_t p = (uint64_t)1073741823ull * (1ull << 20) + 1;  // not nec. prime; arithmetic only
    const uint32_t c = 1073741823u;
    run<0>("mad.lo.u32", blocks, threads, iters, d, p, c);
    run<1>("mad.hi.u32", blocks, threads, iters, d, p, c);
    run<2>("mad.wide.u32", blocks, threads, iters, d, p, c);
    run<3>("mul.lo.u64", blocks, threads, iters, d, p, c);
    run<4>("add.u64", blocks, threads, iters, d, p, c);
    run<5>("shoup_mul_lazy", blocks, threads, iters, d, p, c);
    run<6>("shoup_mul_special", blocks, threads, iters, d, p, c);
    run<7>("shoup_lazy_special", blocks, threads, iters, d, p, c);
    run<8>("mont_mul", blocks, threads, iters, d, p, c);
    run<9>("fwd butterfly", blocks, threads, iters, d, p, c);
    run<10>("shoup wide-q", blocks, threads, iters, d, p, c);
    run<11>("shoup wide-q special", blocks, threads, iters, d, p, c);
    run<12>("shoup all-explicit", blocks, threads, iters, d, p, c);
    run<13>("mont_mul_special", blocks, threads, iters, d, p, c);
    run<14>("fwd butterfly wide-q", blocks, threads, iters, d, p, c);
    cudaFree(d);
    return 0;
}
