// Roofline denominator probe: the device's sustained 32-bit integer multiply-add (IMAD) rate,
// measured with independent mad.lo.u32 chains.  Separate library (libcuckoo_b200_probe.so) used
// only by bench.py; the engine never calls it.
#include <cuda_runtime.h>
#include <stdint.h>

static __global__ void k_imad(uint32_t* out, int iters, uint32_t m) {
    uint32_t x[8];
    for (int i = 0; i < 8; ++i) x[i] = threadIdx.x * 7 + i;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i) asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(x[i]) : "r"(m), "r"(it));
    }
    uint32_t s = 0;
    for (int i = 0; i < 8; ++i) s ^= x[i];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// Returns IMAD operations per second (0 on error), best of `reps` timed launches on `device`.
extern "C" double cfp_imad_ops_per_s(int device, int reps) {
    if (cudaSetDevice(device) != cudaSuccess) return 0;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int blocks = sms * 4, threads = 256, iters = 16384;
    uint32_t* d = nullptr;
    if (cudaMalloc(&d, sizeof(uint32_t) * blocks * threads) != cudaSuccess) return 0;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    k_imad<<<blocks, threads>>>(d, iters, 12345u);
    double best = 0;
    for (int r = 0; r < reps; ++r) {
        cudaEventRecord(a);
        k_imad<<<blocks, threads>>>(d, iters, 12345u);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        const double ops = (double)blocks * threads * 8.0 * iters;
        if (ms > 0 && ops / (ms * 1e-3) > best) best = ops / (ms * 1e-3);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(d);
    return cudaGetLastError() == cudaSuccess ? best : 0;
}
