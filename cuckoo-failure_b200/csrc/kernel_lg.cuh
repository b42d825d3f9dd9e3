// The persistent per-prime kernel: one CTA owns one prime from setup to residues.  Each
// transform length is instantiated in its own translation unit (k_lgNN.cu) so they build in parallel.
#pragma once
#include <cuda_runtime.h>

#include "suffix_engine.cuh"

namespace cfb {

// ------------------------------------------------------------------------------------------
// Device execution policy: `each` runs on the calling thread, `sync` is a block barrier.
// ------------------------------------------------------------------------------------------
template <class G>
struct DevExec {
    Regs<G> r;
    template <class F>
    __device__ __forceinline__ void each(F&& f) {
        f((int)threadIdx.x, r);
    }
    template <class F>
    __device__ __forceinline__ void single(F&& f) {
        if (threadIdx.x == 0) f();
    }
    __device__ __forceinline__ void sync() { __syncthreads(); }
    __device__ __forceinline__ void set_error(int* err, int code) { atomicCAS(err, 0, code); }
    // Sum mod p of v over the calling thread's warp; lane 0 stores it at dst[warp * stride].
    __device__ __forceinline__ void warp_sum_store(int t, u64 v, u64 P, u64* dst, size_t stride) {
        const int T = (int)blockDim.x;
        const unsigned mask = T >= 32 ? 0xffffffffu : ((1u << T) - 1u);
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1)
            if (o < T) v = madd(v, __shfl_xor_sync(mask, v, o), P);
        if ((t & 31) == 0) dst[(size_t)(t >> 5) * stride] = v;
    }
    // red[0..T) holds values in [0, p); leaves their sum mod p in red[T].  Called by all threads.
    __device__ __forceinline__ void reduce_mod(u64* red, int T, u64 P) {
        const int t = threadIdx.x, lane = t & 31, w = t >> 5;
        const unsigned mask = T >= 32 ? 0xffffffffu : ((1u << T) - 1u);
        u64 v = red[t];
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1)
            if (o < T) v = madd(v, __shfl_xor_sync(mask, v, o), P);
        if (lane == 0) red[T + 1 + w] = v;
        __syncthreads();
        if (t == 0) {
            u64 s = 0;
            for (int k = 0; k < (T + 31) / 32; ++k) s = madd(s, red[T + 1 + k], P);
            red[T] = s;
        }
    }
};

template <int LG, int R>
__global__ void __launch_bounds__(Geo<LG, R>::T) k_suffix(KParams kp) {
    typedef Geo<LG, R> G;
    extern __shared__ __align__(16) u64 smem[];
    DevExec<G> ex;
    PrimeRun<G, DevExec<G>> pr(ex, kp, (int)blockIdx.x, smem);
    pr.run();
}

// Elements per thread: 32 for L >= 1024 (one register pass per 5 levels), fewer below so a CTA
// keeps at least a few warps' worth of threads.
template <int LG>
struct RFor {
    static constexpr int R = LG >= 10 ? 5 : (LG >= 6 ? LG - 5 : 1);
};

typedef void (*kfn_t)(KParams);
struct KInfo {
    kfn_t fn;
    int threads;
    size_t smem;
};
template <int LG>
inline KInfo kinfo() {
    typedef Geo<LG, RFor<LG>::R> G;
    return KInfo{&k_suffix<LG, RFor<LG>::R>, G::T, Smem<G>::BYTES};
}

}  // namespace cfb
