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
    // this CTA's rank in its cluster (0 without clusters)
    __device__ __forceinline__ int rank() const {
        if constexpr (G::C == 1) return 0;
        else {
            u32 v;
            asm("mov.u32 %0, %%cluster_ctarank;" : "=r"(v));
            return (int)v;
        }
    }
    // f(t) with t the thread's index in the cluster's T threads (its CTA's CT threads without clusters)
    template <class F>
    __device__ __forceinline__ void each(F&& f) {
        if constexpr (G::C == 1) f((int)threadIdx.x, r);
        else f(rank() * G::CT + (int)threadIdx.x, r);
    }
    template <class F>
    __device__ __forceinline__ void single(F&& f) {
        if (threadIdx.x == 0) f();
    }
    __device__ __forceinline__ void sync() { __syncthreads(); }
    // Barrier of all the cluster's threads; orders their shared (local and distributed) and global
    // memory accesses at cluster scope.
    __device__ __forceinline__ void cluster_sync() {
        asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
        asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
    }
    // Store into CTA `rk`'s shared memory at the offset `p` has in this CTA's (distributed shared memory).
    __device__ __forceinline__ void st_remote(u64* p, int rk, u64 v) const {
        u32 ra;
        asm("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(ra) : "r"((u32)__cvta_generic_to_shared(p)), "r"(rk));
        asm volatile("st.shared::cluster.u64 [%0], %1;" ::"r"(ra), "l"(v) : "memory");
    }
    __device__ __forceinline__ void set_error(int* err, int code) { atomicCAS(err, 0, code); }
    // Tensor memory: one warp allocates the CTA's columns (one CTA per SM uses it): all 512, or
    // for a cluster's CTA the 4 E CT / 128 its threads use (a power of two, at least 32);
    // thread t of warp w owns lane 32 (w % 4) + (t % 32), columns 4E (w / 4) + [0, 4E): E pairs.
    static constexpr u32 TM_COLS = G::C == 1 ? 512 : (4 * G::E * (G::CT / 128) < 32 ? 32 : 4 * G::E * (G::CT / 128));
    static_assert((TM_COLS & (TM_COLS - 1)) == 0 && TM_COLS <= 512, "tensor memory columns: a power of two up to 512");
    __device__ __forceinline__ void tmem_alloc(u32* slot) {
        if ((threadIdx.x >> 5) == 0) {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                             (u32)__cvta_generic_to_shared(slot)), "r"(TM_COLS));
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
        }
        tmem_sync();
    }
    __device__ __forceinline__ void tmem_free(u32 base) {
        tmem_sync();
        if ((threadIdx.x >> 5) == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(TM_COLS));
    }
    __device__ __forceinline__ void tmem_sync() {
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    }
    __device__ __forceinline__ static u32 tmem_addr(u32 base, int t) {
        const int w = t >> 5;
        return base + ((u32)(32 * (w & 3)) << 16) + (u32)(4 * G::E * (w >> 2));
    }
    __device__ __forceinline__ void tmem_st16(int, u32 ta, const u32 (&v)[16]) {
        asm volatile(
            "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(ta),
            "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]),
            "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15]));
    }
    __device__ __forceinline__ void tmem_ld16(int, u32 ta, u32 (&v)[16]) {
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
              "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(ta));
    }
    __device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
    __device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
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

// Resident CTAs per SM the kernel is compiled for (registers per thread <= 65536 / (T x this)).
// Measured on B200 (prime-residues/s, the same batch per SM, n = 2^LG):
//   L = 2^10 (32 threads): 1 -> 6.9k, 12 -> 7.3k, 16 (128 registers, ptxas -O1) -> 8.9k: 16;
//   L = 2^11 .. 2^13 (then with 32 entries per thread): capping registers lost 2 .. 20 %: 1 (no cap);
//   L = 2^14: one CTA per SM is forced by its shared memory and tensor memory anyway.
template <int LG>
struct MinBlocks {
    static constexpr int v = LG == 10 ? 16 : 1;
};
// MB: resident CTAs per SM the variant is compiled for (its register cap).
template <int LG, int R, bool W, int MB = MinBlocks<LG>::v>
__global__ void __launch_bounds__(Geo<LG, R>::T, MB) k_suffix(KParams kp) {
    typedef Geo<LG, R> G;
    extern __shared__ __align__(16) u64 smem[];
    DevExec<G> ex;
    PrimeRun<G, DevExec<G>, W> pr(ex, kp, (int)blockIdx.x, smem);
    pr.run();
}

// ------------------------------------------------------------------------------------------
// Work queue: one persistent launch over many (d, prime) tables of one transform length, each with
// its own n, F, d, model and query list.  A CTA takes the next item from a device counter with an
// atomic add (nothing waits on anything), runs it in its own workspace slot, and takes another
// until the list is exhausted; the host orders the list heaviest first.
// ------------------------------------------------------------------------------------------
struct QItem {
    u64 prime;
    int n, F, d, model, J, q0;  // table size, factorial range, degree, model, queries [q0, q0 + J)
};
struct QueueParams {
    const QItem* items;
    int count;
    int* next;                // next unclaimed item (zeroed before the launch)
    const int* qn;            // [sum J] query sizes, by item
    const int* qM;
    const long long* qout;    // [sum J] output index of each query
};
template <int LG, int R, bool W>
__global__ void __launch_bounds__(Geo<LG, R>::T, MinBlocks<LG>::v) k_suffix_queue(KParams kp, QueueParams qp) {
    typedef Geo<LG, R> G;
    typedef PrimeRun<G, DevExec<G>, W> PR;
    extern __shared__ __align__(16) u64 smem[];
    __shared__ __align__(16) unsigned char ikp_raw[sizeof(KParams)];  // the current item's parameters
    KParams& ikp = *reinterpret_cast<KParams*>(ikp_raw);
    __shared__ int item;
    DevExec<G> ex;
    u32* tm_slot = (u32*)(smem + Smem<G>::MISC + MI_TMEM);
    if constexpr (PR::TM) ex.tmem_alloc(tm_slot);  // once for all the CTA's items
    for (;;) {
        if (threadIdx.x == 0) {
            item = atomicAdd(qp.next, 1);
            if (item < qp.count) {
                const QItem& q = qp.items[item];
                ikp = kp;
                ikp.primes = &q.prime;
                ikp.B = 1;
                ikp.n = q.n, ikp.F = q.F, ikp.d = q.d, ikp.model = q.model, ikp.J = q.J;
                ikp.d0 = q.model == MODEL_SUBSET ? q.d : 1;
                ikp.qn = qp.qn + q.q0, ikp.qM = qp.qM + q.q0, ikp.qout = qp.qout + q.q0;
            }
        }
        __syncthreads();
        if (item >= qp.count) break;
        PR pr(ex, ikp, 0, smem, (int)blockIdx.x);
        pr.run_prime();
        __syncthreads();  // ikp and item are rewritten for the next item
    }
    if constexpr (PR::TM) ex.tmem_free(*tm_slot);
}
typedef void (*qfn_t)(KParams, QueueParams);

// Elements per thread (2^R): 32 at L = 2^10, 16 at L = 2^11 .. 2^14, fewer below so a CTA keeps at
// least a warp.  R = 4 was measured on B200 against R = 5 (twice the threads): n = 2048: 1826 ->
// 2244, n = 4096: 496 -> 540, n = 8192: 122 -> 170, n = 16384: 40.8 -> 48.5 prime-residues/s
// (1024 threads of 64 registers; 32 warps per SM hide the L2 latency of the per-step constants).
template <int LG>
struct RFor {
    static constexpr int R = (LG >= 11 && LG <= 14) ? 4 : (LG >= 10 ? 5 : (LG >= 6 ? LG - 5 : 1));
};

typedef void (*kfn_t)(KParams);
struct KInfo {
    kfn_t fn;
    int threads;  // per CTA
    size_t smem;  // fixed dynamic shared memory; a launch with J queries adds 8 J (threads / 32)
    int r;        // log2 of the entries per thread
    qfn_t qfn;    // the work-queue form (the default geometry only)
    int mb;       // resident CTAs per SM the kernel is compiled for
    int cluster = 1;  // CTAs per prime (a thread-block cluster when above 1)
    size_t smem_for(int J) const { return smem + (size_t)8 * J * (threads >= 32 ? threads / 32 : 1); }
};
// W selects the kernel for primes below 2^62 (otherwise below 2^50).
template <int LG, bool W = false>
inline KInfo kinfo() {
    typedef Geo<LG, RFor<LG>::R> G;
    return KInfo{&k_suffix<LG, RFor<LG>::R, W>, G::T, Smem<G>::BYTES, RFor<LG>::R, &k_suffix_queue<LG, RFor<LG>::R, W>,
                 MinBlocks<LG>::v};
}
// Transform lengths above 2^14 (tables above n = 16384, primes below 2^50): one prime per cluster of
// 2^LC CTAs, one CTA per SM, launched with that cluster size (CTA b 2^LC + c is CTA c of prime b).
template <int LG, int R, int LC, bool W>
__global__ void __launch_bounds__(Geo<LG, R, LC>::CT, 1) k_suffix_cl(KParams kp) {
    typedef Geo<LG, R, LC> G;
    extern __shared__ __align__(16) u64 smem[];
    DevExec<G> ex;
    PrimeRun<G, DevExec<G>, W> pr(ex, kp, (int)blockIdx.x >> LC, smem);
    pr.run();
}
// 2^R entries per thread (16, or 8 for twice the threads per CTA when E = 8 >= C); W: primes
// below 2^62 (otherwise below 2^50).
template <int LG, int LC, int R = 4, bool W = false>
inline KInfo kinfo_cluster() {
    typedef Geo<LG, R, LC> G;
    return KInfo{&k_suffix_cl<LG, R, LC, W>, G::CT, Smem<G>::BYTES, R, nullptr, 1, G::C};
}
// Another geometry of the 50-bit kernel (autotuning candidates): 2^R entries per thread, MB CTAs per SM.
template <int LG, int R, int MB>
inline KInfo kinfo_geo() {
    typedef Geo<LG, R> G;
    return KInfo{&k_suffix<LG, R, false, MB>, G::T, Smem<G>::BYTES, R, nullptr, MB};
}

}  // namespace cfb
