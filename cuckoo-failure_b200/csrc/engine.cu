// CUDA implementation of the C ABI in include/cuckoo_b200.h: the persistent per-prime kernel
// (one CTA per prime, all steps in one launch) and the host-side batching around it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/cuckoo_b200.h"
#include "engine_internal.hpp"
#include "host_common.hpp"
#include "kernel_lg.cuh"
#include "table_query.cuh"

using namespace cfb;

// The kernel for transform length 2^lg: primes below 2^50, or (wide) below 2^62.
KInfo kernel_for(int lg, bool wide) {
    if (wide) switch (lg) {
            case 4: return cf_kinfo_lg4_w();
            case 5: return cf_kinfo_lg5_w();
            case 6: return cf_kinfo_lg6_w();
            case 7: return cf_kinfo_lg7_w();
            case 8: return cf_kinfo_lg8_w();
            case 9: return cf_kinfo_lg9_w();
            case 10: return cf_kinfo_lg10_w();
            case 11: return cf_kinfo_lg11_w();
            case 12: return cf_kinfo_lg12_w();
            case 13: return cf_kinfo_lg13_w();
            case 14: return cf_kinfo_lg14_w();
            case 15: return cf_kinfo_lg15_c4_w();
            case 16: return cf_kinfo_lg16_c8_w();
            default: return KInfo{nullptr, 0, 0, 0};
        }
    switch (lg) {
        case 4: return cf_kinfo_lg4();
        case 5: return cf_kinfo_lg5();
        case 6: return cf_kinfo_lg6();
        case 7: return cf_kinfo_lg7();
        case 8: return cf_kinfo_lg8();
        case 9: return cf_kinfo_lg9();
        case 10: return cf_kinfo_lg10();
        case 11: return cf_kinfo_lg11();
        case 12: return cf_kinfo_lg12();
        case 13: return cf_kinfo_lg13();
        case 14: return cf_kinfo_lg14();
        case 15: return cf_kinfo_lg15_c4();
        case 16: return cf_kinfo_lg16_c16();
        default: return KInfo{nullptr, 0, 0, 0};
    }
}
// The cluster geometries compiled for transform length 2^lg (15, 16): cluster size, and 16 or 8
// entries per thread (8: twice the threads per CTA); smaller clusters first.
static int cluster_variants(int lg, KInfo* v, bool wide = false) {
    if (wide) {  // primes below 2^62: the default geometry only
        if (lg != 15 && lg != 16) return 0;
        v[0] = kernel_for(lg, true);
        return 1;
    }
    if (lg == 15)
        return v[0] = cf_kinfo_lg15_c4(), v[1] = cf_kinfo_lg15_c8(), v[2] = cf_kinfo_lg15_c4_e8(), v[3] = cf_kinfo_lg15_c8_e8(), 4;
    if (lg == 16) return v[0] = cf_kinfo_lg16_c8(), v[1] = cf_kinfo_lg16_c16(), 2;
    return 0;
}
// Clusters of the kernel ki (at smem bytes of dynamic shared memory) the device runs at once.
static int resident_clusters(const KInfo& ki, size_t smem, cudaStream_t s) {
    if (cudaFuncSetAttribute((const void*)ki.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return 0;
    if (ki.cluster > 8 && cudaFuncSetAttribute((const void*)ki.fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
        return 0;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)ki.cluster, at[0].val.clusterDim.y = 1, at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3((unsigned)ki.cluster), cfg.blockDim = dim3((unsigned)ki.threads), cfg.dynamicSmemBytes = smem;
    cfg.stream = s, cfg.attrs = at, cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, (const void*)ki.fn, &cfg) != cudaSuccess) return 0;
    return n;
}
// The cluster geometry a launch at transform length 2^lg runs: the one pinned on the engine
// (cf_tune_set, or cf_autotune's choice), else the default, the first of cluster_variants.
static KInfo pick_cluster(const cf_engine* e, int lg, int nb, int J, cudaStream_t s, bool wide = false) {
    (void)nb, (void)J, (void)s;
    KInfo v[8];
    if (wide) return kernel_for(lg, true);
    const int k = cluster_variants(lg, v);
    const int forced = lg > MAX_LG ? e->cluster_pick[lg - MAX_LG - 1] : -1;
    if (forced >= 0 && forced < k) return v[forced];
    return k > 0 ? v[0] : kernel_for(lg);
}
int cf_kvariants_lg10(KInfo* out, int cap);
int cf_kvariants_lg11(KInfo* out, int cap);
int cf_kvariants_lg12(KInfo* out, int cap);
int cf_kvariants_lg13(KInfo* out, int cap);
int cf_kvariants_lg14(KInfo* out, int cap);
// The geometries compiled for transform length 2^lg (50-bit kernel), the default first.
static int variants_for(int lg, KInfo* v, int cap) {
    switch (lg) {
        case 10: return cf_kvariants_lg10(v, cap);
        case 11: return cf_kvariants_lg11(v, cap);
        case 12: return cf_kvariants_lg12(v, cap);
        case 13: return cf_kvariants_lg13(v, cap);
        case 14: return cf_kvariants_lg14(v, cap);
        default:
            if (cap > 0) v[0] = kernel_for(lg);
            return kernel_for(lg).fn ? 1 : 0;
    }
}
constexpr int MAX_VARIANTS = 8;
// The kernel an engine runs: for primes below 2^50 the geometry it was tuned to, else the default.
static KInfo kernel_of(const cf_engine* e, int lg, bool wide) {
    if (!wide && e && lg >= 0 && lg <= MAX_LG && e->tuned[lg] > 0) {
        KInfo v[MAX_VARIANTS];
        if (e->tuned[lg] < variants_for(lg, v, MAX_VARIANTS)) return v[e->tuned[lg]];
    }
    return kernel_for(lg, wide);
}

struct Plan {
    int lg, F, d0, nmax, J;
    bool wide = false;  // some prime is 2^50 or above: the kernels for primes below 2^62
    KInfo ki;           // the kernel that runs the batch
    Layout lay;
    size_t ws_words;
};
// The kernel this engine runs for the plan and the workspace layout its geometry needs (the
// pass-0 twiddle tables follow the entries per thread); again whenever wide or F changes.
static int finalize(cf_engine* e, Plan& pl) {
    pl.ki = kernel_of(e, pl.lg, pl.wide);
    if (!pl.ki.fn) return fail(e, CF_ERR_UNSUPPORTED, "no kernel for this transform length");
    const int nw = pl.ki.threads >= 32 ? pl.ki.threads / 32 : 1;
    // cluster kernels: row sums for the largest cluster, so any cluster size can run the layout
    pl.lay = make_layout(pl.nmax, pl.F, 1 << pl.lg, pl.J, nw, pl.ki.r, pl.lg > MAX_LG ? MAX_CLUSTER : 1);
    pl.ws_words = pl.lay.total;
    return CF_OK;
}

static int plan(cf_engine* e, int nmax, int d, int model, const int* qn, const int* qM, int J, Plan& pl) {
    if (nmax < 1 || d < 1 || (model != CF_MODEL_SUBSET && model != CF_MODEL_REPLACEMENT) || J < 0)
        return fail(e, CF_ERR_ARG, "bad nmax, d, model or J");
    if (J > 0 && (!qn || !qM)) return fail(e, CF_ERR_ARG, "null query arrays");
    int F = nmax;
    for (int j = 0; j < J; ++j) {
        if (qn[j] < 1 || qn[j] > nmax || qM[j] <= qn[j]) return fail(e, CF_ERR_ARG, "query needs 1 <= n <= nmax and M > n");
        if (model == CF_MODEL_SUBSET && d > qM[j]) return fail(e, CF_ERR_ARG, "subset model needs d <= M");
        F = std::max(F, qM[j]);
    }
    if (model == CF_MODEL_SUBSET && d > F) F = d;  // ifact[d] is read for g(v)
    const u64 L = cfh::transform_length((u64)nmax);
    int lg = 0;
    while ((1ull << lg) < L) ++lg;
    if (e && e->min_lg > lg) lg = e->min_lg;
    if (lg > MAX_LG_CLUSTER)
        return fail(e, CF_ERR_UNSUPPORTED, "transform length above 2^16 (nmax > 65536) is not supported by this build");
    pl.lg = lg;
    pl.F = F;
    pl.d0 = model == CF_MODEL_SUBSET ? d : 1;
    pl.nmax = nmax;
    pl.J = J;
    pl.wide = false;
    return finalize(e, pl);
}

static int check_primes(cf_engine* e, const u64* primes, int B, Plan& pl) {
    const u64 L = 1ull << pl.lg;
    pl.wide = false;
    for (int b = 0; b < B; ++b) {
        const u64 p = primes[b];
        if (p < 3 || (p & 1) == 0 || p >= (1ull << 62) || p <= (u64)pl.F || (p - 1) % L != 0 || !cfh::is_prime(p))
            return fail(e, CF_ERR_ARG, "prime " + std::to_string(p) + " is not an odd prime < 2^62 above max(n, M) with L | p-1");
        if (p >= (1ull << 50)) pl.wide = true;
    }
    return finalize(e, pl);
}

static int ensure_ws(cf_engine* e, size_t bytes) {
    if (e->ws_bytes >= bytes) return CF_OK;
    if (e->ws) cudaFree(e->ws);
    e->ws = nullptr;
    e->ws_bytes = 0;
    CF_CUDA(cudaMalloc(&e->ws, bytes), "workspace allocation");
    e->ws_bytes = bytes;
    return CF_OK;
}
static int ensure_queries(cf_engine* e, const int* qn, const int* qM, int J, cudaStream_t s) {
    if (J > e->qcap) {
        if (e->d_q) cudaFree(e->d_q);
        e->d_q = nullptr;
        CF_CUDA(cudaMalloc(&e->d_q, sizeof(int) * 2 * (size_t)J), "query allocation");
        e->qcap = J;
    }
    if (J) {
        CF_CUDA(cudaMemcpyAsync(e->d_q, qn, sizeof(int) * J, cudaMemcpyHostToDevice, s), "query upload");
        CF_CUDA(cudaMemcpyAsync(e->d_q + e->qcap, qM, sizeof(int) * J, cudaMemcpyHostToDevice, s), "query upload");
    }
    return CF_OK;
}

static long fit_batch(size_t per_prime) {
    // memory the stream-ordered pool keeps from freed resident tables counts as free: give it back
    int dev = 0;
    cudaMemPool_t pool;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess)
        cudaMemPoolTrimTo(pool, 0);
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return 0;
    const size_t reserve = (size_t)1 << 30;  // leave 1 GiB for the context, staging and other users
    if (fr <= reserve) return 0;
    return (long)((fr - reserve) / per_prime);
}

// A launch keeps the per-warp partial sums of its J queries in shared memory (8 J words per warp)
// beside the kernel's fixed part; more queries than the block's opt-in limit allows are refused.
int check_smem(cf_engine* e, size_t smem, int J) {
    int dev = 0, optin = 0;
    CF_CUDA(cudaGetDevice(&dev), "current device");
    CF_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev), "shared memory limit");
    if (smem > (size_t)optin)
        return fail(e, CF_ERR_UNSUPPORTED, std::to_string(J) + " queries need " + std::to_string(smem) +
                                               " bytes of shared memory per block; the device allows " + std::to_string(optin));
    return CF_OK;
}

// fixed_ws: use the workspace as it is (a graph capture, where nothing may be allocated)
// err: the device error word the launch reports to (the engine's unless given)
static int launch_batch(cf_engine* e, const u64* d_primes, int B, int nmax, int d, int model, int J, const Plan& pl,
                        u64* d_out, cudaStream_t s, u64* keep = nullptr, size_t keep_words = 0, bool fixed_ws = false,
                        int* err = nullptr) {
    if (!err) err = e->d_err;
    KInfo ki = pl.ki;
    if (!ki.fn) return fail(e, CF_ERR_UNSUPPORTED, "no kernel for this transform length");
    if (ki.cluster > 1 && keep) return fail(e, CF_ERR_UNSUPPORTED, "resident tables are built up to nmax = 16384");
    if (ki.cluster > 1) ki = pick_cluster(e, pl.lg, B, J, s, pl.wide);  // refined per chunk below
    size_t smem = ki.smem_for(J);
    int rc0 = check_smem(e, smem, J);
    if (rc0) return rc0;
    CF_CUDA(cudaFuncSetAttribute((const void*)ki.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
            "shared memory attribute");
    const size_t per_prime = pl.ws_words * 8;
    // chunk: as many primes as the workspace (grown once) holds
    long cap = (long)(e->ws_bytes / per_prime);
    if (fixed_ws && cap < 1) return fail(e, CF_ERR_NOMEM, "workspace holds no prime");
    // primes per launch this call wants: the batch, or at most max_ctas (whose workspace is then
    // all it takes, so a capped engine leaves the rest of the device to others)
    const long need = e->max_ctas > 0 ? std::min<long>(B, e->max_ctas) : B;
    if (cap < need && !fixed_ws) {
        long fitb = fit_batch(per_prime) + cap;  // what is free plus what is already held
        if (fitb < 1) return fail(e, CF_ERR_NOMEM, "not enough device memory for one prime");
        const long want = std::min<long>(need, fitb);
        int rc = ensure_ws(e, (size_t)want * per_prime);
        if (rc) return rc;
        cap = want;
    }
    if (e->max_ctas > 0) cap = std::min<long>(cap, e->max_ctas);
    CF_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s), "error reset");
    // equal chunks: a short tail launch would cost as much time as a full one
    const long nchunks = (B + cap - 1) / cap, per = (B + nchunks - 1) / nchunks;
    for (int at = 0; at < B; at += (int)per) {
        const int nb = (int)std::min<long>(per, B - at);
        KParams kp;
        kp.primes = d_primes + at;
        kp.B = nb;
        kp.n = nmax;
        kp.F = pl.F;
        kp.d = d;
        kp.d0 = pl.d0;
        kp.model = model;
        kp.J = J;
        kp.qn = e->d_q;
        kp.qM = e->d_q + e->qcap;
        kp.ws = e->ws;
        kp.ws_words = pl.ws_words;
        kp.lay = pl.lay;
        kp.out = d_out + (size_t)at * J;
        kp.err = err;
        kp.keep = keep ? keep + (size_t)at * keep_words : nullptr;
        kp.keep_words = keep_words;
        if (ki.cluster > 1) {  // one cluster of ki.cluster CTAs per prime
            ki = pick_cluster(e, pl.lg, nb, J, s, pl.wide);
            smem = ki.smem_for(J);
            rc0 = check_smem(e, smem, J);
            if (rc0) return rc0;
            CF_CUDA(cudaFuncSetAttribute((const void*)ki.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                    "shared memory attribute");
            if (ki.cluster > 8)
                CF_CUDA(cudaFuncSetAttribute((const void*)ki.fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1),
                        "cluster size attribute");
            cudaLaunchConfig_t cfg = {};
            cudaLaunchAttribute att[1];
            att[0].id = cudaLaunchAttributeClusterDimension;
            att[0].val.clusterDim.x = (unsigned)ki.cluster, att[0].val.clusterDim.y = 1, att[0].val.clusterDim.z = 1;
            cfg.gridDim = dim3((unsigned)(nb * ki.cluster)), cfg.blockDim = dim3((unsigned)ki.threads);
            cfg.dynamicSmemBytes = smem, cfg.stream = s, cfg.attrs = att, cfg.numAttrs = 1;
            CF_CUDA(cudaLaunchKernelEx(&cfg, ki.fn, kp), "cluster kernel launch");
        } else {
            ki.fn<<<nb, ki.threads, smem, s>>>(kp);
        }
        CF_CUDA(cudaGetLastError(), "kernel launch");
        ++e->launches;
    }
    return CF_OK;
}

extern "C" {

long cf_prime_range(long first, long count, uint64_t* out) {
    if (first < 0 || count < 0 || (count > 0 && !out)) return 0;
    const std::vector<u64> v = cfh::prime_range(first, count);
    std::copy(v.begin(), v.end(), out);
    return (long)v.size();
}
long cf_need(int n, int M, int d, int model) { return cfh::need(n, M, d, model); }
long cf_prime_range_bits(long first, long count, int bits, uint64_t* out) {
    if ((bits != 50 && bits != 62) || first < 0 || count < 0 || (count > 0 && !out)) return 0;
    const std::vector<u64> v = cfh::prime_range(first, count, bits);
    std::copy(v.begin(), v.end(), out);
    return (long)v.size();
}
long cf_need_bits(int n, int M, int d, int model, int bits) {
    if (bits != 50 && bits != 62) return -1;
    return cfh::need(n, M, d, model, bits);
}
int cf_engine_set_prime_bits(cf_engine* e, int bits) {
    if (!e || (bits != 50 && bits != 62)) return CF_ERR_ARG;
    e->prime_bits = bits;
    return CF_OK;
}
long cf_lib_primes(int n, int M, int d, int model, uint64_t* out, long cap) {
    if (n < 1 || M < 1 || d < 1 || (model == CF_MODEL_SUBSET && d > M) || cap < 0 || (cap > 0 && !out)) return -1;
    const std::vector<u64> v = cfh::lib_primes_for(n, M, d, model);
    if (v.empty()) return -1;
    std::copy(v.begin(), v.begin() + std::min<long>(cap, (long)v.size()), out);
    return (long)v.size();
}
uint64_t cf_transform_length(uint64_t nmax) { return cfh::transform_length(nmax); }

int cf_engine_create(int device, cf_engine** out) {
    if (!out) return CF_ERR_ARG;
    *out = nullptr;
    cf_engine* e = new cf_engine();
    e->device = device;
    cudaError_t c = cudaSetDevice(device);
    if (c == cudaSuccess) c = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
    if (c == cudaSuccess) c = cudaMalloc(&e->d_err, sizeof(int));
    if (c != cudaSuccess) {
        delete e;
        return CF_ERR_CUDA;
    }
    *out = e;
    return CF_OK;
}

void cf_engine_destroy(cf_engine* e) {
    if (!e) return;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    cudaFree(e->ws);
    cudaFree(e->d_err);
    cudaFree(e->d_q);
    cudaFree(e->d_primes);
    cudaFree(e->d_out);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
}

const char* cf_engine_last_error(const cf_engine* e) { return e ? e->err.c_str() : "no engine"; }
long cf_last_launches(const cf_engine* e) { return e ? e->launches : 0; }

uint64_t cf_workspace_bytes(int nmax, int Mmax, int J) {
    if (nmax < 1 || J < 0) return 0;
    const int F = std::max(nmax, Mmax);
    const u64 L = cfh::transform_length((u64)nmax);
    int lg = 0;
    while ((1ull << lg) < L) ++lg;
    if (lg > MAX_LG_CLUSTER) return 0;
    const KInfo ki = kernel_for(lg);
    return 8 * make_layout(nmax, F, (int)L, J, ki.threads >= 32 ? ki.threads / 32 : 1, ki.r, lg > MAX_LG ? MAX_CLUSTER : 1).total;
}

// ---- resident tables (serving) ----

struct cf_tables {
    int device = 0, n = 0, F = 0, d = 0, d0 = 0, model = 0, B = 0;
    u64* keep = nullptr;  // [B][keep_words]
    size_t keep_words = 0;
    u64* d_primes = nullptr;
    std::vector<u64> primes;
    u64* d_out = nullptr;  // [B][jcap] results of the waiting query form
    int jcap = 0;
    int* d_err = nullptr;     // the build's device error word
    int* h_err = nullptr;     // its pinned host copy, written when the build is done
    cudaEvent_t built = nullptr;
    bool pooled = false;      // keep / d_primes / d_err from the stream-ordered allocator
    bool err_slot = false;    // h_err is a slot of the shared pinned slab
};

// Pinned host words for the stream-ordered builds' error copies, taken from one slab allocated
// once per process: freeing pinned memory (cudaFreeHost) waits for the whole device, which would
// stall a serving loop that frees tables while rebuilds run.  Beyond the slab, plain pinned
// allocations are used.
namespace {
constexpr int ERR_SLOTS = 4096;
std::mutex g_slab_mu;
int* g_slab = nullptr;
std::vector<int> g_slab_free;
int* take_err_slot() {
    std::lock_guard<std::mutex> lk(g_slab_mu);
    if (!g_slab) {
        if (cudaHostAlloc(&g_slab, sizeof(int) * ERR_SLOTS, cudaHostAllocPortable) != cudaSuccess) {
            g_slab = nullptr;
            return nullptr;
        }
        for (int i = ERR_SLOTS - 1; i >= 0; --i) g_slab_free.push_back(i);
    }
    if (g_slab_free.empty()) return nullptr;
    const int i = g_slab_free.back();
    g_slab_free.pop_back();
    return g_slab + i;
}
void give_err_slot(int* p) {
    std::lock_guard<std::mutex> lk(g_slab_mu);
    g_slab_free.push_back((int)(p - g_slab));
}
}  // namespace

uint64_t cf_tables_bytes(int nmax, int Fmax) {
    if (nmax < 1) return 0;
    return 8 * make_keep_layout(nmax, std::max(nmax, Fmax)).total;
}

// The build of both forms: memory, the persistent launch with the table set's own error word, the
// error word's copy to the host and the `built` event, all on stream s; no wait.  The stream-ordered
// form (pooled) allocates and frees on streams, so neither blocks the device.
static int tables_build(cf_engine* e, const uint64_t* primes, int B, int nmax, int Fmax, int d, int model,
                        cudaStream_t s, bool pooled, cf_tables** out) {
    *out = nullptr;
    e->err.clear();
    e->launches = 0;
    if (B < 1 || !primes) return fail(e, CF_ERR_ARG, "bad prime buffer");
    Plan pl;
    int rc = plan(e, nmax, d, model, nullptr, nullptr, 0, pl);
    if (rc) return rc;
    pl.F = std::max(pl.F, Fmax);  // the largest M later queries may use
    rc = check_primes(e, primes, B, pl);  // and the layout for that F
    if (rc) return rc;
    if (pl.wide) return fail(e, CF_ERR_UNSUPPORTED, "resident tables hold primes below 2^50");
    if (pl.lg > MAX_LG) return fail(e, CF_ERR_UNSUPPORTED, "resident tables are built up to nmax = 16384");
    CF_CUDA(cudaSetDevice(e->device), "set device");
    cf_tables* t = new cf_tables();
    t->device = e->device, t->n = nmax, t->F = pl.F, t->d = d, t->d0 = pl.d0, t->model = model, t->B = B;
    t->keep_words = make_keep_layout(nmax, pl.F).total;
    t->primes.assign(primes, primes + B);
    t->pooled = pooled;
    const size_t kb = 8 * t->keep_words * (size_t)B;
    cudaError_t c = pooled ? cudaMallocAsync(&t->keep, kb, s) : cudaMalloc(&t->keep, kb);
    if (c == cudaSuccess) c = pooled ? cudaMallocAsync(&t->d_primes, 8 * (size_t)B, s) : cudaMalloc(&t->d_primes, 8 * (size_t)B);
    if (c == cudaSuccess) c = pooled ? cudaMallocAsync(&t->d_err, sizeof(int), s) : cudaMalloc(&t->d_err, sizeof(int));
    if (c == cudaSuccess && pooled && (t->h_err = take_err_slot()) != nullptr) t->err_slot = true;
    if (c == cudaSuccess && !t->h_err) c = cudaHostAlloc(&t->h_err, sizeof(int), cudaHostAllocDefault);
    if (c == cudaSuccess) c = cudaEventCreateWithFlags(&t->built, cudaEventDisableTiming);
    if (c == cudaSuccess) c = cudaMemcpyAsync(t->d_primes, primes, 8 * (size_t)B, cudaMemcpyHostToDevice, s);
    if (c != cudaSuccess) {
        cf_tables_free(t);
        return cuda_fail(e, c, "resident table allocation");
    }
    *t->h_err = -1;  // not done
    rc = launch_batch(e, t->d_primes, B, nmax, d, model, 0, pl, nullptr, s, t->keep, t->keep_words, false, t->d_err);
    if (rc == CF_OK) {
        c = cudaMemcpyAsync(t->h_err, t->d_err, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (c == cudaSuccess) c = cudaEventRecord(t->built, s);
        if (c != cudaSuccess) rc = cuda_fail(e, c, "table build");
    }
    if (rc) {
        cudaStreamSynchronize(s);
        cf_tables_free(t);
        return rc;
    }
    *out = t;
    return CF_OK;
}

int cf_tables_build(cf_engine* e, const uint64_t* primes, int B, int nmax, int Fmax, int d, int model, cf_tables** out) {
    if (!e || !out) return CF_ERR_ARG;
    int rc = tables_build(e, primes, B, nmax, Fmax, d, model, e->stream, false, out);
    if (rc) return rc;
    CF_CUDA(cudaEventSynchronize((*out)->built), "table build");
    if (*(*out)->h_err) {
        const int herr = *(*out)->h_err;
        cf_tables_free(*out);
        *out = nullptr;
        return fail(e, CF_ERR_DEVICE, "device check failed (code " + std::to_string(herr) + ")");
    }
    return CF_OK;
}

int cf_tables_build_async(cf_engine* e, const uint64_t* primes, int B, int nmax, int Fmax, int d, int model, void* stream,
                          cf_tables** out) {
    if (!e || !out) return CF_ERR_ARG;
    return tables_build(e, primes, B, nmax, Fmax, d, model, (cudaStream_t)stream, true, out);
}

int cf_tables_ready(const cf_tables* t) {
    if (!t || !t->built) return CF_ERR_ARG;
    if (cudaSetDevice(t->device) != cudaSuccess) return CF_ERR_CUDA;
    const cudaError_t c = cudaEventQuery(t->built);
    if (c == cudaErrorNotReady) return 0;
    if (c != cudaSuccess) return CF_ERR_CUDA;
    return *t->h_err ? CF_ERR_DEVICE : 1;
}

// Residues of the queries into d_residues[b * J + j] on stream s, as launches of up to TQ_MAXJ
// queries whose sizes travel in the kernel parameters; no wait.
static int tables_query(cf_engine* e, const cf_tables* t, const int* qn, const int* qM, int J, u64* d_out, cudaStream_t s) {
    if (J < 1 || !qn || !qM || !d_out) return fail(e, CF_ERR_ARG, "bad query buffers");
    for (int j = 0; j < J; ++j) {
        if (qn[j] < 1 || qn[j] > t->n || qM[j] <= qn[j] || qM[j] > t->F)
            return fail(e, CF_ERR_ARG, "query needs 1 <= n <= table n and n < M <= table F");
        if (t->model == CF_MODEL_SUBSET && t->d > qM[j]) return fail(e, CF_ERR_ARG, "subset model needs d <= M");
    }
    const size_t smem = tq_smem_bytes(t->n);
    CF_CUDA(cudaFuncSetAttribute((const void*)k_table_query<TQ_THREADS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
            "shared memory attribute");
    for (int j0 = 0; j0 < J; j0 += TQ_MAXJ) {
        TQParams tp;
        tp.primes = t->d_primes;
        tp.B = t->B, tp.n = t->n, tp.F = t->F, tp.d = t->d, tp.d0 = t->d0, tp.model = t->model;
        tp.J = std::min(TQ_MAXJ, J - j0);
        for (int j = 0; j < tp.J; ++j) tp.qn[j] = qn[j0 + j], tp.qM[j] = qM[j0 + j];
        tp.keep = t->keep;
        tp.keep_words = t->keep_words;
        tp.out = d_out + j0;
        tp.out_stride = (size_t)J;
        k_table_query<TQ_THREADS><<<t->B * tp.J, TQ_THREADS, smem, s>>>(tp);
        CF_CUDA(cudaGetLastError(), "query launch");
        ++e->launches;
    }
    return CF_OK;
}

int cf_tables_query_async(cf_engine* e, const cf_tables* t, const int* qn, const int* qM, int J, uint64_t* d_residues,
                          void* stream) {
    if (!e || !t) return CF_ERR_ARG;
    e->err.clear();
    e->launches = 0;
    CF_CUDA(cudaSetDevice(t->device), "set device");
    return tables_query(e, t, qn, qM, J, d_residues, (cudaStream_t)stream);
}

int cf_tables_query(cf_engine* e, const cf_tables* t, const int* qn, const int* qM, int J, uint64_t* residues) {
    if (!e || !t) return CF_ERR_ARG;
    e->err.clear();
    e->launches = 0;
    if (J < 1 || !qn || !qM || !residues) return fail(e, CF_ERR_ARG, "bad query buffers");
    CF_CUDA(cudaSetDevice(t->device), "set device");
    cf_tables* tm = const_cast<cf_tables*>(t);  // the waiting form's result buffer is per table set
    if (J > tm->jcap) {
        cudaFree(tm->d_out);
        tm->d_out = nullptr;
        tm->jcap = 0;
        CF_CUDA(cudaMalloc(&tm->d_out, 8 * (size_t)t->B * J), "query result buffer");
        tm->jcap = J;
    }
    cudaStream_t s = e->stream;
    CF_CUDA(cudaStreamWaitEvent(s, t->built, 0), "wait for the build");
    int rc = tables_query(e, t, qn, qM, J, tm->d_out, s);
    if (rc) return rc;
    CF_CUDA(cudaMemcpyAsync(residues, tm->d_out, 8 * (size_t)t->B * J, cudaMemcpyDeviceToHost, s), "query download");
    CF_CUDA(cudaStreamSynchronize(s), "query");
    return CF_OK;
}

int cf_tables_count(const cf_tables* t) { return t ? t->B : 0; }

void cf_tables_free(cf_tables* t) {
    if (!t) return;
    cudaSetDevice(t->device);
    if (t->pooled) {  // back to the pool in stream order, without waiting for the device
        cudaFreeAsync(t->keep, 0);
        cudaFreeAsync(t->d_primes, 0);
        cudaFreeAsync(t->d_err, 0);
    } else {
        cudaFree(t->keep);
        cudaFree(t->d_primes);
        cudaFree(t->d_err);
    }
    cudaFree(t->d_out);  // only the waiting query form allocates it
    if (t->err_slot) give_err_slot(t->h_err);
    else if (t->h_err) cudaFreeHost(t->h_err);
    if (t->built) cudaEventDestroy(t->built);
    delete t;
}

int cf_engine_set_max_ctas(cf_engine* e, int n) {
    if (!e || n < 0) return CF_ERR_ARG;
    e->max_ctas = n;
    return CF_OK;
}

long cf_resident_primes(cf_engine* e, int nmax, int Mmax, int J) {
    if (!e || nmax < 1 || J < 0) return 0;
    if (cudaSetDevice(e->device) != cudaSuccess) return 0;
    std::vector<int> qn((size_t)std::max(J, 1), nmax), qM((size_t)std::max(J, 1), std::max(Mmax, nmax + 1));
    Plan pl;
    if (plan(e, nmax, 3, CF_MODEL_SUBSET, qn.data(), qM.data(), J, pl)) return 0;
    const KInfo ki = pl.ki.cluster > 1 ? pick_cluster(e, pl.lg, 1, J, e->stream) : pl.ki;
    const size_t smem = ki.smem_for(J);
    if (ki.cluster > 1) return resident_clusters(ki, smem, e->stream);
    int per_sm = 0, sms = 0;
    if (cudaFuncSetAttribute((const void*)ki.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ki.fn, ki.threads, smem) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device) != cudaSuccess)
        return 0;
    return (long)per_sm * sms;
}

int cf_engine_set_transform_lg(cf_engine* e, int lg) {
    if (!e || lg < 0 || lg > MAX_LG_CLUSTER) return CF_ERR_ARG;
    e->min_lg = lg;
    return CF_OK;
}

long cf_max_batch(cf_engine* e, int nmax, int Mmax, int J) {
    if (!e) return 0;
    cudaSetDevice(e->device);
    const uint64_t per = cf_workspace_bytes(nmax, Mmax, J);
    if (!per) return 0;
    return fit_batch(per) + (long)(e->ws_bytes / per);
}

int cf_residues_async(cf_engine* e, const uint64_t* d_primes, int B, int nmax, int d, int model, const int* qn,
                      const int* qM, int J, uint64_t* d_residues, void* stream) {
    if (!e) return CF_ERR_ARG;
    e->err.clear();
    e->launches = 0;
    if (B < 0 || (B > 0 && (!d_primes || (J > 0 && !d_residues)))) return fail(e, CF_ERR_ARG, "bad batch buffers");
    Plan pl;
    int rc = plan(e, nmax, d, model, qn, qM, J, pl);
    if (rc) return rc;
    if (B == 0) return CF_OK;
    pl.wide = e->prime_bits > 50;
    rc = finalize(e, pl);
    if (rc) return rc;
    CF_CUDA(cudaSetDevice(e->device), "set device");
    cudaStream_t s = (cudaStream_t)stream;  // NULL is the CUDA default stream
    rc = ensure_queries(e, qn, qM, J, s);
    if (rc) return rc;
    return launch_batch(e, d_primes, B, nmax, d, model, J, pl, d_residues, s);
}

int cf_residues(cf_engine* e, const uint64_t* primes, int B, int nmax, int d, int model, const int* qn, const int* qM,
                int J, uint64_t* residues) {
    if (!e) return CF_ERR_ARG;
    e->err.clear();
    e->launches = 0;
    if (B < 0 || (B > 0 && (!primes || (J > 0 && !residues)))) return fail(e, CF_ERR_ARG, "bad batch buffers");
    Plan pl;
    int rc = plan(e, nmax, d, model, qn, qM, J, pl);
    if (rc) return rc;
    rc = check_primes(e, primes, B, pl);
    if (rc) return rc;
    if (B == 0) return CF_OK;
    CF_CUDA(cudaSetDevice(e->device), "set device");
    cudaStream_t s = e->stream;
    if ((size_t)B > e->io_cap || J > e->jcap) {
        cudaFree(e->d_primes);
        cudaFree(e->d_out);
        e->d_primes = nullptr;
        e->d_out = nullptr;
        e->io_cap = 0;
        CF_CUDA(cudaMalloc(&e->d_primes, 8 * (size_t)B), "prime buffer");
        CF_CUDA(cudaMalloc(&e->d_out, 8 * (size_t)B * std::max(J, 1)), "residue buffer");
        e->io_cap = (size_t)B;
        e->jcap = std::max(J, 1);
    }
    CF_CUDA(cudaMemcpyAsync(e->d_primes, primes, 8 * (size_t)B, cudaMemcpyHostToDevice, s), "prime upload");
    rc = ensure_queries(e, qn, qM, J, s);
    if (rc) return rc;
    rc = launch_batch(e, e->d_primes, B, nmax, d, model, J, pl, e->d_out, s);
    if (rc) return rc;
    int herr = 0;
    if (J) CF_CUDA(cudaMemcpyAsync(residues, e->d_out, 8 * (size_t)B * J, cudaMemcpyDeviceToHost, s), "residue download");
    CF_CUDA(cudaMemcpyAsync(&herr, e->d_err, sizeof(int), cudaMemcpyDeviceToHost, s), "error download");
    CF_CUDA(cudaStreamSynchronize(s), "batch");
    if (herr) return fail(e, CF_ERR_DEVICE, "device check failed (code " + std::to_string(herr) + ")");
    return CF_OK;
}

struct cf_batch_graph {
    int device = 0;
    u64* ws = nullptr;  // the batch's own workspace, query table and error word
    size_t ws_bytes = 0;
    int* d_q = nullptr;
    int qcap = 0;
    int* d_err = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    long launches = 0;
};

void cf_batch_graph_destroy(cf_batch_graph* g) {
    if (!g) return;
    cudaSetDevice(g->device);
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    cudaFree(g->ws);
    cudaFree(g->d_q);
    cudaFree(g->d_err);
    delete g;
}

int cf_batch_graph_create(cf_engine* e, const uint64_t* d_primes, int B, int nmax, int d, int model, const int* qn,
                          const int* qM, int J, uint64_t* d_residues, cf_batch_graph** out) {
    if (!e || !out) return CF_ERR_ARG;
    *out = nullptr;
    e->err.clear();
    e->launches = 0;
    if (B < 1 || !d_primes || (J > 0 && !d_residues)) return fail(e, CF_ERR_ARG, "bad batch buffers");
    Plan pl;
    int rc = plan(e, nmax, d, model, qn, qM, J, pl);
    if (rc) return rc;
    pl.wide = e->prime_bits > 50;
    rc = finalize(e, pl);
    if (rc) return rc;
    CF_CUDA(cudaSetDevice(e->device), "set device");
    cf_batch_graph* g = new cf_batch_graph();
    g->device = e->device;
    cudaStream_t cs = nullptr;
    // The graph's buffers stand in for the engine's while the batch is sized and captured, so the
    // captured launches address them; the engine's own come back afterwards.
    std::swap(e->ws, g->ws), std::swap(e->ws_bytes, g->ws_bytes), std::swap(e->d_q, g->d_q), std::swap(e->qcap, g->qcap),
        std::swap(e->d_err, g->d_err);
    auto run = [&]() -> int {
        CF_CUDA(cudaMalloc(&e->d_err, sizeof(int)), "error word");
        CF_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "capture stream");
        int r = ensure_queries(e, qn, qM, J, cs);
        if (r) return r;
        // allocate the workspace outside the capture: the captured call then finds it in place
        const size_t per_prime = pl.ws_words * 8;
        const long fitb = fit_batch(per_prime);
        if (fitb < 1) return fail(e, CF_ERR_NOMEM, "not enough device memory for one prime");
        r = ensure_ws(e, (size_t)std::min<long>(B, fitb) * per_prime);
        if (r) return r;
        CF_CUDA(cudaStreamSynchronize(cs), "query upload");
        CF_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal), "begin capture");
        r = launch_batch(e, d_primes, B, nmax, d, model, J, pl, d_residues, cs, nullptr, 0, true);
        cudaGraph_t gr = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(cs, &gr);
        g->graph = gr;
        if (r) return r;
        CF_CUDA(ce, "end capture");
        CF_CUDA(cudaGraphInstantiate(&g->exec, g->graph, 0), "graph instantiation");
        g->launches = e->launches;
        return CF_OK;
    };
    rc = run();
    std::swap(e->ws, g->ws), std::swap(e->ws_bytes, g->ws_bytes), std::swap(e->d_q, g->d_q), std::swap(e->qcap, g->qcap),
        std::swap(e->d_err, g->d_err);
    if (cs) cudaStreamDestroy(cs);
    if (rc) {
        cf_batch_graph_destroy(g);
        return rc;
    }
    *out = g;
    return CF_OK;
}

int cf_batch_graph_launch(cf_batch_graph* g, void* stream) {
    if (!g || !g->exec) return CF_ERR_ARG;
    if (cudaSetDevice(g->device) != cudaSuccess) return CF_ERR_CUDA;
    return cudaGraphLaunch(g->exec, (cudaStream_t)stream) == cudaSuccess ? CF_OK : CF_ERR_CUDA;
}

int cf_batch_graph_status(cf_batch_graph* g, void* stream) {
    if (!g) return CF_ERR_ARG;
    if (cudaSetDevice(g->device) != cudaSuccess) return CF_ERR_CUDA;
    int herr = 0;
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaMemcpyAsync(&herr, g->d_err, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return CF_ERR_CUDA;
    return herr ? CF_ERR_DEVICE : CF_OK;
}

long cf_batch_graph_launches(const cf_batch_graph* g) { return g ? g->launches : 0; }

// ---- autotuning of the kernel geometry ----

int cf_tune_variants(int lg, int* log2_entries, int* threads, int* ctas_per_sm, int cap) {
    if (lg < 0 || lg > MAX_LG_CLUSTER || cap < 0) return -1;
    KInfo v[MAX_VARIANTS];
    const int k = lg > MAX_LG ? cluster_variants(lg, v) : variants_for(lg, v, MAX_VARIANTS);
    for (int i = 0; i < k && i < cap; ++i) {
        if (log2_entries) log2_entries[i] = v[i].r;
        if (threads) threads[i] = v[i].threads;
        if (ctas_per_sm) ctas_per_sm[i] = v[i].mb;
    }
    return k;
}

int cf_tune_set(cf_engine* e, int lg, int variant) {
    if (e && lg > MAX_LG && lg <= MAX_LG_CLUSTER) {  // a cluster size, or -1: chosen per batch
        KInfo v[8];
        if (variant < -1 || variant >= cluster_variants(lg, v)) return CF_ERR_ARG;
        e->cluster_pick[lg - MAX_LG - 1] = variant;
        return CF_OK;
    }
    if (!e || lg < 0 || lg > MAX_LG || variant < 0) return CF_ERR_ARG;
    KInfo v[MAX_VARIANTS];
    if (variant >= variants_for(lg, v, MAX_VARIANTS)) return CF_ERR_ARG;
    e->tuned[lg] = variant;
    return CF_OK;
}

int cf_tune_get(const cf_engine* e, int lg) {
    if (e && lg > MAX_LG && lg <= MAX_LG_CLUSTER) return e->cluster_pick[lg - MAX_LG - 1];
    return e && lg >= 0 && lg <= MAX_LG ? e->tuned[lg] : -1;
}

int cf_autotune(cf_engine* e, int nmax, int Mmax, int d, int B, double* rates, int cap, int* chosen) {
    if (!e || B < 1 || nmax < 1) return CF_ERR_ARG;
    e->err.clear();
    const u64 L = cfh::transform_length((u64)nmax);
    int lg = 0;
    while ((1ull << lg) < L) ++lg;
    if (lg > MAX_LG_CLUSTER) return fail(e, CF_ERR_UNSUPPORTED, "transform length above 2^16");
    const bool cl = lg > MAX_LG;  // cluster geometries: pinned through cluster_pick
    KInfo v[MAX_VARIANTS];
    const int k = cl ? cluster_variants(lg, v) : variants_for(lg, v, MAX_VARIANTS);
    int& pick = cl ? e->cluster_pick[lg - MAX_LG - 1] : e->tuned[lg];
    const std::vector<u64> primes = cfh::prime_range(0, B);
    const int qn[1] = {nmax}, qM[1] = {std::max(Mmax, nmax + 1)};
    std::vector<u64> first_out, out((size_t)B);
    const int saved = pick;
    int best = 0;
    double best_rate = -1;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CF_CUDA(cudaSetDevice(e->device), "set device");
    CF_CUDA(cudaEventCreate(&e0), "event");
    CF_CUDA(cudaEventCreate(&e1), "event");
    int rc = CF_OK;
    for (int i = 0; i < k && rc == CF_OK; ++i) {
        pick = i;
        float ms = 0;
        for (int rep = 0; rep < 2 && rc == CF_OK; ++rep) {  // a warm-up launch, then the timed one
            if (cudaEventRecord(e0, e->stream) != cudaSuccess) rc = fail(e, CF_ERR_CUDA, "event");
            if (rc == CF_OK) rc = cf_residues(e, primes.data(), B, nmax, d, CF_MODEL_SUBSET, qn, qM, 1, out.data());
            if (rc == CF_OK && (cudaEventRecord(e1, e->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                                cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
                rc = fail(e, CF_ERR_CUDA, "timing");
        }
        if (rc) break;
        if (i == 0) first_out = out;
        else if (out != first_out)  // every geometry computes the same residues
            rc = fail(e, CF_ERR_DEVICE, "geometry " + std::to_string(i) + " disagrees with the default");
        const double rate = B / (ms * 1e-3);
        if (rates && i < cap) rates[i] = rate;
        if (rate > best_rate) best_rate = rate, best = i;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    pick = rc == CF_OK ? best : saved;
    if (chosen) *chosen = pick;
    return rc;
}

}  // extern "C"
