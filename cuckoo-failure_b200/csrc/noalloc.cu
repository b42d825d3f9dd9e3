// cf_residues_noalloc: the batch computation of cf_residues for callers that cannot allocate
// device memory.
//
// Some callers may not call cudaMalloc: a host program whose device memory is owned by another
// allocator (a framework pool sized to the whole card), code running where allocation is
// forbidden or would synchronize the device, or an embedding that must not grow the process's
// device footprint after start-up.  This entry point never allocates: its scratch (the suffix
// tables, per-prime tables, staged primes, queries, residues and the error word) lives in one
// file-scope device array of CF_NOALLOC_SCRATCH_BYTES, which every GPU that loads the library
// holds until the process exits.
//
// Contract:
//  * The first call on a device resolves the array's device address with cudaGetSymbolAddress
//    (with that device current) and caches it; make that first call before any stream capture.
//  * Every call shares the one array and finds the previous call's contents there; the call
//    clears what must start at zero (the error word; the kernel zeroes its own accumulators).
//    Calls whose work overlaps on the GPU (different streams or threads) race on the array.
//  * A request whose single-prime workspace does not fit the array is rejected with
//    CF_ERR_NOMEM and a message naming the limit; nothing is launched.
//  * No cudaMalloc, cudaFree or allocating library routine is called.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "../../include/cuckoo_b200.h"
#include "host_common.hpp"
#include "kernel_lg.cuh"

using namespace cfb;

cfb::KInfo cf_kinfo_lg4();
cfb::KInfo cf_kinfo_lg5();
cfb::KInfo cf_kinfo_lg6();
cfb::KInfo cf_kinfo_lg7();
cfb::KInfo cf_kinfo_lg8();
cfb::KInfo cf_kinfo_lg9();
cfb::KInfo cf_kinfo_lg10();
cfb::KInfo cf_kinfo_lg11();
cfb::KInfo cf_kinfo_lg12();
cfb::KInfo cf_kinfo_lg13();
cfb::KInfo cf_kinfo_lg14();
cfb::KInfo cf_kinfo_lg4_w();
cfb::KInfo cf_kinfo_lg5_w();
cfb::KInfo cf_kinfo_lg6_w();
cfb::KInfo cf_kinfo_lg7_w();
cfb::KInfo cf_kinfo_lg8_w();
cfb::KInfo cf_kinfo_lg9_w();
cfb::KInfo cf_kinfo_lg10_w();
cfb::KInfo cf_kinfo_lg11_w();
cfb::KInfo cf_kinfo_lg12_w();
cfb::KInfo cf_kinfo_lg13_w();
cfb::KInfo cf_kinfo_lg14_w();

namespace {

constexpr size_t SCRATCH_WORDS = CF_NOALLOC_SCRATCH_BYTES / 8;
constexpr size_t HEAD_WORDS = 32;  // error word, padded to 256 bytes
constexpr int MAX_DEVICES = 64;

// The scratch.  In host code this name is only a handle for cudaGetSymbolAddress, never a
// device address.
__device__ __align__(256) u64 g_noalloc_scratch[SCRATCH_WORDS];

std::mutex g_mu;
u64* g_scratch_ptr[MAX_DEVICES] = {};
std::string g_err;

// wide: some prime is 2^50 or above (the kernels for primes below 2^62)
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
        default: return KInfo{nullptr, 0, 0, 0};
    }
}

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

// Device address of the scratch on the current device (resolved once per device).
int scratch_for_current_device(u64** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return fail(CF_ERR_CUDA, "no current CUDA device");
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t c = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (c != cudaSuccess || !p) return fail(CF_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(c));
        g_scratch_ptr[dev] = (u64*)p;
    }
    *out = g_scratch_ptr[dev];
    return CF_OK;
}

}  // namespace

extern "C" const char* cf_noalloc_last_error(void) { return g_err.c_str(); }

extern "C" int cf_residues_noalloc(const uint64_t* primes, int B, int nmax, int d, int model, const int* qn,
                                   const int* qM, int J, uint64_t* residues, void* stream) {
    std::lock_guard<std::mutex> lock(g_mu);
    g_err.clear();
    // arguments (the same rules as cf_residues)
    if (B < 0 || (B > 0 && (!primes || (J > 0 && !residues))) || nmax < 1 || d < 1 ||
        (model != CF_MODEL_SUBSET && model != CF_MODEL_REPLACEMENT) || J < 0 || (J > 0 && (!qn || !qM)))
        return fail(CF_ERR_ARG, "bad arguments");
    int F = nmax;
    for (int j = 0; j < J; ++j) {
        if (qn[j] < 1 || qn[j] > nmax || qM[j] <= qn[j]) return fail(CF_ERR_ARG, "query needs 1 <= n <= nmax and M > n");
        if (model == CF_MODEL_SUBSET && d > qM[j]) return fail(CF_ERR_ARG, "subset model needs d <= M");
        F = std::max(F, qM[j]);
    }
    if (model == CF_MODEL_SUBSET && d > F) F = d;
    const u64 L = cfh::transform_length((u64)nmax);
    int lg = 0;
    while ((1ull << lg) < L) ++lg;
    if (lg > 14) return fail(CF_ERR_UNSUPPORTED, "transform length above 2^14 is not supported");
    bool wide = false;
    for (int b = 0; b < B; ++b) {
        const u64 p = primes[b];
        if (p < 3 || (p & 1) == 0 || p >= (1ull << 62) || p <= (u64)F || (p - 1) % L != 0 || !cfh::is_prime(p))
            return fail(CF_ERR_ARG, "prime " + std::to_string(p) + " is not an odd prime < 2^62 above max(n, M) with L | p-1");
        if (p >= (1ull << 50)) wide = true;
    }
    const KInfo ki = kernel_for(lg, wide);
    if (!ki.fn) return fail(CF_ERR_UNSUPPORTED, "no kernel for this transform length");
    if (B == 0) return CF_OK;
    const Layout lay = make_layout(nmax, F, (int)L, J, ki.threads >= 32 ? ki.threads / 32 : 1, ki.r);
    // scratch layout: [error word][queries: J n's then J M's as ints][primes][residues][workspaces],
    // every region padded to 256 bytes
    auto pad = [](size_t w) { return (w + 31) & ~(size_t)31; };
    const size_t qwords = pad((size_t)J);  // J sizes n and J sizes M, 4 bytes each
    const size_t fixed = HEAD_WORDS + qwords;
    auto words_for = [&](size_t c) { return fixed + pad(c) + pad(c * (size_t)J) + c * lay.total; };
    if (words_for(1) > SCRATCH_WORDS)
        return fail(CF_ERR_NOMEM, "a table of nmax = " + std::to_string(nmax) + " needs " + std::to_string(8 * words_for(1)) +
                                      " bytes of scratch; the static scratch holds " + std::to_string(CF_NOALLOC_SCRATCH_BYTES) + " bytes");
    // primes per launch: as many as the padded layout holds
    size_t cap = std::min<size_t>((SCRATCH_WORDS - fixed) / (lay.total + 1 + (size_t)J), (size_t)B);
    cap = std::max<size_t>(cap, 1);
    while (cap > 1 && words_for(cap) > SCRATCH_WORDS) --cap;

    u64* scr = nullptr;
    int rc = scratch_for_current_device(&scr);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    int* d_err = (int*)scr;
    int* d_qn = (int*)(scr + HEAD_WORDS);
    int* d_qM = d_qn + J;
    u64* d_primes = scr + fixed;
    u64* d_out = d_primes + pad(cap);
    u64* d_ws = d_out + pad(cap * (size_t)J);
#define NA_CUDA(call, what)                                                                     \
    do {                                                                                        \
        cudaError_t c_ = (call);                                                                \
        if (c_ != cudaSuccess) return fail(CF_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(c_)); \
    } while (0)
    const size_t smem = ki.smem_for(J);
    {
        int dev = 0, optin = 0;
        NA_CUDA(cudaGetDevice(&dev), "current device");
        NA_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev), "shared memory limit");
        if (smem > (size_t)optin) return fail(CF_ERR_UNSUPPORTED, std::to_string(J) + " queries exceed the shared memory of one block");
    }
    NA_CUDA(cudaFuncSetAttribute((const void*)ki.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "shared memory attribute");
    NA_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), s), "error reset");
    if (J) {
        NA_CUDA(cudaMemcpyAsync(d_qn, qn, sizeof(int) * J, cudaMemcpyHostToDevice, s), "query upload");
        NA_CUDA(cudaMemcpyAsync(d_qM, qM, sizeof(int) * J, cudaMemcpyHostToDevice, s), "query upload");
    }
    for (int at = 0; at < B; at += (int)cap) {
        const int nb = (int)std::min<size_t>(cap, (size_t)(B - at));
        NA_CUDA(cudaMemcpyAsync(d_primes, primes + at, 8 * (size_t)nb, cudaMemcpyHostToDevice, s), "prime upload");
        KParams kp;
        kp.primes = d_primes;
        kp.B = nb;
        kp.n = nmax;
        kp.F = F;
        kp.d = d;
        kp.d0 = model == CF_MODEL_SUBSET ? d : 1;
        kp.model = model;
        kp.J = J;
        kp.qn = d_qn;
        kp.qM = d_qM;
        kp.ws = d_ws;
        kp.ws_words = lay.total;
        kp.lay = lay;
        kp.out = d_out;
        kp.err = d_err;
        ki.fn<<<nb, ki.threads, smem, s>>>(kp);
        NA_CUDA(cudaGetLastError(), "kernel launch");
        if (J) NA_CUDA(cudaMemcpyAsync(residues + (size_t)at * J, d_out, 8 * (size_t)nb * J, cudaMemcpyDeviceToHost, s), "residue download");
    }
    int herr = 0;
    NA_CUDA(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, s), "error download");
    NA_CUDA(cudaStreamSynchronize(s), "batch");
#undef NA_CUDA
    if (herr) return fail(CF_ERR_DEVICE, "device check failed (code " + std::to_string(herr) + ")");
    return CF_OK;
}
