// Internals shared by the C ABI's translation units (engine.cu, uneven.cu): the engine object,
// its error helpers and the kernel table.
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "../../include/cuckoo_b200.h"
#include "kernel_lg.cuh"

using cfb::u64;

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
// The kernel for transform length 2^lg: primes below 2^50, or (wide) below 2^62 (engine.cu).
cfb::KInfo kernel_for(int lg, bool wide = false);
cfb::KInfo cf_kinfo_lg15_c4();
cfb::KInfo cf_kinfo_lg15_c8();
cfb::KInfo cf_kinfo_lg15_c4_e8();
cfb::KInfo cf_kinfo_lg15_c4_w();
cfb::KInfo cf_kinfo_lg16_c8_w();
cfb::KInfo cf_kinfo_lg15_c8_e8();
cfb::KInfo cf_kinfo_lg16_c8();
cfb::KInfo cf_kinfo_lg16_c16();
constexpr int MAX_LG = 14;          // one CTA per prime (every entry point)
constexpr int MAX_LG_CLUSTER = 16;  // a cluster of CTAs per prime (cf_residues and its forms)
constexpr int MAX_CLUSTER = 16;     // the largest cluster a layout provides row sums for
struct cf_engine;
// CF_OK if a launch with J queries fits the device's shared memory per block (engine.cu)
int check_smem(cf_engine* e, size_t smem, int J);

// ------------------------------------------------------------------------------------------
// Engine
// ------------------------------------------------------------------------------------------
struct cf_engine {
    int device = 0;
    cudaStream_t stream = nullptr;
    u64* ws = nullptr;  // workspace
    size_t ws_bytes = 0;
    int* d_err = nullptr;
    int* d_q = nullptr;  // [2][qcap] query n and M
    int qcap = 0;
    u64* d_primes = nullptr;  // staging for cf_residues
    u64* d_out = nullptr;
    size_t io_cap = 0;  // primes capacity of d_primes; d_out has io_cap * jcap
    int jcap = 0;
    long launches = 0;
    int prime_bits = 50;  // for cf_residues_async, whose primes are not read on the host
    int max_ctas = 0;     // CTAs (primes) per launch at most, 0 = no cap
    int tuned[MAX_LG + 1] = {};  // geometry (index into the compiled variants) per transform length
    int min_lg = 0;              // transforms of at least 2^min_lg entries (cf_engine_set_transform_lg)
    int cluster_pick[MAX_LG_CLUSTER - MAX_LG] = {-1, -1};  // forced cluster variant per length above 2^14 (-1: by batch)
    std::string err;
};

inline int fail(cf_engine* e, int code, const std::string& msg) {
    if (e) e->err = msg;
    return code;
}
inline int cuda_fail(cf_engine* e, cudaError_t c, const char* what) {
    return fail(e, CF_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(c));
}
#define CF_CUDA(call, what)                              \
    do {                                                 \
        cudaError_t c_ = (call);                         \
        if (c_ != cudaSuccess) return cuda_fail(e, c_, what); \
    } while (0)

