// Autotuning candidates for transform length 2^14: the default geometry (k_lg14.cu) first,
// then other (entries per thread, CTAs per SM) pairs of the 50-bit kernel.
#include "kernel_lg.cuh"

cfb::KInfo cf_kinfo_lg14();
int cf_kvariants_lg14(cfb::KInfo* out, int cap) {
    const cfb::KInfo v[] = {
        cf_kinfo_lg14(),
        cfb::kinfo_geo<14, 5, 1>()};
    const int k = (int)(sizeof(v) / sizeof(v[0]));
    for (int i = 0; i < k && i < cap; ++i) out[i] = v[i];
    return k;
}
