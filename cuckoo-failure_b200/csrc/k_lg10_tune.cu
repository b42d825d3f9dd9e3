// Autotuning candidates for transform length 2^10: the default geometry (k_lg10.cu) first,
// then other (entries per thread, CTAs per SM) pairs of the 50-bit kernel.
#include "kernel_lg.cuh"

cfb::KInfo cf_kinfo_lg10();
int cf_kvariants_lg10(cfb::KInfo* out, int cap) {
    const cfb::KInfo v[] = {
        cf_kinfo_lg10(),
        cfb::kinfo_geo<10, 4, 8>(),
        cfb::kinfo_geo<10, 5, 8>()};
    const int k = (int)(sizeof(v) / sizeof(v[0]));
    for (int i = 0; i < k && i < cap; ++i) out[i] = v[i];
    return k;
}
