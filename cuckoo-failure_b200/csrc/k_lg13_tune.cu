// Autotuning candidates for transform length 2^13: the default geometry (k_lg13.cu) first,
// then other (entries per thread, CTAs per SM) pairs of the 50-bit kernel.
#include "kernel_lg.cuh"

cfb::KInfo cf_kinfo_lg13();
int cf_kvariants_lg13(cfb::KInfo* out, int cap) {
    const cfb::KInfo v[] = {
        cf_kinfo_lg13(),
        cfb::kinfo_geo<13, 5, 1>(),
        cfb::kinfo_geo<13, 4, 2>()};
    const int k = (int)(sizeof(v) / sizeof(v[0]));
    for (int i = 0; i < k && i < cap; ++i) out[i] = v[i];
    return k;
}
