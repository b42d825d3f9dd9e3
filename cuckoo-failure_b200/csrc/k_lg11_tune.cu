// Autotuning candidates for transform length 2^11: the default geometry (k_lg11.cu) first,
// then other (entries per thread, CTAs per SM) pairs of the 50-bit kernel.
#include "kernel_lg.cuh"

cfb::KInfo cf_kinfo_lg11();
int cf_kvariants_lg11(cfb::KInfo* out, int cap) {
    const cfb::KInfo v[] = {
        cf_kinfo_lg11(),
        cfb::kinfo_geo<11, 4, 2>(),
        cfb::kinfo_geo<11, 4, 4>(),
        cfb::kinfo_geo<11, 3, 2>()};
    const int k = (int)(sizeof(v) / sizeof(v[0]));
    for (int i = 0; i < k && i < cap; ++i) out[i] = v[i];
    return k;
}
