// Instantiation of the per-prime kernel for transform length 2^6.
#include "kernel_lg.cuh"

cfb::KInfo cf_kinfo_lg6() { return cfb::kinfo<6>(); }
cfb::KInfo cf_kinfo_lg6_w() { return cfb::kinfo<6, true>(); }
