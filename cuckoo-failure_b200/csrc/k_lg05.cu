// Instantiation of the per-prime kernel for transform length 2^5.
#include "kernel_lg.cuh"

cfb::KInfo cf_kinfo_lg5() { return cfb::kinfo<5>(); }
cfb::KInfo cf_kinfo_lg5_w() { return cfb::kinfo<5, true>(); }
