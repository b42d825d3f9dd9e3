// Instantiation of the per-prime kernel for transform length 2^10.
#include "kernel_lg.cuh"

cfb::KInfo cf_kinfo_lg10() { return cfb::kinfo<10>(); }
cfb::KInfo cf_kinfo_lg10_w() { return cfb::kinfo<10, true>(); }
