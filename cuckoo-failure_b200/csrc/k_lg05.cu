// Instantiation of the per-prime kernel for transform length 2^5.
#include "kernel_lg.cuh"

cfb::KInfo cf_kinfo_lg5() { return cfb::kinfo<5>(); }
