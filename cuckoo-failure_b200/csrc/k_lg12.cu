// Instantiation of the per-prime kernel for transform length 2^12.
#include "kernel_lg.cuh"

cfb::KInfo cf_kinfo_lg12() { return cfb::kinfo<12>(); }
cfb::KInfo cf_kinfo_lg12_w() { return cfb::kinfo<12, true>(); }
