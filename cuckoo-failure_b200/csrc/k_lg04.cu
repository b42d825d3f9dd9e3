// Instantiation of the per-prime kernel for transform length 2^4.
#include "kernel_lg.cuh"

cfb::KInfo cf_kinfo_lg4() { return cfb::kinfo<4>(); }
cfb::KInfo cf_kinfo_lg4_w() { return cfb::kinfo<4, true>(); }
