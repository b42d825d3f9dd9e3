// Instantiation of the per-prime kernel for transform length 2^7.
#include "kernel_lg.cuh"

cfb::KInfo cf_kinfo_lg7() { return cfb::kinfo<7>(); }
cfb::KInfo cf_kinfo_lg7_w() { return cfb::kinfo<7, true>(); }
