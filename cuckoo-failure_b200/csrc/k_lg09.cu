// Instantiation of the per-prime kernel for transform length 2^9.
#include "kernel_lg.cuh"

cfb::KInfo cf_kinfo_lg9() { return cfb::kinfo<9>(); }
cfb::KInfo cf_kinfo_lg9_w() { return cfb::kinfo<9, true>(); }
