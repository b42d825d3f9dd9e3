// Instantiation of the per-prime kernel for transform length 2^8.
#include "kernel_lg.cuh"

cfb::KInfo cf_kinfo_lg8() { return cfb::kinfo<8>(); }
cfb::KInfo cf_kinfo_lg8_w() { return cfb::kinfo<8, true>(); }
