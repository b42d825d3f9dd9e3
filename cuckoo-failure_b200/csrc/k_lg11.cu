// Instantiation of the per-prime kernel for transform length 2^11.
#include "kernel_lg.cuh"

cfb::KInfo cf_kinfo_lg11() { return cfb::kinfo<11>(); }
cfb::KInfo cf_kinfo_lg11_w() { return cfb::kinfo<11, true>(); }
