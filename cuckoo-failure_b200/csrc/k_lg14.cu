// Instantiation of the per-prime kernel for transform length 2^14.
#include "kernel_lg.cuh"

cfb::KInfo cf_kinfo_lg14() { return cfb::kinfo<14>(); }
cfb::KInfo cf_kinfo_lg14_w() { return cfb::kinfo<14, true>(); }
