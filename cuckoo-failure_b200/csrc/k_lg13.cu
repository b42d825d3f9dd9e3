// Instantiation of the per-prime kernel for transform length 2^13.
#include "kernel_lg.cuh"

cfb::KInfo cf_kinfo_lg13() { return cfb::kinfo<13>(); }
cfb::KInfo cf_kinfo_lg13_w() { return cfb::kinfo<13, true>(); }
