// Instantiation of the cluster kernel for transform length 2^16 on clusters of 16 CTAs.
#include "kernel_lg.cuh"

cfb::KInfo cf_kinfo_lg16_c16() { return cfb::kinfo_cluster<16, 4>(); }
