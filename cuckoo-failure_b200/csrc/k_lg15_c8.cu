// Instantiation of the cluster kernel for transform length 2^15 on clusters of 8 CTAs.
#include "kernel_lg.cuh"

cfb::KInfo cf_kinfo_lg15_c8() { return cfb::kinfo_cluster<15, 3>(); }
