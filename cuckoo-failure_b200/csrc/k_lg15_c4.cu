// Instantiation of the cluster kernel for transform length 2^15 on clusters of 4 CTAs.
#include "kernel_lg.cuh"

cfb::KInfo cf_kinfo_lg15_c4() { return cfb::kinfo_cluster<15, 2>(); }
