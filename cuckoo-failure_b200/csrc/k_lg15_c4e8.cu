// Instantiation of the cluster kernel for transform length 2^15 on clusters of 4 CTAs, 8 entries per thread.
#include "kernel_lg.cuh"

cfb::KInfo cf_kinfo_lg15_c4_e8() { return cfb::kinfo_cluster<15, 2, 3>(); }
