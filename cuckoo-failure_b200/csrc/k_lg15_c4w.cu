// Instantiation of the cluster kernel for transform length 2^15 on clusters of 4 CTAs, primes below 2^62.
#include "kernel_lg.cuh"

cfb::KInfo cf_kinfo_lg15_c4_w() { return cfb::kinfo_cluster<15, 2, 4, true>(); }
