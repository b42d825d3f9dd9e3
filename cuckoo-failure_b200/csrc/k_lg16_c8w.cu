// Instantiation of the cluster kernel for transform length 2^16 on clusters of 8 CTAs, primes below 2^62.
#include "kernel_lg.cuh"

cfb::KInfo cf_kinfo_lg16_c8_w() { return cfb::kinfo_cluster<16, 3, 4, true>(); }
