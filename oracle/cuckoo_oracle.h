/* CPU oracle for the one-table suffix-table path (TEST INFRASTRUCTURE ONLY).
 *
 * Plain-C restatement of the reference algorithm, used exclusively as the checker by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg.  The product path never links it.
 * Each function cites the reference file:line it restates (paths inside zcy05331/Cuckoo-Failure).
 */
#ifndef CUCKOO_ORACLE_H
#define CUCKOO_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Sampling models: OC_SUBSET g(v) = C(v, d), Q = C(M, d); OC_REPLACEMENT g(v) = v^d, Q = M^d
 * (include/cuckoo/single_table.hpp:16-23). */
enum { OC_SUBSET = 0, OC_REPLACEMENT = 1 };

/* Primes number first .. first+count-1 of the fixed list: p = c 2^20 + 1 < 2^50, prime, largest
 * first (fast/cuckoo_fast.cu:403-432).  Returns how many were written. */
long oc_prime_range(long first, long count, uint64_t* out);

/* Number of 50-bit primes a query needs: ceil((n log2 Q + 3) / 49) + 1, evaluated in long
 * double exactly as fast/cuckoo_fast.cu:452-459 does (model OC_REPLACEMENT uses log2 Q = d log2 M). */
long oc_need(int n, int M, int d, int model);

/* Transform length max(16, next_pow2(nmax)) (fast/cuckoo_fast.cu:460-472). */
uint64_t oc_transform_length(uint64_t nmax);

/* N_bad mod p for J queries (qn[j], qM[j]) from one suffix table built to nmax >= max qn,
 * O(nmax^2 log nmax) with NTT convolutions (include/cuckoo/single_table.hpp:178-229 for the
 * build, :103-119 for nbad; fast/cuckoo_fast.cu:877-890 for the Horner form).  p must be an odd
 * prime with 2^k | p - 1 for 2^k >= the transform length and p > max(nmax, max qM).
 * Writes canonical residues to out[J].  Returns 0, or -1 on bad arguments. */
int oc_residues_ntt(uint64_t p, int nmax, int d, int model, int J, const int* qn, const int* qM, uint64_t* out);

/* The same from the O(nmax^3) construction (include/cuckoo/single_table.hpp:135-166): an
 * independent cross-check for small nmax (no transform, any odd prime p > max(nmax, qM)). */
int oc_residues_cubic(uint64_t p, int nmax, int d, int model, int J, const int* qn, const int* qM, uint64_t* out);

/* The whole suffix table V[p][w] (0 <= w < p <= nmax), packed by rows at offset p(p-1)/2, as
 * canonical residues (for checking retained tables).  out must hold nmax(nmax+1)/2 words. */
int oc_suffix_table(uint64_t p, int nmax, int d, int model, uint64_t* out);

/* N_bad mod p for d = 1 by the closed form M^n - M!/(M-n)! (src/check.cpp:122-146). */
uint64_t oc_birthday(uint64_t p, int n, int M);

#ifdef __cplusplus
}
#endif
#endif
