// Host-side helpers with the reference's exact semantics (fast/cuckoo_fast.cu:391-472): the
// fixed prime list, the prime count need(), the transform length.  Shared by the C ABI and the CLI.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

namespace cfh {

typedef uint64_t u64;
typedef unsigned __int128 u128;

inline u64 mulmod(u64 a, u64 b, u64 p) { return (u64)((u128)a * b % p); }
inline u64 powmod(u64 a, u64 e, u64 p) {
    u64 r = 1;
    a %= p;
    while (e) {
        if (e & 1) r = mulmod(r, a, p);
        a = mulmod(a, a, p);
        e >>= 1;
    }
    return r;
}
// Deterministic Miller-Rabin for n < 2^64 (bases: the first twelve primes).
inline bool is_prime(u64 n) {
    static const u64 bases[12] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    if (n < 2) return false;
    for (u64 q : bases)
        if (n % q == 0) return n == q;
    u64 d = n - 1;
    int s = 0;
    while ((d & 1) == 0) d >>= 1, ++s;
    for (u64 a : bases) {
        u64 x = powmod(a, d, n);
        if (x == 1 || x == n - 1) continue;
        bool comp = true;
        for (int i = 1; i < s && comp; ++i) {
            x = mulmod(x, x, n);
            if (x == n - 1) comp = false;
        }
        if (comp) return false;
    }
    return true;
}

constexpr int PRIME_BITS = 50;  // primes of the fixed list lie in (2^49, 2^50)
constexpr int TWO_ADIC = 20;    // and have 2^20 | p - 1
// The reference's -DFP_RB=64 build uses the list below 2^62 instead (fast/cuckoo_fast.cu:48-57):
// `bits` = 50 or 62 in the two functions below.

// Primes number first .. first+count-1 of the fixed list, largest first (fast/cuckoo_fast.cu:422-432).
inline std::vector<u64> prime_range(long first, long count, int bits = PRIME_BITS) {
    std::vector<u64> out;
    long idx = 0;
    for (u64 c = ((1ull << bits) - 2) >> TWO_ADIC; c >= 1 && (long)out.size() < count; --c) {
        const u64 p = (c << TWO_ADIC) + 1;
        if (!is_prime(p)) continue;
        if (idx++ >= first) out.push_back(p);
    }
    return out;
}

// log2 of the number of candidate sets per item (fast/cuckoo_fast.cu:452-456; the replacement
// model's Q = M^d as in src/cuckoo_fail.cpp:105-106).
inline double log2_Q(int M, int d, int model) {
    if (model == 1) return (double)((long double)d * std::log2((long double)M));
    long double b = 0;
    for (int i = 0; i < d; ++i) b += std::log2((long double)(M - i)) - std::log2((long double)(i + 1));
    return (double)b;
}
// Primes a query needs: the product of that many primes (each > 2^(bits-1)) exceeds 4 Q^n
// (fast/cuckoo_fast.cu:457-459).
inline long need(int n, int M, int d, int model, int bits = PRIME_BITS) {
    return (long)std::ceil(((long double)n * log2_Q(M, d, model) + 3) / (bits - 1)) + 1;
}
inline u64 transform_length(u64 nmax) {
    u64 L = 1;
    while (L < nmax) L <<= 1;
    return L < 16 ? 16 : L;
}

// ---- the 32-bit library's prime choice (src/cuckoo_fail.cpp:151-170) ----

// `count` primes p = c 2^k + 1 < 2^32 with c odd (so 2^k exactly divides p - 1), k from 31 down to
// min_pow2, c from its largest value down; returned largest first
// (include/cuckoo/modint.hpp:183-196).  Empty if there are not that many.
inline std::vector<u64> lib_ntt_primes(int count, int min_pow2) {
    std::vector<u64> out;
    for (int k = 31; k >= min_pow2 && (int)out.size() < count; --k) {
        long long c = (long long)((((1ull << 32) - 2)) >> k);
        if (c % 2 == 0) --c;
        for (; c >= 1 && (int)out.size() < count; c -= 2) {
            const u64 p = ((u64)c << k) + 1;
            if (is_prime(p)) out.push_back(p);
        }
    }
    if ((int)out.size() < count) return {};
    std::sort(out.rbegin(), out.rend());
    return out;
}

// The primes `cuckoo_fail single -n n -M M -d d` reconstructs N_bad from: the fewest primes of the
// list above whose product exceeds 4 Q^n, grown from n log2 Q / 31 + 2 as the library does, with
// its long-double sums.  The transform length there is max(2, next_pow2(n))
// (include/cuckoo/single_table.hpp:175).
inline std::vector<u64> lib_primes_for(int n, int M, int d, int model) {
    long double lq = 0;
    if (model == 1) lq = d * std::log2((long double)M);
    else
        for (int i = 0; i < d; ++i) lq += std::log2((long double)(M - i)) - std::log2((long double)(i + 1));
    const long double bits = n * lq;
    u64 L = 1;
    while (L < (u64)n) L <<= 1;
    if (L < 2) L = 2;
    int min_pow2 = 0;
    while ((1ull << min_pow2) < L) ++min_pow2;
    int count = (int)(bits / 31) + 2;
    while (true) {
        std::vector<u64> ps = lib_ntt_primes(count, min_pow2);
        if (ps.empty()) return ps;
        long double have = 0;
        for (u64 p : ps) have += std::log2((long double)p);
        if (have > bits + 2) return ps;
        count += (int)((bits + 2 - have) / 31) + 1;
    }
}

}  // namespace cfh
