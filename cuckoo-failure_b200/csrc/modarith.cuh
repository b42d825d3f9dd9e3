// Exact modular arithmetic for odd primes p < 2^50, built from 32 x 32 -> 64-bit integer
// multiplies (IMAD.WIDE on sm_100a).  Everything here is __host__ __device__ so the host tests and
// the CPU oracle comparison exercise the very same formulas the kernels run.
//
// Residues are kept in Montgomery form with R = 2^64: x is stored as x R mod p.  Any Montgomery
// radix gives the same canonical residues after from_mont, so the choice only affects speed; the
// reference (fast/cuckoo_fast.cu:84-99) uses R = 2^52 for its IFMA build.
//
// Products:
//  * mont_mul(a, b): a b R^{-1} mod p, fully reduced, for inputs a, b < 2^52 (lazy inputs allowed).
//  * shoup_mul(a, w, w'): a w mod p in [0, 2p) for a fixed multiplier w with the precomputed
//    companion w' = floor(w 2^64 / p) (Shoup's method); a may be any 64-bit value.
//  * shoup_mul_lazy: the same with a cheaper quotient estimate, result in [0, 4p); the hot loops
//    use it.  A Shoup product by a canonical constant preserves whatever form a is in.
//
// Primes of the fixed list have p = c 2^20 + 1 (fast/cuckoo_fast.cu:422-432).  For those, the
// product m p needed by the reduction is m + (m c) 2^20, which saves two wide multiplies; the
// `Special` variants use it, the generic ones work for every odd p < 2^50 (e.g. the 32-bit NTT
// primes of the library CLI, include/cuckoo/modint.hpp:183-196).
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define CF_HD __host__ __device__ __forceinline__
#else
#define CF_HD inline
#endif

namespace cfb {

typedef uint64_t u64;
typedef uint32_t u32;

CF_HD u64 wmul(u32 a, u32 b) { return (u64)a * (u64)b; }
CF_HD u32 lo32(u64 x) { return (u32)x; }
CF_HD u32 hi32(u64 x) { return (u32)(x >> 32); }

// Per-prime constants.  Layout is 32 bytes so a table of them is trivially indexable on device.
struct Mod {
    u64 p;     // the prime (odd, < 2^50)
    u64 pinv;  // p^{-1} mod 2^64
    u64 r1;    // 2^64 mod p: the Montgomery form of 1
    u64 r2;    // 2^128 mod p: converts a canonical residue into Montgomery form
};

// Full product of a, b < 2^56: (hi, lo) with a b = hi 2^64 + lo.
CF_HD void mul_full(u64 a, u64 b, u64& lo, u64& hi) {
    const u32 a0 = lo32(a), a1 = hi32(a), b0 = lo32(b), b1 = hi32(b);
    const u64 p00 = wmul(a0, b0), p01 = wmul(a0, b1), p10 = wmul(a1, b0), p11 = wmul(a1, b1);
    const u64 mid = p01 + p10 + (p00 >> 32);  // < 2^57 + 2^32: no overflow
    lo = (mid << 32) | (u64)lo32(p00);
    hi = p11 + (mid >> 32);
}

// High 64 bits of m p for a 64-bit m and p < 2^56 (generic modulus).
CF_HD u64 mulhi_mp(u64 m, u64 p) {
    const u32 m0 = lo32(m), m1 = hi32(m), p0 = lo32(p), p1 = hi32(p);
    const u64 q00 = wmul(m0, p0), q01 = wmul(m0, p1), q10 = wmul(m1, p0), q11 = wmul(m1, p1);
    const u64 mid = (q00 >> 32) + (u64)lo32(q01) + (u64)lo32(q10);
    return q11 + (q01 >> 32) + (q10 >> 32) + (mid >> 32);
}

// High 64 bits of m p for p = c 2^20 + 1: m p = m + (m c) 2^20.
CF_HD u64 mulhi_mp_special(u64 m, u32 c) {
    const u64 x0 = wmul(lo32(m), c), x1 = wmul(hi32(m), c);  // m c = x0 + x1 2^32 < 2^94
    const u64 xlo = x0 + ((u64)lo32(x1) << 32);
    const u64 xhi = (u64)hi32(x1) + (xlo < x0 ? 1u : 0u);  // m c = xhi 2^64 + xlo
    const u64 b = xlo << 20;                                // (m c 2^20) mod 2^64
    const u64 a = (xhi << 20) | (xlo >> 44);                // floor(m c 2^20 / 2^64)
    const u64 s = b + m;
    return a + (s < m ? 1u : 0u);
}

// Montgomery product a b 2^{-64} mod p in [0, p) for a b < p 2^64 (any a, b < 2^52 qualify).
CF_HD u64 mont_mul(u64 a, u64 b, const Mod& md) {
    u64 tl, th;
    mul_full(a, b, tl, th);
    const u64 m = tl * md.pinv;  // m p = T mod 2^64, so (T - m p) / 2^64 = th - hi(m p)
    const u64 mh = mulhi_mp(m, md.p);
    const u64 r = th - mh;
    return th >= mh ? r : r + md.p;
}
CF_HD u64 mont_mul_special(u64 a, u64 b, const Mod& md, u32 c) {
    u64 tl, th;
    mul_full(a, b, tl, th);
    const u64 m = tl * md.pinv;
    const u64 mh = mulhi_mp_special(m, c);
    const u64 r = th - mh;
    return th >= mh ? r : r + md.p;
}

// Shoup companion floor(w 2^64 / p) for w < p (host or device; a 128/64 division by shifts).
CF_HD u64 shoup_companion(u64 w, u64 p) {
#if defined(__CUDA_ARCH__)
    // Long division of w 2^64 by p, one quotient bit per step (w < p keeps the remainder < p).
    u64 rem = w, q = 0;
    for (int i = 0; i < 64; ++i) {
        const bool top = (rem >> 63) != 0;
        rem <<= 1;
        q <<= 1;
        if (top || rem >= p) {
            rem -= p;
            q |= 1;
        }
    }
    return q;
#else
    return (u64)((((unsigned __int128)w) << 64) / p);
#endif
}

// a w mod p in [0, 4p) for any 64-bit a, given w < p and wq = floor(w 2^64 / p).  The quotient
// estimate keeps only the partial products of a wq that reach the high word (a1 q1 and the high
// halves of a0 q1, a1 q0): it is at most 2 below floor(a wq / 2^64), which in turn is at most 1
// below floor(a w / p), so the remainder lies in [0, 4p).  5 wide + 4 low multiplies.
//
// On sm_100a a 32 x 32 -> high-32 multiply (mul.hi.u32) issues at under half the rate of a
// 32 x 32 -> 64 one (mul.wide.u32: 27 against 58 per SM per clock, measured), so the two high
// halves of the quotient estimate are taken from wide products.
CF_HD u64 shoup_mul_lazy(u64 a, u64 w, u64 wq, u64 p) {
    const u32 a0 = lo32(a), a1 = hi32(a), q0 = lo32(wq), q1 = hi32(wq);
#if defined(__CUDA_ARCH__)
    u64 t1, t2, q;
    asm("mul.wide.u32 %0, %1, %2;" : "=l"(t1) : "r"(a0), "r"(q1));
    asm("mul.wide.u32 %0, %1, %2;" : "=l"(t2) : "r"(a1), "r"(q0));
    asm("mad.wide.u32 %0, %1, %2, %3;" : "=l"(q) : "r"(a1), "r"(q1), "l"((t1 >> 32) + (t2 >> 32)));
    // a w - q p modulo 2^64 with the subtraction folded into the multiplies:
    //   a0 w0 - q0 p0 = a0 w0 + q0 (2^32 - p0) - q0 2^32                       (one mad.wide)
    //   high word += a0 w1 + a1 w0 + q0 (-p1 - 1) + q1 (2^32 - p0)  (mod 2^32)  (four mad.lo)
    // (p odd, so 2^32 - p0 is a 32-bit value); the same value as a w - q p, two instructions fewer.
    const u32 w0 = lo32(w), w1 = hi32(w), qa = lo32(q), qb = hi32(q), np0 = 0u - lo32(p), np1m = ~hi32(p);
    u64 x, y;
    u32 rl, rh;
    asm("mul.wide.u32 %0, %1, %2;" : "=l"(x) : "r"(a0), "r"(w0));
    asm("mad.wide.u32 %0, %1, %2, %3;" : "=l"(y) : "r"(qa), "r"(np0), "l"(x));
    asm("mov.b64 {%0, %1}, %2;" : "=r"(rl), "=r"(rh) : "l"(y));
    asm("mad.lo.u32 %0, %1, %2, %0;" : "+r"(rh) : "r"(a0), "r"(w1));
    asm("mad.lo.u32 %0, %1, %2, %0;" : "+r"(rh) : "r"(a1), "r"(w0));
    asm("mad.lo.u32 %0, %1, %2, %0;" : "+r"(rh) : "r"(qa), "r"(np1m));
    asm("mad.lo.u32 %0, %1, %2, %0;" : "+r"(rh) : "r"(qb), "r"(np0));
    u64 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "r"(rl), "r"(rh));
    return r;  // below 4p < 2^64
#else
    const u64 q = wmul(a1, q1) + (wmul(a0, q1) >> 32) + (wmul(a1, q0) >> 32);
    return a * w - q * p;  // exact modulo 2^64, and the true value is below 4p < 2^64
#endif
}

// Shoup companion floor(w 2^64 / p) for w < p from three per-prime constants: mu = floor(2^64 / p),
// r = 2^64 mod p and rq = floor(r 2^64 / p).  Since w 2^64 = w mu p + w r, the companion is
// w mu + floor(w r / p); the second term is the quotient of a Shoup product by r, whose lazy
// estimate (shoup_mul_lazy's) is at most 3 low and is corrected against the remainder.  Every sum
// is below 2^64, so arithmetic modulo 2^64 is exact.  Replaces the 64-step division in hot code.
CF_HD u64 shoup_companion_fast(u64 w, u64 p, u64 mu, u64 r, u64 rq) {
    const u32 a0 = lo32(w), a1 = hi32(w), q0 = lo32(rq), q1 = hi32(rq);
    u64 q = wmul(a1, q1) + (wmul(a0, q1) >> 32) + (wmul(a1, q0) >> 32);
    u64 rem = w * r - q * p;  // the true remainder, below 4p
#pragma unroll
    for (int k = 0; k < 3; ++k)
        if (rem >= p) rem -= p, ++q;
    return w * mu + q;
}

// a w mod p in [0, 2p) for any 64-bit a, given w < p and wq = floor(w 2^64 / p).
CF_HD u64 shoup_mul(u64 a, u64 w, u64 wq, const Mod& md) {
    const u32 a0 = lo32(a), a1 = hi32(a), q0 = lo32(wq), q1 = hi32(wq);
    const u64 s00 = wmul(a0, q0), s01 = wmul(a0, q1), s10 = wmul(a1, q0), s11 = wmul(a1, q1);
    const u64 mid = (s00 >> 32) + (u64)lo32(s01) + (u64)lo32(s10);
    const u64 q = s11 + (s01 >> 32) + (s10 >> 32) + (mid >> 32);  // floor(a wq / 2^64)
    return a * w - q * md.p;                                        // exact: lies in [0, 2p)
}
CF_HD u64 shoup_mul_special(u64 a, u64 w, u64 wq, const Mod& md, u32 c) {
    const u32 a0 = lo32(a), a1 = hi32(a), q0 = lo32(wq), q1 = hi32(wq);
    const u64 s00 = wmul(a0, q0), s01 = wmul(a0, q1), s10 = wmul(a1, q0), s11 = wmul(a1, q1);
    const u64 mid = (s00 >> 32) + (u64)lo32(s01) + (u64)lo32(s10);
    const u64 q = s11 + (s01 >> 32) + (s10 >> 32) + (mid >> 32);
    const u64 qc = wmul(lo32(q), c) + ((u64)(hi32(q) * c) << 32);  // q c mod 2^64
    return a * w - (q + (qc << 20));                                // q p = q + q c 2^20
    (void)md;
}

CF_HD u64 reduce2p(u64 x, u64 p) { return x >= p ? x - p : x; }  // [0, 2p) -> [0, p)
CF_HD u64 madd(u64 a, u64 b, u64 p) {
    const u64 s = a + b;
    return s >= p ? s - p : s;
}
CF_HD u64 msub(u64 a, u64 b, u64 p) { return a >= b ? a - b : a - b + p; }

CF_HD u64 mont_pow(u64 base, u64 e, const Mod& md) {
    u64 r = md.r1;
    while (e) {
        if (e & 1) r = mont_mul(r, base, md);
        base = mont_mul(base, base, md);
        e >>= 1;
    }
    return r;
}
CF_HD u64 to_mont(u64 x, const Mod& md) { return mont_mul(x, md.r2, md); }  // x < 2^52
CF_HD u64 from_mont(u64 x, const Mod& md) { return mont_mul(x, 1, md); }

// Per-prime constants (host or device).
CF_HD Mod make_mod(u64 p) {
    Mod m;
    m.p = p;
    u64 x = p;  // Newton iteration for p^{-1} mod 2^64 (each step doubles the correct bits)
    for (int i = 0; i < 6; ++i) x *= 2 - p * x;
    m.pinv = x;
    // 2^64 mod p and 2^128 mod p by doubling (no 128-bit division on device)
    u64 r = 1;
    for (int i = 0; i < 64; ++i) r = madd(r, r, p);
    m.r1 = r;
    for (int i = 0; i < 64; ++i) r = madd(r, r, p);
    m.r2 = r;
    return m;
}

}  // namespace cfb
