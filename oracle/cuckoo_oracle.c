/* CPU oracle for the one-table suffix-table path (TEST INFRASTRUCTURE ONLY).
 *
 * A plain-C restatement of the reference algorithm (zcy05331/Cuckoo-Failure), used only as the
 * checker: by tests/, by __graft_entry__.smoke() and by bench.py's cpu_baseline leg.  The product
 * (the CUDA engine behind include/cuckoo_b200.h) never links or calls this file.
 *
 * Arithmetic: Montgomery form with R = 2^64 over unsigned __int128 products; any odd modulus
 * p < 2^63 works.  The formulas follow include/cuckoo/single_table.hpp (library form of the
 * algorithm) and fast/cuckoo_fast.cu (prime list, need(), transform length, Horner finish).
 * Results are canonical residues, so they compare byte for byte with the reference's output.
 *
 * Build: make -C oracle   (liboracle.so; plain gcc, no dependencies)
 */
#include "cuckoo_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef uint64_t u64;
typedef unsigned __int128 u128;

/* ---- modular arithmetic (Montgomery, R = 2^64) ---- */
typedef struct {
    u64 p, pinv, r1, r2;
} om;

static om om_make(u64 p) {
    om m;
    u64 x = p;
    for (int i = 0; i < 6; ++i) x *= 2 - p * x; /* p^{-1} mod 2^64 */
    m.p = p;
    m.pinv = x;
    m.r1 = (u64)((((u128)1) << 64) % p);
    m.r2 = (u64)(((u128)m.r1 * m.r1) % p);
    return m;
}
static inline u64 om_mul(u64 a, u64 b, const om* m) { /* a b R^{-1} mod p, a, b < p */
    const u128 t = (u128)a * b;
    const u64 tl = (u64)t, th = (u64)(t >> 64);
    const u64 q = tl * m->pinv;
    const u64 qh = (u64)(((u128)q * m->p) >> 64);
    const u64 r = th - qh;
    return th >= qh ? r : r + m->p;
}
static inline u64 om_add(u64 a, u64 b, const om* m) {
    const u64 s = a + b;
    return s >= m->p ? s - m->p : s;
}
static inline u64 om_sub(u64 a, u64 b, const om* m) { return a >= b ? a - b : a - b + m->p; }
static inline u64 om_to(u64 x, const om* m) { return om_mul(x % m->p, m->r2, m); }
static inline u64 om_from(u64 x, const om* m) { return om_mul(x, 1, m); }
static u64 om_pow(u64 b, u64 e, const om* m) {
    u64 r = m->r1;
    while (e) {
        if (e & 1) r = om_mul(r, b, m);
        b = om_mul(b, b, m);
        e >>= 1;
    }
    return r;
}
static u64 om_inv(u64 x, const om* m) { return om_pow(x, m->p - 2, m); }

/* ---- prime list and sizes (fast/cuckoo_fast.cu:391-472) ---- */
static u64 h_mulmod(u64 a, u64 b, u64 p) { return (u64)((u128)a * b % p); }
static u64 h_powmod(u64 a, u64 e, u64 p) {
    u64 r = 1;
    a %= p;
    while (e) {
        if (e & 1) r = h_mulmod(r, a, p);
        a = h_mulmod(a, a, p);
        e >>= 1;
    }
    return r;
}
/* deterministic Miller-Rabin for n < 2^64 with the first twelve primes as bases
 * (fast/cuckoo_fast.cu:403-421) */
static int is_prime_u64(u64 n) {
    static const u64 bases[12] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    if (n < 2) return 0;
    for (int i = 0; i < 12; ++i)
        if (n % bases[i] == 0) return n == bases[i];
    u64 d = n - 1;
    int s = 0;
    while ((d & 1) == 0) d >>= 1, ++s;
    for (int i = 0; i < 12; ++i) {
        u64 x = h_powmod(bases[i], d, n);
        if (x == 1 || x == n - 1) continue;
        int comp = 1;
        for (int k = 1; k < s && comp; ++k) {
            x = h_mulmod(x, x, n);
            if (x == n - 1) comp = 0;
        }
        if (comp) return 0;
    }
    return 1;
}

long oc_prime_range(long first, long count, uint64_t* out) { /* fast/cuckoo_fast.cu:422-432 */
    long idx = 0, got = 0;
    for (u64 c = ((1ull << 50) - 2) >> 20; c >= 1 && got < count; --c) {
        const u64 p = (c << 20) + 1;
        if (!is_prime_u64(p)) continue;
        if (idx++ >= first) out[got++] = p;
    }
    return got;
}

static double log2_Q(int M, int d, int model) { /* fast/cuckoo_fast.cu:452-456 */
    long double b = 0;
    if (model == OC_REPLACEMENT) return (double)((long double)d * log2l((long double)M));
    for (int i = 0; i < d; ++i) b += log2l((long double)(M - i)) - log2l((long double)(i + 1));
    return (double)b;
}
long oc_need(int n, int M, int d, int model) { /* fast/cuckoo_fast.cu:457-459, PRIME_BITS = 50 */
    return (long)ceill(((long double)n * log2_Q(M, d, model) + 3) / 49) + 1;
}
uint64_t oc_transform_length(uint64_t nmax) { /* fast/cuckoo_fast.cu:460-472 */
    u64 L = 1;
    while (L < nmax) L <<= 1;
    return L < 16 ? 16 : L;
}

/* ---- NTT (standard iterative radix-2; any primitive root of order L gives the same cyclic
 * convolution, so the oracle need not mirror the reference's butterfly order) ---- */
typedef struct {
    u64 L;
    int lg;
    u64* rt;  /* rt[half + j] = w_{2 half}^j, Montgomery form */
    u64* rti; /* inverse roots */
    u64 linv; /* 1 / L */
} ntt_t;

static int ntt_init(ntt_t* t, u64 L, const om* m) {
    t->L = L;
    t->lg = 0;
    while (((u64)1 << t->lg) < L) ++t->lg;
    if ((m->p - 1) % L) return -1;
    /* a root of order L: x^((p-1)/L) whose (L/2)-th power is -1 (fast/cuckoo_fast.cu:815-820) */
    u64 w = 0;
    const u64 minus1 = om_sub(0, m->r1, m);
    for (u64 x = 2;; ++x) {
        w = om_pow(om_to(x, m), (m->p - 1) / L, m);
        if (om_pow(w, L / 2, m) == minus1) break;
    }
    const u64 wi = om_inv(w, m);
    t->rt = (u64*)calloc(L, 8);
    t->rti = (u64*)calloc(L, 8);
    for (u64 half = 1; half < L; half <<= 1) {
        const u64 wh = om_pow(w, L / (2 * half), m), whi = om_pow(wi, L / (2 * half), m);
        t->rt[half] = t->rti[half] = m->r1;
        for (u64 j = 1; j < half; ++j) {
            t->rt[half + j] = om_mul(t->rt[half + j - 1], wh, m);
            t->rti[half + j] = om_mul(t->rti[half + j - 1], whi, m);
        }
    }
    t->linv = om_inv(om_to(L, m), m);
    return 0;
}
static void ntt_free(ntt_t* t) {
    free(t->rt);
    free(t->rti);
}
static void ntt_run(const ntt_t* t, u64* a, int inverse, const om* m) {
    const u64 L = t->L;
    for (u64 i = 1, j = 0; i < L; ++i) { /* bit reversal */
        u64 bit = L >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            const u64 x = a[i];
            a[i] = a[j];
            a[j] = x;
        }
    }
    const u64* rt = inverse ? t->rti : t->rt;
    for (u64 half = 1; half < L; half <<= 1)
        for (u64 i = 0; i < L; i += 2 * half)
            for (u64 j = 0; j < half; ++j) {
                const u64 u = a[i + j], v = om_mul(a[i + j + half], rt[half + j], m);
                a[i + j] = om_add(u, v, m);
                a[i + j + half] = om_sub(u, v, m);
            }
    if (inverse)
        for (u64 i = 0; i < L; ++i) a[i] = om_mul(a[i], t->linv, m);
}

/* ---- factorials and the model (include/cuckoo/modint.hpp:336-355, single_table.hpp:16-23) ---- */
typedef struct {
    int n;
    u64 *fact, *ifact;
} facts_t;
static void facts_init(facts_t* f, int n, const om* m) {
    f->n = n;
    f->fact = (u64*)malloc(8 * (size_t)(n + 1));
    f->ifact = (u64*)malloc(8 * (size_t)(n + 1));
    f->fact[0] = m->r1;
    for (int i = 1; i <= n; ++i) f->fact[i] = om_mul(f->fact[i - 1], om_to((u64)i, m), m);
    f->ifact[n] = om_inv(f->fact[n], m);
    for (int i = n; i > 0; --i) f->ifact[i - 1] = om_mul(f->ifact[i], om_to((u64)i, m), m);
}
static void facts_free(facts_t* f) {
    free(f->fact);
    free(f->ifact);
}
static u64 binom(const facts_t* f, long a, long b, const om* m) { /* 0 unless 0 <= b <= a */
    if (a < 0 || b < 0 || b > a) return 0;
    return om_mul(om_mul(f->fact[a], f->ifact[b], m), f->ifact[a - b], m);
}
static u64 model_g(const facts_t* f, int v, int d, int model, const om* m) {
    if (v < 0) return 0;
    if (model == OC_REPLACEMENT) return om_pow(om_to((u64)v, m), (u64)d, m);
    return binom(f, v, d, m);
}

static size_t offV(size_t p) { return p * (p - 1) / 2; } /* row p >= 1, entries w = 0..p-1 */
static size_t offS(size_t v) { return v * (v + 1) / 2; } /* row v >= 0, entries q = 0..v */

static int check_args(u64 p, int nmax, int d, int model, int J, const int* qn, const int* qM, int* Fmax) {
    if (p < 3 || !(p & 1) || nmax < 1 || d < 1 || (model != OC_SUBSET && model != OC_REPLACEMENT)) return -1;
    int F = nmax;
    for (int j = 0; j < J; ++j) {
        if (qn[j] < 1 || qn[j] > nmax || qM[j] <= qn[j]) return -1;
        if (qM[j] > F) F = qM[j];
    }
    if ((u64)F >= p) return -1;
    *Fmax = F;
    return 0;
}

/* The suffix table V (Montgomery form), rows packed at offV.  include/cuckoo/single_table.hpp:178-229. */
static u64* build_ntt(const om* m, const facts_t* f, int nmax, int d, int model, int* err) {
    const u64 L = oc_transform_length((u64)nmax);
    ntt_t t;
    *err = 0;
    if (ntt_init(&t, L, m)) {
        *err = -1;
        return NULL;
    }
    u64* hat = (u64*)calloc(L, 8);
    for (int k = 1; k < nmax; ++k) hat[k] = om_mul(f->ifact[k], f->fact[k - 1], m); /* 1/k */
    ntt_run(&t, hat, 0, m);
    u64* gval = (u64*)malloc(8 * (size_t)(nmax + 1));
    u64* ginv = (u64*)malloc(8 * (size_t)(nmax + 1));
    for (int v = 0; v <= nmax; ++v) {
        gval[v] = model_g(f, v, d, model, m);
        ginv[v] = gval[v] ? om_inv(gval[v], m) : 0;
    }
    u64* V = (u64*)calloc(offV((size_t)nmax + 1), 8);
    u64* S = (u64*)calloc(offS((size_t)nmax), 8);
    u64* a = (u64*)malloc(8 * L);
    for (int v = 0; v < nmax; ++v) {
        if (v >= 1) { /* stage 1: S[v'][v] for v <= v' < nmax */
            int any = 0;
            memset(a, 0, 8 * L);
            for (int w = 0; w < v; ++w) {
                a[w] = om_mul(om_mul(V[offV(v) + w], f->ifact[w], m), f->ifact[v - w - 1], m);
                any |= a[w] != 0;
            }
            if (any) {
                ntt_run(&t, a, 0, m);
                for (u64 i = 0; i < L; ++i) a[i] = om_mul(a[i], hat[i], m);
                ntt_run(&t, a, 1, m);
                for (int vp = v; vp < nmax; ++vp)
                    S[offS(vp) + v] = om_mul(om_mul(f->fact[vp], f->ifact[vp - v], m), a[vp], m);
            }
        }
        if (gval[v] == 0) continue; /* V[p][v] = 0 when no candidate set fits in v slots */
        int any = 0;
        u64 gi = m->r1;
        memset(a, 0, 8 * L);
        for (int q = 1; q <= v; ++q) { /* stage 2 input */
            gi = om_mul(gi, ginv[v], m);
            a[q] = om_mul(om_mul(om_mul(S[offS(v) + q], gi, m), f->ifact[q], m), f->ifact[v - q], m);
            any |= a[q] != 0;
        }
        if (any) {
            ntt_run(&t, a, 0, m);
            for (u64 i = 0; i < L; ++i) a[i] = om_mul(a[i], hat[i], m);
            ntt_run(&t, a, 1, m);
        }
        u64 gp = om_pow(gval[v], (u64)v + 1, m);
        for (int p = v + 1; p <= nmax; ++p) {
            u64 val = binom(f, p - 1, v, m);
            if (any) /* c[nmax] is read at index 0 when L = nmax */
                val = om_sub(val, om_mul(om_mul(f->fact[p], f->ifact[p - v - 1], m), a[(u64)p & (L - 1)], m), m);
            V[offV(p) + v] = om_mul(val, gp, m);
            gp = om_mul(gp, gval[v], m);
        }
    }
    free(a);
    free(S);
    free(gval);
    free(ginv);
    free(hat);
    ntt_free(&t);
    return V;
}

/* O(nmax^3) construction, include/cuckoo/single_table.hpp:135-166. */
static u64* build_cubic(const om* m, const facts_t* f, int nmax, int d, int model) {
    u64* V = (u64*)calloc(offV((size_t)nmax + 1), 8);
    u64* S = (u64*)calloc(offS((size_t)nmax), 8);
    u64* gpow = (u64*)malloc(8 * (size_t)(nmax + 1));
    for (int v = 0; v < nmax; ++v) {
        if (v >= 1)
            for (int vp = v; vp < nmax; ++vp) {
                u64 s = 0;
                for (int w = 0; w < v; ++w)
                    if (V[offV(v) + w])
                        s = om_add(s, om_mul(om_mul(binom(f, vp - w - 1, vp - v, m), binom(f, vp, w, m), m), V[offV(v) + w], m), m);
                S[offS(vp) + v] = s;
            }
        const u64 g = model_g(f, v, d, model, m);
        gpow[0] = m->r1;
        for (int e = 1; e <= nmax; ++e) gpow[e] = om_mul(gpow[e - 1], g, m);
        for (int p = v + 1; p <= nmax; ++p) {
            u64 val = om_mul(binom(f, p - 1, v, m), gpow[p], m);
            for (int q = 1; q <= v; ++q)
                if (S[offS(v) + q])
                    val = om_sub(val,
                                 om_mul(om_mul(om_mul(binom(f, p - q - 1, p - v - 1, m), binom(f, p, q, m), m), gpow[p - q], m),
                                        S[offS(v) + q], m),
                                 m);
            V[offV(p) + v] = val;
        }
    }
    free(gpow);
    free(S);
    return V;
}

/* nbad(n, M) from the table, include/cuckoo/single_table.hpp:103-119:
 *   N_bad = sum_{q=1..n} C(n,q) Q^{n-q} sum_{w<q} C(M-w-1, M-q) C(M, w) V[q][w]. */
static u64 nbad(const om* m, const facts_t* f, const u64* V, int n, int M, int d, int model) {
    const u64 Q = model_g(f, M, d, model, m);
    u64 total = 0;
    for (int q = 1; q <= n; ++q) { /* Horner in Q (fast/cuckoo_fast.cu:884-890) */
        u64 inner = 0;
        for (int w = 0; w < q; ++w)
            if (V[offV(q) + w])
                inner = om_add(inner, om_mul(om_mul(binom(f, M - w - 1, M - q, m), binom(f, M, w, m), m), V[offV(q) + w], m), m);
        total = om_add(om_mul(total, Q, m), om_mul(binom(f, n, q, m), inner, m), m);
    }
    return om_from(total, m);
}

static int residues(int cubic, uint64_t p, int nmax, int d, int model, int J, const int* qn, const int* qM, uint64_t* out) {
    int F;
    if (check_args(p, nmax, d, model, J, qn, qM, &F)) return -1;
    const om m = om_make(p);
    facts_t f;
    facts_init(&f, F, &m);
    int err = 0;
    u64* V = cubic ? build_cubic(&m, &f, nmax, d, model) : build_ntt(&m, &f, nmax, d, model, &err);
    if (!V) {
        facts_free(&f);
        return err ? err : -1;
    }
    for (int j = 0; j < J; ++j) out[j] = nbad(&m, &f, V, qn[j], qM[j], d, model);
    free(V);
    facts_free(&f);
    return 0;
}

int oc_residues_ntt(uint64_t p, int nmax, int d, int model, int J, const int* qn, const int* qM, uint64_t* out) {
    return residues(0, p, nmax, d, model, J, qn, qM, out);
}
int oc_residues_cubic(uint64_t p, int nmax, int d, int model, int J, const int* qn, const int* qM, uint64_t* out) {
    return residues(1, p, nmax, d, model, J, qn, qM, out);
}

int oc_suffix_table(uint64_t p, int nmax, int d, int model, uint64_t* out) {
    int F;
    if (check_args(p, nmax, d, model, 0, NULL, NULL, &F)) return -1;
    const om m = om_make(p);
    facts_t f;
    facts_init(&f, F, &m);
    int err = 0;
    u64* V = build_ntt(&m, &f, nmax, d, model, &err);
    if (!V) {
        facts_free(&f);
        return -1;
    }
    const size_t cnt = offV((size_t)nmax + 1);
    for (size_t i = 0; i < cnt; ++i) out[i] = om_from(V[i], &m);
    free(V);
    facts_free(&f);
    return 0;
}

uint64_t oc_birthday(uint64_t p, int n, int M) { /* src/check.cpp:131 */
    const u64 mn = h_powmod((u64)M, (u64)n, p);
    u64 fall = 1;
    for (int i = 0; i < n; ++i) fall = h_mulmod(fall, (u64)(M - i), p);
    return mn >= fall ? mn - fall : mn + p - fall;
}
