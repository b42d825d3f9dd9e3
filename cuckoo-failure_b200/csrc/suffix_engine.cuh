// One-table suffix-table engine: the per-prime build of V[p][v] and the nbad(n, M) queries,
// written as a sequence of block-wide phases so one CTA owns one prime from setup to residues.
//
// Reference semantics (zcy05331/Cuckoo-Failure):
//   include/cuckoo/single_table.hpp:80-119,178-229  the algorithm (two 1/t convolutions per step)
//   fast/cuckoo_fast.cu:145-243                      stage bodies (Stage1Pre/Post, Stage2Pre/Post)
//   fast/cuckoo_fast.cu:306-323,877-890              query sums and the Horner finish
//
// Design (B200, one CTA per prime, persistent over all steps v = 1 .. n-1):
//   * the length-L transform lives in shared memory between radix-2^R register passes;
//   * every multiplication by a constant is a Shoup product with a precomputed companion, and
//     values stay lazily reduced in [0, 2p) / [0, 4p) inside the transforms;
//   * the stage factors are folded into what is stored, so stage 1 needs no multiply on input:
//       Vs[p][w] = V[p][w] / (w! (p-1-w)! (p-1)!)        (stored V, column-major)
//       Ss[v][q] = S[v][q] / (q! (v-q)! v!)              (stored S, column-major)
//     which turns the reference's stage relations into
//       stage 1:  Ss[v'][v] = D[v'-v] inv[v] conv(Vs[v][.])[v'],            D[k] = 1/k!^2
//       stage 2:  Vs[p][v]  = g^p D[p-v-1] (D[v] - p conv(Ss[v][q] g^-q)[p])
//       query:    out(q)    = (q-1)! sum_w Vs[q][w] / (M - w)
//   * the queries are evaluated on the fly from the stage-1 input rows (the same U[w] the
//     reference's k_query builds), so a batch needs no separate pass over V.
//
// The kernel code runs through an Exec policy: on the GPU `each` is the calling thread and
// `sync` is __syncthreads; a CPU harness (tests) runs the same phases thread by thread.
#pragma once
#include "modarith.cuh"

namespace cfb {

enum { MODEL_SUBSET = 0, MODEL_REPLACEMENT = 1 };

#if defined(__CUDA_ARCH__)
#define CF_LDG(p) __ldg(p)
#else
#define CF_LDG(p) (*(p))
#endif

// Transform geometry: L = 2^LG entries, T threads holding E = 2^R entries each.  The LG levels
// are done in passes of R levels (the last pass may have fewer); between passes the entries go
// through shared memory.
template <int LG_, int R_>
struct Geo {
    static constexpr int LG = LG_, R = R_;
    static constexpr int L = 1 << LG, E = 1 << R, T = 1 << (LG - R);
    static constexpr int NP = (LG + R - 1) / R;  // number of passes
    static constexpr int SWZ = R > 4 ? R : 4;    // shared-memory swizzle shift
    static constexpr int HLO = (LG + 1) / 2;     // two-level power tables: x^e = hi[e >> HLO] lo[e & (LO-1)]
    static constexpr int LO = 1 << HLO, HI = (L >> HLO) + 1;
    static constexpr int GT = LO > HI ? LO : HI;  // entries per power table
    CF_HD static constexpr int pass_b(int p) { return LG - (p + 1) * R > 0 ? LG - (p + 1) * R : 0; }
    CF_HD static constexpr int pass_r(int p) { return LG - p * R - pass_b(p); }
    // index of the entry held in slot j by thread t during pass p
    CF_HD static int idx(int p, int t, int j) {
        if (p == NP - 1) return t * E + j;
        const int b = pass_b(p);
        return ((t >> b) << (b + R)) + (t & ((1 << b) - 1)) + (j << b);
    }
    CF_HD static int swz(int i) { return i ^ ((i >> SWZ) & 15); }
};

CF_HD u64 red2(u64 x, u64 m) { return x >= m ? x - m : x; }  // [0, 2m) -> [0, m)

// Per-prime global workspace, in 64-bit words (every table 256-byte aligned).
struct Layout {
    size_t V, S, fact, factq, ifact, ifactq, inv, invq, D, Dq, Kq, W, Wq, hat, hatq, ps, total;
};
CF_HD size_t lay_take(size_t& at, size_t cnt) {
    const size_t r = at;
    at += (cnt + 31) & ~(size_t)31;
    return r;
}
CF_HD Layout make_layout(int n, int F, int L, int J) {
    Layout o;
    size_t at = 0;
    o.V = lay_take(at, (size_t)n * (n + 1) / 2);  // columns w = 0..n-1, rows p = w+1..n
    o.S = lay_take(at, (size_t)n * (n - 1) / 2);  // columns q = 1..n-1, rows v = q..n-1
    o.fact = lay_take(at, (size_t)F + 1);
    o.factq = lay_take(at, (size_t)F + 1);
    o.ifact = lay_take(at, (size_t)F + 1);
    o.ifactq = lay_take(at, (size_t)F + 1);
    o.inv = lay_take(at, (size_t)F + 1);
    o.invq = lay_take(at, (size_t)F + 1);
    o.D = lay_take(at, (size_t)n + 1);
    o.Dq = lay_take(at, (size_t)n + 1);
    o.Kq = lay_take(at, (size_t)n + 1);
    o.W = lay_take(at, (size_t)L / 2 + 1);
    o.Wq = lay_take(at, (size_t)L / 2 + 1);
    o.hat = lay_take(at, (size_t)L);
    o.hatq = lay_take(at, (size_t)L);
    o.ps = lay_take(at, (size_t)J * (n + 1));
    o.total = at;
    return o;
}
CF_HD size_t colV(size_t w, size_t n) { return w * n - w * (w - 1) / 2; }        // V[p][w] at colV(w) + p-w-1
CF_HD size_t colS(size_t q, size_t n) { return (q - 1) * n - (q - 1) * q / 2; }  // S[v][q] at colS(q) + v-q

// Launch parameters shared by all CTAs of a batch (one CTA per prime).
struct KParams {
    const u64* primes;  // [B]
    int B, n, F, d, d0, model, J;
    const int* qn;      // [J] query sizes n_j <= n
    const int* qM;      // [J] query table sizes M_j <= F
    u64* ws;            // workspace base
    size_t ws_words;    // words per prime
    u64* out;           // [B][J] residues
    int* err;           // device error word (0 = ok)
};

// Error codes recorded in *err by the kernel.
enum { KERR_NONE = 0, KERR_NO_ROOT = 1, KERR_BOUNDS = 2 };

// Shared memory per CTA, in 64-bit words.
template <class G>
struct Smem {
    static constexpr int X = 0;                       // [L] transform exchange (swizzled)
    static constexpr int RED = G::L;                  // [2T + 64] reduction and scan scratch
    static constexpr int TAB = RED + 2 * G::T + 64;   // [8][GT] power tables and companions
    static constexpr int MISC = TAB + 8 * G::GT;      // [16] scalars
    static constexpr int WORDS = MISC + 16;
    static constexpr size_t BYTES = (size_t)WORDS * 8;
};

template <class G>
struct Regs {
    u64 x[G::E];
};

template <class G, class X>
struct PrimeRun {
    static constexpr int L = G::L, T = G::T, E = G::E, NP = G::NP;
    X& ex;
    const KParams& kp;
    int b;  // prime index within the batch
    u64 P, P2, one_q;  // one_q = floor(2^64 / p): Shoup companion of 1, reduces any 64-bit value to [0, 2p)
    Mod md;
    int n, F, d, d0, model, J;
    u64 *V, *S, *fact, *factq, *ifact, *ifactq, *inv, *invq, *D, *Dq, *Kq, *W, *Wq, *hat, *hatq, *ps;
    u64* sm;

    CF_HD PrimeRun(X& e, const KParams& k, int bi, u64* smem) : ex(e), kp(k), b(bi), sm(smem) {
        P = kp.primes[b];
        P2 = 2 * P;
        md = make_mod(P);
        one_q = shoup_companion(1, P);
        n = kp.n, F = kp.F, d = kp.d, d0 = kp.d0, model = kp.model, J = kp.J;
        const Layout lo = make_layout(n, F, L, J);
        u64* base = kp.ws + (size_t)b * kp.ws_words;
        V = base + lo.V, S = base + lo.S;
        fact = base + lo.fact, factq = base + lo.factq, ifact = base + lo.ifact, ifactq = base + lo.ifactq;
        inv = base + lo.inv, invq = base + lo.invq, D = base + lo.D, Dq = base + lo.Dq, Kq = base + lo.Kq;
        W = base + lo.W, Wq = base + lo.Wq, hat = base + lo.hat, hatq = base + lo.hatq, ps = base + lo.ps;
    }

    CF_HD u64 sh(u64 a, const u64* tab, const u64* tabq, int k) const {  // a * tab[k] via Shoup
        return shoup_mul(a, CF_LDG(tab + k), CF_LDG(tabq + k), md);
    }
    CF_HD u64 canon_mul(u64 a, u64 bb) const { return mont_mul(mont_mul(a, bb, md), md.r2, md); }  // a b mod p, canonical

    // ---------------------------------------------------------------------------------------
    // Transform passes.  Forward: Gentleman-Sande (natural in, bit-reversed out); inverse:
    // Cooley-Tukey with inverse roots (bit-reversed in, natural out, unscaled), the same pair of
    // transforms as fast/cuckoo_fast.cu:258-305 and include/cuckoo/ntt.hpp:97-123.  W[k] = w^k
    // for k <= L/2 (W[L/2] = -1), so w_{2h}^{-j} = -W[L/2 - j L/2h] for every j, including 0.
    // ---------------------------------------------------------------------------------------
    template <int PASS>
    CF_HD void fwd_pass(int t, u64 (&x)[E]) const {
        constexpr int bb = G::pass_b(PASS), r = G::pass_r(PASS);
        const int off = bb ? (t & ((1 << bb) - 1)) : 0;
#pragma unroll
        for (int m = r - 1; m >= 0; --m) {
            const int shift = G::LG - 1 - bb - m;
#pragma unroll
            for (int ul = 0; ul < (1 << m); ++ul) {
                const bool trivial = (bb == 0 && ul == 0);
                u64 w = 1, wq = 0;
                if (!trivial) {
                    const int k = (off + (ul << bb)) << shift;
                    w = CF_LDG(W + k), wq = CF_LDG(Wq + k);
                }
#pragma unroll
                for (int s = 0; s < (E >> r); ++s)
#pragma unroll
                    for (int uh = 0; uh < (1 << (r - 1 - m)); ++uh) {
                        const int j0 = (s << r) + (uh << (m + 1)) + ul, j1 = j0 + (1 << m);
                        const u64 a = x[j0], c = x[j1];
                        x[j0] = red2(a + c, P2);
                        const u64 dd = a - c + P2;
                        x[j1] = trivial ? red2(dd, P2) : shoup_mul(dd, w, wq, md);
                    }
            }
        }
    }
    template <int PASS>
    CF_HD void inv_pass(int t, u64 (&x)[E]) const {
        constexpr int bb = G::pass_b(PASS), r = G::pass_r(PASS);
        const int off = bb ? (t & ((1 << bb) - 1)) : 0;
#pragma unroll
        for (int m = 0; m < r; ++m) {
            const int shift = G::LG - 1 - bb - m;
#pragma unroll
            for (int ul = 0; ul < (1 << m); ++ul) {
                const bool trivial = (bb == 0 && ul == 0);
                u64 w = 1, wq = 0;
                if (!trivial) {
                    const int k = (L / 2) - ((off + (ul << bb)) << shift);
                    w = CF_LDG(W + k), wq = CF_LDG(Wq + k);
                }
#pragma unroll
                for (int s = 0; s < (E >> r); ++s)
#pragma unroll
                    for (int uh = 0; uh < (1 << (r - 1 - m)); ++uh) {
                        const int j0 = (s << r) + (uh << (m + 1)) + ul, j1 = j0 + (1 << m);
                        const u64 a = red2(x[j0], P2);
                        if (trivial) {
                            const u64 c = red2(x[j1], P2);
                            x[j0] = a + c;
                            x[j1] = a - c + P2;
                        } else {
                            const u64 c = shoup_mul(x[j1], w, wq, md);  // -w_{2h}^{-j} y
                            x[j0] = a - c + P2;
                            x[j1] = a + c;
                        }
                    }
            }
        }
    }
    template <int PASS>
    CF_HD void to_smem(int t, const u64 (&x)[E]) const {
#pragma unroll
        for (int j = 0; j < E; ++j) sm[G::swz(G::idx(PASS, t, j))] = x[j];
    }
    template <int PASS>
    CF_HD void from_smem(int t, u64 (&x)[E]) const {
#pragma unroll
        for (int j = 0; j < E; ++j) x[j] = sm[G::swz(G::idx(PASS, t, j))];
    }

    template <int PASS>
    CF_HD void fwd_chain() {  // passes PASS .. NP-1 of the forward transform (entry: data in smem, PASS >= 1)
        ex.sync();
        ex.each([&](int t, Regs<G>& rg) {
            from_smem<PASS>(t, rg.x);
            fwd_pass<PASS>(t, rg.x);
            if (PASS == NP - 1) {
                pointwise(t, rg.x);
                inv_pass<PASS>(t, rg.x);
            }
            if (PASS > 0) to_smem<PASS>(t, rg.x);
        });
        if constexpr (PASS + 1 < NP) fwd_chain<PASS + 1>();
    }
    template <int PASS>
    CF_HD void inv_chain() {  // inverse passes PASS .. 0 (entry: data in smem in layout PASS)
        ex.sync();
        ex.each([&](int t, Regs<G>& rg) {
            from_smem<PASS>(t, rg.x);
            inv_pass<PASS>(t, rg.x);
            if (PASS > 0) to_smem<PASS>(t, rg.x);
        });
        if constexpr (PASS > 0) inv_chain<PASS - 1>();
    }
    CF_HD void pointwise(int t, u64 (&x)[E]) const {
#pragma unroll
        for (int j = 0; j < E; ++j) {
            const int i = G::idx(NP - 1, t, j);
            x[j] = sh(x[j], hat, hatq, i);
        }
    }
    // Cyclic convolution of the registers (layout of pass 0) with the kernel 1/t; the result comes
    // back in the same layout, in [0, 4p).
    CF_HD void convolve() {
        if constexpr (NP == 1) {
            ex.each([&](int t, Regs<G>& rg) {
                fwd_pass<0>(t, rg.x);
                pointwise(t, rg.x);
                inv_pass<0>(t, rg.x);
            });
        } else {
            ex.each([&](int t, Regs<G>& rg) {
                fwd_pass<0>(t, rg.x);
                to_smem<0>(t, rg.x);
            });
            fwd_chain<1>();
            inv_chain<NP - 2>();
        }
    }

    // ---------------------------------------------------------------------------------------
    // Block reduction of per-thread values mod p: each thread leaves its value in RED[t].
    // ---------------------------------------------------------------------------------------
    CF_HD u64 sum_red() {
        u64* red = sm + Smem<G>::RED;
        ex.sync();
        ex.reduce_mod(red, T, P);  // leaves the total in red[0] (and in red[T] for all readers)
        ex.sync();
        const u64 s = red[T];
        return s;
    }

    // Powers x^e for 0 <= e < L through two tables: tab[0..GT) = x^(j), tab[2GT..) = x^(j LO).
    // Companions in the odd slots.  xm is x in Montgomery form.  Called by every thread.
    CF_HD void power_tables(int t, u64 xm, u64* tab) const {
        for (int k = t; k < G::LO + G::HI; k += T) {
            const bool lo = k < G::LO;
            const u64 e = lo ? (u64)k : (u64)(k - G::LO) << G::HLO;
            const u64 v = from_mont(mont_pow(xm, e, md), md);
            u64* dst = lo ? tab + k : tab + 2 * G::GT + (k - G::LO);
            dst[0] = v;
            dst[G::GT] = shoup_companion(v, P);
        }
    }
    // x^e for e < L from the tables (canonical, [0, 2p) lazily) times a
    CF_HD u64 mul_pow(u64 a, const u64* tab, int e) const {
        const int lo = e & (G::LO - 1), hi = e >> G::HLO;
        a = shoup_mul(a, tab[lo], tab[G::GT + lo], md);
        return shoup_mul(a, tab[2 * G::GT + hi], tab[3 * G::GT + hi], md);
    }

    // g(v) in Montgomery form, and 1/g(v) (g != 0 for v >= d0)
    CF_HD u64 g_mont(int v) const {
        if (model == MODEL_REPLACEMENT) return mont_pow(to_mont((u64)v, md), (u64)d, md);
        const u64 c = red2(sh(sh(CF_LDG(fact + v), ifact, ifactq, d), ifact, ifactq, v - d), P);
        return to_mont(c, md);
    }
    CF_HD u64 ginv_mont(int v) const {
        if (model == MODEL_REPLACEMENT) return mont_pow(to_mont(CF_LDG(inv + v), md), (u64)d, md);
        const u64 c = red2(sh(sh(CF_LDG(ifact + v), fact, factq, d), fact, factq, v - d), P);
        return to_mont(c, md);
    }

    // ---------------------------------------------------------------------------------------
    // Setup: factorials, inverses, D, twiddles and the kernel spectrum of 1/t (the per-batch host
    // work of fast/cuckoo_fast.cu:797-839, done on the device).
    // ---------------------------------------------------------------------------------------
    CF_HD void setup() {
        u64* red = sm + Smem<G>::RED;  // red[t]: prefix before chunk t; red[T + t]: chunk product / suffix
        u64* misc = sm + Smem<G>::MISC;
        const int C = (F + 1 + T - 1) / T;  // factorial entries k = 0..F, chunk of C per thread
        // product of the integers in each chunk (Montgomery form)
        ex.each([&](int t, Regs<G>&) {
            const int k0 = t * C > 1 ? t * C : 1, k1 = (t + 1) * C < F + 1 ? (t + 1) * C : F + 1;
            u64 pr = md.r1;
            u64 km = to_mont((u64)k0, md);
            for (int k = k0; k < k1; ++k) {
                pr = mont_mul(pr, km, md);
                km = madd(km, md.r1, P);
            }
            red[T + t] = pr;
        });
        ex.sync();
        ex.single([&]() {  // exclusive prefix products, F!, 1/F!, exclusive suffix products / F!
            u64 run = md.r1;
            for (int t = 0; t < T; ++t) {
                red[t] = run;
                run = mont_mul(run, red[T + t], md);
            }
            u64 suf = mont_pow(run, P - 2, md);  // 1/F!
            for (int t = T - 1; t >= 0; --t) {
                const u64 c = red[T + t];
                red[T + t] = suf;  // 1/F! times the product of the chunks after t = 1/(last k of chunk t)!
                suf = mont_mul(suf, c, md);
            }
        });
        ex.sync();
        ex.each([&](int t, Regs<G>&) {
            const int k0 = t * C, k1 = (t + 1) * C < F + 1 ? (t + 1) * C : F + 1;
            u64 run = red[t];  // (k0 - 1)! (Montgomery), 1 for the first chunk
            u64 km = to_mont((u64)(k0 > 0 ? k0 : 1), md);
            for (int k = k0; k < k1; ++k) {  // k! = (k-1)! k
                if (k > 0) {
                    run = mont_mul(run, km, md);
                    km = madd(km, md.r1, P);
                }
                const u64 c = from_mont(run, md);
                fact[k] = c;
                factq[k] = shoup_companion(c, P);
            }
            run = red[T + t];  // 1/(k1 - 1)!
            for (int k = k1 - 1; k >= k0; --k) {  // 1/(k-1)! = k / k!
                const u64 c = from_mont(run, md);
                ifact[k] = c;
                ifactq[k] = shoup_companion(c, P);
                if (k > 0) run = mont_mul(run, to_mont((u64)k, md), md);
            }
        });
        ex.sync();
        // inv[k] = (k-1)!/k!, D[k] = 1/k!^2, Kq[k] = companion of k
        ex.each([&](int t, Regs<G>&) {
            for (int k = t; k <= F; k += T) {
                const u64 c = k ? red2(sh(CF_LDG(ifact + k), fact, factq, k - 1), P) : 0;
                inv[k] = c;
                invq[k] = shoup_companion(c, P);
            }
            for (int k = t; k <= n; k += T) {
                const u64 ik = CF_LDG(ifact + k);
                const u64 c = red2(sh(ik, ifact, ifactq, k), P);
                D[k] = c;
                Dq[k] = shoup_companion(c, P);
                Kq[k] = shoup_companion((u64)k % P, P);
            }
            for (int q = 0; q < J; ++q)
                for (int k = t; k <= n; k += T) ps[(size_t)q * (n + 1) + k] = 0;
        });
        // a root of unity of order L: x^((p-1)/L) whose (L/2)-th power is -1 (fast/cuckoo_fast.cu:815-820)
        ex.single([&]() {
            const u64 minus1 = P - md.r1;
            u64 w = 0;
            int found = 0;
            for (u64 x = 2; x < 1000; ++x) {
                w = mont_pow(to_mont(x, md), (P - 1) / L, md);
                if (mont_pow(w, L / 2, md) == minus1) {
                    found = 1;
                    break;
                }
            }
            if (!found) ex.set_error(kp.err, KERR_NO_ROOT);
            misc[2] = w;
            misc[3] = mont_pow(to_mont((u64)L, md), P - 2, md);  // 1/L (Montgomery)
        });
        ex.sync();
        ex.each([&](int t, Regs<G>&) {
            const u64 w = misc[2];
            u64 cur = mont_pow(w, (u64)t, md);
            const u64 step = mont_pow(w, (u64)T, md);
            for (int k = t; k <= L / 2; k += T) {
                const u64 c = from_mont(cur, md);
                W[k] = c;
                Wq[k] = shoup_companion(c, P);
                cur = mont_mul(cur, step, md);
            }
        });
        ex.sync();
        // kernel spectrum: hat = DIF(ker) / L with ker[t] = 1/t for 1 <= t <= n-1 (fast/cuckoo_fast.cu:829,838-839)
        ex.each([&](int t, Regs<G>& rg) {
#pragma unroll
            for (int j = 0; j < E; ++j) {
                const int i = G::idx(0, t, j);
                rg.x[j] = (i >= 1 && i < n) ? CF_LDG(inv + i) : 0;
            }
        });
        fwd_only();
        ex.each([&](int t, Regs<G>& rg) {
            const u64 linv = from_mont(misc[3], md);
            const u64 linvq = shoup_companion(linv, P);
#pragma unroll
            for (int j = 0; j < E; ++j) {
                const int i = G::idx(NP - 1, t, j);
                const u64 c = red2(shoup_mul(rg.x[j], linv, linvq, md), P);
                hat[i] = c;
                hatq[i] = shoup_companion(c, P);
            }
        });
        ex.sync();
    }
    // forward transform only (registers in layout 0 -> registers in layout NP-1)
    template <int PASS>
    CF_HD void fwd_only_chain() {
        ex.sync();
        ex.each([&](int t, Regs<G>& rg) {
            from_smem<PASS>(t, rg.x);
            fwd_pass<PASS>(t, rg.x);
            if (PASS < NP - 1) to_smem<PASS>(t, rg.x);
        });
        if constexpr (PASS + 1 < NP) fwd_only_chain<PASS + 1>();
    }
    CF_HD void fwd_only() {
        if constexpr (NP == 1) {
            ex.each([&](int t, Regs<G>& rg) { fwd_pass<0>(t, rg.x); });
        } else {
            ex.each([&](int t, Regs<G>& rg) {
                fwd_pass<0>(t, rg.x);
                to_smem<0>(t, rg.x);
            });
            fwd_only_chain<1>();
        }
    }

    // ---------------------------------------------------------------------------------------
    // Query partial sums for row q: ps_j[q] = sum_{w<q} Vs[q][w] / (M_j - w), for every query
    // with n_j >= q (the U[w] / (M - w) sums of fast/cuckoo_fast.cu:306-323, 595-622).
    // The row must be in the registers (layout 0, entries w >= q zero).
    // ---------------------------------------------------------------------------------------
    CF_HD void query_row(int q) {
        u64* red = sm + Smem<G>::RED;
        for (int jq = 0; jq < J; ++jq) {
            const int nj = kp.qn[jq], Mj = kp.qM[jq];
            if (nj < q) continue;
            ex.each([&](int t, Regs<G>& rg) {
                u64 acc = 0;
#pragma unroll
                for (int j = 0; j < E; ++j) {
                    const int w = G::idx(0, t, j);
                    if (w < q) acc += sh(rg.x[j], inv, invq, Mj - w);  // < 2^63 for E <= 2^12
                }
                red[t] = red2(shoup_mul(acc, 1, one_q, md), P);
            });
            const u64 s = sum_red();
            ex.single([&]() { ps[(size_t)jq * (n + 1) + q] = s; });
        }
    }

    // One step of the suffix recurrence (fast/cuckoo_fast.cu:841-855).
    CF_HD void step(int v) {
        u64* tab = sm + Smem<G>::TAB;
        if (v > d0) {  // stage 1: column v of S from row v of V
            ex.each([&](int t, Regs<G>& rg) {
#pragma unroll
                for (int j = 0; j < E; ++j) {
                    const int i = G::idx(0, t, j);
                    rg.x[j] = i < v ? CF_LDG(V + colV(i, n) + (v - i - 1)) : 0;
                }
            });
            query_row(v);
            convolve();
            ex.each([&](int t, Regs<G>& rg) {
                const u64 iv = CF_LDG(inv + v), ivq = CF_LDG(invq + v);
                u64* col = S + colS(v, n);
#pragma unroll
                for (int j = 0; j < E; ++j) {
                    const int i = G::idx(0, t, j);
                    if (i >= v && i < n) col[i - v] = red2(shoup_mul(sh(rg.x[j], D, Dq, i - v), iv, ivq, md), P);
                }
            });
        }
        if (v >= d0) {  // stage 2: column v of V from row v of S
            ex.each([&](int t, Regs<G>&) {
                power_tables(t, g_mont(v), tab);                 // g^e
                power_tables(t, ginv_mont(v), tab + 4 * G::GT);  // g^-e
            });
            ex.sync();
            ex.each([&](int t, Regs<G>& rg) {
#pragma unroll
                for (int j = 0; j < E; ++j) {
                    const int i = G::idx(0, t, j);
                    rg.x[j] = (i >= 1 && i <= v) ? mul_pow(CF_LDG(S + colS(i, n) + (v - i)), tab + 4 * G::GT, i) : 0;
                }
            });
            convolve();
            ex.each([&](int t, Regs<G>& rg) {
                const u64 dv = CF_LDG(D + v);
                u64* col = V + colV(v, n);
#pragma unroll
                for (int j = 0; j < E; ++j) {
                    const int i = G::idx(0, t, j);
                    const int p = (i == 0) ? L : i;  // e[n] sits at index 0 when L = n
                    if (p > v && p <= n) {
                        const u64 pe = shoup_mul(rg.x[j], (u64)p % P, CF_LDG(Kq + p), md);
                        u64 y = sh(dv + P2 - pe, D, Dq, p - v - 1);
                        y = mul_pow(y, tab, p);
                        col[p - v - 1] = red2(y, P);
                    }
                }
            });
        }
        ex.sync();  // column v of V is read by the next step
    }

    // Horner finish (fast/cuckoo_fast.cu:877-890): N_bad = M! n! sum_k inv[k] ifact[n-k] ifact[M-k] Q^{n-k} ps[k]
    CF_HD void finish() {
        u64* tab = sm + Smem<G>::TAB;
        u64* red = sm + Smem<G>::RED;
        // the last row n for queries with n_j = n
        if (n > d0) {
            ex.each([&](int t, Regs<G>& rg) {
#pragma unroll
                for (int j = 0; j < E; ++j) {
                    const int i = G::idx(0, t, j);
                    rg.x[j] = i < n ? CF_LDG(V + colV(i, n) + (n - i - 1)) : 0;
                }
            });
            query_row(n);
        }
        for (int jq = 0; jq < J; ++jq) {
            const int nj = kp.qn[jq], Mj = kp.qM[jq];
            ex.sync();
            ex.each([&](int t, Regs<G>&) {
                u64 Qm;
                if (model == MODEL_REPLACEMENT) Qm = mont_pow(to_mont((u64)Mj, md), (u64)d, md);
                else Qm = to_mont(red2(sh(sh(CF_LDG(fact + Mj), ifact, ifactq, d), ifact, ifactq, Mj - d), P), md);
                power_tables(t, Qm, tab);
            });
            ex.sync();
            ex.each([&](int t, Regs<G>&) {
                u64 acc = 0;
                for (int k = t + 1; k <= nj; k += T) {
                    u64 y = CF_LDG(ps + (size_t)jq * (n + 1) + k);
                    y = sh(y, inv, invq, k);
                    y = sh(y, ifact, ifactq, nj - k);
                    y = sh(y, ifact, ifactq, Mj - k);
                    y = mul_pow(y, tab, nj - k);
                    acc = madd(acc, red2(y, P), P);
                }
                red[t] = acc;
            });
            const u64 s = sum_red();
            ex.single([&]() {
                const u64 r = red2(sh(red2(sh(s, fact, factq, nj), P), fact, factq, Mj), P);
                kp.out[(size_t)b * J + jq] = r;
            });
        }
    }

    CF_HD void run() {
        setup();
        for (int v = 1; v < n; ++v) step(v);
        finish();
    }
};

}  // namespace cfb
