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
//   * every multiplication by a stored constant is a Shoup product with a precomputed companion;
//     inside the transforms only the twiddle products are reduced (lazily, to [0, 4p)); the sums
//     grow within the 14 spare bits of a word under bounds tracked per level (Geo);
//   * the stage factors are folded into what is stored, so stage 1 needs no multiply on input:
//       Vs[p][w] = V[p][w] / (w! (p-1-w)! (p-1)!)        (stored V)
//       Ss[v][q] = S[v][q] / (q! (v-q)! v!)              (stored S)
//     which turns the reference's stage relations into
//       stage 1:  Ss[v'][v] = D[v'-v] inv[v] conv(Vs[v][.])[v'],            D[k] = 1/k!^2
//       stage 2:  Vs[p][v]  = g^p D[p-v-1] (D[v] - p conv(Ss[v][q] g^-q)[p])
//       query:    out(q)    = (q-1)! sum_w Vs[q][w] / (M - w)
//   * the powers g^p and g^-q of a step are running Montgomery products per thread (each thread
//     holds the entries t + k T), started from a small per-step table of powers in shared memory;
//   * the queries are evaluated on the fly from the stage-1 input rows (the same U[w] the
//     reference's k_query builds), over the row's live entries only; each warp leaves its partial
//     sum in shared memory and, after the transform's first barrier, one warp per query folds the
//     row's partials into one word, so a batch needs no separate pass over V and no barrier of its
//     own per row.
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

// Scheduling controls for the hot loops.  Constant tables are interleaved (value, companion)
// pairs fetched with one 16-byte load.  `ld_pair` is a volatile load and `pin` an empty volatile
// statement that consumes a result: a load placed after a pin cannot be hoisted above the work
// that produced the pinned value, which bounds how many constants are in flight (registers).
//
// L2 policy: the per-prime constant tables are re-read every step and are loaded with an
// evict-last hint; the rows and column tiles of V and S stream through once per step and use
// evict-first, so they do not push the tables out of L2.  V, S and the tiles are written by the
// kernel itself, so they are read with plain coherent loads, never through the read-only path.
#if defined(__CUDA_ARCH__)
CF_HD void pin(u64& v) { asm volatile("" : "+l"(v)); }
CF_HD void pin_int(int& v) { asm volatile("" : "+r"(v)); }
CF_HD u64 policy_keep() {
    u64 pol;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
CF_HD u64 policy_stream() {
    u64 pol;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
CF_HD void ld_pair(const u64* p, u64& a, u64& b) {
    asm volatile("ld.global.nc.L2::cache_hint.v2.u64 {%0, %1}, [%2], %3;" : "=l"(a), "=l"(b) : "l"(p), "l"(policy_keep()));
}
CF_HD u64 ld_stream(const u64* p) {
    u64 v;
    asm volatile("ld.global.L2::cache_hint.u64 %0, [%1], %2;" : "=l"(v) : "l"(p), "l"(policy_stream()));
    return v;
}
CF_HD void st_stream(u64* p, u64 v) { asm volatile("st.global.L2::cache_hint.u64 [%0], %1, %2;" ::"l"(p), "l"(v), "l"(policy_stream())); }
// one full 32-byte sector (p 32-byte aligned)
CF_HD void st_stream4(u64* p, u64 a, u64 b, u64 c, u64 d) {
    asm volatile("st.global.L2::cache_hint.v4.u64 [%0], {%1, %2, %3, %4}, %5;" ::"l"(p), "l"(a), "l"(b), "l"(c), "l"(d),
                 "l"(policy_stream()));
}
CF_HD void ld_pair_shared(const u64* p, u64& a, u64& b) {
    asm volatile("ld.shared.v2.u64 {%0, %1}, [%2];" : "=l"(a), "=l"(b) : "r"((u32)__cvta_generic_to_shared(p)));
}
#else
CF_HD u64 ld_stream(const u64* p) { return *p; }
CF_HD void st_stream(u64* p, u64 v) { *p = v; }
CF_HD void st_stream4(u64* p, u64 a, u64 b, u64 c, u64 d) { p[0] = a, p[1] = b, p[2] = c, p[3] = d; }
CF_HD void ld_pair_shared(const u64* p, u64& a, u64& b) { a = p[0], b = p[1]; }
CF_HD void pin(u64&) {}
CF_HD void pin_int(int&) {}
CF_HD void ld_pair(const u64* p, u64& a, u64& b) { a = p[0], b = p[1]; }
#endif
// Loads of data a kernel writes itself.  A CTA alone reads its own writes through L1 and the
// read-only path.  In a cluster (CG), data another CTA wrote in this launch is read from L2 (.cg),
// where the writer's release at the cluster barrier has made it visible; L1 lines of an earlier
// read (block cells and tiles are reused) and the read-only path would not see the new values.
template <bool CG>
CF_HD void ldp(const u64* p, u64& a, u64& b) {
#if defined(__CUDA_ARCH__)
    if constexpr (CG)
        asm volatile("ld.global.cg.L2::cache_hint.v2.u64 {%0, %1}, [%2], %3;" : "=l"(a), "=l"(b) : "l"(p), "l"(policy_keep()));
    else ld_pair(p, a, b);
#else
    a = p[0], b = p[1];
#endif
}
template <bool CG>
CF_HD u64 lds(const u64* p) {
#if defined(__CUDA_ARCH__)
    if constexpr (CG) {
        u64 v;
        asm volatile("ld.global.cg.L2::cache_hint.u64 %0, [%1], %2;" : "=l"(v) : "l"(p), "l"(policy_stream()));
        return v;
    } else return ld_stream(p);
#else
    return *p;
#endif
}
template <bool CG>
CF_HD u64 ldc(const u64* p) {
#if defined(__CUDA_ARCH__)
    if constexpr (CG) {
        u64 v;
        asm volatile("ld.global.cg.u64 %0, [%1];" : "=l"(v) : "l"(p));
        return v;
    } else return CF_LDG(p);
#else
    return *p;
#endif
}
// Lambdas that index the register array must be inlined, or the array goes to local memory.
#define CF_INL __attribute__((always_inline))
// Compile-time slot index handed to the bodies below (so register-array indices are constants).
template <int V>
struct IC {
    static constexpr int value = V;
    CF_HD constexpr operator int() const { return V; }
};
// Unrolled loop over N units with a bounded window: body(IC<J>) pins its inputs and computes unit
// J; done(IC<J>) pins unit J's outputs and is issued right after body(IC<J + K>).  Since volatile
// statements keep their order, unit J + K + 1 cannot start before unit J has finished: at most
// K + 1 units are in flight, which bounds the registers the compiler's interleaving may use.
template <int N, int K, int J, class B, class Dn>
CF_HD void window_step(B& body, Dn& done) {
    if constexpr (J < N + K) {
        if constexpr (J < N) body(IC<J>{});
        if constexpr (J >= K && J - K < N) done(IC<J - K>{});
        window_step<N, K, J + 1>(body, done);
    }
}
template <int N, int K, class B, class Dn>
CF_HD void window(B&& body, Dn&& done) {
    window_step<N, K, 0>(body, done);
}
// Per-slot constant pairs over a window: slot J's pair addr(IC<J>) is loaded D slots ahead.
template <int N, int D, int K, bool CG = false, class A, class F, class Dn>
CF_HD void pipe_pairs(A&& addr, F&& apply, Dn&& done) {
    u64 ra[D + 1], rb[D + 1];
    window<D, 0>([&](auto jc) CF_INL {
        constexpr int j = decltype(jc)::value;
        if constexpr (j < N) ldp<CG>(addr(jc), ra[j], rb[j]);
    }, [&](auto) CF_INL {});
    window<N, K>(
        [&](auto jc) CF_INL {
            constexpr int j = decltype(jc)::value;
            if constexpr (j + D < N) ldp<CG>(addr(IC<j + D>{}), ra[(j + D) % (D + 1)], rb[(j + D) % (D + 1)]);
            apply(jc, ra[j % (D + 1)], rb[j % (D + 1)]);
        },
        done);
}
// The same over the slots for which live(IC<J>) holds (a warp-uniform test): the others issue
// neither their constant load nor their unit.
template <int N, int D, int K, bool CG = false, class Lv, class A, class F, class Dn>
CF_HD void pipe_pairs_live(Lv&& live, A&& addr, F&& apply, Dn&& done) {
    u64 ra[D + 1] = {}, rb[D + 1] = {};
    window<D, 0>([&](auto jc) CF_INL {
        constexpr int j = decltype(jc)::value;
        if constexpr (j < N)
            if (live(jc)) ldp<CG>(addr(jc), ra[j], rb[j]);
    }, [&](auto) CF_INL {});
    window<N, K>(
        [&](auto jc) CF_INL {
            constexpr int j = decltype(jc)::value;
            if constexpr (j + D < N)
                if (live(IC<j + D>{})) ldp<CG>(addr(IC<j + D>{}), ra[(j + D) % (D + 1)], rb[(j + D) % (D + 1)]);
            if (live(jc)) apply(jc, ra[j % (D + 1)], rb[j % (D + 1)]);
        },
        done);
}
#ifndef CF_PIPE_D
#define CF_PIPE_D 4
#endif
#ifndef CF_WIN_K
#define CF_WIN_K 3
#endif
constexpr int PIPE_D = CF_PIPE_D;  // constants loaded ahead
constexpr int WIN_K = CF_WIN_K;    // units in flight beyond the current one

// Transform geometry: L = 2^LG entries, T threads holding E = 2^R entries each.  The LG levels
// are done in passes of R levels (the last pass may have fewer); between passes the entries go
// through shared memory.
//
// Clusters (LC > 0): the T threads are spread over C = 2^LC CTAs of CT = T / C threads, thread t
// being thread t % CT of the cluster's CTA t / CT.  Pass 0 holds index t + jT in slot j (a
// column of every one of the E blocks of L / E entries); after it every later pass works inside one
// block, and CTA c holds blocks c E / C .. (c + 1) E / C - 1 (E >= C), i.e. the indices
// [c L / C, (c + 1) L / C).  So the entries cross between CTAs only after the first forward pass
// and before the last inverse pass, through distributed shared memory.
template <int LG_, int R_, int LC_ = 0>
struct Geo {
    static constexpr int LG = LG_, R = R_, LC = LC_;
    static constexpr int L = 1 << LG, E = 1 << R, T = 1 << (LG - R);
    static constexpr int C = 1 << LC, CT = T >> LC, LCN = L >> LC;  // CTAs, threads and entries per CTA
    static constexpr int NP = (LG + R - 1) / R;  // number of passes
    static constexpr int SWZ = R > 4 ? R : 4;    // shared-memory swizzle shift
    static constexpr int NW = (CT + 31) / 32;    // warps per CTA
    static_assert(C == 1 || (E >= C && CT % 128 == 0 && NP >= 3), "a cluster needs E >= C, whole warp quarters and 3 passes");
    // Forward transform for primes below 2^50 (reduction-free, bounds below): up to 2^14 entries the
    // sums grow through every level; above, pass 0's outputs are reduced lazily to [0, 4p) (at the
    // exchange between CTAs) and the later levels grow from there.  flvl(s): the s' with level s's
    // inputs below 2^s' p.
    static constexpr int FRED = LG > 14 ? R : 0;
    CF_HD static constexpr int flvl(int s) { return FRED && s >= FRED ? s - FRED + 2 : s; }
    static_assert(LG <= 14 || LG - FRED + 2 <= 14, "forward bounds need 2^14 p < 2^64");
    CF_HD static constexpr int pass_b(int p) { return LG - (p + 1) * R > 0 ? LG - (p + 1) * R : 0; }
    CF_HD static constexpr int pass_r(int p) { return LG - p * R - pass_b(p); }
    // index of the entry held in slot j by thread t during pass p
    CF_HD static int idx(int p, int t, int j) {
        if (p == NP - 1) return t * E + j;
        const int b = pass_b(p);
        return ((t >> b) << (b + R)) + (t & ((1 << b) - 1)) + (j << b);
    }
    CF_HD static int swz(int i) { return i ^ ((i >> SWZ) & 15); }
    // Value bounds of the transforms for primes below 2^50 (multiples of p, strict upper bounds),
    // by level s in processing order.  Forward: canonical inputs, no reduction of sums, so the
    // inputs of level s lie below 2^s p (2^LG p < 2^64 needs LG <= 14).  Inverse: inputs below 4p;
    // a butterfly with a twiddle adds a product below 4p, a trivial one (first pass, twiddle 1)
    // doubles, so no reduction is needed either.
    static constexpr int R_LAST = LG - (NP - 1) * R;  // levels of the last pass (the trivial groups)
    CF_HD static constexpr u64 inv_bound(int s) {
        return s <= R_LAST ? (u64)4 << s : ((u64)4 << R_LAST) + 4 * (u64)(s - R_LAST);
    }
    static constexpr u64 INV_OUT = inv_bound(LG);  // bound of the inverse transform's outputs
    // Bound (multiple of p) of the stage-2 product p e[p] with the companion p floor(2^64 / p): the
    // quotient estimate loses at most p x / 2^64 < INV_OUT 2^(LG - 14) more for p <= L, P < 2^50.
    static constexpr u64 PE_B = LG <= 14 ? INV_OUT + 4 : (INV_OUT << (LG - 14)) + 5;
};

CF_HD u64 red2(u64 x, u64 m) { return x >= m ? x - m : x; }  // [0, 2m) -> [0, m)

// V and S are read by rows (a step reads row v) but produced by columns (step v writes column v).
// The columns of the current TILE steps are staged column-major in VS / SS (contiguous writes) and
// moved into row storage every TILE steps, the scheme of fast/cuckoo_fast.cu:133-144, 227-243.
//
// Row storage is made of TILE x TILE blocks: block (P, W) holds rows 1 + 16P .. 16 + 16P and
// columns 1 + 16W .. 16 + 16W, row-major (a row's 16 entries are one 128-byte line).  Only blocks
// below the diagonal (W < P) are stored; a row's own group of columns is read from the staging
// tile.  Block (P, W) is written when tile W is flushed and dead once the steps of tile P have read
// its rows (row n of V stays until the finish), so at most (k + 1)(G - 1 - k) blocks are live
// after flush k, G = number of row groups.  The blocks map onto an (G - h) x h array of cells,
// h = ceil(G / 2), that is exactly that peak:
//   W < h <= P : cell (P - h, W)          the rectangle, live through the middle of the run
//   P < h      : cell (W, P)              rows read before step 16h; their cell's rectangle block
//                                        is written at flush P, after its last read
//   h <= W     : cell (W - h, P - h - 1)  written from flush h on, into cells whose rectangle
//                                        block was read in tile W, before that flush
// so a prime's V and S take about n^2 / 4 words each instead of n^2 / 2 for packed triangles.
constexpr int TILE = 16;
CF_HD int grp(int x) { return (x - 1) >> 4; }  // row / column group of index x >= 1
CF_HD int block_h(int n) { return (((n - 1) >> 4) + 2) >> 1; }  // h = ceil(G / 2), G = grp(n) + 1
CF_HD size_t block_count(int n) {
    if (n < 1) return 0;
    const size_t G = (size_t)grp(n) + 1, h = (size_t)block_h(n);
    return (G - h) * h;
}
CF_HD size_t block_cell(int P, int W, int h) {  // W < P
    if (P < h) return (size_t)W * h + P;
    if (W < h) return (size_t)(P - h) * h + W;
    return (size_t)(W - h) * h + (P - h - 1);
}
// word offset of entry (row r, column c), grp(c) < grp(r), inside a block pool
CF_HD size_t blk_off(int r, int c, int h) {
    return (block_cell(grp(r), grp(c), h) << 8) + ((size_t)((r - 1) & 15) << 4) + (size_t)((c - 1) & 15);
}

// Per-prime global workspace, in 64-bit words (every table 256-byte aligned).
// Tables marked "pairs" hold (value, Shoup companion) interleaved: entry k at [2k], [2k+1].
struct Layout {
    size_t V, S, VS, SS, fact, ifact, inv, D, Gm, hat, ps, total;
    size_t WL[8];  // pass-0 twiddles by level: WL[s] holds pairs w^(u 2^s), u = 0 .. L/2^(s+1)
};
CF_HD size_t lay_take(size_t& at, size_t cnt) {
    const size_t r = at;
    at += (cnt + 31) & ~(size_t)31;
    return r;
}
// nw = warps per CTA: query partial sums are kept per warp.  C: CTAs per prime (each keeps its own
// row sums of the queries).
CF_HD Layout make_layout(int n, int F, int L, int J, int nw, int R, int C = 1) {
    Layout o;
    size_t at = 0;
    o.V = lay_take(at, block_count(n) << 8);         // rows p = 1..n, entries w = 1..p-1 (blocks)
    o.S = lay_take(at, block_count(n) << 8);         // rows v = 1..n-1, entries q = 1..v (blocks)
    o.VS = lay_take(at, (size_t)TILE * (n + 1));      // column tiles, [column - v0][row]
    o.SS = lay_take(at, (size_t)TILE * (n + 1));
    o.fact = lay_take(at, 2 * ((size_t)F + 1));   // pairs: k!
    o.ifact = lay_take(at, 2 * ((size_t)F + 1));  // pairs: 1/k!
    o.inv = lay_take(at, 2 * ((size_t)F + 1));    // pairs: 1/k
    o.D = lay_take(at, 2 * ((size_t)n + 1));      // pairs: 1/k!^2
    o.Gm = lay_take(at, 2 * ((size_t)n + 1));     // (g(v), 1/g(v)) in Montgomery form, v = 0 .. n
    for (int l = 0; l < 8; ++l) o.WL[l] = l < R ? lay_take(at, 2 * (((size_t)L >> (l + 1)) + 1)) : 0;  // pairs
    o.hat = lay_take(at, 2 * (size_t)L);          // pairs: spectrum of the kernel 1/t, times 1/L
    o.ps = lay_take(at, (size_t)C * J * (n + 1));  // [C][J][n+1] row sums per query (per CTA of the prime)
    (void)nw;
    o.total = at;
    return o;
}
CF_HD int tile_v0(int v) { return 1 + TILE * ((v - 1) / TILE); }  // first column of v's tile

// Resident tables (serving): per prime, the whole V as a packed triangle (row p at p(p-1)/2,
// entries w = 0..p-1, entries w < d0 unused) and the pair tables fact, ifact, inv up to F, so that
// later queries (n' <= n, M' <= F) need no rebuild.
struct KeepLayout {
    size_t tri, fact, ifact, inv, total;
};
CF_HD KeepLayout make_keep_layout(int n, int F) {
    KeepLayout k;
    size_t at = 0;
    k.tri = lay_take(at, (size_t)n * (n + 1) / 2);
    k.fact = lay_take(at, 2 * ((size_t)F + 1));
    k.ifact = lay_take(at, 2 * ((size_t)F + 1));
    k.inv = lay_take(at, 2 * ((size_t)F + 1));
    k.total = at;
    return k;
}
CF_HD size_t tri_off(size_t p) { return p * (p - 1) / 2; }  // V[p][w] at tri + tri_off(p) + w

// Launch parameters shared by all CTAs of a batch (one CTA per prime).
struct KParams {
    const u64* primes;  // [B]
    int B, n, F, d, d0, model, J;
    const int* qn;      // [J] query sizes n_j <= n
    const int* qM;      // [J] query table sizes M_j <= F
    u64* ws;            // workspace base
    size_t ws_words;    // words per prime
    Layout lay;         // offsets inside a prime's workspace
    u64* out;           // [B][J] residues, or out[qout[j]] when qout is set
    int* err;           // device error word (0 = ok)
    const long long* qout = nullptr;  // [J] output index of each query (work-queue items), or null
    u64* keep = nullptr;  // resident tables [B][keep_words] (serving builds), or null
    size_t keep_words = 0;
};

// Error codes recorded in *err by the kernel.
enum { KERR_NONE = 0, KERR_NO_ROOT = 1 };

// Shared memory per CTA, in 64-bit words.
template <class G>
struct Smem {
    // [L] transform exchange by index (swizzled); a CTA of a cluster holds the LCN indices of its
    // blocks there (by index - c LCN) and, at X0, pass 0's column layout: slot j of thread t at
    // X0 + t % CT + j CT, written by the CTAs that finish the inverse transform's upper levels
    static constexpr int X = 0;
    static constexpr int X0 = G::C > 1 ? G::LCN : 0;
    static constexpr int RED = G::C > 1 ? 2 * G::LCN : G::L;  // [2 CT + 64] reduction and scan scratch
    static constexpr int MISC = RED + 2 * G::CT + 64;        // [16] modulus constants and scalars
    static constexpr int TWS = MISC + 16;             // pairs w^(k 2^R), k = 0 .. L/2^(R+1): passes >= 1
    static constexpr int TWS_N = (G::L >> (G::R + 1)) + 1;
    // [2][PW_STRIDE] powers of 1/g(v) and g(v) for stage 2, rebuilt every step (power_tables)
    static constexpr int PW = TWS + 2 * TWS_N;
    static constexpr int PW_STRIDE = 104;
    static constexpr int WORDS = PW + 2 * PW_STRIDE;
    // A cluster's CTAs take more than half an SM's shared memory, so no two share an SM (a CTA
    // waiting for tensor memory held by another CTA of its own cluster would never get it).
    static constexpr size_t BYTES = G::C > 1 && WORDS * 8 < 120 * 1024 ? 120 * 1024 : (size_t)WORDS * 8;
    // [J][NW] per-warp query partial sums of the current row, after the fixed part (the launch's
    // dynamic shared memory is BYTES + 8 J NW)
    static constexpr int QS = WORDS;
    static constexpr size_t bytes_for(int J) { return BYTES + (size_t)8 * J * G::NW; }
};
enum { MI_P = 0, MI_PINV = 1, MI_R1 = 2, MI_R2 = 3, MI_ONEQ = 4, MI_ROOT = 5, MI_LINV = 6, MI_TMEM = 7, MI_R1Q = 8 };
// Slots of a power table (power_tables): h^k at PW_A + k (k < TA), h^(TA k) at PW_B + k (k < TB),
// h^(T j) at PW_J + j (j < E), the chains' step h^(NCH T) as a plain residue and its Shoup companion
// at PW_STEP, PW_STEPQ, and h^L at PW_L.
enum { PW_A = 0, PW_B = 32, PW_J = 64, PW_STEP = 96, PW_STEPQ = 97, PW_L = 98 };

template <class G>
struct Regs {
    u64 x[G::E];
};

// W = false: primes below 2^50 (the fixed list of fast/cuckoo_fast.cu with FP_RB = 52); the
// transforms reduce only their twiddle products (bounds per level in Geo).
// W = true: primes below 2^62 (the list of the FP_RB = 64 build); with 8p beyond 2^64 every
// transform value stays in [0, 2p) instead (one more conditional subtraction per output), and the
// few products whose lazy factor could reach 2^62 take a canonical one.
template <class G, class X, bool W = false>
struct PrimeRun {
    static constexpr int L = G::L, T = G::T, E = G::E, NP = G::NP, NW = G::NW;
    static constexpr int C = G::C, CT = G::CT, LCN = G::LCN;  // a cluster of C CTAs of CT threads per prime
    static constexpr bool CG = C > 1;  // loads of what other CTAs wrote go to L2 (ldp / lds / ldc)
    static_assert(W || G::LG <= 14 || G::FRED, "reduction-free forward transform needs 2^LG p < 2^64");
    static_assert(NP > 1, "layout 0 must hold index t + jT in slot j of thread t");
    // L = 2^14 (1024 threads x 16 entries): the kernel spectrum lives in tensor memory, each
    // thread's 16 (value, companion) pairs in its own 64 columns (all 512 columns of the SM's 128
    // lanes); smaller transforms, several CTAs to an SM, read it from global.  A cluster's CTAs
    // (one per SM) keep their blocks' part of it in 4 E CT / 128 columns.
    static constexpr bool TM = (T == 1024 && E == 16) || (T == 512 && E == 32) || (C > 1 && 4 * E * (CT / 128) <= 512);
    // Constants in flight and units in flight of the hot loops.  At 1024 threads (64 registers each)
    // the shallowest schedule spills least and measured fastest (49.7 vs 48.9 prime-residues/s).
    static constexpr int PD = CT >= 1024 ? 1 : PIPE_D, WK = CT >= 1024 ? 1 : WIN_K;
    X& ex;
    const KParams& kp;
    int b;      // prime index within the batch
    u64* base;  // this prime's workspace
    u64* sm;    // shared memory
    u64 P;
    int rank_;  // this CTA's rank in its cluster

    // bi: the prime's index in kp.primes (and its output row); slot: its workspace slot (bi if < 0)
    CF_HD PrimeRun(X& e, const KParams& k, int bi, u64* smem, int slot = -1) : ex(e), kp(k), b(bi), sm(smem) {
        P = kp.primes[b];
        base = kp.ws + (size_t)(slot < 0 ? bi : slot) * kp.ws_words;
        rank_ = ex.rank();
    }
    CF_HD int rank() const {
        if constexpr (C == 1) return 0;
        else return rank_;
    }
    CF_HD static int lt(int t) {  // thread index within the CTA
        if constexpr (C == 1) return t;
        else return t & (CT - 1);
    }
    CF_HD void csync() {  // barrier of the whole cluster (of the CTA alone when C = 1)
        if constexpr (C == 1) ex.sync();
        else ex.cluster_sync();
    }
    // workspace tables (offsets live in the kernel parameters, so these hold no registers)
    CF_HD u64* V() const { return base + kp.lay.V; }
    CF_HD u64* S() const { return base + kp.lay.S; }
    CF_HD u64* VS() const { return base + kp.lay.VS; }
    CF_HD u64* SS() const { return base + kp.lay.SS; }
    CF_HD u64* fact() const { return base + kp.lay.fact; }
    CF_HD u64* ifact() const { return base + kp.lay.ifact; }
    CF_HD u64* inv() const { return base + kp.lay.inv; }
    CF_HD u64* D() const { return base + kp.lay.D; }
    CF_HD u64* Gm() const { return base + kp.lay.Gm; }
    CF_HD u64* WL(int l) const { return base + kp.lay.WL[l]; }
    CF_HD u64* tws() const { return sm + Smem<G>::TWS; }
    CF_HD u64* hat() const { return base + kp.lay.hat; }
    CF_HD u64* ps() const { return ps_of(rank()); }
    CF_HD u64* ps_of(int c) const { return base + kp.lay.ps + (size_t)c * kp.J * (kp.n + 1); }  // CTA c's row sums
    CF_HD u64* misc() const { return sm + Smem<G>::MISC; }
    CF_HD Mod md() const {  // modulus constants, kept in shared memory
        const u64* m = misc();
        Mod r;
        r.p = m[MI_P], r.pinv = m[MI_PINV], r.r1 = m[MI_R1], r.r2 = m[MI_R2];
        return r;
    }

    CF_HD u64 sh(u64 a, const u64* pairs, int k) const {  // a * pairs[k], result in [0, 4p)
        return shoup_mul_lazy(a, ldc<CG>(pairs + 2 * k), ldc<CG>(pairs + 2 * k + 1), P);
    }
    // Shoup companion of w < p, from the per-prime constants setup keeps in shared memory
    CF_HD u64 companion(u64 w) const { return shoup_companion_fast(w, P, misc()[MI_ONEQ], misc()[MI_R1], misc()[MI_R1Q]); }
    CF_HD void put_pair(u64* pairs, int k, u64 v) const {
        pairs[2 * k] = v;
        pairs[2 * k + 1] = companion(v);
    }
    CF_HD u64 canon(u64 x) const { return red2(red2(x, 2 * P), P); }  // [0, 4p) -> [0, p)

    // ---------------------------------------------------------------------------------------
    // Transform passes.  Forward: Gentleman-Sande (natural in, bit-reversed out); inverse:
    // Cooley-Tukey with inverse roots (bit-reversed in, natural out, unscaled), the same pair of
    // transforms as fast/cuckoo_fast.cu:258-305 and include/cuckoo/ntt.hpp:97-123.  W[k] = w^k
    // for k <= L/2 (W[L/2] = -1), so w_{2h}^{-j} = -W[L/2 - j L/2h] for every j, including 0.
    // Primes below 2^50: the transforms reduce nothing but the twiddle products (bounds in Geo);
    // primes below 2^62: every value stays in [0, 2p).
    // ---------------------------------------------------------------------------------------
    // Host builds with CF_CHECK_BOUNDS (the CPU harness) verify every bound the transforms rely on.
    CF_HD void check_bound(u64 x, u64 mult) const {
#if defined(CF_CHECK_BOUNDS) && !defined(__CUDA_ARCH__)
        if (x >= mult * P) throw std::runtime_error("transform value above its bound");
#else
        (void)x, (void)mult;
#endif
    }
    // Butterfly schedule of one register pass.  Unit q runs in order of level (forward: m = r-1
    // down to 0; inverse: 0 up), then twiddle group (ul), then register pair; grp(q) numbers the
    // twiddle groups in that order.
    template <int PASS, bool FWD>
    struct Plan {
        static constexpr int bb = G::pass_b(PASS), r = G::pass_r(PASS);
        static constexpr int BPL = E / 2, NB = BPL * r, NG = (1 << r) - 1;
        // levels done before this pass, in processing order (forward: passes 0 ..; inverse: NP-1 ..)
        static constexpr int s0 = FWD ? PASS * G::R : (PASS == NP - 1 ? 0 : G::R_LAST + (NP - 2 - PASS) * G::R);
        CF_HD static constexpr int lvl(int q) { return s0 + q / BPL; }
        CF_HD static constexpr int m(int q) { return FWD ? r - 1 - q / BPL : q / BPL; }
        CF_HD static constexpr int per(int q) { return E >> (m(q) + 1); }  // butterflies per group
        CF_HD static constexpr int ul(int q) { return (q % BPL) / per(q); }
        CF_HD static constexpr int kk(int q) { return (q % BPL) % per(q); }
        CF_HD static constexpr int grp(int q) { return FWD ? (1 << r) - (1 << (m(q) + 1)) + ul(q) : (1 << m(q)) - 1 + ul(q); }
        CF_HD static constexpr int j0(int q) {
            return ((kk(q) >> (r - 1 - m(q))) << r) + ((kk(q) & ((1 << (r - 1 - m(q))) - 1)) << (m(q) + 1)) + ul(q);
        }
        CF_HD static constexpr int j1(int q) { return j0(q) + (1 << m(q)); }
        // level and group-within-level of twiddle group f
        CF_HD static constexpr int gm(int f) {
            int mm = FWD ? r - 1 : 0;
            while (f >= (1 << mm)) f -= (1 << mm), mm += FWD ? -1 : 1;
            return mm;
        }
        CF_HD static constexpr int gul(int f) {
            int mm = FWD ? r - 1 : 0;
            while (f >= (1 << mm)) f -= (1 << mm), mm += FWD ? -1 : 1;
            return f;
        }
        CF_HD static constexpr bool trivial_grp(int f) { return bb == 0 && gul(f) == 0; }
    };
    // pair address of the twiddle of group F (forward: w_{2h}^j; inverse: W[L/2 - j L/2h], whose
    // negation is w_{2h}^{-j})
    // Pass 0 reads its level's table in global memory (a warp's lanes take consecutive pairs);
    // later passes only need multiples of 2^R, kept in shared memory.
    template <int PASS, bool FWD, int F>
    CF_HD const u64* tw_addr(int off) const {
        typedef Plan<PASS, FWD> PL;
        constexpr int mm = PL::gm(F), ul = PL::gul(F), sh = G::LG - 1 - PL::bb - mm;
        const int u = off + (ul << PL::bb);  // twiddle w^(u 2^sh)
        if constexpr (PASS == 0) return WL(sh) + 2 * (FWD ? u : (L >> (sh + 1)) - u);
        else return tws() + 2 * ((FWD ? u << sh : L / 2 - (u << sh)) >> G::R);
    }
    template <int PASS>
    CF_HD static void ld_tw(const u64* p, u64& a, u64& b) {
        if constexpr (PASS == 0) ldp<CG>(p, a, b);
        else ld_pair_shared(p, a, b);
    }
    template <int PASS, bool FWD>
    CF_HD void pass(int t, u64 (&x)[E]) const {
        typedef Plan<PASS, FWD> PL;
        // pass 0 reads its twiddles from L2 (the others from shared memory): at 1024 threads it
        // prefetches them two groups ahead (72.1 against 70.3 prime-residues/s at n = 16384)
        constexpr int D = (PASS == 0 && T >= 1024) ? 2 : PD;
        const int off = PL::bb ? (t & ((1 << PL::bb) - 1)) : 0;
        const u64 P4 = 4 * P, P2 = 2 * P;
        u64 rw[D + 1], rq[D + 1];
        window<D, 0>([&](auto fc) CF_INL {
            constexpr int f = decltype(fc)::value;
            if constexpr (f < PL::NG && !PL::trivial_grp(f)) ld_tw<PASS>(tw_addr<PASS, FWD, f>(off), rw[f], rq[f]);
        }, [&](auto) CF_INL {});
        window<PL::NB, WK>(
            [&](auto qc) CF_INL {
                constexpr int q = decltype(qc)::value, f = PL::grp(q), fn = f + D;
                if constexpr (PL::kk(q) == 0 && fn < PL::NG && !PL::trivial_grp(fn))
                    ld_tw<PASS>(tw_addr<PASS, FWD, fn>(off), rw[fn % (D + 1)], rq[fn % (D + 1)]);
                constexpr int j0 = PL::j0(q), j1 = PL::j1(q);
                constexpr bool trivial = PL::trivial_grp(f);
                pin(x[j0]);
                pin(x[j1]);
                const u64 w = rw[f % (D + 1)], wq = rq[f % (D + 1)];
                if constexpr (FWD && W) {  // inputs and outputs in [0, 2p)
                    const u64 a = x[j0], c = x[j1];
                    x[j0] = red2(a + c, P2);
                    const u64 dd = a - c + P2;
                    x[j1] = red2(trivial ? dd : shoup_mul_lazy(dd, w, wq, P), P2);
                } else if constexpr (W) {
                    const u64 a = x[j0];
                    if constexpr (trivial) {
                        const u64 c = x[j1];
                        x[j0] = red2(a + c, P2);
                        x[j1] = red2(a - c + P2, P2);
                    } else {
                        const u64 c = red2(shoup_mul_lazy(x[j1], w, wq, P), P2);  // -w_{2h}^{-j} y
                        x[j0] = red2(a - c + P2, P2);
                        x[j1] = red2(a + c, P2);
                    }
                } else if constexpr (FWD) {  // inputs below 2^s p, outputs below 2^(s+1) p
                    constexpr int s = G::flvl(PL::lvl(q));
                    const u64 a = x[j0], c = x[j1];
                    x[j0] = a + c;
                    const u64 dd = a - c + (P << s);
                    if constexpr (trivial) x[j1] = dd;
                    else if constexpr (s == 0) x[j1] = red2(shoup_mul_lazy(dd, w, wq, P), P2);
                    else x[j1] = shoup_mul_lazy(dd, w, wq, P);
                    check_bound(x[j0], (u64)2 << s), check_bound(x[j1], (u64)2 << s);
                } else {  // inputs below inv_bound(s) p
                    constexpr int s = PL::lvl(q);
                    const u64 a = x[j0];
                    if constexpr (trivial) {
                        const u64 c = x[j1];
                        x[j0] = a + c;
                        x[j1] = a - c + P * G::inv_bound(s);
                    } else {
                        const u64 c = shoup_mul_lazy(x[j1], w, wq, P);  // -w_{2h}^{-j} y
                        x[j0] = a - c + P4;
                        x[j1] = a + c;
                    }
                    check_bound(x[j0], G::inv_bound(s + 1)), check_bound(x[j1], G::inv_bound(s + 1));
                }
            },
            [&](auto qc) CF_INL {
                constexpr int q = decltype(qc)::value;
                pin(x[PL::j0(q)]);
                pin(x[PL::j1(q)]);
            });
    }
    template <int PASS>
    CF_HD void fwd_pass(int t, u64 (&x)[E]) const { pass<PASS, true>(t, x); }
    template <int PASS>
    CF_HD void inv_pass(int t, u64 (&x)[E]) const { pass<PASS, false>(t, x); }
    // Entries to shared memory by index.  In a cluster, pass 0's outputs (forward) go to the CTA
    // whose block holds them, reduced to [0, 4p) when the forward bounds need it (Geo::FRED), and
    // with TO_L0 the inverse transform's pass-1 outputs go to the CTA that holds them in pass 0.
    template <int PASS, bool TO_L0 = false>
    CF_HD void to_smem(int t, u64 (&x)[E]) const {
        pin_int(t);  // recompute the addresses rather than keep the loads' 32 addresses live across the pass
        if constexpr (C > 1 && PASS == 0) {
#pragma unroll
            for (int j = 0; j < E; ++j) {
                const int i = G::idx(0, t, j);
                const u64 v = (G::FRED && !W) ? shoup_mul_lazy(x[j], 1, misc()[MI_ONEQ], P) : x[j];
                ex.st_remote(sm + G::swz(i & (LCN - 1)), i / LCN, v);
            }
        } else if constexpr (C > 1 && TO_L0) {
#pragma unroll
            for (int j = 0; j < E; ++j) {
                const int i = G::idx(PASS, t, j);
                ex.st_remote(sm + Smem<G>::X0 + (i & (CT - 1)) + (i / T) * CT, (i & (T - 1)) / CT, x[j]);
            }
        } else {
#pragma unroll
            for (int j = 0; j < E; ++j) {
                const int i = G::idx(PASS, t, j);
                if constexpr (G::FRED && !W && PASS == 0) x[j] = shoup_mul_lazy(x[j], 1, misc()[MI_ONEQ], P);
                sm[G::swz(C > 1 ? i & (LCN - 1) : i)] = x[j];
            }
        }
    }
    template <int PASS>
    CF_HD void from_smem(int t, u64 (&x)[E]) const {
        if constexpr (C > 1 && PASS == 0) {
#pragma unroll
            for (int j = 0; j < E; ++j) x[j] = sm[Smem<G>::X0 + lt(t) + j * CT];
        } else {
#pragma unroll
            for (int j = 0; j < E; ++j) {
                const int i = G::idx(PASS, t, j);
                x[j] = sm[G::swz(C > 1 ? i & (LCN - 1) : i)];
            }
        }
    }
    // the barrier before pass PASS reads shared memory: the cluster's at the exchanges
    template <int PASS, bool FWD>
    CF_HD void pass_sync() {
        if constexpr (C > 1 && ((FWD && PASS == 1) || (!FWD && PASS == 0))) ex.cluster_sync();
        else ex.sync();
    }

    template <int PASS>
    CF_HD void fwd_chain() {  // forward passes PASS .. NP-1, pointwise, last inverse pass (PASS >= 1)
        pass_sync<PASS, true>();
        ex.each([&](int t, Regs<G>& rg) CF_INL {
            from_smem<PASS>(t, rg.x);
            fwd_pass<PASS>(t, rg.x);
            if (PASS == NP - 1) {
                pointwise(t, rg.x);
                inv_pass<PASS>(t, rg.x);
            }
            to_smem<PASS, PASS == 1 && NP == 2>(t, rg.x);  // the inverse's pass 1 only when it is the last
        });
        if constexpr (PASS + 1 < NP) fwd_chain<PASS + 1>();
    }
    template <int PASS>
    CF_HD void inv_chain() {  // inverse passes PASS .. 0 (entry: data in smem in layout PASS + 1)
        pass_sync<PASS, false>();
        ex.each([&](int t, Regs<G>& rg) CF_INL {
            from_smem<PASS>(t, rg.x);
            inv_pass<PASS>(t, rg.x);
            if (PASS > 0) to_smem<PASS, PASS == 1>(t, rg.x);
        });
        if constexpr (PASS > 0) inv_chain<PASS - 1>();
    }
    // spectrum pairs of chunk C (entries 4C .. 4C+3) from tensor memory, then the next chunk
    template <int CH>
    CF_HD void tm_pointwise(int t, u32 ta, u64 (&x)[E], u32 (&b0)[16], u32 (&b1)[16]) const {
        if constexpr (CH < E / 4) {
            u32(&cur)[16] = (CH & 1) ? b1 : b0;
            u32(&nxt)[16] = (CH & 1) ? b0 : b1;
            if constexpr (CH + 1 < E / 4) ex.tmem_ld16(t, ta + 16 * (CH + 1), nxt);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const u64 w = (u64)cur[4 * k] | ((u64)cur[4 * k + 1] << 32), wq = (u64)cur[4 * k + 2] | ((u64)cur[4 * k + 3] << 32);
                x[4 * CH + k] = shoup_mul_lazy(x[4 * CH + k], w, wq, P);
                if constexpr (W) x[4 * CH + k] = red2(x[4 * CH + k], 2 * P);
            }
            ex.tmem_wait_ld();
            tm_pointwise<CH + 1>(t, ta, x, b0, b1);
        }
    }
    CF_HD void pointwise(int t, u64 (&x)[E]) const {
        if constexpr (TM) {
            const u32 ta = X::tmem_addr((u32)misc()[MI_TMEM], lt(t));
            u32 b0[16], b1[16];
            ex.tmem_ld16(t, ta, b0);
            ex.tmem_wait_ld();
            tm_pointwise<0>(t, ta, x, b0, b1);
            return;
        }
        const u64* h = hat();
        pipe_pairs<E, PD, WK, CG>(
            [&](auto jc) CF_INL { return h + 2 * G::idx(NP - 1, t, decltype(jc)::value); },
            [&](auto jc, u64 w, u64 wq) CF_INL {
                constexpr int j = decltype(jc)::value;
                pin(x[j]);
                x[j] = shoup_mul_lazy(x[j], w, wq, P);
                if constexpr (W) x[j] = red2(x[j], 2 * P);
            },
            [&](auto jc) CF_INL { pin(x[decltype(jc)::value]); });
    }
    // Cyclic convolution of the registers (layout of pass 0, values < 4p) with the kernel 1/t;
    // the result comes back in the same layout, below INV_OUT p (below 2p for W).
    CF_HD void convolve() {
        if constexpr (NP == 1) {
            ex.each([&](int t, Regs<G>& rg) CF_INL {
                fwd_pass<0>(t, rg.x);
                pointwise(t, rg.x);
                inv_pass<0>(t, rg.x);
            });
        } else {
            ex.each([&](int t, Regs<G>& rg) CF_INL {
                fwd_pass<0>(t, rg.x);
                to_smem<0>(t, rg.x);
            });
            fwd_chain<1>();
            inv_chain<NP - 2>();
        }
    }
    // forward transform only (registers in layout 0 -> registers in layout NP-1), used for the
    // kernel spectrum
    template <int PASS>
    CF_HD void fwd_only_chain() {
        pass_sync<PASS, true>();
        ex.each([&](int t, Regs<G>& rg) CF_INL {
            from_smem<PASS>(t, rg.x);
            fwd_pass<PASS>(t, rg.x);
            if (PASS < NP - 1) to_smem<PASS>(t, rg.x);
        });
        if constexpr (PASS + 1 < NP) fwd_only_chain<PASS + 1>();
    }
    CF_HD void fwd_only() {
        if constexpr (NP == 1) {
            ex.each([&](int t, Regs<G>& rg) CF_INL { fwd_pass<0>(t, rg.x); });
        } else {
            ex.each([&](int t, Regs<G>& rg) CF_INL {
                fwd_pass<0>(t, rg.x);
                to_smem<0>(t, rg.x);
            });
            fwd_only_chain<1>();
        }
    }

    // Block sum mod p of the values the CTA's threads left in RED[t] (returned to every thread).
    CF_HD u64 sum_red() {
        u64* red = sm + Smem<G>::RED;
        ex.sync();
        ex.reduce_mod(red, CT, P);
        ex.sync();
        return red[CT];
    }

    // value of a pair table, canonical
    CF_HD static u64 val(const u64* pairs, int k) { return ldc<CG>(pairs + 2 * k); }

    // The slots' powers h^(t + jT), j = 0 .. E-1, as NCH independent running products: chain c
    // holds h^(t + jT) for j = c (mod NCH) and steps by h^(NCH T), so the products that depend on
    // one another are NCH times fewer than with one chain.
    static constexpr int NCH = E >= 4 ? 4 : E;

    // Stage-2 powers of h = 1/g(v) (base 0: the row products) and h = g(v) (base 1: the stage-2
    // products), Montgomery form, rebuilt at the start of each step in shared memory (the PW_*
    // slots): A[k] = h^k (k < TA = min(T, 32)), B[k] = h^(TA k) (k < TB = T / TA), J[j] = h^(T j)
    // (j < E), the chains' step h^(NCH T) as a plain residue with its Shoup companion (a Shoup product
    // by it keeps a Montgomery-form power in Montgomery form), and h^L.  Slot j of thread t holds
    // index t + jT, whose power is A[t % TA] B[t / TA] J[j].  The six groups (A, B, J for two bases)
    // go to six warps, fewer warps looping over them; a group's lanes raise a common base (h, h^TA
    // or h^T, which every lane squares up itself) to their own small exponent, so the deepest chain
    // is about 20 products, and h comes from the table of g(v) built at setup.  The other warps go
    // straight on with stage 1: the tables are read only after its barriers.  In a cluster, t is the
    // thread's index in its CTA and J[j] = h^(c CT + T j) carries the CTA's offset c CT.
    static constexpr int TA = CT < 32 ? CT : 32, TB = CT / TA;
    static constexpr int LW = CT < 32 ? CT : 32;  // lanes of a warp
    CF_HD static constexpr int log2c(int x) { return x <= 1 ? 0 : 1 + log2c(x / 2); }
    CF_HD void power_tables(int v) {
        u64* pw = sm + Smem<G>::PW;
        const u64* gm = Gm();
        ex.each([&](int t, Regs<G>&) CF_INL {
            const int lane = t & 31;
            for (int gi = lt(t) >> 5; gi < 6; gi += NW) {
                const int base = gi & 1, kind = gi >> 1;
                const int size = kind == 0 ? TA : kind == 1 ? TB : E + 2;
                if (lane >= size) continue;
                const Mod m = md();
                u64* tab = pw + base * Smem<G>::PW_STRIDE;
                u64 b = ldc<CG>(gm + 2 * v + 1 - base);  // 1/g(v) or g(v)
                u64 off = m.r1;                          // h^(c CT): the CTA's offset (clusters)
                if constexpr (C > 1)
                    if (kind == 2 && rank() > 0) off = mont_pow(b, (u64)rank() * CT, m);
                const int sq = kind == 0 ? 0 : kind == 1 ? log2c(TA) : log2c(T);
                for (int i = 0; i < sq; ++i) b = mont_mul(b, b, m);
                for (int k = lane; k < size; k += LW) {
                    if (kind == 0) tab[PW_A + k] = mont_pow(b, (u64)k, m);
                    else if (kind == 1) tab[PW_B + k] = mont_pow(b, (u64)k, m);
                    else if (k < E) tab[PW_J + k] = C > 1 ? mont_mul(mont_pow(b, (u64)k, m), off, m) : mont_pow(b, (u64)k, m);
                    else if (k == E) {
                        const u64 y = from_mont(mont_pow(b, (u64)NCH, m), m);
                        tab[PW_STEP] = y;
                        tab[PW_STEPQ] = shoup_companion_fast(y, P, misc()[MI_ONEQ], m.r1, misc()[MI_R1Q]);
                    } else tab[PW_L] = mont_pow(b, (u64)E, m);
                }
            }
        });
    }
    // chain c of thread t holds h^(t + jT) for j = c (mod NCH) in Montgomery form and steps by a
    // Shoup product with (step, stepq) = h^(NCH T) and its companion: values in [0, 4p) for primes
    // below 2^50; canonical for W, where mont_mul's full product is exact only below 2^62
    CF_HD u64 chain_step(u64 f, u64 step, u64 stepq) const {
        const u64 y = shoup_mul_lazy(f, step, stepq, P);
        if constexpr (W) return canon(y);
        return y;
    }
    // Chains started at slot j0 (the first slot a warp needs): chain c starts at the first slot
    // j >= j0 with j = c (mod NCH), from A[t % TA] B[t / TA] J[j].
    CF_HD void power_chains(int base, int t, const Mod& m, u64 (&f)[NCH], u64& step, u64& stepq, int j0 = 0) const {
        const u64* pw = sm + Smem<G>::PW + base * Smem<G>::PW_STRIDE;
        const int tl = lt(t);
        const u64 ab = TB > 1 ? mont_mul(pw[PW_A + tl % TA], pw[PW_B + tl / TA], m) : pw[PW_A + tl];
#pragma unroll
        for (int c = 0; c < NCH; ++c) {
            const int jc = j0 + ((c - j0) & (NCH - 1));
            // J[0] = 1 on a CTA alone; in a cluster it carries the CTA's offset h^(c CT)
            f[c] = (jc == 0 && C == 1) ? ab : (jc < E ? mont_mul(ab, pw[PW_J + jc], m) : 0);
        }
        step = pw[PW_STEP], stepq = pw[PW_STEPQ];
    }
    // Index range [lo, hi] of slot j (layout 0: index t + jT) over the calling thread's warp: the
    // stage loops skip a slot, warp-uniformly, when no lane of the warp needs it.
    CF_HD static void warp_slot_range(int t, int j, int& lo, int& hi) {
        const int tw = t & ~31;
        lo = tw + j * T;
        hi = (T < 32 ? T - 1 : tw + 31) + j * T;
    }

    // g(v) and 1/g(v) in Montgomery form, from the table built at setup (0 for v < d0, subset model)
    CF_HD u64 g_mont(int v) const { return ldc<CG>(Gm() + 2 * v); }
    CF_HD u64 ginv_mont(int v) const { return ldc<CG>(Gm() + 2 * v + 1); }

    // ---------------------------------------------------------------------------------------
    // Setup: factorials, inverses, D, twiddles and the kernel spectrum of 1/t (the per-batch host
    // work of fast/cuckoo_fast.cu:797-839, done on the device).
    // ---------------------------------------------------------------------------------------
    CF_HD void setup() {
        u64* red = sm + Smem<G>::RED;  // red[t]: prefix before chunk t; red[CT + t]: chunk product / suffix
        u64* mi = misc();
        const int F = kp.F, n = kp.n, J = kp.J;
        ex.single([&]() CF_INL {
            const Mod m = make_mod(P);
            mi[MI_P] = m.p, mi[MI_PINV] = m.pinv, mi[MI_R1] = m.r1, mi[MI_R2] = m.r2;
            mi[MI_ONEQ] = shoup_companion(1, P);
            mi[MI_R1Q] = shoup_companion(m.r1, P);
        });
        ex.sync();
        // The prime's tables in global memory: one CTA builds them (the cluster's first, which its
        // other CTAs wait for at the cluster barrier below).
        if (rank() == 0) {
            const int CH = (F + 1 + CT - 1) / CT;  // factorial entries k = 0..F, chunk of CH per thread
            // product of the integers in each chunk (Montgomery form)
            ex.each([&](int t, Regs<G>&) CF_INL {
                const Mod m = md();
                const int k0 = t * CH > 1 ? t * CH : 1, k1 = (t + 1) * CH < F + 1 ? (t + 1) * CH : F + 1;
                u64 pr = m.r1;
                u64 km = to_mont((u64)k0, m);
                for (int k = k0; k < k1; ++k) {
                    pr = mont_mul(pr, km, m);
                    km = madd(km, m.r1, P);
                }
                red[CT + t] = pr;
            });
            ex.sync();
            ex.single([&]() CF_INL {  // exclusive prefix products, F!, 1/F!, exclusive suffix products / F!
                const Mod m = md();
                u64 run = m.r1;
                for (int t = 0; t < CT; ++t) {
                    red[t] = run;
                    run = mont_mul(run, red[CT + t], m);
                }
                u64 suf = mont_pow(run, P - 2, m);  // 1/F!
                for (int t = CT - 1; t >= 0; --t) {
                    const u64 c = red[CT + t];
                    red[CT + t] = suf;  // 1/F! times the product of the chunks after t = 1/(last k of chunk t)!
                    suf = mont_mul(suf, c, m);
                }
            });
            ex.sync();
            ex.each([&](int t, Regs<G>&) CF_INL {
                const Mod m = md();
                const int k0 = t * CH, k1 = (t + 1) * CH < F + 1 ? (t + 1) * CH : F + 1;
                u64 run = red[t];  // (k0 - 1)! (Montgomery), 1 for the first chunk
                u64 km = to_mont((u64)(k0 > 0 ? k0 : 1), m);
                for (int k = k0; k < k1; ++k) {  // k! = (k-1)! k
                    if (k > 0) {
                        run = mont_mul(run, km, m);
                        km = madd(km, m.r1, P);
                    }
                    put_pair(fact(), k, from_mont(run, m));
                }
                run = red[CT + t];  // 1/(k1 - 1)!
                for (int k = k1 - 1; k >= k0; --k) {  // 1/(k-1)! = k / k!
                    put_pair(ifact(), k, from_mont(run, m));
                    if (k > 0) run = mont_mul(run, to_mont((u64)k, m), m);
                }
            });
            ex.sync();
            // inv[k] = (k-1)!/k!, D[k] = 1/k!^2, Kq[k] = companion of k
            ex.each([&](int t, Regs<G>&) CF_INL {
                for (int k = t; k <= F; k += CT) put_pair(inv(), k, k ? canon(sh(val(ifact(), k), fact(), k - 1)) : 0);
                for (int k = t; k <= n; k += CT) put_pair(D(), k, canon(sh(val(ifact(), k), ifact(), k)));
                // g(k) and 1/g(k), Montgomery form: C(k, d) and its inverse, or k^d and (1/k)^d
                const Mod m = md();
                for (int k = t; k <= n; k += CT) {
                    u64 g = 0, gi = 0;
                    if (kp.model == MODEL_REPLACEMENT) {
                        if (k > 0) {
                            g = mont_pow(to_mont((u64)k, m), (u64)kp.d, m);
                            gi = mont_pow(to_mont(inv()[2 * k], m), (u64)kp.d, m);  // this thread wrote inv[k]
                        }
                    } else if (k >= kp.d) {
                        g = to_mont(canon(sh(sh(val(fact(), k), ifact(), kp.d), ifact(), k - kp.d)), m);
                        gi = to_mont(canon(sh(sh(val(ifact(), k), fact(), kp.d), fact(), k - kp.d)), m);
                    }
                    Gm()[2 * k] = g;
                    Gm()[2 * k + 1] = gi;
                }
            });
        }
        // query partial sums zeroed (each CTA's own)
        ex.each([&](int t, Regs<G>&) CF_INL {
            const size_t nps = (size_t)J * (n + 1);
            for (size_t k = lt(t); k < nps; k += CT) ps()[k] = 0;
        });
        // a root of unity of order L: x^((p-1)/L) whose (L/2)-th power is -1 (fast/cuckoo_fast.cu:815-820)
        ex.single([&]() CF_INL {
            const Mod m = md();
            const u64 minus1 = P - m.r1;
            u64 w = 0;
            int found = 0;
            for (u64 x = 2; x < 1000; ++x) {
                w = mont_pow(to_mont(x, m), (P - 1) / L, m);
                if (mont_pow(w, L / 2, m) == minus1) {
                    found = 1;
                    break;
                }
            }
            if (!found && rank() == 0) ex.set_error(kp.err, KERR_NO_ROOT);
            mi[MI_ROOT] = w;
            mi[MI_LINV] = from_mont(mont_pow(to_mont((u64)L, m), P - 2, m), m);  // 1/L, canonical
        });
        ex.sync();
        // w^k into every table that holds it: the pass-0 tables by level (global, the first CTA)
        // and the multiples of 2^R of the later passes (every CTA's shared memory)
        ex.each([&](int t, Regs<G>&) CF_INL {
            const Mod m = md();
            const u64 w = mi[MI_ROOT];
            const int tl = lt(t);
            u64 cur = mont_pow(w, (u64)tl, m);
            const u64 step = mont_pow(w, (u64)CT, m);
            for (int k = tl; k <= L / 2; k += CT) {
                const bool tw = (k & ((1 << G::R) - 1)) == 0;
                if (rank() == 0 || tw) {
                    const u64 c = from_mont(cur, m), cq = companion(c);
                    if (rank() == 0)
                        for (int l = 0; l < G::R && (k & ((1 << l) - 1)) == 0; ++l) {
                            u64* d = WL(l) + 2 * (k >> l);
                            d[0] = c, d[1] = cq;
                        }
                    if (tw) {
                        u64* d = tws() + 2 * (k >> G::R);
                        d[0] = c, d[1] = cq;
                    }
                }
                cur = mont_mul(cur, step, m);
            }
        });
        csync();  // the first CTA's tables are read below and by every later step
        // kernel spectrum: hat = DIF(ker) / L with ker[t] = 1/t for 1 <= t <= n-1 (fast/cuckoo_fast.cu:829,838-839)
        ex.each([&](int t, Regs<G>& rg) CF_INL {
#pragma unroll
            for (int j = 0; j < E; ++j) {
                const int i = G::idx(0, t, j);
                rg.x[j] = (i >= 1 && i < n) ? val(inv(), i) : 0;
            }
        });
        fwd_only();
        if (kp.keep) {  // the pair tables, for queries served later from this prime's resident V
            const KeepLayout kl = make_keep_layout(n, F);
            u64* kb = kp.keep + (size_t)b * kp.keep_words;
            ex.each([&](int t, Regs<G>&) CF_INL {
                for (size_t k = t; k < 2 * ((size_t)F + 1); k += T) {
                    kb[kl.fact + k] = fact()[k];
                    kb[kl.ifact + k] = ifact()[k];
                    kb[kl.inv + k] = inv()[k];
                }
            });
        }
        ex.each([&](int t, Regs<G>& rg) CF_INL {
            const u64 linv = mi[MI_LINV];
            const u64 linvq = companion(linv);
            if constexpr (TM) {
                const u32 ta = X::tmem_addr((u32)mi[MI_TMEM], lt(t));
#pragma unroll
                for (int c = 0; c < E / 4; ++c) {
                    u32 v[16];
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const u64 h = canon(shoup_mul_lazy(rg.x[4 * c + k], linv, linvq, P)), hq = companion(h);
                        v[4 * k] = lo32(h), v[4 * k + 1] = hi32(h), v[4 * k + 2] = lo32(hq), v[4 * k + 3] = hi32(hq);
                    }
                    ex.tmem_st16(t, ta + 16 * c, v);
                }
                ex.tmem_wait_st();
            } else {
#pragma unroll
                for (int j = 0; j < E; ++j) put_pair(hat(), G::idx(NP - 1, t, j), canon(shoup_mul_lazy(rg.x[j], linv, linvq, P)));
            }
        });
        csync();  // no CTA's transform exchange may start while another still reads its spectrum pass
    }

    // Row r of V or S into the registers (layout 0): the slot of index i gets entry i of the row
    // for lo <= i < hi, zero elsewhere.  Columns of earlier groups come from the blocks, those of
    // r's own group from the staging tile.
    //
    // In layout 0 slot j holds index i = t + jT, so when T is a multiple of 16 the column group of
    // slot j is W0 + j T/16 and the entry's place in its block is the same for every slot.  The
    // block cell of (P, W) is then linear in W on either side of h (block_cell's three cases):
    // W < h: W a_lo + b_lo; W >= h: W h + b_hi.  That replaces blk_off's per-entry case analysis.
    CF_HD void load_row(int t, u64 (&x)[E], const u64* pool, const u64* tile, int r, int lo, int hi) const {
        const int n = kp.n, v0 = tile_v0(r), h = block_h(n);
        const u64* tl = tile + r;
        if constexpr (T % TILE == 0) {
            const int P = grp(r), W0 = (t - 1) >> 4;  // -1 for t = 0, whose slot 0 is never in range
            const int a_lo = P < h ? h : 1, b_lo = P < h ? P : (P - h) * h, b_hi = P - h - 1 - h * h;
            const u64* base = pool + ((size_t)((r - 1) & 15) << 4) + ((t - 1) & 15);
#pragma unroll
            for (int j = 0; j < E; ++j) {
                const int i = t + j * T, wg = W0 + j * (T / TILE);  // column group
                const int cell = wg < h ? wg * a_lo + b_lo : wg * h + b_hi;
                x[j] = (i >= lo && i < hi) ? lds<CG>(i < v0 ? base + ((size_t)cell << 8) : tl + (size_t)(i - v0) * (n + 1)) : 0;
            }
        } else {
#pragma unroll
            for (int j = 0; j < E; ++j) {
                const int i = G::idx(0, t, j);
                x[j] = (i >= lo && i < hi) ? lds<CG>(i < v0 ? pool + blk_off(r, i, h) : tl + (size_t)(i - v0) * (n + 1)) : 0;
            }
        }
    }

    // ---------------------------------------------------------------------------------------
    // Query partial sums for row q: sum_{w<q} Vs[q][w] / (M_j - w) for every query with n_j >= q
    // (the U[w] / (M - w) sums of fast/cuckoo_fast.cu:306-323, 595-622).  The row is in the
    // registers (layout 0, entries outside the row zero).  Only the slots below q are visited: the
    // warp leaves the unrolled slot loop at its first slot wholly at or above q (slot indices grow
    // with j, so the exit is warp-uniform), which makes a query cost about n_j^2 / 2 products
    // instead of n_j L.  Each warp leaves its sum at QS[j][warp] in shared memory; fold_queries
    // combines them after the next barrier.
    // ---------------------------------------------------------------------------------------
    CF_HD void query_row(int q) {
        u64* qs = sm + Smem<G>::QS;
        for (int jq = 0; jq < kp.J; ++jq) {
            const int nj = kp.qn[jq], Mj = kp.qM[jq];
            if (nj < q) continue;
            ex.each([&](int t, Regs<G>& rg) CF_INL {
                const u64* iv = inv() + 2 * (size_t)Mj;  // the pair of 1/(M_j - w) sits at iv - 2w
                const int tw = t & ~31;                  // the warp's first thread
                u64 acc = 0;
                if constexpr (C == 1) {  // the next slot's inverse loaded one slot ahead
                    u64 c0 = 0, q0 = 0;
                    if (G::idx(0, t, 0) < q) ldp<CG>(iv - 2 * G::idx(0, t, 0), c0, q0);
#pragma unroll
                    for (int j = 0; j < E; ++j) {
                        const bool more = j + 1 < E && G::idx(0, tw, j + 1) < q;
                        u64 c1 = 0, q1 = 0;  // slots at or above q multiply by zero
                        if (more && G::idx(0, t, j + 1) < q) ldp<CG>(iv - 2 * G::idx(0, t, j + 1), c1, q1);
                        if constexpr (W) acc = madd(acc, canon(shoup_mul_lazy(rg.x[j], c0, q0, P)), P);
                        else acc += shoup_mul_lazy(rg.x[j], c0, q0, P);  // E terms below 4p: < 2^57
                        if (!more) break;
                        c0 = c1, q0 = q1;
                    }
                } else {
                    // A cluster's CTAs have half the warps of the 2^14 kernel to hide the inverses'
                    // L2 latency: they load QD slots ahead (a ring of QD + 1 pairs).  Measured at
                    // n = 65536 with 126 queries: 8.29 against 8.86 s per launch; with one query the
                    // deeper ring cost the 2^14 kernel 1.5 %, so that kernel keeps one slot.
                    constexpr int QD = 4;
                    u64 rc[QD + 1], rq[QD + 1];
#pragma unroll
                    for (int j = 0; j < QD + 1; ++j) rc[j] = rq[j] = 0;
#pragma unroll
                    for (int j = 0; j < QD && j < E; ++j)
                        if (G::idx(0, t, j) < q) ldp<CG>(iv - 2 * G::idx(0, t, j), rc[j], rq[j]);
#pragma unroll
                    for (int j = 0; j < E; ++j) {
                        if (G::idx(0, tw, j) >= q) break;  // warp-uniform: this slot and the later ones lie past the row
                        const int jn = j + QD;
                        if (jn < E && G::idx(0, t, jn) < q) ldp<CG>(iv - 2 * G::idx(0, t, jn), rc[jn % (QD + 1)], rq[jn % (QD + 1)]);
                        const u64 c0 = G::idx(0, t, j) < q ? rc[j % (QD + 1)] : 0;  // slots at or above q multiply by zero
                        const u64 q0 = G::idx(0, t, j) < q ? rq[j % (QD + 1)] : 0;
                        if constexpr (W) acc = madd(acc, canon(shoup_mul_lazy(rg.x[j], c0, q0, P)), P);
                        else acc += shoup_mul_lazy(rg.x[j], c0, q0, P);  // E terms below 4p: < 2^57
                    }
                }
                const u64 part = canon(shoup_mul_lazy(acc, 1, misc()[MI_ONEQ], P));
                ex.warp_sum_store(lt(t), part, P, qs + (size_t)jq * NW, 1);
            });
        }
    }
    // Row q's per-warp partials (written by query_row before a barrier) into ps[j][q]: warp w folds
    // queries w, w + NW, ... with shuffles.
    CF_HD void fold_queries(int q) {
        const u64* qs = sm + Smem<G>::QS;
        ex.each([&](int t, Regs<G>&) CF_INL {
            const int w = lt(t) >> 5, lane = t & 31;
            for (int jq = w; jq < kp.J; jq += NW) {
                if (kp.qn[jq] < q) continue;
                const u64 v = lane < NW ? qs[(size_t)jq * NW + lane] : 0;
                ex.warp_sum_store(lt(t), v, P, ps() + (size_t)jq * (kp.n + 1) + q, 0);
            }
        });
    }

    // One step of the suffix recurrence (fast/cuckoo_fast.cu:841-855).
    CF_HD void step(int v) {
        const int n = kp.n, d0 = kp.d0;
        if (v >= d0) power_tables(v);  // read after the barriers of stage 1 / the stage-2 barrier
        if (v > d0) {  // stage 1: column v of S from row v of V
            ex.each([&](int t, Regs<G>& rg) CF_INL {
                load_row(t, rg.x, V(), VS(), v, d0, v);  // columns w < d0 of V are zero (g(w) = 0), never written
            });
            query_row(v);
            convolve();
            ex.each([&](int t, Regs<G>& rg) CF_INL {
                const u64 iv = val(inv(), v), ivq = ldc<CG>(inv() + 2 * v + 1);
                u64* col = SS() + (size_t)(v - tile_v0(v)) * (n + 1);  // S[.][v], by row
                const u64* Dt = D();
                pipe_pairs_live<E, PD, WK, CG>(
                    [&](auto jc) CF_INL {  // rows v .. n-1 of column v: slots where the warp holds one
                        int lo, hi;
                        warp_slot_range(t, decltype(jc)::value, lo, hi);
                        return hi >= v && lo < n;
                    },
                    [&](auto jc) CF_INL {
                        const int i = G::idx(0, t, decltype(jc)::value);
                        return Dt + 2 * (i >= v && i < n ? i - v : 0);
                    },
                    [&](auto jc, u64 c, u64 cq) CF_INL {
                        constexpr int j = decltype(jc)::value;
                        const int i = G::idx(0, t, j);
                        pin(rg.x[j]);
                        // S is read only by the stage-2 Montgomery product, which takes factors
                        // below 4p: for primes below 2^50 it is stored lazily reduced
                        rg.x[j] = shoup_mul_lazy(shoup_mul_lazy(rg.x[j], c, cq, P), iv, ivq, P);
                        if constexpr (W) rg.x[j] = canon(rg.x[j]);
                        if (i >= v && i < n) st_stream(col + i, rg.x[j]);
                    },
                    [&](auto jc) CF_INL { pin(rg.x[decltype(jc)::value]); });
            });
            fold_queries(v);  // after the transform's barriers: every warp's partial of row v is in
        }
        if (v >= d0) {  // stage 2: column v of V from row v of S
            csync();  // column v of S is read below
            ex.each([&](int t, Regs<G>& rg) CF_INL {
                const Mod m = md();
                u64 f[NCH], step, stepq;  // g^-(t + jT)
                power_chains(0, t, m, f, step, stepq);
                // columns q <= d0 of S are zero (stage 1 skipped: row q of V is zero), never written
                load_row(t, rg.x, S(), SS(), v, d0 + 1, v + 1);
                window<E, WK>(
                    [&](auto jc) CF_INL {
                        constexpr int j = decltype(jc)::value;
                        int lo, hi;
                        warp_slot_range(t, j, lo, hi);
                        if (lo > v) return;  // entries q <= v only: this slot and the later ones stay zero
                        pin(rg.x[j]);
                        rg.x[j] = mont_mul(rg.x[j], f[j % NCH], m);  // x, f < 4p: exact, canonical
                        f[j % NCH] = chain_step(f[j % NCH], step, stepq);
                    },
                    [&](auto jc) CF_INL { pin(rg.x[decltype(jc)::value]); });
            });
            convolve();
            ex.each([&](int t, Regs<G>& rg) CF_INL {
                const Mod m = md();
                // Entries p = v+1 .. n: the warp's first slot holding one is j0, and its chains start
                // there.  When L = n, e[n] sits at index 0 (thread 0, slot 0): a slot of its own, done
                // below by thread 0 alone when warp 0 skips slot 0, so no warp does more than the rest.
                int j0 = 0;
#pragma unroll
                for (int j = 0; j < E; ++j) {
                    int lo, hi;
                    warp_slot_range(t, j, lo, hi);
                    j0 += hi <= v;
                }
                u64 f[NCH], step, stepq;  // g^(t + jT)
                power_chains(1, t, m, f, step, stepq, j0);
                const u64 dv = val(D(), v);
                u64* col = VS() + (size_t)(v - tile_v0(v)) * (n + 1);  // V[.][v], by row
                const u64* Dt = D();
                const u64 mu = misc()[MI_ONEQ];  // floor(2^64 / p)
                const u64 fwrap = sm[Smem<G>::PW + Smem<G>::PW_STRIDE + PW_L];  // g^L, for e[n] at index 0 when L = n
                // W: the multipliers p of the slots as a running Montgomery form (p = t + j T)
                u64 pm = W ? to_mont((u64)(t + j0 * T), m) : 0;
                const u64 pmT = W ? to_mont((u64)T, m) : 0, pmL = (W && t == 0 && n == L) ? to_mont((u64)L, m) : 0;
                // V[p][v] = g^p D[p-v-1] (D[v] - p e[p]) for a conv output x = e[p], (c, cq) = D[p-v-1],
                // gp = g^p and (W) pmv = p in Montgomery form
                auto entry = [&](u64 x, int p, u64 c, u64 cq, u64 gp, u64 pmv) CF_INL {
                    if constexpr (W) {  // x < 2P and pmv < P keep the product exact below 2^126
                        const u64 pe = mont_mul(x, pmv, m);  // p e[p], canonical
                        const u64 y = canon(shoup_mul_lazy(dv + P - pe, c, cq, P));
                        return mont_mul(y, gp, m);
                    } else {
                        // p e[p]: with p floor(2^64/p) for the companion the quotient estimate loses
                        // at most p x / 2^64 < INV_OUT more (x < INV_OUT P, p <= 2^14, P < 2^50),
                        // so pe < (INV_OUT + 4) P
                        (void)pmv;
                        const u64 pe = shoup_mul_lazy(x, (u64)p, (u64)p * mu, P);
                        check_bound(pe, G::INV_OUT + 4);
                        const u64 y = shoup_mul_lazy(dv + (G::INV_OUT + 4) * P - pe, c, cq, P);
                        return mont_mul(y, gp, m);
                    }
                };
                const bool wrap0 = n == L && t == 0;  // this thread holds e[n] at index 0
                if (wrap0 && j0 > 0 && L > v) {
                    u64 c, cq;
                    ldp<CG>(Dt + 2 * (L - v - 1), c, cq);
                    st_stream(col + L, entry(rg.x[0], L, c, cq, fwrap, pmL));
                }
                pipe_pairs_live<E, PD, WK, CG>(
                    [&](auto jc) CF_INL {
                        int lo, hi;
                        warp_slot_range(t, decltype(jc)::value, lo, hi);
                        return decltype(jc)::value >= j0 && lo <= n;
                    },
                    [&](auto jc) CF_INL {
                        const int i = G::idx(0, t, decltype(jc)::value), p = i == 0 ? L : i;
                        return Dt + 2 * (p > v && p <= n ? p - v - 1 : 0);
                    },
                    [&](auto jc, u64 c, u64 cq) CF_INL {
                        constexpr int j = decltype(jc)::value;
                        const int i = G::idx(0, t, j);
                        const bool wrap = (i == 0);  // e[n] sits at index 0 when L = n
                        const int p = wrap ? L : i;
                        pin(rg.x[j]);
                        if (p > v && p <= n) {
                            rg.x[j] = entry(rg.x[j], p, c, cq, wrap ? fwrap : f[j % NCH], wrap ? pmL : pm);
                            st_stream(col + p, rg.x[j]);
                        }
                        f[j % NCH] = chain_step(f[j % NCH], step, stepq);
                        if constexpr (W) pm = madd(pm, pmT, P);
                    },
                    [&](auto jc) CF_INL { pin(rg.x[decltype(jc)::value]); });
            });
        }
        const int v0 = tile_v0(v);
        if (v - v0 == TILE - 1 || v == n - 1) {  // move the tile's columns v0 .. v into the rows
            csync();
            // Rows of later groups only: a row of this tile's group reads these columns from the tile.
            // A full tile goes out in whole 32-byte sectors (4 columns of a block row).
            ex.each([&](int t, Regs<G>&) CF_INL {
                const int cnt = v - v0 + 1, h = block_h(n);
                const size_t cs = (size_t)n + 1;  // tile column stride
                for (int r = v0 + TILE + t; r <= n; r += T) {
                    const size_t off = blk_off(r, v0, h);  // columns v0 + c at off + c
                    if (r < n) {  // row r of S: entries q = v0 .. v, written for q > d0
                        u64* dst = S() + off;
                        const u64* src = SS() + r;
                        if (cnt == TILE && v0 > d0) {
#pragma unroll
                            for (int c = 0; c < TILE; c += 4)
                                st_stream4(dst + c, lds<CG>(src + c * cs), lds<CG>(src + (c + 1) * cs),
                                           lds<CG>(src + (c + 2) * cs), lds<CG>(src + (c + 3) * cs));
                        } else {
                            for (int c = 0; c < cnt; ++c)
                                if (v0 + c > d0) st_stream(dst + c, lds<CG>(src + c * cs));
                        }
                    }
                    u64* dst = V() + off;  // row r of V: entries w = v0 .. v, written for w >= d0
                    const u64* src = VS() + r;
                    if (cnt == TILE && v0 >= d0) {
#pragma unroll
                        for (int c = 0; c < TILE; c += 4)
                            st_stream4(dst + c, lds<CG>(src + c * cs), lds<CG>(src + (c + 1) * cs),
                                       lds<CG>(src + (c + 2) * cs), lds<CG>(src + (c + 3) * cs));
                    } else {
                        for (int c = 0; c < cnt; ++c)
                            if (v0 + c >= d0) st_stream(dst + c, lds<CG>(src + c * cs));
                    }
                }
            });
            if (kp.keep) keep_tile(v0, v);
        }
        csync();  // row v + 1 is read by the next step
    }

    // Serving builds: the tile's columns v0 .. v of V, for every row below them, into the resident
    // packed triangle.
    CF_HD void keep_tile(int v0, int v) {
        const int n = kp.n, d0 = kp.d0, cnt = v - v0 + 1;
        u64* tri = kp.keep + (size_t)b * kp.keep_words;  // the triangle sits at offset 0
        ex.each([&](int t, Regs<G>&) CF_INL {
            for (int r = v0 + 1 + t; r <= n; r += T) {
                u64* dst = tri + tri_off(r);
                const u64* src = VS() + r;
                for (int c = 0; c < cnt; ++c) {
                    const int w = v0 + c;
                    if (w >= d0 && w < r) dst[w] = lds<CG>(src + (size_t)c * (n + 1));
                }
            }
        });
    }

    // Horner finish (fast/cuckoo_fast.cu:877-890):
    //   N_bad = M! n! sum_k inv[k] ifact[n-k] ifact[M-k] Q^{n-k} ps[k],  ps[k] = sum of the warp partials.
    CF_HD void finish() {
        const int n = kp.n, d0 = kp.d0;
        u64* red = sm + Smem<G>::RED;
        if (n > d0) {  // the last row n for queries with n_j = n
            ex.each([&](int t, Regs<G>& rg) CF_INL { load_row(t, rg.x, V(), VS(), n, d0, n); });
            query_row(n);
            ex.sync();
            fold_queries(n);
        }
        csync();  // every CTA's row sums are in
        if (rank() == 0) {  // in a cluster, the first CTA adds up the CTAs' row sums
            for (int jq = 0; jq < kp.J; ++jq) {
                const int nj = kp.qn[jq], Mj = kp.qM[jq];
                ex.each([&](int t, Regs<G>&) CF_INL {
                    const Mod m = md();
                    u64 Qm;
                    if (kp.model == MODEL_REPLACEMENT) Qm = mont_pow(to_mont((u64)Mj, m), (u64)kp.d, m);
                    else Qm = to_mont(canon(sh(sh(val(fact(), Mj), ifact(), kp.d), ifact(), Mj - kp.d)), m);
                    const size_t pj = (size_t)jq * (n + 1);
                    u64 acc = 0;
                    for (int k = t + 1; k <= nj; k += CT) {
                        u64 y = ldc<CG>(ps_of(0) + pj + k);
                        for (int c = 1; c < C; ++c) y = madd(y, ldc<CG>(ps_of(c) + pj + k), P);
                        y = sh(y, inv(), k);
                        y = sh(y, ifact(), nj - k);
                        y = sh(y, ifact(), Mj - k);
                        if constexpr (W) y = canon(y);  // a factor below 2^62 keeps mont_mul exact
                        y = mont_mul(y, mont_pow(Qm, (u64)(nj - k), m), m);
                        acc = madd(acc, y, P);
                    }
                    red[t] = acc;
                });
                const u64 s = sum_red();
                ex.single([&]() CF_INL {
                    kp.out[kp.qout ? (size_t)kp.qout[jq] : (size_t)b * kp.J + jq] = canon(sh(canon(sh(s, fact(), nj)), fact(), Mj));
                });
            }
        }
    }

    // Tensor memory for the kernel spectrum is taken once per CTA, around all the primes it runs.
    CF_HD void acquire() {
        if constexpr (TM) ex.tmem_alloc((u32*)(misc() + MI_TMEM));
    }
    CF_HD void release() {
        if constexpr (TM) ex.tmem_free((u32)misc()[MI_TMEM]);
    }
    CF_HD void run_prime() {
        setup();
        for (int v = 1; v < kp.n; ++v) step(v);
        finish();
    }
    CF_HD void run() {
        acquire();
        run_prime();
        release();
    }
};

}  // namespace cfb
