// Test harness (not product code): runs the engine's per-prime phase code from
// cuckoo-failure_b200/csrc/suffix_engine.cuh on the CPU, one emulated thread after another between
// barriers, so the index logic of the CUDA kernel can be checked against the oracle without a GPU.
// It is never linked into the product library and is not a fallback for it.
#include "emu_exec.hpp"

using namespace cfb;

// The engine's block map of V / S row storage (suffix_engine.cuh), for the lifetime test.
extern "C" long emu_block_cell(int P, int W, int h) { return (long)block_cell(P, W, h); }
extern "C" long emu_block_count(int n) { return (long)block_count(n); }
extern "C" int emu_block_h(int n) { return block_h(n); }

static int emu_run(const uint64_t* primes, int B, int nmax, int d, int model, const int* qn, const int* qM, int J,
                   uint64_t* out, int Fmin, std::vector<u64>* keep);

extern "C" int emu_residues(const uint64_t* primes, int B, int nmax, int d, int model, const int* qn, const int* qM, int J,
                            uint64_t* out) {
    return emu_run(primes, B, nmax, d, model, qn, qM, J, out, 0, nullptr);
}

// A serving build of one prime (no queries): copies out the resident table (the packed triangle
// of folded V, then fact, ifact, inv pairs up to F) into keep_out[keep_words].
extern "C" long emu_keep_words(int nmax, int F) { return (long)make_keep_layout(nmax, F).total; }
extern "C" int emu_keep_build(uint64_t prime, int nmax, int Fmin, int d, int model, uint64_t* keep_out) {
    std::vector<u64> keep;
    const int rc = emu_run(&prime, 1, nmax, d, model, nullptr, nullptr, 0, nullptr, Fmin, &keep);
    if (rc == 0) std::memcpy(keep_out, keep.data(), keep.size() * sizeof(u64));
    return rc;
}

static int emu_run(const uint64_t* primes, int B, int nmax, int d, int model, const int* qn, const int* qM, int J,
                   uint64_t* out, int Fmin, std::vector<u64>* keep) {
    int F = nmax > Fmin ? nmax : Fmin;
    for (int j = 0; j < J; ++j) F = qM[j] > F ? qM[j] : F;
    if (model == MODEL_SUBSET && d > F) F = d;
    const int L = (int)cfh::transform_length((uint64_t)nmax);
    int lg = 0;
    while ((1 << lg) < L) ++lg;
    const int R = (lg >= 11 && lg <= 14) ? 4 : (lg >= 10 ? 5 : (lg >= 6 ? lg - 5 : 1)), T = 1 << (lg - R);
    const Layout lo = make_layout(nmax, F, L, J, T >= 32 ? T / 32 : 1, R);
    // poisoned, like reused device memory: every word the kernel reads must have been written first
    std::vector<u64> ws(lo.total * (size_t)B, 0xA5A5A5A5A5A5A5A5ull);
    int err = 0;
    KParams kp;
    kp.primes = primes;
    kp.B = B;
    kp.n = nmax;
    kp.F = F;
    kp.d = d;
    kp.d0 = model == MODEL_SUBSET ? d : 1;
    kp.model = model;
    kp.J = J;
    kp.qn = qn;
    kp.qM = qM;
    kp.ws = ws.data();
    kp.ws_words = lo.total;
    kp.lay = lo;
    kp.out = out;
    kp.err = &err;
    if (keep) {  // poisoned too: entries the build never writes must never be read by a query
        keep->assign(make_keep_layout(nmax, F).total * (size_t)B, 0xA5A5A5A5A5A5A5A5ull);
        kp.keep = keep->data();
        kp.keep_words = make_keep_layout(nmax, F).total;
    }
    bool wide = false;  // the kernels for primes below 2^62, as the engine selects them
    for (int b = 0; b < B; ++b) wide = wide || primes[b] >= (1ull << 50);
    try {
    switch (lg) {
        case 4: wide ? run_lg<4, true>(kp) : run_lg<4, false>(kp); break;
        case 5: wide ? run_lg<5, true>(kp) : run_lg<5, false>(kp); break;
        case 6: wide ? run_lg<6, true>(kp) : run_lg<6, false>(kp); break;
        case 7: wide ? run_lg<7, true>(kp) : run_lg<7, false>(kp); break;
        case 8: wide ? run_lg<8, true>(kp) : run_lg<8, false>(kp); break;
        case 9: wide ? run_lg<9, true>(kp) : run_lg<9, false>(kp); break;
        case 10: wide ? run_lg<10, true>(kp) : run_lg<10, false>(kp); break;
        case 11: wide ? run_lg<11, true>(kp) : run_lg<11, false>(kp); break;
        case 12:
        case 13:
        case 14: run_lg_big(lg, wide, kp); break;
        default: return -4;
    }
    } catch (const std::runtime_error&) {
        return -6;  // a value bound of the transforms did not hold (check_bound)
    }
    return err ? -5 : 0;
}

// ---- uneven batches: the work-queue launch's per-table semantics on the CPU ----
// Each table of the plan (uneven_plan.hpp) runs with its own n, F, d, model and query list in a
// workspace slot laid out for the largest table of its transform length (as k_suffix_queue's
// slots are), freshly poisoned, and scatters its residues through the query output indices.
#include "../../cuckoo-failure_b200/csrc/uneven_plan.hpp"

template <int LG, bool W>
static void run_table(const KParams& kp) {
    typedef Geo<LG, RFor<LG>::R> G;
    std::vector<u64> smem(Smem<G>::bytes_for(kp.J) / 8, 0xA5A5A5A5A5A5A5A5ull);
    HostExec<G> ex;
    PrimeRun<G, HostExec<G>, W> pr(ex, kp, 0, smem.data(), 0);
    pr.acquire();
    pr.run_prime();
    pr.release();
}

extern "C" int emu_uneven(const int* n, const int* M, const int* d, int K, int model, int bits, long first, long count,
                          long stride, uint64_t* out) {
    cfh::UnevenPlan pl;
    if (!cfh::plan_uneven(n, M, d, K, model, bits, first, count, stride, 0, pl)) return -1;
    const bool wide = bits == 62;
    int gn[16] = {0}, gF[16] = {0}, gJ[16] = {0};  // largest table of each transform length
    for (const cfh::UnevenTable& t : pl.tables) {
        gn[t.lg] = gn[t.lg] > t.n ? gn[t.lg] : t.n;
        gF[t.lg] = gF[t.lg] > t.F ? gF[t.lg] : t.F;
        gJ[t.lg] = gJ[t.lg] > t.J ? gJ[t.lg] : t.J;
    }
    int err = 0;
    try {
        for (const cfh::UnevenTable& t : pl.tables) {
            const int R = (t.lg >= 11 && t.lg <= 14) ? 4 : (t.lg >= 10 ? 5 : (t.lg >= 6 ? t.lg - 5 : 1)), T = 1 << (t.lg - R);
            const Layout lo = make_layout(gn[t.lg], gF[t.lg], 1 << t.lg, gJ[t.lg], T >= 32 ? T / 32 : 1, R);
            std::vector<u64> ws(lo.total, 0xA5A5A5A5A5A5A5A5ull);
            KParams kp;
            kp.primes = &t.prime;
            kp.B = 1;
            kp.n = t.n, kp.F = t.F, kp.d = t.d, kp.model = model, kp.J = t.J;
            kp.d0 = model == MODEL_SUBSET ? t.d : 1;
            kp.qn = pl.qn.data() + t.q0, kp.qM = pl.qM.data() + t.q0, kp.qout = pl.qout.data() + t.q0;
            kp.ws = ws.data();
            kp.ws_words = lo.total;
            kp.lay = lo;
            kp.out = out;
            kp.err = &err;
            switch (t.lg) {
                case 4: wide ? run_table<4, true>(kp) : run_table<4, false>(kp); break;
                case 5: wide ? run_table<5, true>(kp) : run_table<5, false>(kp); break;
                case 6: wide ? run_table<6, true>(kp) : run_table<6, false>(kp); break;
                case 7: wide ? run_table<7, true>(kp) : run_table<7, false>(kp); break;
                case 8: wide ? run_table<8, true>(kp) : run_table<8, false>(kp); break;
                case 9: wide ? run_table<9, true>(kp) : run_table<9, false>(kp); break;
                case 10: wide ? run_table<10, true>(kp) : run_table<10, false>(kp); break;
                case 11: wide ? run_table<11, true>(kp) : run_table<11, false>(kp); break;
                default: return -4;  // larger lengths are too slow for CPU tests
            }
        }
    } catch (const std::runtime_error&) {
        return -6;
    }
    return err ? -5 : 0;
}
extern "C" long emu_uneven_outputs(const int* n, const int* M, const int* d, int K, int model, int bits) {
    cfh::UnevenPlan pl;
    if (!cfh::plan_uneven(n, M, d, K, model, bits, 0, 0, 1, 0, pl)) return -1;
    return pl.outputs;
}
