// Test harness (not product code): runs the engine's per-prime phase code from
// cuckoo-failure_b200/csrc/suffix_engine.cuh on the CPU, one emulated thread after another between
// barriers, so the index logic of the CUDA kernel can be checked against the oracle without a GPU.
// It is never linked into the product library and is not a fallback for it.
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

// every value bound the transforms rely on is checked here (suffix_engine.cuh: check_bound)
#define CF_CHECK_BOUNDS 1
#include "../../cuckoo-failure_b200/csrc/host_common.hpp"
#include "../../cuckoo-failure_b200/csrc/suffix_engine.cuh"

using namespace cfb;

// A cluster's CTAs run as host threads, one per CTA, meeting at the cluster barriers; each CTA's
// shared memory is its own array, which the others write through st_remote.
struct ClusterShared {
    int C = 1;
    std::vector<u64*> smem;  // each CTA's shared memory
    size_t words = 0;
    std::mutex mu;
    std::condition_variable cv;
    int arrived = 0;
    long gen = 0;
    bool aborted = false;  // a CTA failed: the barriers stop waiting so the others end too
    void wait() {
        std::unique_lock<std::mutex> lk(mu);
        if (aborted) return;
        const long g = gen;
        if (++arrived == C) {
            arrived = 0;
            ++gen;
            cv.notify_all();
        } else {
            cv.wait(lk, [&] { return gen != g || aborted; });
        }
    }
    void abort() {
        std::lock_guard<std::mutex> lk(mu);
        aborted = true;
        cv.notify_all();
    }
};

template <class G>
struct HostExec {
    std::vector<Regs<G>> regs;
    int rk = 0;                   // CTA rank in the cluster
    ClusterShared* cl = nullptr;  // the cluster (null: a lone CTA)
    u64* own = nullptr;           // this CTA's shared memory
    HostExec() : regs(G::CT) {}
    int rank() const { return rk; }
    template <class F>
    void each(F&& f) {
        for (int t = 0; t < G::CT; ++t) f(rk * G::CT + t, regs[t]);
    }
    void cluster_sync() {
        if (cl) cl->wait();
    }
    void st_remote(u64* p, int r, u64 v) {
        const ptrdiff_t off = p - own;
        if (!cl || r < 0 || r >= cl->C || off < 0 || (size_t)off >= cl->words)
            throw std::runtime_error("distributed shared memory store out of range");
        cl->smem[r][off] = v;
    }
    template <class F>
    void single(F&& f) {
        f();
    }
    void sync() {}
    void set_error(int* err, int code) {
        if (*err == 0) *err = code;
    }
    // tensor memory: 128 lanes x 512 columns of 32-bit words, same ownership as on the device
    std::vector<u32> tm = std::vector<u32>(128 * 512, 0xDEADBEEFu);
    void tmem_alloc(u32* slot) { *slot = 0; }
    void tmem_free(u32) {}
    void tmem_sync() {}
    static u32 tmem_addr(u32 base, int t) {
        const int w = t >> 5;
        return base + ((u32)(32 * (w & 3)) << 16) + (u32)(4 * G::E * (w >> 2));
    }
    u32* tmem_word(int t, u32 ta, int k) {
        const int lane = (int)(ta >> 16) + (t & 31), col = (int)(ta & 0xFFFF) + k;
        // the columns the device allocates: all 512, or 4 E CT / 128 (at least 32) for a cluster's CTA
        const int cols = G::C == 1 ? 512 : (4 * G::E * (G::CT / 128) < 32 ? 32 : 4 * G::E * (G::CT / 128));
        if (lane >= 128 || col >= cols) throw std::runtime_error("tensor memory address out of range");
        return &tm[(size_t)lane * 512 + col];
    }
    void tmem_st16(int t, u32 ta, const u32 (&v)[16]) {
        for (int k = 0; k < 16; ++k) *tmem_word(t, ta, k) = v[k];
    }
    void tmem_ld16(int t, u32 ta, u32 (&v)[16]) {
        for (int k = 0; k < 16; ++k) v[k] = *tmem_word(t, ta, k);
    }
    void tmem_wait_ld() {}
    void tmem_wait_st() {}
    // warp sums, as on the device: threads of a warp run one after another, lane 0 first, so lane 0
    // stores and the later lanes add (the destination's old contents never count)
    void warp_sum_store(int t, u64 v, u64 P, u64* dst, size_t stride) {
        u64* c = dst + (size_t)(t >> 5) * stride;
        *c = (t & 31) == 0 ? v : madd(*c, v, P);
    }
    void reduce_mod(u64* red, int T, u64 P) {
        u64 s = 0;
        for (int t = 0; t < T; ++t) s = madd(s, red[t], P);
        red[T] = s;
    }
};

// The cluster kernel (transform length 2^LG on 2^LC CTAs per prime, 16 entries per thread).
template <int LG, int LC, int R = 4>
static int run_cluster(const KParams& kp) {
    typedef Geo<LG, R, LC> G;
    const size_t words = Smem<G>::bytes_for(kp.J) / 8;
    for (int b = 0; b < kp.B; ++b) {
        ClusterShared cs;
        cs.C = G::C;
        cs.words = words;
        std::vector<std::vector<u64>> sm(G::C, std::vector<u64>(words, 0xA5A5A5A5A5A5A5A5ull));
        for (int c = 0; c < G::C; ++c) cs.smem.push_back(sm[c].data());
        std::vector<std::string> errs(G::C);
        std::vector<std::thread> th;
        for (int c = 0; c < G::C; ++c)
            th.emplace_back([&, c] {
                try {
                    HostExec<G> ex;
                    ex.rk = c, ex.cl = &cs, ex.own = sm[c].data();
                    PrimeRun<G, HostExec<G>, false> pr(ex, kp, b, sm[c].data());
                    pr.run();
                } catch (const std::exception& e) {
                    errs[c] = e.what();
                    cs.abort();
                }
            });
        for (std::thread& x : th) x.join();
        for (const std::string& e : errs)
            if (!e.empty()) throw std::runtime_error(e);
    }
    return 0;
}

template <int LG>
struct RFor {
    static constexpr int R = (LG >= 11 && LG <= 14) ? 4 : (LG >= 10 ? 5 : (LG >= 6 ? LG - 5 : 1));
};

template <int LG, bool W>
static int run_lg(const KParams& kp) {
    typedef Geo<LG, RFor<LG>::R> G;
    std::vector<u64> smem(Smem<G>::bytes_for(kp.J) / 8, 0xA5A5A5A5A5A5A5A5ull);
    for (int b = 0; b < kp.B; ++b) {
        HostExec<G> ex;
        PrimeRun<G, HostExec<G>, W> pr(ex, kp, b, smem.data());
        pr.run();
    }
    return 0;
}

// Another register-pass geometry at one transform length (the autotuner's candidates): the same
// phase code with 2^R entries per thread.
template <int LG, int R>
static int run_geo(const KParams& kp) {
    typedef Geo<LG, R> G;
    std::vector<u64> smem(Smem<G>::bytes_for(kp.J) / 8, 0xA5A5A5A5A5A5A5A5ull);
    for (int b = 0; b < kp.B; ++b) {
        HostExec<G> ex;
        PrimeRun<G, HostExec<G>, false> pr(ex, kp, b, smem.data());
        pr.run();
    }
    return 0;
}

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
        case 12: wide ? run_lg<12, true>(kp) : run_lg<12, false>(kp); break;
        case 13: wide ? run_lg<13, true>(kp) : run_lg<13, false>(kp); break;
        case 14: wide ? run_lg<14, true>(kp) : run_lg<14, false>(kp); break;
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
extern "C" int emu_residues_geo(const uint64_t* primes, int B, int nmax, int d, int model, const int* qn, const int* qM,
                                int J, uint64_t* out, int R) {
    int F = nmax;
    for (int j = 0; j < J; ++j) F = qM[j] > F ? qM[j] : F;
    if (model == MODEL_SUBSET && d > F) F = d;
    const int L = (int)cfh::transform_length((uint64_t)nmax);
    int lg = 0;
    while ((1 << lg) < L) ++lg;
    const int T = 1 << (lg - R);
    const Layout lo = make_layout(nmax, F, L, J, T >= 32 ? T / 32 : 1, R);
    std::vector<u64> ws(lo.total * (size_t)B, 0xA5A5A5A5A5A5A5A5ull);
    int err = 0;
    KParams kp;
    kp.primes = primes, kp.B = B, kp.n = nmax, kp.F = F, kp.d = d, kp.d0 = model == MODEL_SUBSET ? d : 1;
    kp.model = model, kp.J = J, kp.qn = qn, kp.qM = qM, kp.ws = ws.data(), kp.ws_words = lo.total, kp.lay = lo;
    kp.out = out, kp.err = &err;
    try {
        if (lg == 10 && R == 4) run_geo<10, 4>(kp);
        else if (lg == 11 && R == 3) run_geo<11, 3>(kp);
        else if (lg == 12 && R == 3) run_geo<12, 3>(kp);
        else if (lg == 12 && R == 5) run_geo<12, 5>(kp);
        else if (lg == 13 && R == 5) run_geo<13, 5>(kp);
        else return -4;
    } catch (const std::runtime_error&) {
        return -6;
    }
    return err ? -5 : 0;
}
// The cluster kernels on a table of any size (the transform length forced to 2^lg, as
// cf_engine_set_transform_lg does): lg = 15 with C = 4 or 8 (-4, -8: 8 entries per thread instead
// of 16), lg = 16 with C = 8 or 16.
extern "C" int emu_residues_cluster(const uint64_t* primes, int B, int nmax, int d, int model, const int* qn,
                                    const int* qM, int J, uint64_t* out, int lg, int C) {
    int F = nmax;
    for (int j = 0; j < J; ++j) F = qM[j] > F ? qM[j] : F;
    if (model == MODEL_SUBSET && d > F) F = d;
    if ((1ull << lg) < cfh::transform_length((uint64_t)nmax)) return -1;
    const Layout lo = make_layout(nmax, F, 1 << lg, J, 1, 4, 16);  // row sums for the largest cluster, as the engine lays out
    std::vector<u64> ws(lo.total * (size_t)B, 0xA5A5A5A5A5A5A5A5ull);
    int err = 0;
    KParams kp;
    kp.primes = primes, kp.B = B, kp.n = nmax, kp.F = F, kp.d = d, kp.d0 = model == MODEL_SUBSET ? d : 1;
    kp.model = model, kp.J = J, kp.qn = qn, kp.qM = qM, kp.ws = ws.data(), kp.ws_words = lo.total, kp.lay = lo;
    kp.out = out, kp.err = &err;
    try {
        if (lg == 15 && C == -4) run_cluster<15, 2, 3>(kp);  // 8 entries per thread
        else if (lg == 15 && C == -8) run_cluster<15, 3, 3>(kp);
        else if (lg == 15 && C == 4) run_cluster<15, 2>(kp);
        else if (lg == 15 && C == 8) run_cluster<15, 3>(kp);
        else if (lg == 16 && C == 8) run_cluster<16, 3>(kp);
        else if (lg == 16 && C == 16) run_cluster<16, 4>(kp);
        else return -4;
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
