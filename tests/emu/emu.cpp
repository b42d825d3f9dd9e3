// Test harness (not product code): runs the engine's per-prime phase code from
// cuckoo-failure_b200/csrc/suffix_engine.cuh on the CPU, one emulated thread after another between
// barriers, so the index logic of the CUDA kernel can be checked against the oracle without a GPU.
// It is never linked into the product library and is not a fallback for it.
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <vector>

// every value bound the transforms rely on is checked here (suffix_engine.cuh: check_bound)
#define CF_CHECK_BOUNDS 1
#include "../../cuckoo-failure_b200/csrc/host_common.hpp"
#include "../../cuckoo-failure_b200/csrc/suffix_engine.cuh"

using namespace cfb;

template <class G>
struct HostExec {
    std::vector<Regs<G>> regs;
    HostExec() : regs(G::T) {}
    template <class F>
    void each(F&& f) {
        for (int t = 0; t < G::T; ++t) f(t, regs[t]);
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
        if (lane >= 128 || col >= 512) throw std::runtime_error("tensor memory address out of range");
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
    // warp sums, as on the device: threads of a warp run one after another, dst starts at zero
    void warp_sum_store(int t, u64 v, u64 P, u64* dst, size_t stride) {
        u64* c = dst + (size_t)(t >> 5) * stride;
        *c = madd(*c, v, P);
    }
    void reduce_mod(u64* red, int T, u64 P) {
        u64 s = 0;
        for (int t = 0; t < T; ++t) s = madd(s, red[t], P);
        red[T] = s;
    }
};

template <int LG>
struct RFor {
    static constexpr int R = (LG >= 11 && LG <= 14) ? 4 : (LG >= 10 ? 5 : (LG >= 6 ? LG - 5 : 1));
};

template <int LG, bool W>
static int run_lg(const KParams& kp) {
    typedef Geo<LG, RFor<LG>::R> G;
    std::vector<u64> smem(Smem<G>::WORDS);
    for (int b = 0; b < kp.B; ++b) {
        HostExec<G> ex;
        PrimeRun<G, HostExec<G>, W> pr(ex, kp, b, smem.data());
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
