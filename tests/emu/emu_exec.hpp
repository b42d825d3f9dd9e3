// Test harness (not product code): the host execution policy that runs the engine's per-prime
// phase code (cuckoo-failure_b200/csrc/suffix_engine.cuh) on the CPU, one emulated thread after
// another between barriers, and the per-geometry runners.  Shared by the harness's translation
// units (emu*.cpp), which compile in parallel.
#pragma once
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
template <int LG, int LC, int R = 4, bool W = false>
inline int run_cluster(const KParams& kp) {
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
                    PrimeRun<G, HostExec<G>, W> pr(ex, kp, b, sm[c].data());
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
inline int run_lg(const KParams& kp) {
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
inline int run_geo(const KParams& kp) {
    typedef Geo<LG, R> G;
    std::vector<u64> smem(Smem<G>::bytes_for(kp.J) / 8, 0xA5A5A5A5A5A5A5A5ull);
    for (int b = 0; b < kp.B; ++b) {
        HostExec<G> ex;
        PrimeRun<G, HostExec<G>, false> pr(ex, kp, b, smem.data());
        pr.run();
    }
    return 0;
}

// lg 12 .. 14 of emu_run's dispatch, compiled in emu_big.cpp
int run_lg_big(int lg, bool wide, const KParams& kp);
