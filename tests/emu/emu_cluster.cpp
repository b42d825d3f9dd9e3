// Test harness (not product code): the cluster kernels (one prime per thread-block
// cluster, its CTAs as host threads), run on the CPU (see emu_exec.hpp).
#include "emu_exec.hpp"

using namespace cfb;

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
    bool wide = false;  // primes below 2^62: the engine's cluster kernels for them
    for (int b = 0; b < B; ++b) wide = wide || primes[b] >= (1ull << 50);
    try {
        if (wide && lg == 15 && C == 4) run_cluster<15, 2, 4, true>(kp);
        else if (wide && lg == 16 && C == 8) run_cluster<16, 3, 4, true>(kp);
        else if (wide) return -4;
        else if (lg == 15 && C == -4) run_cluster<15, 2, 3>(kp);  // 8 entries per thread
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
