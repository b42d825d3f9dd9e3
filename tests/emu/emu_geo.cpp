// Test harness (not product code): the autotuner's other register-pass geometries, run on
// the CPU (see emu_exec.hpp).
#include "emu_exec.hpp"

using namespace cfb;

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
