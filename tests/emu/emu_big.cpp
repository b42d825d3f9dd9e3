// Test harness (not product code): the engine's phase code at transform lengths 2^12 .. 2^14 on the
// CPU (see emu_exec.hpp), in a translation unit of its own so the harness compiles in parallel.
#include "emu_exec.hpp"

using namespace cfb;

int run_lg_big(int lg, bool wide, const KParams& kp) {
    switch (lg) {
        case 12: return wide ? run_lg<12, true>(kp) : run_lg<12, false>(kp);
        case 13: return wide ? run_lg<13, true>(kp) : run_lg<13, false>(kp);
        default: return wide ? run_lg<14, true>(kp) : run_lg<14, false>(kp);
    }
}
