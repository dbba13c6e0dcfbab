// The map passes on compile-time lines of 144–256 points (the sweep's candidate planes and small
// maps); a unit of its own so the instantiations compile in parallel with the others.
#include "passes.cuh"

namespace zc {

bool pass_lines_b(Pass p, const LinePlan& L, const PassArgs& a, cudaStream_t st, cudaError_t* e) {
    switch (L.n) {
        case 144: *e = run_fixed<144, false>(p, L.tw, a, st); return true;
        case 192: *e = run_fixed<192, false>(p, L.tw, a, st); return true;
        case 256: *e = run_fixed<256, false>(p, L.tw, a, st); return true;
        default: return false;
    }
}

}  // namespace zc
