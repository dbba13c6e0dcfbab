// The map passes on compile-time lines of 288–512 points (the sweep's candidate planes and small
// maps); a unit of its own so the instantiations compile in parallel with the others.
#include "passes.cuh"

namespace zc {

bool pass_lines_c(Pass p, const LinePlan& L, const PassArgs& a, cudaStream_t st, cudaError_t* e) {
    switch (L.n) {
        case 288: *e = run_fixed<288, false>(p, L.tw, a, st); return true;
        case 384: *e = run_fixed<384, false>(p, L.tw, a, st); return true;
        case 432: *e = run_fixed<432, false>(p, L.tw, a, st); return true;
        case 512: *e = run_fixed<512, false>(p, L.tw, a, st); return true;
        default: return false;
    }
}

}  // namespace zc
