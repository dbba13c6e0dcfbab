// The map passes on compile-time lines of 48–128 points (the sweep's candidate planes and small
// maps); a unit of its own so the instantiations compile in parallel with the others.
#include "passes.cuh"

namespace zc {

bool pass_lines_a(Pass p, const LinePlan& L, const PassArgs& a, cudaStream_t st, cudaError_t* e) {
    switch (L.n) {
        case 48: *e = run_fixed<48, false>(p, L.tw, a, st); return true;
        case 64: *e = run_fixed<64, false>(p, L.tw, a, st); return true;
        case 96: *e = run_fixed<96, false>(p, L.tw, a, st); return true;
        case 128: *e = run_fixed<128, false>(p, L.tw, a, st); return true;
        default: return false;
    }
}

}  // namespace zc
