// Instances of the lanes-on-transforms spreading kernel for 16 transforms per lane group (one
// compilation unit per transform chunk so they build in parallel).
#include "spread_lc.cuh"

namespace hb {

int spread_lc_cc16(const NufftPlan* p, const GridArgs& a, cudaStream_t s) {
    return p->g.dim == 3 ? launch_spread_lc_w<16, true>(p, a, s) : launch_spread_lc_w<16, false>(p, a, s);
}

}  // namespace hb
