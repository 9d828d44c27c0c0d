// Boundary-frame part of a single-domain column-pair stage (every kernel variant; friction law and wind kind read at run time).
#include "pair_dispatch.cuh"

namespace go {
namespace {
struct Run {
    const PairSingleReq* r;
    template <bool GN, bool RCP, bool LAND>
    cudaError_t run() {
        cdklm_pair_kernel<kPairT, kPairMinBlocksFrame, kPairSlots, kPairUnroll, -1, -1, GN, RCP, LAND, 1>
            <<<pair_frame_count(r->g), kPairT, 0, r->s>>>(*r->a, *r->mp, r->g);
        return cudaGetLastError();
    }
};
}  // namespace

cudaError_t pair_launch_frame(const PairSingleReq& r, const Variant& v) {
    Run l{&r};
    return dispatch_pair_frame_variant(l, v);
}
}  // namespace go
