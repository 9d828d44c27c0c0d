// Boundary tiles of a batched column-pair stage (every kernel variant; friction law and wind kind read at run time).
#include "pair_dispatch.cuh"

namespace go {
namespace {
struct Run {
    const PairBatchReq* r;
    template <bool GN, bool RCP, bool LAND>
    cudaError_t run() {
        cdklm_pair_batch_kernel<kPairT, kPairMinBlocksFrame, kPairSlots, kPairUnroll, -1, -1, GN, RCP, LAND, 1>
            <<<r->grid, kPairT, 0, r->s>>>(r->args, r->dts, r->tiles, r->ntiles, r->rk_step, r->maps);
        return cudaGetLastError();
    }
};
}  // namespace

cudaError_t pair_batch_launch_frame(const PairBatchReq& r, const Variant& v) {
    Run l{&r};
    return dispatch_pair_frame_variant(l, v);
}
}  // namespace go
