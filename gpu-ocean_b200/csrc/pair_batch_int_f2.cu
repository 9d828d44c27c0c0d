// Boundary-free tiles of a batched column-pair stage, friction law 2
// (kFricNone, kFricQuad, kFricLinear), every other kernel variant.
#include "pair_dispatch.cuh"

namespace go {
namespace {
struct Run {
    const PairBatchReq* r;
    template <int WIND, bool GN, bool RCP, bool LAND>
    cudaError_t run() {
        auto kern = cdklm_pair_batch_kernel<kPairT, kPairMinBlocksInterior, kPairSlots, kPairUnroll, 2, WIND, GN, RCP,
                                            LAND, 0>;
        static const cudaError_t attr = cudaFuncSetAttribute(
            kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pair_ring_bytes<kPairT>(kPairSlots, 1));
        if (attr != cudaSuccess) return attr;
        kern<<<r->grid, kPairT, pair_ring_bytes<kPairT>(kPairSlots, r->rk_step), r->s>>>(r->args, r->dts, r->tiles,
                                                                                        r->ntiles, r->rk_step, r->maps);
        return cudaGetLastError();
    }
};
}  // namespace

cudaError_t pair_batch_launch_interior_f2(const PairBatchReq& r, const Variant& v) {
    Run l{&r};
    return dispatch_pair_variant(l, v);
}
}  // namespace go
