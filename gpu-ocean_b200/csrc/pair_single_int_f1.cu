// Boundary-free part of a single-domain column-pair stage, friction law 1
// (kFricNone, kFricQuad, kFricLinear), every other kernel variant.
#include "pair_dispatch.cuh"

namespace go {
namespace {
struct Run {
    const PairSingleReq* r;
    template <int WIND, bool GN, bool RCP, bool LAND>
    cudaError_t run() {
        auto kern = cdklm_pair_kernel<kPairT, kPairMinBlocksInterior, kPairSlots, kPairUnroll, 1, WIND, GN, RCP,
                                      LAND, 0>;
        static const cudaError_t attr = cudaFuncSetAttribute(
            kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pair_ring_bytes<kPairT>(kPairSlots, 1));
        if (attr != cudaSuccess) return attr;
        const PairGrid& g = r->g;
        kern<<<dim3(g.bx1 - g.bx0, g.nby), kPairT, pair_ring_bytes<kPairT>(kPairSlots, r->a->rk_step), r->s>>>(
            *r->a, *r->mp, g);
        return cudaGetLastError();
    }
};
}  // namespace

cudaError_t pair_launch_interior_f1(const PairSingleReq& r, const Variant& v) {
    Run l{&r};
    return dispatch_pair_variant(l, v);
}
}  // namespace go
