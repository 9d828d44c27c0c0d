// Single-domain stage launches: every kernel variant of the marching stage.
#include "cdklm16_pair.cuh"
#include "dispatch.cuh"

using namespace go;

namespace {

struct SingleLaunch {
    const StageArgs* a;
    cudaStream_t s;
    template <int BW, int MINB, int FRIC, bool GN, bool WF, bool RCP, bool LAND, int D>
    cudaError_t run() {
        const dim3 grid((a->k.nx + (BW - 4) - 1) / (BW - 4), (a->k.ny + a->rows_per_block - 1) / a->rows_per_block);
        cdklm_stage_kernel<BW, MINB, FRIC, GN, WF, RCP, LAND, D><<<grid, BW, 0, s>>>(*a);
        return cudaGetLastError();
    }
};

}  // namespace

Variant go_variant(const go_domain* d) {
    Variant v;
    v.shape = d->shape;
    v.fric = go_friction_mode(d);
    v.gen_north = go_general_north(d);
    v.wind_field = d->wx_cur != nullptr;
    v.rcp = d->arith == GO_ARITH_RCP;
    v.land = d->has_land != 0;
    return v;
}

int go_prepare_pair(const StageArgs& a, int shape, PairMapParams* mp, bool* tma);
int go_launch_pair(go_domain* d, cudaStream_t s, const StageArgs& a, const PairMapParams& mp, bool tma);

int go_launch_stage(go_domain* d, cudaStream_t s, const StageArgs& a) {
    if (go_pair_shape(d->shape)) {
        PairMapParams mp;
        bool tma = false;
        int rc = go_prepare_pair(a, d->shape, &mp, &tma);
        if (!rc) rc = go_launch_pair(d, s, a, mp, tma);
        return rc;
    }
    SingleLaunch L{&a, s};
    const cudaError_t e = dispatch_variant(L, go_variant(d));
    if (e != cudaSuccess) return go_fail(GO_ERR_CUDA, "stage launch failed: %s", cudaGetErrorString(e));
    return GO_OK;
}
