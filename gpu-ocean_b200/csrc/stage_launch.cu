// Single-domain stage launches: the column-pair kernel (pair_launch.cu) or
// a variant of the marching kernel.
#include "pair_dispatch.cuh"

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

int go_prepare_stage(go_domain* d, const StageArgs& a, PreparedStage* p) {
    p->a = a;
    p->pair = go_pair_shape(d->shape);
    p->tma = false;
    if (!p->pair) return GO_OK;
    if (d->own_side && !d->side) {
        // the boundary-frame kernel's stream and the events that fork it
        // from, and join it back to, the caller's stream
        int least = 0, greatest = 0;
        GO_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        GO_CUDA(cudaStreamCreateWithPriority(&d->side, cudaStreamNonBlocking, greatest));
        GO_CUDA(cudaEventCreateWithFlags(&d->ev_fork, cudaEventDisableTiming));
        GO_CUDA(cudaEventCreateWithFlags(&d->ev_join, cudaEventDisableTiming));
    }
    return go_prepare_pair(a, &p->mp, &p->tma);
}

int go_launch_prepared(go_domain* d, cudaStream_t s, const PreparedStage& p) {
    if (p.pair) return go_launch_pair(d, s, p.a, p.mp, p.tma);
    d->stage_launches = 1;
    SingleLaunch L{&p.a, s};
    const cudaError_t e = dispatch_variant(L, go_variant(d));
    if (e != cudaSuccess) return go_fail(GO_ERR_CUDA, "stage launch failed: %s", cudaGetErrorString(e));
    return GO_OK;
}

int go_launch_stage(go_domain* d, cudaStream_t s, const StageArgs& a) {
    PreparedStage p;
    int rc = go_prepare_stage(d, a, &p);
    if (!rc) rc = go_launch_prepared(d, s, p);
    return rc;
}
