// Launches of the column-pair stage kernel (cdklm16_pair.cuh): the TMA
// tensor maps of a stage's arrays and the two-part launch of a stage.
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>

#include "pair_dispatch.cuh"

using namespace go;

namespace {

PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_encode_once;

PFN_cuTensorMapEncodeTiled_v12000 encoder() {
    std::call_once(g_encode_once, [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    });
    return g_encode;
}

// 2-D map of a (rows x cols) float array with a pitch in floats; box of
// box_cols x box_rows.
bool encode(CUtensorMap* m, const float* base, int cols, int rows, int pitch, int box_cols, int box_rows) {
    auto fn = encoder();
    if (!fn) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)pitch * sizeof(float)};
    const cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool aligned(const void* p, size_t n) { return ((uintptr_t)p % n) == 0; }

}  // namespace

bool go_pair_shape(int shape) { return shape == GO_SHAPE_PAIR; }

namespace go {
namespace {
// Periodic east/west ghost columns of rows [2, ny+2) of a stage's output
// (boundary_kernels.cu:76-110 restricted to what the region's strips do
// not write themselves): columns 0, 1 from nx, nx+1 and nx+2, nx+3 from 2,
// 3.  blockIdx.y selects the member of a batch (args[2 m + rk_step]).
__global__ void k_periodic_columns(const StageArgs* __restrict__ args, int rk_step, StageArgs one) {
    const StageArgs& a = args ? args[2 * blockIdx.y + rk_step] : one;
    if (a.k.bcE != kPeriodic) return;
    const int nx = a.k.nx;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 4 * a.k.ny; i += gridDim.x * blockDim.x) {
        const int j = 2 + (i >> 2), c = i & 3;
        const int dst = c < 2 ? c : nx + c;
        const int src = c < 2 ? c + nx : c;
        const size_t o = (size_t)j * a.pout;
        a.eta_out[o + dst] = a.eta_out[o + src];
        a.hu_out[o + dst] = a.hu_out[o + src];
        a.hv_out[o + dst] = a.hv_out[o + src];
    }
}

}  // namespace

cudaError_t pair_launch_periodic_columns(const StageArgs* args, int n, int max_ny, int rk_step, const StageArgs& one,
                                         cudaStream_t s) {
    k_periodic_columns<<<dim3((4 * max_ny + 255) / 256, n), 256, 0, s>>>(args, rk_step, one);
    return cudaGetLastError();
}

cudaError_t pair_launch_interior(const PairSingleReq& r, const Variant& v) {
    if (v.fric == kFricQuad) return pair_launch_interior_f1(r, v);
    if (v.fric == kFricLinear) return pair_launch_interior_f2(r, v);
    return pair_launch_interior_f0(r, v);
}
cudaError_t pair_batch_launch_interior(const PairBatchReq& r, const Variant& v) {
    if (v.fric == kFricQuad) return pair_batch_launch_interior_f1(r, v);
    if (v.fric == kFricLinear) return pair_batch_launch_interior_f2(r, v);
    return pair_batch_launch_interior_f0(r, v);
}
}  // namespace go

int go_prepare_pair(const StageArgs& a, PairMapParams* mp, bool* tma) {
    memset(mp, 0, sizeof(*mp));
    constexpr int T = kPairT;
    const int nx = a.k.nx, ny = a.k.ny;
    // TMA needs 16-byte aligned bases and pitches; the vector stores of the
    // boundary-free blocks need 8-byte aligned outputs and an even pitch
    bool ok = encoder() != nullptr && aligned(a.eta_out, 8) && aligned(a.hu_out, 8) && aligned(a.hv_out, 8) &&
              (a.pout % 2) == 0 && (a.pin * 4) % 16 == 0;
    const float* q[3] = {a.eta_in, a.hu_in, a.hv_in};
    const float* qn[3] = {a.qn_eta, a.qn_hu, a.qn_hv};
    for (int f = 0; f < 3 && ok; ++f) {
        ok = aligned(q[f], 16) && encode(&mp->q[f], q[f], nx + 4, ny + 4, a.pin, 2 * T, kPairRingRows);
        if (ok && a.rk_step == 1)
            ok = aligned(qn[f], 16) && (a.pqn * 4) % 16 == 0 &&
                 encode(&mp->qn[f], qn[f], nx + 4, ny + 4, a.pqn, 2 * T, kPairRingRows);
    }
    if (ok) ok = aligned(a.Hi, 16) && (a.phi * 4) % 16 == 0 &&
                 encode(&mp->h, a.Hi, nx + 5, ny + 5, a.phi, 2 * T + 4, kPairRingRows);
    // The region's prime reads each block's 2T (+2 corner) columns straight
    // from global memory, past the end of a row into the following rows for
    // the last column block; its last Q row is ny and its last corner row
    // ny + 1, so the arrays' 4 rows below them must hold that overflow.  On
    // grids narrower than that (nx below about 37 columns) every block takes
    // the boundary path, whose loads are clamped per lane.
    const int last_cl0 = ((nx + (2 * T - 4) - 1) / (2 * T - 4) - 1) * (2 * T - 4);
    if (ok) ok = last_cl0 + 2 * T <= 4 * a.pin && last_cl0 + 2 * T + 1 <= 4 * a.phi;
    *tma = ok;
    return GO_OK;
}

// One stage: the boundary-frame kernel on the domain's high-priority side
// stream (its short strips are scheduled ahead of the region's blocks),
// forked from and joined back to the caller's stream, then the periodic
// east/west ghost columns of the output; without a side stream (the
// allocation-free step) every part runs on the caller's stream.
int go_launch_pair(go_domain* d, cudaStream_t s, const StageArgs& a, const PairMapParams& mp, bool tma) {
    const PairGrid g = pair_grid(a.k, a.rows_per_block, tma);
    const int n_int = (g.bx1 - g.bx0) * g.nby;
    const int n_frame = pair_frame_count(g);
    const Variant v = go_variant(d);
    const bool fork_join = d->side && n_int > 0 && n_frame > 0;
    PairSingleReq r{&a, &mp, g, s};
    if (n_frame > 0) {
        if (fork_join) {
            GO_CUDA(cudaEventRecord(d->ev_fork, s));
            GO_CUDA(cudaStreamWaitEvent(d->side, d->ev_fork, 0));
            r.s = d->side;
        }
        const cudaError_t e = pair_launch_frame(r, v);
        if (e != cudaSuccess) return go_fail(GO_ERR_CUDA, "stage launch (boundary frame) failed: %s", cudaGetErrorString(e));
    }
    if (n_int > 0) {
        r.s = s;
        const cudaError_t e = pair_launch_interior(r, v);
        if (e != cudaSuccess) return go_fail(GO_ERR_CUDA, "stage launch failed: %s", cudaGetErrorString(e));
    }
    if (fork_join) {
        GO_CUDA(cudaEventRecord(d->ev_join, d->side));
        GO_CUDA(cudaStreamWaitEvent(s, d->ev_join, 0));
    }
    d->stage_launches = (n_frame > 0) + (n_int > 0);
    if (n_int > 0 && a.k.bcE == kPeriodic) {
        // the region's strips leave the periodic images of their cells to this copy
        GO_CUDA(pair_launch_periodic_columns(nullptr, 1, a.k.ny, 0, a, s));
        d->stage_launches += 1;
    }
    return GO_OK;
}
