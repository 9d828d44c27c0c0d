// Launches of the column-pair stage kernel (cdklm16_pair.cuh): TMA tensor
// maps of the stage's arrays, ring size, kernel variant.
#include <cudaTypedefs.h>

#include <mutex>

#include "cdklm16_pair.cuh"
#include "dispatch.cuh"

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

int pair_threads(int shape) {
    switch (shape) {
        case GO_SHAPE_PAIR32: return 32;
        case GO_SHAPE_PAIR96: return 96;
        default: return 64;
    }
}

struct PairLaunch {
    const StageArgs* a;
    const PairMapParams* mp;
    bool tma;
    cudaStream_t s;
    template <int T, int MINB, int NS, int FRIC, bool GN, bool WF, bool RCP, bool LAND>
    cudaError_t run() {
        const dim3 grid((a->k.nx + (2 * T - 4) - 1) / (2 * T - 4),
                        (a->k.ny + a->rows_per_block - 1) / a->rows_per_block);
        if (tma) {
            auto kern = cdklm_pair_kernel<T, MINB, NS, FRIC, GN, WF, RCP, LAND, true>;
            const size_t ring = pair_ring_bytes<T>(NS, a->rk_step);
            static cudaError_t attr = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                           (int)pair_ring_bytes<T>(NS, 1));
            if (attr != cudaSuccess) return attr;
            kern<<<grid, T, ring, s>>>(*a, *mp);
        } else {
            cdklm_pair_kernel<T, MINB, NS, FRIC, GN, WF, RCP, LAND, false><<<grid, T, 0, s>>>(*a, *mp);
        }
        return cudaGetLastError();
    }
};

template <class L>
cudaError_t dispatch_pair(L& l, int shape, const Variant& v) {
    // experimental set: north-up, uniform wind, quadratic friction,
    // reciprocal quotients, no land
    if (v.gen_north || v.wind_field || v.fric != kFricQuad || !v.rcp || v.land) return cudaErrorNotSupported;
    switch (shape) {
        case GO_SHAPE_PAIR32: return l.template run<32, 12, 2, kFricQuad, false, false, true, false>();
        case GO_SHAPE_PAIR96: return l.template run<96, 4, 2, kFricQuad, false, false, true, false>();
        default: return l.template run<64, 6, 2, kFricQuad, false, false, true, false>();
    }
}

}  // namespace

bool go_pair_shape(int shape) {
    return shape == GO_SHAPE_PAIR32 || shape == GO_SHAPE_PAIR64 || shape == GO_SHAPE_PAIR96;
}

int go_pair_threads(int shape) { return pair_threads(shape); }

int go_prepare_pair(const StageArgs& a, int shape, PairMapParams* mp, bool* tma) {
    memset(mp, 0, sizeof(*mp));
    const int T = pair_threads(shape);
    const int nx = a.k.nx, ny = a.k.ny;
    // TMA needs 16-byte aligned bases and pitches; the vector stores of the
    // boundary-free blocks need 8-byte aligned outputs and an even pitch
    bool ok = encoder() != nullptr;
    const float* q[3] = {a.eta_in, a.hu_in, a.hv_in};
    const float* qn[3] = {a.qn_eta, a.qn_hu, a.qn_hv};
    for (int f = 0; f < 3 && ok; ++f) {
        ok = aligned(q[f], 16) && (a.pin * 4) % 16 == 0 && aligned(a.eta_out, 8) && aligned(a.hu_out, 8) &&
             aligned(a.hv_out, 8) && (a.pout % 2) == 0;
        if (ok) ok = encode(&mp->q[f], q[f], nx + 4, ny + 4, a.pin, 2 * T, kPairRingRows);
        if (ok && a.rk_step == 1) {
            ok = aligned(qn[f], 16) && (a.pqn * 4) % 16 == 0;
            if (ok) ok = encode(&mp->qn[f], qn[f], nx + 4, ny + 4, a.pqn, 2 * T, kPairRingRows);
        }
    }
    if (ok) ok = aligned(a.Hi, 16) && (a.phi * 4) % 16 == 0 &&
                 encode(&mp->h, a.Hi, nx + 5, ny + 5, a.phi, 2 * T + 4, kPairRingRows);
    *tma = ok;
    return GO_OK;
}

int go_launch_pair(go_domain* d, cudaStream_t s, const StageArgs& a, const PairMapParams& mp, bool tma) {
    PairLaunch L{&a, &mp, tma, s};
    const cudaError_t e = dispatch_pair(L, d->shape, go_variant(d));
    if (e == cudaErrorNotSupported)
        return go_fail(GO_ERR_UNSUPPORTED, "column-pair launch shape %d has no kernel for this variant", d->shape);
    if (e != cudaSuccess) return go_fail(GO_ERR_CUDA, "pair stage launch failed: %s", cudaGetErrorString(e));
    return GO_OK;
}
