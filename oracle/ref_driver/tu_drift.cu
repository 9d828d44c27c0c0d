// Translation unit holding the reference's drifter and observation kernels
// (test oracle only): gpu_ocean/SWESimulators/gpu_kernels/driftKernels.cu and
// observationKernels.cu, built with nvcc's default options as
// GPUDrifterCollection.py:81-83 and OceanNoiseEnsemble.py:322-328 get them,
// launched as GPUDrifterCollection.drift (:209-232, 64 threads per block,
// ceil((n + 2) / 64) blocks) and BaseOceanStateEnsemble (:110-125) do.
#include <cuda_runtime.h>

namespace refr {
#include "driftKernels.cu"
#include "observationKernels.cu"
}

extern "C" int refr_set_drift_wind(cudaTextureObject_t xc, cudaTextureObject_t xn, cudaTextureObject_t yc,
                                   cudaTextureObject_t yn) {
    cudaError_t e = cudaMemcpyToSymbol(refr::wind_X_current, &xc, sizeof(xc));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(refr::wind_X_next, &xn, sizeof(xn));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(refr::wind_Y_current, &yc, sizeof(yc));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(refr::wind_Y_next, &yn, sizeof(yn));
    return (int)e;
}

extern "C" int refr_drift(cudaStream_t s, int nx, int ny, float dx, float dy, float dt, int x0, int y0,
                          float* eta, int pe, float* hu, int pu, float* hv, int pv, float* Hm, int ph, int pns,
                          int pew, int n, float* pos, int pp, float sensitivity, float wind_t, float wdf) {
    const int threads = 64;
    const int blocks = (int)((n + 2 + threads - 1) / threads);
    refr::passiveDrifterKernel<<<blocks, threads, 0, s>>>(nx, ny, dx, dy, dt, x0, y0, eta, pe, hu, pu, hv, pv, Hm,
                                                          ph, pns, pew, n, pos, pp, sensitivity, wind_t, wdf);
    return (int)cudaGetLastError();
}

extern "C" int refr_enforce_bc(cudaStream_t s, float size_x, float size_y, int pns, int pew, int n, float* pos,
                               int pp) {
    const int threads = 64;
    const int blocks = (int)((n + 2 + threads - 1) / threads);
    refr::enforceBoundaryConditions<<<blocks, threads, 0, s>>>(size_x, size_y, pns, pew, n, pos, pp);
    return (int)cudaGetLastError();
}

extern "C" int refr_observe(cudaStream_t s, int nx, int ny, float dx, float dy, int x0, int y0, float* eta,
                            int pe, float* hu, int pu, float* hv, int pv, float H, int n, float* pos, int pp,
                            float* obs, int po) {
    const int threads = 64;
    const int blocks = (int)((n + threads - 1) / threads);
    refr::observeUnderlyingFlow<<<blocks, threads, 0, s>>>(nx, ny, dx, dy, x0, y0, eta, pe, hu, pu, hv, pv, H, n,
                                                           pos, pp, obs, po);
    return (int)cudaGetLastError();
}
