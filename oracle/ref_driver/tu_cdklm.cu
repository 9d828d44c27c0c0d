// Translation unit holding the reference's cdklm_swe_2D (test oracle only).
// The kernel source is gpu_ocean/SWESimulators/gpu_kernels/CDKLM16_kernel.cu
// (+ common.cu) after the texture-reference -> texture-object rewrite done
// by oracle/build_ref.py in a temporary directory; it is included, never
// copied into this repository.  Compiled with the reference's #defines
// (CDKLM16.py:179-191) and flags (CDKLM16.py:196-200).
#include <cuda_runtime.h>

namespace refk {
#include "CDKLM16_kernel.cu"
}

extern "C" int refk_set_textures(cudaTextureObject_t angle, cudaTextureObject_t coriolis,
                                 cudaTextureObject_t wxc, cudaTextureObject_t wxn,
                                 cudaTextureObject_t wyc, cudaTextureObject_t wyn) {
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(refk::angle_tex, &angle, sizeof(angle));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(refk::coriolis_f_tex, &coriolis, sizeof(coriolis));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(refk::windstress_X_current, &wxc, sizeof(wxc));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(refk::windstress_X_next, &wxn, sizeof(wxn));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(refk::windstress_Y_current, &wyc, sizeof(wyc));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(refk::windstress_Y_next, &wyn, sizeof(wyn));
    return (int)e;
}

// One launch as CDKLM16.callKernel does it (CDKLM16.py:613-639): grid
// ceil(NX/block_width) x ceil(NY/block_height) (Simulator.py:134-138).
extern "C" int refk_cdklm_swe_2D(cudaStream_t s, float dt, int rk_step,
                                 float* e0, int pe0, float* u0, int pu0, float* v0, int pv0,
                                 float* e1, int pe1, float* u1, int pu1, float* v1, int pv1,
                                 float* Hi, int phi, float* Hm, int phm, float land, float wind_t,
                                 int bc) {
    dim3 block(block_width, block_height);
    dim3 grid((NX + block_width - 1) / block_width, (NY + block_height - 1) / block_height);
    refk::cdklm_swe_2D<<<grid, block, 0, s>>>(dt, rk_step, e0, pe0, u0, pu0, v0, pv0, e1, pe1, u1, pu1,
                                              v1, pv1, Hi, phi, Hm, phm, land, wind_t, bc);
    return (int)cudaGetLastError();
}
