// Translation unit holding the reference's model-error kernels (test oracle
// only): gpu_ocean/SWESimulators/gpu_kernels/ocean_noise.cu, built with
// --use_fast_math and 16 x 16 blocks as OceanStateNoise.py:222-227 gets it,
// launched with the grids of OceanStateNoise.py:250-282 and :343-496.
// The caller gives the random buffer spare rows and columns: the
// reference's SOAR tile reads one row and one column past a non-periodic
// random field for blocks at the upper edge (ocean_noise.cu:300-330).
#include <cuda_runtime.h>

namespace refn {
#include "ocean_noise.cu"
}

static dim3 grid_for(int nx, int ny) { return dim3((nx + 15) / 16, (ny + 15) / 16); }

extern "C" int refn_set_textures(cudaTextureObject_t angle, cudaTextureObject_t coriolis) {
    cudaError_t e = cudaMemcpyToSymbol(refn::angle_tex, &angle, sizeof(angle));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(refn::coriolis_f_tex, &coriolis, sizeof(coriolis));
    return (int)e;
}

extern "C" int refn_lcg(cudaStream_t s, int normal, int seed_nx, int seed_ny, int random_nx,
                        unsigned long long* seed, int seed_pitch, float* random, int random_pitch) {
    if (normal)
        refn::normalDistribution<<<grid_for(seed_nx, seed_ny), dim3(16, 16), 0, s>>>(
            seed_nx, seed_ny, random_nx, seed, seed_pitch, random, random_pitch);
    else
        refn::uniformDistribution<<<grid_for(seed_nx, seed_ny), dim3(16, 16), 0, s>>>(
            seed_nx, seed_ny, random_nx, seed, seed_pitch, random, random_pitch);
    return (int)cudaGetLastError();
}

extern "C" int refn_soar(cudaStream_t s, int cnx, int cny, float cdx, float cdy, float q0, float L, float scale,
                         int pns, int pew, float* random, int random_pitch, float* coarse, int coarse_pitch,
                         int additive) {
    refn::SOAR<<<grid_for(cnx + 4, cny + 4), dim3(16, 16), 0, s>>>(cnx, cny, cdx, cdy, q0, L, scale, pns, pew,
                                                                     random, random_pitch, coarse, coarse_pitch,
                                                                     additive);
    return (int)cudaGetLastError();
}

extern "C" int refn_geostrophic(cudaStream_t s, int nx, int ny, float dx, float dy, int gx, int gy, float g,
                                float f, float beta, float y0, float* coarse, int cp, float* eta, int pe, float* hu,
                                int pu, float* hv, int pv, float* Hi, int ph, float land) {
    refn::geostrophicBalance<<<grid_for(nx, ny), dim3(16, 16), 0, s>>>(nx, ny, dx, dy, gx, gy, g, f, beta, y0,
                                                                        coarse, cp, eta, pe, hu, pu, hv, pv, Hi, ph,
                                                                        land);
    return (int)cudaGetLastError();
}

extern "C" int refn_bicubic(cudaStream_t s, int nx, int ny, int gx, int gy, float dx, float dy, int cnx, int cny,
                            int cgx, int cgy, float cdx, float cdy, int oi, int oj, float g, float f, float beta,
                            float y0, float* coarse, int cp, float* eta, int pe, float* hu, int pu, float* hv,
                            int pv, float* Hi, int ph, float land) {
    refn::bicubicInterpolation<<<grid_for(nx, ny), dim3(16, 16), 0, s>>>(nx, ny, gx, gy, dx, dy, cnx, cny, cgx,
                                                                          cgy, cdx, cdy, oi, oj, g, f, beta, y0,
                                                                          coarse, cp, eta, pe, hu, pu, hv, pv, Hi,
                                                                          ph, land);
    return (int)cudaGetLastError();
}

extern "C" int refn_make_perpendicular(cudaStream_t s, int nx, int ny, float* xi, int px, float* nu, int pn,
                                       float* red) {
    refn::makePerpendicular<<<grid_for(nx, ny), dim3(16, 16), 0, s>>>(nx, ny, xi, px, nu, pn, red);
    return (int)cudaGetLastError();
}
