// Translation unit holding the reference's boundary and bathymetry kernels
// (test oracle only): gpu_ocean/SWESimulators/gpu_kernels/boundary_kernels.cu
// and initBm_kernel.cu after the texture-object rewrite of oracle/build_ref.py,
// compiled with block_width = block_height = 16 as Common.py:1043,1357,1376 do.
#include <cuda_runtime.h>

namespace refb {
#include "boundary_kernels.cu"
#include "initBm_kernel.cu"
}

static dim3 grid_for(int w, int h) { return dim3((w + 15) / 16, (h + 15) / 16); }

// BoundaryConditionsArakawaA.boundaryCondition for periodic sides
// (Common.py:1219-1259): NS first, then EW.
extern "C" int refb_periodic(cudaStream_t s, int nx, int ny, int periodic_ns, int periodic_ew,
                             float* h, int ph, float* u, int pu, float* v, int pv) {
    dim3 block(16, 16);
    dim3 grid = grid_for(nx + 2 * 2 + 1, ny + 2 * 2 + 1);
    if (periodic_ns) refb::periodicBoundary_NS<<<grid, block, 0, s>>>(nx, ny, 2, 2, h, ph, u, pu, v, pv);
    if (periodic_ew) refb::periodicBoundary_EW<<<grid, block, 0, s>>>(nx, ny, 2, 2, h, ph, u, pu, v, pv);
    return (int)cudaGetLastError();
}

// Bathymetry.__init__ (Common.py:1355-1389): corner fix, then initBm.
extern "C" int refb_bathymetry(cudaStream_t s, int nx, int ny, int periodic_ns, int periodic_ew,
                               float* Bi, int pbi, float land, float* Bm, int pbm) {
    dim3 block(16, 16);
    dim3 grid = grid_for(nx + 4 + 1, ny + 4 + 1);
    if (periodic_ns) refb::periodic_boundary_intersections_NS<<<grid, block, 0, s>>>(nx, ny, 2, 2, Bi, pbi);
    else refb::closed_boundary_intersections_NS<<<grid, block, 0, s>>>(nx, ny, 2, 2, Bi, pbi);
    if (periodic_ew) refb::periodic_boundary_intersections_EW<<<grid, block, 0, s>>>(nx, ny, 2, 2, Bi, pbi);
    else refb::closed_boundary_intersections_EW<<<grid, block, 0, s>>>(nx, ny, 2, 2, Bi, pbi);
    refb::initBm<<<grid, block, 0, s>>>(nx + 4, ny + 4, Bi, pbi, land, Bm, pbm);
    return (int)cudaGetLastError();
}

// Exterior-solution textures of the flow relaxation (Common.py:1098-1216).
extern "C" int refb_set_open_bc_tex(cudaTextureObject_t ns0, cudaTextureObject_t ns1, cudaTextureObject_t ew0,
                                    cudaTextureObject_t ew1) {
    cudaError_t e = cudaMemcpyToSymbol(refb::bc_tex_NS_current, &ns0, sizeof(ns0));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(refb::bc_tex_NS_next, &ns1, sizeof(ns1));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(refb::bc_tex_EW_current, &ew0, sizeof(ew0));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(refb::bc_tex_EW_next, &ew1, sizeof(ew1));
    return (int)e;
}

// BoundaryConditionsArakawaA.boundaryCondition (Common.py:1219-1239) for any
// codes: north-south periodic or open kinds, then east-west.
extern "C" int refb_boundary(cudaStream_t s, int nx, int ny, int north, int east, int south, int west,
                             int sp_north, int sp_east, int sp_south, int sp_west, float bc_t,
                             float* h, int ph, float* u, int pu, float* v, int pv) {
    dim3 block(16, 16);
    dim3 grid = grid_for(nx + 2 * 2 + 1, ny + 2 * 2 + 1);
    if (north == 2) {
        refb::periodicBoundary_NS<<<grid, block, 0, s>>>(nx, ny, 2, 2, h, ph, u, pu, v, pv);
    } else {
        if (north == 3 || south == 3)
            refb::flowRelaxationScheme_NS<<<grid, block, 0, s>>>(north, south, nx, ny, 2, 2, sp_north, sp_south,
                                                                h, ph, u, pu, v, pv, bc_t);
        if (north == 4 || south == 4)
            refb::linearInterpolation_NS<<<grid, block, 0, s>>>(north, south, nx, ny, 2, 2, sp_north, sp_south,
                                                               h, ph, u, pu, v, pv);
    }
    if (east == 2) {
        refb::periodicBoundary_EW<<<grid, block, 0, s>>>(nx, ny, 2, 2, h, ph, u, pu, v, pv);
    } else {
        if (east == 3 || west == 3)
            refb::flowRelaxationScheme_EW<<<grid, block, 0, s>>>(east, west, nx, ny, 2, 2, sp_east, sp_west,
                                                                h, ph, u, pu, v, pv, bc_t);
        if (east == 4 || west == 4)
            refb::linearInterpolation_EW<<<grid, block, 0, s>>>(east, west, nx, ny, 2, 2, sp_east, sp_west,
                                                               h, ph, u, pu, v, pv);
    }
    return (int)cudaGetLastError();
}
