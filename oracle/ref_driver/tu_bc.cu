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
