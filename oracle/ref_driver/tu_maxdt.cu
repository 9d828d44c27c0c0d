// Translation unit holding the reference's CFL kernels (test oracle only):
// gpu_ocean/SWESimulators/gpu_kernels/max_dt.cu with block 12x32 and
// NUM_THREADS 256 (CDKLM16.py:219-228), launched as updateDt does
// (CDKLM16.py:720-736).
#include <cuda_runtime.h>

namespace refd {
#include "max_dt.cu"
}

extern "C" int refd_max_dt(cudaStream_t s, int nx, int ny, float dx, float dy, float g,
                           float* e, int pe, float* u, int pu, float* v, int pv, float* Hm, int phm,
                           float land, float* dt_blocks, float* dt_out) {
    dim3 block(block_width, block_height);
    dim3 grid((nx + block_width - 1) / block_width, (ny + block_height - 1) / block_height);
    refd::per_block_max_dt<<<grid, block, 0, s>>>(nx, ny, dx, dy, g, e, pe, u, pu, v, pv, Hm, phm, land,
                                                  dt_blocks, (int)(grid.x * sizeof(float)));
    refd::max_dt_reduction<<<1, NUM_THREADS, 0, s>>>((int)(grid.x * grid.y), dt_blocks, dt_out);
    return (int)cudaGetLastError();
}
