// Wind stress sampled at the cells, and the north vector of a constant grid
// angle, as the reference's kernel forms them from its textures.
//
// The reference binds each wind array (any size) to a texture with bilinear
// filtering, clamped addressing and normalised coordinates
// (gpu_ocean/SWESimulators/Simulator.py:171-213) and reads it at every
// interior cell (gpu_ocean/SWESimulators/gpu_kernels/common.cu:616-650,
// called from CDKLM16_kernel.cu:827-828 with ti + 0.5, tj + 0.5 and NX, NY):
// s = (ti + 0.5) / NX, t = (tj + 0.5) / NY, ti, tj the ghost-inclusive
// indices.  The texture unit holds the filter weights in fixed point, so the
// result is not the exact bilinear value.  go_sample_wind therefore does the
// same texture lookup once per wind array, with the same coordinate
// arithmetic (this file is built with --prec-div=false like the reference's
// CDKLM16 module, so ti_ / float(nx) is the same approximate division), and
// the step kernels read the sampled per-cell array.
#include "internal.h"

namespace {

__global__ void k_sample_wind(cudaTextureObject_t tex, int nx, int ny, float* out, int pitch) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= nx || j >= ny) return;
    // ti + 0.5 with ti = i + 2 (an int plus a double, converted to the float
    // parameter: exact), then the float quotient
    const float ti_ = (float)((double)(i + 2) + 0.5);
    const float tj_ = (float)((double)(j + 2) + 0.5);
    const float s = ti_ / float(nx);
    const float t = tj_ / float(ny);
    out[(size_t)j * pitch + i] = tex2D<float>(tex, s, t);
}

// North vector of a constant grid angle, as getNorth forms it on the device
// (CDKLM16_kernel.cu:68-77): sinf and cosf of the float angle.
__global__ void k_north(float angle, float* out) {
    out[0] = sinf(angle);
    out[1] = cosf(angle);
}

}  // namespace

extern "C" int go_north_vector(float angle, float* north_x, float* north_y) {
    if (!north_x || !north_y) return go_fail(GO_ERR_INVALID, "null argument");
    float* d = nullptr;
    GO_CUDA(cudaMalloc(&d, 2 * sizeof(float)));
    float h[2] = {0.0f, 1.0f};
    k_north<<<1, 1>>>(angle, d);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return go_fail(GO_ERR_CUDA, "north vector: %s", cudaGetErrorString(e));
    *north_x = h[0];
    *north_y = h[1];
    return GO_OK;
}

extern "C" int go_sample_wind(void* stream, const float* field, int w, int h, int nx, int ny, float* out,
                              int out_pitch) {
    if (!field || !out) return go_fail(GO_ERR_INVALID, "null argument");
    if (w < 1 || h < 1 || nx < 1 || ny < 1) return go_fail(GO_ERR_INVALID, "empty wind field or grid");
    int rc = go_check_pitch(out_pitch, nx, "out");
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    cudaChannelFormatDesc ch = cudaCreateChannelDesc<float>();
    cudaArray_t arr = nullptr;
    GO_CUDA(cudaMallocArray(&arr, &ch, w, h));
    cudaTextureObject_t tex = 0;
    cudaError_t e = cudaMemcpy2DToArrayAsync(arr, 0, 0, field, sizeof(float) * w, sizeof(float) * w, h,
                                             cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        cudaResourceDesc res;
        memset(&res, 0, sizeof(res));
        res.resType = cudaResourceTypeArray;
        res.res.array.array = arr;
        cudaTextureDesc td;
        memset(&td, 0, sizeof(td));
        td.addressMode[0] = cudaAddressModeClamp;
        td.addressMode[1] = cudaAddressModeClamp;
        td.filterMode = cudaFilterModeLinear;
        td.readMode = cudaReadModeElementType;
        td.normalizedCoords = 1;
        e = cudaCreateTextureObject(&tex, &res, &td, nullptr);
    }
    if (e == cudaSuccess) {
        const dim3 b(32, 8), g((nx + 31) / 32, (ny + 7) / 8);
        k_sample_wind<<<g, b, 0, s>>>(tex, nx, ny, out, out_pitch / 4);
        e = cudaGetLastError();
    }
    // the array and texture live until the lookup is done (a set-up call,
    // once per wind interval, as the reference synchronises around its
    // texture uploads)
    const cudaError_t es = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = es;
    if (tex) cudaDestroyTextureObject(tex);
    cudaFreeArray(arr);
    if (e != cudaSuccess) return go_fail(GO_ERR_CUDA, "wind sampling failed: %s", cudaGetErrorString(e));
    return GO_OK;
}
