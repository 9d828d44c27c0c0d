// Open boundaries: flow relaxation (code 3) and linear interpolation
// (code 4) over the sponge rows and columns.
//
// Restates gpu_ocean/SWESimulators/gpu_kernels/boundary_kernels.cu:264-539
// (linearInterpolation_NS/EW, flowRelaxationScheme_NS/EW) as
// BoundaryConditionsArakawaA.boundaryCondition launches them
// (gpu_ocean/SWESimulators/Common.py:1219-1309): north-south first (periodic,
// or the open kinds of the two sides), then east-west.  The reference builds
// boundary_kernels.cu with nvcc's default options (Common.py:1043 passes no
// compile flags), so this unit does too (build.py UNIT_FLAGS), with the
// reference's operand order.
//
// Sponge extents are ghost-inclusive: the south sponge is rows
// [0, sponge_south), the north sponge rows (ny + 3 - sponge_north, ny + 3],
// likewise for west and east.  The exterior solution for the relaxation is
// two float4 (h, hu, hv, -) textures per time level: NS (row 0 south, row 1
// north, one texel per column) and EW (column 0 west, column 1 east, one
// texel per row), sampled bilinearly at ti / nx (or tj / ny) and linear in
// time with weight bc_t.
#include "internal.h"

namespace {

constexpr int kHalo = 2;

__global__ void k_frs_ns(int row0, int bc_north, int bc_south, int nx, int ny, int sponge_north, int sponge_south, float* h,
                         float* u, float* v, int p, cudaTextureObject_t cur, cudaTextureObject_t next, float bc_t) {
    const int ti = blockIdx.x * blockDim.x + threadIdx.x;
    const int tj = row0 + blockIdx.y * blockDim.y + threadIdx.y;   // a band of rows
    if (!(((bc_south == 3 && tj < sponge_south && tj >= 0) ||
           (bc_north == 3 && tj > ny + 2 * kHalo - 1 - sponge_north && tj < ny + 2 * kHalo)) &&
          (ti >= 0 && ti < nx + 2 * kHalo)))
        return;
    // distance from the outer edge, and the relaxation weight
    const float j = (tj <= sponge_south) ? tj - 1 : ((ny + 2 * kHalo - 2) - tj);
    const float alpha = 1.0f - tanhf(fmaxf(0.0f, j) / 2.0f);
    const float s = ti / float(nx);
    const float t = (tj < ny / 2.0) ? 0.25f : 0.75f;        // south row or north row
    const float4 c = tex2D<float4>(cur, s, t);
    const float4 n = tex2D<float4>(next, s, t);
    const float eh = bc_t * n.x + (1.0f - bc_t) * c.x;
    const float eu = bc_t * n.y + (1.0f - bc_t) * c.y;
    const float ev = bc_t * n.z + (1.0f - bc_t) * c.z;
    const size_t o = (size_t)tj * p + ti;
    h[o] = (1.0f - alpha) * h[o] + alpha * eh;
    u[o] = (1.0f - alpha) * u[o] + alpha * eu;
    v[o] = (1.0f - alpha) * v[o] + alpha * ev;
}

__global__ void k_frs_ew(int col0, int bc_east, int bc_west, int nx, int ny, int sponge_east, int sponge_west, float* h,
                         float* u, float* v, int p, cudaTextureObject_t cur, cudaTextureObject_t next, float bc_t) {
    const int ti = col0 + blockIdx.x * blockDim.x + threadIdx.x;   // a band of columns
    const int tj = blockIdx.y * blockDim.y + threadIdx.y;
    if (!(((bc_west == 3 && ti < sponge_west && ti >= 0) ||
           (bc_east == 3 && ti > nx + 2 * kHalo - 1 - sponge_east && ti < nx + 2 * kHalo)) &&
          (tj >= 0) && (tj < ny + 2 * kHalo)))
        return;
    const float j = (ti <= sponge_west) ? ti - 1 : ((nx + 2 * kHalo - 2) - ti);
    const float alpha = 1.0f - tanhf(fmaxf(0.0f, j) / 2.0f);
    const float s = (ti < nx / 2.0) ? 0.25f : 0.75f;        // west column or east column
    const float t = tj / float(ny);
    const float4 c = tex2D<float4>(cur, s, t);
    const float4 n = tex2D<float4>(next, s, t);
    const float eh = bc_t * n.x + (1.0f - bc_t) * c.x;
    const float eu = bc_t * n.y + (1.0f - bc_t) * c.y;
    const float ev = bc_t * n.z + (1.0f - bc_t) * c.z;
    const size_t o = (size_t)tj * p + ti;
    h[o] = (1.0f - alpha) * h[o] + alpha * eh;
    u[o] = (1.0f - alpha) * u[o] + alpha * eu;
    v[o] = (1.0f - alpha) * v[o] + alpha * ev;
}

// Linear between the outer edge and the inner edge of the sponge; the edges
// themselves keep their values.
__global__ void k_lin_ns(int row0, int bc_north, int bc_south, int nx, int ny, int sponge_north, int sponge_south, float* h,
                         float* u, float* v, int p) {
    const int ti = blockIdx.x * blockDim.x + threadIdx.x;
    const int tj = row0 + blockIdx.y * blockDim.y + threadIdx.y;   // a band of rows
    if (!(((bc_south == 4 && tj < sponge_south && tj > 0) ||
           (bc_north == 4 && tj > ny + 2 * kHalo - 1 - sponge_north && tj < ny + 2 * kHalo - 1)) &&
          (ti > 0) && (ti < nx + 2 * kHalo - 1)))
        return;
    int inner = sponge_south, outer = 0;
    if (tj > sponge_south) {
        inner = ny + 2 * kHalo - 1 - sponge_north;
        outer = ny + 2 * kHalo - 1;
    }
    const float ih = h[(size_t)inner * p + ti], iu = u[(size_t)inner * p + ti], iv = v[(size_t)inner * p + ti];
    const float oh = h[(size_t)outer * p + ti], ou = u[(size_t)outer * p + ti], ov = v[(size_t)outer * p + ti];
    const float ratio = ((float)(tj - outer)) / (inner - outer);
    const size_t o = (size_t)tj * p + ti;
    h[o] = oh + ratio * (ih - oh);
    u[o] = ou + ratio * (iu - ou);
    v[o] = ov + ratio * (iv - ov);
}

__global__ void k_lin_ew(int col0, int bc_east, int bc_west, int nx, int ny, int sponge_east, int sponge_west, float* h,
                         float* u, float* v, int p) {
    const int ti = col0 + blockIdx.x * blockDim.x + threadIdx.x;   // a band of columns
    const int tj = blockIdx.y * blockDim.y + threadIdx.y;
    if (!(((bc_west == 4 && ti < sponge_west && ti > 0) ||
           (bc_east == 4 && ti > nx + 2 * kHalo - 1 - sponge_east && ti < nx + 2 * kHalo - 1)) &&
          (tj > 0) && (tj < ny + 2 * kHalo - 1)))
        return;
    int inner = sponge_west, outer = 0;
    if (ti > sponge_west) {
        inner = nx + 2 * kHalo - 1 - sponge_east;
        outer = nx + 2 * kHalo - 1;
    }
    const size_t row = (size_t)tj * p;
    const float ih = h[row + inner], iu = u[row + inner], iv = v[row + inner];
    const float oh = h[row + outer], ou = u[row + outer], ov = v[row + outer];
    const float ratio = ((float)(ti - outer)) / (inner - outer);
    h[row + ti] = oh + ratio * (ih - oh);
    u[row + ti] = ou + ratio * (iu - ou);
    v[row + ti] = ov + ratio * (iv - ov);
}

}  // namespace

// The open kinds of one axis, after that axis's periodic copy would have
// run (go_boundary_condition calls this for the non-periodic axes).
int go_open_bc_ns(const go_domain* d, cudaStream_t s, float* h, float* u, float* v, int p) {
    const go::Scheme& k = d->k;
    if ((k.bcN == 3 || k.bcS == 3) && (!d->bc_tex[0] || !d->bc_tex[1]))
        return go_fail(GO_ERR_INVALID, "flow relaxation north/south needs its exterior textures "
                                       "(go_domain_set_open_bc)");
    // Only the sponge bands are launched: every thread of the reference's
    // full-grid launch outside them does nothing, and a thread's result
    // depends on its own cell and on rows no thread of the launch writes.
    const int rows = k.ny + 2 * kHalo;
    const int south_end = min(d->sponge[2] + 1, rows);
    const int bands[2][2] = {{0, south_end},                                          // south
                             {max(rows - 1 - d->sponge[0], south_end), rows}};        // north, disjoint
    const dim3 b(16, 16);
    for (const auto& band : bands) {
        const int n = band[1] - band[0];
        if (n <= 0) continue;
        const dim3 g((k.nx + 2 * kHalo + 15) / 16, (n + 15) / 16);
        if (k.bcN == 3 || k.bcS == 3)
            k_frs_ns<<<g, b, 0, s>>>(band[0], k.bcN, k.bcS, k.nx, k.ny, d->sponge[0], d->sponge[2], h, u, v, p,
                                     (cudaTextureObject_t)d->bc_tex[0], (cudaTextureObject_t)d->bc_tex[1], d->bc_t);
        if (k.bcN == 4 || k.bcS == 4)
            k_lin_ns<<<g, b, 0, s>>>(band[0], k.bcN, k.bcS, k.nx, k.ny, d->sponge[0], d->sponge[2], h, u, v, p);
    }
    GO_CUDA(cudaGetLastError());
    return GO_OK;
}

int go_open_bc_ew(const go_domain* d, cudaStream_t s, float* h, float* u, float* v, int p) {
    const go::Scheme& k = d->k;
    if ((k.bcE == 3 || k.bcW == 3) && (!d->bc_tex[2] || !d->bc_tex[3]))
        return go_fail(GO_ERR_INVALID, "flow relaxation east/west needs its exterior textures "
                                       "(go_domain_set_open_bc)");
    const int cols = k.nx + 2 * kHalo;
    const int west_end = min(d->sponge[3] + 1, cols);
    const int bands[2][2] = {{0, west_end},                                           // west
                             {max(cols - 1 - d->sponge[1], west_end), cols}};         // east, disjoint
    const dim3 b(16, 16);
    for (const auto& band : bands) {
        const int n = band[1] - band[0];
        if (n <= 0) continue;
        const dim3 g((n + 15) / 16, (k.ny + 2 * kHalo + 15) / 16);
        if (k.bcE == 3 || k.bcW == 3)
            k_frs_ew<<<g, b, 0, s>>>(band[0], k.bcE, k.bcW, k.nx, k.ny, d->sponge[1], d->sponge[3], h, u, v, p,
                                     (cudaTextureObject_t)d->bc_tex[2], (cudaTextureObject_t)d->bc_tex[3], d->bc_t);
        if (k.bcE == 4 || k.bcW == 4)
            k_lin_ew<<<g, b, 0, s>>>(band[0], k.bcE, k.bcW, k.nx, k.ny, d->sponge[1], d->sponge[3], h, u, v, p);
    }
    GO_CUDA(cudaGetLastError());
    return GO_OK;
}

extern "C" {

int go_bc_texture_create(const float* texels, int w, int h, uint64_t* texture) {
    if (!texels || !texture) return go_fail(GO_ERR_INVALID, "null argument");
    if (w < 1 || h < 1) return go_fail(GO_ERR_INVALID, "empty boundary data");
    *texture = 0;
    cudaChannelFormatDesc ch = cudaCreateChannelDesc<float4>();
    cudaArray_t arr = nullptr;
    GO_CUDA(cudaMallocArray(&arr, &ch, w, h));
    cudaError_t e = cudaMemcpy2DToArray(arr, 0, 0, texels, sizeof(float4) * w, sizeof(float4) * w, h,
                                        cudaMemcpyHostToDevice);
    cudaTextureObject_t tex = 0;
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
    if (e != cudaSuccess) {
        cudaFreeArray(arr);
        return go_fail(GO_ERR_CUDA, "boundary texture: %s", cudaGetErrorString(e));
    }
    *texture = (uint64_t)tex;
    return GO_OK;
}

int go_domain_set_sponge(go_domain* d, int north, int east, int south, int west) {
    if (!d) return go_fail(GO_ERR_INVALID, "null domain");
    if (north < 0 || east < 0 || south < 0 || west < 0)
        return go_fail(GO_ERR_INVALID, "sponge widths must be >= 0");
    if (north + south > d->k.ny + 4 || east + west > d->k.nx + 4)
        return go_fail(GO_ERR_INVALID, "sponges wider than the grid");
    d->sponge[0] = north; d->sponge[1] = east; d->sponge[2] = south; d->sponge[3] = west;
    return GO_OK;
}

int go_domain_set_open_bc(go_domain* d, const uint64_t* textures, float bc_t) {
    if (!d || !textures) return go_fail(GO_ERR_INVALID, "null argument");
    for (int i = 0; i < 4; ++i) d->bc_tex[i] = textures[i];
    d->bc_t = bc_t;
    return GO_OK;
}

}  // extern "C"
