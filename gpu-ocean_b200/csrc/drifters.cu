// Lagrangian drifters and flow observation at drifter cells.
//
// Restates the reference's passive drifter advection, its periodic wrap and
// its observation operator:
//   gpu_ocean/SWESimulators/gpu_kernels/driftKernels.cu:108-207  (passiveDrifterKernel)
//   gpu_ocean/SWESimulators/gpu_kernels/driftKernels.cu:211-250  (enforceBoundaryConditions)
//   gpu_ocean/SWESimulators/gpu_kernels/observationKernels.cu:29-81 (observeUnderlyingFlow)
// The reference builds these kernels with nvcc's default options
// (GPUDrifterCollection.py:81-83 passes no compile flags), so this unit is
// built the same way (IEEE division and square root, FMA contraction on,
// no flush to zero; build.py UNIT_FLAGS) and writes each expression with the
// reference's operand order, so the contractions and roundings agree.
//
// Positions: (n + 1) rows of (x, y) floats in metres from the south-west
// interior corner, pitch in bytes; the last row is the observation's
// position, which drifts with the drifters as in the reference.
#include "internal.h"

namespace {

// Water velocity component q / (Hm + eta) at ghost-inclusive cell (i, j)
// (driftKernels.cu:62-100).
__device__ __forceinline__ float cell_velocity(const float* __restrict__ q, int pq, const float* __restrict__ eta,
                                               int pe, const float* __restrict__ Hm, int ph, int i, int j) {
    const float h = Hm[(size_t)j * ph + i] + eta[(size_t)j * pe + i];
    return q[(size_t)j * pq + i] / h;
}

// Wind at a drifter position: normalised texture coordinates over the
// domain, bilinear lookup of current and next, linear in time
// (driftKernels.cu:38-60).
__device__ __forceinline__ float wind_at(cudaTextureObject_t cur, cudaTextureObject_t next, float wind_t,
                                         float x, float y, float size_x, float size_y) {
    const float s = x / size_x;
    const float t = y / size_y;
    const float c = tex2D<float>(cur, s, t);
    const float n = tex2D<float>(next, s, t);
    return wind_t * n + (1.0f - wind_t) * c;
}

__device__ __forceinline__ int clamp_index(int i, int hi) { return min(max(i, 0), hi); }

struct DriftArgs {
    int nx, ny;
    float dx, dy, dt;
    int x0, y0;                       // ghost-inclusive cell of the origin
    const float *eta, *hu, *hv, *Hm;
    int pe, pu, pv, ph;               // pitches, floats
    int periodic_ns, periodic_ew;
    int n;                            // drifters (the observation row is row n)
    float* pos;
    int pp;                           // pitch, floats
    float sensitivity, wind_t, wind_factor;
    cudaTextureObject_t wxc, wxn, wyc, wyn;
};

__global__ void k_drift(const DriftArgs a) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= a.n + 1) return;
    float* p = a.pos + (size_t)d * a.pp;
    float x = p[0], y = p[1];

    // the cell holding the drifter, then the four cell centres around it
    const int ci = (int)(ceil(x / a.dx) + a.x0);
    const int cj = (int)(ceil(y / a.dy) + a.y0);
    const float fx = x / a.dx - floor(x / a.dx);
    const float fy = y / a.dy - floor(y / a.dy);
    const float wx = fx < 0.5f ? fx + 0.5f : fx - 0.5f;
    const float wy = fy < 0.5f ? fy + 0.5f : fy - 0.5f;
    // Cells clamped to the ghost-inclusive array.  A drifter inside the
    // domain (0 <= x <= nx dx, 0 <= y <= ny dy) never meets the clamp; the
    // reference reads outside its arrays for one that left a walled domain.
    const int i0 = clamp_index(fx < 0.5f ? ci - 1 : ci, a.nx + 3);
    const int i1 = clamp_index((fx < 0.5f ? ci - 1 : ci) + 1, a.nx + 3);
    const int j0 = clamp_index(fy < 0.5f ? cj - 1 : cj, a.ny + 3);
    const int j1 = clamp_index((fy < 0.5f ? cj - 1 : cj) + 1, a.ny + 3);

    const float u00 = cell_velocity(a.hu, a.pu, a.eta, a.pe, a.Hm, a.ph, i0, j0);
    const float u10 = cell_velocity(a.hu, a.pu, a.eta, a.pe, a.Hm, a.ph, i1, j0);
    const float u01 = cell_velocity(a.hu, a.pu, a.eta, a.pe, a.Hm, a.ph, i0, j1);
    const float u11 = cell_velocity(a.hu, a.pu, a.eta, a.pe, a.Hm, a.ph, i1, j1);
    const float v00 = cell_velocity(a.hv, a.pv, a.eta, a.pe, a.Hm, a.ph, i0, j0);
    const float v10 = cell_velocity(a.hv, a.pv, a.eta, a.pe, a.Hm, a.ph, i1, j0);
    const float v01 = cell_velocity(a.hv, a.pv, a.eta, a.pe, a.Hm, a.ph, i0, j1);
    const float v11 = cell_velocity(a.hv, a.pv, a.eta, a.pe, a.Hm, a.ph, i1, j1);

    const float uy0 = (1 - wx) * u00 + wx * u10;
    const float uy1 = (1 - wx) * u01 + wx * u11;
    const float vy0 = (1 - wx) * v00 + wx * v10;
    const float vy1 = (1 - wx) * v01 + wx * v11;
    float u = (1 - wy) * uy0 + wy * uy1;
    float v = (1 - wy) * vy0 + wy * vy1;

    if (a.wind_factor) {
        const float size_x = a.nx * a.dx, size_y = a.ny * a.dy;
        u = u + wind_at(a.wxc, a.wxn, a.wind_t, x, y, size_x, size_y) * a.wind_factor;
        v = v + wind_at(a.wyc, a.wyn, a.wind_t, x, y, size_x, size_y) * a.wind_factor;
    }

    x += a.sensitivity * u * a.dt;
    y += a.sensitivity * v * a.dt;

    if (a.periodic_ew && (x < 0)) x += a.nx * a.dx;
    if (a.periodic_ew && (x > a.nx * a.dx)) x -= a.nx * a.dx;
    if (a.periodic_ns && (y < 0)) y += a.ny * a.dy;
    if (a.periodic_ns && (y > a.ny * a.dy)) y -= a.ny * a.dy;
    p[0] = x;
    p[1] = y;
}

__global__ void k_drift_wrap(float size_x, float size_y, int periodic_ns, int periodic_ew, int n, float* pos,
                             int pp) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n + 1) return;
    float* p = pos + (size_t)d * pp;
    float x = p[0], y = p[1];
    if (periodic_ew && (x < 0)) x += size_x;
    if (periodic_ew && (x > size_x)) x -= size_x;
    if (periodic_ns && (y < 0)) y += size_y;
    if (periodic_ns && (y > size_y)) y -= size_y;
    p[0] = x;
    p[1] = y;
}

// (hu, hv) of the cell under each drifter (observationKernels.cu:29-81).
__global__ void k_observe(int nx, int ny, float dx, float dy, int x0, int y0, const float* __restrict__ hu,
                          int pu, const float* __restrict__ hv, int pv, int n, const float* __restrict__ pos,
                          int pp, float* __restrict__ out, int po) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    const float* p = pos + (size_t)d * pp;
    const int i = clamp_index((int)(floor(p[0] / dx) + x0), nx + 3);    // clamp as in k_drift
    const int j = clamp_index((int)(floor(p[1] / dy) + y0), ny + 3);
    float* o = out + (size_t)d * po;
    o[0] = hu[(size_t)j * pu + i];
    o[1] = hv[(size_t)j * pv + i];
}

constexpr int kDriftBlock = 64;     // GPUDrifterCollection block_width

}  // namespace

extern "C" {

int go_wind_texture_create(const float* field, int w, int h, uint64_t* texture) {
    if (!field || !texture) return go_fail(GO_ERR_INVALID, "null argument");
    if (w < 1 || h < 1) return go_fail(GO_ERR_INVALID, "empty wind field");
    *texture = 0;
    cudaChannelFormatDesc ch = cudaCreateChannelDesc<float>();
    cudaArray_t arr = nullptr;
    GO_CUDA(cudaMallocArray(&arr, &ch, w, h));
    cudaError_t e = cudaMemcpy2DToArray(arr, 0, 0, field, sizeof(float) * w, sizeof(float) * w, h,
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
        return go_fail(GO_ERR_CUDA, "wind texture: %s", cudaGetErrorString(e));
    }
    *texture = (uint64_t)tex;
    return GO_OK;
}

int go_wind_texture_destroy(uint64_t texture) {
    if (!texture) return GO_OK;
    cudaResourceDesc res;
    cudaError_t e = cudaGetTextureObjectResourceDesc(&res, (cudaTextureObject_t)texture);
    if (e == cudaSuccess) e = cudaDestroyTextureObject((cudaTextureObject_t)texture);
    if (e == cudaSuccess && res.resType == cudaResourceTypeArray) e = cudaFreeArray(res.res.array.array);
    if (e != cudaSuccess) return go_fail(GO_ERR_CUDA, "wind texture: %s", cudaGetErrorString(e));
    return GO_OK;
}

int go_drift_passive(void* stream, int nx, int ny, float dx, float dy, float dt, int x_zero_cell,
                     int y_zero_cell, const float* eta, int eta_pitch, const float* hu, int hu_pitch,
                     const float* hv, int hv_pitch, const float* Hm, int Hm_pitch, int periodic_north_south,
                     int periodic_east_west, int num_drifters, float* positions, int positions_pitch,
                     float sensitivity, float wind_t, float wind_drift_factor, const uint64_t* wind_textures) {
    if (!eta || !hu || !hv || !Hm || !positions) return go_fail(GO_ERR_INVALID, "null argument");
    if (num_drifters < 0) return go_fail(GO_ERR_INVALID, "num_drifters < 0");
    if (wind_drift_factor != 0.0f && !wind_textures)
        return go_fail(GO_ERR_INVALID, "a wind drift factor needs the four wind textures");
    int rc = go_check_pitch(eta_pitch, nx + 4, "eta");
    if (!rc) rc = go_check_pitch(hu_pitch, nx + 4, "hu");
    if (!rc) rc = go_check_pitch(hv_pitch, nx + 4, "hv");
    if (!rc) rc = go_check_pitch(Hm_pitch, nx + 4, "Hm");
    if (!rc) rc = go_check_pitch(positions_pitch, 2, "positions");
    if (rc) return rc;
    DriftArgs a;
    a.nx = nx; a.ny = ny; a.dx = dx; a.dy = dy; a.dt = dt; a.x0 = x_zero_cell; a.y0 = y_zero_cell;
    a.eta = eta; a.hu = hu; a.hv = hv; a.Hm = Hm;
    a.pe = eta_pitch / 4; a.pu = hu_pitch / 4; a.pv = hv_pitch / 4; a.ph = Hm_pitch / 4;
    a.periodic_ns = periodic_north_south; a.periodic_ew = periodic_east_west;
    a.n = num_drifters; a.pos = positions; a.pp = positions_pitch / 4;
    a.sensitivity = sensitivity; a.wind_t = wind_t; a.wind_factor = wind_drift_factor;
    a.wxc = wind_textures ? wind_textures[0] : 0; a.wxn = wind_textures ? wind_textures[1] : 0;
    a.wyc = wind_textures ? wind_textures[2] : 0; a.wyn = wind_textures ? wind_textures[3] : 0;
    k_drift<<<(num_drifters + 1 + kDriftBlock - 1) / kDriftBlock, kDriftBlock, 0, (cudaStream_t)stream>>>(a);
    GO_CUDA(cudaGetLastError());
    return GO_OK;
}

int go_drift_enforce_bc(void* stream, float domain_size_x, float domain_size_y, int periodic_north_south,
                        int periodic_east_west, int num_drifters, float* positions, int positions_pitch) {
    if (!positions) return go_fail(GO_ERR_INVALID, "null argument");
    int rc = go_check_pitch(positions_pitch, 2, "positions");
    if (rc) return rc;
    if (num_drifters < 0) return go_fail(GO_ERR_INVALID, "num_drifters < 0");
    k_drift_wrap<<<(num_drifters + 1 + kDriftBlock - 1) / kDriftBlock, kDriftBlock, 0, (cudaStream_t)stream>>>(
        domain_size_x, domain_size_y, periodic_north_south, periodic_east_west, num_drifters, positions,
        positions_pitch / 4);
    GO_CUDA(cudaGetLastError());
    return GO_OK;
}

int go_observe_flow(void* stream, int nx, int ny, float dx, float dy, int x_zero_cell, int y_zero_cell,
                    const float* hu, int hu_pitch, const float* hv, int hv_pitch, int num_drifters,
                    const float* positions, int positions_pitch, float* observation, int observation_pitch) {
    if (!hu || !hv || !positions || !observation) return go_fail(GO_ERR_INVALID, "null argument");
    int rc = go_check_pitch(hu_pitch, nx + 4, "hu");
    if (!rc) rc = go_check_pitch(hv_pitch, nx + 4, "hv");
    if (!rc) rc = go_check_pitch(positions_pitch, 2, "positions");
    if (!rc) rc = go_check_pitch(observation_pitch, 2, "observation");
    if (rc) return rc;
    if (num_drifters < 0) return go_fail(GO_ERR_INVALID, "num_drifters < 0");
    if (num_drifters == 0) return GO_OK;
    k_observe<<<(num_drifters + kDriftBlock - 1) / kDriftBlock, kDriftBlock, 0, (cudaStream_t)stream>>>(
        nx, ny, dx, dy, x_zero_cell, y_zero_cell, hu, hu_pitch / 4, hv, hv_pitch / 4, num_drifters, positions,
        positions_pitch / 4, observation, observation_pitch / 4);
    GO_CUDA(cudaGetLastError());
    return GO_OK;
}

}  // extern "C"
