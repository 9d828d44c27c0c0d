// Host driver for the reference's own CDKLM16 kernels (test oracle only).
//
// Replays what gpu_ocean/SWESimulators/CDKLM16.py does around the kernels:
// texture set-up (CDKLM16.py:288-351, Simulator.py:145-223: LINEAR filter,
// CLAMP addressing, normalized coordinates), bathymetry (Common.py:1319-1389)
// and the RK2 launch order of step() (CDKLM16.py:533-544, 585-586).  One
// library is built per compile-time configuration (NX, NY, DX, DY, GRAV,
// FRIC), as the reference JIT-compiles one module per configuration.
#include <cuda_runtime.h>
#include <string.h>

extern "C" int refb_set_open_bc_tex(cudaTextureObject_t, cudaTextureObject_t, cudaTextureObject_t,
                                    cudaTextureObject_t);
extern "C" int refb_boundary(cudaStream_t, int, int, int, int, int, int, int, int, int, int, float, float*, int,
                             float*, int, float*, int);
extern "C" int refr_set_drift_wind(cudaTextureObject_t, cudaTextureObject_t, cudaTextureObject_t,
                                   cudaTextureObject_t);
extern "C" int refn_set_textures(cudaTextureObject_t, cudaTextureObject_t);
extern "C" int refk_set_textures(cudaTextureObject_t, cudaTextureObject_t, cudaTextureObject_t,
                                 cudaTextureObject_t, cudaTextureObject_t, cudaTextureObject_t);
extern "C" int refk_cdklm_swe_2D(cudaStream_t, float, int, float*, int, float*, int, float*, int, float*,
                                 int, float*, int, float*, int, float*, int, float*, int, float, float, int);
extern "C" int refb_periodic(cudaStream_t, int, int, int, int, float*, int, float*, int, float*, int);
extern "C" int refb_bathymetry(cudaStream_t, int, int, int, int, float*, int, float, float*, int);
extern "C" int refd_max_dt(cudaStream_t, int, int, float, float, float, float*, int, float*, int, float*, int,
                           float*, int, float, float*, float*);

namespace {

struct Tex {
    cudaArray_t arr = nullptr;
    cudaTextureObject_t obj = 0;
};

Tex g_angle, g_f, g_wxc, g_wxn, g_wyc, g_wyn;
Tex g_dwxc, g_dwxn, g_dwyc, g_dwyn;     // wind of the drift kernel
Tex g_ns0, g_ns1, g_ew0, g_ew1;         // exterior solution of the flow relaxation
Tex g_nangle, g_nf;                     // angle and Coriolis textures of the model-error kernels


void release(Tex& t) {
    if (t.obj) cudaDestroyTextureObject(t.obj);
    if (t.arr) cudaFreeArray(t.arr);
    t = Tex();
}

int make_tex(Tex& t, const float* host, int w, int h) {
    release(t);
    cudaChannelFormatDesc ch = cudaCreateChannelDesc<float>();
    cudaError_t e = cudaMallocArray(&t.arr, &ch, w, h);
    if (e) return (int)e;
    e = cudaMemcpy2DToArray(t.arr, 0, 0, host, w * sizeof(float), w * sizeof(float), h, cudaMemcpyHostToDevice);
    if (e) return (int)e;
    cudaResourceDesc res;
    memset(&res, 0, sizeof(res));
    res.resType = cudaResourceTypeArray;
    res.res.array.array = t.arr;
    cudaTextureDesc td;
    memset(&td, 0, sizeof(td));
    td.addressMode[0] = cudaAddressModeClamp;
    td.addressMode[1] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 1;
    return (int)cudaCreateTextureObject(&t.obj, &res, &td, nullptr);
}

struct OpenBC {
    int active = 0;
    int codes[4] = {1, 1, 1, 1};        // north, east, south, west
    int sponge[4] = {0, 0, 0, 0};
    float bc_t = 0.0f;
} g_open;

int make_tex4(Tex& t, const float* host, int w, int h) {
    release(t);
    cudaChannelFormatDesc ch = cudaCreateChannelDesc<float4>();
    cudaError_t e = cudaMallocArray(&t.arr, &ch, w, h);
    if (e) return (int)e;
    e = cudaMemcpy2DToArray(t.arr, 0, 0, host, w * sizeof(float4), w * sizeof(float4), h, cudaMemcpyHostToDevice);
    if (e) return (int)e;
    cudaResourceDesc res;
    memset(&res, 0, sizeof(res));
    res.resType = cudaResourceTypeArray;
    res.res.array.array = t.arr;
    cudaTextureDesc td;
    memset(&td, 0, sizeof(td));
    td.addressMode[0] = cudaAddressModeClamp;
    td.addressMode[1] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 1;
    return (int)cudaCreateTextureObject(&t.obj, &res, &td, nullptr);
}

}  // namespace

extern "C" {

// Compile-time configuration of this library.
int ref_config(int* nx, int* ny, float* dx, float* dy, float* g, float* r) {
    *nx = NX; *ny = NY; *dx = DX; *dy = DY; *g = GRAV; *r = FRIC;
    return 0;
}

// Textures: f (fw x fh, 1x1 for an f-plane, (NX+4)x(NY+4) for beta), a
// constant angle, uniform wind current/next.
int ref_setup(const float* f_host, int fw, int fh, float angle, float wxc, float wxn, float wyc, float wyn) {
    int e = make_tex(g_f, f_host, fw, fh);
    if (!e) e = make_tex(g_angle, &angle, 1, 1);
    if (!e) e = make_tex(g_wxc, &wxc, 1, 1);
    if (!e) e = make_tex(g_wxn, &wxn, 1, 1);
    if (!e) e = make_tex(g_wyc, &wyc, 1, 1);
    if (!e) e = make_tex(g_wyn, &wyn, 1, 1);
    if (!e) e = refk_set_textures(g_angle.obj, g_f.obj, g_wxc.obj, g_wxn.obj, g_wyc.obj, g_wyn.obj);
    return e;
}

// Non-uniform wind: current/next X and Y arrays (host, h x w each) bound as
// the wind textures (Simulator.py:171-213 setTexture).
int ref_set_wind(const float* xc, const float* xn, const float* yc, const float* yn, int w, int h) {
    int e = make_tex(g_wxc, xc, w, h);
    if (!e) e = make_tex(g_wxn, xn, w, h);
    if (!e) e = make_tex(g_wyc, yc, w, h);
    if (!e) e = make_tex(g_wyn, yn, w, h);
    if (!e) e = refk_set_textures(g_angle.obj, g_f.obj, g_wxc.obj, g_wxn.obj, g_wyc.obj, g_wyn.obj);
    return e;
}

// Wind textures of the drift kernel (GPUDrifterCollection.py:120-176).
int ref_set_drift_wind(const float* xc, const float* xn, const float* yc, const float* yn, int w, int h) {
    int e = make_tex(g_dwxc, xc, w, h);
    if (!e) e = make_tex(g_dwxn, xn, w, h);
    if (!e) e = make_tex(g_dwyc, yc, w, h);
    if (!e) e = make_tex(g_dwyn, yn, w, h);
    if (!e) e = refr_set_drift_wind(g_dwxc.obj, g_dwxn.obj, g_dwyc.obj, g_dwyn.obj);
    return e;
}

// Angle and Coriolis textures of the model-error kernels
// (OceanStateNoise.py:284-320), host arrays of h rows x w columns.
int ref_noise_textures(const float* angle, int aw, int ah, const float* coriolis, int cw, int ch) {
    int e = make_tex(g_nangle, angle, aw, ah);
    if (!e) e = make_tex(g_nf, coriolis, cw, ch);
    if (!e) e = refn_set_textures(g_nangle.obj, g_nf.obj);
    return e;
}

int ref_bathymetry(void* s, int bc_north, int bc_east, float* Bi, int pbi, float land, float* Bm, int pbm) {
    return refb_bathymetry((cudaStream_t)s, NX, NY, bc_north == 2, bc_east == 2, Bi, pbi, land, Bm, pbm);
}

int ref_boundary(void* s, int bc_north, int bc_east, float* h, float* u, float* v, int p) {
    if (g_open.active)
        return refb_boundary((cudaStream_t)s, NX, NY, g_open.codes[0], g_open.codes[1], g_open.codes[2],
                             g_open.codes[3], g_open.sponge[0], g_open.sponge[1], g_open.sponge[2], g_open.sponge[3],
                             g_open.bc_t, h, p, u, p, v, p);
    return refb_periodic((cudaStream_t)s, NX, NY, bc_north == 2, bc_east == 2, h, p, u, p, v, p);
}

// Open boundaries for ref_boundary / ref_step: codes and sponge widths
// (north, east, south, west), exterior textures (NS: w_ns x 2 float4 texels,
// EW: 2 x h_ew) of the current and next time, and the time weight.
int ref_set_open_bc(const int* codes, const int* sponge, const float* ns0, const float* ns1, int w_ns,
                    const float* ew0, const float* ew1, int h_ew, float bc_t) {
    for (int i = 0; i < 4; ++i) { g_open.codes[i] = codes[i]; g_open.sponge[i] = sponge[i]; }
    g_open.bc_t = bc_t;
    g_open.active = 1;
    int e = make_tex4(g_ns0, ns0, w_ns, 2);
    if (!e) e = make_tex4(g_ns1, ns1, w_ns, 2);
    if (!e) e = make_tex4(g_ew0, ew0, 2, h_ew);
    if (!e) e = make_tex4(g_ew1, ew1, 2, h_ew);
    if (!e) e = refb_set_open_bc_tex(g_ns0.obj, g_ns1.obj, g_ew0.obj, g_ew1.obj);
    return e;
}

int ref_set_bc_t(float bc_t) {
    g_open.bc_t = bc_t;
    return 0;
}

int ref_stage(void* s, float dt, int rk_step, float* e0, float* u0, float* v0, int p0,
              float* e1, float* u1, float* v1, int p1, float* Hi, int phi, float* Hm, int phm,
              float land, float wind_t, int bc_packed) {
    return refk_cdklm_swe_2D((cudaStream_t)s, dt, rk_step, e0, p0, u0, p0, v0, p0, e1, p1, u1, p1, v1, p1,
                             Hi, phi, Hm, phm, land, wind_t, bc_packed);
}

// n RK2 steps in the order of CDKLM16.step (CDKLM16.py:535-544, 585-586).
int ref_step(void* s, int n, float dt, float wind_t, float* e0, float* u0, float* v0, int p0,
             float* e1, float* u1, float* v1, int p1, float* Hi, int phi, float* Hm, int phm,
             float land, int bc_packed) {
    const int north = (bc_packed >> 24) & 0xff, east = (bc_packed >> 8) & 0xff;
    for (int i = 0; i < n; ++i) {
        int e = ref_stage(s, dt, 0, e0, u0, v0, p0, e1, u1, v1, p1, Hi, phi, Hm, phm, land, wind_t, bc_packed);
        if (!e) e = ref_boundary(s, north, east, e1, u1, v1, p1);
        if (!e) e = ref_stage(s, dt, 1, e1, u1, v1, p1, e0, u0, v0, p0, Hi, phi, Hm, phm, land, wind_t, bc_packed);
        if (!e) e = ref_boundary(s, north, east, e0, u0, v0, p0);
        if (e) return e;
    }
    return 0;
}

int ref_max_dt(void* s, float* e, float* u, float* v, int p, float* Hm, int phm, float land,
               float* dt_blocks, float* dt_out) {
    return refd_max_dt((cudaStream_t)s, NX, NY, DX, DY, GRAV, e, p, u, p, v, p, Hm, phm, land, dt_blocks, dt_out);
}

}  // extern "C"
