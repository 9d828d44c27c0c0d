// Internal declarations shared by the translation units of libgocean.
#pragma once

#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "cdklm16_stage.cuh"
#include "gocean.h"

struct go_domain {
    go_domain_desc desc;
    go::Scheme k;
    int device;
    float* d_frows;          // ny+4 Coriolis values
    unsigned int* d_status;  // GO_STATUS_* bits
    float wxc, wxn, wyc, wyn;
    const float *wx_cur, *wx_next, *wy_cur, *wy_next;
    int wpitch;              // floats
    int rows_per_block;
    int shape;               // launch shape, see go_shape_width()
    int arith;               // GO_ARITH_*
    int has_land;            // bathymetry may hold land cells (checks on)
    int adj_kind;            // GO_ADJ_* launch form of the adjoint stage
    int adj_rows;            // rows per strip of the marching adjoint (0: automatic)
    int sponge[4];           // open-boundary sponge widths: north, east, south, west
    uint64_t bc_tex[4];      // exterior solution textures: NS cur, NS next, EW cur, EW next
    float bc_t;              // their time weight
    // column-pair launches: the boundary-frame kernel runs on a second
    // stream beside the boundary-free one (created on first use)
    cudaStream_t side;
    cudaEvent_t ev_fork, ev_join;
    int own_side;            // go_domain_create's handles may create them (not the allocation-free step)
    int stage_launches;      // kernel launches the last RK stage issued
    unsigned debug;          // GO_DEBUG_* test hooks
};

// Records the message of a failed call (go_last_error) and returns code.
int go_fail(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));

#define GO_CUDA(call)                                                                      \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return go_fail(GO_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));  \
    } while (0)

int go_check_pitch(int pitch_bytes, int min_floats, const char* what);

// Default rows per block strip for a grid and launch shape: the power of two
// in [2, 16] nearest below (column strips x ny) / 600, so that small grids
// still launch enough blocks to cover the 148 SMs.
int go_auto_rows(int nx, int ny, int shape);
int go_auto_shape(int nx, int ny);
// Open kinds (codes 3/4) of one axis (csrc/open_boundaries.cu).
int go_open_bc_ns(const go_domain* d, cudaStream_t s, float* h, float* u, float* v, int p);
int go_open_bc_ew(const go_domain* d, cudaStream_t s, float* h, float* u, float* v, int p);
inline bool go_has_open_bc(const go_domain* d) {
    return d->k.bcN > 2 || d->k.bcE > 2 || d->k.bcS > 2 || d->k.bcW > 2;
}

// Kernel-variant selectors of a domain.
int go_friction_mode(const go_domain* d);
bool go_general_north(const go_domain* d);

// Fills the per-stage arguments of one domain.
go::StageArgs go_stage_args(const go_domain* d, float dt, int rk_step, const float* e0, const float* u0,
                            const float* v0, int pin, float* e1, float* u1, float* v1, int pout,
                            const float* Hi, int phi, float land, float wind_t);

namespace go { struct Variant; }
// Kernel variant of a domain (stage_launch.cu).
go::Variant go_variant(const go_domain* d);

// One single-domain stage launch (stage_launch.cu).
int go_launch_stage(go_domain* d, cudaStream_t s, const go::StageArgs& a);

// Column-pair shape (pair_launch.cu).
bool go_pair_shape(int shape);
namespace go { struct PairMapParams; }
int go_prepare_pair(const go::StageArgs& a, go::PairMapParams* mp, bool* tma);
int go_launch_pair(go_domain* d, cudaStream_t s, const go::StageArgs& a, const go::PairMapParams& mp, bool tma);

// A stage launch prepared once (kernel arguments, TMA maps) and launched
// many times (stage_launch.cu).
struct PreparedStage;
int go_prepare_stage(go_domain* d, const go::StageArgs& a, PreparedStage* p);
int go_launch_prepared(go_domain* d, cudaStream_t s, const PreparedStage& p);
