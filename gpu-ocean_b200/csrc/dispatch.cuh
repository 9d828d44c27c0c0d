// Kernel-variant selection shared by the single-domain and batched launchers.
//
// A variant is (launch shape, friction law, general grid angle, per-cell
// wind, reciprocal quotients, land in the bathymetry).  Shapes 5, 6 and 7
// (128 x 5, 96 x 6 and 192 x 3 blocks) read ahead through the ring.  Every variant gives
// the same results; the specialised ones drop work the general one would do
// for nothing.  Instantiated set:
//   * general: shape 4, every friction law, angle and wind combination, land
//     checks on, reciprocal quotients;
//   * common fast path (north up, uniform wind): every shape and friction
//     law, with and without land checks, reciprocal or '/' quotients.
#pragma once

#include "internal.h"

namespace go {

struct Variant {
    int shape, fric;
    bool gen_north, wind_field, rcp, land;
};

// L is a functor with
//   template <int BW, int MINB, int FRIC, bool GN, bool WF, bool RCP, bool LAND, int D> cudaError_t run();
// (D: rows read ahead through the shared-memory ring, 0 = register prefetch)
template <class L>
cudaError_t dispatch_variant(L& launcher, Variant v) {
#define GO_VD(BW, MINB, F, GN, WF, RCP, LAND, D) return launcher.template run<BW, MINB, F, GN, WF, RCP, LAND, D>()
#define GO_V(BW, MINB, F, GN, WF, RCP, LAND) GO_VD(BW, MINB, F, GN, WF, RCP, LAND, 0)
    if (v.gen_north || v.wind_field) {
        // general variants: 128 x 5 blocks, reciprocal quotients; a rotated
        // grid keeps the land checks on; the per-cell wind field of a
        // north-up grid also has the read-ahead form (shapes 5-7) and a form
        // without land checks
#define GO_GEN(F)                                                     \
    do {                                                              \
        if (v.gen_north && v.wind_field) GO_V(128, 5, F, true, true, true, true);   \
        if (v.gen_north) GO_V(128, 5, F, true, false, true, true);    \
        if (v.shape >= 5) {                                           \
            if (v.land) GO_VD(128, 5, F, false, true, true, true, kReadAhead);   \
            GO_VD(128, 5, F, false, true, true, false, kReadAhead);   \
        }                                                             \
        if (v.land) GO_V(128, 5, F, false, true, true, true);         \
        GO_V(128, 5, F, false, true, true, false);                    \
    } while (0)
        if (v.fric == kFricNone) GO_GEN(kFricNone);
        if (v.fric == kFricQuad) GO_GEN(kFricQuad);
        GO_GEN(kFricLinear);
#undef GO_GEN
    }
#define GO_SHAPES(F, RCP, LAND)                                       \
    do {                                                              \
        switch (v.shape) {                                            \
            case 0: GO_V(192, 2, F, false, false, RCP, LAND);         \
            case 1: GO_V(192, 3, F, false, false, RCP, LAND);         \
            case 2: GO_V(128, 4, F, false, false, RCP, LAND);         \
            case 3: GO_V(256, 2, F, false, false, RCP, LAND);         \
            case 5: GO_VD(128, 5, F, false, false, RCP, LAND, kReadAhead); \
            case 6: GO_VD(96, 6, F, false, false, RCP, LAND, kReadAhead); \
            case 7: GO_VD(192, 3, F, false, false, RCP, LAND, kReadAhead); \
            default: GO_V(128, 5, F, false, false, RCP, LAND);        \
        }                                                             \
    } while (0)
#define GO_RL(F)                                                      \
    do {                                                              \
        if (v.rcp) {                                                  \
            if (v.land) GO_SHAPES(F, true, true);                     \
            GO_SHAPES(F, true, false);                                \
        }                                                             \
        if (v.land) GO_V(128, 5, F, false, false, false, true);       \
        GO_V(128, 5, F, false, false, false, false);                  \
    } while (0)
    if (v.fric == kFricNone) GO_RL(kFricNone);
    if (v.fric == kFricQuad) GO_RL(kFricQuad);
    GO_RL(kFricLinear);
#undef GO_RL
#undef GO_SHAPES
#undef GO_V
#undef GO_VD
}

inline int shape_block_width(int shape) {
    switch (shape) {
        case GO_SHAPE_PAIR: return 128;     // columns per block: two per thread
        case 2: case 4: case 5: return 128;
        case 3: return 256;
        case 6: return 96;
        default: return 192;
    }
}

// Block width of the kernel dispatch_variant launches for v: the general
// variants and '/' quotients run 128-wide blocks whatever v.shape says.
inline int dispatch_width(const Variant& v) {
    if (v.gen_north || v.wind_field || !v.rcp) return 128;
    return shape_block_width(v.shape);
}

// Columns a shape computes for an nx-wide grid (strips x block width).
inline long long shape_columns(int shape, int nx) {
    const int w = shape_block_width(shape);
    return (long long)((nx + w - 5) / (w - 4)) * w;
}

// The read-ahead shape for grids whose column work (sum over grids of
// shape_columns x ny) is work5 with 128-wide and work6 with 96-wide blocks:
// 96-wide blocks cost ~4% more per column (measured on a B200: 4096^2 686 vs
// 710 us per step), so shape 6 only when it computes at least 4% fewer
// columns (a 512-wide member: 576 columns against 640).
inline int ring_shape(long long work5, long long work6) { return work6 * 100 < work5 * 96 ? 6 : 5; }

// Resident blocks per SM the shape is compiled for (its __launch_bounds__).
inline int shape_blocks_per_sm(int shape) {
    switch (shape) {
        case GO_SHAPE_PAIR: return 8;
        case 0: case 3: return 2;
        case 1: case 7: return 3;
        case 2: return 4;
        case 6: return 6;
        default: return 5;
    }
}

}  // namespace go
