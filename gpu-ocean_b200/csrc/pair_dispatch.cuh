// Launch configuration and variant dispatch of the column-pair stage kernel
// (cdklm16_pair.cuh), shared by the single-domain and batched launchers.
#pragma once

#include <algorithm>

#include "cdklm16_pair.cuh"
#include "dispatch.cuh"

namespace go {

// 64 threads (128 columns) per block.  The boundary-free kernel is held to
// 128 registers (8 blocks, 16 warps per SM; it needs no spills there) and
// reads its inputs through a ring of 2 chunks of 3 rows; the boundary-frame
// kernel gets 168 registers and strips of 8 rows.  Measured on a B200 at
// 4096^2 (us per RK2 step): 2 ring slots against 3 (3 slots leave room for
// fewer blocks); one row per loop iteration 583 against 729 for two (the
// 2-row loop spills 64 bytes) and against a 3-row unroll whose code thrashes
// the instruction cache (41% issue activity against 59%).
constexpr int kPairT = 64;
constexpr int kPairMinBlocksInterior = 8;
constexpr int kPairMinBlocksFrame = 6;
constexpr int kPairSlots = 2;
constexpr int kPairUnroll = 1;
constexpr int kPairFrameRows = 8;
// default-shape thresholds: a grid of at least this many cells, a batch
// whose members hold at least this many together
constexpr long long kPairAutoCells = 1500LL * 1500LL;
constexpr long long kPairAutoBatchCells = 2LL << 20;

// The block grid of an nx x ny domain (see PairGrid): the region of TMA
// strips of `rows` rows, empty when `tma` is false (every block then takes
// the boundary path), and the frame.
inline PairGrid pair_grid(const Scheme& k, int rows, bool tma) {
    constexpr int T = kPairT;
    PairGrid g;
    g.nbx = (k.nx + (2 * T - 4) - 1) / (2 * T - 4);
    g.rows = rows;
    g.ny = k.ny;
    g.rf = kPairFrameRows;
    g.bx0 = g.bx1 = 0;
    g.nby = 0;
    if (!tma || k.ny <= 4) return g;
    int lo = -1, hi = -1;
    for (int bx = 0; bx < g.nbx; ++bx) {
        if (pair_fast_cols<T>(k, bx * (2 * T - 4))) { if (lo < 0) lo = bx; hi = bx + 1; }
    }
    if (lo < 0) return g;
    g.bx0 = lo;
    g.bx1 = hi;
    g.nby = (k.ny - 4 + rows - 1) / rows;
    return g;
}

inline int pair_frame_count(const PairGrid& g) {
    int nfull, full, nband;
    return pair_frame_strips(g, nfull, full, nband);
}

// Kernel variants.  The boundary-free kernels are compiled per friction law
// (one unit each) and per (wind field, grid angle, quotient mode, land
// checks): L::run<WIND, GN, RCP, LAND>().  Rotated grids run with
// reciprocal quotients and land checks.
template <class L>
cudaError_t dispatch_pair_variant(L& l, const Variant& v) {
    if (v.gen_north) {
        if (v.wind_field) return l.template run<1, true, true, true>();
        return l.template run<0, true, true, true>();
    }
    if (v.wind_field) {
        if (v.land) return l.template run<1, false, true, true>();
        return l.template run<1, false, true, false>();
    }
    if (v.rcp) {
        if (v.land) return l.template run<0, false, true, true>();
        return l.template run<0, false, true, false>();
    }
    if (v.land) return l.template run<0, false, false, true>();
    return l.template run<0, false, false, false>();
}

// The boundary-frame kernels read the friction law and the wind kind at run
// time: L::run<GN, RCP, LAND>().
template <class L>
cudaError_t dispatch_pair_frame_variant(L& l, const Variant& v) {
    if (v.gen_north) return l.template run<true, true, true>();
    if (v.rcp) {
        if (v.land) return l.template run<false, true, true>();
        return l.template run<false, true, false>();
    }
    if (v.land) return l.template run<false, false, true>();
    return l.template run<false, false, false>();
}

// One single-domain stage: the two parts (pair_single_*.cu).
struct PairSingleReq {
    const StageArgs* a;
    const PairMapParams* mp;
    PairGrid g;
    cudaStream_t s;
};
cudaError_t pair_launch_interior(const PairSingleReq& r, const Variant& v);   // by v.fric
cudaError_t pair_launch_interior_f0(const PairSingleReq& r, const Variant& v);
cudaError_t pair_launch_interior_f1(const PairSingleReq& r, const Variant& v);
cudaError_t pair_launch_interior_f2(const PairSingleReq& r, const Variant& v);
cudaError_t pair_launch_frame(const PairSingleReq& r, const Variant& v);


// One batched stage: the two tile lists (pair_batch_*.cu).
struct PairBatchReq {
    const StageArgs* args;
    const float* dts;
    const int4* tiles;
    int ntiles;
    int grid;
    int rk_step;
    const PairMapParams* maps;
    cudaStream_t s;
};
cudaError_t pair_batch_launch_interior(const PairBatchReq& r, const Variant& v);   // by v.fric
cudaError_t pair_batch_launch_interior_f0(const PairBatchReq& r, const Variant& v);
cudaError_t pair_batch_launch_interior_f1(const PairBatchReq& r, const Variant& v);
cudaError_t pair_batch_launch_interior_f2(const PairBatchReq& r, const Variant& v);
cudaError_t pair_batch_launch_frame(const PairBatchReq& r, const Variant& v);

// Periodic east/west ghost columns of rows [2, ny+2) of a stage's output,
// for one domain (args null: `one`) or n batch members (args[2 m + rk]).
cudaError_t pair_launch_periodic_columns(const StageArgs* args, int n, int max_ny, int rk_step, const StageArgs& one,
                                         cudaStream_t s);


}  // namespace go

struct PreparedStage {
    go::StageArgs a;
    go::PairMapParams mp;
    bool pair, tma;
};
