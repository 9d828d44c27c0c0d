// Gaussian-random-field model error: shared declarations (model_error.cu,
// batch.cu).
#pragma once

#include "internal.h"

namespace go {

constexpr int kGrfMaxTaps = 257;        // 2R + 1 filter weights (R <= 128)

struct GrfWeights {
    float w[kGrfMaxTaps];
    int R;
};

// One member's field: eta (interior (ny x nx) at offset (2, 2)), its
// boundary kinds, the second key word and the offset of its (ny + 2R) x nx
// x-filtered noise in the caller's scratch.
struct GrfMember {
    float* eta;
    int pitch;              // floats
    int nx, ny;
    int periodic_x, periodic_y;
    uint32_t key1;
    size_t tmp_off;
};

// Filter weights for a correlation length in cells.
int grf_weights(float corr_cells, GrfWeights* W);

// Scratch floats one member needs.
inline size_t grf_member_scratch(int nx, int ny, int R) { return (size_t)(ny + 2 * R) * (size_t)nx; }

// eta += std_dev * field for n members (members == nullptr: the single
// member passed by value), key (key0, member.key1), counter event -- or,
// when event_dev is given, the event the device holds there when the
// kernels run (a launch captured into a device-driven event loop).
int grf_launch(const GrfMember* d_members, const GrfMember& single, int n_members, int max_nx, int max_ny,
               uint32_t key0, uint32_t event, float std_dev, const GrfWeights& W, float* scratch,
               cudaStream_t s, const uint32_t* event_dev = nullptr);

}  // namespace go
