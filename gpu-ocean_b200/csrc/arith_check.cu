// Self-check of the reciprocal-quotient mode (GO_ARITH_RCP).
//
// The stage kernel evaluates the reference's quotients a / b, which the
// reference compiles with --prec-div=false (CDKLM16.py:196-200), either as
// written (GO_ARITH_EXACT) or as a * rcp.approx.ftz(b) with the reciprocal
// of a shared denominator hoisted (GO_ARITH_RCP).  This unit is compiled
// with the stage kernel's own flags, so the two quotients it returns are
// the ones the two modes evaluate; tests compare them bit for bit over the
// denominators the scheme divides by.
#include "internal.h"

using namespace go;

namespace {

__global__ void k_quotients(const float* __restrict__ a, const float* __restrict__ b, int n,
                            float* __restrict__ q_div, float* __restrict__ q_rcp) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float x = a[i], y = b[i];
        q_div[i] = x / y;
        q_rcp[i] = quot<true>(x, y);
    }
}

}  // namespace

int go_check_quotients(void* stream, const float* a, const float* b, int n, float* q_div, float* q_rcp) {
    if (n < 0 || (n > 0 && (!a || !b || !q_div || !q_rcp)))
        return go_fail(GO_ERR_INVALID, "go_check_quotients: bad arguments");
    if (n == 0) return GO_OK;
    const int blocks = (n + 255) / 256 < 148 * 8 ? (n + 255) / 256 : 148 * 8;
    k_quotients<<<blocks, 256, 0, (cudaStream_t)stream>>>(a, b, n, q_div, q_rcp);
    GO_CUDA(cudaGetLastError());
    return GO_OK;
}
