// fj_lti.cu -- the march of a discrete-time state-space system (LinearSystem.run,
// utils/linear.py:775-822): x_i = A x_{i-1} + (B u)_{i - shift}, one GEMV-with-add per step.
//
// Each step reads the whole of A (n x n, row-major FP64) once: the march is HBM-bound, or
// L2-bound while A fits in the 126 MB L2 (A's loads use the ordinary cached path so that
// it stays there from step to step).  A warp owns a row at a time and reads it in 16-byte
// loads, coalesced across the warp; x_{i-1} (n doubles) comes through the read-only path;
// the warp's partial sums meet in a shuffle reduction.  Up to 8 CTAs of 8 warps per SM
// cover the rows; the steps are one launch each from the host loop, on the caller's
// stream.
#include <algorithm>

#include "fj_common.cuh"

namespace fj {
namespace {

constexpr int kLtiWarps = 8;  // rows in flight per CTA

__global__ void __launch_bounds__(kLtiWarps * 32) lti_step_kernel(const double* __restrict__ a, int n,
                                                                  const double* __restrict__ x_prev,
                                                                  const double* __restrict__ add,
                                                                  double* __restrict__ x_next) {
    const int lane = threadIdx.x & 31;
    const int64_t warp0 = (int64_t)blockIdx.x * kLtiWarps + (threadIdx.x >> 5);
    const int64_t stride = (int64_t)gridDim.x * kLtiWarps;
    const bool vec = (n & 1) == 0;  // rows start 16-byte aligned only for even n
    for (int64_t row = warp0; row < n; row += stride) {
        const double* ar = a + row * (int64_t)n;
        double s = 0.0;
        if (vec) {
            const double2* ar2 = reinterpret_cast<const double2*>(ar);
            const double2* x2 = reinterpret_cast<const double2*>(x_prev);
            for (int c = lane; c < n / 2; c += 32) {
                const double2 av = __ldg(ar2 + c);
                const double2 xv = __ldg(x2 + c);
                s = fma(av.x, xv.x, s);
                s = fma(av.y, xv.y, s);
            }
        } else {
            for (int c = lane; c < n; c += 32) s = fma(__ldg(ar + c), __ldg(x_prev + c), s);
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
        if (lane == 0) x_next[row] = s + add[row];
    }
}

}  // namespace
}  // namespace fj

using namespace fj;

extern "C" int fj_lti_march(const double* d_a, int n, const double* d_bu, int64_t ld_bu, double* d_x,
                            int64_t n_tstep, int shift, fj_stream_t stream) {
    if (n < 1 || n_tstep < 1 || ld_bu < n || (shift != 0 && shift != 1) || !d_a || !d_bu || !d_x)
        return fail(FJ_ERR_SHAPE, "lti_march: n=%d n_tstep=%lld ld_bu=%lld shift=%d", n, (long long)n_tstep,
                    (long long)ld_bu, shift);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t need = ((int64_t)n + kLtiWarps - 1) / kLtiWarps;
    const unsigned grid = (unsigned)std::min<int64_t>(need, (int64_t)sms * 8);
    cudaStream_t s = (cudaStream_t)stream;
    for (int64_t i = 1; i < n_tstep; ++i) {
        lti_step_kernel<<<grid, kLtiWarps * 32, 0, s>>>(d_a, n, d_x + (i - 1) * n, d_bu + (i - shift) * ld_bu,
                                                        d_x + i * n);
        note_launch();
    }
    FJ_LAUNCH_CHECK("lti_step_kernel");
    return FJ_OK;
}
