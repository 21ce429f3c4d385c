// fj_lu.cuh -- dense LU with partial pivoting, solves and FP64 iterative refinement.
#pragma once

#include "fj_common.cuh"

namespace fj {

// Row-major n x n, in place (L unit-lower below the diagonal, U on and above), 0-based
// pivot rows in piv (row i was swapped with piv[i], applied in increasing i, as LAPACK
// getrf).  *d_info (device int) receives 0 or 1 + the first zero-pivot column.
// run_flag (device, may be null): the factor kernels return at once when *run_flag == 0
int lu_factor64(double* a, int n, int32_t* piv, int* d_info, cudaStream_t s, const int* run_flag = nullptr);
int lu_factor32(float* a, int n, int32_t* piv, int* d_info, cudaStream_t s);

// getrs: b <- A^-1 b using the factors (single right-hand side, in place); work: n doubles.
int lu_solve64(const double* lu, int n, const int32_t* piv, double* b, double* work, cudaStream_t s);

// X <- A^-1 (row-major n x n) from FP32 factors.
int lu_inverse32(const float* lu, int n, const int32_t* piv, float* x, cudaStream_t s);

// The factorisation behind the mixed solve: a32 <- FP32 LU of a64 (pivots in piv,
// zero-pivot info in flags[0]) and x32 <- the FP32 inverse.  From n = 256 on the
// products run on the tensor cores (flags[3] <- 1 if one of their bounded waits expired).
// tri: tc_tri_floats(n) floats of scratch.
size_t tc_tri_floats(int n);
int factor_inverse32(const double* a64, int n, float* a32, int32_t* piv, int* flags, float* x32, float* tri,
                     cudaStream_t s);

// Round an FP64 matrix to FP32.
int convert64to32(const double* a, float* b, int64_t count, cudaStream_t s);

// Mixed solve, given FP64 A and the FP32 inverse X of (a matrix close to) A:
//   x = X b;  repeat n_iter times: r = b - A x (FP64);  x += X r.
// Writes ||b - A x||_inf / ||b||_inf of the final x to *d_resid.
// r_buf: n doubles of scratch.
int refine_solve(const double* a, const float* xinv, int n, const double* b, double* x,
                 double* r_buf, double* d_resid, int n_iter, cudaStream_t s);

// Batched refinement: one launch per sweep for many systems (table in device memory).
struct RefineJob {
    const double* a;    // FP64 A (n x n)
    const float* xinv;  // FP32 inverse
    int n;
    const double* b;
    double* x;
    double* r;          // n doubles of scratch
    double* resid;      // 1 double: final relative residual
};
int refine_jobs(const RefineJob* d_jobs, int n_jobs, int max_n, int n_iter, cudaStream_t s);

}  // namespace fj
