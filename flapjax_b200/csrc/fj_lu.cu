// fj_lu.cu -- the dense AIC solve (jnp.linalg.solve, aero/uvlm.py:985).
//
// lu_factor*: blocked right-looking LU with partial pivoting (the LAPACK getrf
// algorithm family XLA calls).  Per panel of NB columns:
//   1. one CTA factors the (n-k) x NB panel held in shared memory (pivot search by
//      block arg-max with LAPACK's first-maximum tie rule, row swap, scale, rank-1);
//   2. the panel's row swaps are applied to the other columns, and U12 = L11^-1 A12;
//   3. the trailing matrix is updated, A22 -= L21 U12.
// lu_solve64: getrs (pivots, unit-lower forward, upper backward substitution) in one CTA.
// lu_inverse32 + refine_solve: the mixed-precision solve.  FP32 factors give an FP32
// explicit inverse X once per factorisation; every solve is then GEMVs over all SMs:
// x = X b, r = b - A x in FP64, x += X r.
#include <climits>

#include "fj_lu.cuh"

namespace fj {

template <typename T>
__device__ __forceinline__ T absval(T v) {
    return v < T(0) ? -v : v;
}

template <typename T, int NB>
__global__ void __launch_bounds__(1024) lu_panel_kernel(T* __restrict__ a, int n, int k,
                                                        int32_t* __restrict__ piv, int* __restrict__ info) {
    extern __shared__ __align__(16) unsigned char smraw[];
    T* P = reinterpret_cast<T*>(smraw);  // (n-k) x NB, row-major
    __shared__ T s_val[32];
    __shared__ int s_idx[32];
    __shared__ int s_piv;
    const int rows = n - k;
    const int nb = min(NB, rows);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
    for (int idx = threadIdx.x; idx < rows * NB; idx += blockDim.x) {
        const int r = idx / NB, c = idx % NB;
        P[idx] = c < nb ? a[(int64_t)(k + r) * n + k + c] : T(0);
    }
    __syncthreads();
    for (int j = 0; j < nb; ++j) {
        T best = T(-1);
        int bi = INT_MAX;
        for (int r = j + threadIdx.x; r < rows; r += blockDim.x) {
            const T v = absval(P[r * NB + j]);
            if (v > best) {
                best = v;
                bi = r;
            }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const T ov = __shfl_down_sync(0xffffffffu, best, off);
            const int oi = __shfl_down_sync(0xffffffffu, bi, off);
            if (ov > best || (ov == best && oi < bi)) {
                best = ov;
                bi = oi;
            }
        }
        if (lane == 0) {
            s_val[warp] = best;
            s_idx[warp] = bi;
        }
        __syncthreads();
        if (warp == 0) {
            best = lane < nwarps ? s_val[lane] : T(-1);
            bi = lane < nwarps ? s_idx[lane] : INT_MAX;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                const T ov = __shfl_down_sync(0xffffffffu, best, off);
                const int oi = __shfl_down_sync(0xffffffffu, bi, off);
                if (ov > best || (ov == best && oi < bi)) {
                    best = ov;
                    bi = oi;
                }
            }
            if (lane == 0) {
                const int p = (bi == INT_MAX) ? j : bi;  // all-NaN column: keep the diagonal
                s_piv = p;
                piv[k + j] = k + p;
            }
        }
        __syncthreads();
        const int p = s_piv;
        if (p != j && threadIdx.x < NB) {
            const T t = P[j * NB + threadIdx.x];
            P[j * NB + threadIdx.x] = P[p * NB + threadIdx.x];
            P[p * NB + threadIdx.x] = t;
        }
        __syncthreads();
        const T pv = P[j * NB + j];
        if (pv == T(0)) {
            if (threadIdx.x == 0 && *info == 0) *info = k + j + 1;
        } else {
            for (int r = j + 1 + threadIdx.x; r < rows; r += blockDim.x) {
                const T l = P[r * NB + j] / pv;
                P[r * NB + j] = l;
                for (int c = j + 1; c < nb; ++c) P[r * NB + c] -= l * P[j * NB + c];
            }
        }
        __syncthreads();
    }
    for (int idx = threadIdx.x; idx < rows * NB; idx += blockDim.x) {
        const int r = idx / NB, c = idx % NB;
        if (c < nb) a[(int64_t)(k + r) * n + k + c] = P[idx];
    }
}

template <typename T, int NB>
__global__ void lu_swap_trsm_kernel(T* __restrict__ a, int n, int k, const int32_t* __restrict__ piv) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int nb = min(NB, n - k);
    if (c >= n || (c >= k && c < k + nb)) return;
    for (int j = 0; j < nb; ++j) {
        const int p = piv[k + j];
        if (p != k + j) {
            const T t = a[(int64_t)(k + j) * n + c];
            a[(int64_t)(k + j) * n + c] = a[(int64_t)p * n + c];
            a[(int64_t)p * n + c] = t;
        }
    }
    if (c >= k + nb) {
        T u[NB];
#pragma unroll
        for (int j = 0; j < NB; ++j)
            if (j < nb) u[j] = a[(int64_t)(k + j) * n + c];
#pragma unroll
        for (int j = 1; j < NB; ++j) {
            if (j < nb) {
                T s = u[j];
#pragma unroll
                for (int jj = 0; jj < j; ++jj) s -= a[(int64_t)(k + j) * n + k + jj] * u[jj];
                u[j] = s;
            }
        }
#pragma unroll
        for (int j = 1; j < NB; ++j)
            if (j < nb) a[(int64_t)(k + j) * n + c] = u[j];
    }
}

template <typename T, int NB>
__global__ void __launch_bounds__(256) lu_update_kernel(T* __restrict__ a, int n, int k) {
    __shared__ T Ls[64][NB + 1];
    __shared__ T Us[NB][64];
    const int k2 = k + NB;
    const int r0 = k2 + blockIdx.y * 64, c0 = k2 + blockIdx.x * 64;
    for (int idx = threadIdx.x; idx < 64 * NB; idx += blockDim.x) {
        const int r = idx / NB, j = idx % NB;
        Ls[r][j] = (r0 + r < n) ? a[(int64_t)(r0 + r) * n + k + j] : T(0);
        const int jj = idx / 64, c = idx % 64;
        Us[jj][c] = (c0 + c < n) ? a[(int64_t)(k + jj) * n + c0 + c] : T(0);
    }
    __syncthreads();
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        const int r = ty + 16 * p;
        if (r0 + r >= n) continue;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int c = tx + 16 * q;
            if (c0 + c >= n) continue;
            T* dst = a + (int64_t)(r0 + r) * n + c0 + c;
            T acc = *dst;
#pragma unroll
            for (int j = 0; j < NB; ++j) acc -= Ls[r][j] * Us[j][c];
            *dst = acc;
        }
    }
}

template <typename T, int NB>
static int lu_factor_impl(T* a, int n, int32_t* piv, int* d_info, cudaStream_t s) {
    if (n <= 0) return fail(FJ_ERR_SHAPE, "lu_factor: n=%d", n);
    const size_t smem = (size_t)n * NB * sizeof(T);
    if (smem > 220 * 1024) return fail(FJ_ERR_UNSUPPORTED, "lu_factor: n=%d too large for the shared-memory panel", n);
    FJ_CUDA(cudaFuncSetAttribute(lu_panel_kernel<T, NB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    FJ_CUDA(cudaMemsetAsync(d_info, 0, sizeof(int), s));
    for (int k = 0; k < n; k += NB) {
        const int nb = min(NB, n - k);
        lu_panel_kernel<T, NB><<<1, 1024, (size_t)(n - k) * NB * sizeof(T), s>>>(a, n, k, piv, d_info); note_launch();
        if (n > nb) {
            lu_swap_trsm_kernel<T, NB><<<(n + 255) / 256, 256, 0, s>>>(a, n, k, piv); note_launch();
        }
        const int rem = n - k - nb;
        if (rem > 0) {
            dim3 g((rem + 63) / 64, (rem + 63) / 64);
            lu_update_kernel<T, NB><<<g, 256, 0, s>>>(a, n, k); note_launch();
        }
    }
    FJ_LAUNCH_CHECK("lu_factor");
    return FJ_OK;
}

int lu_factor64(double* a, int n, int32_t* piv, int* d_info, cudaStream_t s) {
    return lu_factor_impl<double, 8>(a, n, piv, d_info, s);
}
int lu_factor32(float* a, int n, int32_t* piv, int* d_info, cudaStream_t s) {
    return lu_factor_impl<float, 16>(a, n, piv, d_info, s);
}

// ---------------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) lu_solve64_kernel(const double* __restrict__ lu, int n,
                                                          const int32_t* __restrict__ piv,
                                                          double* __restrict__ b) {
    extern __shared__ double x[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = b[i];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 0; i < n; ++i) {
            const int p = piv[i];
            if (p != i) {
                const double t = x[i];
                x[i] = x[p];
                x[p] = t;
            }
        }
    }
    __syncthreads();
    for (int kb = 0; kb < n; kb += 32) {  // forward, unit lower
        const int bw = min(32, n - kb);
        if (warp == 0) {
            for (int jj = 0; jj < bw; ++jj) {
                __syncwarp();
                const double xj = x[kb + jj];
                if (lane > jj && lane < bw) x[kb + lane] -= lu[(int64_t)(kb + lane) * n + kb + jj] * xj;
            }
        }
        __syncthreads();
        for (int i = kb + bw + threadIdx.x; i < n; i += blockDim.x) {
            double sacc = x[i];
            const double* row = lu + (int64_t)i * n + kb;
            for (int jj = 0; jj < bw; ++jj) sacc -= row[jj] * x[kb + jj];
            x[i] = sacc;
        }
        __syncthreads();
    }
    for (int kb = ((n - 1) / 32) * 32; kb >= 0; kb -= 32) {  // backward, upper
        const int be = min(kb + 32, n);
        if (warp == 0) {
            for (int j = be - 1; j >= kb; --j) {
                __syncwarp();
                if (lane == j - kb) x[j] = x[j] / lu[(int64_t)j * n + j];
                __syncwarp();
                const double xj = x[j];
                if (lane < j - kb) x[kb + lane] -= lu[(int64_t)(kb + lane) * n + j] * xj;
            }
        }
        __syncthreads();
        for (int i = threadIdx.x; i < kb; i += blockDim.x) {
            double sacc = x[i];
            const double* row = lu + (int64_t)i * n;
            for (int j = kb; j < be; ++j) sacc -= row[j] * x[j];
            x[i] = sacc;
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) b[i] = x[i];
}

int lu_solve64(const double* lu, int n, const int32_t* piv, double* b, cudaStream_t s) {
    const size_t smem = (size_t)n * sizeof(double);
    if (smem > 220 * 1024) return fail(FJ_ERR_UNSUPPORTED, "lu_solve: n=%d too large", n);
    FJ_CUDA(cudaFuncSetAttribute(lu_solve64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    lu_solve64_kernel<<<1, 1024, smem, s>>>(lu, n, piv, b); note_launch();
    FJ_LAUNCH_CHECK("lu_solve64_kernel");
    return FJ_OK;
}

// ---------------------------------------------------------------------------------
// Explicit inverse from FP32 factors: each CTA solves for 16 columns of the identity.
constexpr int kInvCols = 16;

__global__ void __launch_bounds__(512) lu_inverse32_kernel(const float* __restrict__ lu, int n,
                                                           const int32_t* __restrict__ piv,
                                                           float* __restrict__ xout) {
    extern __shared__ float B[];  // n x kInvCols
    const int c0 = blockIdx.x * kInvCols;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int idx = threadIdx.x; idx < n * kInvCols; idx += blockDim.x) {
        const int i = idx / kInvCols, c = idx % kInvCols;
        B[idx] = (i == c0 + c) ? 1.0f : 0.0f;
    }
    __syncthreads();
    if (threadIdx.x < kInvCols) {  // B <- P B, swaps in getrf order
        const int c = threadIdx.x;
        for (int i = 0; i < n; ++i) {
            const int p = piv[i];
            if (p != i) {
                const float t = B[i * kInvCols + c];
                B[i * kInvCols + c] = B[p * kInvCols + c];
                B[p * kInvCols + c] = t;
            }
        }
    }
    __syncthreads();
    const int r = threadIdx.x / kInvCols;  // 0..31
    const int c = threadIdx.x % kInvCols;
    // forward: unit lower
    for (int i0 = 0; i0 < n; i0 += 32) {
        const int bw = min(32, n - i0);
        if (r < bw) {
            const float* row = lu + (int64_t)(i0 + r) * n;
            float sacc = B[(i0 + r) * kInvCols + c];
            for (int j = 0; j < i0; ++j) sacc -= row[j] * B[j * kInvCols + c];
            B[(i0 + r) * kInvCols + c] = sacc;
        }
        __syncthreads();
        if (warp < kInvCols) {
            const int cc = warp;
            float v = lane < bw ? B[(i0 + lane) * kInvCols + cc] : 0.0f;
            for (int jj = 0; jj < bw; ++jj) {
                const float xj = __shfl_sync(0xffffffffu, v, jj);
                if (lane > jj && lane < bw) v -= lu[(int64_t)(i0 + lane) * n + i0 + jj] * xj;
            }
            if (lane < bw) B[(i0 + lane) * kInvCols + cc] = v;
        }
        __syncthreads();
    }
    // backward: upper
    for (int i0 = ((n - 1) / 32) * 32; i0 >= 0; i0 -= 32) {
        const int be = min(i0 + 32, n);
        const int bw = be - i0;
        if (r < bw) {
            const float* row = lu + (int64_t)(i0 + r) * n;
            float sacc = B[(i0 + r) * kInvCols + c];
            for (int j = be; j < n; ++j) sacc -= row[j] * B[j * kInvCols + c];
            B[(i0 + r) * kInvCols + c] = sacc;
        }
        __syncthreads();
        if (warp < kInvCols) {
            const int cc = warp;
            float v = lane < bw ? B[(i0 + lane) * kInvCols + cc] : 0.0f;
            for (int jj = bw - 1; jj >= 0; --jj) {
                if (lane == jj) v = v / lu[(int64_t)(i0 + jj) * n + i0 + jj];
                const float xj = __shfl_sync(0xffffffffu, v, jj);
                if (lane < jj) v -= lu[(int64_t)(i0 + lane) * n + i0 + jj] * xj;
            }
            if (lane < bw) B[(i0 + lane) * kInvCols + cc] = v;
        }
        __syncthreads();
    }
    for (int idx = threadIdx.x; idx < n * kInvCols; idx += blockDim.x) {
        const int i = idx / kInvCols, cc = idx % kInvCols;
        if (c0 + cc < n) xout[(int64_t)i * n + c0 + cc] = B[idx];
    }
}

int lu_inverse32(const float* lu, int n, const int32_t* piv, float* x, cudaStream_t s) {
    const size_t smem = (size_t)n * kInvCols * sizeof(float);
    if (smem > 220 * 1024) return fail(FJ_ERR_UNSUPPORTED, "lu_inverse32: n=%d too large", n);
    FJ_CUDA(cudaFuncSetAttribute(lu_inverse32_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    lu_inverse32_kernel<<<(n + kInvCols - 1) / kInvCols, 512, smem, s>>>(lu, n, piv, x); note_launch();
    FJ_LAUNCH_CHECK("lu_inverse32_kernel");
    return FJ_OK;
}

__global__ void convert64to32_kernel(const double* __restrict__ a, float* __restrict__ b, int64_t count) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) b[i] = (float)a[i];
}

int convert64to32(const double* a, float* b, int64_t count, cudaStream_t s) {
    if (count == 0) return FJ_OK;
    convert64to32_kernel<<<(unsigned)((count + 255) / 256), 256, 0, s>>>(a, b, count); note_launch();
    FJ_LAUNCH_CHECK("convert64to32_kernel");
    return FJ_OK;
}

// ---------------------------------------------------------------------------------
// Refinement GEMVs: one warp per row, FP64 accumulation.
//   mode 0: y = X v        mode 1: y += X v        (X FP32)
//   residual: r = b - A x  (A FP64)
__global__ void gemv32_kernel(const float* __restrict__ X, const double* __restrict__ v, int n,
                              double* __restrict__ y, int accumulate) {
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    const float* xr = X + (int64_t)row * n;
    double acc = 0.0;
    for (int j = lane; j < n; j += 32) acc += (double)xr[j] * v[j];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if (lane == 0) y[row] = accumulate ? y[row] + acc : acc;
}

__global__ void residual64_kernel(const double* __restrict__ A, const double* __restrict__ x,
                                  const double* __restrict__ b, int n, double* __restrict__ r) {
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    const double* ar = A + (int64_t)row * n;
    double acc = 0.0;
    for (int j = lane; j < n; j += 32) acc += ar[j] * x[j];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if (lane == 0) r[row] = b[row] - acc;
}

__global__ void rel_resid_kernel(const double* __restrict__ r, const double* __restrict__ b, int n,
                                 double* __restrict__ out) {
    __shared__ double sr[32], sb[32];
    double mr = 0.0, mb = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        mr = fmax(mr, fabs(r[i]));
        mb = fmax(mb, fabs(b[i]));
        if (r[i] != r[i]) mr = INFINITY;  // NaN propagates as a failure
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        mr = fmax(mr, __shfl_down_sync(0xffffffffu, mr, off));
        mb = fmax(mb, __shfl_down_sync(0xffffffffu, mb, off));
    }
    if ((threadIdx.x & 31) == 0) {
        sr[threadIdx.x >> 5] = mr;
        sb[threadIdx.x >> 5] = mb;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
            mr = fmax(mr, sr[w]);
            mb = fmax(mb, sb[w]);
        }
        *out = mb > 0.0 ? mr / mb : mr;
    }
}

int refine_solve(const double* a, const float* xinv, int n, const double* b, double* x, double* r_buf,
                 double* d_resid, int n_iter, cudaStream_t s) {
    const int wpb = 8;
    const unsigned grid = (unsigned)((n + wpb - 1) / wpb);
    gemv32_kernel<<<grid, wpb * 32, 0, s>>>(xinv, b, n, x, 0); note_launch();
    for (int it = 0; it < n_iter; ++it) {
        residual64_kernel<<<grid, wpb * 32, 0, s>>>(a, x, b, n, r_buf); note_launch();
        gemv32_kernel<<<grid, wpb * 32, 0, s>>>(xinv, r_buf, n, x, 1); note_launch();
    }
    residual64_kernel<<<grid, wpb * 32, 0, s>>>(a, x, b, n, r_buf); note_launch();
    rel_resid_kernel<<<1, 1024, 0, s>>>(r_buf, b, n, d_resid); note_launch();
    FJ_LAUNCH_CHECK("refine_solve");
    return FJ_OK;
}

}  // namespace fj
