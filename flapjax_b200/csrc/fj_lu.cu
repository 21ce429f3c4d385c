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
#include <cstdlib>
#include <cstring>
#include <mutex>

#include <cooperative_groups.h>

#include "fj_lu.cuh"
#include "fj_tc.cuh"

namespace fj {

template <typename T>
__device__ __forceinline__ T absval(T v) {
    return v < T(0) ? -v : v;
}

template <typename T, int NB>
__global__ void __launch_bounds__(1024) lu_panel_kernel(T* __restrict__ a, int n, int k,
                                                        int32_t* __restrict__ piv, int* __restrict__ info,
                                                        const int* __restrict__ run_flag) {
    if (run_flag != nullptr && *run_flag == 0) return;
    extern __shared__ __align__(16) unsigned char smraw[];
    T* P = reinterpret_cast<T*>(smraw);  // (n-k) x LDP, row-major; odd stride avoids bank conflicts
    constexpr int LDP = NB + 1;
    __shared__ T s_val[32];
    __shared__ int s_idx[32];
    const int rows = n - k;
    const int nb = min(NB, rows);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
    // asynchronous copies of the panel: every element in flight at once (columns past nb
    // zero-filled)
    for (int idx = threadIdx.x; idx < rows * NB; idx += blockDim.x) {
        const int r = idx / NB, c = idx % NB;
        const T* src = a + (int64_t)(k + r) * n + k + min(c, nb - 1);
        const unsigned dst = (unsigned)__cvta_generic_to_shared(P + r * LDP + c);
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(dst), "l"(src), "n"(sizeof(T)),
                     "r"(c < nb ? (int)sizeof(T) : 0)
                     : "memory");
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    for (int j = 0; j < nb; ++j) {
        T best = T(-1);
        int bi = INT_MAX;
        for (int r = j + threadIdx.x; r < rows; r += blockDim.x) {
            const T v = absval(P[r * LDP + j]);
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
        // every warp reduces the partials itself: no second barrier
        best = lane < nwarps ? s_val[lane] : T(-1);
        bi = lane < nwarps ? s_idx[lane] : INT_MAX;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const T ov = __shfl_xor_sync(0xffffffffu, best, off);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
            if (ov > best || (ov == best && oi < bi)) {
                best = ov;
                bi = oi;
            }
        }
        const int p = (bi == INT_MAX) ? j : bi;  // all-NaN column: keep the diagonal
        if (threadIdx.x == 0) piv[k + j] = k + p;
        if (p != j && threadIdx.x < NB) {
            const T t = P[j * LDP + threadIdx.x];
            P[j * LDP + threadIdx.x] = P[p * LDP + threadIdx.x];
            P[p * LDP + threadIdx.x] = t;
        }
        __syncthreads();
        const T pv = P[j * LDP + j];
        if (pv == T(0)) {
            if (threadIdx.x == 0 && *info == 0) *info = k + j + 1;
        } else {
            for (int r = j + 1 + threadIdx.x; r < rows; r += blockDim.x) {
                const T l = P[r * LDP + j] / pv;
                P[r * LDP + j] = l;
                for (int c = j + 1; c < nb; ++c) P[r * LDP + c] -= l * P[j * LDP + c];
            }
        }
        __syncthreads();
    }
#pragma unroll 8
    for (int idx = threadIdx.x; idx < rows * NB; idx += blockDim.x) {
        const int r = idx / NB, c = idx % NB;
        if (c < nb) a[(int64_t)(k + r) * n + k + c] = P[r * LDP + c];
    }
}

// The same panel with its rows in registers, for panels of at most RPT * 1024 rows.  The
// panel comes in and goes out through shared memory (coalesced cp.async loads and row-
// contiguous stores, as lu_panel_kernel); between, thread t owns rows t + 1024 i (i < RPT)
// in registers, and a column costs two barriers: one to combine the warps' pivot
// candidates, one to exchange the pivot row and row j.  Pivots (first maximum, as getrf)
// and every arithmetic operation are those of lu_panel_kernel, so the factors are bitwise
// the same.
template <typename T, int NB, int RPT>
__global__ void __launch_bounds__(1024) lu_panel_reg_kernel(T* __restrict__ a, int n, int k,
                                                            int32_t* __restrict__ piv, int* __restrict__ info,
                                                            const int* __restrict__ run_flag) {
    if (run_flag != nullptr && *run_flag == 0) return;
    extern __shared__ __align__(16) unsigned char smraw[];
    T* P = reinterpret_cast<T*>(smraw);  // (n-k) x LDP staging
    constexpr int LDP = NB + 1;
    __shared__ T s_val[32];
    __shared__ int s_idx[32];
    __shared__ T s_rowp[NB], s_rowj[NB];
    const int rows = n - k;
    const int nb = min(NB, rows);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nwarps = blockDim.x >> 5;
    for (int idx = tid; idx < rows * NB; idx += blockDim.x) {
        const int r = idx / NB, c = idx % NB;
        const T* src = a + (int64_t)(k + r) * n + k + min(c, nb - 1);
        const unsigned dst = (unsigned)__cvta_generic_to_shared(P + r * LDP + c);
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(dst), "l"(src), "n"(sizeof(T)),
                     "r"(c < nb ? (int)sizeof(T) : 0)
                     : "memory");
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    T v[RPT][NB];
#pragma unroll
    for (int i = 0; i < RPT; ++i) {
        const int r = tid + i * (int)blockDim.x;
#pragma unroll
        for (int c = 0; c < NB; ++c) v[i][c] = r < rows ? P[r * LDP + c] : T(0);
    }
#pragma unroll
    for (int j = 0; j < NB; ++j) {
        if (j >= nb) break;  // uniform over the CTA
        T best = T(-1);
        int bi = INT_MAX;
#pragma unroll
        for (int i = 0; i < RPT; ++i) {
            const int r = tid + i * (int)blockDim.x;
            if (r >= j && r < rows) {
                const T x = absval(v[i][j]);
                if (x > best) {
                    best = x;
                    bi = r;
                }
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
        best = lane < nwarps ? s_val[lane] : T(-1);
        bi = lane < nwarps ? s_idx[lane] : INT_MAX;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const T ov = __shfl_xor_sync(0xffffffffu, best, off);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
            if (ov > best || (ov == best && oi < bi)) {
                best = ov;
                bi = oi;
            }
        }
        const int p = (bi == INT_MAX) ? j : bi;  // all-NaN column: keep the diagonal
        if (tid == 0) piv[k + j] = k + p;
#pragma unroll
        for (int i = 0; i < RPT; ++i) {  // the owners of rows p and j publish them
            const int r = tid + i * (int)blockDim.x;
            if (r == p) {
#pragma unroll
                for (int c = 0; c < NB; ++c) s_rowp[c] = v[i][c];
            }
            if (r == j) {
#pragma unroll
                for (int c = 0; c < NB; ++c) s_rowj[c] = v[i][c];
            }
        }
        __syncthreads();
        if (p != j) {  // the swap: row j takes the pivot row, row p takes row j
#pragma unroll
            for (int i = 0; i < RPT; ++i) {
                const int r = tid + i * (int)blockDim.x;
                if (r == j) {
#pragma unroll
                    for (int c = 0; c < NB; ++c) v[i][c] = s_rowp[c];
                }
                if (r == p) {
#pragma unroll
                    for (int c = 0; c < NB; ++c) v[i][c] = s_rowj[c];
                }
            }
        }
        const T pv = s_rowp[j];
        if (pv == T(0)) {
            if (tid == 0 && *info == 0) *info = k + j + 1;
        } else {
#pragma unroll
            for (int i = 0; i < RPT; ++i) {
                const int r = tid + i * (int)blockDim.x;
                if (r > j && r < rows) {
                    const T l = v[i][j] / pv;
                    v[i][j] = l;
#pragma unroll
                    for (int c = j + 1; c < NB; ++c)
                        if (c < nb) v[i][c] -= l * s_rowp[c];
                }
            }
        }
    }
#pragma unroll
    for (int i = 0; i < RPT; ++i) {
        const int r = tid + i * (int)blockDim.x;
        if (r < rows) {
#pragma unroll
            for (int c = 0; c < NB; ++c) P[r * LDP + c] = v[i][c];
        }
    }
    __syncthreads();
    for (int idx = tid; idx < rows * NB; idx += blockDim.x) {
        const int r = idx / NB, c = idx % NB;
        if (c < nb) a[(int64_t)(k + r) * n + k + c] = P[r * LDP + c];
    }
}

// One panel at column k: the register form where its rows fit (at most 2048), else the
// shared-memory form; both stage the panel in the same dynamic shared memory.
template <typename T, int NB>
static void launch_panel(T* a, int n, int k, int32_t* piv, int* info, const int* run_flag, cudaStream_t s) {
    const int rows = n - k;
    const size_t smem = (size_t)rows * (NB + 1) * sizeof(T);
    if (rows <= 1024)
        lu_panel_reg_kernel<T, NB, 1><<<1, 1024, smem, s>>>(a, n, k, piv, info, run_flag);
    else if (rows <= 2048)
        lu_panel_reg_kernel<T, NB, 2><<<1, 1024, smem, s>>>(a, n, k, piv, info, run_flag);
    else
        lu_panel_kernel<T, NB><<<1, 1024, smem, s>>>(a, n, k, piv, info, run_flag);
    note_launch();
}

// Row swaps of the panel at column k for every other column; U12 = L11^-1 A12 for the
// columns [k + nb, c_end).  The panel's swaps (applied in order, as getrf) compose to one
// permutation of the at most 2 NB rows they touch; thread 0 works it out in shared memory,
// then each column thread loads all the touched values before storing any, one memory
// round trip instead of one per swap.
template <typename T, int NB>
__global__ void lu_swap_trsm_kernel(T* __restrict__ a, int n, int k, const int32_t* __restrict__ piv, int c_end,
                                    const int* __restrict__ run_flag) {
    if (run_flag != nullptr && *run_flag == 0) return;
    __shared__ int s_dst[2 * NB], s_src[2 * NB], s_piv[NB];
    __shared__ int s_cnt;
    __shared__ T s_l[NB][NB];  // the panel's unit-lower diagonal block, for the triangular solve
    const int nb = min(NB, n - k);
    if (threadIdx.x < nb) s_piv[threadIdx.x] = piv[k + threadIdx.x];
    for (int idx = threadIdx.x; idx < NB * NB; idx += blockDim.x) {
        const int r = idx / NB, c = idx % NB;
        s_l[r][c] = (r < nb && c < r) ? a[(int64_t)(k + r) * n + k + c] : T(0);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int cnt = 0;
        for (int jj = 0; jj < nb; ++jj) {
            const int r1 = k + jj, r2 = s_piv[jj];
            if (r1 == r2) continue;
            int i1 = -1, i2 = -1;
            for (int e = 0; e < cnt; ++e) {
                if (s_dst[e] == r1) i1 = e;
                if (s_dst[e] == r2) i2 = e;
            }
            if (i1 < 0) {
                i1 = cnt++;
                s_dst[i1] = r1;
                s_src[i1] = r1;
            }
            if (i2 < 0) {
                i2 = cnt++;
                s_dst[i2] = r2;
                s_src[i2] = r2;
            }
            const int tmp = s_src[i1];
            s_src[i1] = s_src[i2];
            s_src[i2] = tmp;
        }
        s_cnt = cnt;
    }
    __syncthreads();
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n || (c >= k && c < k + nb)) return;
    const int cnt = s_cnt;
    T val[2 * NB];
#pragma unroll
    for (int e = 0; e < 2 * NB; ++e)
        if (e < cnt) val[e] = a[(int64_t)s_src[e] * n + c];
#pragma unroll
    for (int e = 0; e < 2 * NB; ++e)
        if (e < cnt) a[(int64_t)s_dst[e] * n + c] = val[e];
    if (c >= k + nb && c < c_end) {
        T u[NB];
#pragma unroll
        for (int j = 0; j < NB; ++j)
            if (j < nb) u[j] = a[(int64_t)(k + j) * n + c];
#pragma unroll
        for (int j = 1; j < NB; ++j) {
            if (j < nb) {
                T s = u[j];
#pragma unroll
                for (int jj = 0; jj < j; ++jj) s -= s_l[j][jj] * u[jj];
                u[j] = s;
            }
        }
#pragma unroll
        for (int j = 1; j < NB; ++j)
            if (j < nb) a[(int64_t)(k + j) * n + c] = u[j];
    }
}

// A[r0.., c0..] -= L[., k..k+NB) U[k..k+NB, .] on one 64 x 64 tile, rows < r_end and
// columns < c_end.
template <typename T, int NB>
__device__ __forceinline__ void lu_update_tile(T* __restrict__ a, int n, int k, int r0, int c0, int r_end,
                                               int c_end) {
    __shared__ T Ls[64][NB + 1];
    __shared__ T Us[NB][64];
    for (int idx = threadIdx.x; idx < 64 * NB; idx += blockDim.x) {
        const int r = idx / NB, j = idx % NB;
        Ls[r][j] = (r0 + r < r_end) ? a[(int64_t)(r0 + r) * n + k + j] : T(0);
        const int jj = idx / 64, c = idx % 64;
        Us[jj][c] = (c0 + c < c_end) ? a[(int64_t)(k + jj) * n + c0 + c] : T(0);
    }
    // the 16 elements of this thread are loaded before any is computed: one memory round
    // trip per tile
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    T acc[4][4];
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = ty + 16 * p, c = tx + 16 * q;
            acc[p][q] = (r0 + r < r_end && c0 + c < c_end) ? a[(int64_t)(r0 + r) * n + c0 + c] : T(0);
        }
    __syncthreads();
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = ty + 16 * p, c = tx + 16 * q;
#pragma unroll
            for (int j = 0; j < NB; ++j) acc[p][q] -= Ls[r][j] * Us[j][c];
        }
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = ty + 16 * p, c = tx + 16 * q;
            if (r0 + r < r_end && c0 + c < c_end) a[(int64_t)(r0 + r) * n + c0 + c] = acc[p][q];
        }
}

// A22 -= L21 U12 over rows [k + NB, n) and columns [k + NB, c_end).
template <typename T, int NB>
__global__ void __launch_bounds__(256) lu_update_kernel(T* __restrict__ a, int n, int k, int c_end,
                                                        const int* __restrict__ run_flag) {
    if (run_flag != nullptr && *run_flag == 0) return;
    const int k2 = k + NB;
    lu_update_tile<T, NB>(a, n, k, k2 + blockIdx.y * 64, k2 + blockIdx.x * 64, n, c_end);
}

template <typename T, int NB>
static int lu_factor_impl(T* a, int n, int32_t* piv, int* d_info, cudaStream_t s, const int* run_flag) {
    if (n <= 0) return fail(FJ_ERR_SHAPE, "lu_factor: n=%d", n);
    const size_t smem = (size_t)n * (NB + 1) * sizeof(T);
    if (smem > 220 * 1024) return fail(FJ_ERR_UNSUPPORTED, "lu_factor: n=%d too large for the shared-memory panel", n);
    FJ_TRY(allow_dynamic_smem((const void*)lu_panel_kernel<T, NB>, (size_t)smem));
    FJ_TRY(allow_dynamic_smem((const void*)lu_panel_reg_kernel<T, NB, 1>, (size_t)smem));
    FJ_TRY(allow_dynamic_smem((const void*)lu_panel_reg_kernel<T, NB, 2>, (size_t)smem));
    FJ_CUDA(cudaMemsetAsync(d_info, 0, sizeof(int), s));
    for (int k = 0; k < n; k += NB) {
        const int nb = min(NB, n - k);
        launch_panel<T, NB>(a, n, k, piv, d_info, run_flag, s);
        if (n > nb) {
            lu_swap_trsm_kernel<T, NB><<<(n + 255) / 256, 256, 0, s>>>(a, n, k, piv, n, run_flag); note_launch();
        }
        const int rem = n - k - nb;
        if (rem > 0) {
            dim3 g((rem + 63) / 64, (rem + 63) / 64);
            lu_update_kernel<T, NB><<<g, 256, 0, s>>>(a, n, k, n, run_flag); note_launch();
        }
    }
    FJ_LAUNCH_CHECK("lu_factor");
    return FJ_OK;
}

// Panel width: the widest whose (n x (NB + 1)) panel fits the shared-memory budget, so that
// the largest validated AIC order (6144) factors too.
template <typename T>
static bool panel_fits(int n, int nb) {
    return (size_t)n * (nb + 1) * sizeof(T) <= (size_t)220 * 1024;
}

int lu_factor32(float* a, int n, int32_t* piv, int* d_info, cudaStream_t s) {
    if (panel_fits<float>(n, 16)) return lu_factor_impl<float, 16>(a, n, piv, d_info, s, nullptr);
    return lu_factor_impl<float, 8>(a, n, piv, d_info, s, nullptr);
}

// ---------------------------------------------------------------------------------
// getrs: x = P b, then blocked substitution.  Per block of kTrsvBlk rows one CTA solves
// the diagonal block in shared memory and a grid of warps (one per remaining row) applies
// the block's contribution to the rows still to be solved.
constexpr int kTrsvBlk = 128;

// x[i] = b[perm[i]], perm from the getrf row swaps applied in order to the identity.
__global__ void __launch_bounds__(1024) permute_kernel(const int32_t* __restrict__ piv, int n,
                                                       const double* __restrict__ b, double* __restrict__ x) {
    extern __shared__ int perm[];  // n permutation entries, then n pivots
    int* sp = perm + n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        perm[i] = i;
        sp[i] = piv[i];
    }
    __syncthreads();
    if (threadIdx.x == 0) {  // the swaps compose in order; from shared memory only
        for (int i = 0; i < n; ++i) {
            const int p = sp[i];
            if (p != i) {
                const int t = perm[i];
                perm[i] = perm[p];
                perm[p] = t;
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = b[perm[i]];
}

// Solve the diagonal block [i0, i0+bw) of L (unit lower, upper = false) or U (upper = true)
// in place on x.  The block comes into shared memory with every element's cp.async in
// flight at once; then one warp substitutes, lane l holding x of rows l + 32 q (q < 4) in
// registers and x_j reaching every lane by a shuffle, so no step waits on a CTA barrier.
// Per row the operations are getrs's, in its order.
__device__ __forceinline__ double pick4(const double (&v)[4], int q) {
    return q == 0 ? v[0] : q == 1 ? v[1] : q == 2 ? v[2] : v[3];
}

__global__ void __launch_bounds__(kTrsvBlk) trsv_diag_kernel(const double* __restrict__ lu, int n, int i0, int bw,
                                                             bool upper, double* __restrict__ x) {
    static_assert(kTrsvBlk == 128, "four rows per lane");
    extern __shared__ double blk[];  // bw x (bw + 1)
    const int ld = bw + 1;
    for (int idx = threadIdx.x; idx < bw * bw; idx += blockDim.x) {
        const int r = idx / bw, c = idx % bw;
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(blk + r * ld + c)),
                     "l"(lu + (int64_t)(i0 + r) * n + i0 + c)
                     : "memory");
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    if (threadIdx.x >= 32) return;
    const int lane = threadIdx.x;
    const unsigned full = 0xffffffffu;
    double v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) v[q] = lane + 32 * q < bw ? x[i0 + lane + 32 * q] : 0.0;
    if (!upper) {
#pragma unroll 1
        for (int j = 0; j < bw; ++j) {
            const double xj = __shfl_sync(full, pick4(v, j >> 5), j & 31);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int r = lane + 32 * q;
                if (r > j && r < bw) v[q] -= blk[r * ld + j] * xj;
            }
        }
    } else {
#pragma unroll 1
        for (int j = bw - 1; j >= 0; --j) {
            const int qj = j >> 5;
            if (lane == (j & 31)) {
                const double d = blk[j * ld + j];
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (q == qj) v[q] = v[q] / d;
            }
            const double xj = __shfl_sync(full, pick4(v, qj), j & 31);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int r = lane + 32 * q;
                if (r < j) v[q] -= blk[r * ld + j] * xj;
            }
        }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
        if (lane + 32 * q < bw) x[i0 + lane + 32 * q] = v[q];
}

// x[i] -= sum_{j in [j0, j0+bw)} lu[i][j] x[j] for i in [r0, r1): one warp per row.
__global__ void trsv_update_kernel(const double* __restrict__ lu, int n, int j0, int bw, int r0, int r1,
                                   double* __restrict__ x) {
    const int row = r0 + blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= r1) return;
    const double* a = lu + (int64_t)row * n + j0;
    double acc = 0.0;
    for (int j = lane; j < bw; j += 32) acc += a[j] * x[j0 + j];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if (lane == 0) x[row] -= acc;
}

int lu_solve64(const double* lu, int n, const int32_t* piv, double* b, double* work, cudaStream_t s) {
    if (n <= 0) return fail(FJ_ERR_SHAPE, "lu_solve: n=%d", n);
    if ((size_t)n * sizeof(int) > 220 * 1024) return fail(FJ_ERR_UNSUPPORTED, "lu_solve: n=%d too large", n);
    const size_t dsm = (size_t)kTrsvBlk * (kTrsvBlk + 1) * sizeof(double);
    FJ_TRY(allow_dynamic_smem((const void*)permute_kernel, (size_t)(2 * n * sizeof(int))));
    FJ_TRY(allow_dynamic_smem((const void*)trsv_diag_kernel, (size_t)dsm));
    permute_kernel<<<1, 1024, 2 * n * sizeof(int), s>>>(piv, n, b, work); note_launch();
    const int wpb = 8;
    for (int i0 = 0; i0 < n; i0 += kTrsvBlk) {  // forward, unit lower
        const int bw = min(kTrsvBlk, n - i0);
        trsv_diag_kernel<<<1, kTrsvBlk, (size_t)bw * (bw + 1) * sizeof(double), s>>>(lu, n, i0, bw, false, work); note_launch();
        const int r0 = i0 + bw;
        if (r0 < n) {
            trsv_update_kernel<<<(n - r0 + wpb - 1) / wpb, wpb * 32, 0, s>>>(lu, n, i0, bw, r0, n, work); note_launch();
        }
    }
    for (int i0 = ((n - 1) / kTrsvBlk) * kTrsvBlk; i0 >= 0; i0 -= kTrsvBlk) {  // backward, upper
        const int bw = min(kTrsvBlk, n - i0);
        trsv_diag_kernel<<<1, kTrsvBlk, (size_t)bw * (bw + 1) * sizeof(double), s>>>(lu, n, i0, bw, true, work); note_launch();
        if (i0 > 0) {
            trsv_update_kernel<<<(i0 + wpb - 1) / wpb, wpb * 32, 0, s>>>(lu, n, i0, bw, 0, i0, work); note_launch();
        }
    }
    FJ_CUDA(cudaMemcpyAsync(b, work, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    FJ_LAUNCH_CHECK("lu_solve64");
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
    FJ_TRY(allow_dynamic_smem((const void*)lu_inverse32_kernel, (size_t)smem));
    lu_inverse32_kernel<<<(n + kInvCols - 1) / kInvCols, 512, smem, s>>>(lu, n, piv, x); note_launch();
    FJ_LAUNCH_CHECK("lu_inverse32_kernel");
    return FJ_OK;
}

// ---------------------------------------------------------------------------------
// Tensor-core factorisation and inverse (mixed path, n >= kTcMinN).
//
// lu_factor32_tc: the same partial-pivoting LU, blocked twice.  One thread-block cluster
// factors each outer panel of 128 columns (lu_panel_cluster_kernel; the 16-column panels
// above where the rows exceed one cluster, their U rows and updates confined to the outer
// panel).  The columns to its right receive only the row swaps until the outer panel is
// done; then
//   U12 = L11^-1 A12        (lu_trsm32_kernel: forward substitution, CUDA cores, in place)
//   A22 -= L21 U12          (tensor cores, K = 128)
//
// lu_inverse32_tc: X = U^-1 L^-1 P by blocked substitution on the n x n right-hand side
// P (the getrf row swaps applied to the identity), 128 rows at a time:
//   forward   Y_i = L_ii^-1 Y_i,  Y_below -= L_below,i Y_i
//   backward  X_i = U_ii^-1 Y_i,  Y_above -= U_above,i X_i
// Every product is a tensor-core GEMM; 2 n^3 flop in all.
constexpr int kTcBlk = 128;

// tri: the 2 x nblk inverted diagonal blocks (L's, then U's), then the TMA products'
// operand-split scratch, enough for the largest product (m, n <= nblk x 128, K = 128),
// then the row-swap list of one outer panel (kSwapInts ints).
constexpr int kSwapInts = 1 + 2 * 2 * kTcBlk;  // count, then (destination, source) row pairs

static size_t tc_inv_floats(int n) {
    return (size_t)2 * ((n + kTcBlk - 1) / kTcBlk) * kTcBlk * kTcBlk;
}

static size_t tc_scratch_floats(int n) {
    const int np = (n + kTcBlk - 1) / kTcBlk * kTcBlk;
    return tc_gemm_scratch_floats(np, np, kTcBlk, 3);
}

size_t tc_tri_floats(int n) {
    return tc_inv_floats(n) + tc_scratch_floats(n) + (size_t)kSwapInts;
}

// ---------------------------------------------------------------------------------
// One 128-column outer panel, (n - k) rows, factored by a single thread-block cluster
// of 16-warp CTAs (up to 16 CTAs of 8-row warps where the device allows that cluster
// size, else up to 8 CTAs of 16-row warps): getrf's partial pivoting and rank-1 updates
// column by column, with the panel in registers.  Lanes are columns: lane L of a warp
// holds columns L, L + 32, L + 64, L + 96 of the warp's RPW rows; CTA q holds panel rows
// 16 RPW q .. in order over its warps.  The column loop runs in four groups of 32
// (unrolled), so that a column's register is a compile-time index.  Per column j:
//   a. every warp gathers column j of its rows (lane i takes row i from lane j % 32),
//      finds the first maximum of |a(r, j)| over rows r >= j (keys are the magnitude's
//      bits + 1, so one redux.sync orders them; NaN is never a candidate; the lowest
//      lane, i.e. row, wins a tie) and copies the winning row into its candidate slot;
//      the warp holding row j copies row j;
//   b. one CTA barrier; four warps take the CTA's first maximum over its warps and push
//      that row, its key, index and origin into every CTA's slot q (distributed shared
//      memory stores); in CTA 0 four more warps push row j the same way;
//   c. one cluster barrier;
//   d. every warp reads the nc slot keys from its own shared memory and takes the first
//      maximum (lowest CTA: the lowest row, getrf's tie rule; no candidate keeps the
//      diagonal); rows j and p trade places (the pivot row and row j from the local
//      slots); the rows below j are scaled as getrf scales them (by the reciprocal of the
//      pivot when its magnitude is at least the smallest normal, else by division) and
//      updated.
// All slots alternate between two buffers with the column's parity: a buffer is written
// again only after the next column's cluster barrier, which every CTA reaches after its
// reads of it.  Lane i < RPW of a warp carries the original index of the warp's row i;
// at the end the moved rows are listed as (destination, source) global row pairs, at
// most 2 x 128, for lu_swap_rows_kernel.  Every thread passes every barrier (the loop
// bounds are uniform over the cluster), so no wait depends on data.
namespace cg = cooperative_groups;

constexpr int kPcThreads = 512;
constexpr int kPcWarps = kPcThreads / 32;
constexpr int kPcMaxCtas = 16;

// Panel element types.  A panel row is 512 bytes either way: 128 FP32 columns (the mixed
// path's outer panel) or 64 FP64 columns (the FP64 path's); lane L holds columns L + 32 c,
// c < NG.  The candidate key is the magnitude's bits + 1, ordered as the magnitudes; 0 = no
// candidate (inactive, or NaN, which never wins a getrf pivot search).
template <typename T>
struct PanelType;
template <>
struct PanelType<float> {
    static constexpr int NG = 4;
    using Key = uint32_t;
    __device__ static __forceinline__ Key key(float x) {
        const float ax = fabsf(x);
        return ax == ax ? __float_as_uint(ax) + 1u : 0u;
    }
    __device__ static __forceinline__ bool normal(float x) { return fabsf(x) >= 1.17549435e-38f; }  // FLT_MIN
};
template <>
struct PanelType<double> {
    static constexpr int NG = 2;
    using Key = unsigned long long;
    __device__ static __forceinline__ Key key(double x) {
        const double ax = fabs(x);
        return ax == ax ? (Key)__double_as_longlong(ax) + 1ull : 0ull;
    }
    __device__ static __forceinline__ bool normal(double x) { return fabs(x) >= 2.2250738585072014e-308; }  // DBL_MIN
};

// The warp's largest key (every lane gets it).
__device__ __forceinline__ uint32_t warp_key_max(uint32_t k) { return __reduce_max_sync(0xffffffffu, k); }
__device__ __forceinline__ unsigned long long warp_key_max(unsigned long long k) {
    const uint32_t hi = (uint32_t)(k >> 32);
    const uint32_t mhi = __reduce_max_sync(0xffffffffu, hi);
    const uint32_t mlo = __reduce_max_sync(0xffffffffu, hi == mhi ? (uint32_t)k : 0u);
    return ((unsigned long long)mhi << 32) | mlo;
}

// Row `i` (a runtime index) of a thread's rows, as the NG columns this lane holds.
template <typename T, int NG, int RPW>
__device__ __forceinline__ void pick_row(const T (&v)[RPW][NG], int i, T (&out)[NG]) {
#pragma unroll
    for (int c = 0; c < NG; ++c) out[c] = v[0][c];
#pragma unroll
    for (int r = 1; r < RPW; ++r)
        if (r == i) {
#pragma unroll
            for (int c = 0; c < NG; ++c) out[c] = v[r][c];
        }
}

template <typename T, int NG, int RPW>
__device__ __forceinline__ void put_row(T (&v)[RPW][NG], int i, const T (&in)[NG]) {
#pragma unroll
    for (int r = 0; r < RPW; ++r)
        if (r == i) {
#pragma unroll
            for (int c = 0; c < NG; ++c) v[r][c] = in[c];
        }
}

// Rank-1 update of the rows below j with multipliers column(j) * s (mul) or / s (div).
template <typename T, int NG, int RPW, int G, bool kDiv>
__device__ __forceinline__ void panel_update(T (&v)[RPW][NG], int rbase, int rows, int j, int jj, int lane, T s,
                                             const T (&pc)[NG]) {
#pragma unroll
    for (int i = 0; i < RPW; ++i) {
        const int r = rbase + i;
        if (r > j && r < rows) {  // uniform over the warp
            T l = kDiv ? v[i][G] / s : v[i][G] * s;
            l = __shfl_sync(0xffffffffu, l, jj);  // lane jj's is the multiplier
            if (lane == jj) v[i][G] = l;
#pragma unroll
            for (int c = G + 1; c < NG; ++c) v[i][c] -= l * pc[c];
            if (lane > jj) v[i][G] -= l * pc[G];
        }
    }
}

// The panel's shared state (static shared memory of lu_panel_cluster_kernel).
template <typename T>
struct PanelShared {
    static constexpr int KB = 32 * PanelType<T>::NG;
    using Key = typename PanelType<T>::Key;
    T cand[2][kPcWarps][KB];  // this CTA's warp candidates
    Key wkey[2][kPcWarps];
    int wrow[2][kPcWarps], wsrc[2][kPcWarps];
    T rowj_loc[2][KB];                // row j, in CTA 0
    T slot[2][kPcMaxCtas][KB];        // every CTA's candidate, pushed by that CTA
    Key slot_key[2][kPcMaxCtas];
    int slot_row[2][kPcMaxCtas], slot_src[2][kPcMaxCtas];
    T rowj[2][KB];                    // row j, pushed by CTA 0
    int rowj_src[2];
    int rowj_src_loc[2];
    int piv[KB];  // written out at the end: no global store inside the column loop
    int info;
    int wcnt[kPcWarps], cnt, off;
};

template <typename T, int RPW, int G>
__device__ __forceinline__ void panel_columns(T (&v)[RPW][PanelType<T>::NG], int& orig, int k, int kb, int rows,
                                              int q, int nc, int tid, cg::cluster_group& cl, PanelShared<T>& S) {
    constexpr int NG = PanelType<T>::NG;
    using Key = typename PanelType<T>::Key;
    const int lane = tid & 31, warp = tid >> 5;
    const int rbase = (q * kPcWarps + warp) * RPW;
    const unsigned full = 0xffffffffu;
    const int jend = min(kb, 32 * G + 32);
#pragma unroll 1
    for (int j = 32 * G; j < jend; ++j) {
        const int jj = j & 31, par = j & 1;
        // a. the warp's candidate: lane i < RPW takes column j of row i
        T xj = T(0);
#pragma unroll
        for (int i = 0; i < RPW; ++i) {
            const T t = __shfl_sync(full, v[i][G], jj);
            if (lane == i) xj = t;
        }
        const int r = rbase + lane;
        const Key key = (lane < RPW && r >= j && r < rows) ? PanelType<T>::key(xj) : Key(0);
        const Key wmax = warp_key_max(key);
        const unsigned hit = __ballot_sync(full, wmax != Key(0) && key == wmax);
        const int bi = hit ? __ffs(hit) - 1 : 0;
        const int bsrc = __shfl_sync(full, orig, bi);
        if (hit != 0u) {
            T row[NG];
            pick_row<T, NG, RPW>(v, bi, row);
#pragma unroll
            for (int c = 0; c < NG; ++c) S.cand[par][warp][lane + 32 * c] = row[c];
        }
        if (lane == 0) {
            S.wkey[par][warp] = wmax;
            S.wrow[par][warp] = rbase + bi;
            S.wsrc[par][warp] = bsrc;
        }
        const bool holds_j = j >= rbase && j < rbase + RPW;
        const int ij = j - rbase;
        const int jsrc = __shfl_sync(full, orig, holds_j ? ij : 0);
        if (holds_j) {
            T row[NG];
            pick_row<T, NG, RPW>(v, ij, row);
#pragma unroll
            for (int c = 0; c < NG; ++c) S.rowj_loc[par][lane + 32 * c] = row[c];
            if (lane == 0) S.rowj_src_loc[par] = jsrc;
        }
        __syncthreads();
        // b. push: warps 0-3 the CTA's candidate, warps 4-7 of the CTA holding row j that
        //    row; a row is 512 bytes, and thread t stores its float4 t % 32 into CTAs
        //    t / 32 % 4, + 4, + 8, + 12
        if (warp < 8) {
            const int t = tid & 127, f = t & 31, c0 = t >> 5;
            if (warp < 4) {
                const Key kw = lane < kPcWarps ? S.wkey[par][lane] : Key(0);
                const Key m = warp_key_max(kw);
                const unsigned h = __ballot_sync(full, m != Key(0) && kw == m);
                const int w = h ? __ffs(h) - 1 : 0;
                const float4 val = reinterpret_cast<const float4*>(S.cand[par][w])[f];
                const int prow_r = S.wrow[par][w], prow_s = S.wsrc[par][w];
#pragma unroll
                for (int u = 0; u < kPcMaxCtas / 4; ++u) {
                    const int c = c0 + 4 * u;
                    if (c < nc) {
                        PanelShared<T>* R = cl.map_shared_rank(&S, c);
                        reinterpret_cast<float4*>(R->slot[par][q])[f] = val;
                        if (f == 0) {
                            R->slot_key[par][q] = m;
                            R->slot_row[par][q] = prow_r;
                            R->slot_src[par][q] = prow_s;
                        }
                    }
                }
            } else if (q == j / (kPcWarps * RPW)) {
                const float4 val = reinterpret_cast<const float4*>(S.rowj_loc[par])[f];
                const int js = S.rowj_src_loc[par];
#pragma unroll
                for (int u = 0; u < kPcMaxCtas / 4; ++u) {
                    const int c = c0 + 4 * u;
                    if (c < nc) {
                        PanelShared<T>* R = cl.map_shared_rank(&S, c);
                        reinterpret_cast<float4*>(R->rowj[par])[f] = val;
                        if (f == 0) R->rowj_src[par] = js;
                    }
                }
            }
        }
        cl.sync();
        // d. the cluster's pivot, from this CTA's own slots (every warp)
        const Key ks = lane < nc ? S.slot_key[par][lane] : Key(0);
        const Key m = warp_key_max(ks);
        const unsigned h = __ballot_sync(full, m != Key(0) && ks == m);
        const int o = h ? __ffs(h) - 1 : 0;  // the lowest CTA with the maximum
        const T* prow = m != Key(0) ? S.slot[par][o] : S.rowj[par];
        const int p = m != Key(0) ? S.slot_row[par][o] : j;  // no candidate: row j stays the pivot row
        if (p != j) {
            if (holds_j) {  // row j takes the pivot row
                T row[NG];
#pragma unroll
                for (int c = 0; c < NG; ++c) row[c] = prow[lane + 32 * c];
                put_row<T, NG, RPW>(v, ij, row);
                if (lane == ij) orig = S.slot_src[par][o];
            }
            if (p >= rbase && p < rbase + RPW) {  // row p takes row j
                T row[NG];
#pragma unroll
                for (int c = 0; c < NG; ++c) row[c] = S.rowj[par][lane + 32 * c];
                put_row<T, NG, RPW>(v, p - rbase, row);
                if (lane == p - rbase) orig = S.rowj_src[par];
            }
        }
        const T pv = prow[j];
        if (tid == 0) {
            S.piv[j] = k + p;
            if (pv == T(0) && S.info == 0) S.info = k + j + 1;
        }
        if (pv != T(0)) {
            T pc[NG];
#pragma unroll
            for (int c = 0; c < NG; ++c) pc[c] = prow[lane + 32 * c];
            if (PanelType<T>::normal(pv))  // getrf's sfmin test
                panel_update<T, NG, RPW, G, false>(v, rbase, rows, j, jj, lane, T(1) / pv, pc);
            else
                panel_update<T, NG, RPW, G, true>(v, rbase, rows, j, jj, lane, pv, pc);
        }
    }
}

// swaps (may be null: the FP64 path derives the moves from the pivots instead) receives
// the moved rows; run_flag (may be null): every CTA returns at once when *run_flag == 0.
template <typename T, int RPW>
__global__ void __launch_bounds__(kPcThreads, 1)
    lu_panel_cluster_kernel(T* __restrict__ a, int n, int k, int kb, int32_t* __restrict__ piv,
                            int* __restrict__ info, int* __restrict__ swaps, const int* __restrict__ run_flag) {
    if (run_flag != nullptr && *run_flag == 0) return;  // the same for every CTA of the cluster
    constexpr int NG = PanelType<T>::NG;
    cg::cluster_group cl = cg::this_cluster();
    __shared__ __align__(16) PanelShared<T> S;
    const int q = (int)cl.block_rank(), nc = (int)cl.num_blocks();
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int rows = n - k;
    const int rbase = (q * kPcWarps + warp) * RPW;  // the warp's first panel row
    const unsigned full = 0xffffffffu;
    if (tid == 0) S.info = 0;

    T v[RPW][NG];
#pragma unroll
    for (int i = 0; i < RPW; ++i) {
        const bool has = rbase + i < rows;
        const T* src = a + (int64_t)(k + (has ? rbase + i : 0)) * n + k + lane;
#pragma unroll
        for (int c = 0; c < NG; ++c) v[i][c] = (has && lane + 32 * c < kb) ? src[32 * c] : T(0);
    }
    int orig = rbase + lane;  // lanes < RPW: original panel row of the warp's row `lane`
    cl.sync();                // every CTA of the cluster runs before any shared memory is written remotely

    panel_columns<T, RPW, 0>(v, orig, k, kb, rows, q, nc, tid, cl, S);
    panel_columns<T, RPW, 1>(v, orig, k, kb, rows, q, nc, tid, cl, S);
    if constexpr (NG > 2) {
        panel_columns<T, RPW, 2>(v, orig, k, kb, rows, q, nc, tid, cl, S);
        panel_columns<T, RPW, 3>(v, orig, k, kb, rows, q, nc, tid, cl, S);
    }
#pragma unroll
    for (int i = 0; i < RPW; ++i) {
        if (rbase + i < rows) {
            T* dst = a + (int64_t)(k + rbase + i) * n + k + lane;
#pragma unroll
            for (int c = 0; c < NG; ++c)
                if (lane + 32 * c < kb) dst[32 * c] = v[i][c];
        }
    }
    // the moved rows, in row order: (destination, source) global rows
    const bool moved = lane < RPW && rbase + lane < rows && orig != rbase + lane;
    const unsigned mb = __ballot_sync(full, moved);
    if (lane == 0) S.wcnt[warp] = __popc(mb);
    __syncthreads();  // also orders the last column's piv and info before their reads
    if (q == 0) {
        for (int j = tid; j < kb; j += kPcThreads) piv[k + j] = S.piv[j];
        if (tid == 0 && S.info != 0 && *info == 0) *info = S.info;
    }
    if (warp == 0) {
        const int cw = lane < kPcWarps ? S.wcnt[lane] : 0;
        int inc = cw;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int y = __shfl_up_sync(full, inc, off);
            if (lane >= off) inc += y;
        }
        if (lane < kPcWarps) S.wcnt[lane] = inc - cw;  // exclusive prefix over the warps
        if (lane == 31) S.cnt = inc;
    }
    cl.sync();  // every CTA's count is published
    if (tid == 0) {
        int off = 0;
        for (int c = 0; c < q; ++c) off += cl.map_shared_rank(&S, c)->cnt;
        S.off = off;
        if (q == nc - 1 && swaps != nullptr) swaps[0] = off + S.cnt;
    }
    __syncthreads();
    if (moved && swaps != nullptr) {
        const int e = S.off + S.wcnt[warp] + __popc(mb & ((1u << lane) - 1u));
        swaps[1 + 2 * e] = k + rbase + lane;
        swaps[2 + 2 * e] = k + orig;
    }
    cl.sync();  // no CTA exits while another may still read its shared memory
}

// The outer panel's row permutation (lu_panel_cluster_kernel's list) for every column
// outside the panel: a CTA takes 32 columns, loads every listed source row's values into
// shared memory, then stores them to their destinations (all loads before any store, so
// the permutation's cycles need no order).
__global__ void __launch_bounds__(256) lu_swap_rows_kernel(float* __restrict__ a, int n, int k, int kb,
                                                           const int* __restrict__ swaps) {
    __shared__ int s_dst[2 * kTcBlk], s_src[2 * kTcBlk];
    __shared__ float tile[2 * kTcBlk][33];
    const int cnt = min(swaps[0], 2 * kTcBlk);
    for (int e = threadIdx.x; e < cnt; e += blockDim.x) {
        s_dst[e] = swaps[1 + 2 * e];
        s_src[e] = swaps[2 + 2 * e];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int c = blockIdx.x * 32 + lane;
    const bool col = c < n && (c < k || c >= k + kb);
    for (int e = warp; e < cnt; e += 8)
        if (col) tile[e][lane] = a[(int64_t)s_src[e] * n + c];
    __syncthreads();
    for (int e = warp; e < cnt; e += 8)
        if (col) a[(int64_t)s_dst[e] * n + c] = tile[e][lane];
}

// The largest cluster of lu_panel_cluster_kernel<T> CTAs the device runs (16 where the
// non-portable size is allowed, else 8; 0 if none), checked once per element type.
template <typename T>
static int cluster_panel_max() {
    static std::once_flag once;
    static int best = 0;
    std::call_once(once, [] {
        for (int size : {16, 8}) {
            const void* fn = size == 16 ? (const void*)lu_panel_cluster_kernel<T, 8> : (const void*)lu_panel_cluster_kernel<T, 16>;
            if (size == 16 && cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
                cudaGetLastError();
                continue;
            }
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3((unsigned)size);
            cfg.blockDim = dim3(kPcThreads);
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = (unsigned)size;
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            int clusters = 0;
            const cudaError_t e = size == 16 ? cudaOccupancyMaxActiveClusters(&clusters, lu_panel_cluster_kernel<T, 8>, &cfg)
                                             : cudaOccupancyMaxActiveClusters(&clusters, lu_panel_cluster_kernel<T, 16>, &cfg);
            cudaGetLastError();
            if (e == cudaSuccess && clusters > 0) {
                best = size;
                break;
            }
        }
    });
    return best;
}

// Rows of the outer panel one cluster takes: 16 CTAs of 8-row warps, or 8 CTAs of
// 16-row warps.
template <typename T>
static int cluster_panel_rows() {
    const int m = cluster_panel_max<T>();
    return m == 16 ? 16 * 8 * kPcWarps : m == 8 ? 8 * 16 * kPcWarps : 0;
}

// One cluster panel launch with RPW rows per warp: nc CTAs of kPcWarps warps.
template <typename T, int RPW>
static int launch_cluster_rpw(T* a, int n, int k, int kb, int32_t* piv, int* info, int* swaps, const int* run_flag,
                              int nc, cudaStream_t s) {
    if (nc > 8) {  // non-portable cluster size: allowed once per instantiation
        static std::once_flag once;
        static cudaError_t e = cudaSuccess;
        std::call_once(once, [] {
            e = cudaFuncSetAttribute((const void*)lu_panel_cluster_kernel<T, RPW>,
                                     cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        });
        FJ_CUDA(e);
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)nc);
    cfg.blockDim = dim3(kPcThreads);
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)nc;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    FJ_CUDA(cudaLaunchKernelEx(&cfg, lu_panel_cluster_kernel<T, RPW>, a, n, k, kb, piv, info, swaps, run_flag));
    note_launch();
    return FJ_OK;
}

// The cluster panel at column k (kb columns, n - k <= cluster_panel_rows<T>() rows), with
// the fewest rows per warp (2, 4, 8 or 16) whose cluster the device runs: a column's
// serial work in a warp grows with its rows (8-CTA clusters of 16-row warps factor the
// 2048-row AIC 18 % slower than 16-CTA clusters of 8-row warps).
template <typename T>
static int launch_cluster_panel(T* a, int n, int k, int kb, int32_t* piv, int* info, int* swaps,
                                const int* run_flag, cudaStream_t s) {
    const int max_nc = cluster_panel_max<T>();
    const int rows = n - k;
    int rpw = 2;
    while (rpw < 16 && (rows + kPcWarps * rpw - 1) / (kPcWarps * rpw) > max_nc) rpw *= 2;
    const int nc = (rows + kPcWarps * rpw - 1) / (kPcWarps * rpw);
    if (nc > max_nc || nc < 1) return fail(FJ_ERR_UNSUPPORTED, "cluster panel: %d rows", rows);
    switch (rpw) {
        case 2: return launch_cluster_rpw<T, 2>(a, n, k, kb, piv, info, swaps, run_flag, nc, s);
        case 4: return launch_cluster_rpw<T, 4>(a, n, k, kb, piv, info, swaps, run_flag, nc, s);
        case 8: return launch_cluster_rpw<T, 8>(a, n, k, kb, piv, info, swaps, run_flag, nc, s);
        default: return launch_cluster_rpw<T, 16>(a, n, k, kb, piv, info, swaps, run_flag, nc, s);
    }
}

static int launch_panel_cluster(float* a, int n, int k, int kb, int32_t* piv, int* info, int* swaps,
                                cudaStream_t s) {
    FJ_TRY(launch_cluster_panel<float>(a, n, k, kb, piv, info, swaps, nullptr, s));
    lu_swap_rows_kernel<<<(unsigned)((n + 31) / 32), 256, 0, s>>>(a, n, k, kb, swaps);
    note_launch();
    return FJ_OK;
}

// U12 = L11^-1 A12 for the mixed factorisation's outer panel at column k (kb <= 128
// rows, L11 unit lower from the factored panel), in place on the columns [c0, n).  A CTA
// of 16 warps takes 16 columns: L11 and the columns' panel rows come into shared memory
// (coalesced), then warp w substitutes column w, lane l holding rows l + 32 q (q < 4) in
// registers, each x_j reaching every lane by a shuffle.  Forward substitution in FP32,
// as the CUDA-core path's lu_swap_trsm_kernel computes its U rows.
constexpr int kTrsmCols = 16;
constexpr size_t kTrsm32Smem = (size_t)(kTcBlk * (kTcBlk + 1) + kTcBlk * (kTrsmCols + 1)) * sizeof(float);

__device__ __forceinline__ float pick4f(const float (&v)[4], int q) {
    return q == 0 ? v[0] : q == 1 ? v[1] : q == 2 ? v[2] : v[3];
}

constexpr int kTrsmThreads = 32 * kTrsmCols;

__global__ void __launch_bounds__(kTrsmThreads) lu_trsm32_kernel(float* __restrict__ a, int n, int k, int kb, int c0) {
    extern __shared__ __align__(16) float smt[];
    float* ls = smt;                               // [128][129]
    float* xs = smt + kTcBlk * (kTcBlk + 1);       // [128][17]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int cb = c0 + blockIdx.x * kTrsmCols;
    for (int idx = threadIdx.x; idx < kTcBlk * kTcBlk; idx += blockDim.x) {
        const int r = idx >> 7, j = idx & 127;
        ls[r * (kTcBlk + 1) + j] = (r < kb && j < r) ? a[(int64_t)(k + r) * n + k + j] : 0.0f;
    }
    for (int idx = threadIdx.x; idx < kTcBlk * kTrsmCols; idx += blockDim.x) {
        const int r = idx / kTrsmCols, cc = idx % kTrsmCols, col = cb + cc;
        xs[r * (kTrsmCols + 1) + cc] = (r < kb && col < n) ? a[(int64_t)(k + r) * n + col] : 0.0f;
    }
    __syncthreads();
    const unsigned full = 0xffffffffu;
    {
        const int cc = warp;
        float x[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) x[q] = xs[(lane + 32 * q) * (kTrsmCols + 1) + cc];
#pragma unroll 4
        for (int j = 0; j < kb - 1; ++j) {
            const float xj = __shfl_sync(full, pick4f(x, j >> 5), j & 31);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int r = lane + 32 * q;
                if (r > j) x[q] -= ls[r * (kTcBlk + 1) + j] * xj;  // rows >= kb: zero multipliers
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) xs[(lane + 32 * q) * (kTrsmCols + 1) + cc] = x[q];
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < kTcBlk * kTrsmCols; idx += blockDim.x) {
        const int r = idx / kTrsmCols, cc = idx % kTrsmCols, col = cb + cc;
        if (r >= 1 && r < kb && col < n) a[(int64_t)(k + r) * n + col] = xs[r * (kTrsmCols + 1) + cc];
    }
}

// The factorisation's and the inverse's products: the TMA-fed tensor-core GEMM, its
// operand split in the scratch that follows the diagonal-block inverses.
static int tc_mul(const float* a, int lda, const float* b, int ldb, float* c, int ldc, int m, int n, int k,
                  float alpha, float beta, int passes, float* tri, int nn, int* d_err, cudaStream_t s) {
    return tc_gemm_tf32_tma(a, lda, b, ldb, c, ldc, m, n, k, alpha, beta, passes, tri + tc_inv_floats(nn),
                            tc_scratch_floats(nn), d_err, s);
}

template <int NB>
static int lu_factor32_tc_impl(float* a, int n, int32_t* piv, int* d_info, int* d_err, float* tri_l, int passes,
                               cudaStream_t s) {
    static_assert(kTcBlk % NB == 0, "inner panels tile the outer one");
    if (n <= 0) return fail(FJ_ERR_SHAPE, "lu_factor: n=%d", n);
    const size_t smem = (size_t)n * (NB + 1) * sizeof(float);
    if (smem > 220 * 1024) return fail(FJ_ERR_UNSUPPORTED, "lu_factor: n=%d too large for the shared-memory panel", n);
    FJ_TRY(allow_dynamic_smem((const void*)lu_panel_kernel<float, NB>, smem));
    FJ_TRY(allow_dynamic_smem((const void*)lu_panel_reg_kernel<float, NB, 1>, smem));
    FJ_TRY(allow_dynamic_smem((const void*)lu_panel_reg_kernel<float, NB, 2>, smem));
    FJ_TRY(allow_dynamic_smem((const void*)lu_trsm32_kernel, kTrsm32Smem));
    FJ_CUDA(cudaMemsetAsync(d_info, 0, sizeof(int), s));
    int* swaps = reinterpret_cast<int*>(tri_l + tc_inv_floats(n) + tc_scratch_floats(n));
    const int cluster_rows = cluster_panel_rows<float>();
    for (int k = 0; k < n; k += kTcBlk) {
        const int kb = min(kTcBlk, n - k), ke = k + kb;
        if (n - k <= cluster_rows) {
            FJ_TRY(launch_panel_cluster(a, n, k, kb, piv, d_info, swaps, s));
        } else {
          for (int j = k; j < ke; j += NB) {
            const int nb = min(NB, n - j);
            launch_panel<float, NB>(a, n, j, piv, d_info, nullptr, s);
            if (n > nb) {
                lu_swap_trsm_kernel<float, NB><<<(n + 255) / 256, 256, 0, s>>>(a, n, j, piv, ke, nullptr);
                note_launch();
            }
            const int rows = n - j - nb, cols = ke - j - nb;
            if (nb == NB && rows > 0 && cols > 0) {
                lu_update_kernel<float, NB><<<dim3((cols + 63) / 64, (rows + 63) / 64), 256, 0, s>>>(a, n, j, ke, nullptr);
                note_launch();
            }
          }
        }
        const int rest = n - ke;
        if (rest > 0) {  // U12 = L11^-1 A12 (CUDA cores), then A22 -= L21 U12 (tensor cores)
            float* a12 = a + (int64_t)k * n + ke;
            lu_trsm32_kernel<<<(unsigned)((rest + kTrsmCols - 1) / kTrsmCols), kTrsmThreads, kTrsm32Smem, s>>>(a, n, k,
                                                                                                          kb, ke);
            note_launch();
            FJ_TRY(tc_mul(a + (int64_t)ke * n + k, n, a12, n, a + (int64_t)ke * n + ke, n, rest, rest, kb, -1.0f, 1.0f,
                          passes, tri_l, n, d_err, s));
        }
    }
    FJ_LAUNCH_CHECK("lu_factor32_tc");
    return FJ_OK;
}

int lu_factor32_tc(float* a, int n, int32_t* piv, int* d_info, int* d_err, float* tri_l, int passes,
                   cudaStream_t s) {
    if (panel_fits<float>(n, 16)) return lu_factor32_tc_impl<16>(a, n, piv, d_info, d_err, tri_l, passes, s);
    return lu_factor32_tc_impl<8>(a, n, piv, d_info, d_err, tri_l, passes, s);
}

// Y = P I: row i holds a one in column perm[i].  Y must be zero on entry.
__global__ void __launch_bounds__(1024) perm_identity_kernel(const int32_t* __restrict__ piv, int n,
                                                             float* __restrict__ y) {
    extern __shared__ int perm_sm[];  // n permutation entries, then n pivots
    int* sp = perm_sm + n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        perm_sm[i] = i;
        sp[i] = piv[i];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 0; i < n; ++i) {
            const int p = sp[i];
            if (p != i) {
                const int t = perm_sm[i];
                perm_sm[i] = perm_sm[p];
                perm_sm[p] = t;
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) y[(int64_t)i * n + perm_sm[i]] = 1.0f;
}

int lu_inverse32_tc(const float* lu, int n, const int32_t* piv, float* x, float* tri, int passes, int* d_err,
                    cudaStream_t s) {
    const int nblk = (n + kTcBlk - 1) / kTcBlk;
    float* tri_l = tri;
    float* tri_u = tri + (size_t)nblk * kTcBlk * kTcBlk;
    // the diagonal blocks' inverses, L's and U's, each set in one launch (a CTA per block);
    // L's blocks are final once their panel is factored (later swaps touch lower rows only)
    FJ_TRY(tri_inverse32_blocks(lu, n, 0, nblk, false, tri_l, s));
    FJ_TRY(tri_inverse32_blocks(lu, n, 0, nblk, true, tri_u, s));
    FJ_CUDA(cudaMemsetAsync(x, 0, (size_t)n * n * sizeof(float), s));
    FJ_TRY(allow_dynamic_smem((const void*)perm_identity_kernel, (size_t)2 * n * sizeof(int)));
    perm_identity_kernel<<<1, 1024, (size_t)2 * n * sizeof(int), s>>>(piv, n, x);
    note_launch();
    FJ_LAUNCH_CHECK("perm_identity_kernel");
    for (int b = 0; b < nblk; ++b) {  // forward: unit lower
        const int i0 = b * kTcBlk, ib = min(kTcBlk, n - i0), below = n - i0 - ib;
        float* yi = x + (int64_t)i0 * n;
        FJ_TRY(tc_mul(tri_l + (size_t)b * kTcBlk * kTcBlk, kTcBlk, yi, n, yi, n, ib, n, ib, 1.0f, 0.0f, passes, tri,
                      n, d_err, s));
        if (below > 0)
            FJ_TRY(tc_mul(lu + (int64_t)(i0 + ib) * n + i0, n, yi, n, yi + (int64_t)ib * n, n, below, n, ib, -1.0f,
                          1.0f, passes, tri, n, d_err, s));
    }
    for (int b = nblk - 1; b >= 0; --b) {  // backward: upper
        const int i0 = b * kTcBlk, ib = min(kTcBlk, n - i0);
        float* yi = x + (int64_t)i0 * n;
        FJ_TRY(tc_mul(tri_u + (size_t)b * kTcBlk * kTcBlk, kTcBlk, yi, n, yi, n, ib, n, ib, 1.0f, 0.0f, passes, tri,
                      n, d_err, s));
        if (i0 > 0) FJ_TRY(tc_mul(lu + i0, n, yi, n, x, n, i0, n, ib, -1.0f, 1.0f, passes, tri, n, d_err, s));
    }
    return FJ_OK;
}

// ---------------------------------------------------------------------------------
// FP64 factorisation (the plain path's getrf), blocked twice.  Outer panels of kDB = 64
// columns; where a panel's rows fit one cluster (n - k <= cluster_panel_rows<double>())
// one lu_panel_cluster_kernel<double> launch factors it, else 2- to 8-column panels do,
// with their U rows and updates confined to the outer panel.  Then
//   lu_swap_trsm64_kernel: the outer panel's row swaps for every column outside it, and
//                          U12 = L11^-1 A12 for the columns to its right;
//   lu_gemm64_kernel:      A22 -= L21 U12 (K = 64, FP64 FMA).
// Pivots are getrf's (first maximum of the column below the diagonal); the trailing
// matrix is updated once per 64 columns instead of once per column, so the factors
// differ from a column-by-column getrf only by rounding.
constexpr int kDB = 64;

// The composed row moves of the outer panel at column k, from its kb pivots applied in
// order (getrf's laswp): map[i] = the panel row whose values end at panel row i.  A move
// lands on a row < k + kb, or on a pivot row at or below k + kb.  For the columns outside
// the panel each CTA (32 columns, one per lane) loads every moved value before it stores
// any.  Then, for the CTA's columns right of the panel, the kb x kb unit-lower L11 solves
// its rows k .. k + kb: warp w (of 16) takes columns 2w and 2w + 1, lane l rows l and l + 32.
constexpr int kSwapTrsm64Warps = 16;

__global__ void __launch_bounds__(32 * kSwapTrsm64Warps)
    lu_swap_trsm64_kernel(double* __restrict__ a, int n, int k, int kb, const int32_t* __restrict__ piv,
                          int do_swaps, const int* __restrict__ run_flag) {
    if (run_flag != nullptr && *run_flag == 0) return;
    extern __shared__ __align__(16) unsigned char sm64[];
    double* tile = reinterpret_cast<double*>(sm64);            // [2 kDB][32] moved values; then x [kDB][33]
    double* ls = tile + 2 * kDB * 33;                          // [kDB][kDB + 1] L11
    int* map = reinterpret_cast<int*>(ls + kDB * (kDB + 1));  // [n - k]
    __shared__ int s_dst[2 * kDB], s_src[2 * kDB];
    __shared__ int s_cnt;
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int rows = n - k, c0 = blockIdx.x * 32, c = c0 + lane;
    if (do_swaps) {
        for (int i = threadIdx.x; i < rows; i += blockDim.x) map[i] = i;
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int j = 0; j < kb; ++j) {
                const int p = piv[k + j] - k;
                if (p != j && p > j && p < rows) {
                    const int t = map[j];
                    map[j] = map[p];
                    map[p] = t;
                }
            }
        }
        __syncthreads();
        if (warp == 0) {  // the moves, listed: rows [0, kb), then the pivot rows at or below kb
            int base = 0;
            for (int e0 = 0; e0 < 2 * kb; e0 += 32) {
                const int e = e0 + lane;
                int pos = -1;
                if (e < kb) {
                    pos = e;
                } else if (e < 2 * kb) {
                    const int p = piv[k + e - kb] - k;
                    if (p >= kb && p < rows) pos = p;
                }
                const bool mv = pos >= 0 && map[pos] != pos;
                const unsigned m = __ballot_sync(full, mv);
                if (mv) {
                    const int o = base + __popc(m & ((1u << lane) - 1u));
                    s_dst[o] = k + pos;
                    s_src[o] = k + map[pos];
                }
                base += __popc(m);
            }
            if (lane == 0) s_cnt = base;
        }
        __syncthreads();
        const int cnt = s_cnt;
        const bool col = c < n && (c < k || c >= k + kb);
        for (int e = warp; e < cnt; e += kSwapTrsm64Warps)
            if (col) tile[e * 32 + lane] = a[(int64_t)s_src[e] * n + c];
        __syncthreads();
        for (int e = warp; e < cnt; e += kSwapTrsm64Warps)
            if (col) a[(int64_t)s_dst[e] * n + c] = tile[e * 32 + lane];
        __syncthreads();  // the CTA's stores are seen by its loads below
    }
    if (c0 + 31 < k + kb || kb < 2) return;  // no column right of the panel (uniform over the CTA)
    for (int idx = threadIdx.x; idx < kDB * kDB; idx += blockDim.x) {
        const int r = idx / kDB, j = idx % kDB;
        ls[r * (kDB + 1) + j] = (r < kb && j < r) ? a[(int64_t)(k + r) * n + k + j] : 0.0;
    }
    double* xs = tile;
    for (int idx = threadIdx.x; idx < kDB * 32; idx += blockDim.x) {
        const int r = idx >> 5, cc = idx & 31, cg_ = c0 + cc;
        xs[r * 33 + cc] = (r < kb && cg_ >= k + kb && cg_ < n) ? a[(int64_t)(k + r) * n + cg_] : 0.0;
    }
    __syncthreads();
#pragma unroll 1
    for (int t = 0; t < 2; ++t) {
        const int cc = warp * 2 + t;
        double x0 = xs[lane * 33 + cc], x1 = xs[(lane + 32) * 33 + cc];
#pragma unroll 4
        for (int j = 0; j < kb - 1; ++j) {
            const double xj = __shfl_sync(full, j < 32 ? x0 : x1, j & 31);
            if (lane > j) x0 -= ls[lane * (kDB + 1) + j] * xj;
            x1 -= ls[(lane + 32) * (kDB + 1) + j] * xj;  // rows >= kb: zero multipliers
        }
        xs[lane * 33 + cc] = x0;
        xs[(lane + 32) * 33 + cc] = x1;
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < kDB * 32; idx += blockDim.x) {
        const int r = idx >> 5, cc = idx & 31, cg_ = c0 + cc;
        if (r >= 1 && r < kb && cg_ >= k + kb && cg_ < n) a[(int64_t)(k + r) * n + cg_] = xs[r * 33 + cc];
    }
}

constexpr size_t kSwapTrsm64Fixed = (size_t)(2 * kDB * 33 + kDB * (kDB + 1)) * sizeof(double);

// A22 -= L21 U12 with K = kDB, on one 64 x 64 tile of the trailing matrix per CTA: the
// CTA's 64 rows of L21 and 64 columns of U12 come into shared memory (cp.async, zero past
// the matrix), then thread (tx, ty) updates rows ty + 16 p and columns tx + 16 q (p, q < 4)
// with the 64 products in order, as the column-by-column update would.
__global__ void __launch_bounds__(256)
    lu_gemm64_kernel(double* __restrict__ a, int n, int k, const int* __restrict__ run_flag) {
    if (run_flag != nullptr && *run_flag == 0) return;
    extern __shared__ __align__(16) unsigned char smg64[];
    double* as = reinterpret_cast<double*>(smg64);  // [64][kDB]: L21 rows
    double* bs = as + 64 * kDB;                      // [kDB][64]: U12 columns
    const int k2 = k + kDB;
    const int r0 = k2 + blockIdx.y * 64, c0 = k2 + blockIdx.x * 64;
    for (int idx = threadIdx.x; idx < 64 * kDB; idx += blockDim.x) {
        const int r = idx / kDB, j = idx % kDB;
        const bool oka = r0 + r < n;
        const double* srca = a + (int64_t)(oka ? r0 + r : 0) * n + k + j;
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"((unsigned)__cvta_generic_to_shared(as + idx)),
                     "l"(srca), "r"(oka ? 8 : 0)
                     : "memory");
        const int jb = idx / 64, cb = idx % 64;
        const bool okb = c0 + cb < n;
        const double* srcb = a + (int64_t)(k + jb) * n + (okb ? c0 + cb : 0);
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"((unsigned)__cvta_generic_to_shared(bs + idx)),
                     "l"(srcb), "r"(okb ? 8 : 0)
                     : "memory");
    }
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    double acc[4][4];
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = r0 + ty + 16 * p, cc = c0 + tx + 16 * q;
            acc[p][q] = (r < n && cc < n) ? a[(int64_t)r * n + cc] : 0.0;
        }
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
#pragma unroll 8
    for (int j = 0; j < kDB; ++j) {
        double ar[4], br[4];
#pragma unroll
        for (int p = 0; p < 4; ++p) ar[p] = as[(ty + 16 * p) * kDB + j];
#pragma unroll
        for (int q = 0; q < 4; ++q) br[q] = bs[j * 64 + tx + 16 * q];
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[p][q] -= ar[p] * br[q];
    }
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = r0 + ty + 16 * p, cc = c0 + tx + 16 * q;
            if (r < n && cc < n) a[(int64_t)r * n + cc] = acc[p][q];
        }
}

constexpr size_t kGemm64Smem = (size_t)2 * 64 * kDB * sizeof(double);

// The outer panel at column k in NB-column panels (rows beyond one cluster): swaps over
// every column, U rows and updates inside the outer panel [k, ke).
template <int NB>
static int lu_outer_panel_narrow64(double* a, int n, int k, int ke, int32_t* piv, int* d_info, const int* run_flag,
                                   cudaStream_t s) {
    const size_t smem = (size_t)n * (NB + 1) * sizeof(double);
    FJ_TRY(allow_dynamic_smem((const void*)lu_panel_kernel<double, NB>, smem));
    FJ_TRY(allow_dynamic_smem((const void*)lu_panel_reg_kernel<double, NB, 1>, smem));
    FJ_TRY(allow_dynamic_smem((const void*)lu_panel_reg_kernel<double, NB, 2>, smem));
    for (int j = k; j < ke; j += NB) {
        const int nb = min(NB, n - j);
        launch_panel<double, NB>(a, n, j, piv, d_info, run_flag, s);
        if (n > nb) {
            lu_swap_trsm_kernel<double, NB><<<(n + 255) / 256, 256, 0, s>>>(a, n, j, piv, ke, run_flag);
            note_launch();
        }
        const int rows = n - j - nb, cols = ke - j - nb;
        if (nb == NB && rows > 0 && cols > 0) {
            lu_update_kernel<double, NB><<<dim3((cols + 63) / 64, (rows + 63) / 64), 256, 0, s>>>(a, n, j, ke, run_flag);
            note_launch();
        }
    }
    return FJ_OK;
}

int lu_factor64(double* a, int n, int32_t* piv, int* d_info, cudaStream_t s, const int* run_flag) {
    if (n <= 0) return fail(FJ_ERR_SHAPE, "lu_factor: n=%d", n);
    int nb_narrow = 0;
    for (int nb : {8, 4, 2})
        if (nb_narrow == 0 && panel_fits<double>(n, nb)) nb_narrow = nb;
    const int cluster_rows = cluster_panel_rows<double>();
    if (nb_narrow == 0 && n > cluster_rows)
        return fail(FJ_ERR_UNSUPPORTED, "lu_factor: n=%d too large for the shared-memory panel", n);
    const size_t st_smem = kSwapTrsm64Fixed + (size_t)n * sizeof(int);
    FJ_TRY(allow_dynamic_smem((const void*)lu_swap_trsm64_kernel, st_smem));
    FJ_TRY(allow_dynamic_smem((const void*)lu_gemm64_kernel, kGemm64Smem));
    FJ_CUDA(cudaMemsetAsync(d_info, 0, sizeof(int), s));
    for (int k = 0; k < n; k += kDB) {
        const int kb = min(kDB, n - k), ke = k + kb;
        const bool cluster = n - k <= cluster_rows;
        if (cluster) {
            FJ_TRY(launch_cluster_panel<double>(a, n, k, kb, piv, d_info, nullptr, run_flag, s));
        } else if (nb_narrow == 8) {
            FJ_TRY(lu_outer_panel_narrow64<8>(a, n, k, ke, piv, d_info, run_flag, s));
        } else if (nb_narrow == 4) {
            FJ_TRY(lu_outer_panel_narrow64<4>(a, n, k, ke, piv, d_info, run_flag, s));
        } else {
            FJ_TRY(lu_outer_panel_narrow64<2>(a, n, k, ke, piv, d_info, run_flag, s));
        }
        if (n > kb) {
            lu_swap_trsm64_kernel<<<(unsigned)((n + 31) / 32), 32 * kSwapTrsm64Warps, st_smem, s>>>(
                a, n, k, kb, piv, cluster ? 1 : 0, run_flag);
            note_launch();
        }
        const int rest = n - ke;
        if (rest > 0) {  // kb == kDB here
            lu_gemm64_kernel<<<dim3((unsigned)((rest + 63) / 64), (unsigned)((rest + 63) / 64)), 256, kGemm64Smem, s>>>(
                a, n, k, run_flag);
            note_launch();
        }
    }
    FJ_LAUNCH_CHECK("lu_factor64");
    return FJ_OK;
}

// Factor path of the mixed solve.  FJ_MIXED_FACTOR selects it: "cuda" (FP32 CUDA cores),
// "tf32" (tensor cores, one TF32 pass) or the default "tf32x3" (three-pass split); the
// tensor-core paths apply from n >= kTcMinN.
constexpr int kTcMinN = 256;

int factor_inverse32(const double* a64, int n, float* a32, int32_t* piv, int* flags, float* x32, float* tri,
                     cudaStream_t s) {
    int passes = 3;
    if (const char* e = getenv("FJ_MIXED_FACTOR")) {
        if (!strcmp(e, "cuda")) passes = 0;
        else if (!strcmp(e, "tf32")) passes = 1;
        else if (strcmp(e, "tf32x3") != 0) return fail(FJ_ERR_SHAPE, "FJ_MIXED_FACTOR=%s (cuda, tf32 or tf32x3)", e);
    }
    FJ_TRY(convert64to32(a64, a32, (int64_t)n * n, s));
    if (passes == 0 || n < kTcMinN) {
        FJ_TRY(lu_factor32(a32, n, piv, flags, s));
        return lu_inverse32(a32, n, piv, x32, s);
    }
    FJ_CUDA(cudaMemsetAsync(flags + 3, 0, sizeof(int), s));
    FJ_TRY(lu_factor32_tc(a32, n, piv, flags, flags + 3, tri, passes, s));
    return lu_inverse32_tc(a32, n, piv, x32, tri, passes, flags + 3, s);
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
// Row dot products of the refinement (HBM-bound: one pass over the matrix row).  A warp
// takes a row; where the row and the vector are 16-byte aligned and n a multiple of 4 (2
// for FP64 rows) each lane loads whole 16-byte vectors, four in flight, into four
// independent FP64 partial sums; else element by element.  The warp's sum comes back in
// every lane.
__device__ __forceinline__ double warp_sum(double a) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) a += __shfl_xor_sync(0xffffffffu, a, off);
    return a;
}

__device__ __forceinline__ double row_dot32(const float* __restrict__ xr, const double* __restrict__ v, int n,
                                            int lane) {
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    if ((n & 3) == 0 && (((uintptr_t)xr | (uintptr_t)v) & 15) == 0) {
        const float4* x4 = reinterpret_cast<const float4*>(xr);
        const double2* v2 = reinterpret_cast<const double2*>(v);
        const int n4 = n >> 2;
#pragma unroll 4
        for (int j = lane; j < n4; j += 32) {
            const float4 x = __ldg(x4 + j);
            const double2 p = v2[2 * j], q = v2[2 * j + 1];
            a0 = fma((double)x.x, p.x, a0);
            a1 = fma((double)x.y, p.y, a1);
            a2 = fma((double)x.z, q.x, a2);
            a3 = fma((double)x.w, q.y, a3);
        }
    } else {
        for (int j = lane; j < n; j += 32) a0 = fma((double)xr[j], v[j], a0);
    }
    return warp_sum((a0 + a1) + (a2 + a3));
}

__device__ __forceinline__ double row_dot64(const double* __restrict__ ar, const double* __restrict__ x, int n,
                                            int lane) {
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    if ((n & 1) == 0 && (((uintptr_t)ar | (uintptr_t)x) & 15) == 0) {
        const double2* r2 = reinterpret_cast<const double2*>(ar);
        const double2* x2 = reinterpret_cast<const double2*>(x);
        const int n2 = n >> 1;
        int j = lane;
#pragma unroll 2
        for (; j + 32 < n2; j += 64) {
            const double2 p = __ldg(r2 + j), q = __ldg(r2 + j + 32);
            const double2 u = x2[j], w = x2[j + 32];
            a0 = fma(p.x, u.x, a0);
            a1 = fma(p.y, u.y, a1);
            a2 = fma(q.x, w.x, a2);
            a3 = fma(q.y, w.y, a3);
        }
        if (j < n2) {
            const double2 p = __ldg(r2 + j), u = x2[j];
            a0 = fma(p.x, u.x, a0);
            a1 = fma(p.y, u.y, a1);
        }
    } else {
        for (int j = lane; j < n; j += 32) a0 = fma(ar[j], x[j], a0);
    }
    return warp_sum((a0 + a1) + (a2 + a3));
}

__global__ void gemv32_kernel(const float* __restrict__ X, const double* __restrict__ v, int n,
                              double* __restrict__ y, int accumulate) {
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    const double acc = row_dot32(X + (int64_t)row * n, v, n, lane);
    if (lane == 0) y[row] = accumulate ? y[row] + acc : acc;
}

__global__ void residual64_kernel(const double* __restrict__ A, const double* __restrict__ x,
                                  const double* __restrict__ b, int n, double* __restrict__ r) {
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    const double acc = row_dot64(A + (int64_t)row * n, x, n, lane);
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

// ---------------------------------------------------------------------------------
// Batched refinement sweeps (grid.y = system).
__global__ void gemv32_jobs_kernel(const RefineJob* __restrict__ jobs, int from_residual, int accumulate) {
    const RefineJob& J = jobs[blockIdx.y];
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= J.n) return;
    const double acc = row_dot32(J.xinv + (int64_t)row * J.n, from_residual ? J.r : J.b, J.n, lane);
    if (lane == 0) J.x[row] = accumulate ? J.x[row] + acc : acc;
}

__global__ void residual64_jobs_kernel(const RefineJob* __restrict__ jobs) {
    const RefineJob& J = jobs[blockIdx.y];
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= J.n) return;
    const double acc = row_dot64(J.a + (int64_t)row * J.n, J.x, J.n, lane);
    if (lane == 0) J.r[row] = J.b[row] - acc;
}

__global__ void rel_resid_jobs_kernel(const RefineJob* __restrict__ jobs) {
    const RefineJob& J = jobs[blockIdx.x];
    __shared__ double sr[32], sb[32];
    double mr = 0.0, mb = 0.0;
    for (int i = threadIdx.x; i < J.n; i += blockDim.x) {
        mr = fmax(mr, fabs(J.r[i]));
        mb = fmax(mb, fabs(J.b[i]));
        if (J.r[i] != J.r[i]) mr = INFINITY;
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
        *J.resid = mb > 0.0 ? mr / mb : mr;
    }
}

int refine_jobs(const RefineJob* d_jobs, int n_jobs, int max_n, int n_iter, cudaStream_t s) {
    if (n_jobs == 0 || max_n == 0) return FJ_OK;
    const int wpb = 8;
    dim3 g((unsigned)((max_n + wpb - 1) / wpb), (unsigned)n_jobs);
    gemv32_jobs_kernel<<<g, wpb * 32, 0, s>>>(d_jobs, 0, 0); note_launch();
    for (int it = 0; it < n_iter; ++it) {
        residual64_jobs_kernel<<<g, wpb * 32, 0, s>>>(d_jobs); note_launch();
        gemv32_jobs_kernel<<<g, wpb * 32, 0, s>>>(d_jobs, 1, 1); note_launch();
    }
    residual64_jobs_kernel<<<g, wpb * 32, 0, s>>>(d_jobs); note_launch();
    rel_resid_jobs_kernel<<<n_jobs, 1024, 0, s>>>(d_jobs); note_launch();
    FJ_LAUNCH_CHECK("refine_jobs");
    return FJ_OK;
}

}  // namespace fj
