// fj_jac.cu -- dense influence Jacobians of the Biot-Savart sum, for the linearised UVLM
// (aero/linear/linear_uvlm.py, whose state-space matrices the reference forms by jax.jacrev
// of one UVLM step).
//
// Two matrices per (target set, source lattice), FP64, written into caller-owned
// row-major blocks (leading dimension ld, so a block can sit inside a larger matrix):
//   * ring influence  V[t, r]  = velocity at target t of unit circulation on ring r,
//     ring(k,l) = M[k,l] - M[k,l+1] + N[k+1,l] - N[k,l] over the chordwise filaments
//     M[k,l]: (k,l)->(k+1,l) and spanwise N[k,l]: (k,l)->(k,l+1) (aero/aic.py:55-57), a
//     mirror image subtracted (aero/aic.py:101-110, 306-308).  The derivative of
//     compute_v_ind (aero/aic.py:248-310) with respect to the circulations.
//   * vertex Jacobian J[t, v] = d v(x_t) / d zeta_v for given circulations: each vertex
//     collects the endpoint derivatives of its (up to four) filaments, each filament with
//     its strength G[k,l]-G[k,l-1] (chordwise) or G[k-1,l]-G[k,l] (spanwise)
//     (aero/aic.py:284-287); an image vertex M(zeta_v) carries the reflection R = I - 2mm^T.
// With a normal per target the rows are projected (n_t . v), as the AIC rows are; without
// one each target has three rows (x, y, z).  Thread per (target, ring) or (target, vertex);
// every filament is evaluated once per adjacent ring or vertex, the column index runs along
// the warp so the stores coalesce.
//
// fj_lu_solve_many: B <- A^-1 B for many right-hand sides (columns of a row-major B) from
// the getrf factors of fj_lu_factor: blocked forward and backward substitution, 32-column
// tiles per CTA, the off-diagonal updates as shared-memory tile products.
#include <algorithm>

#include "fj_bs.cuh"
#include "fj_bsgrad.cuh"
#include "fj_vind.cuh"

namespace fj {
namespace {

constexpr int kJacBlock = 128;

__device__ __forceinline__ void reflect(const MirrorPlane& mp, const double* z, double o[3]) {
    // mirror_grid, aero/utils.py:651-663
    const double d = (z[0] - mp.p[0]) * mp.nrm[0] + (z[1] - mp.p[1]) * mp.nrm[1] + (z[2] - mp.p[2]) * mp.nrm[2];
    o[0] = z[0] - 2.0 * d * mp.nrm[0];
    o[1] = z[1] - 2.0 * d * mp.nrm[1];
    o[2] = z[2] - 2.0 * d * mp.nrm[2];
}

__device__ __forceinline__ double ring_g(const double* gamma, int R, int C, int k, int l) {
    return (k < 0 || l < 0 || k >= R || l >= C) ? 0.0 : gamma[(int64_t)k * C + l];
}

// K(x; y0 -> y1) with unit strength, the forward arithmetic of the sums.
template <int KER>
__device__ __forceinline__ void seg_velocity(const double x[3], const double y0[3], const double y1[3], double rc2,
                                             double acc[3]) {
    Vtx64<KER> a, b;
    vtx64<KER>(x, y0[0], y0[1], y0[2], a);
    vtx64<KER>(x, y1[0], y1[1], y1[2], b);
    const double r0x = y1[0] - y0[0], r0y = y1[1] - y0[1], r0z = y1[2] - y0[2];
    const double r0sq = r0x * r0x + r0y * r0y + r0z * r0z;
    const double q = KER == FJ_KERNEL_EPSILON ? kEps * r0sq * r0sq : r0sq;
    link64<KER>(a, b, 1.0, r0x, r0y, r0z, q, rc2, acc);
}

template <int KER, bool NRM>
__global__ void __launch_bounds__(kJacBlock) ring_influence_kernel(const double* __restrict__ tgt,
                                                                   const double* __restrict__ nrm, int64_t nt,
                                                                   const double* __restrict__ zeta, int R, int C,
                                                                   int mirror, MirrorPlane mp, double rc2,
                                                                   double* __restrict__ out, int64_t ld) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= (int64_t)R * C) return;
    const int k = (int)(r / C), l = (int)(r % C);
    const int C1 = C + 1;
    const double* z00 = zeta + ((int64_t)k * C1 + l) * 3;
    const double* z01 = z00 + 3;
    const double* z10 = z00 + (int64_t)C1 * 3;
    const double* z11 = z10 + 3;
    double p[2][4][3];  // [image][corner 00, 01, 10, 11]
    for (int d = 0; d < 3; ++d) {
        p[0][0][d] = z00[d];
        p[0][1][d] = z01[d];
        p[0][2][d] = z10[d];
        p[0][3][d] = z11[d];
    }
    if (mirror) {
        reflect(mp, z00, p[1][0]);
        reflect(mp, z01, p[1][1]);
        reflect(mp, z10, p[1][2]);
        reflect(mp, z11, p[1][3]);
    }
    for (int64_t t = blockIdx.y; t < nt; t += gridDim.y) {
        const double x[3] = {tgt[t * 3 + 0], tgt[t * 3 + 1], tgt[t * 3 + 2]};
        double v[3] = {0.0, 0.0, 0.0};
        for (int img = 0; img < (mirror ? 2 : 1); ++img) {
            double m0[3] = {0.0, 0.0, 0.0}, m1[3] = {0.0, 0.0, 0.0}, n0[3] = {0.0, 0.0, 0.0}, n1[3] = {0.0, 0.0, 0.0};
            seg_velocity<KER>(x, p[img][0], p[img][2], rc2, m0);  // M[k,l]
            seg_velocity<KER>(x, p[img][1], p[img][3], rc2, m1);  // M[k,l+1]
            seg_velocity<KER>(x, p[img][2], p[img][3], rc2, n1);  // N[k+1,l]
            seg_velocity<KER>(x, p[img][0], p[img][1], rc2, n0);  // N[k,l]
            const double sg = img ? -1.0 : 1.0;
            for (int d = 0; d < 3; ++d) v[d] += sg * ((m0[d] - m1[d]) + (n1[d] - n0[d]));
        }
        if (NRM) {
            out[t * ld + r] = v[0] * nrm[t * 3 + 0] + v[1] * nrm[t * 3 + 1] + v[2] * nrm[t * 3 + 2];
        } else {
            out[(t * 3 + 0) * ld + r] = v[0];
            out[(t * 3 + 1) * ld + r] = v[1];
            out[(t * 3 + 2) * ld + r] = v[2];
        }
    }
}

// d(lam . K g)/d(endpoint) for filament p0 -> p1 at x; end = 0: p0, 1: p1.
template <int KER>
__device__ __forceinline__ void endpoint_grad(const double x[3], const double p0[3], const double p1[3], double g,
                                              const double lam[3], double rc2, int end, double o[3]) {
    VtxA A, B;
    vtxa(x, p0[0], p0[1], p0[2], A);
    vtxa(x, p1[0], p1[1], p1[2], B);
    const double r0[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
    double g1[3], g2[3], lk;
    link_vjp<KER>(A, B, r0, g, lam, rc2, g1, g2, lk);
    const double* src = end ? g2 : g1;
    o[0] = -src[0];
    o[1] = -src[1];
    o[2] = -src[2];
}

template <int KER, bool NRM>
__global__ void __launch_bounds__(kJacBlock) vertex_jacobian_kernel(const double* __restrict__ tgt,
                                                                    const double* __restrict__ nrm, int64_t nt,
                                                                    const double* __restrict__ zeta,
                                                                    const double* __restrict__ gamma, int R, int C,
                                                                    int mirror, MirrorPlane mp, double rc2,
                                                                    double* __restrict__ out, int64_t ld) {
    const int64_t vi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int C1 = C + 1;
    if (vi >= (int64_t)(R + 1) * C1) return;
    const int k = (int)(vi / C1), l = (int)(vi % C1);
    // incident filaments: (other endpoint, which end this vertex is, strength)
    int nf = 0;
    int ok[4], ol[4], end[4];
    double gs[4];
    if (k >= 1) {  // chordwise (k-1,l) -> (k,l)
        ok[nf] = k - 1, ol[nf] = l, end[nf] = 1;
        gs[nf++] = ring_g(gamma, R, C, k - 1, l) - ring_g(gamma, R, C, k - 1, l - 1);
    }
    if (k < R) {  // chordwise (k,l) -> (k+1,l)
        ok[nf] = k + 1, ol[nf] = l, end[nf] = 0;
        gs[nf++] = ring_g(gamma, R, C, k, l) - ring_g(gamma, R, C, k, l - 1);
    }
    if (l >= 1) {  // spanwise (k,l-1) -> (k,l)
        ok[nf] = k, ol[nf] = l - 1, end[nf] = 1;
        gs[nf++] = ring_g(gamma, R, C, k - 1, l - 1) - ring_g(gamma, R, C, k, l - 1);
    }
    if (l < C) {  // spanwise (k,l) -> (k,l+1)
        ok[nf] = k, ol[nf] = l + 1, end[nf] = 0;
        gs[nf++] = ring_g(gamma, R, C, k - 1, l) - ring_g(gamma, R, C, k, l);
    }
    const double* zv = zeta + vi * 3;
    double pv[2][3], po[2][4][3];
    for (int d = 0; d < 3; ++d) pv[0][d] = zv[d];
    for (int f = 0; f < nf; ++f)
        for (int d = 0; d < 3; ++d) po[0][f][d] = zeta[((int64_t)ok[f] * C1 + ol[f]) * 3 + d];
    if (mirror) {
        reflect(mp, zv, pv[1]);
        for (int f = 0; f < nf; ++f) reflect(mp, po[0][f], po[1][f]);
    }
    const int nrows = NRM ? 1 : 3;
    for (int64_t t = blockIdx.y; t < nt; t += gridDim.y) {
        const double x[3] = {tgt[t * 3 + 0], tgt[t * 3 + 1], tgt[t * 3 + 2]};
#pragma unroll 1
        for (int a = 0; a < nrows; ++a) {
            double lam[3];
            if (NRM) {
                lam[0] = nrm[t * 3 + 0];
                lam[1] = nrm[t * 3 + 1];
                lam[2] = nrm[t * 3 + 2];
            } else {
                lam[0] = a == 0 ? 1.0 : 0.0;
                lam[1] = a == 1 ? 1.0 : 0.0;
                lam[2] = a == 2 ? 1.0 : 0.0;
            }
            double acc[3] = {0.0, 0.0, 0.0};
#pragma unroll 1
            for (int img = 0; img < (mirror ? 2 : 1); ++img) {
                double s[3] = {0.0, 0.0, 0.0};
#pragma unroll 1
                for (int f = 0; f < nf; ++f) {
                    if (gs[f] == 0.0) continue;
                    double o[3];
                    if (end[f]) endpoint_grad<KER>(x, po[img][f], pv[img], gs[f], lam, rc2, 1, o);
                    else endpoint_grad<KER>(x, pv[img], po[img][f], gs[f], lam, rc2, 0, o);
                    s[0] += o[0];
                    s[1] += o[1];
                    s[2] += o[2];
                }
                if (img == 0) {
                    acc[0] += s[0];
                    acc[1] += s[1];
                    acc[2] += s[2];
                } else {
                    // image vertex M(z): d/dz = R d/dM(z), R = I - 2 m m^T; image sign -1
                    const double sm = s[0] * mp.nrm[0] + s[1] * mp.nrm[1] + s[2] * mp.nrm[2];
                    acc[0] -= s[0] - 2.0 * sm * mp.nrm[0];
                    acc[1] -= s[1] - 2.0 * sm * mp.nrm[1];
                    acc[2] -= s[2] - 2.0 * sm * mp.nrm[2];
                }
            }
            double* row = out + (t * nrows + a) * ld + vi * 3;
            row[0] = acc[0];
            row[1] = acc[1];
            row[2] = acc[2];
        }
    }
}

// perm = the getrf row swaps of piv applied in order to the identity
__global__ void perm_from_piv_kernel(const int32_t* __restrict__ piv, int n, int32_t* __restrict__ perm) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    for (int i = 0; i < n; ++i) perm[i] = i;
    for (int i = 0; i < n; ++i) {
        const int p = piv[i];
        if (p != i && p >= 0 && p < n) {
            const int32_t t = perm[i];
            perm[i] = perm[p];
            perm[p] = t;
        }
    }
}

// Blocked substitution for many right-hand sides.  CTA = 256 threads on a tile of 32
// columns; rows in blocks of 32.  For each row block: subtract the already-solved rows
// (a 32 x 32 x k0 product, staged through shared memory in 32 x 32 chunks of the factor
// and of the solved rows), then solve the block's own triangle in shared memory.  Thread
// (c = lane, y = warp) owns rows y, y+8, y+16, y+24 of the block in column c.
constexpr int kSolveCols = 32, kSolveRows = 32, kSolveThreads = 256;

__device__ __forceinline__ void tile_update(const double* __restrict__ lu, int n, const double* __restrict__ w,
                                            int64_t nrhs, int64_t col, bool col_ok, int i0, int k0, int k1,
                                            double (*ls)[kSolveRows + 1], double (*ws)[kSolveCols + 1],
                                            double acc[4]) {
    const int c = threadIdx.x & 31, y = threadIdx.x >> 5;
    for (int kb = k0; kb < k1; kb += kSolveRows) {
        const int kw = min(kSolveRows, k1 - kb);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = y + 8 * q;
            ls[r][c] = (i0 + r < n && c < kw) ? lu[(int64_t)(i0 + r) * n + kb + c] : 0.0;
            ws[r][c] = (r < kw && col_ok) ? w[(int64_t)(kb + r) * nrhs + col] : 0.0;
        }
        __syncthreads();
#pragma unroll 8
        for (int kk = 0; kk < kSolveRows; ++kk) {
            const double x = ws[kk][c];
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[q] -= ls[y + 8 * q][kk] * x;
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kSolveThreads) lu_solve_many_kernel(const double* __restrict__ lu, int n,
                                                                      const int32_t* __restrict__ perm,
                                                                      double* __restrict__ b, int64_t nrhs,
                                                                      int64_t ldb, double* __restrict__ w) {
    __shared__ double ls[kSolveRows][kSolveRows + 1];
    __shared__ double ws[kSolveRows][kSolveCols + 1];
    const int c = threadIdx.x & 31, y = threadIdx.x >> 5;
    const int64_t col = (int64_t)blockIdx.x * kSolveCols + c;
    const bool col_ok = col < nrhs;
    // gather the permuted right-hand sides: w[i] = b[perm[i]]
    if (col_ok)
        for (int i = y; i < n; i += 8) w[(int64_t)i * nrhs + col] = b[(int64_t)perm[i] * ldb + col];
    __syncthreads();
    // forward: unit lower
    for (int i0 = 0; i0 < n; i0 += kSolveRows) {
        const int rb = min(kSolveRows, n - i0);
        double acc[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = y + 8 * q;
            acc[q] = (r < rb && col_ok) ? w[(int64_t)(i0 + r) * nrhs + col] : 0.0;
        }
        tile_update(lu, n, w, nrhs, col, col_ok, i0, 0, i0, ls, ws, acc);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = y + 8 * q;
            ws[r][c] = acc[q];
            ls[r][c] = (r < rb && c < rb) ? lu[(int64_t)(i0 + r) * n + i0 + c] : 0.0;
        }
        __syncthreads();
        for (int rr = 0; rr + 1 < rb; ++rr) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int r = y + 8 * q;
                if (r > rr && r < rb) ws[r][c] -= ls[r][rr] * ws[rr][c];
            }
            __syncthreads();
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = y + 8 * q;
            if (r < rb && col_ok) w[(int64_t)(i0 + r) * nrhs + col] = ws[r][c];
        }
        __syncthreads();
    }
    // backward: upper, with the diagonal
    for (int i0 = ((n - 1) / kSolveRows) * kSolveRows; i0 >= 0; i0 -= kSolveRows) {
        const int rb = min(kSolveRows, n - i0);
        double acc[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = y + 8 * q;
            acc[q] = (r < rb && col_ok) ? w[(int64_t)(i0 + r) * nrhs + col] : 0.0;
        }
        tile_update(lu, n, w, nrhs, col, col_ok, i0, i0 + rb, n, ls, ws, acc);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = y + 8 * q;
            ws[r][c] = acc[q];
            ls[r][c] = (r < rb && c < rb) ? lu[(int64_t)(i0 + r) * n + i0 + c] : 1.0;
        }
        __syncthreads();
        for (int rr = rb - 1; rr >= 0; --rr) {
            if (y == (rr & 7)) ws[rr][c] /= ls[rr][rr];
            __syncthreads();
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int r = y + 8 * q;
                if (r < rr) ws[r][c] -= ls[r][rr] * ws[rr][c];
            }
            __syncthreads();
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = y + 8 * q;
            if (r < rb && col_ok) {
                w[(int64_t)(i0 + r) * nrhs + col] = ws[r][c];
                b[(int64_t)(i0 + r) * ldb + col] = ws[r][c];
            }
        }
        __syncthreads();
    }
}

int check_lattice(const double* tgt, int64_t nt, const double* zeta, int rows, int cols, double* out, int64_t ld,
                  int64_t min_ld, const char* what) {
    if (nt < 0 || rows < 0 || cols < 0) return fail(FJ_ERR_SHAPE, "%s: negative size", what);
    if (nt > 0 && (tgt == nullptr || out == nullptr)) return fail(FJ_ERR_SHAPE, "%s: null pointer", what);
    if (zeta == nullptr && (int64_t)(rows + 1) * (cols + 1) > 0) return fail(FJ_ERR_SHAPE, "%s: null lattice", what);
    if (ld < min_ld) return fail(FJ_ERR_SHAPE, "%s: ld %lld < %lld", what, (long long)ld, (long long)min_ld);
    return FJ_OK;
}

MirrorPlane mirror_of(const double* p, const double* m, int* on) {
    MirrorPlane mp{};
    *on = p != nullptr && m != nullptr;
    if (*on)
        for (int d = 0; d < 3; ++d) {
            mp.p[d] = p[d];
            mp.nrm[d] = m[d];
        }
    return mp;
}

unsigned target_grid(int64_t nt) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>(nt, 65535)); }

}  // namespace
}  // namespace fj

using namespace fj;

extern "C" {

int fj_ring_influence(const double* d_targets, int64_t n_targets, const double* d_normals, const double* d_zeta,
                      int rows, int cols, const double* mirror_point, const double* mirror_normal, int kernel,
                      double r_cut, double* d_out, int64_t ld_out, fj_stream_t stream) {
    cudaStream_t s = (cudaStream_t)stream;
    FJ_TRY(check_lattice(d_targets, n_targets, d_zeta, rows, cols, d_out, ld_out, (int64_t)rows * cols,
                         "fj_ring_influence"));
    if (kernel != FJ_KERNEL_EPSILON && kernel != FJ_KERNEL_CUTOFF)
        return fail(FJ_ERR_UNSUPPORTED, "fj_ring_influence: the epsilon and cutoff kernels only");
    const int64_t nr = (int64_t)rows * cols;
    if (n_targets == 0 || nr == 0) return FJ_OK;
    int mir;
    const MirrorPlane mp = mirror_of(mirror_point, mirror_normal, &mir);
    const double rc2 = r_cut * r_cut;
    dim3 g((unsigned)((nr + kJacBlock - 1) / kJacBlock), target_grid(n_targets));
    if (kernel == FJ_KERNEL_EPSILON) {
        if (d_normals)
            ring_influence_kernel<FJ_KERNEL_EPSILON, true><<<g, kJacBlock, 0, s>>>(d_targets, d_normals, n_targets,
                                                                                   d_zeta, rows, cols, mir, mp, rc2,
                                                                                   d_out, ld_out);
        else
            ring_influence_kernel<FJ_KERNEL_EPSILON, false><<<g, kJacBlock, 0, s>>>(d_targets, nullptr, n_targets,
                                                                                    d_zeta, rows, cols, mir, mp, rc2,
                                                                                    d_out, ld_out);
    } else {
        if (d_normals)
            ring_influence_kernel<FJ_KERNEL_CUTOFF, true><<<g, kJacBlock, 0, s>>>(d_targets, d_normals, n_targets,
                                                                                  d_zeta, rows, cols, mir, mp, rc2,
                                                                                  d_out, ld_out);
        else
            ring_influence_kernel<FJ_KERNEL_CUTOFF, false><<<g, kJacBlock, 0, s>>>(d_targets, nullptr, n_targets,
                                                                                   d_zeta, rows, cols, mir, mp, rc2,
                                                                                   d_out, ld_out);
    }
    note_launch();
    FJ_LAUNCH_CHECK("fj_ring_influence");
    return FJ_OK;
}

int fj_vertex_jacobian(const double* d_targets, int64_t n_targets, const double* d_normals, const double* d_zeta,
                       const double* d_gamma, int rows, int cols, const double* mirror_point,
                       const double* mirror_normal, int kernel, double r_cut, double* d_out, int64_t ld_out,
                       fj_stream_t stream) {
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t nv = (int64_t)(rows + 1) * (cols + 1);
    FJ_TRY(check_lattice(d_targets, n_targets, d_zeta, rows, cols, d_out, ld_out, 3 * nv, "fj_vertex_jacobian"));
    if (kernel != FJ_KERNEL_EPSILON && kernel != FJ_KERNEL_CUTOFF)
        return fail(FJ_ERR_UNSUPPORTED, "fj_vertex_jacobian: the epsilon and cutoff kernels only");
    if (rows * cols > 0 && d_gamma == nullptr) return fail(FJ_ERR_SHAPE, "fj_vertex_jacobian: null circulation");
    if (n_targets == 0 || nv == 0) return FJ_OK;
    int mir;
    const MirrorPlane mp = mirror_of(mirror_point, mirror_normal, &mir);
    const double rc2 = r_cut * r_cut;
    dim3 g((unsigned)((nv + kJacBlock - 1) / kJacBlock), target_grid(n_targets));
    if (kernel == FJ_KERNEL_EPSILON) {
        if (d_normals)
            vertex_jacobian_kernel<FJ_KERNEL_EPSILON, true><<<g, kJacBlock, 0, s>>>(
                d_targets, d_normals, n_targets, d_zeta, d_gamma, rows, cols, mir, mp, rc2, d_out, ld_out);
        else
            vertex_jacobian_kernel<FJ_KERNEL_EPSILON, false><<<g, kJacBlock, 0, s>>>(
                d_targets, nullptr, n_targets, d_zeta, d_gamma, rows, cols, mir, mp, rc2, d_out, ld_out);
    } else {
        if (d_normals)
            vertex_jacobian_kernel<FJ_KERNEL_CUTOFF, true><<<g, kJacBlock, 0, s>>>(
                d_targets, d_normals, n_targets, d_zeta, d_gamma, rows, cols, mir, mp, rc2, d_out, ld_out);
        else
            vertex_jacobian_kernel<FJ_KERNEL_CUTOFF, false><<<g, kJacBlock, 0, s>>>(
                d_targets, nullptr, n_targets, d_zeta, d_gamma, rows, cols, mir, mp, rc2, d_out, ld_out);
    }
    note_launch();
    FJ_LAUNCH_CHECK("fj_vertex_jacobian");
    return FJ_OK;
}

int fj_lu_solve_many_workspace_size(int n, int64_t nrhs, size_t* bytes) {
    if (bytes == nullptr || n <= 0 || nrhs < 0) return fail(FJ_ERR_SHAPE, "lu_solve_many workspace: bad arguments");
    *bytes = 256 + ((size_t)n * sizeof(int32_t) + 255) / 256 * 256 + (size_t)n * (size_t)nrhs * sizeof(double);
    return FJ_OK;
}

int fj_lu_solve_many(const double* d_lu, int n, const int32_t* d_piv, double* d_b, int64_t nrhs, int64_t ldb,
                     void* d_ws, size_t ws_bytes, fj_stream_t stream) {
    cudaStream_t s = (cudaStream_t)stream;
    size_t need;
    FJ_TRY(fj_lu_solve_many_workspace_size(n, nrhs, &need));
    if (ws_bytes < need) return fail(FJ_ERR_NOMEM, "lu_solve_many workspace %zu < %zu", ws_bytes, need);
    if (ldb < nrhs) return fail(FJ_ERR_SHAPE, "lu_solve_many: ldb %lld < nrhs %lld", (long long)ldb, (long long)nrhs);
    if (nrhs == 0) return FJ_OK;
    if (!d_lu || !d_piv || !d_b || !d_ws) return fail(FJ_ERR_SHAPE, "lu_solve_many: null pointer");
    char* base = (char*)(((uintptr_t)d_ws + 255) / 256 * 256);
    int32_t* perm = (int32_t*)base;
    double* w = (double*)(base + ((size_t)n * sizeof(int32_t) + 255) / 256 * 256);
    perm_from_piv_kernel<<<1, 32, 0, s>>>(d_piv, n, perm);
    lu_solve_many_kernel<<<(unsigned)((nrhs + kSolveCols - 1) / kSolveCols), kSolveThreads, 0, s>>>(d_lu, n, perm, d_b,
                                                                                             nrhs, ldb, w);
    note_launch(2);
    FJ_LAUNCH_CHECK("fj_lu_solve_many");
    return FJ_OK;
}

}  // extern "C"
