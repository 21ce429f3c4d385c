// fj_adjoint.cu -- hand-written adjoints of the induced-velocity sum and of the solve.
//
// The reference differentiates its UVLM by reverse-mode AD (jax.vjp through
// solve_prescribed_dynamic / the residuals of aero/uvlm.py:1529-1940).  Here the two
// operators that carry the cost have hand-written adjoints:
//   * the Biot-Savart sum v(x) = sum_s K(x; y0_s, y1_s) g_s (compute_v_ind,
//     aero/aic.py:248-310) -- cotangent lam(x) -> x_bar, vertex adjoints of every source
//     lattice, ring-circulation adjoints (FP64; epsilon kernel aero/utils.py:606-623, and
//     the cutoff kernel :626-648, whose D is |c|^2 and whose pairs within the cutoff
//     radius of the filament line contribute nothing, derivative included);
//   * the dense solve (aero/uvlm.py:985) -- A^T mu = lam with the getrf factors of A.
// K's derivative: with r1 = x - y0, r2 = x - y1, r0 = y1 - y0, c = r1 x r2,
// u_i = r_i / n_i, n_i = sqrt(|r_i|^2 + eps^2), dot = r0.(u1 - u2), D = |c|^2 + eps|r0|^4,
// s = dot / (4 pi D), a = lam.c:
//   d(lam.K)/dr1 = s (r2 x lam) + a [ddot/dr1 - (dot / D) dD/dr1] / (4 pi D)
//   d(lam.K)/dr2 = s (lam x r1) + a [ddot/dr2 - (dot / D) dD/dr2] / (4 pi D)
//   ddot/dr1 = (u1 - u2) + (r0 - (r0.u1) u1) / n1,  ddot/dr2 = -(u1 - u2) - (r0 - (r0.u2) u2) / n2
//   dD/dr1 = 2 (r2 x c) + 4 eps |r0|^2 r0,          dD/dr2 = 2 (c x r1) - 4 eps |r0|^2 r0
// and x_bar = d/dr1 + d/dr2, y0_bar = -d/dr1, y1_bar = -d/dr2, g_bar = lam.K / g.
#include <algorithm>
#include <cstring>
#include <vector>

#include "fj_lu.cuh"
#include "fj_bsgrad.cuh"
#include "fj_vind.cuh"

namespace fj {

constexpr int kAdjBlock = 128;

// Pass 1: target adjoints.  Walks the stream as the forward sum does.
template <int KER>
__global__ void __launch_bounds__(kAdjBlock) vjp_targets_kernel(const double* __restrict__ tgt,
                                                                const double* __restrict__ lam, int64_t n_t,
                                                                const Elem64* __restrict__ st, int64_t n_elem,
                                                                int n_split, double rc2, double* __restrict__ part) {
    __shared__ Elem64 sh[kAdjBlock];
    const int split = blockIdx.y;
    const int64_t per = (n_elem + n_split - 1) / n_split;
    const int64_t e0 = (int64_t)split * per;
    const int64_t e1 = min(n_elem, e0 + per);
    const int64_t vend = min(e1, n_elem - 1);
    const int64_t ti = (int64_t)blockIdx.x * kAdjBlock + threadIdx.x;
    const int64_t tc = min(ti, n_t - 1);
    const double x[3] = {tgt[tc * 3], tgt[tc * 3 + 1], tgt[tc * 3 + 2]};
    const double lm[3] = {lam[tc * 3], lam[tc * 3 + 1], lam[tc * 3 + 2]};
    double acc[3] = {0.0, 0.0, 0.0};
    if (e0 < e1) {
        VtxA prev;
        Elem64 pl = st[e0];
        vtxa(x, pl.x, pl.y, pl.z, prev);
        for (int64_t c0 = e0 + 1; c0 <= vend; c0 += kAdjBlock) {
            const int cnt = (int)min((int64_t)kAdjBlock, vend + 1 - c0);
            __syncthreads();
            if (threadIdx.x < cnt) sh[threadIdx.x] = st[c0 + threadIdx.x];
            __syncthreads();
            for (int i = 0; i < cnt; ++i) {
                const Elem64 cur = sh[i];
                VtxA v;
                vtxa(x, cur.x, cur.y, cur.z, v);
                if (pl.q >= 0.0) {
                    const double r0[3] = {pl.r0x, pl.r0y, pl.r0z};
                    double g1[3], g2[3], lk;
                    link_vjp<KER>(prev, v, r0, pl.g, lm, rc2, g1, g2, lk);
                    acc[0] += g1[0] + g2[0];
                    acc[1] += g1[1] + g2[1];
                    acc[2] += g1[2] + g2[2];
                }
                prev = v;
                pl = cur;
            }
        }
    }
    if (ti < n_t) {
        double* o = part + ((int64_t)split * n_t + ti) * 3;
        o[0] = acc[0];
        o[1] = acc[1];
        o[2] = acc[2];
    }
}

// Pass 2: filament adjoints.  Thread per stream element e (the link e -> e+1); targets
// of this CTA's split staged through shared memory.  Output per element and split:
// [y0_bar(3), y1_bar(3), g_bar].
template <int KER>
__global__ void __launch_bounds__(kAdjBlock) vjp_links_kernel(const double* __restrict__ tgt,
                                                              const double* __restrict__ lam, int64_t n_t,
                                                              const Elem64* __restrict__ st, int64_t n_elem,
                                                              int n_split, double rc2, double* __restrict__ part) {
    __shared__ double sx[kAdjBlock][6];
    const int split = blockIdx.y;
    const int64_t per = (n_t + n_split - 1) / n_split;
    const int64_t t0 = (int64_t)split * per;
    const int64_t t1 = min(n_t, t0 + per);
    const int64_t e = (int64_t)blockIdx.x * kAdjBlock + threadIdx.x;
    const bool live = e + 1 < n_elem && st[min(e, n_elem - 1)].q >= 0.0;
    Elem64 a, b;
    if (live) {
        a = st[e];
        b = st[e + 1];
    } else {
        memset(&a, 0, sizeof(a));
        memset(&b, 0, sizeof(b));
    }
    double y0b[3] = {0, 0, 0}, y1b[3] = {0, 0, 0}, gb = 0.0;
    for (int64_t c0 = t0; c0 < t1; c0 += kAdjBlock) {
        const int cnt = (int)min((int64_t)kAdjBlock, t1 - c0);
        __syncthreads();
        if (threadIdx.x < cnt) {
            const int64_t t = c0 + threadIdx.x;
            for (int k = 0; k < 3; ++k) {
                sx[threadIdx.x][k] = tgt[t * 3 + k];
                sx[threadIdx.x][3 + k] = lam[t * 3 + k];
            }
        }
        __syncthreads();
        if (live) {
            const double r0[3] = {a.r0x, a.r0y, a.r0z};
            for (int i = 0; i < cnt; ++i) {
                const double x[3] = {sx[i][0], sx[i][1], sx[i][2]};
                const double lm[3] = {sx[i][3], sx[i][4], sx[i][5]};
                VtxA A, B;
                vtxa(x, a.x, a.y, a.z, A);
                vtxa(x, b.x, b.y, b.z, B);
                double g1[3], g2[3], lk;
                link_vjp<KER>(A, B, r0, a.g, lm, rc2, g1, g2, lk);
                for (int k = 0; k < 3; ++k) {
                    y0b[k] -= g1[k];
                    y1b[k] -= g2[k];
                }
                gb += lk;
            }
        }
    }
    if (e < n_elem) {
        double* o = part + ((int64_t)split * n_elem + e) * 7;
        for (int k = 0; k < 3; ++k) {
            o[k] = y0b[k];
            o[3 + k] = y1b[k];
        }
        o[6] = gb;
    }
}

__global__ void sum_splits_kernel(const double* __restrict__ part, int n_split, int64_t n, double* __restrict__ out,
                                  int accumulate) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0.0;
    for (int k = 0; k < n_split; ++k) s += part[(int64_t)k * n + i];
    out[i] = accumulate ? out[i] + s : s;
}

// Element adjoints -> lattice vertex and ring-circulation adjoints (accumulated).
struct UnpackArgs {
    LatticeRef lat[kMaxPack];
    int64_t offset[kMaxPack + 1];
    double* zeta_bar[kMaxPack];   // per packed lattice (images point at their original)
    double* gamma_bar[kMaxPack];
    int n_lat;
    MirrorPlane mirror;
};

__global__ void unpack_vertices_kernel(UnpackArgs u, const double* __restrict__ el, int li) {
    const LatticeRef& L = u.lat[li];
    const int R = L.rows, C = L.cols;
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= (int64_t)(R + 1) * (C + 1)) return;
    const int k = (int)(v / (C + 1)), l = (int)(v % (C + 1));
    const int64_t off = u.offset[li];
    const int64_t n_chord = (int64_t)(C + 1) * (R + 1);
    const int64_t ec = off + (int64_t)l * (R + 1) + k;        // chordwise chain element
    const int64_t es = off + n_chord + (int64_t)k * (C + 1) + l;  // spanwise chain element
    double y[3];
    for (int d = 0; d < 3; ++d) {
        double s = el[ec * 7 + d] + el[es * 7 + d];          // vertex as link start
        if (k > 0) s += el[(ec - 1) * 7 + 3 + d];             // vertex as end of chordwise link
        if (l > 0) s += el[(es - 1) * 7 + 3 + d];             // vertex as end of spanwise link
        y[d] = s;
    }
    if (L.mirrored) {  // y' = y - 2((y - p).n) n  =>  y_bar += (I - 2 n n^T) y'_bar
        const double* nn = u.mirror.nrm;
        const double dn = y[0] * nn[0] + y[1] * nn[1] + y[2] * nn[2];
        for (int d = 0; d < 3; ++d) y[d] -= 2.0 * dn * nn[d];
    }
    double* zb = u.zeta_bar[li] + v * 3;
    for (int d = 0; d < 3; ++d) zb[d] += y[d];
}

__global__ void unpack_gamma_kernel(UnpackArgs u, const double* __restrict__ el, int li) {
    const LatticeRef& L = u.lat[li];
    const int R = L.rows, C = L.cols;
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= (int64_t)R * C || u.gamma_bar[li] == nullptr) return;
    const int k = (int)(r / C), l = (int)(r % C);
    const int64_t off = u.offset[li];
    const int64_t n_chord = (int64_t)(C + 1) * (R + 1);
    auto gm = [&](int kk, int ll) { return el[(off + (int64_t)ll * (R + 1) + kk) * 7 + 6]; };
    auto gn = [&](int kk, int ll) { return el[(off + n_chord + (int64_t)kk * (C + 1) + ll) * 7 + 6]; };
    // G_eff_m[k,l] = G[k,l] - G[k,l-1];  G_eff_n[k,l] = G[k-1,l] - G[k,l]  (aero/aic.py:284-287)
    const double gbar = gm(k, l) - gm(k, l + 1) - gn(k, l) + gn(k + 1, l);
    u.gamma_bar[li][r] += (double)L.sign * gbar;
}

// ------------------------------------------------------------------------------------
// getrs with A^T: A = P^T L U  =>  U^T L^T (P x) = b
// ------------------------------------------------------------------------------------
constexpr int kTBlk = 64;

// The diagonal block [i0, i0 + bw) of the factors comes into shared memory as it lies in
// memory (row-major, every element's cp.async in flight at once); one warp substitutes,
// lane l holding x of rows l and l + 32 in registers and x_j reaching every lane by a
// shuffle, reading the block transposed.  Per row the operations are those of the
// column-by-column transposed substitution, in its order.
__global__ void __launch_bounds__(kTBlk) trsv_t_diag_kernel(const double* __restrict__ lu, int n, int i0, int bw,
                                                            bool upper_of_lt, double* __restrict__ x) {
    // upper_of_lt == false: solve with U^T (lower, diagonal U[j][j]) forward
    // upper_of_lt == true:  solve with L^T (upper, unit diagonal) backward
    static_assert(kTBlk == 64, "two rows per lane");
    __shared__ __align__(16) double blk[kTBlk][kTBlk + 1];  // blk[j][r] = lu[i0 + j][i0 + r]
    for (int idx = threadIdx.x; idx < bw * bw; idx += blockDim.x) {
        const int j = idx / bw, r = idx % bw;
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(&blk[j][r])),
                     "l"(lu + (int64_t)(i0 + j) * n + i0 + r)
                     : "memory");
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    if (threadIdx.x >= 32) return;
    const int lane = threadIdx.x;
    const unsigned full = 0xffffffffu;
    double v0 = lane < bw ? x[i0 + lane] : 0.0;
    double v1 = lane + 32 < bw ? x[i0 + lane + 32] : 0.0;
    if (!upper_of_lt) {
#pragma unroll 1
        for (int j = 0; j < bw; ++j) {
            const bool hi = j >= 32;
            if (lane == (j & 31)) {
                if (hi) v1 = v1 / blk[j][j];
                else v0 = v0 / blk[j][j];
            }
            const double xj = __shfl_sync(full, hi ? v1 : v0, j & 31);
            if (lane > j && lane < bw) v0 -= blk[j][lane] * xj;
            if (lane + 32 > j && lane + 32 < bw) v1 -= blk[j][lane + 32] * xj;
        }
    } else {
#pragma unroll 1
        for (int j = bw - 1; j >= 0; --j) {
            const double xj = __shfl_sync(full, j >= 32 ? v1 : v0, j & 31);
            if (lane < j) v0 -= blk[j][lane] * xj;
            if (lane + 32 < j) v1 -= blk[j][lane + 32] * xj;
        }
    }
    if (lane < bw) x[i0 + lane] = v0;
    if (lane + 32 < bw) x[i0 + lane + 32] = v1;
}

// x[i] -= sum_{j in [j0, j0+bw)} lu[j][i] x[j] for i in [r0, r1)
__global__ void trsv_t_update_kernel(const double* __restrict__ lu, int n, int j0, int bw, int r0, int r1,
                                     double* __restrict__ x) {
    const int i = r0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= r1) return;
    double acc = 0.0;
    for (int j = 0; j < bw; ++j) acc += lu[(int64_t)(j0 + j) * n + i] * x[j0 + j];
    x[i] -= acc;
}

__global__ void __launch_bounds__(1024) unpermute_kernel(const int32_t* __restrict__ piv, int n,
                                                         const double* __restrict__ w, double* __restrict__ x) {
    extern __shared__ int perm[];
    for (int i = threadIdx.x; i < n; i += blockDim.x) perm[i] = i;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 0; i < n; ++i) {
            const int p = piv[i];
            if (p != i) {
                const int t = perm[i];
                perm[i] = perm[p];
                perm[p] = t;
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) x[perm[i]] = w[i];
}

int lu_solve_t64(const double* lu, int n, const int32_t* piv, double* b, double* work, cudaStream_t s) {
    if (n <= 0) return fail(FJ_ERR_SHAPE, "lu_solve_t: n=%d", n);
    if ((size_t)n * sizeof(int) > 220 * 1024) return fail(FJ_ERR_UNSUPPORTED, "lu_solve_t: n=%d too large", n);
    FJ_CUDA(cudaMemcpyAsync(work, b, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    for (int i0 = 0; i0 < n; i0 += kTBlk) {  // U^T z = b, forward
        const int bw = min(kTBlk, n - i0);
        trsv_t_diag_kernel<<<1, kTBlk, 0, s>>>(lu, n, i0, bw, false, work); note_launch();
        if (i0 + bw < n) {
            trsv_t_update_kernel<<<(n - i0 - bw + 127) / 128, 128, 0, s>>>(lu, n, i0, bw, i0 + bw, n, work); note_launch();
        }
    }
    for (int i0 = ((n - 1) / kTBlk) * kTBlk; i0 >= 0; i0 -= kTBlk) {  // L^T w = z, backward
        const int bw = min(kTBlk, n - i0);
        trsv_t_diag_kernel<<<1, kTBlk, 0, s>>>(lu, n, i0, bw, true, work); note_launch();
        if (i0 > 0) {
            trsv_t_update_kernel<<<(i0 + 127) / 128, 128, 0, s>>>(lu, n, i0, bw, 0, i0, work); note_launch();
        }
    }
    FJ_TRY(allow_dynamic_smem((const void*)unpermute_kernel, (size_t)(n * sizeof(int))));
    unpermute_kernel<<<1, 1024, n * sizeof(int), s>>>(piv, n, work, b); note_launch();
    FJ_LAUNCH_CHECK("lu_solve_t64");
    return FJ_OK;
}

static int64_t vjp_elems(const int* rows, const int* cols, int n_lattices, int img) {
    int64_t n = 0;
    for (int i = 0; i < n_lattices; ++i) n += img * stream_len(rows[i], cols[i]);
    return n;
}

static int vjp_splits_t(int64_t n_t) { return (int)std::max<int64_t>(1, std::min<int64_t>(64, 1184 / std::max<int64_t>(1, (n_t + kAdjBlock - 1) / kAdjBlock))); }
static int vjp_splits_l(int64_t n_elem, int64_t n_t) {
    const int64_t ctas = (n_elem + kAdjBlock - 1) / kAdjBlock;
    return (int)std::max<int64_t>(1, std::min<int64_t>({64, 1184 / std::max<int64_t>(1, ctas), std::max<int64_t>(1, n_t / 64)}));
}

}  // namespace fj

using namespace fj;

extern "C" {

int fj_vind_vjp_workspace_size(int64_t n_targets, const int* rows, const int* cols, int n_lattices, int mirror,
                               size_t* bytes) {
    if (bytes == nullptr || n_targets < 0 || n_lattices < 0 || n_lattices > FJ_MAX_SURF * 2)
        return fail(FJ_ERR_SHAPE, "vind_vjp workspace: bad arguments");
    const int64_t ne = vjp_elems(rows, cols, n_lattices, mirror ? 2 : 1);
    const int64_t nt = std::max<int64_t>(n_targets, 1);
    Arena a(nullptr, 0);
    a.carve<Elem64>(ne);
    a.carve<double>((int64_t)vjp_splits_t(nt) * nt * 3);
    a.carve<double>((int64_t)vjp_splits_l(ne, nt) * std::max<int64_t>(ne, 1) * 7);
    a.carve<double>(std::max<int64_t>(ne, 1) * 7);
    *bytes = a.used + 256;
    return FJ_OK;
}

int fj_vind_vjp(const double* d_targets, int64_t n_targets, const double* const* d_zetas,
                const double* const* d_gammas, const int* rows, const int* cols, int n_lattices,
                const double* mirror_point, const double* mirror_normal, int kernel, double r_cut,
                const double* d_lam, double* d_targets_bar, double* const* d_zetas_bar, double* const* d_gammas_bar,
                void* d_ws, size_t ws_bytes, fj_stream_t stream) {
    cudaStream_t s = (cudaStream_t)stream;
    if (kernel != FJ_KERNEL_EPSILON && kernel != FJ_KERNEL_CUTOFF)
        return fail(FJ_ERR_UNSUPPORTED, "fj_vind_vjp: the epsilon and cutoff kernels have hand-written adjoints");
    const double rc2 = r_cut * r_cut;
    const int mirror = mirror_point != nullptr && mirror_normal != nullptr;
    const int img = mirror ? 2 : 1;
    size_t need;
    FJ_TRY(fj_vind_vjp_workspace_size(n_targets, rows, cols, n_lattices, mirror, &need));
    if (ws_bytes < need) return fail(FJ_ERR_NOMEM, "vind_vjp workspace %zu < %zu", ws_bytes, need);
    if (n_targets == 0) return FJ_OK;
    const int64_t ne = vjp_elems(rows, cols, n_lattices, img);
    if (ne == 0) return FJ_OK;  // nothing to accumulate
    const int st_split = vjp_splits_t(n_targets), l_split = vjp_splits_l(ne, n_targets);
    Arena a(d_ws, ws_bytes);
    Elem64* st = a.carve<Elem64>(ne);
    double* part_t = a.carve<double>((int64_t)st_split * n_targets * 3);
    double* part_l = a.carve<double>((int64_t)l_split * ne * 7);
    double* el = a.carve<double>(ne * 7);
    PackArgs pa;
    UnpackArgs ua;
    memset(&pa, 0, sizeof(pa));
    memset(&ua, 0, sizeof(ua));
    pa.kernel = kernel;
    pa.r_cut = r_cut;
    if (mirror)
        for (int d = 0; d < 3; ++d) {
            pa.mirror.p[d] = mirror_point[d];
            pa.mirror.nrm[d] = mirror_normal[d];
        }
    ua.mirror = pa.mirror;
    int n = 0;
    for (int i = 0; i < n_lattices; ++i) {
        for (int k = 0; k < img; ++k) {
            LatticeRef& L = pa.lat[n];
            L.zeta = d_zetas[i];
            L.gamma = d_gammas[i];
            L.rows = rows[i];
            L.cols = cols[i];
            L.sign = k ? -1.0f : 1.0f;
            L.mirrored = k;
            pa.offset[n + 1] = pa.offset[n] + stream_len(rows[i], cols[i]);
            ua.lat[n] = L;
            ua.offset[n] = pa.offset[n];
            ua.zeta_bar[n] = d_zetas_bar ? d_zetas_bar[i] : nullptr;
            ua.gamma_bar[n] = d_gammas_bar ? d_gammas_bar[i] : nullptr;
            ++n;
        }
    }
    pa.n_lat = n;
    ua.n_lat = n;
    ua.offset[n] = pa.offset[n];
    FJ_TRY(pack_stream64(pa, st, s));
    if (d_targets_bar) {
        dim3 g((unsigned)((n_targets + kAdjBlock - 1) / kAdjBlock), (unsigned)st_split);
        if (kernel == FJ_KERNEL_EPSILON)
            vjp_targets_kernel<FJ_KERNEL_EPSILON><<<g, kAdjBlock, 0, s>>>(d_targets, d_lam, n_targets, st, ne,
                                                                          st_split, rc2, part_t);
        else
            vjp_targets_kernel<FJ_KERNEL_CUTOFF><<<g, kAdjBlock, 0, s>>>(d_targets, d_lam, n_targets, st, ne,
                                                                         st_split, rc2, part_t);
        note_launch();
        sum_splits_kernel<<<(unsigned)((n_targets * 3 + 255) / 256), 256, 0, s>>>(part_t, st_split, n_targets * 3,
                                                                                 d_targets_bar, 1); note_launch();
    }
    if (d_zetas_bar || d_gammas_bar) {
        dim3 g((unsigned)((ne + kAdjBlock - 1) / kAdjBlock), (unsigned)l_split);
        if (kernel == FJ_KERNEL_EPSILON)
            vjp_links_kernel<FJ_KERNEL_EPSILON><<<g, kAdjBlock, 0, s>>>(d_targets, d_lam, n_targets, st, ne, l_split,
                                                                        rc2, part_l);
        else
            vjp_links_kernel<FJ_KERNEL_CUTOFF><<<g, kAdjBlock, 0, s>>>(d_targets, d_lam, n_targets, st, ne, l_split,
                                                                       rc2, part_l);
        note_launch();
        sum_splits_kernel<<<(unsigned)((ne * 7 + 255) / 256), 256, 0, s>>>(part_l, l_split, ne * 7, el, 0); note_launch();
        for (int li = 0; li < n; ++li) {
            const int64_t nv = (int64_t)(ua.lat[li].rows + 1) * (ua.lat[li].cols + 1);
            if (ua.zeta_bar[li]) {
                unpack_vertices_kernel<<<(unsigned)((nv + 255) / 256), 256, 0, s>>>(ua, el, li); note_launch();
            }
            const int64_t nr = (int64_t)ua.lat[li].rows * ua.lat[li].cols;
            if (ua.gamma_bar[li] && nr > 0) {
                unpack_gamma_kernel<<<(unsigned)((nr + 255) / 256), 256, 0, s>>>(ua, el, li); note_launch();
            }
        }
    }
    FJ_LAUNCH_CHECK("fj_vind_vjp");
    return FJ_OK;
}

int fj_lu_solve_t(const double* d_lu, int n, const int32_t* d_piv, double* d_b, void* d_ws, size_t ws_bytes,
                  fj_stream_t stream) {
    if (ws_bytes < 256 + (size_t)n * sizeof(double)) return fail(FJ_ERR_NOMEM, "lu_solve_t workspace too small");
    return lu_solve_t64(d_lu, n, d_piv, d_b, (double*)((char*)d_ws + 256), (cudaStream_t)stream);
}

}  // extern "C"
