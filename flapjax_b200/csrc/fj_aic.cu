// fj_aic.cu -- bound-on-collocation influence matrix (compute_aic_solve, aero/aic.py:11-205).
//
// One CTA per collocation point i (row i of the AIC).  For each source surface the CTA
// evaluates the influence of every chordwise and spanwise filament at c_i, projects it
// on the area normal n_i (aero/aic.py:47-54) into shared memory, and combines filaments
// into rings as -diff(m, axis=1) + diff(n, axis=0) (aero/aic.py:55-57), so each filament
// is evaluated once per target, in FP64, with the reference's own association order.
// Mirror images are assembled the same way and subtracted ring by ring
// (aero/aic.py:101-110).  In the static solve the wake rings' influence, summed over wake
// rows, is added to the trailing-edge column (add_wake_influence, aero/aic.py:190-205).
#include "fj_aic.cuh"
#include "fj_bs.cuh"

namespace fj {

template <int KER>
__device__ __forceinline__ double seg_normal_influence(const double x[3], const double nrm[3],
                                                       const double* y0, const double* y1,
                                                       double rc2) {
    Vtx64<KER> a, b;
    vtx64<KER>(x, y0[0], y0[1], y0[2], a);
    vtx64<KER>(x, y1[0], y1[1], y1[2], b);
    const double r0x = y1[0] - y0[0], r0y = y1[1] - y0[1], r0z = y1[2] - y0[2];
    const double r0sq = r0x * r0x + r0y * r0y + r0z * r0z;
    const double q = (KER == FJ_KERNEL_EPSILON) ? kEps * r0sq * r0sq : r0sq;
    double k[3] = {0.0, 0.0, 0.0};
    link64<KER>(a, b, 1.0, r0x, r0y, r0z, q, rc2, k);
    return k[0] * nrm[0] + k[1] * nrm[1] + k[2] * nrm[2];  // jnp.dot(K, n_i)
}

__device__ __forceinline__ void mirror_pt(const MirrorPlane& mp, const double* z, double o[3]) {
    const double d0 = z[0] - mp.p[0], d1 = z[1] - mp.p[1], d2 = z[2] - mp.p[2];
    const double dn = d0 * mp.nrm[0] + d1 * mp.nrm[1] + d2 * mp.nrm[2];
    o[0] = z[0] - 2.0 * dn * mp.nrm[0];
    o[1] = z[1] - 2.0 * dn * mp.nrm[1];
    o[2] = z[2] - 2.0 * dn * mp.nrm[2];
}

// Influence of filament `s` of lattice zeta (R rows, C cols) at x projected on nrm.
// s < R*(C+1): chordwise (k,l)->(k+1,l) with k = s / (C+1); else spanwise.
template <int KER>
__device__ __forceinline__ double filament_influence(const double* zeta, int R, int C, int s,
                                                     bool mirrored, const MirrorPlane& mp,
                                                     const double x[3], const double nrm[3],
                                                     double rc2) {
    int k0, l0, k1, l1;
    const int nm = R * (C + 1);
    if (s < nm) {
        k0 = s / (C + 1);
        l0 = s % (C + 1);
        k1 = k0 + 1;
        l1 = l0;
    } else {
        const int t = s - nm;
        k0 = t / C;
        l0 = t % C;
        k1 = k0;
        l1 = l0 + 1;
    }
    const double* p0 = zeta + ((int64_t)k0 * (C + 1) + l0) * 3;
    const double* p1 = zeta + ((int64_t)k1 * (C + 1) + l1) * 3;
    if (!mirrored) return seg_normal_influence<KER>(x, nrm, p0, p1, rc2);
    double q0[3], q1[3];
    mirror_pt(mp, p0, q0);
    mirror_pt(mp, p1, q1);
    return seg_normal_influence<KER>(x, nrm, q0, q1, rc2);
}

template <int KER>
__device__ __forceinline__ void aic_row(const AicArgs& a, int64_t i, double* sm_inf) {
    const double x[3] = {a.c[i * 3 + 0], a.c[i * 3 + 1], a.c[i * 3 + 2]};
    const double nrm[3] = {a.nc[i * 3 + 0], a.nc[i * 3 + 1], a.nc[i * 3 + 2]};
    double* row = a.aic + i * a.ld;
    const int n_img = a.mirror ? 2 : 1;

    for (int sb = 0; sb < a.n_surf; ++sb) {
        const int R = a.m[sb], C = a.n[sb];
        const int nfil = R * (C + 1) + (R + 1) * C;
        __syncthreads();
        for (int img = 0; img < n_img; ++img) {
            double* buf = sm_inf + img * a.max_fil;
            for (int s = threadIdx.x; s < nfil; s += blockDim.x)
                buf[s] = filament_influence<KER>(a.zeta_b[sb], R, C, s, img == 1, a.mp, x, nrm, a.rc2);
        }
        __syncthreads();
        const int nm = R * (C + 1);
        for (int r = threadIdx.x; r < R * C; r += blockDim.x) {
            const int k = r / C, l = r % C;
            double v = 0.0;
            for (int img = 0; img < n_img; ++img) {
                const double* m_inf = sm_inf + img * a.max_fil;
                const double* n_inf = m_inf + nm;
                const double ring = -(m_inf[k * (C + 1) + l + 1] - m_inf[k * (C + 1) + l]) +
                                    (n_inf[(k + 1) * C + l] - n_inf[k * C + l]);
                v = img == 0 ? ring : v - ring;
            }
            row[a.col_off[sb] + r] = v;
        }
        // static solve: lump the wake of surface sb onto its trailing-edge column
        if (a.zeta_w[sb] != nullptr && a.m_star[sb] > 0) {
            __syncthreads();
            const int W = a.m_star[sb];
            const double* zw = a.zeta_w[sb];
            for (int l = threadIdx.x; l < C; l += blockDim.x) {
                double total = 0.0;
                for (int r = 0; r < W; ++r) {
                    double ring_v = 0.0;
                    for (int img = 0; img < n_img; ++img) {
                        const bool mir = img == 1;
                        const int nmw = W * (C + 1);
                        const double m_l = filament_influence<KER>(zw, W, C, r * (C + 1) + l, mir, a.mp, x, nrm, a.rc2);
                        const double m_l1 = filament_influence<KER>(zw, W, C, r * (C + 1) + l + 1, mir, a.mp, x, nrm, a.rc2);
                        const double n_r = filament_influence<KER>(zw, W, C, nmw + r * C + l, mir, a.mp, x, nrm, a.rc2);
                        const double n_r1 = filament_influence<KER>(zw, W, C, nmw + (r + 1) * C + l, mir, a.mp, x, nrm, a.rc2);
                        const double ring = -(m_l1 - m_l) + (n_r1 - n_r);
                        ring_v = img == 0 ? ring : ring_v - ring;
                    }
                    total += ring_v;
                }
                row[a.col_off[sb] + (R - 1) * C + l] += total;
            }
        }
    }
}

template <int KER>
__global__ void __launch_bounds__(256) aic_kernel(AicArgs a, const int* __restrict__ run_flag) {
    if (run_flag != nullptr && *run_flag == 0) return;
    extern __shared__ double sm_inf[];  // [2][max filaments]
    aic_row<KER>(a, blockIdx.x, sm_inf);
}

template <int KER>
__global__ void __launch_bounds__(256) aic_jobs_kernel(const AicArgs* __restrict__ tab) {
    const AicArgs& a = tab[blockIdx.y];
    if (blockIdx.x >= a.n_rows) return;
    if (a.run_flag != nullptr && *a.run_flag == 0) return;
    extern __shared__ double sm_inf[];
    aic_row<KER>(a, blockIdx.x, sm_inf);
}

int aic_launch_jobs(const AicArgs* d_tab, int n_jobs, int64_t max_rows, int max_fil, int any_mirror, int kernel,
                    cudaStream_t s) {
    const size_t smem = (size_t)(any_mirror ? 2 : 1) * max_fil * sizeof(double);
    if (smem > 200 * 1024)
        return fail(FJ_ERR_UNSUPPORTED, "aic: a surface with %d filaments exceeds shared memory", max_fil);
    if (n_jobs == 0 || max_rows == 0) return FJ_OK;
    dim3 g((unsigned)max_rows, (unsigned)n_jobs);
    switch (kernel) {
        case FJ_KERNEL_EPSILON:
            FJ_TRY(allow_dynamic_smem((const void*)aic_jobs_kernel<FJ_KERNEL_EPSILON>, (size_t)smem));
            aic_jobs_kernel<FJ_KERNEL_EPSILON><<<g, 256, smem, s>>>(d_tab); note_launch();
            break;
        case FJ_KERNEL_CUTOFF:
            FJ_TRY(allow_dynamic_smem((const void*)aic_jobs_kernel<FJ_KERNEL_CUTOFF>, (size_t)smem));
            aic_jobs_kernel<FJ_KERNEL_CUTOFF><<<g, 256, smem, s>>>(d_tab); note_launch();
            break;
        case FJ_KERNEL_PLAIN:
            FJ_TRY(allow_dynamic_smem((const void*)aic_jobs_kernel<FJ_KERNEL_PLAIN>, (size_t)smem));
            aic_jobs_kernel<FJ_KERNEL_PLAIN><<<g, 256, smem, s>>>(d_tab); note_launch();
            break;
        default:
            return fail(FJ_ERR_UNSUPPORTED, "aic: unknown kernel %d", kernel);
    }
    FJ_LAUNCH_CHECK("aic_jobs_kernel");
    return FJ_OK;
}

int aic_launch(const AicArgs& a, const int* d_run_flag, cudaStream_t s) {
    const size_t smem = (size_t)(a.mirror ? 2 : 1) * a.max_fil * sizeof(double);
    if (smem > 200 * 1024)
        return fail(FJ_ERR_UNSUPPORTED, "aic: a surface with %d filaments exceeds shared memory", a.max_fil);
    if (a.n_rows == 0) return FJ_OK;
    switch (a.kernel) {
        case FJ_KERNEL_EPSILON:
            FJ_TRY(allow_dynamic_smem((const void*)aic_kernel<FJ_KERNEL_EPSILON>, (size_t)smem));
            aic_kernel<FJ_KERNEL_EPSILON><<<(unsigned)a.n_rows, 256, smem, s>>>(a, d_run_flag); note_launch();
            break;
        case FJ_KERNEL_CUTOFF:
            FJ_TRY(allow_dynamic_smem((const void*)aic_kernel<FJ_KERNEL_CUTOFF>, (size_t)smem));
            aic_kernel<FJ_KERNEL_CUTOFF><<<(unsigned)a.n_rows, 256, smem, s>>>(a, d_run_flag); note_launch();
            break;
        case FJ_KERNEL_PLAIN:
            FJ_TRY(allow_dynamic_smem((const void*)aic_kernel<FJ_KERNEL_PLAIN>, (size_t)smem));
            aic_kernel<FJ_KERNEL_PLAIN><<<(unsigned)a.n_rows, 256, smem, s>>>(a, d_run_flag); note_launch();
            break;
        default:
            return fail(FJ_ERR_UNSUPPORTED, "aic: unknown kernel %d", a.kernel);
    }
    FJ_LAUNCH_CHECK("aic_kernel");
    return FJ_OK;
}

}  // namespace fj
