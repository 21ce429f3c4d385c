// fj_func.cu -- function-level entry points for the pieces of one UVLM step that the
// reference calls separately: the right-hand side (aero/uvlm.py:961-983), wake shedding
// and convection (propagate_surf_wake, aero/utils.py:400-450), forces
// (calculate_steady_forcing aero/utils.py:126-223 and the unsteady term uvlm.py:1086-1103),
// and the adjoint twins of the AIC product and of the wake shift.  Each works on one
// surface (one lattice); the induced-velocity sums inside them take any list of
// lattices through fj_vind / fj_vind_vjp.
#include <algorithm>
#include <cstring>

#include "fj_flow.cuh"
#include "fj_vind.cuh"

namespace fj {

namespace {

constexpr int kFB = 256;

inline unsigned nblk(int64_t n) { return (unsigned)std::max<int64_t>(1, (n + kFB - 1) / kFB); }

// b_i = -((U(c_i, t) - c_dot_i + v_i) . nc_i)
__global__ void rhs_kernel(const double* __restrict__ c, const double* __restrict__ nc,
                           const double* __restrict__ c_dot, const double* __restrict__ v, int64_t n_pan,
                           fj_flowfield flow, double t, double* __restrict__ b) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_pan) return;
    const double x[3] = {c[i * 3], c[i * 3 + 1], c[i * 3 + 2]};
    double u[3];
    flow_eval(flow, x, t, u);
    double s = 0.0;
    for (int d = 0; d < 3; ++d) {
        double w = u[d];
        if (c_dot) w -= c_dot[i * 3 + d];
        if (v) w += v[i * 3 + d];
        s += w * nc[i * 3 + d];
    }
    b[i] = -s;
}

// propagate_surf_wake, uniform branch (aero/utils.py:400-450):
// zeta_w_n = [zeta_te_n; zeta_w_nm1[:-1] + dt (U + v_conv)], gamma_w_n = [gamma_te_nm1; gamma_w_nm1[:-1]]
__global__ void wake_shed_kernel(const double* __restrict__ zeta_te, const double* __restrict__ gamma_te,
                                 const double* __restrict__ zw_nm1, const double* __restrict__ gw_nm1,
                                 const double* __restrict__ v_conv, int n, int m_star, fj_flowfield flow, double t,
                                 double dt, double* __restrict__ zw_n, double* __restrict__ gw_n) {
    const int64_t nv = (int64_t)(m_star + 1) * (n + 1);
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nv) {
        const int r = (int)(i / (n + 1)), l = (int)(i % (n + 1));
        if (r == 0) {
            for (int d = 0; d < 3; ++d) zw_n[i * 3 + d] = zeta_te[l * 3 + d];
        } else {
            const int64_t src = (int64_t)(r - 1) * (n + 1) + l;
            const double x[3] = {zw_nm1[src * 3], zw_nm1[src * 3 + 1], zw_nm1[src * 3 + 2]};
            double u[3];
            flow_eval(flow, x, t, u);
            if (v_conv)
                for (int d = 0; d < 3; ++d) u[d] += v_conv[src * 3 + d];
            for (int d = 0; d < 3; ++d) zw_n[i * 3 + d] = x[d] + dt * u[d];
        }
    }
    const int64_t ng = (int64_t)m_star * n;
    if (i < ng) {
        const int r = (int)(i / n), l = (int)(i % n);
        gw_n[i] = r == 0 ? gamma_te[l] : gw_nm1[(int64_t)(r - 1) * n + l];
    }
}

// Filament midpoints: chordwise (m, n+1) then spanwise (m+1, n); with their velocities.
__global__ void midpoints_kernel(const double* __restrict__ zeta, const double* __restrict__ zeta_dot, int m, int n,
                                 double* __restrict__ mp, double* __restrict__ mpd) {
    const int64_t nc = (int64_t)m * (n + 1), nf = nc + (int64_t)(m + 1) * n;
    const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    int64_t a, b;
    if (f < nc) {
        const int k = (int)(f / (n + 1)), l = (int)(f % (n + 1));
        a = (int64_t)k * (n + 1) + l;
        b = a + (n + 1);
    } else {
        const int64_t g = f - nc;
        const int k = (int)(g / n), l = (int)(g % n);
        a = (int64_t)k * (n + 1) + l;
        b = a + 1;
    }
    for (int d = 0; d < 3; ++d) {
        mp[f * 3 + d] = 0.5 * (zeta[a * 3 + d] + zeta[b * 3 + d]);
        mpd[f * 3 + d] = zeta_dot ? 0.5 * (zeta_dot[a * 3 + d] + zeta_dot[b * 3 + d]) : 0.0;
    }
}

// f = rho g (v_rel x r) per filament (aero/utils.py:167-210), g from the zero-padded
// ring differences and the TE spanwise filament's -gamma_w[0].
__global__ void filament_force_kernel(const double* __restrict__ zeta, const double* __restrict__ gamma_b,
                                      const double* __restrict__ gamma_w0, int m, int n,
                                      const double* __restrict__ mp, const double* __restrict__ mpd,
                                      const double* __restrict__ v, fj_flowfield flow, double t,
                                      double* __restrict__ ff) {
    const int64_t nc = (int64_t)m * (n + 1), nf = nc + (int64_t)(m + 1) * n;
    const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    auto G = [&](int k, int l) { return (k < 0 || l < 0 || k >= m || l >= n) ? 0.0 : gamma_b[(int64_t)k * n + l]; };
    int64_t a, b;
    double g;
    if (f < nc) {
        const int k = (int)(f / (n + 1)), l = (int)(f % (n + 1));
        a = (int64_t)k * (n + 1) + l;
        b = a + (n + 1);
        g = G(k, l) - G(k, l - 1);
    } else {
        const int64_t q = f - nc;
        const int k = (int)(q / n), l = (int)(q % n);
        a = (int64_t)k * (n + 1) + l;
        b = a + 1;
        g = G(k - 1, l) - G(k, l);
        if (k == m && gamma_w0) g -= gamma_w0[l];
    }
    const double x[3] = {mp[f * 3], mp[f * 3 + 1], mp[f * 3 + 2]};
    double u[3];
    flow_eval(flow, x, t, u);
    double vr[3], r[3];
    for (int d = 0; d < 3; ++d) {
        vr[d] = u[d] + v[f * 3 + d] - mpd[f * 3 + d];
        r[d] = zeta[b * 3 + d] - zeta[a * 3 + d];
    }
    const double s = flow.rho * g;
    ff[f * 3 + 0] = s * (vr[1] * r[2] - vr[2] * r[1]);
    ff[f * 3 + 1] = s * (vr[2] * r[0] - vr[0] * r[2]);
    ff[f * 3 + 2] = s * (vr[0] * r[1] - vr[1] * r[0]);
}

// split_to_vertex (algebra/array_utils.py:332-367) of the filament forces, plus the
// unsteady term split_to_vertex(rho gamma_dot nc, (0, 1)).
__global__ void vertex_force_kernel(const double* __restrict__ zeta, const double* __restrict__ ff,
                                    const double* __restrict__ gamma_dot, int m, int n, double rho,
                                    double* __restrict__ f_steady, double* __restrict__ f_unsteady) {
    const int64_t nv = (int64_t)(m + 1) * (n + 1);
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nv) return;
    const int k = (int)(i / (n + 1)), l = (int)(i % (n + 1));
    const int64_t nc = (int64_t)m * (n + 1);
    double fs[3] = {0.0, 0.0, 0.0};
    for (int d = 0; d < 3; ++d) {
        if (k < m) fs[d] += 0.5 * ff[((int64_t)k * (n + 1) + l) * 3 + d];
        if (k > 0) fs[d] += 0.5 * ff[((int64_t)(k - 1) * (n + 1) + l) * 3 + d];
        if (l < n) fs[d] += 0.5 * ff[(nc + (int64_t)k * n + l) * 3 + d];
        if (l > 0) fs[d] += 0.5 * ff[(nc + (int64_t)k * n + l - 1) * 3 + d];
        f_steady[i * 3 + d] = fs[d];
    }
    if (f_unsteady == nullptr) return;
    double fu[3] = {0.0, 0.0, 0.0};
    for (int dk = -1; dk <= 0; ++dk)
        for (int dl = -1; dl <= 0; ++dl) {
            const int pk = k + dk, pl = l + dl;
            if (pk < 0 || pl < 0 || pk >= m || pl >= n) continue;
            // nc of panel (pk, pl): (z11 - z00) x (z10 - z01), aero/utils.py:96-105
            const double* z00 = zeta + ((int64_t)pk * (n + 1) + pl) * 3;
            const double* z01 = z00 + 3;
            const double* z10 = z00 + (n + 1) * 3;
            const double* z11 = z10 + 3;
            double d1[3], d2[3];
            for (int d = 0; d < 3; ++d) {
                d1[d] = z11[d] - z00[d];
                d2[d] = z10[d] - z01[d];
            }
            const double ncp[3] = {d1[1] * d2[2] - d1[2] * d2[1], d1[2] * d2[0] - d1[0] * d2[2],
                                   d1[0] * d2[1] - d1[1] * d2[0]};
            const double w = 0.25 * rho * gamma_dot[(int64_t)pk * n + pl];
            for (int d = 0; d < 3; ++d) fu[d] += w * ncp[d];
        }
    for (int d = 0; d < 3; ++d) f_unsteady[i * 3 + d] = fu[d];
}

// Collocation points and area normals of a lattice (aero/utils.py:87-105).
__global__ void c_nc_kernel(const double* __restrict__ zeta, int m, int n, double* __restrict__ c,
                            double* __restrict__ nc) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (int64_t)m * n) return;
    const int k = (int)(p / n), l = (int)(p % n);
    const double* z00 = zeta + ((int64_t)k * (n + 1) + l) * 3;
    const double* z01 = z00 + 3;
    const double* z10 = z00 + (n + 1) * 3;
    const double* z11 = z10 + 3;
    double d1[3], d2[3];
    for (int d = 0; d < 3; ++d) {
        c[p * 3 + d] = 0.5 * (0.5 * (z00[d] + z10[d]) + 0.5 * (z01[d] + z11[d]));
        d1[d] = z11[d] - z00[d];
        d2[d] = z10[d] - z01[d];
    }
    nc[p * 3 + 0] = d1[1] * d2[2] - d1[2] * d2[1];
    nc[p * 3 + 1] = d1[2] * d2[0] - d1[0] * d2[2];
    nc[p * 3 + 2] = d1[0] * d2[1] - d1[1] * d2[0];
}

// lam_i = mu_i nc_i (the cotangent of the bound-lattice velocity at c_i) and the normal
// cotangent ncbar_i = mu_i V_i.
__global__ void aic_vjp_prep_kernel(const double* __restrict__ mu, const double* __restrict__ nc,
                                    const double* __restrict__ v, int64_t n_pan, double* __restrict__ lam,
                                    double* __restrict__ ncbar) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n_pan) return;
    for (int d = 0; d < 3; ++d) {
        lam[p * 3 + d] = mu[p] * nc[p * 3 + d];
        ncbar[p * 3 + d] = mu[p] * v[p * 3 + d];
    }
}

// Vertex cotangents of c (mean of the 4 panel vertices) and nc = d1 x d2 (gathered per
// vertex over its <= 4 panels, so no atomics): accumulated into zeta_bar.
__global__ void c_nc_transpose_kernel(const double* __restrict__ zeta, const double* __restrict__ cbar,
                                      const double* __restrict__ ncbar, int m, int n, double* __restrict__ zeta_bar) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)(m + 1) * (n + 1)) return;
    const int k = (int)(i / (n + 1)), l = (int)(i % (n + 1));
    double acc[3] = {0.0, 0.0, 0.0};
    for (int dk = -1; dk <= 0; ++dk)
        for (int dl = -1; dl <= 0; ++dl) {
            const int pk = k + dk, pl = l + dl;
            if (pk < 0 || pl < 0 || pk >= m || pl >= n) continue;
            const int64_t p = (int64_t)pk * n + pl;
            const double* z00 = zeta + ((int64_t)pk * (n + 1) + pl) * 3;
            const double* z01 = z00 + 3;
            const double* z10 = z00 + (n + 1) * 3;
            const double* z11 = z10 + 3;
            double d1[3], d2[3];
            for (int d = 0; d < 3; ++d) {
                d1[d] = z11[d] - z00[d];
                d2[d] = z10[d] - z01[d];
                acc[d] += 0.25 * cbar[p * 3 + d];
            }
            const double* nb = ncbar + p * 3;
            // d(nb . (d1 x d2))/d d1 = d2 x nb ; /d d2 = nb x d1
            const double b1[3] = {d2[1] * nb[2] - d2[2] * nb[1], d2[2] * nb[0] - d2[0] * nb[2],
                                  d2[0] * nb[1] - d2[1] * nb[0]};
            const double b2[3] = {nb[1] * d1[2] - nb[2] * d1[1], nb[2] * d1[0] - nb[0] * d1[2],
                                  nb[0] * d1[1] - nb[1] * d1[0]};
            // this vertex is z00 (dk=0,dl=0), z01 (dk=0,dl=-1), z10 (dk=-1,dl=0) or z11 (dk=-1,dl=-1)
            for (int d = 0; d < 3; ++d) {
                if (dk == 0 && dl == 0) acc[d] -= b1[d];
                if (dk == -1 && dl == -1) acc[d] += b1[d];
                if (dk == -1 && dl == 0) acc[d] += b2[d];
                if (dk == 0 && dl == -1) acc[d] -= b2[d];
            }
        }
    for (int d = 0; d < 3; ++d) zeta_bar[i * 3 + d] += acc[d];
}

// Transpose of the prescribed wake shift.
__global__ void wake_vjp_kernel(const double* __restrict__ zw_bar_n, const double* __restrict__ gw_bar_n, int n,
                                int m_star, double* __restrict__ zeta_te_bar, double* __restrict__ gamma_te_bar,
                                double* __restrict__ zw_bar_nm1, double* __restrict__ gw_bar_nm1) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nv = (int64_t)(m_star + 1) * (n + 1);
    if (i < nv) {
        const int r = (int)(i / (n + 1)), l = (int)(i % (n + 1));
        for (int d = 0; d < 3; ++d) {
            const double z = zw_bar_n[i * 3 + d];
            if (r == 0) {
                if (zeta_te_bar) zeta_te_bar[l * 3 + d] += z;
            } else if (zw_bar_nm1) {
                zw_bar_nm1[((int64_t)(r - 1) * (n + 1) + l) * 3 + d] += z;
            }
        }
    }
    if (i < (int64_t)m_star * n && gw_bar_n) {
        const int r = (int)(i / n), l = (int)(i % n);
        if (r == 0) {
            if (gamma_te_bar) gamma_te_bar[l] += gw_bar_n[i];
        } else if (gw_bar_nm1) {
            gw_bar_nm1[(int64_t)(r - 1) * n + l] += gw_bar_n[i];
        }
    }
}

}  // namespace

}  // namespace fj

using namespace fj;

extern "C" {

int fj_rhs_workspace_size(int64_t n_pan, const int* rows_w, const int* cols_w, int n_wake, int mirror,
                          int precision, size_t* bytes) {
    if (bytes == nullptr || n_pan < 0 || n_wake < 0) return fail(FJ_ERR_SHAPE, "rhs workspace: bad arguments");
    size_t vb = 0;
    if (n_wake > 0) FJ_TRY(fj_vind_workspace_size(n_pan, rows_w, cols_w, n_wake, mirror, precision, &vb));
    Arena a;
    a.carve<double>(std::max<int64_t>(n_pan, 1) * 3);
    a.carve<char>(vb);
    *bytes = a.used + 256;
    return FJ_OK;
}

int fj_rhs(const double* d_c, const double* d_nc, const double* d_c_dot, int64_t n_pan, const fj_flowfield* flow,
           double t, const double* const* d_zetas_w, const double* const* d_gammas_w, const int* rows_w,
           const int* cols_w, int n_wake, const double* mirror_point, const double* mirror_normal, int kernel,
           double r_cut, int precision, double* d_b, void* d_ws, size_t ws_bytes, fj_stream_t stream) {
    if (flow == nullptr) return fail(FJ_ERR_SHAPE, "fj_rhs: flow is null");
    const int mirror = mirror_point != nullptr && mirror_normal != nullptr;
    size_t need;
    FJ_TRY(fj_rhs_workspace_size(n_pan, rows_w, cols_w, n_wake, mirror, precision, &need));
    if (ws_bytes < need) return fail(FJ_ERR_NOMEM, "rhs workspace %zu < %zu", ws_bytes, need);
    if (n_pan == 0) return FJ_OK;
    cudaStream_t s = (cudaStream_t)stream;
    Arena a(d_ws, ws_bytes);
    double* v = a.carve<double>(n_pan * 3);
    char* vws = a.carve<char>(0);
    const size_t vws_bytes = ws_bytes - (size_t)(vws - (char*)d_ws);
    bool have_v = false;
    if (n_wake > 0) {
        FJ_TRY(fj_vind(d_c, n_pan, d_zetas_w, d_gammas_w, rows_w, cols_w, n_wake, mirror_point, mirror_normal,
                       kernel, r_cut, precision, v, vws, vws_bytes, stream));
        have_v = true;
    }
    rhs_kernel<<<nblk(n_pan), kFB, 0, s>>>(d_c, d_nc, d_c_dot, have_v ? v : nullptr, n_pan, *flow, t, d_b);
    note_launch();
    FJ_LAUNCH_CHECK("fj_rhs");
    return FJ_OK;
}

int fj_wake_shed_convect(const double* d_zeta_te_n, const double* d_gamma_te_nm1, const double* d_zeta_w_nm1,
                         const double* d_gamma_w_nm1, const double* d_v_conv, int n, int m_star,
                         const fj_flowfield* flow, double t, double dt, double* d_zeta_w_n, double* d_gamma_w_n,
                         fj_stream_t stream) {
    if (flow == nullptr || n <= 0 || m_star < 0) return fail(FJ_ERR_SHAPE, "fj_wake_shed_convect: n=%d m_star=%d", n, m_star);
    const int64_t nv = (int64_t)(m_star + 1) * (n + 1);
    wake_shed_kernel<<<nblk(nv), kFB, 0, (cudaStream_t)stream>>>(d_zeta_te_n, d_gamma_te_nm1, d_zeta_w_nm1,
                                                                   d_gamma_w_nm1, d_v_conv, n, m_star, *flow, t, dt,
                                                                   d_zeta_w_n, d_gamma_w_n);
    note_launch();
    FJ_LAUNCH_CHECK("fj_wake_shed_convect");
    return FJ_OK;
}

int fj_forces_workspace_size(int m, int n, const int* rows, const int* cols, int n_lat, int mirror, int precision,
                             size_t* bytes) {
    if (bytes == nullptr || m <= 0 || n <= 0) return fail(FJ_ERR_SHAPE, "forces workspace: m=%d n=%d", m, n);
    const int64_t nf = (int64_t)m * (n + 1) + (int64_t)(m + 1) * n;
    size_t vb = 0;
    FJ_TRY(fj_vind_workspace_size(nf, rows, cols, n_lat, mirror, precision, &vb));
    Arena a;
    a.carve<double>(nf * 3);  // midpoints
    a.carve<double>(nf * 3);  // midpoint velocities
    a.carve<double>(nf * 3);  // induced velocity
    a.carve<double>(nf * 3);  // filament forces
    a.carve<char>(vb);
    *bytes = a.used + 256;
    return FJ_OK;
}

int fj_forces(const double* d_zeta_b, const double* d_zeta_b_dot, const double* d_gamma_b, const double* d_gamma_w0,
              const double* d_gamma_b_dot, int m, int n, const fj_flowfield* flow, double t,
              const double* const* d_zetas, const double* const* d_gammas, const int* rows, const int* cols, int n_lat,
              const double* mirror_point, const double* mirror_normal, int kernel, double r_cut, int precision,
              double* d_f_steady, double* d_f_unsteady, void* d_ws, size_t ws_bytes, fj_stream_t stream) {
    if (flow == nullptr) return fail(FJ_ERR_SHAPE, "fj_forces: flow is null");
    const int mirror = mirror_point != nullptr && mirror_normal != nullptr;
    size_t need;
    FJ_TRY(fj_forces_workspace_size(m, n, rows, cols, n_lat, mirror, precision, &need));
    if (ws_bytes < need) return fail(FJ_ERR_NOMEM, "forces workspace %zu < %zu", ws_bytes, need);
    if (d_f_unsteady != nullptr && d_gamma_b_dot == nullptr)
        return fail(FJ_ERR_SHAPE, "fj_forces: f_unsteady requested without gamma_b_dot");
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t nf = (int64_t)m * (n + 1) + (int64_t)(m + 1) * n;
    Arena a(d_ws, ws_bytes);
    double* mp = a.carve<double>(nf * 3);
    double* mpd = a.carve<double>(nf * 3);
    double* v = a.carve<double>(nf * 3);
    double* ff = a.carve<double>(nf * 3);
    char* vws = a.carve<char>(0);
    const size_t vws_bytes = ws_bytes - (size_t)(vws - (char*)d_ws);
    midpoints_kernel<<<nblk(nf), kFB, 0, s>>>(d_zeta_b, d_zeta_b_dot, m, n, mp, mpd);
    note_launch();
    FJ_TRY(fj_vind(mp, nf, d_zetas, d_gammas, rows, cols, n_lat, mirror_point, mirror_normal, kernel, r_cut,
                   precision, v, vws, vws_bytes, stream));
    filament_force_kernel<<<nblk(nf), kFB, 0, s>>>(d_zeta_b, d_gamma_b, d_gamma_w0, m, n, mp, mpd, v, *flow, t, ff);
    note_launch();
    const int64_t nv = (int64_t)(m + 1) * (n + 1);
    vertex_force_kernel<<<nblk(nv), kFB, 0, s>>>(d_zeta_b, ff, d_gamma_b_dot, m, n, flow->rho, d_f_steady,
                                                  d_f_unsteady);
    note_launch();
    FJ_LAUNCH_CHECK("fj_forces");
    return FJ_OK;
}

int fj_aic_vjp_workspace_size(int m, int n, size_t* bytes) {
    if (bytes == nullptr || m <= 0 || n <= 0) return fail(FJ_ERR_SHAPE, "aic_vjp workspace: m=%d n=%d", m, n);
    const int64_t np = (int64_t)m * n;
    size_t vb = 0, jb = 0;
    FJ_TRY(fj_vind_workspace_size(np, &m, &n, 1, 0, FJ_PREC_FP64, &vb));
    FJ_TRY(fj_vind_vjp_workspace_size(np, &m, &n, 1, 0, &jb));
    Arena a;
    for (int k = 0; k < 5; ++k) a.carve<double>(np * 3);  // c, nc, v, lam, ncbar
    a.carve<double>(np * 3);                              // cbar
    a.carve<char>(std::max(vb, jb));
    *bytes = a.used + 256;
    return FJ_OK;
}

int fj_aic_vjp(const double* d_zeta, int m, int n, const double* d_gamma, const double* d_mu, int kernel,
               double* d_zeta_bar, void* d_ws, size_t ws_bytes, fj_stream_t stream) {
    if (kernel != FJ_KERNEL_EPSILON)
        return fail(FJ_ERR_UNSUPPORTED, "fj_aic_vjp: only the epsilon kernel has a hand-written adjoint");
    size_t need;
    FJ_TRY(fj_aic_vjp_workspace_size(m, n, &need));
    if (ws_bytes < need) return fail(FJ_ERR_NOMEM, "aic_vjp workspace %zu < %zu", ws_bytes, need);
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t np = (int64_t)m * n;
    Arena a(d_ws, ws_bytes);
    double* c = a.carve<double>(np * 3);
    double* nc = a.carve<double>(np * 3);
    double* v = a.carve<double>(np * 3);
    double* lam = a.carve<double>(np * 3);
    double* ncbar = a.carve<double>(np * 3);
    double* cbar = a.carve<double>(np * 3);
    char* vws = a.carve<char>(0);
    const size_t vws_bytes = ws_bytes - (size_t)(vws - (char*)d_ws);
    c_nc_kernel<<<nblk(np), kFB, 0, s>>>(d_zeta, m, n, c, nc);
    note_launch();
    // V_i = bound-lattice velocity at c_i; mu^T A Gamma = sum_i mu_i nc_i . V_i
    FJ_TRY(fj_vind(c, np, &d_zeta, &d_gamma, &m, &n, 1, nullptr, nullptr, kernel, 0.0, FJ_PREC_FP64, v, vws, vws_bytes,
                   stream));
    aic_vjp_prep_kernel<<<nblk(np), kFB, 0, s>>>(d_mu, nc, v, np, lam, ncbar);
    note_launch();
    FJ_CUDA(cudaMemsetAsync(cbar, 0, np * 3 * sizeof(double), s));
    double* zb[1] = {d_zeta_bar};
    FJ_TRY(fj_vind_vjp(c, np, &d_zeta, &d_gamma, &m, &n, 1, nullptr, nullptr, kernel, 0.0, lam, cbar, zb, nullptr,
                       vws, vws_bytes, stream));
    c_nc_transpose_kernel<<<nblk((int64_t)(m + 1) * (n + 1)), kFB, 0, s>>>(d_zeta, cbar, ncbar, m, n, d_zeta_bar);
    note_launch();
    FJ_LAUNCH_CHECK("fj_aic_vjp");
    return FJ_OK;
}

int fj_wake_vjp(const double* d_zeta_w_bar_n, const double* d_gamma_w_bar_n, int n, int m_star, double* d_zeta_te_bar,
                double* d_gamma_te_bar, double* d_zeta_w_bar_nm1, double* d_gamma_w_bar_nm1, fj_stream_t stream) {
    if (n <= 0 || m_star < 0) return fail(FJ_ERR_SHAPE, "fj_wake_vjp: n=%d m_star=%d", n, m_star);
    const int64_t nv = (int64_t)(m_star + 1) * (n + 1);
    wake_vjp_kernel<<<nblk(nv), kFB, 0, (cudaStream_t)stream>>>(d_zeta_w_bar_n, d_gamma_w_bar_n, n, m_star,
                                                                  d_zeta_te_bar, d_gamma_te_bar, d_zeta_w_bar_nm1,
                                                                  d_gamma_w_bar_nm1);
    note_launch();
    FJ_LAUNCH_CHECK("fj_wake_vjp");
    return FJ_OK;
}

}  // extern "C"
