// fj_bsgrad.cuh -- derivatives of one Biot-Savart filament (FP64), shared by the
// adjoint sums (fj_adjoint.cu) and the dense influence Jacobians (fj_jac.cu).
//
// With r1 = x - y0, r2 = x - y1, r0 = y1 - y0 = r1 - r2, c = r1 x r2,
// u_i = r_i / n_i, n_i = sqrt(|r_i|^2 + eps^2), dot = r0.(u1 - u2), D = |c|^2 + eps|r0|^4
// (epsilon kernel, aero/utils.py:606-623) or |c|^2 (cutoff kernel, :626-648, whose pairs
// within the cutoff radius of the filament line contribute nothing, derivative included),
// s = dot / (4 pi D), a = lam.c:
//   d(lam.K)/dr1 = s (r2 x lam) + a [ddot/dr1 - (dot / D) dD/dr1] / (4 pi D)
//   d(lam.K)/dr2 = s (lam x r1) + a [ddot/dr2 - (dot / D) dD/dr2] / (4 pi D)
//   ddot/dr1 = (u1 - u2) + (r0 - (r0.u1) u1) / n1,  ddot/dr2 = -(u1 - u2) - (r0 - (r0.u2) u2) / n2
//   dD/dr1 = 2 (r2 x c) + 4 eps |r0|^2 r0,          dD/dr2 = 2 (c x r1) - 4 eps |r0|^2 r0
// and x_bar = d/dr1 + d/dr2, y0_bar = -d/dr1, y1_bar = -d/dr2.
#pragma once

#include "fj_common.cuh"

namespace fj {

// Per vertex one reciprocal square root and per link one division (1 / (4 pi D)); the
// other quotients are products with these reciprocals (the FP64 divide and square root
// are multi-instruction sequences on the FP64 pipe).
struct VtxA {
    double d[3];  // x - y
    double u[3];  // d / n
    double rn;    // 1 / n, n = sqrt(|d|^2 + eps^2)
};

__device__ __forceinline__ void vtxa(const double x[3], double yx, double yy, double yz, VtxA& o) {
    o.d[0] = x[0] - yx;
    o.d[1] = x[1] - yy;
    o.d[2] = x[2] - yz;
    o.rn = rsqrt(o.d[0] * o.d[0] + o.d[1] * o.d[1] + o.d[2] * o.d[2] + kEps * kEps);
    o.u[0] = o.d[0] * o.rn;
    o.u[1] = o.d[1] * o.rn;
    o.u[2] = o.d[2] * o.rn;
}

__device__ __forceinline__ void cross3(const double a[3], const double b[3], double o[3]) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

__device__ __forceinline__ double dot3(const double a[3], const double b[3]) {
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

// d(lam . K)/dr1 -> g1, d(lam . K)/dr2 -> g2 (each scaled by g), and lam . K (unit g).
// KER: FJ_KERNEL_EPSILON (D = |c|^2 + eps |r0|^4) or FJ_KERNEL_CUTOFF (D = |c|^2, zero
// within rc2 of the filament line, aero/utils.py:637-648).
template <int KER>
__device__ __forceinline__ void link_vjp(const VtxA& A, const VtxA& B, const double r0[3], double g,
                                         const double lam[3], double rc2, double g1[3], double g2[3], double& lk) {
    double c[3];
    cross3(A.d, B.d, c);
    const double du[3] = {A.u[0] - B.u[0], A.u[1] - B.u[1], A.u[2] - B.u[2]};
    const double dot = dot3(r0, du);
    const double r0sq = dot3(r0, r0);
    if (KER == FJ_KERNEL_CUTOFF) {
        const double sm = dot3(r0, A.d) / r0sq;
        const double mx = A.d[0] - sm * r0[0], my = A.d[1] - sm * r0[1], mz = A.d[2] - sm * r0[2];
        if (!(mx * mx + my * my + mz * mz > rc2)) {
            g1[0] = g1[1] = g1[2] = g2[0] = g2[1] = g2[2] = 0.0;
            lk = 0.0;
            return;
        }
    }
    const double eps_term = KER == FJ_KERNEL_EPSILON ? kEps * r0sq * r0sq : 0.0;
    const double D = dot3(c, c) + eps_term;
    const double inv = 1.0 / (kFourPi * D);
    const double s = dot * inv;
    const double a = dot3(lam, c);
    lk = s * a;
    const double r0u1 = dot3(r0, A.u), r0u2 = dot3(r0, B.u);
    double t1[3], t2[3], dD1[3], dD2[3];
    cross3(B.d, lam, t1);  // r2 x lam
    cross3(lam, A.d, t2);  // lam x r1
    double r2c[3], cr1[3];
    cross3(B.d, c, r2c);
    cross3(c, A.d, cr1);
    const double e4 = KER == FJ_KERNEL_EPSILON ? 4.0 * kEps * r0sq : 0.0;
    for (int k = 0; k < 3; ++k) {
        dD1[k] = 2.0 * r2c[k] + e4 * r0[k];
        dD2[k] = 2.0 * cr1[k] - e4 * r0[k];
    }
    const double q = kFourPi * s;  // dot / D
    for (int k = 0; k < 3; ++k) {
        const double dd1 = du[k] + (r0[k] - r0u1 * A.u[k]) * A.rn;
        const double dd2 = -du[k] - (r0[k] - r0u2 * B.u[k]) * B.rn;
        g1[k] = g * (s * t1[k] + a * (dd1 - q * dD1[k]) * inv);
        g2[k] = g * (s * t2[k] + a * (dd2 - q * dD2[k]) * inv);
    }
}

}  // namespace fj
