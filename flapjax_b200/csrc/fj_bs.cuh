// fj_bs.cuh -- the reference's Biot-Savart segment kernels in FP64, split into a
// per-(target, vertex) part and a per-(target, filament) part so that chains of
// filaments can share vertex work.  The formulas of each filament are those of
// aero/utils.py:580-648; the quotients are formed as products with one reciprocal square
// root per vertex and one division per filament (the FP64 divide and square root are
// multi-instruction sequences on the FP64 pipe), and the cutoff kernel's radial distance
// from the filament line is computed as the reference computes it.
#pragma once

#include "fj_common.cuh"

namespace fj {

template <int KER>
struct Vtx64 {
    double d[3];  // x - y
    double u[3];  // (x - y) / ||x - y||_eps  (plain kernel: / ||x - y||)
};

template <int KER>
__device__ __forceinline__ void vtx64(const double x[3], double yx, double yy, double yz,
                                      Vtx64<KER>& o) {
    o.d[0] = x[0] - yx;
    o.d[1] = x[1] - yy;
    o.d[2] = x[2] - yz;
    const double n2 = o.d[0] * o.d[0] + o.d[1] * o.d[1] + o.d[2] * o.d[2];
    // r / jnp.linalg.norm(r) (plain, aero/utils.py:591); r / ||r||_eps (make_unit_epsilon,
    // :603, and the epsilon kernel's rsqrt, :617-618)
    const double inv = rsqrt(KER == FJ_KERNEL_PLAIN ? n2 : n2 + kEps * kEps);
    o.u[0] = o.d[0] * inv;
    o.u[1] = o.d[1] * inv;
    o.u[2] = o.d[2] * inv;
}

template <int KER>
__device__ __forceinline__ void link64(const Vtx64<KER>& a, const Vtx64<KER>& b, double g,
                                       double r0x, double r0y, double r0z, double q, double rc2,
                                       double acc[3]) {
    // r1 = a.d (x - y0), r2 = b.d (x - y1), r0 = y1 - y0
    const double cx = a.d[1] * b.d[2] - a.d[2] * b.d[1];
    const double cy = a.d[2] * b.d[0] - a.d[0] * b.d[2];
    const double cz = a.d[0] * b.d[1] - a.d[1] * b.d[0];
    const double dot = r0x * (a.u[0] - b.u[0]) + r0y * (a.u[1] - b.u[1]) + r0z * (a.u[2] - b.u[2]);
    const double c2 = cx * cx + cy * cy + cz * cz;
    if (KER == FJ_KERNEL_EPSILON) {
        // aero/utils.py:619-623
        const double val = dot / (kFourPi * (c2 + q));
        acc[0] += (cx * val) * g;
        acc[1] += (cy * val) * g;
        acc[2] += (cz * val) * g;
    } else if (KER == FJ_KERNEL_CUTOFF) {
        // aero/utils.py:637-648: radial distance from the filament line
        const double sm = (r0x * a.d[0] + r0y * a.d[1] + r0z * a.d[2]) / q;
        const double mx = a.d[0] - sm * r0x, my = a.d[1] - sm * r0y, mz = a.d[2] - sm * r0z;
        const double r2 = mx * mx + my * my + mz * mz;
        if (r2 > rc2) {
            const double val = dot / (kFourPi * c2);
            acc[0] += (cx * val) * g;
            acc[1] += (cy * val) * g;
            acc[2] += (cz * val) * g;
        }
    } else {
        // aero/utils.py:587-592
        const double val = dot / (c2 * 4.0 * kPi);
        acc[0] += (cx * val) * g;
        acc[1] += (cy * val) * g;
        acc[2] += (cz * val) * g;
    }
}

}  // namespace fj
