// fj_flow.cuh -- background flow fields on the device (aero/flowfields.py).
#pragma once

#include "fj_common.cuh"

namespace fj {

// Background flow, aero/flowfields.py:87-181.
__device__ __forceinline__ void flow_eval(const fj_flowfield& f, const double x[3], double t, double u[3]) {
    if (f.kind == FJ_FLOW_ONE_MINUS_COSINE) {
        double rx = x[0] - f.gust_x0[0], ry = x[1] - f.gust_x0[1], rz = x[2] - f.gust_x0[2];
        if (f.relative_motion) {
            rx -= f.u_inf[0] * t;
            ry -= f.u_inf[1] * t;
            rz -= f.u_inf[2] * t;
        }
        const double gx = rx * f.gust_travel_dir[0] + ry * f.gust_travel_dir[1] + rz * f.gust_travel_dir[2];
        if (gx > 0.0 && gx < 2.0 * f.gust_length) {
            const double w = 1.0 - cos(kPi * gx / f.gust_length);
            u[0] = f.gust_amplitude_dir[0] * f.gust_amplitude * 0.5 * w;
            u[1] = f.gust_amplitude_dir[1] * f.gust_amplitude * 0.5 * w;
            u[2] = f.gust_amplitude_dir[2] * f.gust_amplitude * 0.5 * w;
        } else {
            u[0] = u[1] = u[2] = 0.0;
        }
        if (f.relative_motion) {
            u[0] += f.u_inf[0];
            u[1] += f.u_inf[1];
            u[2] += f.u_inf[2];
        }
    } else {
        if (f.relative_motion) {
            u[0] = f.u_inf[0];
            u[1] = f.u_inf[1];
            u[2] = f.u_inf[2];
        } else {
            u[0] = u[1] = u[2] = 0.0;
        }
    }
}

}  // namespace fj
