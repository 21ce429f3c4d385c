// fj_step.cu -- one UVLM time step on the device, the case driver and the C ABI.
//
// A dynamic step at slot i (case_solve -> base_solve_from_grid, aero/uvlm.py:824-1215):
//   1. node frames -> lattices: zeta_b(i), zeta_b_dot(i), zeta_b(i-1)   (uvlm.py:537-621)
//      and collocation points / area normals / c_dot                     (uvlm.py:885-893)
//   2. free wake: v at wake vertices of slot i-1 from bound(i-1) + wake(i-1)
//      (uvlm.py:914-929); shed the TE row and convect (aero/utils.py:400-500)
//   3. AIC of the bound lattice (aero/aic.py:137-187)
//   4. RHS = -((U - c_dot + v_wake) . n)                                 (uvlm.py:961-983)
//   5. solve                                                               (uvlm.py:985)
//   6. forces: v at filament midpoints from bound(i) + wake(i), Kutta-Joukowski per
//      filament, split to vertices                                        (aero/utils.py:126-223)
//   7. gamma_dot filter, unsteady force, strip alpha, force total         (uvlm.py:1048-1103)
// Every array is addressed as field + slot * slot_size, surfaces concatenated.
#include <cmath>
#include <cstring>
#include <algorithm>
#include <atomic>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "fj_aic.cuh"
#include "fj_lu.cuh"
#include "fj_flow.cuh"
#include "fj_vind.cuh"

namespace fj {

const char* last_error();
int biot_savart_pairs(const double* x, const double* y, int64_t n, int kernel, double r_cut, double* out,
                      cudaStream_t s);

// ------------------------------------------------------------------------------------
// Layout of the per-surface blocks inside one time slot
// ------------------------------------------------------------------------------------
struct Layout {
    int n_surf;
    int m[FJ_MAX_SURF], n[FJ_MAX_SURF], ms[FJ_MAX_SURF];
    int64_t vo[FJ_MAX_SURF + 1];   // bound vertices
    int64_t po[FJ_MAX_SURF + 1];   // bound panels
    int64_t wvo[FJ_MAX_SURF + 1];  // wake vertices
    int64_t wpo[FJ_MAX_SURF + 1];  // wake panels
    int64_t so[FJ_MAX_SURF + 1];   // strips
    int64_t dofo[FJ_MAX_SURF + 1]; // dof mapping entries (n+1)
    int64_t fo[FJ_MAX_SURF + 1];   // bound filaments m(n+1) + (m+1)n
    int64_t wto[FJ_MAX_SURF + 1];  // free-wake targets (m_star + var)(n+1)
    int64_t dwo[FJ_MAX_SURF + 1];  // delta_w entries m_star
    int64_t xvo[FJ_MAX_SURF + 1];  // variable wake: vertices before re-discretisation (m_star+2)(n+1)
    int64_t xpo[FJ_MAX_SURF + 1];  // variable wake: circulations before re-discretisation (m_star+1)n
    int var[FJ_MAX_SURF];          // 1: variable wake discretisation (delta_w)
    int any_var;
    int n_nodes;                   // beam nodes in the frame arrays
    int pp[FJ_MAX_SURF];           // polar table points per strip (0: no polar correction)
    int64_t plo[FJ_MAX_SURF + 1];  // polar tables: doubles before surface s (n * pp * 4 each)
    int any_polar;
};

static Layout make_layout(const fj_case_config& c) {
    Layout L;
    memset(&L, 0, sizeof(L));
    L.n_surf = c.n_surf;
    L.n_nodes = c.n_nodes;
    for (int s = 0; s < c.n_surf; ++s) {
        const int m = c.m[s], n = c.n[s], ms = c.m_star[s];
        L.m[s] = m;
        L.n[s] = n;
        L.ms[s] = ms;
        L.vo[s + 1] = L.vo[s] + (int64_t)(m + 1) * (n + 1);
        L.po[s + 1] = L.po[s] + (int64_t)m * n;
        L.wvo[s + 1] = L.wvo[s] + (int64_t)(ms + 1) * (n + 1);
        L.wpo[s + 1] = L.wpo[s] + (int64_t)ms * n;
        L.so[s + 1] = L.so[s] + n;
        L.dofo[s + 1] = L.dofo[s] + n + 1;
        L.fo[s + 1] = L.fo[s] + (int64_t)m * (n + 1) + (int64_t)(m + 1) * n;
        const int var = c.variable_wake[s] ? 1 : 0;
        L.var[s] = var;
        L.any_var |= var;
        // with delta_w every wake row is convected (aero/utils.py:431-436)
        L.wto[s + 1] = L.wto[s] + (int64_t)(ms + var) * (n + 1);
        L.dwo[s + 1] = L.dwo[s] + ms;
        L.xvo[s + 1] = L.xvo[s] + (var ? (int64_t)(ms + 2) * (n + 1) : 0);
        L.xpo[s + 1] = L.xpo[s] + (var ? (int64_t)(ms + 1) * n : 0);
        L.pp[s] = c.polar_points[s];
        L.plo[s + 1] = L.plo[s] + (int64_t)n * c.polar_points[s] * 4;
        L.any_polar |= c.polar_points[s] > 0 ? 1 : 0;
    }
    return L;
}

__device__ __forceinline__ int find_surf(const int64_t* off, int n_surf, int64_t idx) {
    int s = 0;
    while (s + 1 < n_surf && idx >= off[s + 1]) ++s;
    return s;
}

// ------------------------------------------------------------------------------------
// 1. geometry
// ------------------------------------------------------------------------------------
// se3.vect_product (algebra/se3.py:209-216): hg[:3,:3] @ x + hg[:3,3]
__device__ __forceinline__ void se3_apply(const double* hg, const double x[3], double o[3]) {
#pragma unroll
    for (int r = 0; r < 3; ++r) o[r] = (hg[r * 4 + 0] * x[0] + hg[r * 4 + 1] * x[1] + hg[r * 4 + 2] * x[2]) + hg[r * 4 + 3];
}

// ------------------------------------------------------------------------------------
// Per-step kernels.  Each reads its case from a table (blockIdx.y = case), so one launch
// advances one case or a whole batch of cases.
// ------------------------------------------------------------------------------------
struct StepCase {
    Layout L;
    int nb;
    int i;            // slot written by this step
    int free_wake;
    double dt, relax;
    fj_flowfield flow;
    const double* zeta0;
    const int32_t* dof;
    const double* hg_n;
    const double* hgd_n;   // null: zero lattice velocity (static solve)
    const double* hg_nm1;  // null: no lattice at n-1 (static solve)
    double* t;             // time array; t[i] = t[i-1] + dt when i > 0 and advance_time
    int advance_time;
    double* zb_n;
    double* zbd_n;
    double* zw_n;
    const double* zw_nm1;
    double* c;
    double* nc;
    double* gb_n;
    const double* gb_nm1;
    double* gbd_n;
    const double* gbd_nm1;  // null: no gamma_dot (static solve)
    double* gw_n;
    const double* gw_nm1;
    const double* gw_force; // wake circulation seen by the trailing-edge filament force
    double* fs;
    double* fu;
    double* alpha;
    double* ft;
    double* zb_nm1;         // workspace
    double* c_dot;          // null: no lattice velocity in the RHS (static solve)
    double* targets;
    double* v;
    double* ffil;
    double* rhs;
    const double* v_wake;   // free-wake convection velocities (null: prescribed wake)
    const double* delta_w;  // variable wake segment lengths (Layout::dwo blocks)
    double* zw_tmp;         // variable wake before re-discretisation (Layout::xvo blocks)
    double* gw_tmp;         // (Layout::xpo blocks)
    double* s_tmp;          // arc length along each wake column (Layout::xvo blocks)
    const double* v_rhs;    // wake velocity at collocation points (null: static solve)
    const double* zeta_ref; // mixed path: lattice of the cached AIC (null: no comparison)
    int* changed;           // mixed path: set to 1 when zb_n differs from zeta_ref
    int* nonfinite;         // lowest slot whose total force is not finite (sentinel: none)
    const double* polars;   // polar tables (Layout::plo blocks; null: no polar correction)
    double* polar_tmp;      // per strip: sectional force (3), couple (3), lift scale
    double polar_scale;     // polar_circulation_scale
};

// Also clears the lattice-changed flag that k_changed sets later in the step (nothing in
// between reads it).
__global__ void k_time(const StepCase* __restrict__ T) {
    const StepCase& C = T[blockIdx.y];
    if (threadIdx.x == 0 && C.advance_time && C.i > 0) C.t[C.i] = C.t[C.i - 1] + C.dt;  // uvlm.py:1158-1161
    if (threadIdx.x == 0 && C.changed != nullptr) *C.changed = 0;
}

// hg_to_zeta_b / hg_dot_to_zeta_b_dot (aero/uvlm.py:537-621), one thread per vertex.
__global__ void k_geom_vertices(const StepCase* __restrict__ T) {
    const StepCase& C = T[blockIdx.y];
    const Layout& L = C.L;
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= L.vo[L.n_surf]) return;
    const int s = find_surf(L.vo, L.n_surf, v);
    const int j = (int)((v - L.vo[s]) % (L.n[s] + 1));
    // the host validates the mapping; the clamp only keeps a bad entry in bounds
    const int node = min(max(C.dof[L.dofo[s] + j], 0), L.n_nodes - 1);
    const double x0[3] = {C.zeta0[v * 3], C.zeta0[v * 3 + 1], C.zeta0[v * 3 + 2]};
    double o[3];
    se3_apply(C.hg_n + (int64_t)node * 16, x0, o);
    for (int d = 0; d < 3; ++d) C.zb_n[v * 3 + d] = o[d];
    if (C.hgd_n != nullptr) {
        se3_apply(C.hgd_n + (int64_t)node * 16, x0, o);
    } else {
        o[0] = o[1] = o[2] = 0.0;
    }
    for (int d = 0; d < 3; ++d) C.zbd_n[v * 3 + d] = o[d];
    if (C.hg_nm1 != nullptr) {
        se3_apply(C.hg_nm1 + (int64_t)node * 16, x0, o);
        for (int d = 0; d < 3; ++d) C.zb_nm1[v * 3 + d] = o[d];
    }
}

// compute_surf_c / compute_surf_nc (aero/utils.py:87-105) and c_dot (uvlm.py:891-893).
__global__ void k_geom_panels(const StepCase* __restrict__ T) {
    const StepCase& C = T[blockIdx.y];
    const Layout& L = C.L;
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= L.po[L.n_surf]) return;
    const int s = find_surf(L.po, L.n_surf, p);
    const int64_t lp = p - L.po[s];
    const int n = L.n[s];
    const int k = (int)(lp / n), l = (int)(lp % n);
    const double* z00 = C.zb_n + (L.vo[s] + (int64_t)k * (n + 1) + l) * 3;
    const double* z01 = z00 + 3;
    const double* z10 = z00 + (n + 1) * 3;
    const double* z11 = z10 + 3;
    for (int d = 0; d < 3; ++d) {
        // neighbour_average over axis 0 then axis 1 (algebra/array_utils.py:106-136)
        const double a0 = 0.5 * (z00[d] + z10[d]);
        const double a1 = 0.5 * (z01[d] + z11[d]);
        C.c[p * 3 + d] = 0.5 * (a0 + a1);
    }
    const double d1[3] = {z11[0] - z00[0], z11[1] - z00[1], z11[2] - z00[2]};
    const double d2[3] = {z10[0] - z01[0], z10[1] - z01[1], z10[2] - z01[2]};
    C.nc[p * 3 + 0] = d1[1] * d2[2] - d1[2] * d2[1];
    C.nc[p * 3 + 1] = d1[2] * d2[0] - d1[0] * d2[2];
    C.nc[p * 3 + 2] = d1[0] * d2[1] - d1[1] * d2[0];
    if (C.c_dot != nullptr) {
        const double* w00 = C.zbd_n + (L.vo[s] + (int64_t)k * (n + 1) + l) * 3;
        const double* w01 = w00 + 3;
        const double* w10 = w00 + (n + 1) * 3;
        const double* w11 = w10 + 3;
        for (int d = 0; d < 3; ++d) {
            const double a0 = 0.5 * (w00[d] + w10[d]);
            const double a1 = 0.5 * (w01[d] + w11[d]);
            C.c_dot[p * 3 + d] = 0.5 * (a0 + a1);
        }
    }
}

// ------------------------------------------------------------------------------------
// wake
// ------------------------------------------------------------------------------------
// initialise_wake (uvlm.py:662-689): TE + cumsum(dt |U|) along the freestream direction.
// `hs_len` > 0 builds the 2-row horseshoe wake instead (uvlm.py:642-660).
__global__ void init_wake_kernel(Layout L, const double* __restrict__ zeta_b, fj_flowfield f, double dt,
                                 double hs_len, double* __restrict__ zeta_w, int rows_override,
                                 const double* __restrict__ delta_w) {
    // rows_override > 0: that many rows for every surface that has a wake, 0 rows
    // (the TE only) for surfaces with m_star == 0 (uvlm.py:652-660)
    int64_t tot = 0;
    for (int q = 0; q < L.n_surf; ++q) {
        const int rows = rows_override > 0 ? (L.ms[q] == 0 ? 0 : rows_override) : L.ms[q];
        tot += (int64_t)(rows + 1) * (L.n[q] + 1);
    }
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= tot) return;
    int s = 0;
    int64_t base = 0, nxt = 0;
    for (s = 0; s < L.n_surf; ++s) {
        const int rows = rows_override > 0 ? (L.ms[s] == 0 ? 0 : rows_override) : L.ms[s];
        nxt = base + (int64_t)(rows + 1) * (L.n[s] + 1);
        if (v < nxt) break;
        base = nxt;
    }
    const int64_t lv = v - base;
    const int n = L.n[s];
    const int r = (int)(lv / (n + 1)), l = (int)(lv % (n + 1));
    const double* te = zeta_b + (L.vo[s] + (int64_t)L.m[s] * (n + 1) + l) * 3;
    const double umag = sqrt(f.u_inf[0] * f.u_inf[0] + f.u_inf[1] * f.u_inf[1] + f.u_inf[2] * f.u_inf[2]);
    double sdist;
    if (hs_len > 0.0) {
        sdist = r == 0 ? 0.0 : hs_len;
    } else if (L.var[s] && delta_w != nullptr) {
        sdist = 0.0;  // cumsum(delta_w), uvlm.py:672-683
        for (int q = 0; q < r; ++q) sdist += delta_w[L.dwo[s] + q];
    } else {
        sdist = 0.0;  // cumsum of equal increments, summed in order as jnp.cumsum
        const double inc = 1.0 * dt * umag;
        for (int q = 0; q < r; ++q) sdist += inc;
    }
    for (int d = 0; d < 3; ++d) zeta_w[v * 3 + d] = te[d] + sdist * (f.u_inf[d] / umag);
}

// Rows 0..m_star-1 of every surface's wake at n-1, packed as the free-wake target list.
__global__ void k_gather_wake_targets(const StepCase* __restrict__ T) {
    const StepCase& C = T[blockIdx.y];
    const Layout& L = C.L;
    if (!C.free_wake) return;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= L.wto[L.n_surf]) return;
    const int s = find_surf(L.wto, L.n_surf, t);
    const int64_t src = L.wvo[s] + (t - L.wto[s]);
    for (int d = 0; d < 3; ++d) C.targets[t * 3 + d] = C.zw_nm1[src * 3 + d];
}

// propagate_surf_wake, uniform branch (aero/utils.py:427-450): shed the TE row and
// circulation of step n-1, drop the last row, convect the rest by dt * (U + v_ind).
__global__ void k_wake_shed(const StepCase* __restrict__ T) {
    const StepCase& C = T[blockIdx.y];
    const Layout& L = C.L;
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nv = L.wvo[L.n_surf];
    const double t = C.t[C.i];
    if (v < nv) {
        const int s = find_surf(L.wvo, L.n_surf, v);
        const int64_t lv = v - L.wvo[s];
        const int n = L.n[s];
        const int r = (int)(lv / (n + 1)), l = (int)(lv % (n + 1));
        if (L.var[s]) {
            // variable wake: k_wake_shed_var and the re-discretisation write this surface
        } else if (r == 0) {
            const double* te = C.zb_n + (L.vo[s] + (int64_t)L.m[s] * (n + 1) + l) * 3;
            for (int d = 0; d < 3; ++d) C.zw_n[v * 3 + d] = te[d];
        } else {
            const int64_t src = L.wvo[s] + (int64_t)(r - 1) * (n + 1) + l;
            const double x[3] = {C.zw_nm1[src * 3], C.zw_nm1[src * 3 + 1], C.zw_nm1[src * 3 + 2]};
            double u[3];
            flow_eval(C.flow, x, t, u);
            if (C.v_wake != nullptr) {
                const int64_t ti = L.wto[s] + (int64_t)(r - 1) * (n + 1) + l;
                u[0] += C.v_wake[ti * 3];
                u[1] += C.v_wake[ti * 3 + 1];
                u[2] += C.v_wake[ti * 3 + 2];
            }
            for (int d = 0; d < 3; ++d) C.zw_n[v * 3 + d] = x[d] + C.dt * u[d];
        }
    }
    const int64_t g = v - nv;
    if (g >= 0 && g < L.wpo[L.n_surf]) {
        const int s = find_surf(L.wpo, L.n_surf, g);
        const int64_t lg = g - L.wpo[s];
        const int n = L.n[s];
        const int r = (int)(lg / n), l = (int)(lg % n);
        if (!L.var[s])
            C.gw_n[g] = r == 0 ? C.gb_nm1[L.po[s] + (int64_t)(L.m[s] - 1) * n + l]
                               : C.gw_nm1[L.wpo[s] + (int64_t)(r - 1) * n + l];
    }
}

// propagate_surf_wake with delta_w (aero/utils.py:427-491), part 1: shed the TE row and
// convect EVERY row of the wake at n-1 (m_star+2 vertex rows, m_star+1 circulation rows).
__global__ void k_wake_shed_var(const StepCase* __restrict__ T) {
    const StepCase& C = T[blockIdx.y];
    const Layout& L = C.L;
    if (!L.any_var || C.zw_tmp == nullptr) return;
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nv = L.xvo[L.n_surf];
    const double t = C.t[C.i];
    if (v < nv) {
        const int s = find_surf(L.xvo, L.n_surf, v);
        const int64_t lv = v - L.xvo[s];
        const int n = L.n[s];
        const int r = (int)(lv / (n + 1)), l = (int)(lv % (n + 1));
        if (r == 0) {
            const double* te = C.zb_n + (L.vo[s] + (int64_t)L.m[s] * (n + 1) + l) * 3;
            for (int d = 0; d < 3; ++d) C.zw_tmp[v * 3 + d] = te[d];
        } else {
            const int64_t src = L.wvo[s] + (int64_t)(r - 1) * (n + 1) + l;
            const double x[3] = {C.zw_nm1[src * 3], C.zw_nm1[src * 3 + 1], C.zw_nm1[src * 3 + 2]};
            double u[3];
            flow_eval(C.flow, x, t, u);
            if (C.v_wake != nullptr) {
                const int64_t ti = L.wto[s] + (int64_t)(r - 1) * (n + 1) + l;
                u[0] += C.v_wake[ti * 3];
                u[1] += C.v_wake[ti * 3 + 1];
                u[2] += C.v_wake[ti * 3 + 2];
            }
            for (int d = 0; d < 3; ++d) C.zw_tmp[v * 3 + d] = x[d] + C.dt * u[d];
        }
    }
    const int64_t g = v - nv;
    if (g >= 0 && g < L.xpo[L.n_surf]) {
        const int s = find_surf(L.xpo, L.n_surf, g);
        const int64_t lg = g - L.xpo[s];
        const int n = L.n[s];
        const int r = (int)(lg / n), l = (int)(lg % n);
        C.gw_tmp[g] = r == 0 ? C.gb_nm1[L.po[s] + (int64_t)(L.m[s] - 1) * n + l]
                             : C.gw_nm1[L.wpo[s] + (int64_t)(r - 1) * n + l];
    }
}

// np.interp(x, xp, fp) for increasing xp of length np_ (strided by `st`): fp[0] left of
// xp[0], fp[-1] right of xp[-1], else fp[j] + slope (x - xp[j]) on xp[j] <= x < xp[j+1].
template <typename XP, typename FP>
__device__ __forceinline__ double interp1(double x, int np_, XP xp, FP fp) {
    if (!(x >= xp(0))) return fp(0);
    if (x >= xp(np_ - 1)) return fp(np_ - 1);
    int lo = 0, hi = np_ - 1;  // invariant xp(lo) <= x < xp(hi)
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (xp(mid) <= x) lo = mid; else hi = mid;
    }
    const double slope = (fp(hi) - fp(lo)) / (xp(hi) - xp(lo));
    return slope * (x - xp(lo)) + fp(lo);
}

// Part 2: arc length along each vertex column of the convected wake, and the vertices
// re-interpolated at the prescribed arc lengths [0, cumsum(delta_w)].  Thread per
// (surface, column).
__global__ void k_wake_redisc_z(const StepCase* __restrict__ T) {
    const StepCase& C = T[blockIdx.y];
    const Layout& L = C.L;
    if (!L.any_var || C.zw_tmp == nullptr) return;
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= L.dofo[L.n_surf]) return;
    const int s = find_surf(L.dofo, L.n_surf, idx);
    if (!L.var[s]) return;
    const int n = L.n[s], ms = L.ms[s];
    const int l = (int)(idx - L.dofo[s]);
    const double* X = C.zw_tmp + L.xvo[s] * 3;
    double* S = C.s_tmp + L.xvo[s];
    const int np_ = ms + 2;
    S[l] = 0.0;
    for (int r = 1; r < np_; ++r) {
        const double* a = X + ((int64_t)(r - 1) * (n + 1) + l) * 3;
        const double* b = X + ((int64_t)r * (n + 1) + l) * 3;
        const double dx = b[0] - a[0], dy = b[1] - a[1], dz = b[2] - a[2];
        S[(int64_t)r * (n + 1) + l] = S[(int64_t)(r - 1) * (n + 1) + l] + sqrt(dx * dx + dy * dy + dz * dz);
    }
    auto xp = [&](int r) { return S[(int64_t)r * (n + 1) + l]; };
    const double* dw = C.delta_w + L.dwo[s];
    double sd = 0.0;
    for (int q = 0; q <= ms; ++q) {
        if (q > 0) sd += dw[q - 1];
        double* out = C.zw_n + (L.wvo[s] + (int64_t)q * (n + 1) + l) * 3;
        for (int d = 0; d < 3; ++d)
            out[d] = interp1(sd, np_, xp, [&](int r) { return X[((int64_t)r * (n + 1) + l) * 3 + d]; });
    }
}

// Part 3: circulations re-interpolated from the panel-centre arc lengths
// (neighbour_average of the vertex arc lengths over both axes) at the midpoints of the
// prescribed segments.  Thread per (surface, circulation column).
__global__ void k_wake_redisc_g(const StepCase* __restrict__ T) {
    const StepCase& C = T[blockIdx.y];
    const Layout& L = C.L;
    if (!L.any_var || C.zw_tmp == nullptr) return;
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= L.so[L.n_surf]) return;
    const int s = find_surf(L.so, L.n_surf, idx);
    if (!L.var[s] || L.ms[s] == 0) return;
    const int n = L.n[s], ms = L.ms[s];
    const int l = (int)(idx - L.so[s]);
    const double* S = C.s_tmp + L.xvo[s];
    const double* G = C.gw_tmp + L.xpo[s];
    auto sz = [&](int r, int c) { return S[(int64_t)r * (n + 1) + c]; };
    auto xp = [&](int r) {
        return 0.5 * (0.5 * (sz(r, l) + sz(r + 1, l)) + 0.5 * (sz(r, l + 1) + sz(r + 1, l + 1)));
    };
    auto fp = [&](int r) { return G[(int64_t)r * n + l]; };
    const double* dw = C.delta_w + L.dwo[s];
    double s0 = 0.0;
    for (int q = 0; q < ms; ++q) {
        const double s1 = s0 + dw[q];
        C.gw_n[L.wpo[s] + (int64_t)q * n + l] = interp1(0.5 * (s0 + s1), ms + 1, xp, fp);
        s0 = s1;
    }
}

// Static wake circulation: broadcast of the TE row (uvlm.py:995-1012).
__global__ void static_gamma_w_kernel(Layout L, const double* __restrict__ gamma_b, double* __restrict__ gamma_w,
                                      int rows_override) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t base = 0;
    for (int s = 0; s < L.n_surf; ++s) {
        const int rows = rows_override >= 0 ? (L.ms[s] == 0 ? 0 : rows_override) : L.ms[s];
        const int64_t cnt = (int64_t)rows * L.n[s];
        if (g < base + cnt) {
            const int l = (int)((g - base) % L.n[s]);
            gamma_w[g] = gamma_b[L.po[s] + (int64_t)(L.m[s] - 1) * L.n[s] + l];
            return;
        }
        base += cnt;
    }
}

// Mixed path: flag a lattice that differs (bitwise) from the one of the cached AIC.
__global__ void k_changed(const StepCase* __restrict__ T) {
    const StepCase& C = T[blockIdx.y];
    if (C.changed == nullptr) return;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < C.L.vo[C.L.n_surf] * 3 && C.zb_n[i] != C.zeta_ref[i]) *C.changed = 1;
}

// ------------------------------------------------------------------------------------
// right-hand side (uvlm.py:961-985): b = -((U(c) - c_dot + v_wake) . n)
// ------------------------------------------------------------------------------------
__global__ void k_rhs(const StepCase* __restrict__ T) {
    const StepCase& C = T[blockIdx.y];
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= C.nb) return;
    const double t = C.t[C.i];
    const double x[3] = {C.c[p * 3], C.c[p * 3 + 1], C.c[p * 3 + 2]};
    double u[3];
    flow_eval(C.flow, x, t, u);
    if (C.c_dot != nullptr)
        for (int d = 0; d < 3; ++d) u[d] -= C.c_dot[p * 3 + d];
    if (C.v_rhs != nullptr)
        for (int d = 0; d < 3; ++d) u[d] += C.v_rhs[p * 3 + d];
    C.rhs[p] = -(u[0] * C.nc[p * 3] + u[1] * C.nc[p * 3 + 1] + u[2] * C.nc[p * 3 + 2]);
}

// ------------------------------------------------------------------------------------
// forces (aero/utils.py:126-223)
// ------------------------------------------------------------------------------------
// Filament f of surface s: f < m(n+1): chordwise (k,l)->(k+1,l); else spanwise (k,l)->(k,l+1).
__device__ __forceinline__ void filament_ends(const Layout& L, int s, int64_t lf, int& k0, int& l0, int& k1,
                                              int& l1, bool& chord) {
    const int m = L.m[s], n = L.n[s];
    const int64_t nm = (int64_t)m * (n + 1);
    if (lf < nm) {
        chord = true;
        k0 = (int)(lf / (n + 1));
        l0 = (int)(lf % (n + 1));
        k1 = k0 + 1;
        l1 = l0;
    } else {
        chord = false;
        const int64_t t = lf - nm;
        k0 = (int)(t / n);
        l0 = (int)(t % n);
        k1 = k0;
        l1 = l0 + 1;
    }
}

__global__ void k_force_targets(const StepCase* __restrict__ T) {
    const StepCase& C = T[blockIdx.y];
    const Layout& L = C.L;
    const int64_t fi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (fi >= L.fo[L.n_surf]) return;
    const int s = find_surf(L.fo, L.n_surf, fi);
    int k0, l0, k1, l1;
    bool chord;
    filament_ends(L, s, fi - L.fo[s], k0, l0, k1, l1, chord);
    const int n = L.n[s];
    const double* a = C.zb_n + (L.vo[s] + (int64_t)k0 * (n + 1) + l0) * 3;
    const double* b = C.zb_n + (L.vo[s] + (int64_t)k1 * (n + 1) + l1) * 3;
    for (int d = 0; d < 3; ++d) C.targets[fi * 3 + d] = 0.5 * (a[d] + b[d]);
}

__global__ void k_force_filament(const StepCase* __restrict__ T) {
    const StepCase& C = T[blockIdx.y];
    const Layout& L = C.L;
    const int64_t fi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (fi >= L.fo[L.n_surf]) return;
    const double t = C.t[C.i];
    const int s = find_surf(L.fo, L.n_surf, fi);
    int k0, l0, k1, l1;
    bool chord;
    filament_ends(L, s, fi - L.fo[s], k0, l0, k1, l1, chord);
    const int m = L.m[s], n = L.n[s];
    const double* gb = C.gb_n + L.po[s];
    const int64_t ia = L.vo[s] + (int64_t)k0 * (n + 1) + l0;
    const int64_t ib = L.vo[s] + (int64_t)k1 * (n + 1) + l1;
    const double* a = C.zb_n + ia * 3;
    const double* b = C.zb_n + ib * 3;
    const double x[3] = {C.targets[fi * 3], C.targets[fi * 3 + 1], C.targets[fi * 3 + 2]};
    double u[3];
    flow_eval(C.flow, x, t, u);
    double vr[3];
    for (int d = 0; d < 3; ++d) {
        const double mpd = 0.5 * (C.zbd_n[ia * 3 + d] + C.zbd_n[ib * 3 + d]);
        vr[d] = (u[d] + C.v[fi * 3 + d]) - mpd;
    }
    double g;
    if (chord) {  // gamma_chordwise[:, :-1] = G; gamma_chordwise[:, 1:] += -G
        g = 0.0;
        if (l0 < n) g = gb[(int64_t)k0 * n + l0];
        if (l0 >= 1) g += -gb[(int64_t)k0 * n + l0 - 1];
    } else {      // gamma_spanwise[:-1, :] = -G; gamma_spanwise[1:, :] += G; [-1] += -Gw[0]
        g = 0.0;
        if (k0 < m) g = -gb[(int64_t)k0 * n + l0];
        if (k0 >= 1) g += gb[(int64_t)(k0 - 1) * n + l0];
        if (k0 == m && C.gw_force != nullptr && L.ms[s] > 0) g += -C.gw_force[L.wpo[s] + l0];
    }
    const double r[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
    const double cr[3] = {vr[1] * r[2] - vr[2] * r[1], vr[2] * r[0] - vr[0] * r[2], vr[0] * r[1] - vr[1] * r[0]};
    for (int d = 0; d < 3; ++d) C.ffil[fi * 3 + d] = C.flow.rho * (g * cr[d]);
}

// compute_gamma_dot (uvlm.py:691-715)
__global__ void k_gamma_dot(const StepCase* __restrict__ T) {
    const StepCase& C = T[blockIdx.y];
    if (C.gbd_nm1 == nullptr) return;
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= C.nb) return;
    const double cur = (C.gb_n[p] - C.gb_nm1[p]) / C.dt;
    C.gbd_n[p] = cur * C.relax + C.gbd_nm1[p] * (1.0 - C.relax);
}

// split_to_vertex of the filament forces (aero/utils.py:220-222) and of
// rho * gamma_dot * n (uvlm.py:1093-1103), algebra/array_utils.py:332-367.
// parts: 1 the steady forces, 2 the unsteady ones, 3 both.
__global__ void k_vertex_forces(const StepCase* __restrict__ T, int parts) {
    const StepCase& C = T[blockIdx.y];
    const Layout& L = C.L;
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= L.vo[L.n_surf]) return;
    const int s = find_surf(L.vo, L.n_surf, v);
    const int64_t lv = v - L.vo[s];
    const int m = L.m[s], n = L.n[s];
    const int k = (int)(lv / (n + 1)), l = (int)(lv % (n + 1));
    const double* fc = C.ffil + L.fo[s] * 3;                          // (m, n+1, 3)
    const double* fsp = C.ffil + (L.fo[s] + (int64_t)m * (n + 1)) * 3;  // (m+1, n, 3)
    const double rho = C.flow.rho;
    for (int d = 0; d < 3 && (parts & 1); ++d) {
        double a = 0.0;  // split_to_vertex(f_chordwise, 0)
        if (k < m) a = 0.5 * fc[((int64_t)k * (n + 1) + l) * 3 + d];
        if (k >= 1) a += 0.5 * fc[((int64_t)(k - 1) * (n + 1) + l) * 3 + d];
        double b = 0.0;  // split_to_vertex(f_spanwise, 1)
        if (l < n) b = 0.5 * fsp[((int64_t)k * n + l) * 3 + d];
        if (l >= 1) b += 0.5 * fsp[((int64_t)k * n + l - 1) * 3 + d];
        C.fs[v * 3 + d] = a + b;
    }
    const bool has_gd = C.gbd_nm1 != nullptr;
    for (int d = 0; d < 3 && (parts & 2); ++d) {
        double out = 0.0;
        if (has_gd) {
            const double* g = C.gbd_n + L.po[s];
            const double* nn = C.nc + L.po[s] * 3;
            // split along axis 0 into (m+1, n), then along axis 1 into (m+1, n+1)
            auto s0 = [&](int kk, int ll) -> double {
                double r = 0.0;
                if (kk < m) r = 0.5 * (rho * g[(int64_t)kk * n + ll] * nn[((int64_t)kk * n + ll) * 3 + d]);
                if (kk >= 1) r += 0.5 * (rho * g[(int64_t)(kk - 1) * n + ll] * nn[((int64_t)(kk - 1) * n + ll) * 3 + d]);
                return r;
            };
            if (l < n) out = 0.5 * s0(k, l);
            if (l >= 1) out += 0.5 * s0(k, l - 1);
        }
        C.fu[v * 3 + d] = out;
    }
}

// strip_alpha (aero/utils.py:226-273), one thread per strip.
__global__ void k_strip_alpha(const StepCase* __restrict__ T) {
    const StepCase& C = T[blockIdx.y];
    const Layout& L = C.L;
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= L.so[L.n_surf]) return;
    const double t = C.t[C.i];
    const int s = find_surf(L.so, L.n_surf, j);
    const int l = (int)(j - L.so[s]);
    const int m = L.m[s], n = L.n[s];
    const double* z = C.zb_n + L.vo[s] * 3;
    const double* le0 = z + (int64_t)l * 3;
    const double* le1 = le0 + 3;
    const double* te0 = z + ((int64_t)m * (n + 1) + l) * 3;
    const double* te1 = te0 + 3;
    double le[3], te[3], chord[3], span[3], mid[3];
    for (int d = 0; d < 3; ++d) {
        le[d] = 0.5 * (le0[d] + le1[d]);
        te[d] = 0.5 * (te0[d] + te1[d]);
        chord[d] = te[d] - le[d];
        span[d] = 0.5 * ((le1[d] + te1[d]) - (le0[d] + te0[d]));
        mid[d] = 0.5 * (le[d] + te[d]);
    }
    const double c_len = sqrt(chord[0] * chord[0] + chord[1] * chord[1] + chord[2] * chord[2]);
    const double b_len = sqrt(span[0] * span[0] + span[1] * span[1] + span[2] * span[2]);
    const double es[3] = {span[0] / b_len, span[1] / b_len, span[2] / b_len};
    double vr[3];
    flow_eval(C.flow, mid, t, vr);
    const double vmag2 = vr[0] * vr[0] + vr[1] * vr[1] + vr[2] * vr[2];
    double el[3] = {vr[1] * es[2] - vr[2] * es[1], vr[2] * es[0] - vr[0] * es[2], vr[0] * es[1] - vr[1] * es[0]};
    const double eln = sqrt(el[0] * el[0] + el[1] * el[1] + el[2] * el[2]);
    el[0] /= eln;
    el[1] /= eln;
    el[2] /= eln;
    double fst[3] = {0.0, 0.0, 0.0};
    const double* fsv = C.fs + L.vo[s] * 3;
    for (int k = 0; k <= m; ++k)
        for (int d = 0; d < 3; ++d)
            fst[d] += 0.5 * (fsv[((int64_t)k * (n + 1) + l) * 3 + d] + fsv[((int64_t)k * (n + 1) + l + 1) * 3 + d]);
    const double q = 0.5 * C.flow.rho * vmag2;
    const double cl = (fst[0] * el[0] + fst[1] * el[1] + fst[2] * el[2]) / (q * c_len * b_len);
    C.alpha[j] = cl / (2.0 * kPi);
}

// apply_polar_correction (aero/utils.py:276-397), per strip of a surface with polars:
// strip frame (e_c, e_s, e_n), freestream at the strip centre, polar(alpha) by linear
// interpolation in the strip's table with the end values held (np.interp), the lift
// scale cl / (2 pi alpha), the sectional force q c b (cl e_l + cd e_d) and couple
// q c b cm e_n into polar_tmp.
__device__ __forceinline__ void polar_lookup(const double* tab, int np_, double a, double out[3]) {
    // tab: np_ rows of (alpha, cl, cd, cm), alpha ascending
    if (!(a > tab[0])) {  // below the table (and NaN, which np.interp maps to the end too)
        for (int q = 0; q < 3; ++q) out[q] = tab[1 + q];
        if (a != a)
            for (int q = 0; q < 3; ++q) out[q] = a;
        return;
    }
    if (a >= tab[(int64_t)(np_ - 1) * 4]) {
        for (int q = 0; q < 3; ++q) out[q] = tab[(int64_t)(np_ - 1) * 4 + 1 + q];
        return;
    }
    int lo = 0, hi = np_ - 1;  // tab[lo].alpha <= a < tab[hi].alpha
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (tab[(int64_t)mid * 4] <= a) lo = mid;
        else hi = mid;
    }
    const double* r0 = tab + (int64_t)lo * 4;
    const double* r1 = tab + (int64_t)hi * 4;
    for (int q = 0; q < 3; ++q) {
        const double slope = (r1[1 + q] - r0[1 + q]) / (r1[0] - r0[0]);
        out[q] = r0[1 + q] + slope * (a - r0[0]);
    }
}

__global__ void k_polar_strips(const StepCase* __restrict__ T) {
    const StepCase& C = T[blockIdx.y];
    const Layout& L = C.L;
    if (C.polars == nullptr) return;
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= L.so[L.n_surf]) return;
    const int s = find_surf(L.so, L.n_surf, j);
    if (L.pp[s] == 0) return;
    const double t = C.t[C.i];
    const int l = (int)(j - L.so[s]);
    const int m = L.m[s], n = L.n[s];
    const double* z = C.zb_n + L.vo[s] * 3;
    const double* le0 = z + (int64_t)l * 3;
    const double* le1 = le0 + 3;
    const double* te0 = z + ((int64_t)m * (n + 1) + l) * 3;
    const double* te1 = te0 + 3;
    double le[3], te[3], chord[3], span[3], mid[3];
    for (int d = 0; d < 3; ++d) {
        le[d] = 0.5 * (le0[d] + le1[d]);
        te[d] = 0.5 * (te0[d] + te1[d]);
        chord[d] = te[d] - le[d];
        span[d] = 0.5 * ((le1[d] + te1[d]) - (le0[d] + te0[d]));
        mid[d] = 0.5 * (le[d] + te[d]);
    }
    const double c_len = sqrt(chord[0] * chord[0] + chord[1] * chord[1] + chord[2] * chord[2]);
    const double b_len = sqrt(span[0] * span[0] + span[1] * span[1] + span[2] * span[2]);
    const double ec[3] = {chord[0] / c_len, chord[1] / c_len, chord[2] / c_len};
    const double es[3] = {span[0] / b_len, span[1] / b_len, span[2] / b_len};
    double en[3] = {ec[1] * es[2] - ec[2] * es[1], ec[2] * es[0] - ec[0] * es[2], ec[0] * es[1] - ec[1] * es[0]};
    const double enn = sqrt(en[0] * en[0] + en[1] * en[1] + en[2] * en[2]);
    for (int d = 0; d < 3; ++d) en[d] /= enn;
    double vr[3];
    flow_eval(C.flow, mid, t, vr);
    const double vmag2 = vr[0] * vr[0] + vr[1] * vr[1] + vr[2] * vr[2];
    const double vmag = sqrt(vmag2);
    const double q = 0.5 * C.flow.rho * vmag2;
    double el[3] = {vr[1] * es[2] - vr[2] * es[1], vr[2] * es[0] - vr[0] * es[2], vr[0] * es[1] - vr[1] * es[0]};
    const double eln = sqrt(el[0] * el[0] + el[1] * el[1] + el[2] * el[2]);
    for (int d = 0; d < 3; ++d) el[d] /= eln;
    const double ed[3] = {vr[0] / vmag, vr[1] / vmag, vr[2] / vmag};
    const double a = C.alpha[j];
    double cf[3];
    polar_lookup(C.polars + L.plo[s] + (int64_t)l * L.pp[s] * 4, L.pp[s], a, cf);
    const double cl_uvlm = 2.0 * kPi * a;
    const double qcb = q * c_len * b_len;
    double* o = C.polar_tmp + j * 7;
    for (int d = 0; d < 3; ++d) {
        o[d] = qcb * (cf[0] * el[d] + cf[1] * ed[d]);
        o[3 + d] = (qcb * cf[2]) * en[d];
    }
    o[6] = fabs(cl_uvlm) > kEps ? cf[0] / cl_uvlm : 1.0;
}

// The corrected steady forces of a surface with polars, one thread per vertex: the
// sectional force at c/4 by the triangular chordwise weights, half to each of the strip's
// two vertex columns, and the couple as opposing leading/trailing-edge forces.
__global__ void k_polar_vertices(const StepCase* __restrict__ T) {
    const StepCase& C = T[blockIdx.y];
    const Layout& L = C.L;
    if (C.polars == nullptr) return;
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= L.vo[L.n_surf]) return;
    const int s = find_surf(L.vo, L.n_surf, v);
    if (L.pp[s] == 0) return;
    const int64_t lv = v - L.vo[s];
    const int m = L.m[s], n = L.n[s];
    const int k = (int)(lv / (n + 1)), l = (int)(lv % (n + 1));
    const double frac = (double)k / (double)m;  // linspace(0, 1, m + 1)
    const double w = fmin(fmax(1.0 - fabs(frac - 0.25) * m, 0.0), 1.0);
    double f[3] = {0.0, 0.0, 0.0};
    for (int sj = l - 1; sj <= l; ++sj) {
        if (sj < 0 || sj >= n) continue;
        const double* o = C.polar_tmp + (L.so[s] + sj) * 7;
        for (int d = 0; d < 3; ++d) {
            f[d] += 0.5 * w * o[d];
            if (k == 0) f[d] += 0.5 * o[3 + d];
            if (k == m) f[d] -= 0.5 * o[3 + d];
        }
    }
    for (int d = 0; d < 3; ++d) C.fs[v * 3 + d] = f[d];
}

// Blend Gamma_b towards the polar lift: gamma *= 1 + scale (lift_scale - 1) per strip
// (uvlm.py:1066-1075).
__global__ void k_polar_gamma(const StepCase* __restrict__ T) {
    const StepCase& C = T[blockIdx.y];
    const Layout& L = C.L;
    if (C.polars == nullptr || C.polar_scale == 0.0) return;
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= L.po[L.n_surf]) return;
    const int s = find_surf(L.po, L.n_surf, p);
    if (L.pp[s] == 0) return;
    const int l = (int)((p - L.po[s]) % L.n[s]);
    C.gb_n[p] *= 1.0 + C.polar_scale * (C.polar_tmp[(L.so[s] + l) * 7 + 6] - 1.0);
}

// Sum over vertices of f_steady + f_unsteady (one CTA per case, fixed order).
__global__ void k_force_total(const StepCase* __restrict__ T) {
    const StepCase& C = T[blockIdx.y];
    const int64_t nv = C.L.vo[C.L.n_surf];
    __shared__ double sh[3][256];
    double a[3] = {0.0, 0.0, 0.0};
    for (int64_t v = threadIdx.x; v < nv; v += blockDim.x)
        for (int d = 0; d < 3; ++d) a[d] += C.fs[v * 3 + d] + C.fu[v * 3 + d];
    for (int d = 0; d < 3; ++d) sh[d][threadIdx.x] = a[d];
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int d = 0; d < 3; ++d) sh[d][threadIdx.x] += sh[d][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        for (int d = 0; d < 3; ++d) C.ft[d] = sh[d][0];
        // every output of the step feeds the total force: a NaN/Inf anywhere shows here
        if (C.nonfinite != nullptr && !(isfinite(sh[0][0]) && isfinite(sh[1][0]) && isfinite(sh[2][0])))
            atomicMin(C.nonfinite, C.i);
    }
}

static inline unsigned nblk(int64_t n, int b = 256) { return (unsigned)((n + b - 1) / b); }

// ------------------------------------------------------------------------------------
// Case plan: layout, workspace carve-up, validation
// ------------------------------------------------------------------------------------
// Mixed path: the RHS sums the first kNearWakeRows wake rows in FP64 and the rest in FP32.
// Row 0's leading filament lies on the trailing edge, a quarter panel from the last row of
// collocation points, where one filament's term is several times the whole normalwash: its
// FP32 rounding alone moved Gamma by ~2e-7 relative, and the unsteady force
// rho (dGamma/dt) A n turns that into ~2e-6 of the drag.  With four rows in FP64 the rest
// of the wake moves Gamma by ~1e-8 (16 x 128 wing, W = 200); the FP64 part is 2 % of the
// wake's links.  The force and convection sums stay FP32 whole.
constexpr int kNearWakeRows = 4;

struct Plan {
    fj_case_config cfg;
    Layout L;
    int nb;                      // AIC order
    int64_t sz_zb, sz_zw, sz_pan, sz_gw, sz_strip;  // per-slot element counts
    int64_t max_targets, max_stream;
    int64_t part_elems;
    size_t ws_needed;    // bytes of workspace this plan carves
    // workspace
    int* flags;          // [0] lu info, [1] geometry changed
    double* zeta_nm1;    // bound vertices at n-1
    double* c_dot;
    double* targets;
    double* v;
    double* part;
    void* stream;
    Elem64* stream_near; // mixed path: FP64 stream of the near-wake rows for the RHS (null on FP64)
    double* hs_zw;       // horseshoe wake scratch
    double* hs_gw;
    double* v_conv;      // free-wake convection velocities of the last step solved (wake targets x 3)
    double* zw_tmp;      // variable wake scratch (null when no surface has delta_w)
    double* gw_tmp;
    double* s_tmp;
    double* a64;         // FP64 AIC (factored in place on the FP64 path)
    float* a32;          // FP32 LU factors (mixed)
    float* x32;          // FP32 inverse (mixed)
    float* tri32;        // triangular-block inverses of the tensor-core factorisation (mixed)
    double* zeta_ref;    // lattice of the cached AIC (mixed) or of the cached FP64 factors
    int32_t* piv;
    double* rhs;
    double* r;
    double* resid;       // per-slot refinement residual (mixed)
    double* ffil;
    double* polar_tmp;   // polar correction: 7 doubles per strip (null without polars)
    char* tab;           // device table of a one-case step
    size_t tab_bytes;
    char* tab_all;       // graph-replayed steps: the table of every slot (n_tstep x tab_bytes)
    int* step_ctr;       // graph-replayed steps: slot whose table the next replay selects
};

static int validate(const fj_case_config* c) {
    if (c == nullptr) return fail(FJ_ERR_SHAPE, "config is NULL");
    if (c->n_surf < 1 || c->n_surf > FJ_MAX_SURF) return fail(FJ_ERR_SHAPE, "n_surf=%d not in [1,%d]", c->n_surf, FJ_MAX_SURF);
    for (int s = 0; s < c->n_surf; ++s) {
        if (c->m[s] < 1 || c->n[s] < 1 || c->m_star[s] < 0)
            return fail(FJ_ERR_SHAPE, "surface %d: m=%d n=%d m_star=%d", s, c->m[s], c->n[s], c->m_star[s]);
    }
    for (int s = 0; s < c->n_surf; ++s)
        if (c->variable_wake[s] != 0 && c->variable_wake[s] != 1)
            return fail(FJ_ERR_SHAPE, "variable_wake[%d]=%d must be 0 or 1", s, c->variable_wake[s]);
    for (int s = 0; s < c->n_surf; ++s)
        if (c->polar_points[s] < 0) return fail(FJ_ERR_SHAPE, "polar_points[%d]=%d", s, c->polar_points[s]);
    if (!(c->polar_circulation_scale >= 0.0 && c->polar_circulation_scale <= 1.0))
        return fail(FJ_ERR_SHAPE, "polar_circulation_scale=%g not in [0, 1]", c->polar_circulation_scale);
    if (c->n_tstep < 1) return fail(FJ_ERR_SHAPE, "n_tstep=%d", c->n_tstep);
    if (c->n_nodes < 1) return fail(FJ_ERR_SHAPE, "n_nodes=%d", c->n_nodes);
    if (!(c->dt > 0.0) || !std::isfinite(c->dt)) return fail(FJ_ERR_SHAPE, "dt=%g must be positive", c->dt);
    if (c->kernel < 0 || c->kernel > 2) return fail(FJ_ERR_UNSUPPORTED, "kernel id %d", c->kernel);
    if (c->precision != FJ_PREC_FP64 && c->precision != FJ_PREC_MIXED)
        return fail(FJ_ERR_UNSUPPORTED, "precision id %d", c->precision);
    if (c->precision == FJ_PREC_MIXED && c->kernel == FJ_KERNEL_PLAIN)
        return fail(FJ_ERR_UNSUPPORTED, "the unregularised kernel is FP64-only");
    if (c->kernel == FJ_KERNEL_CUTOFF && !(c->r_cut >= 0.0)) return fail(FJ_ERR_SHAPE, "r_cut=%g", c->r_cut);
    const double* u = c->flow.u_inf;
    if (!(u[0] * u[0] + u[1] * u[1] + u[2] * u[2] > 0.0)) return fail(FJ_ERR_SHAPE, "u_inf must be non-zero");
    int64_t nb = 0;
    for (int s = 0; s < c->n_surf; ++s) nb += (int64_t)c->m[s] * c->n[s];
    if (nb > 6144) return fail(FJ_ERR_UNSUPPORTED, "AIC order %lld exceeds 6144", (long long)nb);
    return FJ_OK;
}

struct TableLayout {
    size_t step, pack_free, pack_wake, pack_bound, pack_near, job_free, job_rhs, job_force, job_near, cta_free,
        cta_rhs, cta_force, cta_near, aic, refine, total;
};

static TableLayout table_layout(int k) {
    TableLayout t;
    size_t o = 0;
    auto take = [&](size_t bytes) {
        o = align_up(o, 256);
        const size_t at = o;
        o += bytes;
        return at;
    };
    t.step = take(k * sizeof(StepCase));
    t.pack_free = take(k * sizeof(PackJob));
    t.pack_wake = take(k * sizeof(PackJob));
    t.pack_bound = take(k * sizeof(PackJob));
    t.pack_near = take(k * sizeof(PackJob));
    t.job_free = take(k * sizeof(VindJob));
    t.job_rhs = take(k * sizeof(VindJob));
    t.job_force = take(k * sizeof(VindJob));
    t.job_near = take(k * sizeof(VindJob));
    t.cta_free = take((k + 1) * sizeof(int64_t));
    t.cta_rhs = take((k + 1) * sizeof(int64_t));
    t.cta_force = take((k + 1) * sizeof(int64_t));
    t.cta_near = take((k + 1) * sizeof(int64_t));
    t.aic = take(k * sizeof(AicArgs));
    t.refine = take(k * sizeof(RefineJob));
    t.total = align_up(o, 256);
    return t;
}

static int make_plan(const fj_case_config* cfg, void* ws, size_t ws_bytes, Plan& p) {
    FJ_TRY(validate(cfg));
    p.cfg = *cfg;
    p.L = make_layout(*cfg);
    const Layout& L = p.L;
    const int ns = L.n_surf;
    p.nb = (int)L.po[ns];
    p.sz_zb = L.vo[ns] * 3;
    p.sz_zw = L.wvo[ns] * 3;
    p.sz_pan = L.po[ns];
    p.sz_gw = L.wpo[ns];
    p.sz_strip = L.so[ns];
    const int img = cfg->mirror ? 2 : 1;
    int64_t stream = 0;
    for (int s = 0; s < ns; ++s) {
        stream += img * (stream_len(L.m[s], L.n[s]) + stream_len(std::max(L.ms[s], 1), L.n[s]));
        // mixed: a wake longer than the near rows goes in as two lattices that both hold the
        // split row: one more spanwise chain (n+1 elements) and one more element in each of
        // the n+1 chordwise chains
        if (cfg->precision == FJ_PREC_MIXED && L.ms[s] > kNearWakeRows) stream += img * 2ll * (L.n[s] + 1);
    }
    p.max_stream = stream;
    p.max_targets = std::max<int64_t>(std::max<int64_t>(L.wto[ns], L.fo[ns]), L.po[ns]);
    // partial buffers for each of the three target sets at the full stream length
    int64_t part = 0;
    const int64_t sets[3] = {L.wto[ns], L.fo[ns], L.po[ns]};
    for (int64_t nt : sets) {
        if (nt == 0) continue;
        part = std::max<int64_t>(part, (int64_t)split_bound(nt, stream, cfg->precision) * nt * 3);
    }
    p.part_elems = part;

    Arena a(ws, ws_bytes);
    p.flags = a.carve<int>(16);
    p.zeta_nm1 = a.carve<double>(p.sz_zb);
    p.c_dot = a.carve<double>(p.sz_pan * 3);
    p.targets = a.carve<double>(p.max_targets * 3);
    p.v = a.carve<double>(p.max_targets * 3);
    p.part = a.carve<double>(std::max<int64_t>(part, 1));
    p.stream = a.carve<Elem64>(stream);
    if (cfg->precision == FJ_PREC_MIXED) {
        int64_t near = 0;
        for (int s = 0; s < ns; ++s)
            if (L.ms[s] > 0) near += img * stream_len(std::min(L.ms[s], kNearWakeRows), L.n[s]);
        p.stream_near = a.carve<Elem64>(std::max<int64_t>(near, 1));
    } else {
        p.stream_near = nullptr;
    }
    int64_t hs = 0, hsg = 0;
    for (int s = 0; s < ns; ++s) {
        hs += 2ll * (L.n[s] + 1) * 3;
        hsg += L.n[s];
    }
    p.hs_zw = a.carve<double>(hs);
    p.hs_gw = a.carve<double>(hsg);
    p.v_conv = a.carve<double>(std::max<int64_t>(L.wto[ns], 1) * 3);
    if (L.any_var) {
        p.zw_tmp = a.carve<double>(L.xvo[ns] * 3);
        p.gw_tmp = a.carve<double>(std::max<int64_t>(L.xpo[ns], 1));
        p.s_tmp = a.carve<double>(L.xvo[ns]);
    } else {
        p.zw_tmp = p.gw_tmp = p.s_tmp = nullptr;
    }
    p.a64 = a.carve<double>((int64_t)p.nb * p.nb);
    if (cfg->precision == FJ_PREC_MIXED) {
        p.a32 = a.carve<float>((int64_t)p.nb * p.nb);
        p.x32 = a.carve<float>((int64_t)p.nb * p.nb);
        p.tri32 = a.carve<float>(tc_tri_floats(p.nb));
    } else {
        p.a32 = nullptr;
        p.x32 = nullptr;
        p.tri32 = nullptr;
    }
    p.zeta_ref = a.carve<double>(p.sz_zb);
    p.piv = a.carve<int32_t>(p.nb);
    p.rhs = a.carve<double>(p.nb);
    p.r = a.carve<double>(p.nb);
    p.resid = a.carve<double>(cfg->n_tstep);
    p.ffil = a.carve<double>(L.fo[ns] * 3);
    p.polar_tmp = L.any_polar ? a.carve<double>(L.so[ns] * 7) : nullptr;
    p.tab_bytes = table_layout(1).total;
    p.tab = a.carve<char>(p.tab_bytes);
    p.tab_all = a.carve<char>((size_t)cfg->n_tstep * p.tab_bytes);
    p.step_ctr = a.carve<int>(4);
    if (ws != nullptr && !a.fits())
        return fail(FJ_ERR_NOMEM, "workspace of %zu bytes is smaller than the %zu required", ws_bytes, a.used);
    p.ws_needed = a.used;
    return FJ_OK;
}

// ------------------------------------------------------------------------------------
// Stream packing jobs and induced-velocity jobs
// ------------------------------------------------------------------------------------
struct StreamBuilder {
    PackArgs a;
    int n = 0;
    int64_t n_links = 0;
    void init(const Plan& p) {
        memset(&a, 0, sizeof(a));
        a.kernel = p.cfg.kernel;
        a.r_cut = p.cfg.r_cut;
        for (int d = 0; d < 3; ++d) {
            a.mirror.p[d] = p.cfg.mirror_point[d];
            a.mirror.nrm[d] = p.cfg.mirror_normal[d];
        }
        n = 0;
        n_links = 0;
        a.offset[0] = 0;
    }
    void add(const Plan& p, const double* zeta, const double* gamma, int rows, int cols) {
        const int img = p.cfg.mirror ? 2 : 1;
        for (int i = 0; i < img; ++i) {
            LatticeRef& L = a.lat[n];
            L.zeta = zeta;
            L.gamma = gamma;
            L.rows = rows;
            L.cols = cols;
            L.sign = i == 0 ? 1.0f : -1.0f;
            L.mirrored = i;
            a.offset[n + 1] = a.offset[n] + stream_len(rows, cols);
            n_links += lattice_links(rows, cols);
            ++n;
        }
        a.n_lat = n;
    }
    int64_t len() const { return a.offset[n]; }
};

static void* stream_at(const Plan& p, int64_t elem_offset) {
    const size_t es = p.cfg.precision == FJ_PREC_FP64 ? sizeof(Elem64) : sizeof(Elem32);
    return (char*)p.stream + elem_offset * es;
}

static int pack(const Plan& p, const StreamBuilder& sb, int64_t elem_offset, cudaStream_t s) {
    PackArgs a = sb.a;
    if (p.cfg.precision == FJ_PREC_FP64) return pack_stream64(a, (Elem64*)stream_at(p, elem_offset), s);
    return pack_stream32(a, (Elem32*)stream_at(p, elem_offset), s);
}

static int vind_sum(const Plan& p, const double* targets, int64_t nt, int64_t n_elem, int64_t n_links, double* out,
                    cudaStream_t s) {
    if (nt == 0) return FJ_OK;
    if (n_elem == 0) {
        FJ_CUDA(cudaMemsetAsync(out, 0, nt * 3 * sizeof(double), s));
        return FJ_OK;
    }
    VindJob j;
    memset(&j, 0, sizeof(j));
    j.targets = targets;
    j.n_targets = nt;
    j.stream = p.stream;
    j.n_elem = n_elem;
    j.n_split = choose_split(nt, n_elem, p.cfg.precision);
    j.part = p.part;
    j.n_links = n_links;
    j.out = out;
    if ((int64_t)j.n_split * nt * 3 > p.part_elems) return fail(FJ_ERR_NOMEM, "partial buffer too small");
    FJ_TRY(vind_launch(j, p.cfg.precision, p.cfg.kernel, p.cfg.r_cut, s));
    return reduce_partials(p.part, j.n_split, nt, out, 0, 1.0, s);
}

static void fill_aic_args(const Plan& p, AicArgs& a, const double* zeta, const double* c, const double* nc,
                          const double* zeta_w_static, int rows_static) {
    memset(&a, 0, sizeof(a));
    const Layout& L = p.L;
    a.n_surf = L.n_surf;
    int64_t wo = 0;
    a.max_fil = 0;
    for (int s = 0; s < L.n_surf; ++s) {
        a.zeta_b[s] = zeta + L.vo[s] * 3;
        a.m[s] = L.m[s];
        a.n[s] = L.n[s];
        a.col_off[s] = L.po[s];
        a.max_fil = std::max(a.max_fil, L.m[s] * (L.n[s] + 1) + (L.m[s] + 1) * L.n[s]);
        if (zeta_w_static != nullptr) {
            const int rows = rows_static >= 0 ? (L.ms[s] == 0 ? 0 : rows_static) : L.ms[s];
            a.zeta_w[s] = rows > 0 ? zeta_w_static + wo : nullptr;
            a.m_star[s] = rows;
            wo += (int64_t)(rows + 1) * (L.n[s] + 1) * 3;
        }
    }
    a.n_rows = L.po[L.n_surf];
    a.mirror = p.cfg.mirror;
    for (int d = 0; d < 3; ++d) {
        a.mp.p[d] = p.cfg.mirror_point[d];
        a.mp.nrm[d] = p.cfg.mirror_normal[d];
    }
    a.kernel = p.cfg.kernel;
    a.rc2 = p.cfg.r_cut * p.cfg.r_cut;
    a.c = c;
    a.nc = nc;
    a.aic = p.a64;
    a.ld = p.nb;
    a.run_flag = nullptr;
}

static int upload(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    return cuda_status(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s), "table upload");
}

// The solved circulations into the step's slot (the slot pointer comes from the table,
// so a graph-replayed step writes the slot of its replay).
__global__ void k_take_solution(const StepCase* __restrict__ C, const double* __restrict__ x, int nb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nb) C->gb_n[i] = x[i];
}

// The lattice the cached factors belong to (mixed path).
__global__ void k_keep_lattice(const StepCase* __restrict__ C, double* __restrict__ zeta_ref, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) zeta_ref[i] = C->zb_n[i];
}

// Graph-replayed steps: copy the table of slot *ctr into the fixed table area, and
// advance *ctr after the step.
// The slot counter is checked against the slot count the graph was captured with: out of
// range, nothing is copied and *bad (a status word) is set.
__global__ void k_select_table(const char* __restrict__ all, size_t stride, const int* __restrict__ ctr,
                               int n_slots, char* __restrict__ tab, int* __restrict__ bad) {
    const int c = *ctr;
    if (c < 0 || c >= n_slots) {
        if (threadIdx.x == 0 && blockIdx.x == 0) *bad = 1;
        return;
    }
    const int4* src = reinterpret_cast<const int4*>(all + (size_t)c * stride);
    int4* dst = reinterpret_cast<int4*>(tab);
    for (size_t w = (size_t)blockIdx.x * blockDim.x + threadIdx.x; w < stride / 16; w += (size_t)gridDim.x * blockDim.x)
        dst[w] = src[w];
}

__global__ void k_advance(int* ctr) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *ctr += 1;
}

// ------------------------------------------------------------------------------------
// Static solve (uvlm.py:1286-1333 through base_solve_from_grid with static=True)
// ------------------------------------------------------------------------------------
static int run_static(const Plan& p, const fj_case_buffers* B, const double* hg, int horseshoe, double t0,
                      cudaStream_t s) {
    const Layout& L = p.L;
    const fj_case_config& c = p.cfg;
    double* zb = B->d_zeta_b;
    double* zw = B->d_zeta_w;
    double* gb = B->d_gamma_b;
    double* gw = B->d_gamma_w;
    FJ_CUDA(cudaMemcpyAsync(B->d_t, &t0, sizeof(double), cudaMemcpyHostToDevice, s));
    // wake of the solve: initialise_wake or the horseshoe (rows 1, far end at HORSESHOE_LENGTH)
    const double* zw_solve = zw;
    const double* gw_solve = gw;
    int rows_solve = -1;
    if (horseshoe) {
        zw_solve = p.hs_zw;
        gw_solve = p.hs_gw;
        rows_solve = 1;
    }
    StepCase C;
    memset(&C, 0, sizeof(C));
    C.L = L;
    C.nb = p.nb;
    C.i = 0;
    C.dt = c.dt;
    C.relax = c.gamma_dot_relaxation;
    C.flow = c.flow;
    C.zeta0 = B->d_zeta_b0;
    C.dof = B->d_dof_mapping;
    C.hg_n = hg;
    C.t = B->d_t;
    C.zb_n = zb;
    C.zbd_n = B->d_zeta_b_dot;
    C.zw_n = zw;
    C.c = B->d_c;
    C.nc = B->d_nc;
    C.gb_n = gb;
    C.gbd_n = B->d_gamma_b_dot;
    C.gw_n = gw;
    C.gw_force = gw_solve;
    C.fs = B->d_f_steady;
    C.fu = B->d_f_unsteady;
    C.alpha = B->d_alpha;
    C.ft = B->d_force_total;
    C.zb_nm1 = p.zeta_nm1;
    C.targets = p.targets;
    C.v = p.v;
    C.ffil = p.ffil;
    C.rhs = p.rhs;
    C.nonfinite = p.flags + 2;
    C.polars = L.any_polar ? B->d_polars : nullptr;
    C.polar_tmp = p.polar_tmp;
    C.polar_scale = c.polar_circulation_scale;
    const TableLayout tl = table_layout(1);
    StepCase* dC = (StepCase*)(p.tab + tl.step);
    FJ_TRY(upload(dC, &C, sizeof(C), s));
    k_geom_vertices<<<nblk(L.vo[L.n_surf]), 256, 0, s>>>(dC); note_launch();
    k_geom_panels<<<nblk(L.po[L.n_surf]), 256, 0, s>>>(dC); note_launch();
    if (horseshoe) {
        int64_t rows_tot = 0;
        for (int q = 0; q < L.n_surf; ++q) rows_tot += (int64_t)((L.ms[q] == 0 ? 0 : 1) + 1) * (L.n[q] + 1);
        init_wake_kernel<<<nblk(rows_tot), 256, 0, s>>>(L, zb, c.flow, c.dt, 1e3, p.hs_zw, 1, nullptr); note_launch();
    }
    if (L.any_var && B->d_delta_w == nullptr) return fail(FJ_ERR_SHAPE, "variable_wake set but d_delta_w is NULL");
    init_wake_kernel<<<nblk(L.wvo[L.n_surf]), 256, 0, s>>>(L, zb, c.flow, c.dt, 0.0, zw, 0, B->d_delta_w); note_launch();
    FJ_LAUNCH_CHECK("static geometry");
    AicArgs aa;
    fill_aic_args(p, aa, zb, B->d_c, B->d_nc, zw_solve, rows_solve);
    FJ_TRY(aic_launch(aa, nullptr, s));
    k_rhs<<<nblk(p.nb), 256, 0, s>>>(dC); note_launch();
    FJ_TRY(lu_factor64(p.a64, p.nb, p.piv, p.flags, s));
    FJ_TRY(lu_solve64(p.a64, p.nb, p.piv, p.rhs, p.r, s));
    FJ_CUDA(cudaMemcpyAsync(gb, p.rhs, p.nb * sizeof(double), cudaMemcpyDeviceToDevice, s));
    // the static AIC (with the wake lumped in) now occupies the AIC buffer: a NaN in the
    // cached lattice makes the next dynamic step that compares lattices rebuild it
    FJ_CUDA(cudaMemsetAsync(p.zeta_ref, 0xFF, sizeof(double), s));
    // wake circulation of the solve (horseshoe: one row) and of the stored slot
    if (horseshoe) {
        static_gamma_w_kernel<<<nblk(p.sz_strip), 256, 0, s>>>(L, gb, p.hs_gw, 1); note_launch();
    }
    static_gamma_w_kernel<<<nblk(p.sz_gw + 1), 256, 0, s>>>(L, gb, gw, -1); note_launch();
    // forces: v at midpoints from the solve wake + bound, zeta_dot = 0
    StreamBuilder sb;
    sb.init(p);
    int64_t wo = 0, go = 0;
    for (int q = 0; q < L.n_surf; ++q) {
        const int rows = horseshoe ? (L.ms[q] == 0 ? 0 : 1) : L.ms[q];
        sb.add(p, zw_solve + wo, gw_solve + go, rows, L.n[q]);
        wo += (int64_t)(rows + 1) * (L.n[q] + 1) * 3;
        go += (int64_t)rows * L.n[q];
    }
    for (int q = 0; q < L.n_surf; ++q) sb.add(p, zb + L.vo[q] * 3, gb + L.po[q], L.m[q], L.n[q]);
    FJ_TRY(pack(p, sb, 0, s));
    k_force_targets<<<nblk(L.fo[L.n_surf]), 256, 0, s>>>(dC); note_launch();
    FJ_TRY(vind_sum(p, p.targets, L.fo[L.n_surf], sb.len(), sb.n_links, p.v, s));
    k_force_filament<<<nblk(L.fo[L.n_surf]), 256, 0, s>>>(dC); note_launch();
    k_vertex_forces<<<nblk(L.vo[L.n_surf]), 256, 0, s>>>(dC, 3); note_launch();
    k_strip_alpha<<<nblk(p.sz_strip), 256, 0, s>>>(dC); note_launch();
    if (L.any_polar) {  // uvlm.py:1055-1075: forces, then the circulations and the static wake
        k_polar_strips<<<nblk(p.sz_strip), 256, 0, s>>>(dC); note_launch();
        k_polar_vertices<<<nblk(L.vo[L.n_surf]), 256, 0, s>>>(dC); note_launch();
        if (c.polar_circulation_scale != 0.0) {
            k_polar_gamma<<<nblk(p.sz_pan), 256, 0, s>>>(dC); note_launch();
            static_gamma_w_kernel<<<nblk(p.sz_gw + 1), 256, 0, s>>>(L, gb, gw, -1); note_launch();
        }
    }
    FJ_CUDA(cudaMemsetAsync(B->d_gamma_b_dot, 0, p.sz_pan * sizeof(double), s));
    k_force_total<<<1, 256, 0, s>>>(dC); note_launch();
    FJ_LAUNCH_CHECK("static solve");
    return FJ_OK;
}

// ------------------------------------------------------------------------------------
// Dynamic steps of a batch of cases (case_solve, uvlm.py:1119-1215)
// ------------------------------------------------------------------------------------
struct BatchItem {
    Plan p;
    const fj_case_buffers* B;
    int i;
    bool refactor;
    const double* hg_n;
    const double* hgd_n;
    const double* hg_nm1;
    bool reuse_convection = false;  // free wake: the previous call's convection velocities hold
};

// Target CTAs for a batched sum; each job gets a share proportional to its pairs.
static void assign_splits(std::vector<VindJob>& jobs, int precision) {
    if (jobs.size() == 1) {
        jobs[0].n_split = choose_split(jobs[0].n_targets, jobs[0].n_elem, precision);
        return;
    }
    double total = 0.0;
    for (const VindJob& j : jobs) total += (double)j.n_targets * (double)j.n_links;
    const double target_ctas = 4.0 * 148 * 6;
    for (VindJob& j : jobs) {
        const int64_t cx = vind_ctas(j.n_targets, 1, precision);
        const double share = total > 0 ? target_ctas * ((double)j.n_targets * (double)j.n_links) / total : 1.0;
        int64_t sp = (int64_t)(share / std::max<int64_t>(cx, 1) + 0.5);
        sp = std::max<int64_t>(1, std::min<int64_t>(sp, split_bound(j.n_targets, j.n_elem, precision)));
        j.n_split = (int)sp;
    }
}

static int launch_sum(const std::vector<VindJob>& jobs, const std::vector<int64_t>& cta0, char* d_jobs, char* d_cta0,
                      int precision, int kernel, double r_cut, cudaStream_t s, bool persistent, int tile) {
    if (jobs.empty()) return FJ_OK;
    double pairs = 0.0;
    int64_t max_t = 0;
    for (const VindJob& j : jobs) {
        pairs += (double)j.n_targets * (double)j.n_links;
        max_t = std::max(max_t, j.n_targets);
    }
    FJ_TRY(vind_launch_jobs((const VindJob*)d_jobs, (const int64_t*)d_cta0, (int)jobs.size(), cta0.back(), pairs,
                            precision, kernel, r_cut, s, persistent, tile));
    return reduce_jobs((const VindJob*)d_jobs, (int)jobs.size(), max_t, s);
}

// run_steps modes: build the table and launch (normal); only build the table into a
// host buffer (build); launch with the table already in place on the device (launch:
// the graph-replayed steps, whose table a select kernel copies in first).
enum { kStepNormal = 0, kStepBuild = 1, kStepLaunch = 2 };

static int run_steps(std::vector<BatchItem>& items, char* d_tab, size_t tab_bytes, cudaStream_t s,
                     int mode = kStepNormal, char* h_out = nullptr, std::vector<int64_t>* sig = nullptr,
                     bool persistent_sums = false) {
    const int K = (int)items.size();
    if (K == 0) return FJ_OK;
    const int precision = items[0].p.cfg.precision;
    const int kernel = items[0].p.cfg.kernel;
    const double r_cut = items[0].p.cfg.r_cut;
    for (const BatchItem& it : items)
        if (it.p.cfg.precision != precision || it.p.cfg.kernel != kernel || it.p.cfg.r_cut != r_cut)
            return fail(FJ_ERR_UNSUPPORTED, "a batch must share precision, kernel and cutoff radius");
    const TableLayout tl = table_layout(K);
    if (tl.total > tab_bytes) return fail(FJ_ERR_NOMEM, "batch table needs %zu bytes, %zu given", tl.total, tab_bytes);

    std::vector<char> h(tl.total, 0);
    StepCase* hC = (StepCase*)(h.data() + tl.step);
    std::vector<VindJob> jf, jr, jfo, jrn;
    std::vector<PackJob> pf(K), pw(K), pb(K), pwn(K);
    std::vector<int64_t> rhs_far(K, 0), near_cap;
    std::vector<AicArgs> aic(K);
    std::vector<RefineJob> ref;
    std::vector<int> free_idx;
    int64_t max_v = 0, max_p = 0, max_w = 0, max_wt = 0, max_f = 0, max_e_free = 0, max_e_wake = 0, max_e_bound = 0,
            max_e_near = 0;
    int max_n = 0, max_fil = 0, any_mirror = 0, any_free = 0, any_changed = 0, any_var = 0, any_polar = 0;
    int64_t max_xw = 0, max_cols = 0;
    for (int k = 0; k < K; ++k) {
        BatchItem& it = items[k];
        const Plan& p = it.p;
        const Layout& L = p.L;
        const fj_case_config& c = p.cfg;
        const fj_case_buffers* B = it.B;
        const int i = it.i;
        const bool mixed = c.precision == FJ_PREC_MIXED;
        StepCase& C = hC[k];
        C.L = L;
        C.nb = p.nb;
        C.i = i;
        // convection velocities: computed into p.v_conv (kept for the next call), or
        // reused from there when the caller says the step's n-1 state is the same
        const bool fw = c.free_wake && L.wto[L.n_surf] > 0;
        C.free_wake = fw && !it.reuse_convection;
        C.dt = c.dt;
        C.relax = c.gamma_dot_relaxation;
        C.flow = c.flow;
        C.zeta0 = B->d_zeta_b0;
        C.dof = B->d_dof_mapping;
        C.hg_n = it.hg_n;
        C.hgd_n = it.hgd_n;
        C.hg_nm1 = it.hg_nm1;
        C.t = B->d_t;
        C.advance_time = 1;
        C.zb_n = B->d_zeta_b + (int64_t)i * p.sz_zb;
        C.zbd_n = B->d_zeta_b_dot + (int64_t)i * p.sz_zb;
        C.zw_n = B->d_zeta_w + (int64_t)i * p.sz_zw;
        C.zw_nm1 = B->d_zeta_w + (int64_t)(i - 1) * p.sz_zw;
        C.c = B->d_c + (int64_t)i * p.sz_pan * 3;
        C.nc = B->d_nc + (int64_t)i * p.sz_pan * 3;
        C.gb_n = B->d_gamma_b + (int64_t)i * p.sz_pan;
        C.gb_nm1 = B->d_gamma_b + (int64_t)(i - 1) * p.sz_pan;
        C.gbd_n = B->d_gamma_b_dot + (int64_t)i * p.sz_pan;
        C.gbd_nm1 = B->d_gamma_b_dot + (int64_t)(i - 1) * p.sz_pan;
        C.gw_n = B->d_gamma_w + (int64_t)i * p.sz_gw;
        C.gw_nm1 = B->d_gamma_w + (int64_t)(i - 1) * p.sz_gw;
        C.gw_force = C.gw_n;
        C.fs = B->d_f_steady + (int64_t)i * p.sz_zb;
        C.fu = B->d_f_unsteady + (int64_t)i * p.sz_zb;
        C.alpha = B->d_alpha + (int64_t)i * p.sz_strip;
        C.ft = B->d_force_total + (int64_t)i * 3;
        C.zb_nm1 = p.zeta_nm1;
        C.c_dot = p.c_dot;
        C.targets = p.targets;
        C.v = p.v;
        C.ffil = p.ffil;
        C.rhs = p.rhs;
        C.nonfinite = p.flags + 2;
        C.v_wake = fw ? p.v_conv : nullptr;
        C.v_rhs = p.v;
        if (L.any_var && B->d_delta_w == nullptr)
            return fail(FJ_ERR_SHAPE, "variable_wake set but d_delta_w is NULL");
        C.delta_w = B->d_delta_w;
        C.zw_tmp = p.zw_tmp;
        C.gw_tmp = p.gw_tmp;
        C.s_tmp = p.s_tmp;
        any_var |= L.any_var;
        max_xw = std::max(max_xw, L.xvo[L.n_surf] + L.xpo[L.n_surf]);
        max_cols = std::max(max_cols, L.dofo[L.n_surf]);
        // a step that does not refactorise compares its lattice with the one of the cached
        // AIC (mixed) or FP64 factors and rebuilds them only where it changed
        C.zeta_ref = !it.refactor ? p.zeta_ref : nullptr;
        C.changed = !it.refactor ? p.flags + 1 : nullptr;
        C.polars = L.any_polar ? B->d_polars : nullptr;
        C.polar_tmp = p.polar_tmp;
        C.polar_scale = c.polar_circulation_scale;
        any_polar |= L.any_polar;
        any_changed |= C.changed != nullptr;
        max_v = std::max(max_v, L.vo[L.n_surf]);
        max_p = std::max(max_p, L.po[L.n_surf]);
        max_w = std::max(max_w, L.wvo[L.n_surf] + L.wpo[L.n_surf]);
        max_wt = std::max(max_wt, L.wto[L.n_surf]);
        max_f = std::max(max_f, L.fo[L.n_surf]);
        max_n = std::max(max_n, p.nb);
        any_mirror |= c.mirror;

        // free-wake sum: bound(n-1) + wake(n-1) at the wake vertices of n-1
        if (C.free_wake) {
            any_free = 1;
            StreamBuilder sb;
            sb.init(p);
            for (int q = 0; q < L.n_surf; ++q)
                sb.add(p, p.zeta_nm1 + L.vo[q] * 3, C.gb_nm1 + L.po[q], L.m[q], L.n[q]);
            for (int q = 0; q < L.n_surf; ++q)
                sb.add(p, C.zw_nm1 + L.wvo[q] * 3, C.gw_nm1 + L.wpo[q], L.ms[q], L.n[q]);
            pf[k].a = sb.a;
            pf[k].out = stream_at(p, 0);
            max_e_free = std::max(max_e_free, sb.len());
            VindJob j;
            memset(&j, 0, sizeof(j));
            j.targets = p.targets;
            j.n_targets = L.wto[L.n_surf];
            j.stream = p.stream;
            j.n_elem = sb.len();
            j.part = p.part;
            j.n_links = sb.n_links;
            j.out = p.v_conv;
            jf.push_back(j);
        } else {
            memset(&pf[k], 0, sizeof(PackJob));  // empty job: offset[0] = 0 packs nothing
        }
        // wake(n) stream, then bound(n) appended.  Mixed: each wake goes in as two lattices,
        // rows [kNearWakeRows, m_star) first and rows [0, kNearWakeRows) after them (the two
        // together carry the same filaments as the whole wake), so that the RHS sums the
        // stream's leading far part in FP32 and takes the near rows, in FP64, from their own
        // stream; the force sum reads the whole wake part.
        StreamBuilder sw, swn;
        sw.init(p);
        swn.init(p);
        if (!mixed) {
            for (int q = 0; q < L.n_surf; ++q) sw.add(p, C.zw_n + L.wvo[q] * 3, C.gw_n + L.wpo[q], L.ms[q], L.n[q]);
        } else {
            for (int q = 0; q < L.n_surf; ++q) {
                const int kn = std::min(L.ms[q], kNearWakeRows);
                if (L.ms[q] > kn)
                    sw.add(p, C.zw_n + (L.wvo[q] + (int64_t)kn * (L.n[q] + 1)) * 3, C.gw_n + L.wpo[q] + (int64_t)kn * L.n[q],
                           L.ms[q] - kn, L.n[q]);
            }
        }
        rhs_far[k] = sw.len();
        const int64_t far_links = sw.n_links;
        if (mixed) {
            for (int q = 0; q < L.n_surf; ++q) {
                const int kn = std::min(L.ms[q], kNearWakeRows);
                if (kn == 0) continue;
                sw.add(p, C.zw_n + L.wvo[q] * 3, C.gw_n + L.wpo[q], kn, L.n[q]);
                swn.add(p, C.zw_n + L.wvo[q] * 3, C.gw_n + L.wpo[q], kn, L.n[q]);
            }
        }
        pwn[k].a = swn.a;
        pwn[k].out = p.stream_near;
        max_e_near = std::max(max_e_near, swn.len());
        pw[k].a = sw.a;
        pw[k].out = stream_at(p, 0);
        max_e_wake = std::max(max_e_wake, sw.len());
        StreamBuilder sbd;
        sbd.init(p);
        for (int q = 0; q < L.n_surf; ++q) sbd.add(p, C.zb_n + L.vo[q] * 3, C.gb_n + L.po[q], L.m[q], L.n[q]);
        pb[k].a = sbd.a;
        pb[k].out = stream_at(p, sw.len());
        max_e_bound = std::max(max_e_bound, sbd.len());
        if (p.nb > 0) {
            VindJob j;
            memset(&j, 0, sizeof(j));
            j.targets = C.c;
            j.n_targets = p.nb;
            j.stream = p.stream;
            j.n_elem = rhs_far[k];
            j.part = p.part;
            j.n_links = far_links;
            j.out = p.v;
            if (j.n_elem > 0) jr.push_back(j);
        }
        if (p.nb > 0 && swn.len() > 0) {  // the near rows in FP64, added to the far sum
            VindJob j;
            memset(&j, 0, sizeof(j));
            j.targets = C.c;
            j.n_targets = p.nb;
            j.stream = p.stream_near;
            j.n_elem = swn.len();
            j.part = p.part;
            j.n_links = swn.n_links;
            j.out = p.v;
            j.accumulate = 1;
            jrn.push_back(j);
            near_cap.push_back(p.part_elems / ((int64_t)p.nb * 3));
        }
        {
            VindJob j;
            memset(&j, 0, sizeof(j));
            j.targets = p.targets;
            j.n_targets = L.fo[L.n_surf];
            j.stream = p.stream;
            j.n_elem = sw.len() + sbd.len();
            j.part = p.part;
            j.n_links = sw.n_links + sbd.n_links;
            j.out = p.v;
            jfo.push_back(j);
        }
        // AIC of the bound lattice (dynamic: no wake lumping)
        fill_aic_args(p, aic[k], C.zb_n, C.c, C.nc, nullptr, -1);
        aic[k].run_flag = C.changed;
        max_fil = std::max(max_fil, aic[k].max_fil);
        if (mixed) {
            RefineJob rj;
            rj.a = p.a64;
            rj.xinv = p.x32;
            rj.n = p.nb;
            rj.b = p.rhs;
            rj.x = C.gb_n;
            rj.r = p.r;
            rj.resid = p.resid + i;
            ref.push_back(rj);
        }
    }
    // RHS jobs of cases whose wake stream is empty: zero velocity
    assign_splits(jf, precision);
    assign_splits(jr, precision);
    assign_splits(jfo, precision);
    // The near-row sums are short (a few rows of links): 32 elements per split so that they
    // spread over the GPU instead of running as a handful of long FP64 CTAs; each reuses
    // its case's partial buffer.
    for (size_t q = 0; q < jrn.size(); ++q)
        jrn[q].n_split = (int)std::max<int64_t>(1, std::min<int64_t>({(jrn[q].n_elem + 31) / 32, 1024, near_cap[q]}));
    // every job's partials must fit its case's partial buffer (the kernels take any split)
    std::unordered_map<const double*, int64_t> part_elems;
    for (const BatchItem& it : items) part_elems[it.p.part] = it.p.part_elems;
    for (std::vector<VindJob>* jobs : {&jf, &jr, &jfo, &jrn})
        for (VindJob& j : *jobs) {
            const int64_t cap = part_elems[j.part] / std::max<int64_t>(1, j.n_targets * 3);
            if (cap < 1) return fail(FJ_ERR_NOMEM, "partial buffer too small for %lld targets", (long long)j.n_targets);
            j.n_split = (int)std::min<int64_t>(j.n_split, cap);
        }
    // one tile (targets per thread) per FP32 launch: the autotuned choice of its largest job
    auto phase_tile = [&](const std::vector<VindJob>& jobs) {
        double most = -1.0;
        int tile = 0;
        for (const VindJob& j : jobs) {
            const double w = (double)j.n_targets * (double)j.n_links;
            if (w > most) {
                most = w;
                tile = choose_tile(j.n_targets, j.n_elem, precision);
            }
        }
        return tile;
    };
    const int tf = phase_tile(jf), tr = phase_tile(jr), tfo = phase_tile(jfo);
    auto fill_cta = [&](const std::vector<VindJob>& jobs, size_t off, int prec, int tile) {
        int64_t* c0 = (int64_t*)(h.data() + off);
        c0[0] = 0;
        for (size_t q = 0; q < jobs.size(); ++q)
            c0[q + 1] = c0[q] + vind_ctas(jobs[q].n_targets, jobs[q].n_split, prec, tile);
        return std::vector<int64_t>(c0, c0 + jobs.size() + 1);
    };
    const std::vector<int64_t> cf = fill_cta(jf, tl.cta_free, precision, tf),
                               cr = fill_cta(jr, tl.cta_rhs, precision, tr),
                               cfo = fill_cta(jfo, tl.cta_force, precision, tfo),
                               crn = fill_cta(jrn, tl.cta_near, FJ_PREC_FP64, 0);
    memcpy(h.data() + tl.pack_free, pf.data(), K * sizeof(PackJob));
    memcpy(h.data() + tl.pack_wake, pw.data(), K * sizeof(PackJob));
    memcpy(h.data() + tl.pack_bound, pb.data(), K * sizeof(PackJob));
    memcpy(h.data() + tl.pack_near, pwn.data(), K * sizeof(PackJob));
    if (!jf.empty()) memcpy(h.data() + tl.job_free, jf.data(), jf.size() * sizeof(VindJob));
    if (!jr.empty()) memcpy(h.data() + tl.job_rhs, jr.data(), jr.size() * sizeof(VindJob));
    memcpy(h.data() + tl.job_force, jfo.data(), jfo.size() * sizeof(VindJob));
    if (!jrn.empty()) memcpy(h.data() + tl.job_near, jrn.data(), jrn.size() * sizeof(VindJob));
    memcpy(h.data() + tl.aic, aic.data(), K * sizeof(AicArgs));
    if (!ref.empty()) memcpy(h.data() + tl.refine, ref.data(), ref.size() * sizeof(RefineJob));
    if (sig != nullptr) {
        // Every host value the launches below take outside the table: grid extents, job
        // counts, and the per-case pointers of the launches that are not table-driven (the
        // FP64 and refactorising solves, the zeroing of cases without far-wake rows).  Two
        // builds with equal signatures launch the same kernels with the same arguments, so
        // a graph captured for one replays the other once its table is in place.
        std::vector<int64_t>& g = *sig;
        double rc = r_cut;
        int64_t rc_bits = 0;
        memcpy(&rc_bits, &rc, sizeof(rc_bits));
        auto sum_sig = [&](const std::vector<VindJob>& jobs) {
            int64_t mt = 0;
            for (const VindJob& j : jobs) mt = std::max(mt, j.n_targets);
            g.push_back((int64_t)jobs.size());
            g.push_back(mt);
        };
        g = {precision, kernel, rc_bits, K, max_v, max_p, max_w, max_wt, max_f, max_n, max_fil, any_mirror, any_free,
             any_changed, any_var, any_polar, max_xw, max_cols, max_e_free, max_e_wake, max_e_bound, max_e_near,
             (int64_t)ref.size(), tf, tr, tfo};
        sum_sig(jf);
        sum_sig(jr);
        sum_sig(jrn);
        sum_sig(jfo);
        for (int k = 0; k < K; ++k) {
            const Plan& p = items[k].p;
            g.push_back(p.sz_strip);
            if (rhs_far[k] == 0) g.push_back((int64_t)(uintptr_t)p.v);
            if (precision == FJ_PREC_FP64 || items[k].refactor) {
                g.push_back(items[k].refactor);
                for (const void* ptr : {(const void*)p.a64, (const void*)p.piv, (const void*)p.flags,
                                        (const void*)p.rhs, (const void*)p.r, (const void*)p.a32, (const void*)p.x32,
                                        (const void*)p.tri32, (const void*)p.zeta_ref})
                    g.push_back((int64_t)(uintptr_t)ptr);
                g.push_back((int64_t)(uintptr_t)hC[k].changed);
                g.push_back(p.nb);
                g.push_back(p.sz_zb);
            }
        }
    }
    if (mode == kStepBuild) {
        memcpy(h_out, h.data(), tl.total);
        return FJ_OK;
    }
    if (mode == kStepNormal) FJ_TRY(upload(d_tab, h.data(), tl.total, s));
    const StepCase* dC = (const StepCase*)(d_tab + tl.step);
    const dim3 b(256);

    // 1. time, geometry
    k_time<<<dim3(1, K), 32, 0, s>>>(dC); note_launch();
    k_geom_vertices<<<dim3(nblk(max_v), K), b, 0, s>>>(dC); note_launch();
    k_geom_panels<<<dim3(nblk(max_p), K), b, 0, s>>>(dC); note_launch();
    // 2. free wake, shed + convect
    if (any_free) {
        FJ_TRY(pack_jobs((const PackJob*)(d_tab + tl.pack_free), K, max_e_free, precision, s));
        k_gather_wake_targets<<<dim3(nblk(max_wt), K), b, 0, s>>>(dC); note_launch();
        FJ_TRY(launch_sum(jf, cf, d_tab + tl.job_free, d_tab + tl.cta_free, precision, kernel, r_cut, s, persistent_sums,
                          tf));
    }
    k_wake_shed<<<dim3(nblk(max_w), K), b, 0, s>>>(dC); note_launch();
    if (any_var) {  // delta_w surfaces: convect all rows, then re-discretise (aero/utils.py:452-491)
        k_wake_shed_var<<<dim3(nblk(max_xw), K), b, 0, s>>>(dC); note_launch();
        k_wake_redisc_z<<<dim3(nblk(max_cols), K), b, 0, s>>>(dC); note_launch();
        k_wake_redisc_g<<<dim3(nblk(max_cols), K), b, 0, s>>>(dC); note_launch();
    }
    // 3. AIC (mixed: only where the lattice changed since the factorisation)
    if (any_changed) {
        k_changed<<<dim3(nblk(max_v * 3), K), b, 0, s>>>(dC); note_launch();
    }
    FJ_TRY(aic_launch_jobs((const AicArgs*)(d_tab + tl.aic), K, max_n, max_fil, any_mirror, kernel, s));
    // 4. RHS
    FJ_TRY(pack_jobs((const PackJob*)(d_tab + tl.pack_wake), K, max_e_wake, precision, s));
    if (!jrn.empty()) FJ_TRY(pack_jobs((const PackJob*)(d_tab + tl.pack_near), K, max_e_near, FJ_PREC_FP64, s));
    for (int k = 0; k < K; ++k)  // cases without (far) wake filaments: zero, then the near rows add
        if (rhs_far[k] == 0 && items[k].p.nb > 0)
            FJ_CUDA(cudaMemsetAsync(items[k].p.v, 0, items[k].p.nb * 3 * sizeof(double), s));
    FJ_TRY(launch_sum(jr, cr, d_tab + tl.job_rhs, d_tab + tl.cta_rhs, precision, kernel, r_cut, s, persistent_sums, tr));
    FJ_TRY(launch_sum(jrn, crn, d_tab + tl.job_near, d_tab + tl.cta_near, FJ_PREC_FP64, kernel, r_cut, s, persistent_sums,
                      0));
    k_rhs<<<dim3(nblk(max_n), K), b, 0, s>>>(dC); note_launch();
    FJ_LAUNCH_CHECK("step: geometry, wake, RHS");
    // 5. solve
    if (precision == FJ_PREC_FP64) {
        for (int k = 0; k < K; ++k) {
            const Plan& p = items[k].p;
            // factor only when the lattice changed since the cached factors (the factor
            // kernels read the flag and return at once when it is clear)
            FJ_TRY(lu_factor64(p.a64, p.nb, p.piv, p.flags, s, hC[k].changed));
            FJ_TRY(lu_solve64(p.a64, p.nb, p.piv, p.rhs, p.r, s));
            k_take_solution<<<nblk(p.nb), 256, 0, s>>>(dC + k, p.rhs, p.nb); note_launch();
            k_keep_lattice<<<nblk(p.sz_zb), 256, 0, s>>>(dC + k, p.zeta_ref, p.sz_zb); note_launch();
        }
    } else {
        for (int k = 0; k < K; ++k) {
            if (!items[k].refactor) continue;
            const Plan& p = items[k].p;
            FJ_TRY(factor_inverse32(p.a64, p.nb, p.a32, p.piv, p.flags, p.x32, p.tri32, s));
            k_keep_lattice<<<nblk(p.sz_zb), 256, 0, s>>>(dC + k, p.zeta_ref, p.sz_zb); note_launch();
        }
        FJ_TRY(refine_jobs((const RefineJob*)(d_tab + tl.refine), (int)ref.size(), max_n, 3, s));
    }
    // 6. forces with bound(n) + wake(n)
    FJ_TRY(pack_jobs((const PackJob*)(d_tab + tl.pack_bound), K, max_e_bound, precision, s));
    k_force_targets<<<dim3(nblk(max_f), K), b, 0, s>>>(dC); note_launch();
    FJ_TRY(launch_sum(jfo, cfo, d_tab + tl.job_force, d_tab + tl.cta_force, precision, kernel, r_cut, s, persistent_sums,
                      tfo));
    k_force_filament<<<dim3(nblk(max_f), K), b, 0, s>>>(dC); note_launch();
    // 7. gamma_dot, vertex forces, strip alpha, totals
    if (!any_polar) {
        k_gamma_dot<<<dim3(nblk(max_n), K), b, 0, s>>>(dC); note_launch();
        k_vertex_forces<<<dim3(nblk(max_v), K), b, 0, s>>>(dC, 3); note_launch();
    } else {
        // uvlm.py:1055-1103: steady forces and strip alpha from the solved Gamma, the polar
        // forces and circulation blend, then gamma_dot and the unsteady forces from the
        // blended Gamma (the same kernels; a case without polars skips the polar ones)
        int64_t max_s = 0;
        for (const BatchItem& it : items) max_s = std::max(max_s, it.p.sz_strip);
        k_vertex_forces<<<dim3(nblk(max_v), K), b, 0, s>>>(dC, 1); note_launch();
        k_strip_alpha<<<dim3(nblk(max_s), K), b, 0, s>>>(dC); note_launch();
        k_polar_strips<<<dim3(nblk(max_s), K), b, 0, s>>>(dC); note_launch();
        k_polar_vertices<<<dim3(nblk(max_v), K), b, 0, s>>>(dC); note_launch();
        k_polar_gamma<<<dim3(nblk(max_n), K), b, 0, s>>>(dC); note_launch();
        k_gamma_dot<<<dim3(nblk(max_n), K), b, 0, s>>>(dC); note_launch();
        k_vertex_forces<<<dim3(nblk(max_v), K), b, 0, s>>>(dC, 2); note_launch();
    }
    if (!any_polar) {
        int64_t max_strip = 0;
        for (const BatchItem& it : items) max_strip = std::max(max_strip, it.p.sz_strip);
        k_strip_alpha<<<dim3(nblk(max_strip), K), b, 0, s>>>(dC); note_launch();
    }
    k_force_total<<<dim3(1, K), b, 0, s>>>(dC); note_launch();
    FJ_LAUNCH_CHECK("step: forces");
    return FJ_OK;
}

// Collocation points and area normals of one lattice (compute_surf_c / compute_surf_nc).
__global__ void surface_c_nc_kernel(int m, int n, const double* __restrict__ zeta, double* __restrict__ c,
                                    double* __restrict__ nc) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (int64_t)m * n) return;
    const int k = (int)(p / n), l = (int)(p % n);
    const double* z00 = zeta + ((int64_t)k * (n + 1) + l) * 3;
    const double* z01 = z00 + 3;
    const double* z10 = z00 + (n + 1) * 3;
    const double* z11 = z10 + 3;
    for (int d = 0; d < 3; ++d) c[p * 3 + d] = 0.5 * (0.5 * (z00[d] + z10[d]) + 0.5 * (z01[d] + z11[d]));
    const double d1[3] = {z11[0] - z00[0], z11[1] - z00[1], z11[2] - z00[2]};
    const double d2[3] = {z10[0] - z01[0], z10[1] - z01[1], z10[2] - z01[2]};
    nc[p * 3 + 0] = d1[1] * d2[2] - d1[2] * d2[1];
    nc[p * 3 + 1] = d1[2] * d2[0] - d1[0] * d2[2];
    nc[p * 3 + 2] = d1[0] * d2[1] - d1[1] * d2[0];
}

static int check_buffers(const Plan& p, const fj_case_buffers* B, bool dynamic) {
    if (B == nullptr) return fail(FJ_ERR_SHAPE, "buffers struct is NULL");
    if (!B->d_zeta_b0 || !B->d_dof_mapping || !B->d_t || !B->d_zeta_b || !B->d_zeta_b_dot || !B->d_zeta_w ||
        !B->d_c || !B->d_nc || !B->d_gamma_b || !B->d_gamma_b_dot || !B->d_f_steady ||
        !B->d_f_unsteady || !B->d_alpha || !B->d_force_total)
        return fail(FJ_ERR_SHAPE, "a required device buffer is NULL");
    // gamma_w has no entries when no surface has a wake (m_star = 0 everywhere)
    if (!B->d_gamma_w && p.sz_gw > 0) return fail(FJ_ERR_SHAPE, "d_gamma_w is NULL");
    if (dynamic && (!B->d_hg_t || !B->d_hg_dot_t)) return fail(FJ_ERR_SHAPE, "hg_t / hg_dot_t are NULL");
    if (p.L.any_polar && !B->d_polars) return fail(FJ_ERR_SHAPE, "polar_points set but d_polars is NULL");
    return FJ_OK;
}

// Status words of a case-level call: flags[0] the LU info of the last factorisation
// (first zero pivot + 1), flags[2] the lowest slot with a non-finite total force,
// flags[3] set when a bounded wait of the tensor-core factorisation expired, flags[4] set
// when a replayed step graph found its slot counter out of range.
static constexpr int kNoSlot = 0x7f7f7f7f;  // the byte pattern 0x7f repeated

static int clear_status(const Plan& p, cudaStream_t s) {
    FJ_CUDA(cudaMemsetAsync(p.flags + 3, 0, 2 * sizeof(int), s));
    return cuda_status(cudaMemsetAsync(p.flags + 2, 0x7f, sizeof(int), s), "status reset");
}

static int read_status(const Plan& p, cudaStream_t s) {
    int w[5] = {0, 0, 0, 0, 0};
    FJ_CUDA(cudaMemcpyAsync(w, p.flags, sizeof(w), cudaMemcpyDeviceToHost, s));
    FJ_CUDA(cudaStreamSynchronize(s));
    if (w[4] != 0) return fail(FJ_ERR_CUDA, "a replayed step graph found its slot counter out of range");
    if (w[3] != 0) return fail(FJ_ERR_TIMEOUT, "a tensor-core wait of the AIC factorisation expired");
    if (w[2] != kNoSlot) return fail(FJ_ERR_NONFINITE, "non-finite forces at time slot %d", w[2]);
    if (w[0] != 0) return fail(FJ_ERR_SINGULAR, "zero pivot in column %d of the AIC factorisation", w[0] - 1);
    return FJ_OK;
}

static BatchItem step_item(const Plan& p, const fj_case_buffers* B, int k, bool refactor) {
    const int64_t hs = (int64_t)p.cfg.n_nodes * 16;
    BatchItem it;
    it.p = p;
    it.B = B;
    it.i = k;
    it.refactor = refactor;
    it.hg_n = B->d_hg_t + (int64_t)k * hs;
    it.hgd_n = B->d_hg_dot_t + (int64_t)k * hs;
    it.hg_nm1 = B->d_hg_t + (int64_t)(k - 1) * hs;
    return it;
}

// Steps g0..g1-1 (none refactorising) replayed from one captured step: every slot's
// table is built on the host and uploaded once; the graph selects the table of slot
// *step_ctr, runs the step's kernels on the fixed table area and advances the counter.
// The capture runs on a private stream (the legacy default stream cannot be captured);
// the replays go to the caller's stream.
//
// The executable graph is kept for later calls on the same workspace: its kernels take
// only workspace pointers and the host values of the step's launch signature, so a call
// whose first step has the same signature replays it without a new capture.  A small
// cache (least recently used out) bounds the graphs held.
struct RangeGraph {
    const void* tab = nullptr;
    std::vector<int64_t> sig;
    cudaGraphExec_t exec = nullptr;
    int64_t kernels = 0;
    uint64_t used = 0;
};
constexpr int kRangeGraphs = 16;
static std::mutex g_rg_mu;
static std::vector<RangeGraph> g_rg;
static uint64_t g_rg_clock = 0;

static int run_range_graph(const Plan& p, const fj_case_buffers* B, int g0, int g1, cudaStream_t s) {
    std::vector<char> h((size_t)(g1 - g0) * p.tab_bytes);
    std::vector<int64_t> sig;
    for (int k = g0; k < g1; ++k) {
        std::vector<BatchItem> one(1, step_item(p, B, k, false));
        FJ_TRY(run_steps(one, p.tab, p.tab_bytes, s, kStepBuild, h.data() + (size_t)(k - g0) * p.tab_bytes,
                         k == g0 ? &sig : nullptr));
    }
    // the graph's own select and advance kernels take the slot tables, the counter and a
    // status word: the counter's place in the workspace follows the slot count, so a
    // workspace at the same address for a case of another length must not replay this graph
    sig.push_back((int64_t)(uintptr_t)p.tab_all);
    sig.push_back((int64_t)(uintptr_t)p.step_ctr);
    sig.push_back((int64_t)(uintptr_t)p.flags);
    sig.push_back((int64_t)p.tab_bytes);
    sig.push_back((int64_t)p.cfg.n_tstep);
    FJ_TRY(upload(p.tab_all + (size_t)g0 * p.tab_bytes, h.data(), h.size(), s));
    FJ_TRY(upload(p.step_ctr, &g0, sizeof(int), s));

    std::lock_guard<std::mutex> lk(g_rg_mu);
    RangeGraph* rg = nullptr;
    for (RangeGraph& r : g_rg)
        if (r.tab == p.tab) rg = &r;
    if (rg == nullptr || rg->sig != sig || rg->exec == nullptr) {
        cudaStream_t cs = nullptr;
        FJ_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaGraph_t graph = nullptr;
        const int64_t launches0 = launch_count();
        int st = cuda_status(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal), "step graph capture");
        if (st == FJ_OK) {
            k_select_table<<<32, 256, 0, cs>>>(p.tab_all, p.tab_bytes, p.step_ctr, p.cfg.n_tstep, p.tab, p.flags + 4);
            note_launch();
            std::vector<BatchItem> one(1, step_item(p, B, g0, false));
            st = run_steps(one, p.tab, p.tab_bytes, cs, kStepLaunch);
            k_advance<<<1, 32, 0, cs>>>(p.step_ctr); note_launch();
            const int st_end = cuda_status(cudaStreamEndCapture(cs, &graph), "step graph capture");
            if (st == FJ_OK) st = st_end;
        }
        cudaStreamDestroy(cs);
        cudaGraphExec_t exec = nullptr;
        if (st == FJ_OK) st = cuda_status(cudaGraphInstantiate(&exec, graph, 0), "step graph instantiate");
        if (graph) cudaGraphDestroy(graph);
        if (st != FJ_OK) return st;
        if (rg == nullptr) {
            if ((int)g_rg.size() < kRangeGraphs) {
                g_rg.emplace_back();
                rg = &g_rg.back();
            } else {  // least recently used out
                rg = &g_rg[0];
                for (RangeGraph& r : g_rg)
                    if (r.used < rg->used) rg = &r;
            }
        }
        if (rg->exec) cudaGraphExecDestroy(rg->exec);
        rg->tab = p.tab;
        rg->sig.swap(sig);
        rg->exec = exec;
        // the capture counted the step's kernels once; the first replay runs them
        rg->kernels = launch_count() - launches0;
        note_launch((int)(-rg->kernels));
    }
    rg->used = ++g_rg_clock;
    int st = FJ_OK;
    for (int k = g0; k < g1 && st == FJ_OK; ++k) {
        st = cuda_status(cudaGraphLaunch(rg->exec, s), "step graph launch");
        note_launch((int)rg->kernels);
    }
    if (st == FJ_OK) st = cuda_status(cudaStreamSynchronize(s), "step graph replay");
    return st;
}

static int run_dynamic(const Plan& p, const fj_case_buffers* B, int i_first, int i_last, int flags, cudaStream_t s) {
    const bool mixed = p.cfg.precision == FJ_PREC_MIXED;
    const bool graphs = !(flags & FJ_NO_GRAPH) && !prof_active();
    bool refactor_all = false;
    int i = i_first;
    for (int attempt = 0; attempt < 2; ++attempt) {
        int k = i;
        while (k < i_last) {
            const bool first = (k == i) && !(attempt == 0 && (flags & FJ_REUSE_FACTORS));
            const bool refactor = refactor_all || first;
            // the first step always runs directly (it also does the one-time set-up)
            if (graphs && !refactor && k > i && i_last - k >= 2) break;
            std::vector<BatchItem> one(1, step_item(p, B, k, refactor));
            // the cached convection velocities belong to the previous call's step: only the
            // first step of the first attempt may take them
            one[0].reuse_convection = attempt == 0 && k == i_first && (flags & FJ_REUSE_CONVECTION);
            FJ_TRY(run_steps(one, p.tab, p.tab_bytes, s));
            ++k;
        }
        if (k < i_last) FJ_TRY(run_range_graph(p, B, k, i_last, s));
        if (!mixed) break;
        // read the refinement residuals back once; re-run from the first failure with a
        // fresh factorisation every step if the cached factors were not good enough
        std::vector<double> res(i_last - i);
        FJ_CUDA(cudaMemcpyAsync(res.data(), p.resid + i, res.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
        FJ_TRY(read_status(p, s));  // non-finite data is not a refinement failure
        int bad = -1;
        for (size_t q = 0; q < res.size(); ++q)
            if (!(res[q] <= 1e-12)) {
                bad = (int)q + i;
                break;
            }
        if (bad < 0) return FJ_OK;
        if (refactor_all)
            return fail(FJ_ERR_NOT_CONVERGED, "refinement residual %.3g at slot %d after refactorisation",
                        res[bad - i], bad);
        refactor_all = true;
        i = bad;
    }
    return FJ_OK;
}

}  // namespace fj

// =====================================================================================
// C ABI
// =====================================================================================
using namespace fj;

extern "C" {

const char* fj_last_error_string(void) { return fj::last_error(); }

int fj_version(void) { return 100; }

int fj_case_workspace_size(const fj_case_config* cfg, size_t* bytes) {
    if (bytes == nullptr) return fail(FJ_ERR_SHAPE, "bytes is NULL");
    Plan p;
    FJ_TRY(make_plan(cfg, nullptr, 0, p));
    *bytes = p.ws_needed + 256;
    return FJ_OK;
}

int fj_solve_static(const fj_case_config* cfg, const fj_case_buffers* bufs, int horseshoe, double t0, void* d_ws,
                    size_t ws_bytes, fj_stream_t stream) {
    Plan p;
    FJ_TRY(make_plan(cfg, d_ws, ws_bytes, p));
    FJ_TRY(check_buffers(p, bufs, false));
    const double* hg = bufs->d_hg_t;
    if (hg == nullptr) return fail(FJ_ERR_SHAPE, "d_hg_t is NULL (slot 0 holds the static frames)");
    cudaStream_t s = (cudaStream_t)stream;
    FJ_TRY(clear_status(p, s));
    FJ_TRY(run_static(p, bufs, hg, horseshoe, t0, s));
    return read_status(p, s);
}

int fj_solve_prescribed_dynamic(const fj_case_config* cfg, const fj_case_buffers* bufs, int i_first, int i_last,
                                int flags, void* d_ws, size_t ws_bytes, fj_stream_t stream) {
    Plan p;
    FJ_TRY(make_plan(cfg, d_ws, ws_bytes, p));
    FJ_TRY(check_buffers(p, bufs, true));
    if (i_first < 1 || i_last > cfg->n_tstep || i_first > i_last)
        return fail(FJ_ERR_SHAPE, "step range [%d, %d) not within [1, %d)", i_first, i_last, cfg->n_tstep);
    if (i_first == i_last) return FJ_OK;
    cudaStream_t s = (cudaStream_t)stream;
    FJ_TRY(clear_status(p, s));
    FJ_TRY(run_dynamic(p, bufs, i_first, i_last, flags, s));
    return read_status(p, s);
}

int fj_case_step(const fj_case_config* cfg, const fj_case_buffers* bufs, int i_ts, int flags, void* d_ws,
                 size_t ws_bytes, fj_stream_t stream) {
    return fj_solve_prescribed_dynamic(cfg, bufs, i_ts, i_ts + 1, flags, d_ws, ws_bytes, stream);
}

int fj_batch_workspace_size(int max_items, size_t* bytes) {
    if (bytes == nullptr || max_items < 1) return fail(FJ_ERR_SHAPE, "batch workspace: max_items=%d", max_items);
    *bytes = table_layout(max_items).total + 256;
    return FJ_OK;
}

}  // extern "C"

namespace fj {

// Captured batched steps, one per batch workspace.  A batch whose launch signature (the
// grid extents, job counts and out-of-table pointers run_steps reports) equals that of the
// last capture on its workspace uploads its table and replays the graph; any other batch
// re-captures (updating the executable graph in place where CUDA allows).  The sum kernels
// are persistent, so the cases' sizes enter only through the grid maxima.
struct BatchGraph {
    std::vector<int64_t> sig;
    cudaGraphExec_t exec = nullptr;
    int64_t kernels = 0;
};
static std::mutex g_bg_mu;
static std::unordered_map<const void*, BatchGraph> g_bg;
static std::atomic<int64_t> g_bg_replays{0}, g_bg_captures{0};

static int step_batched_graph(std::vector<BatchItem>& v, char* d_tab, size_t tab_bytes, cudaStream_t s) {
    std::vector<char> h(table_layout((int)v.size()).total);
    std::vector<int64_t> sig;
    FJ_TRY(run_steps(v, d_tab, tab_bytes, s, kStepBuild, h.data(), &sig));
    FJ_TRY(upload(d_tab, h.data(), h.size(), s));
    std::lock_guard<std::mutex> lk(g_bg_mu);
    BatchGraph& bg = g_bg[d_tab];
    if (bg.exec != nullptr && bg.sig == sig) {
        note_launch((int)bg.kernels);  // the replay runs the captured kernels once more
        g_bg_replays.fetch_add(1);
        return cuda_status(cudaGraphLaunch(bg.exec, s), "batched step graph launch");
    }
    cudaStream_t cs = nullptr;
    FJ_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t graph = nullptr;
    const int64_t launches0 = launch_count();
    int st = cuda_status(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal), "batched step capture");
    if (st == FJ_OK) {
        st = run_steps(v, d_tab, tab_bytes, cs, kStepLaunch, nullptr, nullptr, true);
        const int st_end = cuda_status(cudaStreamEndCapture(cs, &graph), "batched step capture");
        if (st == FJ_OK) st = st_end;
    }
    cudaStreamDestroy(cs);
    if (st == FJ_OK) {
        cudaGraphExecUpdateResultInfo info;
        if (bg.exec != nullptr && cudaGraphExecUpdate(bg.exec, graph, &info) != cudaSuccess) {
            cudaGetLastError();  // an update that does not apply is not an error: instantiate anew
            cudaGraphExecDestroy(bg.exec);
            bg.exec = nullptr;
        }
        if (bg.exec == nullptr) st = cuda_status(cudaGraphInstantiate(&bg.exec, graph, 0), "batched step instantiate");
    }
    if (graph) cudaGraphDestroy(graph);
    if (st != FJ_OK) {
        if (bg.exec) cudaGraphExecDestroy(bg.exec);
        g_bg.erase(d_tab);
        return st;
    }
    bg.sig.swap(sig);
    bg.kernels = launch_count() - launches0;
    g_bg_captures.fetch_add(1);
    return cuda_status(cudaGraphLaunch(bg.exec, s), "batched step graph launch");
}

}  // namespace fj

extern "C" {

int fj_batch_release(void* d_batch_ws) {
    std::lock_guard<std::mutex> lk(g_bg_mu);
    auto it = g_bg.find(d_batch_ws);
    if (it == g_bg.end()) return FJ_OK;
    if (it->second.exec) FJ_CUDA(cudaGraphExecDestroy(it->second.exec));
    g_bg.erase(it);
    return FJ_OK;
}

int fj_batch_graph_stats(int64_t* replays, int64_t* captures) {
    if (replays) *replays = g_bg_replays.load();
    if (captures) *captures = g_bg_captures.load();
    return FJ_OK;
}

int fj_step_batched(const fj_batch_item* items, int n_items, void* d_batch_ws, size_t batch_ws_bytes,
                    fj_stream_t stream) {
    if (n_items < 0 || (n_items > 0 && items == nullptr)) return fail(FJ_ERR_SHAPE, "n_items=%d", n_items);
    if (n_items == 0) return FJ_OK;
    // graph replay unless a caller opts out, a case refactorises (its factorisation is
    // direct launches) or the event profiler is recording launch times
    bool graphs = !prof_active();
    std::vector<BatchItem> v(n_items);
    for (int k = 0; k < n_items; ++k) {
        const fj_batch_item& it = items[k];
        FJ_TRY(make_plan(it.cfg, it.d_ws, it.ws_bytes, v[k].p));
        FJ_TRY(check_buffers(v[k].p, it.bufs, true));
        if (it.i_ts < 1 || it.i_ts >= it.cfg->n_tstep)
            return fail(FJ_ERR_SHAPE, "item %d: slot %d not in [1, %d)", k, it.i_ts, it.cfg->n_tstep);
        const int64_t hs = (int64_t)it.cfg->n_nodes * 16;
        v[k].B = it.bufs;
        v[k].i = it.i_ts;
        v[k].refactor = !(it.flags & FJ_REUSE_FACTORS);
        v[k].reuse_convection = (it.flags & FJ_REUSE_CONVECTION) != 0;
        v[k].hg_n = it.bufs->d_hg_t + it.i_ts * hs;
        v[k].hgd_n = it.bufs->d_hg_dot_t + it.i_ts * hs;
        v[k].hg_nm1 = it.bufs->d_hg_t + (it.i_ts - 1) * hs;
        graphs = graphs && !(it.flags & FJ_NO_GRAPH) && !v[k].refactor;
    }
    if (!graphs) return run_steps(v, (char*)d_batch_ws, batch_ws_bytes, (cudaStream_t)stream);
    return step_batched_graph(v, (char*)d_batch_ws, batch_ws_bytes, (cudaStream_t)stream);
}

int fj_case_residual(const fj_case_config* cfg, void* d_ws, size_t ws_bytes, int i_ts, double* h_out,
                     fj_stream_t stream) {
    Plan p;
    FJ_TRY(make_plan(cfg, d_ws, ws_bytes, p));
    if (i_ts < 0 || i_ts >= cfg->n_tstep || h_out == nullptr) return fail(FJ_ERR_SHAPE, "slot %d", i_ts);
    FJ_CUDA(cudaMemcpyAsync(h_out, p.resid + i_ts, sizeof(double), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    FJ_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    return FJ_OK;
}

int fj_case_factors_copy(const fj_case_config* cfg, const void* d_ws, size_t ws_bytes, double* d_lu,
                         int32_t* d_piv, fj_stream_t stream) {
    if (cfg == nullptr || d_lu == nullptr || d_piv == nullptr) return fail(FJ_ERR_SHAPE, "factors_copy: null argument");
    if (cfg->precision != FJ_PREC_FP64)
        return fail(FJ_ERR_UNSUPPORTED, "factors_copy: only FP64 cases keep FP64 factors");
    Plan p;
    FJ_TRY(make_plan(cfg, const_cast<void*>(d_ws), ws_bytes, p));
    cudaStream_t s = (cudaStream_t)stream;
    FJ_CUDA(cudaMemcpyAsync(d_lu, p.a64, (size_t)p.nb * p.nb * sizeof(double), cudaMemcpyDeviceToDevice, s));
    FJ_CUDA(cudaMemcpyAsync(d_piv, p.piv, (size_t)p.nb * sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
    return FJ_OK;
}

int fj_biot_savart(const double* d_x, const double* d_y, int64_t n_pairs, int kernel, double r_cut, double* d_out,
                   fj_stream_t stream) {
    return biot_savart_pairs(d_x, d_y, n_pairs, kernel, r_cut, d_out, (cudaStream_t)stream);
}

static int vind_plan(int64_t n_targets, const int* rows, const int* cols, int n_lattices, int mirror, int precision,
                     int64_t& n_elem, int& n_split, size_t& bytes) {
    if (n_targets < 0 || n_lattices < 0 || n_lattices > FJ_MAX_SURF * 2)
        return fail(FJ_ERR_SHAPE, "vind: n_targets=%lld n_lattices=%d", (long long)n_targets, n_lattices);
    if (precision != FJ_PREC_FP64 && precision != FJ_PREC_MIXED) return fail(FJ_ERR_UNSUPPORTED, "precision %d", precision);
    n_elem = 0;
    for (int i = 0; i < n_lattices; ++i) {
        if (rows[i] < 0 || cols[i] < 0) return fail(FJ_ERR_SHAPE, "vind: lattice %d has rows=%d cols=%d", i, rows[i], cols[i]);
        n_elem += (mirror ? 2 : 1) * stream_len(rows[i], cols[i]);
    }
    n_split = split_bound(std::max<int64_t>(n_targets, 1), n_elem, precision);
    Arena a(nullptr, 0);
    a.carve<Elem64>(n_elem);
    a.carve<double>((int64_t)n_split * std::max<int64_t>(n_targets, 1) * 3);
    bytes = a.used + 256;
    return FJ_OK;
}

int fj_vind_workspace_size(int64_t n_targets, const int* rows, const int* cols, int n_lattices, int mirror,
                           int precision, size_t* bytes) {
    int64_t ne;
    int sp;
    size_t b;
    FJ_TRY(vind_plan(n_targets, rows, cols, n_lattices, mirror, precision, ne, sp, b));
    *bytes = b;
    return FJ_OK;
}

int fj_vind(const double* d_targets, int64_t n_targets, const double* const* d_zetas, const double* const* d_gammas,
            const int* rows, const int* cols, int n_lattices, const double* mirror_point, const double* mirror_normal,
            int kernel, double r_cut, int precision, double* d_v_out, void* d_ws, size_t ws_bytes,
            fj_stream_t stream) {
    cudaStream_t s = (cudaStream_t)stream;
    const int mirror = mirror_point != nullptr && mirror_normal != nullptr;
    int64_t ne;
    int sp;
    size_t need;
    FJ_TRY(vind_plan(n_targets, rows, cols, n_lattices, mirror, precision, ne, sp, need));
    if (kernel < 0 || kernel > 2) return fail(FJ_ERR_UNSUPPORTED, "kernel %d", kernel);
    if (precision == FJ_PREC_MIXED && kernel == FJ_KERNEL_PLAIN)
        return fail(FJ_ERR_UNSUPPORTED, "the unregularised kernel is FP64-only");
    if (ws_bytes < need) return fail(FJ_ERR_NOMEM, "vind workspace %zu < %zu", ws_bytes, need);
    if (n_targets == 0) return FJ_OK;
    Arena a(d_ws, ws_bytes);
    void* st = a.carve<Elem64>(ne);
    double* part = a.carve<double>((int64_t)sp * n_targets * 3);
    PackArgs pa;
    memset(&pa, 0, sizeof(pa));
    pa.kernel = kernel;
    pa.r_cut = r_cut;
    if (mirror)
        for (int d = 0; d < 3; ++d) {
            pa.mirror.p[d] = mirror_point[d];
            pa.mirror.nrm[d] = mirror_normal[d];
        }
    int n = 0;
    for (int i = 0; i < n_lattices; ++i) {
        for (int img = 0; img < (mirror ? 2 : 1); ++img) {
            LatticeRef& L = pa.lat[n];
            L.zeta = d_zetas[i];
            L.gamma = d_gammas[i];
            L.rows = rows[i];
            L.cols = cols[i];
            L.sign = img ? -1.0f : 1.0f;
            L.mirrored = img;
            pa.offset[n + 1] = pa.offset[n] + stream_len(rows[i], cols[i]);
            ++n;
        }
    }
    pa.n_lat = n;
    if (ne == 0) {
        FJ_CUDA(cudaMemsetAsync(d_v_out, 0, n_targets * 3 * sizeof(double), s));
        return FJ_OK;
    }
    if (precision == FJ_PREC_FP64)
        FJ_TRY(pack_stream64(pa, (Elem64*)st, s));
    else
        FJ_TRY(pack_stream32(pa, (Elem32*)st, s));
    VindJob j;
    j.targets = d_targets;
    j.n_targets = n_targets;
    j.stream = st;
    j.n_elem = ne;
    j.n_split = std::min(sp, choose_split(n_targets, ne, precision));
    j.part = part;
    j.out = d_v_out;
    j.n_links = 0;
    for (int i = 0; i < n_lattices; ++i) j.n_links += (mirror ? 2 : 1) * lattice_links(rows[i], cols[i]);
    FJ_TRY(vind_launch(j, precision, kernel, r_cut, s));
    return reduce_partials(part, j.n_split, n_targets, d_v_out, 0, 1.0, s);
}

int fj_aic_workspace_size(const int* m, const int* n, int n_surf, size_t* bytes) {
    if (bytes == nullptr || n_surf < 1 || n_surf > FJ_MAX_SURF) return fail(FJ_ERR_SHAPE, "aic workspace: n_surf=%d", n_surf);
    int64_t nb = 0;
    for (int s = 0; s < n_surf; ++s) nb += (int64_t)m[s] * n[s];
    Arena a(nullptr, 0);
    a.carve<double>(nb * 3);
    a.carve<double>(nb * 3);
    *bytes = a.used + 256;
    return FJ_OK;
}

int fj_aic_assemble(const double* const* d_zetas_b, const int* m, const int* n, int n_surf,
                    const double* const* d_zetas_w, const int* m_star, const double* mirror_point,
                    const double* mirror_normal, int kernel, double r_cut, double* d_aic, void* d_ws, size_t ws_bytes,
                    fj_stream_t stream) {
    cudaStream_t st = (cudaStream_t)stream;
    size_t need;
    FJ_TRY(fj_aic_workspace_size(m, n, n_surf, &need));
    if (ws_bytes < need) return fail(FJ_ERR_NOMEM, "aic workspace %zu < %zu", ws_bytes, need);
    if (kernel < 0 || kernel > 2) return fail(FJ_ERR_UNSUPPORTED, "kernel %d", kernel);
    fj_case_config cfg;
    memset(&cfg, 0, sizeof(cfg));
    cfg.n_surf = n_surf;
    for (int s = 0; s < n_surf; ++s) {
        if (m[s] < 1 || n[s] < 1) return fail(FJ_ERR_SHAPE, "surface %d: m=%d n=%d", s, m[s], n[s]);
        cfg.m[s] = m[s];
        cfg.n[s] = n[s];
        cfg.m_star[s] = d_zetas_w != nullptr ? m_star[s] : 0;
    }
    Layout L = make_layout(cfg);
    const int64_t nb = L.po[n_surf];
    Arena a(d_ws, ws_bytes);
    double* c = a.carve<double>(nb * 3);
    double* nc = a.carve<double>(nb * 3);
    for (int s = 0; s < n_surf; ++s) {
        surface_c_nc_kernel<<<nblk((int64_t)m[s] * n[s]), 256, 0, st>>>(m[s], n[s], d_zetas_b[s], c + L.po[s] * 3,
                                                                       nc + L.po[s] * 3); note_launch();
    }
    FJ_LAUNCH_CHECK("aic geometry");
    AicArgs aa;
    memset(&aa, 0, sizeof(aa));
    aa.n_surf = n_surf;
    aa.max_fil = 0;
    for (int s = 0; s < n_surf; ++s) {
        aa.zeta_b[s] = d_zetas_b[s];
        aa.m[s] = m[s];
        aa.n[s] = n[s];
        aa.col_off[s] = L.po[s];
        aa.max_fil = std::max(aa.max_fil, m[s] * (n[s] + 1) + (m[s] + 1) * n[s]);
        aa.zeta_w[s] = (d_zetas_w != nullptr && m_star[s] > 0) ? d_zetas_w[s] : nullptr;
        aa.m_star[s] = d_zetas_w != nullptr ? m_star[s] : 0;
    }
    aa.n_rows = nb;
    aa.mirror = mirror_point != nullptr && mirror_normal != nullptr;
    if (aa.mirror)
        for (int d = 0; d < 3; ++d) {
            aa.mp.p[d] = mirror_point[d];
            aa.mp.nrm[d] = mirror_normal[d];
        }
    aa.kernel = kernel;
    aa.rc2 = r_cut * r_cut;
    aa.c = c;
    aa.nc = nc;
    aa.aic = d_aic;
    aa.ld = nb;
    return aic_launch(aa, nullptr, st);
}

int fj_lu_workspace_size(int n, size_t* bytes) {
    if (bytes == nullptr || n < 0) return fail(FJ_ERR_SHAPE, "lu workspace: n=%d", n);
    *bytes = 256 + (size_t)n * sizeof(double);  // info word, then n doubles of solve scratch
    return FJ_OK;
}

int fj_lu_factor(double* d_a, int n, int32_t* d_piv, void* d_ws, size_t ws_bytes, fj_stream_t stream) {
    if (ws_bytes < sizeof(int)) return fail(FJ_ERR_NOMEM, "lu workspace too small");
    return lu_factor64(d_a, n, d_piv, (int*)d_ws, (cudaStream_t)stream);
}

int fj_lu_solve(const double* d_lu, int n, const int32_t* d_piv, double* d_b, void* d_ws, size_t ws_bytes,
                fj_stream_t stream) {
    if (ws_bytes < 256 + (size_t)n * sizeof(double)) return fail(FJ_ERR_NOMEM, "lu_solve workspace too small");
    return lu_solve64(d_lu, n, d_piv, d_b, (double*)((char*)d_ws + 256), (cudaStream_t)stream);
}

int fj_solve_mixed_workspace_size(int n, size_t* bytes) {
    Arena a(nullptr, 0);
    a.carve<float>((int64_t)n * n);
    a.carve<float>((int64_t)n * n);
    a.carve<int32_t>(n);
    a.carve<double>(n);
    a.carve<int>(4);
    a.carve<float>(tc_tri_floats(n));
    *bytes = a.used + 256;
    return FJ_OK;
}

int fj_solve_mixed(const double* d_a, int n, const double* d_b, double* d_x, int refactor, double* d_resid, void* d_ws,
                   size_t ws_bytes, fj_stream_t stream) {
    cudaStream_t s = (cudaStream_t)stream;
    size_t need;
    FJ_TRY(fj_solve_mixed_workspace_size(n, &need));
    if (ws_bytes < need) return fail(FJ_ERR_NOMEM, "solve_mixed workspace %zu < %zu", ws_bytes, need);
    Arena a(d_ws, ws_bytes);
    float* a32 = a.carve<float>((int64_t)n * n);
    float* x32 = a.carve<float>((int64_t)n * n);
    int32_t* piv = a.carve<int32_t>(n);
    double* r = a.carve<double>(n);
    int* info = a.carve<int>(4);
    float* tri = a.carve<float>(tc_tri_floats(n));
    if (refactor) {
        FJ_TRY(factor_inverse32(d_a, n, a32, piv, info, x32, tri, s));
    }
    return refine_solve(d_a, x32, n, d_b, d_x, r, d_resid, 3, s);
}

}  // extern "C"
