// C++ FP64 restatement of the pair-heavy part of the UVLM step (TEST INFRASTRUCTURE AND
// CPU BASELINE ONLY; the product is the CUDA library).
//
// Restates, with OpenMP over target points and SIMD over filaments:
//   * the Biot-Savart kernels biot_savart_epsilon / biot_savart_cutoff / biot_savart
//     (aero/utils.py:580-648; epsilon = 1e-7, utils/constants.py:16);
//   * compute_v_ind (aero/aic.py:248-310): v(x) = sum over lattices and filaments of
//     K(x; y0, y1) * G_eff, chordwise G_eff = G[k,l] - G[k,l-1], spanwise
//     G_eff = G[k-1,l] - G[k,l] (zero-padded, aic.py:284-287), mirror images subtracted
//     (aic.py:295-308, mirror_grid aero/utils.py:651-663);
//   * compute_aic_solve (aero/aic.py:11-205): per collocation point the normal component
//     of every filament's unit-strength influence, ring (k,l) =
//     -(M[k,l+1] - M[k,l]) + (N[k+1,l] - N[k,l]) (aic.py:55-57), mirror grid subtracted,
//     and for the static solve the wake rings summed over rows onto the trailing-edge
//     bound row (add_wake_influence, aic.py:190-205).
// The Python side (oracle/uvlm_cpp.py) keeps the O(M N) arithmetic and the LAPACK solve.
#include <cmath>
#include <cstdint>
#include <vector>

#include <omp.h>

namespace {

constexpr double kEps = 1e-7;
constexpr double kInvFourPi = 1.0 / (4.0 * M_PI);

enum { KER_EPSILON = 0, KER_CUTOFF = 1, KER_PLAIN = 2 };

// Filaments as structure-of-arrays: start y0, end y1, strength g.
struct Filaments {
    std::vector<double> ax, ay, az, bx, by, bz, g;
    void add(const double* p, const double* q, double s) {
        ax.push_back(p[0]);
        ay.push_back(p[1]);
        az.push_back(p[2]);
        bx.push_back(q[0]);
        by.push_back(q[1]);
        bz.push_back(q[2]);
        g.push_back(s);
    }
    int64_t size() const { return (int64_t)g.size(); }
};

void reflect(const double* y, const double* mp, const double* mn, double* o) {
    const double d = (y[0] - mp[0]) * mn[0] + (y[1] - mp[1]) * mn[1] + (y[2] - mp[2]) * mn[2];
    for (int k = 0; k < 3; ++k) o[k] = y[k] - 2.0 * d * mn[k];
}

// Vertex (k, l) of a (R+1, C+1, 3) lattice, reflected when mp != nullptr.
void vertex(const double* zeta, int C, int k, int l, const double* mp, const double* mn, double* o) {
    const double* y = zeta + ((int64_t)k * (C + 1) + l) * 3;
    if (mp)
        reflect(y, mp, mn, o);
    else
        for (int d = 0; d < 3; ++d) o[d] = y[d];
}

// Chordwise filaments (k,l)->(k+1,l) in (k, l) order, then spanwise (k,l)->(k,l+1).
// Strength: G_eff * sign when gamma is given, else 1 (unit influences for the AIC).
void add_lattice(Filaments& f, const double* zeta, const double* gamma, int R, int C, double sign,
                 const double* mp, const double* mn) {
    double p[3], q[3];
    auto G = [&](int k, int l) { return (k < 0 || l < 0 || k >= R || l >= C) ? 0.0 : gamma[(int64_t)k * C + l]; };
    for (int k = 0; k < R; ++k)
        for (int l = 0; l <= C; ++l) {
            vertex(zeta, C, k, l, mp, mn, p);
            vertex(zeta, C, k + 1, l, mp, mn, q);
            f.add(p, q, gamma ? sign * (G(k, l) - G(k, l - 1)) : sign);
        }
    for (int k = 0; k <= R; ++k)
        for (int l = 0; l < C; ++l) {
            vertex(zeta, C, k, l, mp, mn, p);
            vertex(zeta, C, k, l + 1, mp, mn, q);
            f.add(p, q, gamma ? sign * (G(k - 1, l) - G(k, l)) : sign);
        }
}

// K(x; y0, y1) for one pair (aero/utils.py:580-648), written branch-free for SIMD.
template <int KER>
inline void kernel_pair(double x, double y, double z, double ax, double ay, double az, double bx, double by,
                        double bz, double rc, double& kx, double& ky, double& kz) {
    const double r0x = bx - ax, r0y = by - ay, r0z = bz - az;
    const double r1x = x - ax, r1y = y - ay, r1z = z - az;
    const double r2x = x - bx, r2y = y - by, r2z = z - bz;
    const double cx = r1y * r2z - r1z * r2y;
    const double cy = r1z * r2x - r1x * r2z;
    const double cz = r1x * r2y - r1y * r2x;
    const double c2 = cx * cx + cy * cy + cz * cz;
    const double n1sq = r1x * r1x + r1y * r1y + r1z * r1z;
    const double n2sq = r2x * r2x + r2y * r2y + r2z * r2z;
    const double r0sq = r0x * r0x + r0y * r0y + r0z * r0z;
    double i1, i2, coef;
    if (KER == KER_PLAIN) {
        i1 = 1.0 / std::sqrt(n1sq);
        i2 = 1.0 / std::sqrt(n2sq);
    } else {
        i1 = 1.0 / std::sqrt(n1sq + kEps * kEps);
        i2 = 1.0 / std::sqrt(n2sq + kEps * kEps);
    }
    const double dot = r0x * (r1x * i1 - r2x * i2) + r0y * (r1y * i1 - r2y * i2) + r0z * (r1z * i1 - r2z * i2);
    if (KER == KER_EPSILON) {
        coef = dot * kInvFourPi / (c2 + kEps * r0sq * r0sq);
    } else if (KER == KER_CUTOFF) {
        // perpendicular distance from x to the filament line: |x - (y0 + s r0)|
        const double s = (r0x * r1x + r0y * r1y + r0z * r1z) / r0sq;
        const double dx = r1x - s * r0x, dy = r1y - s * r0y, dz = r1z - s * r0z;
        const double r = std::sqrt(dx * dx + dy * dy + dz * dz);
        coef = (r > rc) ? dot * kInvFourPi / c2 : 0.0;
    } else {
        coef = dot * kInvFourPi / c2;
    }
    kx = coef * cx;
    ky = coef * cy;
    kz = coef * cz;
}

template <int KER>
void vind_all(const double* t, int64_t n_t, const Filaments& f, double rc, double* out) {
    const int64_t ns = f.size();
    const double *ax = f.ax.data(), *ay = f.ay.data(), *az = f.az.data();
    const double *bx = f.bx.data(), *by = f.by.data(), *bz = f.bz.data(), *g = f.g.data();
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n_t; ++i) {
        const double x = t[i * 3], y = t[i * 3 + 1], z = t[i * 3 + 2];
        double vx = 0.0, vy = 0.0, vz = 0.0;
#pragma omp simd reduction(+ : vx, vy, vz)
        for (int64_t s = 0; s < ns; ++s) {
            double kx, ky, kz;
            kernel_pair<KER>(x, y, z, ax[s], ay[s], az[s], bx[s], by[s], bz[s], rc, kx, ky, kz);
            vx += g[s] * kx;
            vy += g[s] * ky;
            vz += g[s] * kz;
        }
        out[i * 3] = vx;
        out[i * 3 + 1] = vy;
        out[i * 3 + 2] = vz;
    }
}

// Normal component of each unit filament's influence at x: infl[s] = n . K(x; s).
template <int KER>
inline void normal_influences(double x, double y, double z, const double* nrm, const Filaments& f, double rc,
                              double* infl) {
    const int64_t ns = f.size();
    const double *ax = f.ax.data(), *ay = f.ay.data(), *az = f.az.data();
    const double *bx = f.bx.data(), *by = f.by.data(), *bz = f.bz.data();
    const double n0 = nrm[0], n1 = nrm[1], n2 = nrm[2];
#pragma omp simd
    for (int64_t s = 0; s < ns; ++s) {
        double kx, ky, kz;
        kernel_pair<KER>(x, y, z, ax[s], ay[s], az[s], bx[s], by[s], bz[s], rc, kx, ky, kz);
        infl[s] = kx * n0 + ky * n1 + kz * n2;
    }
}

// Ring influences of an R x C lattice from its filament influences (chordwise block
// R*(C+1), then spanwise (R+1)*C), aic.py:55-57.
inline void rings(const double* infl, int R, int C, double* out /* R*C */) {
    const double* m = infl;
    const double* n = infl + (int64_t)R * (C + 1);
    for (int k = 0; k < R; ++k)
        for (int l = 0; l < C; ++l) {
            const double dm = m[(int64_t)k * (C + 1) + l + 1] - m[(int64_t)k * (C + 1) + l];
            const double dn = n[(int64_t)(k + 1) * C + l] - n[(int64_t)k * C + l];
            out[(int64_t)k * C + l] = -dm + dn;
        }
}

struct LatticeFils {
    Filaments direct, image;
    int R, C;
};

template <int KER>
void aic_all(const double* c, const double* nc, int64_t n_c, const std::vector<LatticeFils>& bound,
             const std::vector<LatticeFils>& wake, bool mirror, double rc, int64_t n_cols, double* out) {
    int64_t max_f = 1, max_r = 1;
    for (const auto& L : bound) {
        max_f = std::max<int64_t>(max_f, L.direct.size());
        max_r = std::max<int64_t>(max_r, (int64_t)L.R * L.C);
    }
    for (const auto& L : wake) {
        max_f = std::max<int64_t>(max_f, L.direct.size());
        max_r = std::max<int64_t>(max_r, (int64_t)L.R * L.C);
    }
#pragma omp parallel
    {
        std::vector<double> infl(max_f), r_dir(max_r), r_img(max_r);
#pragma omp for schedule(static)
        for (int64_t i = 0; i < n_c; ++i) {
            const double x = c[i * 3], y = c[i * 3 + 1], z = c[i * 3 + 2];
            double* row = out + i * n_cols;
            int64_t off = 0;
            for (size_t j = 0; j < bound.size(); ++j) {
                const LatticeFils& L = bound[j];
                const int64_t nr = (int64_t)L.R * L.C;
                normal_influences<KER>(x, y, z, nc + i * 3, L.direct, rc, infl.data());
                rings(infl.data(), L.R, L.C, r_dir.data());
                if (mirror) {
                    normal_influences<KER>(x, y, z, nc + i * 3, L.image, rc, infl.data());
                    rings(infl.data(), L.R, L.C, r_img.data());
                    for (int64_t r = 0; r < nr; ++r) row[off + r] = r_dir[r] - r_img[r];
                } else {
                    for (int64_t r = 0; r < nr; ++r) row[off + r] = r_dir[r];
                }
                if (j < wake.size() && wake[j].R > 0) {  // static: wake rings lumped onto the TE row
                    const LatticeFils& W = wake[j];
                    normal_influences<KER>(x, y, z, nc + i * 3, W.direct, rc, infl.data());
                    rings(infl.data(), W.R, W.C, r_dir.data());
                    if (mirror) {
                        normal_influences<KER>(x, y, z, nc + i * 3, W.image, rc, infl.data());
                        rings(infl.data(), W.R, W.C, r_img.data());
                        for (int64_t r = 0; r < (int64_t)W.R * W.C; ++r) r_dir[r] -= r_img[r];
                    }
                    for (int l = 0; l < W.C; ++l) {
                        double s = 0.0;
                        for (int k = 0; k < W.R; ++k) s += r_dir[(int64_t)k * W.C + l];
                        row[off + (int64_t)(L.R - 1) * L.C + l] += s;
                    }
                }
                off += nr;
            }
        }
    }
}

}  // namespace

extern "C" {

int uvref_max_threads() { return omp_get_max_threads(); }

void uvref_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }

// compute_v_ind: targets (n_t, 3); lattices zeta_i (rows_i+1, cols_i+1, 3) with gamma_i
// (rows_i, cols_i); mirror plane (point, unit normal) or nulls; out (n_t, 3).
int uvref_vind(const double* targets, int64_t n_t, const double* const* zetas, const double* const* gammas,
               const int* rows, const int* cols, int n_lat, const double* mirror_point,
               const double* mirror_normal, int kernel, double r_cut, double* out) {
    Filaments f;
    for (int i = 0; i < n_lat; ++i) {
        add_lattice(f, zetas[i], gammas[i], rows[i], cols[i], 1.0, nullptr, nullptr);
        if (mirror_point && mirror_normal)
            add_lattice(f, zetas[i], gammas[i], rows[i], cols[i], -1.0, mirror_point, mirror_normal);
    }
    switch (kernel) {
        case KER_EPSILON: vind_all<KER_EPSILON>(targets, n_t, f, r_cut, out); break;
        case KER_CUTOFF: vind_all<KER_CUTOFF>(targets, n_t, f, r_cut, out); break;
        case KER_PLAIN: vind_all<KER_PLAIN>(targets, n_t, f, r_cut, out); break;
        default: return -1;
    }
    return 0;
}

// compute_aic_solve for collocation points c / normals nc (n_c, 3) against the bound
// lattices (m_i, n_i); zetas_w (m_star_i) given for the static solve only.  out is
// (n_c, sum m_i n_i) row-major.
int uvref_aic(const double* c, const double* nc, int64_t n_c, const double* const* zetas_b, const int* m,
              const int* n, int n_surf, const double* const* zetas_w, const int* m_star, const double* mirror_point,
              const double* mirror_normal, int kernel, double r_cut, double* out) {
    const bool mirror = mirror_point && mirror_normal;
    std::vector<LatticeFils> bound(n_surf), wake;
    int64_t n_cols = 0;
    for (int i = 0; i < n_surf; ++i) {
        bound[i].R = m[i];
        bound[i].C = n[i];
        add_lattice(bound[i].direct, zetas_b[i], nullptr, m[i], n[i], 1.0, nullptr, nullptr);
        if (mirror) add_lattice(bound[i].image, zetas_b[i], nullptr, m[i], n[i], 1.0, mirror_point, mirror_normal);
        n_cols += (int64_t)m[i] * n[i];
    }
    if (zetas_w) {
        wake.resize(n_surf);
        for (int i = 0; i < n_surf; ++i) {
            wake[i].R = m_star[i];
            wake[i].C = n[i];
            if (m_star[i] == 0) continue;
            add_lattice(wake[i].direct, zetas_w[i], nullptr, m_star[i], n[i], 1.0, nullptr, nullptr);
            if (mirror)
                add_lattice(wake[i].image, zetas_w[i], nullptr, m_star[i], n[i], 1.0, mirror_point, mirror_normal);
        }
    }
    switch (kernel) {
        case KER_EPSILON: aic_all<KER_EPSILON>(c, nc, n_c, bound, wake, mirror, r_cut, n_cols, out); break;
        case KER_CUTOFF: aic_all<KER_CUTOFF>(c, nc, n_c, bound, wake, mirror, r_cut, n_cols, out); break;
        case KER_PLAIN: aic_all<KER_PLAIN>(c, nc, n_c, bound, wake, mirror, r_cut, n_cols, out); break;
        default: return -1;
    }
    return 0;
}

}  // extern "C"
