// fj_aic.cuh -- AIC assembly and the geometry kernels that feed it.
#pragma once

#include "fj_vind.cuh"

namespace fj {

struct AicArgs {
    int n_surf;
    const double* zeta_b[FJ_MAX_SURF];  // (m+1, n+1, 3)
    int m[FJ_MAX_SURF], n[FJ_MAX_SURF];
    const double* zeta_w[FJ_MAX_SURF];  // static solve only; else null
    int m_star[FJ_MAX_SURF];
    int64_t col_off[FJ_MAX_SURF];       // first AIC column of each surface
    int64_t n_rows;                     // sum m*n
    int max_fil;                        // max over surfaces of m(n+1) + (m+1)n
    int mirror;
    MirrorPlane mp;
    int kernel;
    double rc2;
    const double* c;   // (n_rows, 3) collocation points, surfaces concatenated
    const double* nc;  // (n_rows, 3) area normals
    double* aic;       // row-major (n_rows, ld)
    int64_t ld;
    const int* run_flag;  // batched launches: skip this job when *run_flag == 0 (may be null)
};

// Batched: one launch for many AIC jobs (table in device memory); grid = (max rows, jobs).
int aic_launch_jobs(const AicArgs* d_tab, int n_jobs, int64_t max_rows, int max_fil, int any_mirror, int kernel,
                    cudaStream_t s);

// d_run_flag (device int, may be null): when *d_run_flag == 0 the kernel returns at once
// (used to skip re-assembly when the bound lattice is bitwise unchanged).
int aic_launch(const AicArgs& a, const int* d_run_flag, cudaStream_t s);

}  // namespace fj
