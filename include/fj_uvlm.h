/*
 * fj_uvlm.h -- C ABI of libfj_uvlm.so, the B200 (sm_100a) UVLM hot path.
 *
 * The reference (FLAPJAX, src/flapjax/aero/) has no FFI layer: its hot path is a set of
 * JAX functions that uvlm.py imports by name.  Each entry point below replaces one of
 * them, with the same array layouts (C-contiguous float64, lattice zeta
 * (rows+1, cols+1, 3), circulation (rows, cols)).  The reference function replaced is
 * cited beside each declaration (paths relative to src/flapjax/).
 *
 * Conventions
 *   - Every pointer argument named d_* is DEVICE memory; everything else is host memory.
 *   - The caller owns every buffer.  No entry point allocates device memory: scratch
 *     space comes from the caller through (ws, ws_bytes), sized by the matching
 *     *_workspace_size function.
 *   - Calls are ordered on the given stream and return without synchronising, except
 *     where a function says it reads a device result back.
 *   - The return value is FJ_OK (0) or a negative FJ_ERR_* code; fj_last_error_string()
 *     (thread-local) then describes the failure.
 */
#ifndef FJ_UVLM_H
#define FJ_UVLM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define FJ_API __attribute__((visibility("default")))
#else
#define FJ_API
#endif

typedef struct CUstream_st* fj_stream_t; /* a cudaStream_t; NULL = legacy default stream */

/* status codes */
#define FJ_OK 0
#define FJ_ERR_SHAPE (-1)         /* a size/shape argument is invalid */
#define FJ_ERR_NONFINITE (-2)     /* a NaN/Inf was found where it is not allowed */
#define FJ_ERR_SINGULAR (-3)      /* exact zero pivot in a factorisation */
#define FJ_ERR_TIMEOUT (-4)       /* a bounded device wait gave up */
#define FJ_ERR_NOMEM (-5)         /* the workspace given is smaller than required */
#define FJ_ERR_CUDA (-6)          /* a CUDA runtime call failed */
#define FJ_ERR_UNSUPPORTED (-7)   /* option combination not implemented */
#define FJ_ERR_NOT_CONVERGED (-8) /* iterative refinement did not reach its tolerance */

/* Biot-Savart segment kernels, aero/utils.py:580-648 (selected by UVLM(kernel=...),
 * aero/uvlm.py:173, 280-285). */
#define FJ_KERNEL_EPSILON 0 /* biot_savart_epsilon, aero/utils.py:606-623 (default) */
#define FJ_KERNEL_CUTOFF 1  /* biot_savart_cutoff, aero/utils.py:626-648, run-time radius */
#define FJ_KERNEL_PLAIN 2   /* biot_savart, aero/utils.py:580-592 (FP64 only) */

/* arithmetic of the Biot-Savart sums and the solve */
#define FJ_PREC_FP64 0  /* plain FP64 everywhere: the reference's arithmetic */
#define FJ_PREC_MIXED 1 /* FP32 Biot-Savart with FP64 accumulation, FP32 factors + FP64 refinement */

/* background flow, aero/flowfields.py */
#define FJ_FLOW_CONSTANT 0         /* Constant, aero/flowfields.py:87-97 */
#define FJ_FLOW_ONE_MINUS_COSINE 1 /* OneMinusCosine, aero/flowfields.py:100-181 */

#define FJ_MAX_SURF 8

typedef struct fj_flowfield {
    int kind;            /* FJ_FLOW_* */
    int relative_motion; /* FlowField.relative_motion */
    double u_inf[3];
    double rho;
    double gust_length;        /* OneMinusCosine: half the full gust length */
    double gust_amplitude;
    double gust_travel_dir[3]; /* unit vectors, normalised by the caller */
    double gust_amplitude_dir[3];
    double gust_x0[3];
} fj_flowfield;

/* Everything about a UVLM case that is fixed for its lifetime: UVLM.__init__
 * (aero/uvlm.py:166-339) plus set_design_variables (:387-472) scalars. */
typedef struct fj_case_config {
    int n_surf;
    int m[FJ_MAX_SURF];      /* chordwise bound panels per surface */
    int n[FJ_MAX_SURF];      /* spanwise panels per surface */
    int m_star[FJ_MAX_SURF]; /* wake rows per surface */
    int n_nodes;             /* beam nodes in the hg arrays */
    int n_tstep;             /* time slots in the output arrays */
    int kernel;              /* FJ_KERNEL_* */
    double r_cut;            /* cutoff radius for FJ_KERNEL_CUTOFF */
    int free_wake;
    int mirror;              /* 1: image system across (mirror_point, mirror_normal) */
    double mirror_point[3];
    double mirror_normal[3]; /* unit */
    double dt;
    double gamma_dot_relaxation;
    fj_flowfield flow;
    int precision;           /* FJ_PREC_* */
    /* 1: surface s uses the variable wake discretisation (propagate_surf_wake with
     * delta_w, aero/utils.py:452-491): its segment lengths are d_delta_w's block */
    int variable_wake[FJ_MAX_SURF];
    /* polar correction (apply_polar_correction, aero/utils.py:276-397, applied as
     * uvlm.py:1055-1075): table points per strip of surface s in d_polars, 0 = none */
    int polar_points[FJ_MAX_SURF];
    /* 0..1: Gamma_b (and a static solve's Gamma_w) blended towards the polar lift scale */
    double polar_circulation_scale;
} fj_case_config;

/* Device buffers of one case.  Surfaces are concatenated in the innermost extent of
 * each time slot: field[i_ts][sum over surfaces of the per-surface block], so slot
 * i_ts of surface s is a C-contiguous block in the AeroCase layout
 * (aero/data_structures.py:43-615, AeroCase fields). */
typedef struct fj_case_buffers {
    /* inputs */
    const double* d_zeta_b0;   /* sum_s (m+1)(n+1)*3: local grid (UVLM.zeta_b0) */
    const int32_t* d_dof_mapping; /* sum_s (n+1): spanwise vertex -> beam node */
    const double* d_hg_t;      /* (n_tstep, n_nodes, 4, 4) SE(3) node frames */
    const double* d_hg_dot_t;  /* (n_tstep, n_nodes, 4, 4) their time derivatives */
    const double* d_delta_w;   /* sum_s m_star: wake segment lengths (UVLM.delta_w) of the
                                  surfaces with variable_wake set; NULL when none is */
    /* outputs, time-major (n_tstep, ...) */
    double* d_t;               /* (n_tstep,) */
    double* d_zeta_b;          /* (m+1, n+1, 3) per surface */
    double* d_zeta_b_dot;      /* (m+1, n+1, 3) */
    double* d_zeta_w;          /* (m_star+1, n+1, 3) */
    double* d_c;               /* (m, n, 3) collocation points */
    double* d_nc;              /* (m, n, 3) area normals */
    double* d_gamma_b;         /* (m, n) */
    double* d_gamma_b_dot;     /* (m, n) */
    double* d_gamma_w;         /* (m_star, n) */
    double* d_f_steady;        /* (m+1, n+1, 3) */
    double* d_f_unsteady;      /* (m+1, n+1, 3) */
    double* d_alpha;           /* (n,) strip angle of attack */
    double* d_force_total;     /* (3,) per slot: sum over vertices of f_steady+f_unsteady */
    /* polar tables of the surfaces with polar_points > 0, in surface order: per strip
     * polar_points rows of (alpha, cl, cd, cm), alpha ascending (linear interpolation,
     * end values held outside); NULL when no surface has polars */
    const double* d_polars;
} fj_case_buffers;

/* ---------------------------------------------------------------------------------
 * Library
 * ------------------------------------------------------------------------------- */
FJ_API const char* fj_last_error_string(void);
FJ_API int fj_version(void); /* major*10000 + minor*100 + patch */

/* Instrumentation (no counterpart in the reference, which has no timers beyond
 * utils/utils.py:130-175).  fj_launch_count: kernels launched by this library so far.
 * fj_profile_begin/_end bracket a region in which every Biot-Savart sum kernel is timed
 * with CUDA events on its own stream; _end waits for those events. */
typedef struct fj_profile {
    int64_t launches;      /* kernels launched in the region */
    int64_t vind_launches; /* Biot-Savart sum kernels timed */
    double vind_ms;        /* their summed device time */
    double vind_ms_max;    /* longest single launch */
    double vind_pairs;     /* (target, filament) pairs they evaluated */
    int64_t vind64_launches; /* the FP64 sums among them (the FP32 ones are the rest) */
    double vind64_ms;
    double vind64_pairs;
} fj_profile;
FJ_API int64_t fj_launch_count(void);
FJ_API int fj_profile_begin(void);
FJ_API int fj_profile_end(fj_profile* out);

/* ---------------------------------------------------------------------------------
 * Case-level entry points (replace UVLM.solve_static / solve_prescribed_dynamic /
 * case_solve, aero/uvlm.py:1119-1406).  The workspace carries cached state between
 * calls of one case (factors, streams) and must stay alive for the case's lifetime.
 * ------------------------------------------------------------------------------- */
FJ_API int fj_case_workspace_size(const fj_case_config* cfg, size_t* bytes);

/* UVLM.solve_static (aero/uvlm.py:1286-1333): writes time slot 0 of the outputs
 * (zeta_b from hg_t[0]; zeta_b_dot, gamma_b_dot, f_unsteady zero). */
FJ_API int fj_solve_static(const fj_case_config* cfg, const fj_case_buffers* bufs, int horseshoe,
                    double t0, void* d_ws, size_t ws_bytes, fj_stream_t stream);

/* UVLM.solve_prescribed_dynamic (aero/uvlm.py:1335-1406): time steps
 * i_first..i_last-1 (1 <= i_first), each a case_solve (aero/uvlm.py:1119-1215) reading
 * slot i-1 and writing slot i.  Slot i_first-1 must hold a solution (e.g. from
 * fj_solve_static).
 * FJ_PREC_MIXED: the FP32 factors are computed at step i_first, unless flags has
 * FJ_REUSE_FACTORS and an earlier call on this workspace left factors there; the
 * refinement residuals are read back after the last step (one synchronisation) and
 * the steps from the first one above 1e-12 are re-run with fresh factors.
 * Runs of three or more steps that reuse their factors (FP64: every step after the
 * first) are replayed from one CUDA graph captured for a single step; FJ_NO_GRAPH
 * launches every step directly instead (same arithmetic).
 * fj_solve_static and fj_solve_prescribed_dynamic synchronise the stream before
 * returning and scan their slots: FJ_ERR_NONFINITE names the first slot whose total
 * force is NaN/Inf (a NaN anywhere in the step reaches it), FJ_ERR_SINGULAR an exact
 * zero pivot of the last factorisation. */
#define FJ_REUSE_FACTORS 1
#define FJ_NO_GRAPH 2
/* Fluid-structure iterations re-solve one slot i with new frames hg_t[i] but the same
 * converged slot i-1.  The free-wake convection velocity (aero/uvlm.py:912-941) depends
 * only on slot i-1 and hg_t[i-1], so with FJ_REUSE_CONVECTION the first step of the call
 * takes the velocities the previous call on this workspace computed for that slot instead
 * of recomputing them (the caller guarantees slot i-1 and hg_t[i-1] are unchanged). */
#define FJ_REUSE_CONVECTION 4
FJ_API int fj_solve_prescribed_dynamic(const fj_case_config* cfg, const fj_case_buffers* bufs,
                                int i_first, int i_last, int flags, void* d_ws,
                                size_t ws_bytes, fj_stream_t stream);

/* One case_solve (aero/uvlm.py:1119-1215) at slot i_ts >= 1 with the node frames of
 * slots i_ts (hg_n, hg_dot_n) and i_ts-1 (hg_nm1) taken from the hg arrays.  This is
 * the call the coupled FSI loop makes (structure/beam.py:2656-2667). */
FJ_API int fj_case_step(const fj_case_config* cfg, const fj_case_buffers* bufs, int i_ts,
                 int flags, void* d_ws, size_t ws_bytes, fj_stream_t stream);

/* One time step for each of many cases in one set of kernel launches (the serving
 * path).  Each item is a case (its config, buffers and own workspace) and the slot it
 * solves; the step is case_solve (aero/uvlm.py:1119-1215) with the node frames of slots
 * i_ts and i_ts-1 of the case's hg arrays.  All items must share precision, kernel and
 * cutoff radius.  FJ_PREC_MIXED items reuse the factors cached in their workspace when
 * flags has FJ_REUSE_FACTORS, else factorise at this step.  Does not synchronise: the
 * refinement residual of a slot is read with fj_case_residual. */
typedef struct fj_batch_item {
    const fj_case_config* cfg;
    const fj_case_buffers* bufs;
    void* d_ws;
    size_t ws_bytes;
    int i_ts;
    int flags;
} fj_batch_item;
FJ_API int fj_batch_workspace_size(int max_items, size_t* bytes);
/* Unless an item has FJ_NO_GRAPH or factorises (no FJ_REUSE_FACTORS), the step runs as a
 * CUDA graph captured on the first call for its batch workspace and replayed by later calls
 * whose batch has the same launch signature: the same number of cases, the same grid
 * maxima and the same sum-job counts (the per-case data travel in the uploaded table; the
 * Biot-Savart sums are persistent kernels whose grid is fixed).  A different signature
 * re-captures.  Calls that share a batch workspace must not overlap. */
FJ_API int fj_step_batched(const fj_batch_item* items, int n_items, void* d_batch_ws,
                           size_t batch_ws_bytes, fj_stream_t stream);
/* Drops the captured graph held for a batch workspace (call before freeing it). */
FJ_API int fj_batch_release(void* d_batch_ws);
/* Replays and captures of batched-step graphs since the library was loaded. */
FJ_API int fj_batch_graph_stats(int64_t* replays, int64_t* captures);
/* Relative refinement residual of slot i_ts of a mixed-precision case (synchronises). */
FJ_API int fj_case_residual(const fj_case_config* cfg, void* d_ws, size_t ws_bytes, int i_ts,
                            double* h_out, fj_stream_t stream);

/* Copies the getrf factors (row-major L\U, n x n) and 0-based pivots of the AIC that the
 * last dynamic step of an FP64 case solved with, into caller buffers (stream-ordered).
 * The adjoint keeps them per step to solve A^T mu = lam with fj_lu_solve_t instead of
 * re-assembling and re-factorising; the reference has no counterpart (jax.vjp through
 * jnp.linalg.solve recomputes, aero/uvlm.py:985). */
FJ_API int fj_case_factors_copy(const fj_case_config* cfg, const void* d_ws, size_t ws_bytes, double* d_lu,
                                int32_t* d_piv, fj_stream_t stream);

/* Measured FP32 FMA throughput of the current device (TFLOP/s, an FMA counted as two):
 * the larger of a scalar and a packed (f32x2) register-resident FMA-chain kernel, timed
 * with CUDA events.  Synchronises. */
FJ_API int fj_peak_fp32(double* tflops, fj_stream_t stream);

/* ---------------------------------------------------------------------------------
 * Function-level entry points (the names uvlm.py imports, aero/uvlm.py:15, :32-43).
 * ------------------------------------------------------------------------------- */

/* biot_savart_epsilon / biot_savart_cutoff / biot_savart (aero/utils.py:580-648)
 * evaluated pairwise: d_x (n_pairs, 3), d_y (n_pairs, 2, 3) -> d_out (n_pairs, 3). */
FJ_API int fj_biot_savart(const double* d_x, const double* d_y, int64_t n_pairs, int kernel,
                   double r_cut, double* d_out, fj_stream_t stream);

/* compute_v_ind (aero/aic.py:248-310): induced velocity at n_targets points of the
 * lattices d_zetas[i] ((rows[i]+1, cols[i]+1, 3)) with ring circulations d_gammas[i]
 * ((rows[i], cols[i])), minus their images when mirror_point != NULL.  d_zetas and
 * d_gammas are HOST arrays of device pointers. */
FJ_API int fj_vind_workspace_size(int64_t n_targets, const int* rows, const int* cols,
                           int n_lattices, int mirror, int precision, size_t* bytes);
FJ_API int fj_vind(const double* d_targets, int64_t n_targets, const double* const* d_zetas,
            const double* const* d_gammas, const int* rows, const int* cols, int n_lattices,
            const double* mirror_point, const double* mirror_normal, int kernel, double r_cut,
            int precision, double* d_v_out, void* d_ws, size_t ws_bytes, fj_stream_t stream);

/* Adjoint of compute_v_ind (the reference differentiates it with jax.vjp): given the
 * cotangent d_lam (n_targets, 3) of the velocities, ACCUMULATES (+=) into d_targets_bar
 * (n_targets, 3), d_zetas_bar[i] (vertex adjoints of lattice i) and d_gammas_bar[i]
 * (ring-circulation adjoints); any of the three may be NULL to skip it.  FP64, epsilon
 * kernel only. */
FJ_API int fj_vind_vjp_workspace_size(int64_t n_targets, const int* rows, const int* cols,
                                      int n_lattices, int mirror, size_t* bytes);
FJ_API int fj_vind_vjp(const double* d_targets, int64_t n_targets, const double* const* d_zetas,
                       const double* const* d_gammas, const int* rows, const int* cols,
                       int n_lattices, const double* mirror_point, const double* mirror_normal,
                       int kernel, double r_cut, const double* d_lam, double* d_targets_bar,
                       double* const* d_zetas_bar, double* const* d_gammas_bar, void* d_ws,
                       size_t ws_bytes, fj_stream_t stream);

/* Dense influence Jacobians of compute_v_ind (aero/aic.py:248-310) for one source lattice
 * zeta (rows+1, cols+1, 3), for the linearised UVLM (aero/linear/linear_uvlm.py forms its
 * state-space matrices by jax.jacrev of one step).  FP64, epsilon or cutoff kernel, the
 * mirror image subtracted when mirror_point/mirror_normal are given.  Each writes a
 * row-major block with leading dimension ld_out (overwritten, not accumulated):
 *   fj_ring_influence:  d v(x_t) / d gamma_r, the velocity of unit circulation on ring
 *     r = k*cols + l;  (n_targets, ld_out) projected on d_normals (n_targets, 3) when given,
 *     else (3 n_targets, ld_out) with rows t*3 + {x, y, z};  ld_out >= rows*cols.
 *   fj_vertex_jacobian: d v(x_t) / d zeta_v for circulations d_gamma (rows, cols), column
 *     v*3 + {x, y, z} for vertex v = k*(cols+1) + l;  rows as above;  ld_out >= 3 vertices. */
FJ_API int fj_ring_influence(const double* d_targets, int64_t n_targets, const double* d_normals,
                             const double* d_zeta, int rows, int cols, const double* mirror_point,
                             const double* mirror_normal, int kernel, double r_cut, double* d_out,
                             int64_t ld_out, fj_stream_t stream);
FJ_API int fj_vertex_jacobian(const double* d_targets, int64_t n_targets, const double* d_normals,
                              const double* d_zeta, const double* d_gamma, int rows, int cols,
                              const double* mirror_point, const double* mirror_normal, int kernel,
                              double r_cut, double* d_out, int64_t ld_out, fj_stream_t stream);

/* B <- A^-1 B for nrhs right-hand sides, the columns of the row-major (n, ldb) d_b, from the
 * factors of fj_lu_factor (jax.scipy.linalg.lu_solve / jnp.linalg.solve with a matrix
 * right-hand side, as the linear model's Jacobians need). */
FJ_API int fj_lu_solve_many_workspace_size(int n, int64_t nrhs, size_t* bytes);
FJ_API int fj_lu_solve_many(const double* d_lu, int n, const int32_t* d_piv, double* d_b, int64_t nrhs,
                            int64_t ldb, void* d_ws, size_t ws_bytes, fj_stream_t stream);

/* The state march of LinearSystem.run (utils/linear.py:775-822): for i = 1 .. n_tstep-1,
 * x_i = A x_{i-1} + bu_{i-shift}, with A (n, n) row-major, the input terms bu (n_tstep rows
 * of leading dimension ld_bu, bu_i = B u_i) and x (n_tstep, n) whose row 0 holds x_0.
 * shift = 1 after remove_u_np1 (the system takes the input of step i-1), else 0.  One
 * GEMV-with-add launch per step on the caller's stream; FP64. */
FJ_API int fj_lti_march(const double* d_a, int n, const double* d_bu, int64_t ld_bu, double* d_x,
                        int64_t n_tstep, int shift, fj_stream_t stream);

/* fj_vind without a caller workspace, for callers that cannot allocate device memory
 * (a plugin host that owns the device memory pool, a real-time loop that may not block in
 * cudaMalloc).  No counterpart in the reference.  Its scratch is a fixed 8 MiB array in
 * the library's device memory, reserved on every GPU that loads the library; sizes whose
 * filament stream plus one set of partial velocities exceed it are refused with
 * FJ_ERR_SHAPE.  The first call on a device looks the array up (cudaGetSymbolAddress) and
 * should come before any stream capture; the address it keeps does not survive a
 * cudaDeviceReset of that device.  All calls share the array: calls that overlap on the
 * GPU (other streams, other host threads) race and must be serialised. */
FJ_API int fj_vind_noalloc(const double* d_targets, int64_t n_targets, const double* const* d_zetas,
                           const double* const* d_gammas, const int* rows, const int* cols,
                           int n_lattices, const double* mirror_point, const double* mirror_normal,
                           int kernel, double r_cut, int precision, double* d_v_out,
                           fj_stream_t stream);

/* compute_aic_solve (aero/aic.py:137-187): the (sum m*n)^2 row-major AIC of the bound
 * lattices at their own collocation points, projected on the area normals.  When
 * d_zetas_w != NULL (static solve) each surface's wake influence is lumped onto its
 * trailing-edge column (add_wake_influence, aero/aic.py:190-205). */
FJ_API int fj_aic_assemble(const double* const* d_zetas_b, const int* m, const int* n, int n_surf,
                    const double* const* d_zetas_w, const int* m_star,
                    const double* mirror_point, const double* mirror_normal, int kernel,
                    double r_cut, double* d_aic, void* d_ws, size_t ws_bytes,
                    fj_stream_t stream);
FJ_API int fj_aic_workspace_size(const int* m, const int* n, int n_surf, size_t* bytes);

/* jnp.linalg.solve (aero/uvlm.py:985) split as LAPACK getrf/getrs, row-major A.
 * fj_lu_factor overwrites d_a with L\U and writes 0-based pivot rows to d_piv (n). */
FJ_API int fj_lu_workspace_size(int n, size_t* bytes);
FJ_API int fj_lu_factor(double* d_a, int n, int32_t* d_piv, void* d_ws, size_t ws_bytes,
                 fj_stream_t stream);
FJ_API int fj_lu_solve(const double* d_lu, int n, const int32_t* d_piv, double* d_b, void* d_ws,
                size_t ws_bytes, fj_stream_t stream);

/* Transpose solve A^T x = b with the factors of fj_lu_factor (the adjoint of the solve at
 * aero/uvlm.py:985); workspace as fj_lu_workspace_size. */
FJ_API int fj_lu_solve_t(const double* d_lu, int n, const int32_t* d_piv, double* d_b, void* d_ws,
                         size_t ws_bytes, fj_stream_t stream);

/* ---- One surface's pieces of a step, as the reference calls them separately ---------
 * Right-hand side of the dynamic solve, aero/uvlm.py:961-983: b_i = -(v_bc_i . nc_i) with
 * v_bc = U(c, t) - c_dot + v_ind(c; wake lattices) -- the vector the reference passes to
 * jnp.linalg.solve(aic, -rhs).  The static solve is n_wake = 0 and d_c_dot = NULL. */
FJ_API int fj_rhs_workspace_size(int64_t n_pan, const int* rows_w, const int* cols_w, int n_wake,
                                 int mirror, int precision, size_t* bytes);
FJ_API int fj_rhs(const double* d_c, const double* d_nc, const double* d_c_dot, int64_t n_pan,
                  const fj_flowfield* flow, double t, const double* const* d_zetas_w,
                  const double* const* d_gammas_w, const int* rows_w, const int* cols_w, int n_wake,
                  const double* mirror_point, const double* mirror_normal, int kernel, double r_cut,
                  int precision, double* d_b, void* d_ws, size_t ws_bytes, fj_stream_t stream);

/* propagate_surf_wake, uniform branch (aero/utils.py:400-450): zeta_w_n (m_star+1, n+1, 3)
 * = [TE row of zeta_b_n; zeta_w_nm1[:-1] + dt (U(x, t) + v_conv)] and gamma_w_n (m_star, n)
 * = [TE row of gamma_b_nm1; gamma_w_nm1[:-1]].  d_v_conv (m_star, n+1, 3): the free-wake
 * induced velocity at zeta_w_nm1[:-1] (fj_vind over the lattices of step n-1), or NULL
 * for a prescribed wake. */
FJ_API int fj_wake_shed_convect(const double* d_zeta_te_n, const double* d_gamma_te_nm1,
                                const double* d_zeta_w_nm1, const double* d_gamma_w_nm1,
                                const double* d_v_conv, int n, int m_star, const fj_flowfield* flow,
                                double t, double dt, double* d_zeta_w_n, double* d_gamma_w_n,
                                fj_stream_t stream);

/* calculate_steady_forcing (aero/utils.py:126-223) of one lattice zeta_b (m+1, n+1, 3):
 * per filament rho G_eff (v_rel x r) at its midpoint, v_rel = U + v_ind(midpoint; the
 * given lattices, normally bound + wake) - zeta_b_dot (averaged), the TE spanwise
 * filament less gamma_w[0] (d_gamma_w0, n values, or NULL), split to the vertices; and
 * with d_gamma_b_dot the unsteady force split_to_vertex(rho gamma_dot nc)
 * (aero/uvlm.py:1086-1103) into d_f_unsteady (or NULL to skip). */
FJ_API int fj_forces_workspace_size(int m, int n, const int* rows, const int* cols, int n_lat,
                                    int mirror, int precision, size_t* bytes);
FJ_API int fj_forces(const double* d_zeta_b, const double* d_zeta_b_dot, const double* d_gamma_b,
                     const double* d_gamma_w0, const double* d_gamma_b_dot, int m, int n,
                     const fj_flowfield* flow, double t, const double* const* d_zetas,
                     const double* const* d_gammas, const int* rows, const int* cols, int n_lat,
                     const double* mirror_point, const double* mirror_normal, int kernel, double r_cut,
                     int precision, double* d_f_steady, double* d_f_unsteady, void* d_ws, size_t ws_bytes,
                     fj_stream_t stream);

/* Adjoint twin of the AIC (compute_aic_solve, aero/aic.py:11-187; the reference
 * differentiates it with jax.vjp): ACCUMULATES into d_zeta_bar (m+1, n+1, 3) the lattice
 * cotangent of s = mu^T A(zeta) Gamma for one surface's bound AIC (epsilon kernel, no
 * mirror), through the filaments, the collocation points and the normals. */
FJ_API int fj_aic_vjp_workspace_size(int m, int n, size_t* bytes);
FJ_API int fj_aic_vjp(const double* d_zeta, int m, int n, const double* d_gamma, const double* d_mu,
                      int kernel, double* d_zeta_bar, void* d_ws, size_t ws_bytes, fj_stream_t stream);

/* Adjoint twin of the prescribed wake shift (aero/utils.py:427-450): given the cotangents
 * of zeta_w_n and gamma_w_n, ACCUMULATES row 0 into the TE cotangents (of zeta_b_n's last
 * row and gamma_b_nm1's last row) and rows 1.. into the cotangents of zeta_w_nm1[:-1] and
 * gamma_w_nm1[:-1].  Any output may be NULL. */
FJ_API int fj_wake_vjp(const double* d_zeta_w_bar_n, const double* d_gamma_w_bar_n, int n, int m_star,
                       double* d_zeta_te_bar, double* d_gamma_te_bar, double* d_zeta_w_bar_nm1,
                       double* d_gamma_w_bar_nm1, fj_stream_t stream);

/* Mixed-precision solve of A x = b (jnp.linalg.solve, aero/uvlm.py:985): FP32 factors
 * of A and the FP32 inverse M (recomputed when refactor != 0) kept in the workspace, then
 * FP64 iterative refinement x += M (b - A x) with the FP64 residual.  Writes the final
 * relative residual ||b-Ax||_inf / ||b||_inf to *d_resid (device, 1 double).  From
 * n = 256 the factorisation's and the inverse's products run on the tensor cores
 * (fj_gemm_tf32, three-pass split); the environment variable FJ_MIXED_FACTOR = "cuda" |
 * "tf32" | "tf32x3" selects the FP32 CUDA-core path, a single TF32 pass or the default. */
FJ_API int fj_solve_mixed_workspace_size(int n, size_t* bytes);
FJ_API int fj_solve_mixed(const double* d_a, int n, const double* d_b, double* d_x, int refactor,
                   double* d_resid, void* d_ws, size_t ws_bytes, fj_stream_t stream);

/* C <- alpha A B + beta C on the tensor cores (tcgen05, TF32 operands, FP32 accumulation
 * in tensor memory): A (m x k, lda), B (k x n, ldb), C (m x n, ldc), row-major FP32
 * device arrays.  passes = 1 multiplies the TF32-rounded operands; passes = 3 adds the
 * products with the operands' rounding remainders (hi*hi + hi*lo + lo*hi), close to
 * FP32 accuracy.  beta = 0 does not read C.  *d_err (device int) is set to 1 if a bounded
 * device wait expired.  The product building block of the mixed factorisation (the
 * reference's solve runs inside jnp.linalg.solve, aero/uvlm.py:985). */
FJ_API int fj_gemm_tf32(const float* d_a, int lda, const float* d_b, int ldb, float* d_c, int ldc, int m, int n,
                        int k, float alpha, float beta, int passes, int* d_err, fj_stream_t stream);

/* The same product through the factorisation's TMA pipeline: the operands are first
 * split into TF32 hi/lo copies in d_scratch (K-major, fj_gemm_tf32_scratch_floats
 * floats, 16-byte aligned), which cp.async.bulk.tensor loads feed to the MMAs through a
 * three-stage mbarrier ring (a producer thread apart from the MMA issuer).  C may alias
 * A or B. */
FJ_API int fj_gemm_tf32_scratch_floats(int m, int n, int k, int passes, size_t* floats);
FJ_API int fj_gemm_tf32_tma(const float* d_a, int lda, const float* d_b, int ldb, float* d_c, int ldc, int m,
                            int n, int k, float alpha, float beta, int passes, float* d_scratch,
                            size_t scratch_floats, int* d_err, fj_stream_t stream);

/* Failure-detection self-test of the tensor-core kernel's bounded waits: launches
 * fj_gemm_tf32's kernel with its MMAs and commits withheld, so that the mbarrier it waits
 * on never completes.  After about two seconds (the wait and a bounded drain) the kernel
 * has set *d_err (device int) to 1, freed its tensor memory and returned; the context
 * stays usable.  d_scratch: 4 device floats. */
FJ_API int fj_tc_wait_selftest(int* d_err, float* d_scratch, fj_stream_t stream);

/* Autotuner of the Biot-Savart sum launches (the reference's vmap/lax.map chunking,
 * aero/aic.py:47-63, 237-245, has no tunable).  A sum of n_targets points over a stream of
 * n_elem filament elements runs as target tiles x splits CTAs; for each shape this times
 * the sum and its reduction at candidate split counts on a synthetic lattice of that
 * stream length (CUDA events; synchronises) and publishes the fastest into a new
 * immutable table, by precision, log2 n_targets and log2 stream length, that every later
 * launch consults.  Per shape it reports the split chosen, the rule's split and both
 * times (ms); any of those arrays may be NULL.  precision: FJ_PREC_FP64 or
 * FJ_PREC_MIXED (the FP32 sums).  The FP32 sums are also tried with four targets per
 * thread instead of two (the tile shape): chosen[i] is then the split plus 4096 when the
 * four-target tile won. */
FJ_API int fj_autotune_vind_workspace_size(int precision, const int64_t* n_targets, const int64_t* n_elem,
                                           int n_shapes, size_t* bytes);
FJ_API int fj_autotune_vind(int precision, int kernel, double r_cut, const int64_t* n_targets,
                            const int64_t* n_elem, int n_shapes, int* chosen, int* heuristic, double* chosen_ms,
                            double* heuristic_ms, void* d_ws, size_t ws_bytes, fj_stream_t stream);
/* The published table as int16 entries (fj_autotune_table_size of them; 0 = not tuned),
 * to save it and load it into another process; fj_autotune_set(NULL, 0) drops it.  The
 * first half is the FP64 sums' split counts (1..1024), the second the FP32 sums', each
 * plus 4096 where four targets per thread won; fj_autotune_set refuses anything else. */
FJ_API int fj_autotune_table_size(int* n_entries);
FJ_API int fj_autotune_get(int16_t* entries, int n_entries);
FJ_API int fj_autotune_set(const int16_t* entries, int n_entries);

#ifdef __cplusplus
}
#endif
#endif /* FJ_UVLM_H */
