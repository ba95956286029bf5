/*
 * nfgs_b200.h - C ABI of the B200-native NFGS (Gaussian-separated NFPT)
 * reconstruction library (libnfgs_b200.so).
 *
 * The reference exposes this path as the Python class NFGSSolverGPU
 * (nfgs_solver.py:3905 in spaceprod/NFGS).  Each entry point below replaces
 * one method of that class; the citation beside it names the reference
 * method.  Plain C types only: host pointers for host data, no torch types,
 * no C++ exceptions across the boundary.  Every call returns an NFGS_*
 * status; nfgs_last_error() gives a message for the calling thread.
 *
 * Threading: a handle is used by one host thread at a time.  Each handle
 * owns a CUDA stream on the device that was current at nfgs_create().
 */
#ifndef NFGS_B200_H
#define NFGS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define NFGS_OK 0
#define NFGS_EINVAL 1         /* invalid argument (ValueError in the reference) */
#define NFGS_ECUDA 2          /* CUDA runtime error */
#define NFGS_ENOMEM 3         /* device allocation failed */
#define NFGS_ESTATE 4         /* wrong call order (RuntimeError in the reference) */
#define NFGS_EPOLICY 5        /* zero-mode / harmonic policy violation (ValueError) */
#define NFGS_ETIMEDOUT 6      /* a bounded device wait ran out */
#define NFGS_EUNSUPPORTED 7   /* option outside the production NFGS branch */

/* storage types */
#define NFGS_F32 0
#define NFGS_F64 1

/* enumerations of reference string options */
#define NFGS_HZM_OMIT 0                    /* horizontal_zero_mode_policy="omit" */
#define NFGS_HZM_FROZEN_LINEAR_HARMONIC 1  /* "frozen_linear_harmonic" (default) */
#define NFGS_HZM_COUPLED_K0 2              /* "coupled_k0" (nfgs_solver.py:5058-5431) */
#define NFGS_HZM_CONSTRAINED_SPLINE 3      /* "constrained_spline_harmonic" (nfgs_solver.py:5099-5260) */
#define NFGS_MEANBZ_UNIFORM_OPEN 0
#define NFGS_MEANBZ_REQUIRE_BALANCED 1
#define NFGS_MEANBZ_USER_SUPPLIED 2
#define NFGS_POLICY_ERROR 0                /* zero-mode policies */
#define NFGS_POLICY_WARN_PROJECT 1
#define NFGS_POLICY_PROJECT 2
#define NFGS_HARM_DIAGNOSE 0               /* harmonic_residual_policy */
#define NFGS_HARM_WARN 1
#define NFGS_HARM_ERROR 2
#define NFGS_POLARITY_BOTH 0
#define NFGS_POLARITY_POSITIVE 1
#define NFGS_POLARITY_NEGATIVE 2
#define NFGS_JZ_DERIVE_LEGACY_HELPER 0     /* bottom_current_grid_mode="legacy_helper" */
#define NFGS_JZ_DERIVE_CALC_GRID 1         /* "calculation_grid" */
#define NFGS_JZ_PROVIDED 2                 /* "provided" */

/* stop reasons (history["stop_reason"]) */
#define NFGS_STOP_RUNNING 0
#define NFGS_STOP_MAX_ITER 1
#define NFGS_STOP_TOL 2
#define NFGS_STOP_SIGMA_IMPROVEMENT 3
#define NFGS_STOP_SIGMA_STALL 4
#define NFGS_STOP_MAX_ROLLBACKS 5
#define NFGS_STOP_POLICY_ERROR 6
#define NFGS_STOP_FIXED_POINT 7

/* Calculation grid and observed field of view (host-computed sizing,
 * nfgs_solver.py:771-819). */
typedef struct NfgsGeom {
    int32_t nx, ny, nz;          /* calculation grid */
    double dx, dy, dz;
    int32_t input_nx, input_ny, input_nz; /* constructor grid */
    int32_t pad_x, pad_y;        /* calculation_pad_xy */
    int32_t dtype;               /* NFGS_F32 or NFGS_F64 */
    int32_t device;              /* CUDA device ordinal */
} NfgsGeom;

/* NFGS policy (constructor keywords, nfgs_solver.py:3925-4349). */
typedef struct NfgsParams {
    double robin_weight;           /* bottom_divergence_robin_weight (rho) */
    double projection_weight;      /* bottom_divergence_projection_weight */
    double alpha_max;              /* alpha clip bound 1/h * factor; <= 0 disables */
    double weak_field_floor_b2;
    double mean_mode_tolerance;
    double source_zero_mode_tolerance;
    double user_open_bz;           /* user_supplied_open_bz (MEANBZ_USER_SUPPLIED) */
    int32_t horizontal_zero_mode;  /* NFGS_HZM_* */
    int32_t mean_bz_policy;        /* NFGS_MEANBZ_* */
    int32_t d0_policy;             /* NFGS_POLICY_* */
    int32_t source_policy;         /* NFGS_POLICY_* */
    int32_t harmonic_policy;       /* NFGS_HARM_* */
    int32_t gaussian_spectral;     /* 1: "spectral", 0: "fd" */
    int32_t face_parallel_exact_jz;/* bottom_parallel_current_mode */
    int32_t buffer_thickness;      /* 0: no window */
    int32_t buffer_xy_only;
    /* k_h=0 closures (NFGS_HZM_COUPLED_K0, NFGS_HZM_CONSTRAINED_SPLINE) */
    double k0_smoothness;          /* k0_ode_smoothness (>= 0) */
    double k0_update_mu;           /* k0_update_mu in (0, 1]; <= 0: the step's scalar mu */
    int32_t k0_spline_basis;       /* k0_spline_basis_size (4 <= n <= nz) */
    int32_t k0_legacy;             /* coupled_k0_discretization="legacy_plane_centred" */
    int32_t k0_face_target;        /* k0_current_target_placement="face" */
    int32_t k0_reserved;
} NfgsParams;

/* set_bottom_vector_boundary keywords (nfgs_solver.py:4661, 2000-2113). */
typedef struct NfgsBoundaryOpts {
    int32_t ny_obs, nx_obs;   /* shape of the supplied maps */
    int32_t zero_net_current;
    int32_t smooth_passes;
    int32_t ijzbcor;
    int32_t jz_mode;          /* NFGS_JZ_* */
    int32_t nzo;              /* observed height (fields crop and sigma box) */
    int32_t fov_y0, fov_x0;   /* placement of the observed maps in the calc grid */
    int32_t src_y0, src_x0;   /* first copied row/column of the maps (crop) */
    int32_t copy_ny, copy_nx; /* copied extent */
} NfgsBoundaryOpts;

/* Number of doubles nfgs_set_boundary() writes to diag_out. */
#define NFGS_NDIAG 40

/* iterate() stop rule (nfgs_solver.py:3522-3562). */
typedef struct NfgsStop {
    int32_t max_iter;
    int32_t patience;
    double tol;
    double mu;
    double sigma_improvement_tol;  /* <= 0 disables */
    int32_t polarity_mask;         /* NFGS_POLARITY_* */
    int32_t adaptive_mu;
    double mu_min, mu_max, mu_backoff, mu_growth;
    int32_t growth_streak;
    int32_t max_rollbacks;
    double divergence_factor;
    int32_t check_every;           /* iterations per host status poll (>= 1) */
    int32_t use_graph;             /* capture the per-iteration launches in a CUDA graph */
} NfgsStop;

/* Number of doubles per history row written by nfgs_iterate_end(). */
#define NFGS_HIST_COLS 8
/* columns: sigma, divB, energy, mu, rollback, sigma_rel_change,
 *          energy_rel_change, source_zero_mode_ratio */

typedef struct NfgsIterResult {
    int32_t n_hist;          /* rows written to hist */
    int32_t best_iter;
    int32_t final_iter;
    int32_t stop_reason;     /* NFGS_STOP_* */
    int32_t rollbacks;
    int32_t kernel_launches; /* kernels this library launched in the call */
    double best_sigma;
    double final_sigma;
    double final_vs_best_B_relative;
    double sigma0, divB0, energy0;
    double last_sigma_improvement; /* NaN when no step was accepted */
    double init_source_zero_mode_ratio;
    double device_ms;        /* CUDA-event time of the whole iterate call */
} NfgsIterResult;

/* NFGSSolverGPU.__init__ (nfgs_solver.py:3925-4349 -> 736-937):
 * validates the geometry, allocates every device buffer for the grid. */
int nfgs_create(const NfgsGeom* geom, const NfgsParams* params, void** handle_out);

/* NFGSSolverGPU.set_bottom_vector_boundary / set_bottom_boundary
 * (nfgs_solver.py:4661, 4548-4596): host maps (row-major ny_obs x nx_obs,
 * FP64) are copied to the device, embedded, bottom Jz is derived (or jz is
 * used when jz_mode == NFGS_JZ_PROVIDED), the toroidal boundary and the
 * Gaussian separation (nfgs_solver.py:4671-4919) are built on the device.
 * diag_out (NFGS_NDIAG doubles, may be NULL) receives the separation
 * diagnostics in the order documented in nfgs_b200/solver.py. */
int nfgs_set_boundary(void* handle, const double* bx, const double* by, const double* bz,
                      const double* jz, const NfgsBoundaryOpts* opts, double* diag_out);

/* NFGSSolverGPU.iterate, split so that a per-step host callback can run
 * between steps (nfgs_solver.py:6937 -> 3522-3850):
 *   begin   - gs_cfcf initial state (nfgs_solver.py:6613-6645) and its sigma;
 *   advance - up to max_steps NFPT iterations on the device (no host sync
 *             inside), returns the stop reason (NFGS_STOP_RUNNING if none);
 *   end     - selects the best-sigma state, fills the result and history. */
int nfgs_iterate_begin(void* handle, const NfgsStop* stop);
/* sigma, divB, energy of the initial state after nfgs_iterate_begin()
 * (the "Initial" line of verbose iterate, nfgs_solver.py:3612-3622). */
int nfgs_iterate_initial(void* handle, double* scalars3);
int nfgs_iterate_advance(void* handle, int32_t max_steps, int32_t* stop_reason, int32_t* n_done);
int nfgs_iterate_end(void* handle, NfgsIterResult* result, double* hist, int32_t hist_rows);

/* History rows [first, first + n) written so far by the running iterate
 * (for verbose printing and per-step callbacks); returns the row count
 * in *n_total. */
int nfgs_get_history(void* handle, int32_t first, int32_t n, double* out, int32_t* n_total);

/* Convenience: begin + advance until stopped + end. */
int nfgs_iterate(void* handle, const NfgsStop* stop, NfgsIterResult* result, double* hist,
                 int32_t hist_rows);

/* NFGSSolverGPU.fields_to_numpy (nfgs_solver.py:2881-2903).
 * which: 0 = stored solution (best state after iterate), 1 = current state.
 * out: 6 consecutive (nz_out, ny_out, nx_out) FP64 blocks Bx,By,Bz,Jx,Jy,Jz;
 * crop != 0 crops to the observed field of view. dims_out (3 ints) gets
 * the output shape. */
int nfgs_fields(void* handle, int32_t which, int32_t crop, double* out, int32_t* dims_out);

/* NFGSSolverGPU.fields_to_numpy (nfgs_solver.py:2881-2903) in the dtype the
 * reference returns there (the solver dtype, `B[0].cpu().numpy()`):
 * as nfgs_fields, with out holding 6 blocks of out_dtype (NFGS_F32 or
 * NFGS_F64) in host memory of any kind.  The gather buffer on the device is
 * kept by the handle between calls; the copy to the host goes through two
 * pinned 32 MB chunks. */
int nfgs_fields_into(void* handle, int32_t which, int32_t crop, void* out, int32_t out_dtype, int32_t* dims_out);

/* The same six fields gathered into caller-owned DEVICE memory (no host
 * copy), for evaluation on the GPU: out_dev holds 6 * nz_out * ny_out *
 * nx_out values of out_dtype.  out_dev == NULL only reports dims_out.
 * Returns after the gather has been queued on the solver's stream and that
 * stream has completed it. */
int nfgs_fields_device(void* handle, int32_t which, int32_t crop, void* out_dev, int32_t out_dtype, int32_t* dims_out);

/* Single-step access used by parity tests and by per_step_callback:
 * reconstructs the state of `which` and returns phi_c, A_z (FP64, full
 * calc grid), and its sigma/divB/energy. */
int nfgs_get_scalars_state(void* handle, int32_t which, double* phi, double* az, double* scalars3);

/* One NFPT step from the current state with relaxation mu (no stop logic),
 * nfgs_solver.py:6647-6935.  The new state becomes current. */
int nfgs_step(void* handle, double mu, int32_t polarity_mask);

/* NFGSSolverGPU.gaussian_above_bottom_field (nfgs_solver.py:4921-4946):
 * out is (3, ny, nx) FP64. */
int nfgs_gaussian_above(void* handle, double* out);

/* Allocation-free variant of nfgs_gaussian_above; no counterpart in the
 * reference.  For callers that cannot allocate device memory while they
 * run: applications whose own pool allocator holds the free HBM, and
 * applications sharing the GPU with latency-critical work (cudaMalloc and
 * cudaFree synchronise the device).  The handle must have been created and
 * given a boundary beforehand.  Writes (3, ny, nx) FP64 to the caller's
 * device buffer out_dev, enqueued on `stream` (a cudaStream_t; NULL is the
 * default stream) without synchronising; scratch comes from one static
 * 16 MiB device array that this library reserves on every GPU it loads on,
 * so the calculation plane may hold at most 419,430 cells (NFGS_EINVAL
 * beyond that).  Every call looks the array's device address up on the
 * handle's device (so a device reset leaves no stale address behind); the
 * first call on a device also loads the module, and should come before any
 * stream capture.  The call is ordered after the work already queued on the
 * handle's own stream, and a later nfgs_set_boundary or nfgs_destroy of the
 * handle waits for it to finish.  The caller's current device is restored on
 * return.  All calls share the array: calls that overlap on the GPU race. */
int nfgs_gaussian_above_noalloc(void* handle, double* out_dev, void* stream);

/* Fixed 2-D products of the boundary set-up (FP64, calc grid, (ny, nx)):
 * which = 0 Bz_obs, 1 Bx_obs, 2 By_obs, 3 Jz_obs, 4 Az_bottom, 5 Jz_T,
 * 6 Phi_above_bottom, 7 Bz_above, 8 D0, 9 bottom_dphi_c_target. */
int nfgs_get_plane(void* handle, int32_t which, double* out);

/* B_background volume (3, nz, ny, nx), FP64. */
int nfgs_get_background(void* handle, double* out);

/* Post-solve source diagnostics (nfgs_solver.py:7014-7196), scalar keys in
 * the order documented in nfgs_b200/solver.py (NFGS_NSRCDIAG doubles). */
#define NFGS_NSRCDIAG 12
int nfgs_source_diagnostics(void* handle, double* out);

/* Per-phase device time of n_iters NFPT iterations from the current
 * state (no stop rule), CUDA events on the handle's stream.  ms_out[5]:
 * 0 stencil passes (reconstruction, face current, sources, reductions),
 * 1 forward DCT-I/DST-I transforms, 2 modal z-solves, 3 inverse
 * transforms, 4 finalisation/control.  Instrumentation for roofline
 * reporting; the state advances as in nfgs_step. */
int nfgs_time_phases(void* handle, int32_t n_iters, double* ms_out);

/* The 2-D transforms of one iteration applied to host data (instrumentation
 * for transform parity tests; uses the handle's work buffers and its third
 * state buffer).  chain 0: DCT-I in x then y of an (nz, ny, nx) volume
 * (nfgs_solver.py:4354-4355, 4445-4446); chain 1: DST-I of the interior
 * (nz, ny-2, nx-2) volume (nfgs_solver.py:1019-1050).  inverse != 0 applies
 * the inverse transforms.  Forward: all planes of chain 0, planes 1..nz-2 of
 * chain 1; inverse: planes 1..nz-1 (chain 0) and 1..nz-2 (chain 1); other
 * planes of out are left unspecified. */
int nfgs_apply_transform(void* handle, int32_t chain, int32_t inverse, const double* in, double* out);

int nfgs_destroy(void* handle);

/* Message for the last failing call on this thread ("" if none). */
const char* nfgs_last_error(void);

/* Library build identification (sm arch, version). */
const char* nfgs_version(void);

/* Device memory of every solver handle (state, tables, set-up scratch)
 * comes from one stream-ordered memory pool per device that keeps freed
 * memory reserved, so creating and destroying solvers does not pay
 * cudaMalloc / cudaFree after the first one; device-to-host staging uses
 * pinned chunks shared by the process, the transform matrices are one
 * device copy per grid size shared by the solvers of a device, and the
 * page-locked control mirrors are reused.  This call hands the reserved
 * device memory of `device`, the idle pinned chunks and mirrors, and (when no
 * solver of `device` is alive) its shared matrices back, after a device
 * synchronisation.  No reference counterpart: the reference's PyTorch
 * tensors come from torch's caching allocator, whose equivalent is
 * torch.cuda.empty_cache(). */
int nfgs_release_cached_memory(int32_t device);

/* Batched scan (the reference runs its weight x rho sweeps as a serial loop
 * of solves, run_nfgs_td_robin_weight_sweep.py:510-660): handles that have
 * each been through nfgs_iterate_begin (graph mode) are advanced together.
 * nfgs_scan_create builds one CUDA graph holding `iters` iterations of every
 * handle (independent chains, so the solves run concurrently); each
 * nfgs_scan_launch launches it once, waits, and returns how many solves have
 * not stopped (stopped solves skip their work on the device).  Finish each
 * handle with nfgs_iterate_end.  All handles must be on one device. */
int nfgs_scan_create(void* const* handles, int32_t n, int32_t iters, void** scan_out);
int nfgs_scan_launch(void* scan, int32_t* n_active_out);
/* Add solves begun since (nfgs_iterate_begin with use_graph) to a scan
 * between launches: the scan's graph is rebuilt with them, so a caller can
 * start launching while the rest of its solves are still being set up. */
int nfgs_scan_add(void* scan, void* const* handles, int32_t n);
int nfgs_scan_destroy(void* scan);

/* Learned warm start (no reference counterpart; the reference always starts
 * from the zero-source state, nfgs_solver.py:6613-6645).
 * nfgs_iterate_start_state: device views (storage type, (nz, ny, nx)) of the
 * gs_cfcf start state that nfgs_iterate_begin prepared; the library's stream
 * is synchronised, so the views are complete for any stream; valid until the
 * first nfgs_iterate_advance.
 * nfgs_iterate_restart_from: phi, az are device arrays of the same shape and
 * type, complete when called (the library reads them on its own stream).
 * mode 0: only evaluate their sigma_J; 1: make them the start when their
 * sigma_J is lower than the gs_cfcf start's; 2: make them the start;
 * 3: evaluate like 0 but leave the start's sources to be restored by the
 * next call of another mode or by the first nfgs_iterate_advance (several
 * candidates in a row then cost one restore); 4: only that restore (phi and
 * az may be NULL; out3[0] NaN).
 * out3 = {sigma of the supplied state, sigma of the gs_cfcf start, 1 if it
 * became the start}.  Must come before the first nfgs_iterate_advance
 * (NFGS_ESTATE otherwise). */
int nfgs_iterate_start_state(void* handle, void** phi_out, void** az_out);
int nfgs_iterate_restart_from(void* handle, const void* phi, const void* az, int32_t mode, double* out3);

/* soft_cfcf start: replaces the gs_cfcf start prepared by nfgs_iterate_begin
 * (call it between nfgs_iterate_begin and the first nfgs_iterate_advance,
 * NFGS_ESTATE otherwise).  Replaces NFGSSolverGPU._soft_cfcf_initial_state
 * (nfgs_solver.py:6427-6484), which compute_initial_conditions /
 * iterate(init_mode="soft_cfcf") call (nfgs_solver.py:6613-6628,
 * 6937-6955): per horizontal mode, the z profile minimising
 * |D_z L_k Phi|^2 + (k^2 + epsilon)|L_k Phi|^2 (Phi) and
 * |L_k A_z|^2 + epsilon(|D_z A_z|^2 + k^2|A_z|^2) (A_z), L_k = D_zz - k^2,
 * with the bottom data and the transparent top Robin row exact, solved by a
 * banded Cholesky of the normal equations (normal_ridge * max(1, max diag)
 * added to the diagonal).  epsilon, normal_ridge >= 0 (NFGS_EINVAL), the
 * reference's soft_cfcf_epsilon (default 1e-4 / min(dx, dy, dz)^2) and
 * soft_cfcf_normal_ridge.  Nz >= 5 and Nx, Ny >= 3 (NFGS_EINVAL).  A
 * non-finite solve is NFGS_ESTATE (the reference's RuntimeError).
 * out4 = {curl-current energy, current energy, objective = curl-current +
 * epsilon * current (the modal quadrature, nfgs_solver.py:6486-6540),
 * sigma_J of the start}. */
int nfgs_iterate_soft_cfcf_start(void* handle, double epsilon, double normal_ridge, double* out4);

/* The cfcf start: between nfgs_iterate_begin and the first advance, the
 * gs_cfcf start is replaced by the Stable-NFPT curl-free-current state
 * projected into the NFGS scalars.  Replaces
 * NFGSSolverGPU._build_stable_cfcf_initial_state (nfgs_solver.py:6080-6147),
 * which compute_initial_conditions / iterate(init_mode="cfcf") call
 * (nfgs_solver.py:6613-6628, 6937-6955).  A_z is the zero-source Dirichlet
 * extension of the stable solver's T = Poisson2D(-Jz), its Jz the legacy
 * helper-grid current (nfgs_solver.py:2331-2351, 3394-3398, 1498-1567);
 * Phi_c solves lap_xy Phi_c = B_z - B_background,z on planes 1..nz-1, B_z
 * the potential field's harmonic extension of Bz_obs with a Neumann top
 * (nfgs_solver.py:1611-1627) with the BC1 wall and top copies when
 * lateral_bc1 != 0 (the lateral_wall "paper_bc1" / "BC1" / "paper";
 * nfgs_solver.py:2138-2164).  mean_bcz_out (nz doubles, may be NULL): the
 * mean B_c,z per height (stable_cfcf_mean_bcz_by_height).  out2 = {sigma_J
 * of the start, 1 if A_z differs from the gs_cfcf start's}. */
int nfgs_iterate_cfcf_start(void* handle, int32_t lateral_bc1, double* mean_bcz_out, double* out2);

/* Per-step diagnostics of record_iteration_diagnostics=True
 * (nfgs_solver.py:6660-6681, 6806-6933) for the candidate of the last step,
 * after nfgs_iterate_advance(handle, 1, ...): out15 = {phi_update,
 * az_update, phi_map_residual, az_map_residual, h_k0_update,
 * h_k0_map_residual, bcz_pde_residual, jz_pde_residual,
 * poloidal_pde_residual, toroidal_pde_residual, mixed_row_residual,
 * bottom_field_imprint, bottom_jz_imprint (all relative),
 * alpha_clip_fraction, weak_field_floor_fraction}.  NFGS_ESTATE unless the
 * last advance ran exactly one step. */
#define NFGS_NSTEPDIAG 15
int nfgs_step_diagnostics(void* handle, double* out15);

/* stop_mode="fixed_point" (nfgs_solver.py:3707-3776, 3815-3818): the
 * solution becomes the final accepted iterate rather than the best-sigma
 * state; stop_now != 0 also ends the iteration with NFGS_STOP_FIXED_POINT
 * (the host decides the fixed point from the step diagnostics). */
int nfgs_iterate_fixed_point(void* handle, int32_t stop_now);

/* State of the k_h=0 closure (coupled_k0, constrained_spline_harmonic):
 * the horizontally uniform field H(z) = (H_x, H_y) by plane that the next
 * start state carries (the selected state's after iterate, the target
 * constant after set_boundary; nfgs_solver.py:5058-5097, 6991-7004), and
 * the last update's fit (nfgs_solver.py:5952-6067).  Layout, nz planes:
 *   out[0 .. 2nz)    H of the selected state (x then y)
 *   out[2nz .. 4nz)  last fitted profile H* (before the k0_update_mu blend)
 *   out[4nz .. 6nz)  last target mean current (mean J_x, mean J_y) by plane
 *   out[6nz]         running maximum of the relative fit residual
 *   out[6nz + 1]     2-norm condition number of the spline KKT matrix (NaN
 *                    for coupled_k0)
 *   out[6nz + 2]     number of updates since iterate_begin
 * n >= 6nz + 3.  NFGS_EUNSUPPORTED for the other horizontal policies. */
#define NFGS_K0_EXTRA 3
int nfgs_k0_state(void* handle, double* out, int32_t n);

/* The k_h=0 closure's fit as a linear map, host only (no device needed):
 * profile = G q + m h0 for a target mean current q by plane and bottom
 * value h0, G row-major nz x nz, m of length nz.  spline != 0 selects
 * constrained_spline_harmonic (basis n_basis), else coupled_k0 (legacy != 0:
 * "legacy_plane_centred").  cond_out: the spline KKT matrix's 2-norm
 * condition number, NaN for coupled_k0 (nfgs_solver.py:5149-5404). */
int nfgs_k0_operator(int32_t nz, double dz, int32_t spline, int32_t legacy, int32_t n_basis, double smoothness,
                     double* G, double* m, double* cond_out);

/* ------------------------------------------------------------------------
 * Evaluation metrics of a solution on a region of interest, in one FP64-
 * accumulating pass on the GPU.  Replaces the NumPy metrics the reference
 * runs on host copies of the fields:
 *   compute_reference_metrics   nfgs/_backend/util/metrics.py:123-178
 *   compute_metrics             nfgs/_backend/scripts/recompute_td_referee_diagnostics.py:344-400
 *   roi_cwsin / fortran_cwsin   nfgs/_backend/util/metrics.py:64-120
 *   curl, divergence, sigma_j   nfgs/diagnostics/common_fd2.py:21-78
 * ref, sol, cur: device pointers to component-major (3, nz, ny, nx) volumes
 * of dtype (NFGS_F32 or NFGS_F64); ref and cur may be NULL.  spacing3 =
 * {dx, dy, dz}.  roi6 = {z0, z1, y0, y1, x0, x1}, half-open, non-empty and
 * inside the volume.  The finite-difference curl and divergence are those
 * of the full volume (one-sided at its walls), evaluated on the region.
 * out (host, NFGS_MET_COUNT doubles) gets the metrics below; those that need
 * ref (or cur) are NaN when it is NULL.  stream is a cudaStream_t; the call
 * returns when the result is on the host.
 * ------------------------------------------------------------------------ */
enum {
    NFGS_MET_C_VEC = 0,        /* sum b.B / sqrt(sum |B|^2 sum |b|^2) */
    NFGS_MET_C_CS,             /* mean b.B / (|B||b|) */
    NFGS_MET_EPRIME_N,         /* 1 - sum |b - B| / sum |B| */
    NFGS_MET_EPRIME_M,         /* 1 - mean |b - B| / |B| */
    NFGS_MET_EPSILON,          /* sum |b|^2 / sum |B|^2 */
    NFGS_MET_SIGMA_J,          /* on cur: sum |J x b| / max(|b|, 1e-10) / sum |J| */
    NFGS_MET_SIGMA_J_FD2,      /* the same on the second-order curl of sol */
    NFGS_MET_DIVB_NORM,        /* mean |div b| / (6 mean |b| / h_eff), h_eff = 3 / (1/dx + 1/dy + 1/dz) */
    NFGS_MET_CELLS,            /* cells in the region */
    NFGS_MET_SUM_B2,           /* sum |b|^2 */
    NFGS_MET_SUM_REF2,         /* sum |B|^2 */
    NFGS_MET_NONFINITE_B,      /* cells with a non-finite b or B component */
    NFGS_MET_NONFINITE_J,      /* cells with a non-finite cur component */
    NFGS_MET_COUNT
};
int nfgs_field_metrics(const void* ref, const void* sol, const void* cur, int32_t dtype, int32_t nz, int32_t ny,
                       int32_t nx, const double* spacing3, const int32_t* roi6, double* out, void* stream);

/* ------------------------------------------------------------------------
 * Field-line tracing and squashing-factor (Q) maps on a seed plane.
 * Replace the FastQSL tracer and Q step that the reference drives through
 * CuPy for its topology maps: compute_y0_qmap / compute_bottom_qmap
 * (nfgs/_backend/util/fastqsl_plane.py:203-506), which launch TraceAllBline
 * (third_party/FastQSL/fastqslpy/cu/TraceBlineAdaptive.cu:429) over the seeds
 * and then QCalcPlane.  Written from the published definition of Q (Titov,
 * Hornig & Demoulin 2002; Titov 2007), not from that source.
 *
 * nfgs_trace_field_lines: b = device (3, nz, ny, nx) volume of dtype (NFGS_F32
 * or NFGS_F64), at least 2 nodes per axis.  Positions are grid-index units
 * (x in [0, nx-1], y in [0, ny-1], z in [0, nz-1]), B trilinear between
 * nodes.  Each of the n seeds (device (n, 3) xyz of dtype; clamped into the
 * box) is traced along +B and along -B with classical RK4 steps of length
 * `step` along the unit field direction, until the step that leaves the box
 * (cut where its chord meets the first face, the end snapped onto that face)
 * or max_steps steps.  normal3 = unit normal n0 of the seed plane.
 * Outputs (device, dtype unless stated):
 *   ends   (2, n, 3)  forward then backward end points;
 *   flags  (2, n)     int32: face reached 1..6 = x=0, x=nx-1, y=0, y=ny-1,
 *                     z=0, z=nz-1; 0 max_steps reached; -1 zero field met;
 *   bn     (3, n)     B.n0 at the seed, |B.n| at the forward and backward
 *                     ends (n the face normal; NaN without a face);
 *   length (2, n)     path length of each half, grid units;
 *   twist  (2, n)     NULL, or the twist of each half: the integral of
 *                     J.B / (4 pi |B|^2) ds along it (J = curl B by
 *                     second-order differences in grid units, one-sided at
 *                     the walls; at least 3 nodes per axis), with the RK4
 *                     stages of the line (as the reference's include_twist,
 *                     fastqsl_plane.py:287-305).
 * stream: a cudaStream_t (NULL for the legacy default stream) on the current
 * device; the call returns when the outputs are complete.
 *
 * nfgs_qmap_plane: the n = nu * nv seeds of the trace formed a regular grid
 * of unit spacing on the plane (seed iu + nu * iv, iu along the unit in-plane
 * axis u, iv along v).  q (nv, nu) of dtype: with a = dr/du, b = dr/dv of the
 * forward (+) and backward (-) end points by central differences,
 *   Q = [|a+|^2 |b-|^2 + |b+|^2 |a-|^2 - 2 (a+.b+)(a-.b-)] |Bn+ Bn-| / Bn0^2;
 * NaN on the plane's border and where the five lines of a direction (the
 * seed and its four neighbours) do not all end on one face.
 * ------------------------------------------------------------------------ */
int nfgs_trace_field_lines(const void* b, int32_t dtype, int32_t nz, int32_t ny, int32_t nx, const void* seeds,
                           int64_t n, const double* normal3, double step, int32_t max_steps, void* ends,
                           int32_t* flags, void* bn, void* length, void* twist, void* stream);
int nfgs_qmap_plane(int32_t dtype, int32_t nu, int32_t nv, const void* ends, const int32_t* flags, const void* bn,
                    void* q, void* stream);

/* nfgs_trace_qperp: Q_perp of Titov (2007) at each seed, which needs no seed
 * plane and stays defined where B lies in the plane of the seeds (where the
 * plane form above divides by Bn0 = 0).  Per seed, five lines are traced both
 * ways: through the seed and through seed +- delta e1, seed +- delta e2, with
 * e1, e2 unit vectors perpendicular to B at the seed (e1 = unit(b x a), a the
 * coordinate axis least aligned with b = B/|B|; e2 = b x e1).  With
 * a = dr/dp, b = dr/dq of the end points by central differences over
 * +-delta,
 *   Q = [|a+|^2 |b-|^2 + |b+|^2 |a-|^2 - 2 (a+.b+)(a-.b-)] |Bn+ Bn-| / |B0|^2;
 * NaN unless all five lines of each direction end on one face, or where
 * B0 = 0.  Outputs as nfgs_trace_field_lines for the central line (ends
 * (2, n, 3), flags (2, n), length (2, n), twist (2, n) or NULL) except
 * bn (3, n) = |B0|, |Bn+|, |Bn-|; q (n).  delta > 0 in grid units. */
int nfgs_trace_qperp(const void* b, int32_t dtype, int32_t nz, int32_t ny, int32_t nx, const void* seeds, int64_t n,
                     double delta, double step, int32_t max_steps, void* ends, int32_t* flags, void* bn, void* length,
                     void* q, void* twist, void* stream);

/* FastQSL-compatible tracing and Q: the reference's topology maps
 * (compute_y0_qmap / compute_bottom_qmap, nfgs/_backend/util/
 * fastqsl_plane.py:203-506) trace with the vendored FastQSL adaptive tracer
 * (TraceAllBline, third_party/FastQSL/fastqslpy/cu/TraceBlineAdaptive.cu:
 * 429-512) and form Q with QCalcPlane (fastqslpy/FastQSL.py:65-122).  These
 * two entry points restate both in the reference's FP32 arithmetic.
 *
 * nfgs_trace_fastqsl: b (3, nz, ny, nx) FP32 device field; seeds (n, 3) xyz
 * grid coordinates; normal3 the seed plane's unit normal; step the initial
 * step (1/8 in the reference), tol_coef its tol (0.1).  Per seed, the line
 * along +B gives the end and along -B the start (embedded RKF4(5) with the
 * reference's step control, face handling and limits).  Outputs (device):
 * ends (2, n, 3): [0] end, [1] start; flags (2, n): 1..6 the face reached
 * (x min, x max, y min, y max, z min, z max), 0 stopped inside, 42 through an
 * edge or corner; bsamp (3, 3, n): B (x, y, z rows) at the seed, the end and
 * the start; bflag (n): 1 where |B.n| < |B| / 100 at the seed; length (n):
 * both halves' path length; twist (n, with_twist != 0): both halves'
 * integral of J.B / (4 pi |B|^2) ds with J the centred grid curl.
 *
 * nfgs_qcalc_plane: the seeds formed an nv x nu plane (seed u + nu v);
 * q (nv, nu) FP32: QCalcPlane's Q from the face-projected end coordinates
 * and the z components of B at the ends, at least 1, NaN on the border and
 * where a neighbour's flags differ; stride the seed spacing (1). */
int nfgs_trace_fastqsl(const float* b, int32_t nz, int32_t ny, int32_t nx, const float* seeds, int64_t n,
                       const double* normal3, double step, double tol_coef, int32_t with_twist, float* ends,
                       int32_t* flags, float* bsamp, int32_t* bflag, double* length, double* twist, void* stream);
int nfgs_qcalc_plane(int32_t nu, int32_t nv, const float* ends, const int32_t* flags, const float* bsamp,
                     const double* normal3, double stride, float* q, void* stream);

/* ------------------------------------------------------------------------
 * Learned warm start: operator kernels of a 3-D neural operator on a
 * truncated cosine basis.  No reference counterpart (the reference starts
 * every solve from the zero-source state, nfgs_solver.py:6613-6645).
 * All pointers are device pointers; activations are FP32, channel-major
 * (C, Nz, Ny, Nx); stream is a cudaStream_t (NULL = legacy stream).
 * Reductions are fixed-order (bitwise repeatable).
 * ------------------------------------------------------------------------ */
const char* nfgs_nn_last_error(void);
/* y[o,v] (+)= sum_i W[o*ci + i] x[i,v] + b[o] (b may be NULL) */
int nfgs_nn_pointwise(const float* x, const float* W, const float* b, float* y, int32_t ci, int32_t co, int64_t nvox,
                      int32_t accumulate, void* stream);
/* gx (+)= W^T gy (gx may be NULL); gW += gy x^T; gb += sum_v gy (gb may be NULL).
 * scratch holds ceil(nvox/1024) * (co*ci + co) floats. */
int nfgs_nn_pointwise_bwd(const float* x, const float* W, const float* gy, float* gx, float* gW, float* gb, int32_t ci,
                          int32_t co, int64_t nvox, int32_t accumulate_gx, float* scratch, int64_t scratch_len,
                          void* stream);
int nfgs_nn_gelu(const float* x, float* y, int64_t n, void* stream);
int nfgs_nn_gelu_bwd(const float* x, const float* gy, float* gx, int64_t n, int32_t accumulate, void* stream);
/* out[c,kz,ky,kx] = sum Mz[kz,z] My[ky,y] Mx[kx,x] in[c,z,y,x]; bases row-major (K, N), kx <= 32.
 * t1: C*nz*ny*kx floats, t2: C*nz*ky*kx floats. */
int nfgs_nn_reduce3(const float* in, float* out, int32_t C, int32_t nz, int32_t ny, int32_t nx, const float* Mz,
                    const float* My, const float* Mx, int32_t kz, int32_t ky, int32_t kx, float* t1, float* t2,
                    void* stream);
/* out[c,z,y,x] (+)= sum Mz[kz,z] My[ky,y] Mx[kx,x] in[c,kz,ky,kx].
 * t1: C*nz*ky*kx floats, t2: C*nz*ny*kx floats. */
int nfgs_nn_expand3(const float* in, float* out, int32_t C, int32_t nz, int32_t ny, int32_t nx, const float* Mz,
                    const float* My, const float* Mx, int32_t kz, int32_t ky, int32_t kx, int32_t accumulate,
                    float* t1, float* t2, void* stream);
/* out (C, mz, my, mx) = trilinear resampling of in (C, nz, ny, nx) between node grids spanning the same box
 * (target node z' at source coordinate z' (nz-1)/(mz-1), likewise y, x). */
int nfgs_nn_resample_linear(const float* in, float* out, int32_t C, int32_t nz, int32_t ny, int32_t nx, int32_t mz,
                            int32_t my, int32_t mx, void* stream);
/* yh[o,k] = sum_i W[(k*ci + i)*co + o] xh[i,k] */
int nfgs_nn_modemix(const float* xh, const float* W, float* yh, int32_t ci, int32_t co, int32_t nm, void* stream);
/* gxh = W^T gyh per mode; gW += xh gyh^T per mode */
int nfgs_nn_modemix_bwd(const float* xh, const float* W, const float* gyh, float* gxh, float* gW, int32_t ci,
                        int32_t co, int32_t nm, void* stream);
/* loss_out (device double) = sum mask (pred - target)^2 / count; grad = 2 mask (pred - target) / count.
 * part: device doubles, at least ceil(n/256). mask may be NULL. */
int nfgs_nn_mse(const float* pred, const float* target, const float* mask, float* grad, int64_t n, double count,
                double* part, double* loss_out, void* stream);
/* Adam with decoupled weight decay, step >= 1 */
int nfgs_nn_adam(float* p, const float* g, float* m, float* v, int64_t n, float lr, float b1, float b2, float eps,
                 float wd, int32_t step, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* NFGS_B200_H */
