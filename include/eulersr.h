/*
 * eulersr.h -- C ABI of the B200-native explicit finite-volume Euler solver.
 *
 * This is the boundary a host (Python through ctypes, or any FFI) binds to
 * replace EulerSR's JAX solve path. Every entry point is extern "C", takes
 * plain pointers and sizes, returns an int status (ESR_OK = 0) and never lets
 * an exception cross the boundary; the text of the last error of the calling
 * thread is returned by esr_last_error().
 *
 * Reference interfaces each call replaces (paths inside the EulerSR checkout):
 *   esr_mesh_create      Mesh (euler/jax_fvm/src/mesh.py:28-150) + its geometry
 *                        (mesh.py:223-260), loaded by euler/config.py:63-79
 *   esr_solver_create    kwargs + scheme selection of euler/main.py:43-60
 *   esr_set_case         euler/main.py:28-41 initialize(); the warm-start init
 *                        field of eval/_fvm_solve_worker.py:97-105
 *   esr_compute_dt       euler/jax_fvm/src/helper.py:8-18 get_dt (with the CFL
 *                        clamp of euler/main.py:117-121)
 *   esr_step             euler/jax_fvm/src/euler_solver.py:635-643
 *                        time_step_RK2_SSP (and :630-653 EE/RK2)
 *   esr_run              the lax.scan loop and stop rule of euler/main.py:141-216
 *   esr_residual_probe   euler/main.py:228-230 and eval/_fvm_solve_worker.py:120-139
 *   esr_forces           euler/jax_fvm/src/helper.py:366-415 (get_drag/lift_coefficient)
 *   esr_entropy          euler/jax_fvm/src/helper.py:312-320 get_total_entropy
 *   esr_batch_solve      the serial grid loop of slurm/run_euler_grid.py:94-104,
 *                        run as one batch with retire/refill
 *   esr_batch_submit /   the same batch in three non-blocking steps (the grid
 *   _poll / _results /   loop's calls to euler.main.run, :103-104, issued
 *   _cancel              together and collected when done)
 *   esr_idw_apply        eval/core.py:135-142 predict_idw (weights utils/metrics.py:9-14)
 *   esr_set_cases /      esr_set_case / esr_get_state for many slots at once (the
 *   esr_get_states       per-case initialize + np.asarray(W) of the grid loop)
 *   esr_gemm_bf16 and    the network forward/backward that produces the warm start
 *   the esr_mlp_*        (models/dam.py:306-308 with loss.py:20-23), here a residual
 *                        MLP on IDW
 *   esr_solver_tuning    no counterpart (XLA chooses launch shapes itself)
 *
 * Threading: a solver handle owns one CUDA stream and must not be used from
 * two threads at once. Handles of different solvers are independent.
 */
#ifndef EULERSR_H
#define EULERSR_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ESR_API_VERSION 1

/* status codes */
#define ESR_OK             0
#define ESR_ERR_ARG        1   /* invalid argument (ValueError in the reference) */
#define ESR_ERR_CUDA       2   /* CUDA runtime error */
#define ESR_ERR_NONFINITE  3   /* non-finite value met where a finite one is required */
#define ESR_ERR_TIMEOUT    4   /* a bounded device wait gave up */
#define ESR_ERR_OOM        5   /* device allocation failed */
#define ESR_ERR_STATE      6   /* call not valid in the handle's current state */

/* per-case status words (esr_result.status) */
#define ESR_CASE_EMPTY      0
#define ESR_CASE_RUNNING    1
#define ESR_CASE_CONVERGED  2   /* stop rule met `patience` times in a row */
#define ESR_CASE_MAXSTEP    3   /* reached N = int(tf/dt)+1 (or max_steps) unconverged */
#define ESR_CASE_NONFINITE  4   /* NaN/Inf in the state norm: case retired */

/* options */
#define ESR_PREC_F32 0
#define ESR_PREC_F64 1
#define ESR_FLUX_HLLC 0
#define ESR_FLUX_RUSANOV 1
#define ESR_RECON_MUSCL 0
#define ESR_RECON_CONSTANT 1
#define ESR_TIME_SRK2 0
#define ESR_TIME_EE 1
#define ESR_TIME_RK2 2
#define ESR_DT_GLOBAL 0        /* one dt per case from the initial field (reference) */
#define ESR_DT_LOCAL 1         /* per-cell CFL dt recomputed every step */
#define ESR_STOP_REFERENCE 0   /* ||W_n - W_ref||_F / (steps (||W_ref||_F + 1e-16)) */
#define ESR_STOP_DENSITY_L2 1  /* RMS over cells of the density residual */
#define ESR_STOP_ENGINEERING 2 /* stop when the engineering criterion (force coefficients
                                * within tolerance of given targets) is confirmed */
#define ESR_BLOCK_PATCHES (-1)  /* esr_params.block_size: K2 by patches of <= 24 cells, each inner
                                  * face's flux evaluated once and exchanged in shared memory
                                  * (float32 fast fidelity, HLLC + MUSCL; the fluxes are bitwise
                                  * those of the per-cell K2) */
#define ESR_FIDELITY_FAST 0      /* geometry formed in float64 and rounded once; float32 kernels
                                  * with approximate division and the direct HLLC flux */
#define ESR_FIDELITY_REFERENCE 1 /* the reference's rounding: geometry formed in the run's
                                  * precision in its operation order (mesh.py:223-240,
                                  * euler_solver.py:49,74,79, helper.py:136-150), the
                                  * least-squares gradient solved per call (helper.py:136-153)
                                  * and float32 kernels with IEEE division, the central-flux
                                  * identity and no fused multiply-add */

/* Mesh description; all host arrays are owned by the caller and copied. */
typedef struct esr_mesh_desc {
    int32_t n_points;
    int32_t n_cells;
    int32_t n_faces;
    const double*  points;            /* (n_points, 2) */
    const int32_t* tris;              /* (n_cells, 3), counter-clockwise */
    const int32_t* neighbors;         /* (n_cells, 3), cell across edge k (v_k, v_k+1), -1 = boundary */
    const int32_t* faces;             /* (n_faces, 2) vertex ids */
    const int32_t* face_markers;      /* (n_faces,) 0 interior, 2 wall, 3 inlet, 4 outlet, 5 subsonic inlet */
    const int32_t* face_connectivity; /* (n_cells, 3) face id of edge k */
    const int32_t* wall_markers;      /* markers treated as slip walls (NULL -> {2}) */
    int32_t n_wall_markers;
    int32_t force_marker;             /* marker of the faces the force coefficients integrate (2) */
    int32_t sponge;                   /* 1: top/bottom sponge layer (all cases but 'bump') */
    double sponge_width;              /* <= 0: 0.2 * (y_max - y_min) */
    double inlet_subsonic[4];         /* rho, u, v, p of the subsonic inlet (marker 5) */
    int32_t renumber;                 /* 1: reorder cells (reverse Cuthill-McKee) for locality */
} esr_mesh_desc;

typedef struct esr_mesh_info {
    int32_t n_cells;
    int32_t n_faces;
    int32_t n_wall_faces;
    int32_t n_boundary_slots;
    double y_min, y_max;
    int64_t device_bytes_f32;
    int64_t device_bytes_f64;
} esr_mesh_info;

typedef struct esr_params {
    int32_t precision;        /* ESR_PREC_* */
    int32_t flux;             /* ESR_FLUX_* */
    int32_t reconstruction;   /* ESR_RECON_* */
    int32_t time_scheme;      /* ESR_TIME_* */
    int32_t dt_mode;          /* ESR_DT_* */
    int32_t stop_rule;        /* ESR_STOP_* */
    double gamma;             /* ratio of specific heats of the run (1.4) */
    double threshold;         /* stationarity threshold */
    int32_t check_every;      /* steps between stop-rule checks (>= 1) */
    int32_t patience;         /* consecutive checks under the threshold (>= 1) */
    int32_t device;           /* CUDA device ordinal */
    int32_t use_graphs;       /* 1: capture step chunks in CUDA graphs */
    int32_t block_size;       /* threads per block for the cell kernels: 64, 128, 256, 0 = autotuned,
                               * or ESR_BLOCK_PATCHES: cell kernels at 128 with K2 formed by patches */
    int32_t fidelity;         /* ESR_FIDELITY_* (0: fast) */
    int32_t stream_priority;  /* CUDA priority of the solver's stream (0: default; lower is
                               * higher, clamped to the device's range): a solver whose small
                               * launches run beside another solver's long chunks gets SMs first */
} esr_params;

/* One (Mach, alpha) case. inlet = conserved freestream (euler/main.py:39). */
typedef struct esr_case {
    int32_t mesh;             /* index of the mesh the case runs on */
    int32_t reserved;
    double mach;
    double aoa_deg;
    double cfl;               /* already clamped by the caller or not: see esr_params */
    double tf;                /* N = int(tf/dt) + 1 */
    int64_t max_steps;        /* extra cap on N (0: none) */
    double inlet[4];          /* conserved inlet state */
    double rho_inf;           /* force reference density */
    double u_inf;             /* force reference speed |U_inf| */
    double l_ref;             /* force reference length (obstacle_length) */
    /* engineering criterion tracked beside the stop rule, never stopping the
     * case (euler/main.py:66-113,160-171): |cd - target_cd| <= cd_tol *
     * max(|target_cd|, 1e-8) and the same for cl, `eng_patience` checks in a row */
    int32_t eng_track;
    int32_t eng_patience;
    double eng_target_cd, eng_target_cl;
    double eng_cd_tol, eng_cl_tol;
    /* stop-rule threshold of this case; <= 0: the solver's esr_params.threshold
     * (eval/convergence_case.py:61-65 gives each case its own: the reference
     * field's one-step residual x 1.001) */
    double threshold;
} esr_case;

typedef struct esr_result {
    int32_t status;           /* ESR_CASE_* */
    int32_t converged;        /* 1 when the stop rule confirmed */
    int32_t stopping_step;    /* first step of the confirming streak, else N */
    int32_t steps;            /* steps actually advanced */
    int32_t n_max;            /* N = int(tf/dt)+1 (capped by max_steps) */
    int32_t case_index;       /* batch solves: index into the submitted case list; esr_run /
                                 esr_get_results: the slot of a case set on it, else -1 */
    double dt;                /* global dt of the case (0 in local mode) */
    double last_rel;          /* last stop-rule value */
    double cd, cl;            /* body-axis pressure force coefficients at the end */
    double solve_time_s;      /* device time from the case's start to its retirement */
    int32_t eng_converged;    /* engineering criterion confirmed (0 when not tracked) */
    int32_t eng_stopping_step;/* first step of its confirming streak, else N */
    double final_residual;    /* esr_batch_solve: one more step of the final state with the
                                 case's own dt, ||W' - W||_F / (||W||_F + 1e-16)
                                 (euler/main.py:228-230); esr_run leaves 0, use
                                 esr_residual_probe */
} esr_result;

typedef struct esr_mesh esr_mesh;
typedef struct esr_solver esr_solver;

int32_t     esr_api_version(void);
const char* esr_last_error(void);

int esr_mesh_create(const esr_mesh_desc* desc, esr_mesh** out);
int esr_mesh_destroy(esr_mesh* mesh);
int esr_mesh_get_info(const esr_mesh* mesh, esr_mesh_info* info);
/* new-to-old cell permutation chosen by the renumbering (n_cells entries) */
int esr_mesh_get_permutation(const esr_mesh* mesh, int32_t* perm);
/* The renumbering's patches (at most 24 cells each; the face-flux kernel of
 * batched float32 solves exchanges the fluxes of a patch's inner faces in
 * shared memory): *n_patches, and when start is not NULL the first new cell
 * of every patch plus n_cells (n_patches + 1 entries). */
int esr_mesh_get_patches(const esr_mesh* mesh, int32_t* n_patches, int32_t* start);
/* The per-cell geometry the kernels read, in the caller's cell order, for a
 * fidelity (ESR_FIDELITY_*) and precision (ESR_PREC_*): geo receives
 * n_cells x 24 values (normals n_kx, n_ky of the three edges, face lengths,
 * area, sponge blend^3, pad, least-squares coefficients c_kx, c_ky, face
 * offsets f_kx, f_ky); lsq, when not NULL and the pair is reference
 * fidelity in float32, receives n_cells x 13 values (weights w_k, offsets
 * dx_k, the 2x2 matrix a00 a01 a10 a11 of the per-call solve). Inspection
 * only (mesh.py:223-260 computes the same quantities). */
int esr_mesh_get_geometry(const esr_mesh* mesh, int32_t fidelity, int32_t precision, double* geo, double* lsq);

/* A solver holds `n_meshes` meshes and slots_per_mesh[m] concurrent case
 * slots on mesh m; all slots advance together in one launch per kernel. It
 * keeps its own copy of each mesh, so a mesh may be destroyed once the
 * solvers made from it exist. */
int esr_solver_create(const esr_mesh* const* meshes, const int32_t* slots_per_mesh, int32_t n_meshes,
                      const esr_params* params, esr_solver** out);
int esr_solver_destroy(esr_solver* solver);
int esr_solver_num_slots(const esr_solver* solver, int32_t* n_slots);
/* Slot `slot` gets case `c`; W_init = (n_cells, 4) conserved state in the
 * caller's cell order, or NULL for the freestream of c->inlet. Computes the
 * case's dt (global mode) and resets its stop-rule counters. */
int esr_set_case(esr_solver* solver, int32_t slot, const esr_case* c, const double* W_init);
int esr_clear_slot(esr_solver* solver, int32_t slot);
/* esr_set_case for n slots at once: slots[i] gets cases[i] and W_init[i]
 * (W_init NULL, or a NULL entry: freestream). The host fields are copied
 * asynchronously (pinned buffers copy fastest), the dt of every filled slot
 * comes from one reduction, and the call synchronises once. A slot may be
 * listed once; as in esr_set_case, the slot decides the mesh. Every case is
 * checked before anything changes: a call that fails on an argument leaves
 * every slot as it was. */
int esr_set_cases(esr_solver* solver, int32_t n, const int32_t* slots, const esr_case* cases,
                  const double* const* W_init);
/* esr_get_state for n slots at once into out[i] (caller's cell order); one
 * synchronisation at the end. */
int esr_get_states(esr_solver* solver, int32_t n, const int32_t* slots, double* const* out);
/* The same with float32 host fields (half the bytes over PCIe; a float32
 * solver stores exactly these values). */
int esr_set_cases_f32(esr_solver* solver, int32_t n, const int32_t* slots, const esr_case* cases,
                      const float* const* W_init);
int esr_get_states_f32(esr_solver* solver, int32_t n, const int32_t* slots, float* const* out);
/* The same moves overlapped with the solver's work, for pipelines that feed
 * one batch while the previous one runs (the upload of the next cases and
 * the download of the last fields run on a copy stream of the solver):
 * esr_stage_cases_f32 checks the cases and starts copying their float32
 * fields (host memory; page-locked copies overlap) and returns; the fields
 * must stay unchanged until the copy ends (esr_wait_transfers, or the next
 * esr_stage_cases_f32). esr_apply_staged places the staged cases in their
 * slots on the solver's stream (as esr_set_cases_f32 would) without waiting
 * for them. esr_fetch_states_f32 gathers the slots' fields on the solver's
 * stream (after everything issued before it) and starts copying them into
 * out[i], returning at once; esr_wait_transfers waits for every staged and
 * fetched copy. Results equal esr_set_cases_f32 / esr_get_states_f32 bit for
 * bit. (Same calls as esr_set_cases / esr_get_state, euler/main.py:28-41 and
 * the grid loop's np.asarray(W), issued ahead.) */
int esr_stage_cases_f32(esr_solver* solver, int32_t n, const int32_t* slots, const esr_case* cases,
                        const float* const* W_init);
int esr_apply_staged(esr_solver* solver);
int esr_fetch_states_f32(esr_solver* solver, int32_t n, const int32_t* slots, float* const* out);
int esr_wait_transfers(esr_solver* solver);
/* Slot `slot` restarts from state W (caller's cell order): stop-rule counters
 * reset and dt recomputed from W, as esr_set_case with W_init does. */
int esr_set_state(esr_solver* solver, int32_t slot, const double* W);
int esr_get_state(esr_solver* solver, int32_t slot, double* W);
/* device-resident float32/float64 state of a slot in the caller's cell order;
 * d_W must be memory of the solver's GPU (or managed memory) aligned to 16
 * bytes, else ESR_ERR_ARG before any launch */
int esr_set_state_device(esr_solver* solver, int32_t slot, const void* d_W);
int esr_get_state_device(esr_solver* solver, int32_t slot, void* d_W);
int esr_compute_dt(esr_solver* solver, double* dt_per_slot);
/* Advance every running slot by nsteps (no stop rule). */
int esr_step(esr_solver* solver, int32_t nsteps);
/* Run every running slot to its stop (stop rule, N, or non-finite). */
int esr_run(esr_solver* solver, esr_result* results_per_slot);
int esr_get_results(esr_solver* solver, esr_result* results_per_slot);
int esr_residual_probe(esr_solver* solver, double* rel_per_slot);
int esr_forces(esr_solver* solver, double* cd_per_slot, double* cl_per_slot);
int esr_entropy(esr_solver* solver, double* total_per_slot);
/* Unlimited LSQ gradient of the primitives of one slot, boundary ghosts
 * included: grad[(cell*4 + var)*2 + dim], caller's cell order. Replaces the
 * host gradient of the bundle export (euler/utils.py:33-39, helper.py:136-153). */
int esr_gradients(esr_solver* solver, int32_t slot, double* grad);
int esr_synchronize(esr_solver* solver);
/* Device milliseconds of the solver's stream between the last two esr_run /
 * esr_step / esr_batch_solve boundaries. */
int esr_last_elapsed_ms(esr_solver* solver, double* ms);
/* Number of kernel launches issued by the solver since creation. */
int esr_kernel_launches(const esr_solver* solver, int64_t* n);

/* Average device time of each kernel kind over `nsteps` plain steps issued
 * without graphs, CUDA events recorded on the solver's stream around every
 * launch. The steps advance the state like esr_step. */
typedef struct esr_kernel_times {
    double recon_ms;          /* K1: gradient, limiter, MUSCL face states */
    double flux_ms;           /* K2: face fluxes, residual, stage update */
    double other_ms;          /* bookkeeping kernels */
    int32_t recon_launches;
    int32_t flux_launches;
    int32_t other_launches;
    int32_t reserved;
} esr_kernel_times;
int esr_profile_step(esr_solver* solver, int32_t nsteps, esr_kernel_times* out);

/* The autotuner's record: with esr_params.block_size = 0 the solver times one
 * full step of all its slots for each launch shape at creation and keeps the
 * fastest (no reference counterpart: XLA picks launch shapes). Shapes: the
 * cell kernels at 64, 128 and 256 threads per block; at the best of those,
 * where the float32 fast kernels run, K2's second register budget, K2 by
 * patches at both of its budgets (float32 fast fidelity, HLLC + MUSCL), and
 * K1's second budget with the best K2. A register budget is the number of
 * resident blocks per SM a kernel is compiled for. The choice is kept for
 * the process per solver shape (device, precision, scheme, each mesh's cells
 * and slots): a second solver of the same shape takes it without timing
 * (cached = 1). Results do not depend on the choice. */
#define ESR_TUNING_MAX_VARIANTS 12
typedef struct esr_tuning_variant {
    int32_t block_size;       /* threads per block of K1 (and of the per-cell K2) */
    int32_t k2_patches;       /* 1: K2 by patches */
    int32_t k1_minb;          /* register budget of K1 (0: not constrained; the K1 that
                                 also writes the local time step keeps its own) */
    int32_t k2_minb;          /* register budget of K2, per-cell or patch form */
    double step_ms;           /* device ms of one step */
} esr_tuning_variant;
typedef struct esr_tuning {
    int32_t block_size;       /* threads per block of the cell kernels in use */
    int32_t n_candidates;     /* 0 when block_size was given */
    int32_t candidates[4];    /* 64, 128, 256 and ESR_BLOCK_PATCHES at the default budgets */
    int32_t k2_patches;       /* 1: K2 runs by patches */
    int32_t cached;           /* 1: taken from an earlier solver of the same shape */
    double step_ms[4];        /* device ms of one step per candidate */
    int32_t k1_minb;          /* register budgets in use (0: not constrained) */
    int32_t k2_minb;
    int32_t n_variants;       /* every shape timed, in order */
    int32_t reserved;
    esr_tuning_variant variants[ESR_TUNING_MAX_VARIANTS];
} esr_tuning;
int esr_solver_tuning(const esr_solver* solver, esr_tuning* out);
/* Run the solver with the given launch shape (a variant recorded by an
 * earlier autotuning, or chosen by hand); step_ms is ignored, a budget of 0
 * means the kernel's default. ESR_ERR_ARG for a shape this solver cannot run
 * (K2 by patches or a second budget outside float32 fast fidelity, HLLC +
 * MUSCL), ESR_ERR_STATE while a submitted batch owns the slots. Results do
 * not depend on the shape. */
int esr_solver_set_shape(esr_solver* solver, const esr_tuning_variant* shape);

/* Solve n_cases cases through the solver's slots: every slot retired by the
 * stop rule is refilled in place with the next queued case. init_fields[i]
 * is a (n_cells,4) conserved warm start or NULL; final_states[i] receives the
 * final state when non-NULL. results has n_cases entries. A solver on K2 by
 * patches runs the batch's tail (every mesh down to 24 running cases or
 * fewer) with the per-cell K2, whose threads cover the running slots alone;
 * the results are the same. */
int esr_batch_solve(esr_solver* solver, const esr_case* cases, int32_t n_cases,
                    const double* const* init_fields, double* const* final_states,
                    esr_result* results);

/* esr_batch_solve split so that the caller keeps its thread between polls
 * (slurm/run_euler_grid.py:94-104 run as one batch, as above).
 * esr_batch_submit uploads the cases (init_fields as in esr_batch_solve; the
 * fields are copied before it returns), fills every slot and returns; from
 * then on the batch owns the slots, and every other call on the solver except
 * esr_batch_poll, esr_batch_results, esr_batch_cancel, esr_solver_num_slots,
 * esr_solver_tuning, esr_synchronize, esr_last_elapsed_ms and
 * esr_kernel_launches fails with ESR_ERR_STATE. want_states != 0 keeps every
 * case's final state for esr_batch_results. esr_batch_poll advances the batch
 * by a few captured chunks (doubling from 4 up to 32 per call), waits for
 * them, and reports how many cases have finished; results are bitwise those
 * of esr_batch_solve. esr_batch_results (valid once *n_done == n_cases)
 * fills results[n_cases] and, when final_states is non-NULL, final_states[i]
 * (NULL entries skipped), then releases the batch. esr_batch_cancel
 * abandons a pending batch: running cases stop and their slots go inactive
 * (without a pending batch it does nothing). A failing poll cancels the
 * batch itself. */
int esr_batch_submit(esr_solver* solver, const esr_case* cases, int32_t n_cases,
                     const double* const* init_fields, int32_t want_states);
int esr_batch_poll(esr_solver* solver, int32_t* n_done);
int esr_batch_results(esr_solver* solver, double* const* final_states, esr_result* results);
int esr_batch_cancel(esr_solver* solver);

/* Relative change ||A - B||_F / (||B||_F + 1e-16) of two device fields of
 * n_rows x 4 values (float4 rows for ESR_PREC_F32, double4 rows for
 * ESR_PREC_F64), written to the device double *d_out on `stream`. d_A and
 * d_B must be memory of the current GPU (or managed memory) aligned to 16
 * bytes, d_out the same aligned to 8 bytes; anything else (a host address,
 * another GPU's memory) is ESR_ERR_ARG before any launch. No counterpart in the reference: it is the allocation-free form
 * of the solver's stop-rule norm, for callers that cannot allocate device
 * memory when they need it (a host allocator that owns the whole device
 * budget, a pre-sized arena that forbids allocation after start-up). Its
 * scratch is a fixed 16 KiB device array inside the library: at most
 * 2,097,152 rows (larger n_rows is rejected with ESR_ERR_ARG); every GPU that
 * loads the library holds the array until exit; the first call on a device
 * looks up the array's address once (make it before any stream capture);
 * calls that overlap on the GPU race on the shared array. */
int esr_rel_change_noalloc(const void* d_A, const void* d_B, int64_t n_rows, int32_t precision,
                           double* d_out, void* stream);

/* IDW (k neighbours, weights 1/(d^2+1e-12) normalised) of a source field onto
 * target points; all pointers are device pointers, float32, row-major. A
 * neighbour index outside [0, n_src) is never read: that target row is set
 * to NaN and the library's IDW error flag is raised. */
int esr_idw_apply(const float* d_src, int32_t n_src, int32_t n_vars,
                  const int32_t* d_idx, const float* d_dist, int32_t n_dst, int32_t k,
                  float* d_out, void* stream);
/* Synchronous: 1 in *bad when an esr_idw_apply since the last call met an
 * out-of-range neighbour index, then clears the flag. */
int esr_idw_status(int32_t* bad);

/* ---- learned warm start: BF16 training/inference kernels of the residual
 * MLP that corrects the IDW interpolation (replaces the DAM/AMNet forward of
 * models/dam.py:306-308 with a 4 x 256 residual MLP; loss of loss.py:20-23).
 * All pointers are device pointers; `stream` is a cudaStream_t or NULL. */

/* C[M x N] = A[M x K] B[K x N] on the fifth-generation tensor cores
 * (tcgen05.mma, accumulators in tensor memory), BF16 operands, FP32
 * accumulation. trans_a: A stored [K][M] else [M][K]; trans_b: B stored
 * [K][N] else [N][K] (a torch Linear weight). epi 0: FP32 partial tiles
 * (out0 + split * M * ldo); epi 1: z = acc + bias -> out1, out0 = res +
 * relu(z); epi 2: dh = acc + res -> out0, out1 = dh * (aux > 0).
 * M, N multiples of 128, K a multiple of 64 * splits. */
int esr_gemm_bf16(int32_t trans_a, int32_t trans_b, int32_t M, int32_t N, int32_t K, const void* A, int32_t lda,
                  const void* B, int32_t ldb, int32_t epi, const float* bias, const void* res, const void* aux,
                  void* out0, void* out1, int32_t ldo, int32_t splits, void* stream);
/* The same GEMM on the warp-level mma.sync path (K a multiple of 32 *
 * splits), kept as the cross-check of the tcgen05 kernel. */
int esr_gemm_bf16_mma_sync(int32_t trans_a, int32_t trans_b, int32_t M, int32_t N, int32_t K, const void* A,
                           int32_t lda, const void* B, int32_t ldb, int32_t epi, const float* bias, const void* res,
                           const void* aux, void* out0, void* out1, int32_t ldo, int32_t splits, void* stream);
/* Synchronous: 1 in *gave_up when a tcgen05 GEMM stopped waiting on its
 * pipeline barriers (bounded waits) since the last call, then clears it. */
int esr_gemm_tc_status(int32_t* gave_up);
/* 4-wide output layer: y = H W^T + b (+ base), H BF16 [rows x K], W FP32 [4 x K] */
int esr_mlp_head_fwd(const void* H, int32_t rows, int32_t K, const float* W, const float* b, const float* base,
                     float* y, void* stream);
/* its backward: dH = dY W, dZ = dH * (Z > 0) (BF16), dW/db partials per `rpb` rows */
int esr_mlp_head_bwd(const float* dY, const void* H, const void* Z, int32_t rows, int32_t K, const float* W, void* dH,
                     void* dZ, float* part, int32_t rpb, void* stream);
/* per-cell input rows (13 features, zero padded to ld columns, BF16) and,
 * when base != NULL, the normalised IDW primitives the MLP corrects (FP32) */
int esr_mlp_features(const float* stat5, const float* idw_prim, const float* idw_gradp, int32_t rows, float mach_n,
                     float aoa_n, const float* mu, const float* sig, int32_t ld, void* X, float* base, void* stream);
/* normalised primitive prediction -> conserved float64 rows (density and pressure floored) */
int esr_mlp_decode(const float* pred_n, int32_t rows, const float* mu, const float* sig, float gamma, float rho_floor,
                   float p_floor, double* W, void* stream);
/* shock-weighted relative MSE: per-block loss partials and d loss / d pred */
int esr_mlp_loss(const float* pred, const float* tgt, const float* w, int32_t rows, const float* inv_den,
                 float* dpred, float* part, void* stream);
/* fixed-order sums: out[i] = sum_s part[s*stride + i]; column sums of BF16 rows */
int esr_reduce_splits(const float* part, int32_t splits, int64_t stride, int64_t n, float* out, void* stream);
int esr_colsum_bf16(const void* X, int32_t rows, int32_t C, int32_t rpb, float* part, void* stream);
/* AdamW on FP32 master weights, refreshing an optional BF16 copy */
int esr_adamw(float* p, const float* g, float* m, float* v, int64_t n, float lr, float b1, float b2, float eps,
              float wd, int32_t step, void* p_bf16, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* EULERSR_H */
