/* C ABI of the B200-native ARS(2,2,2) IMEX step for 2-D resistive MHD.
 *
 * Drop-in replacement for the hot path of RikibabManos/Magnetohydrodynamics_Simulator: its IMEX()
 * integrator (include/solvers.hpp:491-613), the implicit matrix set-up (solvers.hpp:404-443 +
 * ConjugateGradient::compute at src/integrator_main.cpp:58-60, 87-95), the CFL time-step selector
 * (include/diagnostics.hpp:44-88) and the div B diagnostic (diagnostics.hpp:15-42).
 *
 * Conventions
 *  - All arithmetic is IEEE FP64 on the GPU (sm_100a); there is no CPU fallback.
 *  - A context owns its device memory; the caller owns every host buffer it passes.
 *  - Field order everywhere: rho, mx, my, E, bxf, byf (conserved state of Grid.hpp:19-22);
 *    bxf(i,j) is B_x on the left face of cell (i,j), byf(i,j) is B_y on its bottom face.
 *  - Host layouts: MHD_LAYOUT_DENSE = nx*ny doubles, row-major (j*nx + i), physical cells only;
 *    MHD_LAYOUT_PADDED = the reference Grid vectors, (nx+2ng)*(ny+2ng) doubles with the first
 *    physical cell at (ng, ng) (Grid.hpp:29-62).
 *  - Every call returns an mhd_status. Calls that enqueue work (mhd_step, mhd_run, ...) are
 *    asynchronous on the context's stream; conditions found on the device (non-finite state, CG
 *    not converged, barrier timeout) are reported by mhd_synchronize.
 *  - Grids are periodic; nx, ny >= 2 (the reference's ghost fill needs two physical cells).
 */
#ifndef MHD_B200_H
#define MHD_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    MHD_OK = 0,
    MHD_ERR_INVALID_ARGUMENT = 1,
    MHD_ERR_CUDA = 2,
    MHD_ERR_NONFINITE = 3,          /* a NaN/Inf appeared in the state or the CG broke down */
    MHD_ERR_CG_NOT_CONVERGED = 4,   /* an implicit solve hit its iteration cap */
    MHD_ERR_TIMEOUT = 5,            /* a grid-wide wait of the persistent CG ran out of time */
    MHD_ERR_NO_DEVICE = 6,          /* no sm_100 device, or the library was not built for it */
    MHD_ERR_OUT_OF_MEMORY = 7,
    MHD_ERR_NO_STATE = 8,           /* a state must be set before stepping */
    MHD_ERR_TOO_LARGE = 9,          /* grid larger than the fixed scratch of the no-alloc call */
    MHD_ERR_IO = 10                 /* a snapshot file could not be written */
} mhd_status;

typedef enum { MHD_LAYOUT_DENSE = 0, MHD_LAYOUT_PADDED = 1 } mhd_layout;

/* Corner-velocity test of the upwind constrained transport (solvers.hpp:326,333). The reference
 * calls an unqualified abs() on a double there, which GCC resolves to int abs(int): the face
 * fields are averaged whenever |v| < 1. MHD_CT_TRUE_ABS applies the literal |v| < 1e-12. */
typedef enum { MHD_CT_REFERENCE = 0, MHD_CT_TRUE_ABS = 1 } mhd_ct_mode;

typedef struct {
    int nx, ny;              /* physical cells (Grid::nx, Grid::ny) */
    double dx, dy;           /* Grid::cell_width, Grid::cell_height */
    double eta;              /* Grid::resistivity */
    int ct_mode;             /* mhd_ct_mode */
    double cg_tol;           /* <= 0: machine epsilon (Eigen's default) */
    long long cg_max_iters;  /* <= 0: 2*nx*ny (Eigen's default) */
    double courant;          /* CFL factor (diagnostics.hpp:82 uses 0.5); <= 0 selects 0.5 */
    double safety;           /* CFL safety (diagnostics.hpp:84 uses 0.9); <= 0 selects 0.9 */
    double cg_timeout_s;     /* wall-clock limit of one implicit solve; <= 0 selects 30 s */
} mhd_params;

typedef struct mhd_context mhd_context;

/* Fill *p with the reference's defaults for an nx*ny grid of cell size dx*dy. */
mhd_status mhd_default_params(mhd_params* p, int nx, int ny, double dx, double dy, double eta);

/* Allocate the device state and workspace: replaces Grid x3 + integrator_reserved_memory +
 * ReconstructedValues + the Eigen solver (src/integrator_main.cpp:34-48, solvers.hpp:68-193).
 * stream: a cudaStream_t (NULL = a new non-blocking stream owned by the context). */
mhd_status mhd_create(const mhd_params* p, void* stream, mhd_context** out);
mhd_status mhd_destroy(mhd_context* ctx);

/* Upload / download the conserved state. The upload applies nothing (no floors); like the
 * reference driver (integrator_main.cpp:52-53) the first step floors the density. */
mhd_status mhd_set_state(mhd_context* ctx, const double* const fields[6], int layout, int ng);
mhd_status mhd_get_state(mhd_context* ctx, double* const fields[6], int layout, int ng);
/* Pipelined host transfers, for streaming states through host memory step after step (no
 * counterpart in the reference, whose state lives on the host). Dense nx*ny host planes, pinned for
 * the copies to overlap (pageable memory works but serialises). Both calls only enqueue: the copies
 * run on two copy streams of the context, in quarter planes, so that a state's read-back and the
 * next state's upload overlap in the two directions of the host link. mhd_set_state_async: the next
 * step waits for the upload, and each piece's upload waits for the previous mhd_get_state_async's
 * copy of that piece (the same host buffer may be passed to both). mhd_get_state_async: copies the
 * current state once the work queued so far is done; later steps wait for these copies before
 * they overwrite the state. The host buffers are ready after mhd_transfers_wait (or
 * mhd_synchronize). */
mhd_status mhd_set_state_async(mhd_context* ctx, const double* const fields[6]);
mhd_status mhd_get_state_async(mhd_context* ctx, double* const fields[6]);
mhd_status mhd_transfers_wait(mhd_context* ctx);
/* Same, with device pointers to dense nx*ny planes (device-to-device copies). */
mhd_status mhd_set_state_device(mhd_context* ctx, const double* const fields[6]);
mhd_status mhd_get_state_device(mhd_context* ctx, double* const fields[6]);

/* Grid::fillGhostPeriodic + computePrimitives of the current state (Grid.hpp:64-136):
 * rho (floored), vx, vy, p, bxc, byc; any pointer may be NULL. */
mhd_status mhd_get_primitives(mhd_context* ctx, double* const prims[6], int layout, int ng);

/* generate_A_matrix(grid, workspace, alpha) + ConjugateGradient::compute (solvers.hpp:404-443,
 * integrator_main.cpp:58-60): the implicit solves use (I - alpha L) until the next call. Until it
 * is first called, each step uses alpha = dt * eta * (1 - 1/sqrt 2). */
mhd_status mhd_set_implicit_coefficient(mhd_context* ctx, double alpha);

/* IMEX(grid, ..., dt) (solvers.hpp:491-613): one ARS(2,2,2) step in place. dt <= 0 takes the
 * CFL step of the current state instead (computed on the device). Asynchronous. */
mhd_status mhd_step(mhd_context* ctx, double dt);

/* The driver loop of src/integrator_main.cpp:76-112 on the device: nsteps steps, each with
 * dt = dt_fixed, or the CFL step when dt_fixed <= 0, clipped so the time does not pass t_end
 * (t_end <= 0: no clipping); the implicit matrix is regenerated only when dt moved by more than
 * 1e-10 relative, as the reference driver does. Captured into a CUDA graph. dts_out and
 * cg_products_out (2 per step), if not NULL, are host arrays filled on return (synchronous). */
mhd_status mhd_run(mhd_context* ctx, int nsteps, double dt_fixed, double t_end, double* dts_out,
                   long long* cg_products_out);

/* resistive_B_term(grid, bx_rate, by_rate, solver, workspace, solve_implicitly)
 * (solvers.hpp:445-489) on device arrays: the rate of the face field, -curl E, from the corner field
 * E = eta*J_z(B) (solve_implicitly == 0) or the solution of (I - alpha L) E = eta*J_z(B)
 * (solve_implicitly != 0; the reference's matrix of generate_A_matrix(grid, workspace, alpha)).
 * bxf, byf, bx_rate, by_rate are device pointers to dense nx*ny planes of the context's grid.
 * cg_products (host, may be NULL) receives the solve's matrix-vector products; when it is given
 * the call waits for the result. Uses the context's solver workspace (not concurrent with a step
 * on another stream). */
mhd_status mhd_resistive_rate(mhd_context* ctx, int solve_implicitly, double alpha,
                              const double* bxf, const double* byf, double* bx_rate,
                              double* by_rate, long long* cg_products);

/* Allocation-free variant of mhd_resistive_rate (no counterpart in the reference).
 *
 * For callers that cannot allocate device memory where they need the solve: plugins whose host
 * application owns every device buffer and hands out only its own, processes running under a
 * device-memory budget where a new allocation fails or is not allowed, and latency-sensitive loops
 * in which cudaMalloc/cudaFree would stall on an implicit device synchronisation. It takes no
 * context; the caller passes the inputs and outputs (device pointers to dense nx*ny planes) and
 * the grid parameters (nx, ny, dx, dy, eta, cg_tol, cg_max_iters, cg_timeout_s are used).
 *
 * Scratch lives in one file-scope device array sized for at most MHD_NOALLOC_MAX_CELLS cells
 * (256 x 256; about 2.7 MB, held on every device that loads this library until the process
 * exits). Larger grids are rejected with MHD_ERR_TOO_LARGE. The function calls no cudaMalloc,
 * cudaFree or allocating library routine. The first call on a device resolves the array's device
 * address (cudaGetSymbolAddress) and sets up the solver kernel; make that first call before any
 * stream capture. All calls share the one array: calls that overlap on the GPU (other streams,
 * other threads) race on it, so serialise them. stream: a cudaStream_t (NULL = legacy default).
 * With solve_implicitly != 0 the call always waits for the solve and returns its device status
 * (MHD_ERR_NONFINITE, MHD_ERR_CG_NOT_CONVERGED, MHD_ERR_TIMEOUT or MHD_OK), whether or not
 * cg_products (host, may be NULL) is given to receive the matrix-vector products; the solver runs
 * with the same geometry as a context's, so its result equals mhd_resistive_rate's bit for bit.
 * With solve_implicitly == 0 (no solve) the call only enqueues the rate kernel and returns. */
#define MHD_NOALLOC_MAX_CELLS 65536
mhd_status mhd_resistive_rate_noalloc(const mhd_params* p, int solve_implicitly, double alpha,
                                      const double* bxf, const double* byf, double* bx_rate,
                                      double* by_rate, long long* cg_products, void* stream);

/* CFL_condition_checker(grid) (diagnostics.hpp:44-88) with the context's courant/safety. */
mhd_status mhd_cfl_dt(mhd_context* ctx, double* dt);

/* calculate_current_div_B(grid) (diagnostics.hpp:15-42): RMS and max |div B|. Synchronous. */
mhd_status mhd_divb(mhd_context* ctx, double* rms, double* maxabs);

/* Wait for the context's stream; return and clear the device-side status (first of:
 * MHD_ERR_TIMEOUT, MHD_ERR_NONFINITE, MHD_ERR_CG_NOT_CONVERGED). */
mhd_status mhd_synchronize(mhd_context* ctx);

/* Matrix-vector products of the last step's two implicit solves (after mhd_synchronize). */
mhd_status mhd_last_cg_products(mhd_context* ctx, long long out[2]);
/* Matrix-vector products of the first (out[0]) and second (out[1]) implicit solve of every step
 * since the context was created, summed (for per-step averages over a timed run; no counterpart
 * in the reference). Synchronises. */
mhd_status mhd_cg_products_sum(mhd_context* ctx, long long out[2]);

/* Device planes of the current state (dense nx*ny, valid until the next step). */
mhd_status mhd_state_device_pointers(mhd_context* ctx, double* out[6]);

/* Record CUDA events around every kernel of the following mhd_step calls (enable != 0), for
 * per-kernel device times; no counterpart in the reference (which only prints a wall-clock total,
 * src/integrator_main.cpp:114-120). */
mhd_status mhd_set_kernel_timing(mhd_context* ctx, int enable);

/* Device time of each kernel summed over the steps recorded since timing was enabled or last read,
 * in ms: out[0] stage 1, out[1] first implicit solve, out[2] stage 2, out[3] second solve,
 * out[4] finalize. *steps receives the number of steps. Synchronises; clears the record. */
mhd_status mhd_kernel_times(mhd_context* ctx, double out_ms[5], long long* steps);

/* The stream the context enqueues on (a cudaStream_t). */
void* mhd_stream(mhd_context* ctx);

/* Number of kernel launches one mhd_step enqueues (for launch accounting). */
int mhd_launches_per_step(mhd_context* ctx);

/* Snapshots in the reference's file format: the bytes write_data_to_binary_file
 * (diagnostics.hpp:90-131) writes for the Grid after fillGhostPeriodic + computePrimitives, as the
 * driver calls it every snapshot_frequency steps (integrator_main.cpp:102-109). 9 doubles
 * [nx, ny, ng, snapshot_rate, dx, dy, dt, divB_rms, divB_max], then 7 padded planes of
 * (nx+2ng)*(ny+2ng) doubles with periodic ghost layers, in the order rho (floored), E, p, vx, vy,
 * bxc, byc (the reader scripts/display_functions.py:3-22 reshapes them so). 0 <= ng <= min(nx, ny);
 * the reference's Grid has ng = 2. */
size_t mhd_snapshot_bytes(mhd_context* ctx, int ng);  /* 0 for an invalid ng */
/* Write the current state's snapshot to the file `path` asynchronously: packed on the device in
 * stream order (later steps do not disturb it), copied to pinned host memory on a copy stream of
 * its own and written by a host thread while the caller keeps stepping. Two snapshots can be in
 * flight; a third call waits for the older one. */
mhd_status mhd_snapshot_write(mhd_context* ctx, const char* path, int ng, int snapshot_rate,
                              double dt);
/* Wait until every snapshot written so far is on disk; MHD_ERR_IO if a file could not be written
 * (since the last wait). */
mhd_status mhd_snapshot_wait(mhd_context* ctx);
/* The same bytes into host memory `out` (mhd_snapshot_bytes long), synchronously. */
mhd_status mhd_snapshot_pack(mhd_context* ctx, int ng, int snapshot_rate, double dt, void* out);

/* ---------------------------------------------------------------------------------------------
 * Batched stepping (no counterpart in the reference, which advances one Grid per process):
 * `count` independent periodic simulations, each with its own mhd_params (size, spacing, eta,
 * courant, safety, ct_mode, solver tolerance), advanced together. Each step is one launch per
 * stage for the whole batch (coefficients, stage 1, implicit solve, stage 2, implicit solve,
 * finalize; the solves take one launch per 64 instances). Every instance gets exactly the step
 * it would get from its own mhd_context: its own CFL dt, its own matrix coefficient, its own CG
 * convergence. States are dense nx*ny planes in the order rho, mx, my, E, bxf, byf. */
typedef struct mhd_batch mhd_batch;

/* Work decomposition of the batch kernels, chosen by mhd_batch_autotune. */
typedef struct mhd_batch_tuning {
    int stage_rows;  /* rows per work item of the explicit stages and the finalize (>= 1; a strip
                      * is cut into equal items of at most this many rows) */
    int cg_rows;     /* implicit solve: rows of a band (cg_order 0) or of a tile (1), >= 1; with
                      * cg_order 1, 0 lets every phase choose its tile height (16-256 rows) for the
                      * instances still iterating */
    int cg_order;    /* implicit solve: each phase deals the work of the instances still
                      * iterating evenly over the warps, 0: as equal row ranges (numbered in bands
                      * of cg_rows rows, strip by strip within a band), 1: as 28 x cg_rows tiles,
                      * round robin */
    int stage_tail_rows; /* > 0: the last min(stage_rows, ny) rows of every strip go in items of this many
                          * rows, which largest-first scheduling runs last (fills the launch's
                          * tail); 0: none */
    double stage_ms; /* device time of the explicit kernels in the tuning step (output only) */
    double cg_ms;    /* device time of the solver launches in the tuning step (output only) */
} mhd_batch_tuning;

/* params: count parameter blocks. stream: a cudaStream_t (NULL = a new non-blocking stream). */
mhd_status mhd_batch_create(const mhd_params* params, int count, void* stream, mhd_batch** out);
mhd_status mhd_batch_destroy(mhd_batch* b);
int mhd_batch_count(mhd_batch* b);
/* Upload / download instance `index`'s state: host (or device) pointers to dense planes. */
mhd_status mhd_batch_set_state(mhd_batch* b, int index, const double* const fields[6]);
mhd_status mhd_batch_get_state(mhd_batch* b, int index, double* const fields[6]);
mhd_status mhd_batch_set_state_device(mhd_batch* b, int index, const double* const fields[6]);
mhd_status mhd_batch_get_state_device(mhd_batch* b, int index, double* const fields[6]);
/* As mhd_set_implicit_coefficient, for one instance. */
mhd_status mhd_batch_set_implicit_coefficient(mhd_batch* b, int index, double alpha);
/* One step of every instance; dts: host array of count steps (<= 0: that instance's CFL step),
 * or NULL for CFL steps throughout. Asynchronous. */
mhd_status mhd_batch_step(mhd_batch* b, const double* dts);
/* mhd_run for every instance at once (the driver loop of src/integrator_main.cpp:76-112 per
 * instance), captured as a CUDA graph. dts_out[count][nsteps] and
 * cg_products_out[count][nsteps][2], if not NULL, are host arrays filled on return. */
mhd_status mhd_batch_run(mhd_batch* b, int nsteps, double dt_fixed, double t_end, double* dts_out,
                         long long* cg_products_out);
/* Time one step of the current states under candidate decompositions and keep the fastest
 * (the states, times and step counters are restored afterwards). All states must be set.
 * *out (may be NULL) receives the choice. Synchronous. */
mhd_status mhd_batch_autotune(mhd_batch* b, mhd_batch_tuning* out);
mhd_status mhd_batch_set_tuning(mhd_batch* b, const mhd_batch_tuning* t);
mhd_status mhd_batch_get_tuning(mhd_batch* b, mhd_batch_tuning* t);
/* Wait; return the worst device status over the batch and clear it. per_instance (may be NULL)
 * receives count statuses. */
mhd_status mhd_batch_synchronize(mhd_batch* b, mhd_status* per_instance);
/* Matrix-vector products of each instance's last two solves: out[count][2] (after synchronize). */
mhd_status mhd_batch_last_cg_products(mhd_batch* b, long long* out);
/* As mhd_cfl_dt and mhd_divb, for one instance. */
mhd_status mhd_batch_cfl_dt(mhd_batch* b, int index, double* dt);
mhd_status mhd_batch_divb(mhd_batch* b, int index, double* rms, double* maxabs);
void* mhd_batch_stream(mhd_batch* b);
/* Kernel launches one mhd_batch_step enqueues. */
int mhd_batch_launches_per_step(mhd_batch* b);

/* ---------------------------------------------------------------------------------------------
 * Differentiation (no counterpart in the reference): the discrete adjoint of a fixed-dt
 * trajectory of IMEX steps (solvers.hpp:491-613 with the driver's matrix alpha = dt*eta*g),
 * computed by hand-written adjoint kernels of the reconstruction, HLL flux, CT and stage update
 * and by the (self-adjoint) implicit solve. The forward pass keeps every checkpoint_every-th
 * state; the backward pass recomputes each segment of steps from its checkpoint and runs the
 * adjoint steps backwards through it. All state arguments are device pointers to dense nx*ny
 * planes in the order rho, mx, my, E, bxf, byf. Density and pressure floors are differentiated as
 * clamps (zero derivative where active); minmod, HLL and CT branches as selections. */
typedef struct mhd_adjoint mhd_adjoint;

/* p: the grid (nx, ny, dx, dy, eta, ct_mode, cg_tol, cg_max_iters, cg_timeout_s are used);
 * dt > 0 the fixed step; nsteps >= 1; checkpoint_every >= 1. */
mhd_status mhd_adj_create(const mhd_params* p, double dt, int nsteps, int checkpoint_every,
                          void* stream, mhd_adjoint** out);
/* Memory mode of mhd_adj_create_ex. By default the forward pass keeps the two implicit solutions
 * of every step (2 * nsteps planes) and the backward pass recomputes only each segment's explicit
 * stages. MHD_ADJ_RECOMPUTE_SOLVES keeps the solutions of one segment (2 * checkpoint_every planes)
 * and re-solves each segment in the backward pass: device memory of O(nsteps / checkpoint_every +
 * checkpoint_every) planes for two more solves per step; the gradients are bit-identical. */
#define MHD_ADJ_RECOMPUTE_SOLVES 1
mhd_status mhd_adj_create_ex(const mhd_params* p, double dt, int nsteps, int checkpoint_every,
                             int flags, void* stream, mhd_adjoint** out);
/* Device memory the adjoint object holds for its planes, in bytes. */
size_t mhd_adj_device_bytes(mhd_adjoint* a);
mhd_status mhd_adj_destroy(mhd_adjoint* a);
/* Resistivity of the following passes (the matrix coefficient follows: alpha = dt*eta*g). */
mhd_status mhd_adj_set_eta(mhd_adjoint* a, double eta);
/* nsteps steps from u0; the final state is written to uT. Keeps the checkpoints. */
mhd_status mhd_adj_forward(mhd_adjoint* a, const double* const u0[6], double* const uT[6]);
/* Given dL/duT (device), write dL/du0 (device) and dL/deta (host, may be NULL) of the trajectory
 * of the last mhd_adj_forward. Synchronous. */
mhd_status mhd_adj_backward(mhd_adjoint* a, const double* const grad_uT[6],
                            double* const grad_u0[6], double* grad_eta);
/* One step's vector-Jacobian product at state u: lam = (dU^{n+1}/dU^n)^T lam_next, and
 * *grad_eta (host, may be NULL) = lam_next . dU^{n+1}/deta. Synchronous. */
mhd_status mhd_adj_step_vjp(mhd_adjoint* a, const double* const u[6],
                            const double* const lam_next[6], double* const lam[6],
                            double* grad_eta);
/* Vector-Jacobian product of the explicit rate (solvers.hpp:393-402) at u: out = F'(u)^T w. */
mhd_status mhd_adj_rate_vjp(mhd_adjoint* a, const double* const u[6], const double* const w[6],
                            double* const out[6]);
/* Kernel launches of one forward step and of one adjoint step (for launch accounting). */
mhd_status mhd_adj_launch_counts(mhd_adjoint* a, int* forward_step, int* adjoint_step);
/* The stream the adjoint object enqueues on (a cudaStream_t). */
void* mhd_adj_stream(mhd_adjoint* a);

/* ---------------------------------------------------------------------------------------------
 * Domain decomposition (no counterpart in the reference, which grows one Grid on one thread:
 * src/integrator_main.cpp:29-30). A grid is split into P x Q subdomains, one mhd_subdomain each
 * (one per GPU; several may share a GPU). A subdomain keeps its nx x ny interior cells inside
 * extended planes with a ring of MHD_SUB_HALO cells on every side; the explicit kernels run on the
 * extended planes, and the caller (the decomposition driver) refreshes the rings between kernels
 * by packing strips of each interior into buffers (mhd_sub_pack), moving them to the neighbours
 * (device copies, or NCCL between GPUs) and unpacking them into the neighbours' rings
 * (mhd_sub_unpack): west/east first, then south/north, whose strips span the extended width and so
 * also fill the corners. The implicit solve is a conjugate gradient on the interior corners with
 * one call per phase; calls that return partial sums wait for them, and the driver adds the
 * subdomains' partials in a fixed order and takes Eigen's decisions (x0 = 0, Jacobi scaling, stop
 * at |r|^2 < max(tol^2 |b|^2, DBL_MIN)). One step, with exchanges (set, ring width):
 *   set_step(dt, alpha); stage(1); exchange(PREDICTOR, H); solve on T_B; exchange(SOLUTION, H);
 *   stage(2); exchange(ACCUMULATOR_B, H); solve on A_B; exchange(SOLUTION, H); finalize();
 *   exchange(STATE, H)
 * where a solve is cg_rhs, then per product exchange(DIRECTION, 1), cg_matvec, cg_update and
 * cg_direction. dt comes from the largest interior CFL speed (mhd_sub_cfl_speed) of all
 * subdomains, by the formula of diagnostics.hpp:82-84. */
#define MHD_SUB_HALO 4
enum { MHD_SUB_WEST = 0, MHD_SUB_EAST = 1, MHD_SUB_SOUTH = 2, MHD_SUB_NORTH = 3 };
enum {
    MHD_SUB_SET_STATE = 0,          /* rho, mx, my, E, bxf, byf */
    MHD_SUB_SET_PREDICTOR = 1,      /* U1* (6 planes) */
    MHD_SUB_SET_ACCUMULATOR_B = 2,  /* the face fields of U2* (2 planes) */
    MHD_SUB_SET_SOLUTION = 3,       /* the corner field of the last solve */
    MHD_SUB_SET_DIRECTION = 4,      /* the CG direction p */
    MHD_SUB_SET_CG_EVEN = 5,        /* single-sweep solve: r_k and p_{k-1} before an even iteration */
    MHD_SUB_SET_CG_ODD = 6          /* ... before an odd iteration */
};
typedef struct mhd_subdomain mhd_subdomain;
int mhd_sub_halo(void);
/* p: the interior (nx, ny >= MHD_SUB_HALO), spacing, eta, ct_mode. stream: a cudaStream_t or NULL. */
mhd_status mhd_sub_create(const mhd_params* p, void* stream, mhd_subdomain** out);
mhd_status mhd_sub_destroy(mhd_subdomain* s);
void* mhd_sub_stream(mhd_subdomain* s);
/* Interior state from / to dense nx*ny planes (host or device pointers). Synchronous. */
mhd_status mhd_sub_set_state(mhd_subdomain* s, const double* const fields[6]);
mhd_status mhd_sub_get_state(mhd_subdomain* s, double* const fields[6]);
/* Doubles of the strip that `side` exchanges for `set` with a ring of `width` (1..MHD_SUB_HALO):
 * planes x width x ny (west/east) or planes x (nx + 2 MHD_SUB_HALO) x width (south/north). */
size_t mhd_sub_strip_doubles(mhd_subdomain* s, int set, int side, int width);
/* Pack the strip of the interior next to `side` into the device buffer buf; unpack a neighbour's
 * strip into the ring beyond `side` (the strip the neighbour packed for its opposite side).
 * Asynchronous on the subdomain's stream. */
mhd_status mhd_sub_pack(mhd_subdomain* s, int set, int side, int width, double* buf);
mhd_status mhd_sub_unpack(mhd_subdomain* s, int set, int side, int width, const double* buf);
/* Every ring of `set` (width 1..MHD_SUB_HALO) refreshed for P x Q subdomains that live in this
 * process on one device (subs[q * P + p]): device-to-device copies from each neighbour's interior
 * strips, west/east then south/north, on the receiving subdomain's stream, ordered by events; no
 * host wait. Neighbours along x must have equal rows, along y equal columns. */
mhd_status mhd_sub_exchange_local(mhd_subdomain* const* subs, int P, int Q, int set, int width);
/* Largest CFL signal speed over the interior of the state (diagnostics.hpp:60-78), and whether a
 * value is not finite. Synchronous. */
mhd_status mhd_sub_cfl_speed(mhd_subdomain* s, double* smax, int* nonfinite);
/* Coefficients of the next step: dt and the implicit matrix coefficient alpha. */
mhd_status mhd_sub_set_step(mhd_subdomain* s, double dt, double alpha);
/* Explicit stage 1 or 2 (solvers.hpp:509-517, 522-566) and the finalize (:571-611). */
mhd_status mhd_sub_stage(mhd_subdomain* s, int stage);
mhd_status mhd_sub_finalize(mhd_subdomain* s);
/* CG phases on the interior corners. cg_rhs: b = eta J_z(B*) of the predictor's (solve 0) or the
 * accumulator's (solve 1) faces, r = b, p = z = b/d, x = 0; out = partial |b|^2, r.z. cg_matvec:
 * q = (I - alpha L) p, *pq = partial p.q. cg_update: x += alpha p, r -= alpha q, z = r/d;
 * out = partial |r|^2, r.z. cg_direction: p = z + beta p. cg_zero_solution: x = 0.
 * cg_rhs, cg_matvec and cg_update wait for their sums when given an output pointer; with NULL they
 * only enqueue (several subdomains' phases then run together) and mhd_sub_sums(s, out, n) waits
 * and returns the n sums of the last such phase. */
mhd_status mhd_sub_cg_rhs(mhd_subdomain* s, int solve_index, double out[2]);
mhd_status mhd_sub_cg_matvec(mhd_subdomain* s, double* pq);
mhd_status mhd_sub_cg_update(mhd_subdomain* s, double alpha, double out[2]);
mhd_status mhd_sub_cg_direction(mhd_subdomain* s, double beta);
mhd_status mhd_sub_cg_zero_solution(mhd_subdomain* s);
mhd_status mhd_sub_sums(mhd_subdomain* s, double* out, int n);
/* Decisions of the decomposed solve on the device. A group (mhd_subcg) holds a control block of
 * MHD_SUBCG_CTL doubles and count sum slots of 4 doubles, in device memory. The *_dev phases write
 * their subdomain's sums into its slot (mhd_subcg_slots(g) + 4 index; across ranks the slots are
 * all-gathered into the group's array) and read alpha, beta and "still iterating" from the control
 * block, doing nothing once the solve has ended; mhd_subcg_decide (phase 0 after cg_rhs_dev, 1
 * after cg_matvec_dev, 2 after cg_update_dev) adds the slots in subdomain order and takes the
 * decisions of the host driver, with the same arithmetic: the results are bit-identical. The
 * subdomains and the group's stream must be ordered by the caller (one shared stream in one
 * process). mhd_subcg_post(g, tag) enqueues a copy of the control block to pinned memory and
 * mhd_subcg_read(g, tag, out) waits for it (four copies in flight: tags equal modulo 4 share one).
 * cg_finish_dev zeroes x after a solve that met a non-finite value (as cg_zero_solution).
 * mhd_subcg_decide_host applies the same rules to host arrays (no device needed). Phases 3 and 4
 * are those of the single-sweep form below. */
#define MHD_SUBCG_CTL 16
enum {
    MHD_SUBCG_ACTIVE = 0,     /* 1.0 while the solve iterates */
    MHD_SUBCG_STATUS = 1,     /* MHD_SUBCG_OK / _NOT_CONVERGED / _NONFINITE */
    MHD_SUBCG_PRODUCTS = 2,   /* matrix products so far */
    MHD_SUBCG_BB = 3,         /* |b|^2 */
    MHD_SUBCG_THRESHOLD = 4,  /* max(tol^2 |b|^2, DBL_MIN) */
    MHD_SUBCG_ABSNEW = 5,     /* r.z */
    MHD_SUBCG_ALPHA = 6,
    MHD_SUBCG_BETA = 7,
    MHD_SUBCG_RR = 8,         /* |r|^2 after the last update */
    MHD_SUBCG_PQ = 9,         /* p.q of the last product (single-sweep form: p.Ap of the next) */
    MHD_SUBCG_ALPHA_PREV = 10, /* single-sweep form: alpha of the previous iteration */
    MHD_SUBCG_K_LAST = 11,    /* single-sweep form: the last iteration swept (-1: none) */
    MHD_SUBCG_ALPHA_LAST = 12, /* single-sweep form: its alpha */
    MHD_SUBCG_ZERO = 13,      /* single-sweep form: 1 when the solution is x = 0 */
    MHD_SUBCG_DT = 14,        /* the step of the last mhd_subcg_cfl_step */
    MHD_SUBCG_CFL_NONFINITE = 15 /* 1 when that step's scan met a non-finite value */
};
enum { MHD_SUBCG_OK = 0, MHD_SUBCG_NOT_CONVERGED = 1, MHD_SUBCG_NONFINITE = 2 };
typedef struct mhd_subcg mhd_subcg;
mhd_status mhd_sub_cg_rhs_dev(mhd_subdomain* s, int solve_index, double* slot);
mhd_status mhd_sub_cg_matvec_dev(mhd_subdomain* s, const double* ctl, double* slot);
mhd_status mhd_sub_cg_update_dev(mhd_subdomain* s, const double* ctl, double* slot);
mhd_status mhd_sub_cg_direction_dev(mhd_subdomain* s, const double* ctl);
mhd_status mhd_sub_cg_finish_dev(mhd_subdomain* s, const double* ctl);
/* count: subdomains of the solve; stream: a cudaStream_t, or NULL for a stream of the group's own;
 * slots: count x 4 doubles of device memory that the caller owns, or NULL (the group allocates). */
mhd_status mhd_subcg_create(int count, void* stream, double* slots, mhd_subcg** out);
mhd_status mhd_subcg_destroy(mhd_subcg* g);
double* mhd_subcg_slots(mhd_subcg* g);
const double* mhd_subcg_control(mhd_subcg* g);
mhd_status mhd_subcg_decide(mhd_subcg* g, int phase, double tol, long long max_products);
mhd_status mhd_subcg_post(mhd_subcg* g, int tag);
mhd_status mhd_subcg_read(mhd_subcg* g, int tag, double* out);
mhd_status mhd_subcg_decide_host(double* ctl, const double* slots, int count, int phase, double tol,
                                 long long max_products);
/* For subdomains of this process on their own streams (subs[i] writes slot i): decide_on orders the
 * decision after every subdomain's work so far and their later work after it (events);
 * mhd_subcg_product enqueues one whole product of the solve -- the exchange of p's 1-cell ring
 * (mhd_sub_exchange_local), cg_matvec_dev, decision 1, cg_update_dev, decision 2,
 * cg_direction_dev on all P x Q subdomains -- as one CUDA graph on the group's stream, captured at
 * the first call for these arguments and replayed after, then posts the control block under `tag`.
 * The subdomains' streams must not be the legacy default stream (MHD_ERR_INVALID_ARGUMENT). */
mhd_status mhd_subcg_decide_on(mhd_subcg* g, mhd_subdomain* const* subs, int phase, double tol,
                               long long max_products);
mhd_status mhd_subcg_product(mhd_subcg* g, mhd_subdomain* const* subs, int P, int Q, double tol,
                             long long max_products, int tag);
/* The CFL step of every subdomain (at most 64, of one grid: equal spacing and eta) on the device:
 * the largest interior signal speed of all of them (diagnostics.hpp:60-78), dt by
 * diagnostics.hpp:82-86 with `courant` and `safety` (the host driver's arithmetic), and each
 * subdomain's step set to dt with the reference driver's matrix alpha = (dt eta) g, as
 * mhd_sub_set_step would. dt lands in ctl[MHD_SUBCG_DT] and a non-finite state in
 * ctl[MHD_SUBCG_CFL_NONFINITE], read with the next mhd_subcg_post/read. Ordered after the
 * subdomains' work so far and before their later work; no host wait. */
mhd_status mhd_subcg_cfl_step(mhd_subcg* g, mhd_subdomain* const* subs, double courant, double safety);
/* The single-sweep form of the decomposed solve: the single context's solver (one sweep per
 * product forming q = A p, r, z and the sums r.r, r.z, z.Az, z.q, with p.Ap carried by a
 * recurrence, and the solution moved every second iteration) on each subdomain's interior.
 * cg_sweep_rhs_dev: b = eta J_z(B*), r0 = b, slot = |b|^2, b.z0, z0.A z0 (then decision phase 3;
 * the predictor's or accumulator's rings must hold 2 cells). Iteration k: exchange
 * MHD_SUB_SET_CG_EVEN / _ODD (k even / odd) with a ring of 2, cg_sweep_iter_dev, decision phase 4.
 * mhd_subcg_sweep_product enqueues iteration k of subdomains that share a device as a replayed
 * graph (one per parity), with no exchange: each sweep reads the cells around its interior from
 * its neighbours' interiors (same results); it then posts the control block under `tag`.
 * cg_sweep_finish_dev ends the solve (x = 0 after a zero right-hand
 * side or a breakdown, the last alpha_k p_k after an even last iteration). */
mhd_status mhd_sub_cg_sweep_rhs_dev(mhd_subdomain* s, int solve_index, double* slot);
mhd_status mhd_sub_cg_sweep_iter_dev(mhd_subdomain* s, const double* ctl, double* slot);
mhd_status mhd_sub_cg_sweep_finish_dev(mhd_subdomain* s, const double* ctl);
mhd_status mhd_subcg_sweep_product(mhd_subcg* g, mhd_subdomain* const* subs, int P, int Q, double tol,
                                   long long max_products, int k, int tag);
/* Interior div B partials (diagnostics.hpp:15-42): out[0] = sum of div^2, out[1] = max |div|. */
mhd_status mhd_sub_divb_sums(mhd_subdomain* s, double out[2]);
mhd_status mhd_sub_synchronize(mhd_subdomain* s);

const char* mhd_status_string(mhd_status s);

/* 1 when a device this library was built for is present, else 0. */
int mhd_device_available(void);

#ifdef __cplusplus
}
#endif

#endif /* MHD_B200_H */
