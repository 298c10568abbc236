/* Test infrastructure only: the CPU oracle for the ARS(2,2,2) IMEX step.
 *
 * A plain-C restatement of the reference solver's hot path (RikibabManos/Magnetohydrodynamics_Simulator,
 * include/{Grid,MUSCL,HLL,solvers,diagnostics,benchmarks}.hpp). It is only ever used as the checker
 * in tests/, in __graft_entry__.smoke() and in bench.py's CPU-baseline leg -- never by the product.
 *
 * Layout: every field is a dense, row-major nx*ny array of doubles (index j*nx + i) holding the
 * physical cells of the reference's padded Grid (Grid.hpp:58, (ng,ng) = first physical cell).
 * Ghost cells are not stored: the reference's ghost fill is a periodic copy (Grid.hpp:143-161), so
 * every neighbour access here wraps periodically instead.
 *   bxf(i,j) = B_x on the LEFT face of cell (i,j);  byf(i,j) = B_y on the BOTTOM face;
 *   corner (i,j) = bottom-left corner of cell (i,j).
 */
#ifndef MHD_ORACLE_H
#define MHD_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int nx, ny;
    double dx, dy;       /* cell width / height (Grid::cell_width/cell_height) */
    double eta;          /* resistivity (Grid::resistivity) */
    int ct_abs_mode;     /* 0: corner-velocity test truncates to int, as GCC compiles the
                            unqualified abs() at solvers.hpp:326,333; 1: true |v| < 1e-12 */
    double cg_tol;       /* <= 0 selects machine epsilon (Eigen default) */
    long cg_max_iters;   /* <= 0 selects 2 * nx * ny (Eigen default) */
} orc_params;

/* state: 6 planes in the order rho, mx, my, E, bxf, byf */
enum { ORC_RHO = 0, ORC_MX, ORC_MY, ORC_E, ORC_BX, ORC_BY, ORC_NFIELDS };

/* Grid.hpp:82-136: cell-centred B, velocities (before the density floor), floored density and
 * pressure. Outputs may be NULL. */
void orc_primitives(const orc_params* P, const double* const state[6], double* rho_floored,
                    double* vx, double* vy, double* p, double* bxc, double* byc);

/* solvers.hpp:393-402 explicit_rhs: the six explicit rates of a state. */
void orc_explicit_rhs(const orc_params* P, const double* const state[6], double* const rate[6]);

/* solvers.hpp:450-463: right-hand side eta * J_z at every corner (nx*ny, row-major). */
void orc_corner_current_rhs(const orc_params* P, const double* bxf, const double* byf, double* rhs);

/* Eigen ConjugateGradient<SparseMatrix, Lower|Upper> defaults on the matrix of solvers.hpp:404-443,
 * (I - alpha*L) x = rhs, x0 = 0. Returns the number of matrix-vector products; *iters gets
 * Eigen's iteration count. */
long orc_cg_solve(const orc_params* P, double alpha, const double* rhs, double* x, long* iters);

/* solvers.hpp:445-489 resistive_B_term: rate of bxf/byf from the corner field; implicit when
 * alpha_or_neg >= 0 (solve with that alpha), explicit when alpha_or_neg < 0. Returns products. */
long orc_resistive_rate(const orc_params* P, const double* bxf, const double* byf,
                        double alpha_or_neg, double* bx_rate, double* by_rate);

/* solvers.hpp:491-613 IMEX: one ARS(2,2,2) step in place. alpha is the coefficient the implicit
 * matrix was generated with (dt*eta*gamma_ARS in the reference driver). cg_products[2] (may be
 * NULL) receives the products of the two solves. */
void orc_imex_step(const orc_params* P, double* const state[6], double dt, double alpha,
                   long* cg_products);

/* diagnostics.hpp:44-88 with the hyperbolic Courant factor and safety factor as parameters
 * (reference: courant = 0.5, safety = 0.9). */
double orc_cfl_dt(const orc_params* P, const double* const state[6], double courant, double safety);

/* diagnostics.hpp:15-42: RMS and max |div B| over physical cells. */
void orc_divb(const orc_params* P, const double* bxf, const double* byf, double* rms, double* maxabs);

/* diagnostics.hpp:90-131 write_data_to_binary_file of the Grid after fillGhostPeriodic +
 * computePrimitives (Grid.hpp:64-136), as the driver calls it (integrator_main.cpp:106-108): into
 * out, 9 doubles [nx, ny, ng, snapshot_rate, dx, dy, dt, divB rms, divB max], then the padded
 * (nx+2ng)*(ny+2ng) planes rho (floored), E, p, vx, vy, bxc, byc with periodic ghost layers. */
void orc_snapshot(const orc_params* P, const double* const state[6], int ng, int snapshot_rate,
                  double dt, double* out);

/* benchmarks.hpp:15-76 Orszag-Tang vortex (face B from Az at corners, E from face B). */
void orc_init_orszag_tang(const orc_params* P, double* const state[6]);

/* benchmarks.hpp:352-417 decaying magnetic sine wave with a vector potential
 * Az = az_amp * f(kx x) * sin(ky y), f = cos (reference: az_amp = 1/kx, use_sin = 0) or sin
 * (use_sin = 1); rho = p = 1, v = 0. kx, ky <= 0 select the reference's 2*pi/L. */
void orc_init_sine_wave(const orc_params* P, double* const state[6], double az_amp, double kx,
                        double ky, int use_sin);

#ifdef __cplusplus
}
#endif

#endif
