/* Test infrastructure only: CPU oracle for the ARS(2,2,2) IMEX step (see mhd_oracle.h).
 *
 * Every function restates one part of the reference solver, RikibabManos/Magnetohydrodynamics_Simulator,
 * in the same arithmetic order, on dense periodic arrays (the reference's 2-wide ghost layers are a
 * periodic copy, Grid.hpp:143-161, so neighbours wrap instead). Compiled without fast-math so that
 * it is deterministic; it is used only as the checker (tests, smoke, CPU baseline).
 */
#include "mhd_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

static const double GAMMA_GAS = 5.0 / 3.0;   /* Grid.hpp:104, HLL.hpp:31,62,85,108 */
static const double RHO_FLOOR = 1e-8;        /* Grid.hpp:115 */
static const double P_FLOOR = 1e-8;          /* Grid.hpp:124 */

static inline int wrap(int i, int n) { return (i < 0) ? i + n : ((i >= n) ? i - n : i); }
#define AT(a, i, j) (a)[(size_t)wrap((j), ny) * (size_t)nx + (size_t)wrap((i), nx)]

/* ---------------------------------------------------------------- primitives (Grid.hpp) */

void orc_primitives(const orc_params* P, const double* const s[6], double* rho_f, double* vx,
                    double* vy, double* p, double* bxc, double* byc) {
    const int nx = P->nx, ny = P->ny;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const size_t id = (size_t)j * nx + i;
            /* Grid.hpp:91,94 computeCellB: average of the two faces */
            const double bx = (s[ORC_BX][id] + AT(s[ORC_BX], i + 1, j)) / 2.0;
            const double by = (s[ORC_BY][id] + AT(s[ORC_BY], i, j + 1)) / 2.0;
            /* Grid.hpp:112-115: velocities use the density BEFORE the floor */
            double rho = s[ORC_RHO][id];
            const double u = s[ORC_MX][id] / rho;
            const double v = s[ORC_MY][id] / rho;
            if (rho < RHO_FLOOR) rho = RHO_FLOOR;
            /* Grid.hpp:118-125: EoS; the low-pressure branch leaves E untouched */
            const double kin = 0.5 * rho * (u * u + v * v);
            const double mag = (bx * bx + by * by) / 2;
            const double eint = s[ORC_E][id] - kin - mag;
            double pr = (GAMMA_GAS - 1) * eint;
            if (pr < P_FLOOR) pr = P_FLOOR;
            if (rho_f) rho_f[id] = rho;
            if (vx) vx[id] = u;
            if (vy) vy[id] = v;
            if (p) p[id] = pr;
            if (bxc) bxc[id] = bx;
            if (byc) byc[id] = by;
        }
}

/* diagnostics.hpp:90-131 (header, then the 7 planes in the order written at :121-127). The ghost
 * fill (Grid.hpp:64-80, 143-161) copies every field periodically -- bxc/byc after computeCellB --
 * and computePrimitives then runs over the whole padded grid, so each padded cell holds the
 * primitives of its periodic image. */
void orc_snapshot(const orc_params* P, const double* const s[6], int ng, int snapshot_rate,
                  double dt, double* out) {
    const int nx = P->nx, ny = P->ny;
    const int nxt = nx + 2 * ng, nyt = ny + 2 * ng;
    const size_t n = (size_t)nx * ny, plane = (size_t)nxt * nyt;
    double rms, maxabs;
    orc_divb(P, s[ORC_BX], s[ORC_BY], &rms, &maxabs);
    out[0] = nx;
    out[1] = ny;
    out[2] = ng;
    out[3] = snapshot_rate;
    out[4] = P->dx;
    out[5] = P->dy;
    out[6] = dt;
    out[7] = rms;
    out[8] = maxabs;
    double* prim = (double*)malloc(6 * n * sizeof(double));
    double* rho_f = prim;
    double* vx = prim + n;
    double* vy = prim + 2 * n;
    double* p = prim + 3 * n;
    double* bxc = prim + 4 * n;
    double* byc = prim + 5 * n;
    orc_primitives(P, s, rho_f, vx, vy, p, bxc, byc);
    const double* src[7] = {rho_f, s[ORC_E], p, vx, vy, bxc, byc};
    for (int q = 0; q < 7; ++q)
        for (int J = 0; J < nyt; ++J)
            for (int I = 0; I < nxt; ++I) {
                const int i = ((I - ng) % nx + nx) % nx, j = ((J - ng) % ny + ny) % ny;
                out[9 + q * plane + (size_t)J * nxt + I] = src[q][(size_t)j * nx + i];
            }
    free(prim);
}

/* ---------------------------------------------------------------- MUSCL (MUSCL.hpp) */

/* MUSCL.hpp:11-17 */
static inline double minmod(double a, double b) {
    if (a * b > 0.0) return (fabs(a) < fabs(b)) ? a : b;
    return 0.0;
}

/* MUSCL.hpp:26-47: lower (L) and upper (R) extrapolation of a cell from its two neighbours. */
static inline void recon(double fm, double f0, double fp, double* L, double* R) {
    const double s = minmod(f0 - fm, fp - f0);
    *L = f0 - 0.5 * s;
    *R = f0 + 0.5 * s;
}

/* ---------------------------------------------------------------- HLL (HLL.hpp) */

typedef struct { double rho, vx, vy, p, bx, by; } prim_t;
typedef struct { double rho, mx, my, E, bx, by; } flux_t;

/* HLL.hpp:31-47 ConservedState::fromPrimitive */
static inline flux_t to_conserved(prim_t w) {
    flux_t u;
    u.rho = w.rho;
    u.mx = w.rho * w.vx;
    u.my = w.rho * w.vy;
    const double v2 = w.vx * w.vx + w.vy * w.vy;
    const double b2 = w.bx * w.bx + w.by * w.by;
    u.E = w.p / (GAMMA_GAS - 1.0) + 0.5 * w.rho * v2 + 0.5 * b2;
    u.bx = w.bx;
    u.by = w.by;
    return u;
}

/* HLL.hpp:61-81 */
static inline flux_t flux_x(prim_t p) {
    const double v2 = p.vx * p.vx + p.vy * p.vy;
    const double b2 = p.bx * p.bx + p.by * p.by;
    const double pt = p.p + 0.5 * b2;
    const double vb = p.vx * p.bx + p.vy * p.by;
    const double E = p.p / (GAMMA_GAS - 1.0) + 0.5 * (p.rho * v2 + b2);
    flux_t F;
    F.rho = p.rho * p.vx;
    F.mx = p.rho * p.vx * p.vx + pt - p.bx * p.bx;
    F.my = p.rho * p.vx * p.vy - p.bx * p.by;
    F.E = (E + pt) * p.vx - p.bx * vb;
    F.bx = 0.0;
    F.by = p.vx * p.by - p.vy * p.bx;
    return F;
}

/* HLL.hpp:84-104 */
static inline flux_t flux_y(prim_t p) {
    const double v2 = p.vx * p.vx + p.vy * p.vy;
    const double b2 = p.bx * p.bx + p.by * p.by;
    const double pt = p.p + 0.5 * b2;
    const double vb = p.vx * p.bx + p.vy * p.by;
    const double E = p.p / (GAMMA_GAS - 1.0) + 0.5 * (p.rho * v2 + b2);
    flux_t F;
    F.rho = p.rho * p.vy;
    F.my = p.rho * p.vy * p.vy + pt - p.by * p.by;
    F.mx = p.rho * p.vx * p.vy - p.bx * p.by;
    F.E = (E + pt) * p.vy - p.by * vb;
    F.by = 0.0;
    F.bx = p.vy * p.bx - p.vx * p.by;
    return F;
}

/* HLL.hpp:107-122 */
static inline double fast_speed(prim_t p, double bn) {
    const double b2 = p.bx * p.bx + p.by * p.by;
    const double a2 = GAMMA_GAS * p.p / p.rho;
    const double t2 = b2 / p.rho;
    const double n2 = bn * bn / p.rho;
    const double sum = t2 + a2;
    const double term = sum * sum - 4.0 * a2 * n2;
    return sqrt(0.5 * (sum + sqrt(term > 0.0 ? term : 0.0)));
}

static inline double dmin(double a, double b) { return (b < a) ? b : a; } /* std::min */
static inline double dmax(double a, double b) { return (a < b) ? b : a; } /* std::max */

/* HLL.hpp:126-172 (x) and :177-218 (y): the normal direction is selected by `dir`. */
static inline flux_t hll(prim_t L, prim_t R, int dir) {
    const flux_t FL = dir == 0 ? flux_x(L) : flux_y(L);
    const flux_t FR = dir == 0 ? flux_x(R) : flux_y(R);
    const double cL = fast_speed(L, dir == 0 ? L.bx : L.by);
    const double cR = fast_speed(R, dir == 0 ? R.bx : R.by);
    const double vnL = dir == 0 ? L.vx : L.vy;
    const double vnR = dir == 0 ? R.vx : R.vy;
    const double sL = dmin(vnL - cL, vnR - cR);
    const double sR = dmax(vnL + cL, vnR + cR);
    if (sL >= 0) return FL;
    if (sR <= 0) return FR;
    const flux_t UL = to_conserved(L), UR = to_conserved(R);
    const double inv = 1.0 / (sR - sL);
    flux_t F;
    F.rho = (sR * FL.rho - sL * FR.rho + sL * sR * (UR.rho - UL.rho)) * inv;
    F.mx = (sR * FL.mx - sL * FR.mx + sL * sR * (UR.mx - UL.mx)) * inv;
    F.my = (sR * FL.my - sL * FR.my + sL * sR * (UR.my - UL.my)) * inv;
    F.E = (sR * FL.E - sL * FR.E + sL * sR * (UR.E - UL.E)) * inv;
    if (dir == 0) {
        F.bx = 0.0;
        F.by = (sR * FL.by - sL * FR.by + sL * sR * (UR.by - UL.by)) * inv;
    } else {
        F.bx = (sR * FL.bx - sL * FR.bx + sL * sR * (UR.bx - UL.bx)) * inv;
        F.by = 0.0;
    }
    return F;
}

/* ---------------------------------------------------------------- explicit RHS (solvers.hpp) */

/* solvers.hpp:326,333 corner-velocity test. GCC resolves the unqualified abs(double) there to
 * int abs(int) (only <cmath>/<cstdlib> are in scope), so the test is "(int)v == 0"; on x86 an
 * out-of-range or NaN conversion yields INT_MIN, whose abs is still negative (< 1e-12). */
static inline int ct_average(double v, int mode) {
    if (mode == 1) return fabs(v) < 1e-12;
    return !(fabs(v) >= 1.0 && fabs(v) < 2147483648.0);
}

void orc_explicit_rhs(const orc_params* P, const double* const s[6], double* const f[6]) {
    const int nx = P->nx, ny = P->ny;
    const size_t n = (size_t)nx * ny;
    double* buf = (double*)malloc(sizeof(double) * n * 20);
    double *rho = buf, *vx = buf + n, *vy = buf + 2 * n, *p = buf + 3 * n, *bxc = buf + 4 * n,
           *byc = buf + 5 * n;
    /* x-face (right face of cell i) fluxes and y-face (top face of cell j) fluxes */
    double *fx_rho = buf + 6 * n, *fx_mx = buf + 7 * n, *fx_my = buf + 8 * n, *fx_E = buf + 9 * n,
           *fx_by = buf + 10 * n;
    double *fy_rho = buf + 11 * n, *fy_mx = buf + 12 * n, *fy_my = buf + 13 * n,
           *fy_E = buf + 14 * n, *fy_bx = buf + 15 * n;
    double* ez = buf + 16 * n;

    orc_primitives(P, s, rho, vx, vy, p, bxc, byc); /* solvers.hpp:395-396 */

    /* solvers.hpp:348-391 flux_population + :216-251 generate_cell_properties +
     * MUSCL.hpp:82-119. Face (i+1/2, j): L state = upper x-extrapolation of cell i, R state =
     * lower x-extrapolation of cell i+1; normal B = bxf(i+1). */
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            prim_t L, R;
            double t;
            recon(AT(rho, i - 1, j), AT(rho, i, j), AT(rho, i + 1, j), &t, &L.rho);
            recon(AT(vx, i - 1, j), AT(vx, i, j), AT(vx, i + 1, j), &t, &L.vx);
            recon(AT(vy, i - 1, j), AT(vy, i, j), AT(vy, i + 1, j), &t, &L.vy);
            recon(AT(p, i - 1, j), AT(p, i, j), AT(p, i + 1, j), &t, &L.p);
            recon(AT(byc, i - 1, j), AT(byc, i, j), AT(byc, i + 1, j), &t, &L.by);
            recon(AT(rho, i, j), AT(rho, i + 1, j), AT(rho, i + 2, j), &R.rho, &t);
            recon(AT(vx, i, j), AT(vx, i + 1, j), AT(vx, i + 2, j), &R.vx, &t);
            recon(AT(vy, i, j), AT(vy, i + 1, j), AT(vy, i + 2, j), &R.vy, &t);
            recon(AT(p, i, j), AT(p, i + 1, j), AT(p, i + 2, j), &R.p, &t);
            recon(AT(byc, i, j), AT(byc, i + 1, j), AT(byc, i + 2, j), &R.by, &t);
            L.bx = R.bx = AT(s[ORC_BX], i + 1, j);
            const flux_t F = hll(L, R, 0);
            const size_t id = (size_t)j * nx + i;
            fx_rho[id] = F.rho; fx_mx[id] = F.mx; fx_my[id] = F.my; fx_E[id] = F.E; fx_by[id] = F.by;
        }
    /* Face (i, j+1/2): D state = upper y-extrapolation of cell j, U state = lower y-extrapolation
     * of cell j+1; tangential B from bxc, normal B = byf(j+1). */
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            prim_t D, U;
            double t;
            recon(AT(rho, i, j - 1), AT(rho, i, j), AT(rho, i, j + 1), &t, &D.rho);
            recon(AT(vx, i, j - 1), AT(vx, i, j), AT(vx, i, j + 1), &t, &D.vx);
            recon(AT(vy, i, j - 1), AT(vy, i, j), AT(vy, i, j + 1), &t, &D.vy);
            recon(AT(p, i, j - 1), AT(p, i, j), AT(p, i, j + 1), &t, &D.p);
            recon(AT(bxc, i, j - 1), AT(bxc, i, j), AT(bxc, i, j + 1), &t, &D.bx);
            recon(AT(rho, i, j), AT(rho, i, j + 1), AT(rho, i, j + 2), &U.rho, &t);
            recon(AT(vx, i, j), AT(vx, i, j + 1), AT(vx, i, j + 2), &U.vx, &t);
            recon(AT(vy, i, j), AT(vy, i, j + 1), AT(vy, i, j + 2), &U.vy, &t);
            recon(AT(p, i, j), AT(p, i, j + 1), AT(p, i, j + 2), &U.p, &t);
            recon(AT(bxc, i, j), AT(bxc, i, j + 1), AT(bxc, i, j + 2), &U.bx, &t);
            D.by = U.by = AT(s[ORC_BY], i, j + 1);
            const flux_t F = hll(D, U, 1);
            const size_t id = (size_t)j * nx + i;
            fy_rho[id] = F.rho; fy_mx[id] = F.mx; fy_my[id] = F.my; fy_E[id] = F.E; fy_bx[id] = F.bx;
        }
    /* solvers.hpp:294-346 cell_corner_electric_fields at corner (i,j) */
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const double eN = -AT(fx_by, i - 1, j);
            const double eS = -AT(fx_by, i - 1, j - 1);
            const double eE = AT(fy_bx, i, j - 1);
            const double eW = AT(fy_bx, i - 1, j - 1);
            const double vxc = 0.25 * (AT(vx, i, j) + AT(vx, i - 1, j) + AT(vx, i, j - 1) +
                                       AT(vx, i - 1, j - 1));
            const double vyc = 0.25 * (AT(vy, i, j) + AT(vy, i - 1, j) + AT(vy, i, j - 1) +
                                       AT(vy, i - 1, j - 1));
            double ezy, ezx;
            if (ct_average(vyc, P->ct_abs_mode)) ezy = 0.5 * (eS + eN);
            else ezy = (vyc > 0.0) ? eS : eN;
            if (ct_average(vxc, P->ct_abs_mode)) ezx = 0.5 * (eE + eW);
            else ezx = (vxc > 0.0) ? eW : eE;
            ez[(size_t)j * nx + i] = 0.5 * (ezx + ezy);
        }
    /* solvers.hpp:253-292 time_derivatives */
    const double dx = P->dx, dy = P->dy;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const size_t id = (size_t)j * nx + i;
            f[ORC_RHO][id] = -((fx_rho[id] - AT(fx_rho, i - 1, j)) / dx + (fy_rho[id] - AT(fy_rho, i, j - 1)) / dy);
            f[ORC_E][id] = -((fx_E[id] - AT(fx_E, i - 1, j)) / dx + (fy_E[id] - AT(fy_E, i, j - 1)) / dy);
            f[ORC_MX][id] = -((fx_mx[id] - AT(fx_mx, i - 1, j)) / dx + (fy_mx[id] - AT(fy_mx, i, j - 1)) / dy);
            f[ORC_MY][id] = -((fx_my[id] - AT(fx_my, i - 1, j)) / dx + (fy_my[id] - AT(fy_my, i, j - 1)) / dy);
            f[ORC_BX][id] = -(AT(ez, i, j + 1) - ez[id]) / dy;
            f[ORC_BY][id] = (AT(ez, i + 1, j) - ez[id]) / dx;
        }
    free(buf);
}

/* ---------------------------------------------------------------- resistive term + CG */

void orc_corner_current_rhs(const orc_params* P, const double* bxf, const double* byf, double* rhs) {
    const int nx = P->nx, ny = P->ny;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const size_t id = (size_t)j * nx + i;
            const double dBy_dx = (byf[id] - AT(byf, i - 1, j)) / P->dx;  /* solvers.hpp:457 */
            const double dBx_dy = (bxf[id] - AT(bxf, i, j - 1)) / P->dy;  /* solvers.hpp:458 */
            rhs[id] = P->eta * (dBy_dx - dBx_dy);                          /* solvers.hpp:460 */
        }
}

/* (I - alpha L) p, row r = j*nx+i, summed over the row's entries in increasing column index
 * (the order of the compressed, symmetric matrix of solvers.hpp:404-443). */
static void apply_matrix(const orc_params* P, double alpha, const double* p, double* out) {
    const int nx = P->nx, ny = P->ny;
    const double cx = alpha / (P->dx * P->dx);   /* solvers.hpp:409 */
    const double cy = alpha / (P->dy * P->dy);   /* solvers.hpp:410 */
    const double diag = 1 + 2 * (cx + cy);       /* solvers.hpp:432 */
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            long col[5];
            double val[5];
            const long r = (long)j * nx + i;
            col[0] = (long)wrap(j - 1, ny) * nx + i; val[0] = -cy;
            col[1] = (long)wrap(j + 1, ny) * nx + i; val[1] = -cy;
            col[2] = (long)j * nx + wrap(i - 1, nx); val[2] = -cx;
            col[3] = (long)j * nx + wrap(i + 1, nx); val[3] = -cx;
            col[4] = r; val[4] = diag;
            /* insertion sort by column; equal columns are merged (duplicates summed) */
            for (int a = 1; a < 5; ++a)
                for (int b = a; b > 0 && col[b] < col[b - 1]; --b) {
                    long tc = col[b]; col[b] = col[b - 1]; col[b - 1] = tc;
                    double tv = val[b]; val[b] = val[b - 1]; val[b - 1] = tv;
                }
            double acc = 0.0;
            int a = 0;
            while (a < 5) {
                double v = val[a];
                int b = a + 1;
                while (b < 5 && col[b] == col[a]) v += val[b++];
                acc += v * p[col[a]];
                a = b;
            }
            out[r] = acc;
        }
}

long orc_cg_solve(const orc_params* P, double alpha, const double* b, double* x, long* iters_out) {
    const long n = (long)P->nx * P->ny;
    const double cx = alpha / (P->dx * P->dx), cy = alpha / (P->dy * P->dy);
    const double d = 1 + 2 * (cx + cy);
    const double invdiag = (d == 0.0) ? 1.0 : 1.0 / d;
    const double tol = P->cg_tol > 0 ? P->cg_tol : DBL_EPSILON;
    const long max_iters = P->cg_max_iters > 0 ? P->cg_max_iters : 2 * n;
    long products = 0;
    for (long k = 0; k < n; ++k) x[k] = 0.0;
    double bb = 0.0;
    for (long k = 0; k < n; ++k) bb += b[k] * b[k];
    if (iters_out) *iters_out = 0;
    if (bb == 0.0) return 0;
    const double threshold = fmax(tol * tol * bb, DBL_MIN);
    double* r = (double*)malloc(sizeof(double) * n * 3);
    double *p = r + n, *q = r + 2 * n;
    for (long k = 0; k < n; ++k) r[k] = b[k];
    double rr = bb;
    if (rr < threshold) { free(r); return 0; }
    double absNew = 0.0;
    for (long k = 0; k < n; ++k) { p[k] = invdiag * r[k]; absNew += r[k] * p[k]; }
    long i = 0;
    while (i < max_iters) {
        apply_matrix(P, alpha, p, q);
        ++products;
        double pq = 0.0;
        for (long k = 0; k < n; ++k) pq += p[k] * q[k];
        const double a = absNew / pq;
        for (long k = 0; k < n; ++k) x[k] += a * p[k];
        rr = 0.0;
        for (long k = 0; k < n; ++k) { r[k] -= a * q[k]; rr += r[k] * r[k]; }
        if (rr < threshold) break;
        const double absOld = absNew;
        absNew = 0.0;
        for (long k = 0; k < n; ++k) absNew += r[k] * (invdiag * r[k]);
        const double beta = absNew / absOld;
        for (long k = 0; k < n; ++k) p[k] = invdiag * r[k] + beta * p[k];
        ++i;
    }
    if (iters_out) *iters_out = i;
    free(r);
    return products;
}

long orc_resistive_rate(const orc_params* P, const double* bxf, const double* byf, double alpha,
                        double* bx_rate, double* by_rate) {
    const int nx = P->nx, ny = P->ny;
    const size_t n = (size_t)nx * ny;
    double* rhs = (double*)malloc(sizeof(double) * n * 2);
    double* ez = rhs + n;
    long products = 0;
    orc_corner_current_rhs(P, bxf, byf, rhs);
    if (alpha >= 0) products = orc_cg_solve(P, alpha, rhs, ez, NULL);  /* solvers.hpp:469 */
    else memcpy(ez, rhs, sizeof(double) * n);                            /* solvers.hpp:470 */
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const size_t id = (size_t)j * nx + i;
            bx_rate[id] = -(AT(ez, i, j + 1) - ez[id]) / P->dy;   /* solvers.hpp:484 */
            by_rate[id] = (AT(ez, i + 1, j) - ez[id]) / P->dx;    /* solvers.hpp:485 */
        }
    free(rhs);
    return products;
}

/* ---------------------------------------------------------------- IMEX (solvers.hpp:491-613) */

/* Grid::computePrimitives floors the density in place (Grid.hpp:115). */
static void floor_density(size_t n, double* rho) {
    for (size_t k = 0; k < n; ++k)
        if (rho[k] < RHO_FLOOR) rho[k] = RHO_FLOOR;
}

void orc_imex_step(const orc_params* P, double* const s[6], double dt, double alpha,
                   long* cg_products) {
    const size_t n = (size_t)P->nx * P->ny;
    /* solvers.hpp:39-66 ARS(2,2,2) tableau */
    const double gamma = (2.0 - sqrt(2.0)) / 2.0;
    const double delta = 1.0 - (1.0 / (2.0 * gamma));
    const double A_ex3 = gamma, A_ex6 = delta, A_ex7 = 1.0 - delta;
    const double A_im4 = gamma, A_im7 = 1.0 - gamma;
    const double b_ex0 = delta, b_ex1 = 1.0 - delta, b_im1 = 1.0 - gamma, b_im2 = gamma;

    double* buf = (double*)malloc(sizeof(double) * n * 30);
    double *f1[6], *f2[6], *u1[6], *u2[6], *ini[6];
    for (int k = 0; k < 6; ++k) {
        f1[k] = buf + (size_t)k * n;
        f2[k] = buf + (size_t)(6 + k) * n;
        u1[k] = buf + (size_t)(12 + k) * n;
        u2[k] = buf + (size_t)(18 + k) * n;
        ini[k] = buf + (size_t)(24 + k) * n;
    }
    double* sx = (double*)malloc(sizeof(double) * n * 4);
    double *sy = sx + n, *gx = sx + 2 * n, *gy = sx + 3 * n;
    long prod[2] = {0, 0};

    for (int k = 0; k < 6; ++k) memcpy(ini[k], s[k], sizeof(double) * n); /* :493 copy */
    /* :495-496 f1 = explicit_rhs(U^n); explicit_rhs floors U^n's density in place */
    orc_explicit_rhs(P, (const double* const*)s, f1);
    floor_density(n, s[ORC_RHO]);
    /* :499 g1 enters only with the zero weights A_im[3], A_im[6], b_im[0]: skipped */

    /* :501-520 U1 = U^n(copy) + dt*A_ex[3]*f1 */
    const double c1 = dt * A_ex3;
    for (int k = 0; k < 6; ++k) {
        memcpy(u1[k], ini[k], sizeof(double) * n);
        for (size_t q = 0; q < n; ++q) u1[k][q] += f1[k][q] * c1;
    }
    floor_density(n, u1[ORC_RHO]);                                         /* :522-523 */
    prod[0] = orc_resistive_rate(P, u1[ORC_BX], u1[ORC_BY], alpha, sx, sy); /* :526 */
    const double diag = dt * A_im4;                                         /* :503 */
    for (size_t q = 0; q < n; ++q) {                                        /* :528-529 */
        u1[ORC_BX][q] += sx[q] * diag;
        u1[ORC_BY][q] += sy[q] * diag;
    }
    orc_explicit_rhs(P, (const double* const*)u1, f2);                      /* :535 */
    orc_resistive_rate(P, u1[ORC_BX], u1[ORC_BY], -1.0, gx, gy);            /* :537 g2 */

    /* :543-566 U2 = U^n(copy) + dt*A_ex[6]*f1 + dt*A_ex[7]*f2 (+0*g1) + dt*A_im[7]*g2 */
    const double c2 = dt * A_ex6, c3 = dt * A_ex7, ci3 = dt * A_im7;
    for (int k = 0; k < 6; ++k) {
        memcpy(u2[k], ini[k], sizeof(double) * n);
        for (size_t q = 0; q < n; ++q) u2[k][q] += f1[k][q] * c2;
        for (size_t q = 0; q < n; ++q) u2[k][q] += f2[k][q] * c3;
    }
    for (size_t q = 0; q < n; ++q) {
        u2[ORC_BX][q] += gx[q] * ci3;
        u2[ORC_BY][q] += gy[q] * ci3;
    }
    floor_density(n, u2[ORC_RHO]);                                          /* :568-569 */
    prod[1] = orc_resistive_rate(P, u2[ORC_BX], u2[ORC_BY], alpha, sx, sy); /* :571 */
    for (size_t q = 0; q < n; ++q) {                                        /* :573-574 */
        u2[ORC_BX][q] += sx[q] * diag;
        u2[ORC_BY][q] += sy[q] * diag;
    }
    double* g3x = sx;
    double* g3y = sy;
    orc_resistive_rate(P, u2[ORC_BX], u2[ORC_BY], -1.0, g3x, g3y);          /* :579 g3 */

    /* :585-608 final combination on the (density-floored) U^n */
    const double fc1 = dt * b_ex0, fc2 = dt * b_ex1, gc2 = dt * b_im1, gc3 = dt * b_im2;
    for (int k = 0; k < 6; ++k)
        for (size_t q = 0; q < n; ++q) s[k][q] += f1[k][q] * fc1;
    for (int k = 0; k < 6; ++k)
        for (size_t q = 0; q < n; ++q) s[k][q] += f2[k][q] * fc2;
    for (size_t q = 0; q < n; ++q) {
        s[ORC_BX][q] += gx[q] * gc2;
        s[ORC_BY][q] += gy[q] * gc2;
    }
    for (size_t q = 0; q < n; ++q) {
        s[ORC_BX][q] += g3x[q] * gc3;
        s[ORC_BY][q] += g3y[q] * gc3;
    }
    floor_density(n, s[ORC_RHO]);                                           /* :610-611 */
    if (cg_products) { cg_products[0] = prod[0]; cg_products[1] = prod[1]; }
    free(sx);
    free(buf);
}

/* ---------------------------------------------------------------- diagnostics */

double orc_cfl_dt(const orc_params* P, const double* const s[6], double courant, double safety) {
    const int nx = P->nx, ny = P->ny;
    const size_t n = (size_t)nx * ny;
    double* buf = (double*)malloc(sizeof(double) * n * 6);
    double *rho = buf, *vx = buf + n, *vy = buf + 2 * n, *p = buf + 3 * n, *bxc = buf + 4 * n,
           *byc = buf + 5 * n;
    orc_primitives(P, s, rho, vx, vy, p, bxc, byc);
    const double dx = P->dx, dy = P->dy;
    double dt_res = INFINITY;                                               /* diagnostics.hpp:52 */
    if (P->eta != 0.0) dt_res = dmin(dx, dy) * dmin(dx, dy) / (4.0 * P->eta);
    double smax = 1e-8;                                                     /* :58 */
    for (size_t k = 0; k < n; ++k) {
        const double r = dmax(rho[k], 1e-8), pr = dmax(p[k], 1e-8);
        const double a2 = GAMMA_GAS * pr / r;
        const double b2 = (bxc[k] * bxc[k] + byc[k] * byc[k]) / r;
        const double s_ = sqrt(a2 + b2) + sqrt(vx[k] * vx[k] + vy[k] * vy[k]);
        if (s_ > smax) smax = s_;
    }
    free(buf);
    const double dt_hyp = courant * dmin(dx, dy) / smax;                    /* :82 */
    return dmin(dt_hyp, dt_res) * safety;                                   /* :83-84 */
}

void orc_divb(const orc_params* P, const double* bxf, const double* byf, double* rms,
              double* maxabs) {
    const int nx = P->nx, ny = P->ny;
    double s2 = 0.0, mx = 0.0;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const size_t id = (size_t)j * nx + i;
            const double d = (AT(bxf, i + 1, j) - bxf[id]) / P->dx + (AT(byf, i, j + 1) - byf[id]) / P->dy;
            s2 += d * d;
            if (fabs(d) > mx) mx = fabs(d);
        }
    *rms = sqrt(s2 / (nx * ny));
    *maxabs = mx;
}

/* ---------------------------------------------------------------- initial conditions */

/* Face B from a corner vector potential (benchmarks.hpp:58-59, :399-400), then conserved state
 * with E built from the FACE values (benchmarks.hpp:61-62 / :402-403). */
static void fill_from_potential(const orc_params* P, double* const s[6], const double* az,
                                double rho0, double p0, const double* vx, const double* vy) {
    const int nx = P->nx, ny = P->ny;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const size_t id = (size_t)j * nx + i;
            const size_t a = (size_t)j * (nx + 1) + i;
            const double bx = (az[a + (nx + 1)] - az[a]) / P->dy;
            const double by = -(az[a + 1] - az[a]) / P->dx;
            prim_t w = {rho0, vx[id], vy[id], p0, bx, by};
            flux_t u = to_conserved(w);
            s[ORC_RHO][id] = u.rho; s[ORC_MX][id] = u.mx; s[ORC_MY][id] = u.my; s[ORC_E][id] = u.E;
            s[ORC_BX][id] = bx; s[ORC_BY][id] = by;
        }
}

void orc_init_orszag_tang(const orc_params* P, double* const s[6]) {
    const int nx = P->nx, ny = P->ny;
    double* az = (double*)malloc(sizeof(double) * (size_t)(nx + 1) * (ny + 1));
    double* v = (double*)malloc(sizeof(double) * (size_t)nx * ny * 2);
    for (int j = 0; j <= ny; ++j)
        for (int i = 0; i <= nx; ++i) {
            const double xc = i * P->dx, yc = j * P->dy;                    /* :37-38 */
            az[(size_t)j * (nx + 1) + i] = 0.5 * cos(2 * xc) + cos(yc);     /* :41 */
        }
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const double x = (i + 0.5) * P->dx, y = (j + 0.5) * P->dy;      /* :53-54 */
            v[(size_t)j * nx + i] = -sin(y);                                /* :56 */
            v[(size_t)nx * ny + (size_t)j * nx + i] = sin(x);               /* :57 */
        }
    fill_from_potential(P, s, az, 25.0 / 9.0, 5.0 / 3.0, v, v + (size_t)nx * ny); /* :27-28 */
    free(az);
    free(v);
}

void orc_init_sine_wave(const orc_params* P, double* const s[6], double az_amp, double kx,
                        double ky, int use_sin) {
    const int nx = P->nx, ny = P->ny;
    const double pi = 3.14159265359;                                         /* :363 */
    if (kx <= 0) kx = 2 * pi / (nx * P->dx);                                 /* :365 */
    if (ky <= 0) ky = 2 * pi / (ny * P->dy);                                 /* :366 */
    double* az = (double*)malloc(sizeof(double) * (size_t)(nx + 1) * (ny + 1));
    double* v = (double*)calloc((size_t)nx * ny * 2, sizeof(double));
    for (int j = 0; j <= ny; ++j)
        for (int i = 0; i <= nx; ++i) {
            const double xl = i * P->dx, yb = j * P->dy;                    /* :384-385 */
            const double fx = use_sin ? sin(kx * xl) : cos(kx * xl);
            az[(size_t)j * (nx + 1) + i] = az_amp * fx * sin(ky * yb);      /* :387 */
        }
    fill_from_potential(P, s, az, 1.0, 1.0, v, v + (size_t)nx * ny);
    free(az);
    free(v);
}
