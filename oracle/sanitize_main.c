/* Test infrastructure only: a driver for the CPU oracle built with AddressSanitizer and
 * UndefinedBehaviorSanitizer (`make sanitize`), so that a memory error or undefined behaviour in
 * the oracle -- the checker every parity test relies on -- stops the run with a report instead of
 * skewing a comparison.
 *
 * It exercises every oracle entry point on small grids (dx != dy, odd sizes): Orszag-Tang 36 x 28
 * for 4 CFL steps (CFL step, IMEX with both solves, div B, primitives, explicit and implicit
 * resistive rates, a snapshot with 2 ghost layers) and the decaying sine wave 32 x 20 for 3 fixed
 * steps in the true-|v| corner mode with a capped solver. It writes the final states to the file
 * named by argv[1] (raw doubles: 6 planes of each run, then the snapshot), which the test compares
 * with the same calls through the unsanitized liboracle.so. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "mhd_oracle.h"

static double* alloc_planes(int n, double* s[6]) {
    double* pool = (double*)calloc((size_t)6 * n, sizeof(double));
    if (!pool) return NULL;
    for (int k = 0; k < 6; ++k) s[k] = pool + (size_t)k * n;
    return pool;
}

static int run_case(const orc_params* P, int orszag_tang, int steps, double fixed_dt, FILE* out,
                    double* snap, int ng) {
    const int n = P->nx * P->ny;
    double* s[6];
    double* pool = alloc_planes(n, s);
    double* aux = (double*)calloc((size_t)8 * n, sizeof(double));
    if (!pool || !aux) return 1;
    if (orszag_tang) orc_init_orszag_tang(P, s);
    else orc_init_sine_wave(P, s, 1e-3, -1.0, -1.0, 1);
    double dt = fixed_dt;
    for (int t = 0; t < steps; ++t) {
        if (fixed_dt <= 0) dt = orc_cfl_dt(P, (const double* const*)s, 0.4, 0.9);
        long prods[2] = {0, 0};
        const double g = (2.0 - sqrt(2.0)) / 2.0;  /* ARS(2,2,2) gamma; the driver's matrix alpha */
        orc_imex_step(P, s, dt, dt * P->eta * g, prods);
    }
    double rms = 0, mx = 0;
    orc_divb(P, s[ORC_BX], s[ORC_BY], &rms, &mx);
    orc_primitives(P, (const double* const*)s, aux, aux + n, aux + 2 * n, aux + 3 * n, aux + 4 * n,
                   aux + 5 * n);
    double* f[6];
    double* rates = alloc_planes(n, f);
    if (!rates) return 1;
    orc_explicit_rhs(P, (const double* const*)s, f);
    orc_corner_current_rhs(P, s[ORC_BX], s[ORC_BY], aux + 6 * n);
    orc_resistive_rate(P, s[ORC_BX], s[ORC_BY], -1.0, aux, aux + n);
    orc_resistive_rate(P, s[ORC_BX], s[ORC_BY], 1e-3, aux + 2 * n, aux + 3 * n);
    if (snap) orc_snapshot(P, (const double* const*)s, ng, 5, dt, snap);
    const size_t wrote = fwrite(pool, sizeof(double), (size_t)6 * n, out);
    free(rates);
    free(aux);
    free(pool);
    return wrote == (size_t)6 * n ? 0 : 1;
}

int main(int argc, char** argv) {
    if (argc != 2) return 2;
    FILE* out = fopen(argv[1], "wb");
    if (!out) return 2;
    const double pi = 3.14159265358979323846;
    orc_params ot = {36, 28, 2 * pi / 36, 1.7 * pi / 28, 1e-2, 0, 0.0, 0};
    orc_params sw = {32, 20, 2 * pi / 32, 2 * pi / 20, 0.5, 1, 1e-12, 40};
    const int ng = 2;
    const size_t snap_n = 9 + (size_t)7 * (ot.nx + 2 * ng) * (ot.ny + 2 * ng);
    double* snap = (double*)calloc(snap_n, sizeof(double));
    int rc = snap ? 0 : 1;
    if (!rc) rc = run_case(&ot, 1, 4, 0.0, out, snap, ng);
    if (!rc) rc = run_case(&sw, 0, 3, 1e-3, out, NULL, ng);
    if (!rc && fwrite(snap, sizeof(double), snap_n, out) != snap_n) rc = 1;
    free(snap);
    fclose(out);
    return rc;
}
