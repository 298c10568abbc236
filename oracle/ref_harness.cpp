// Test infrastructure only (never shipped, never on the product path).
//
// Wraps the reference solver's own headers -- include/Grid.hpp, MUSCL.hpp, HLL.hpp, solvers.hpp,
// diagnostics.hpp, benchmarks.hpp of RikibabManos/Magnetohydrodynamics_Simulator, compiled
// unmodified from where they lie (see oracle/Makefile) -- behind a small C ABI, so the tests and the
// CPU baseline can drive the reference's real IMEX step without its interactive main().
// Eigen3 is replaced by oracle/eigen_subset (project-written; documented CG defaults).
//
// What each entry point mirrors in the reference:
//   ref_create            src/integrator_main.cpp:34-48   (grids, workspace, tableau, solver)
//   ref_init_orszag_tang  benchmarks.hpp:15-76 + integrator_main.cpp:52-53
//   ref_init_dsw          benchmarks.hpp:352-417 + integrator_main.cpp:52-53
//   ref_init_fixture      benchmarks.hpp:78-350 (Alfven wave, Gaussian pulse, acoustic wave,
//                         sausage, kink) + integrator_main.cpp:52-53
//   ref_set_alpha         integrator_main.cpp:58-60 / :87-95 (generate_A_matrix + compute)
//   ref_step              integrator_main.cpp:99 (IMEX, solvers.hpp:491-613)
//   ref_cfl               diagnostics.hpp:44-88
//   ref_divb              diagnostics.hpp:15-42
//   ref_explicit_rhs      solvers.hpp:393-402 (on a copy of the state)
//   ref_run               integrator_main.cpp:76-112 (dt loop, matrix regeneration rule)
//   ref_write_snapshot    integrator_main.cpp:107-109 (ghost fill, primitives,
//                         write_data_to_binary_file into output/ of the working directory)
#include <iostream>
#include <fstream>
#include <vector>
#include <array>
#include <string>
#include <cmath>
#include <cstdlib>
#include <sstream>
#include <iomanip>
#include <chrono>
#include "Grid.hpp"
#include "MUSCL.hpp"
#include "HLL.hpp"
#include "solvers.hpp"
#include <Eigen/Dense>
#include <Eigen/Sparse>
#include "diagnostics.hpp"
#include "benchmarks.hpp"

namespace {

using Solver = Eigen::ConjugateGradient<Eigen::SparseMatrix<double>, Eigen::Lower | Eigen::Upper>;

struct RefSim {
    Grid state, g1, g2;
    integrator_reserved_memory mem;
    ReconstructedValues rv;
    IMEX_Butcher_Tableus tab;
    Solver solver;
    std::vector<long> cg_products;  // matrix-vector products per implicit solve, in call order
    bool have_matrix = false;

    RefSim(int nx, int ny, double dx, double dy, double eta)
        : state(nx, ny, 2), g1(nx, ny, 2), g2(nx, ny, 2),
          mem(state.nxt * state.nyt, nx * ny, (state.nxt + 1) * (state.nyt + 1)),
          rv(static_cast<size_t>(state.nxt) * state.nyt) {
        state.cell_width = dx;
        state.cell_height = dy;
        state.resistivity = eta;
        g1 = state;
        g2 = state;
    }
};

void finish_setup(RefSim* s) {
    s->state.fillGhostPeriodic();
    s->state.computePrimitives();
}

}  // namespace

extern "C" {

void* ref_create(int nx, int ny, double dx, double dy, double eta) {
    return new RefSim(nx, ny, dx, dy, eta);
}

void ref_destroy(void* h) { delete static_cast<RefSim*>(h); }

void ref_init_orszag_tang(void* h) {
    RefSim* s = static_cast<RefSim*>(h);
    orszag_tang_initial_conditions(s->state, s->mem);
    finish_setup(s);
}

void ref_init_dsw(void* h) {
    RefSim* s = static_cast<RefSim*>(h);
    decaying_magnetic_sine_wave_initial_conditions(s->state, s->mem);
    finish_setup(s);
}

// which: 0 Alfven wave, 1 Gaussian density pulse, 2 acoustic wave, 3 sausage, 4 kink.
int ref_init_fixture(void* h, int which) {
    RefSim* s = static_cast<RefSim*>(h);
    switch (which) {
        case 0: alfven_wave_test_initial_values(s->state); break;
        case 1: gaussian_density_pulse_test_initial_values(s->state); break;
        case 2: acoustic_wave_test_initial_values(s->state); break;
        case 3: sausage_instability_initial_conditions(s->state); break;
        case 4: kink_instability_initial_conditions(s->state); break;
        default: return -1;
    }
    finish_setup(s);
    return 0;
}

// Dense row-major (j*nx + i) physical arrays -> padded Grid, then ghosts + primitives.
void ref_set_state(void* h, const double* rho, const double* mx, const double* my, const double* E,
                   const double* bxf, const double* byf) {
    RefSim* s = static_cast<RefSim*>(h);
    Grid& g = s->state;
    for (int j = 0; j < g.ny; ++j)
        for (int i = 0; i < g.nx; ++i) {
            const int id = g.indexC(g.gi(i), g.gj(j));
            const int d = j * g.nx + i;
            g.rho[id] = rho[d]; g.mx[id] = mx[d]; g.my[id] = my[d]; g.E[id] = E[d];
            g.bxf[id] = bxf[d]; g.byf[id] = byf[d];
        }
    finish_setup(s);
}

void ref_get_state(void* h, double* rho, double* mx, double* my, double* E, double* bxf,
                   double* byf) {
    RefSim* s = static_cast<RefSim*>(h);
    const Grid& g = s->state;
    for (int j = 0; j < g.ny; ++j)
        for (int i = 0; i < g.nx; ++i) {
            const int id = g.indexC(g.gi(i), g.gj(j));
            const int d = j * g.nx + i;
            rho[d] = g.rho[id]; mx[d] = g.mx[id]; my[d] = g.my[id]; E[d] = g.E[id];
            bxf[d] = g.bxf[id]; byf[d] = g.byf[id];
        }
}

void ref_get_primitives(void* h, double* vx, double* vy, double* p, double* bxc, double* byc) {
    RefSim* s = static_cast<RefSim*>(h);
    const Grid& g = s->state;
    for (int j = 0; j < g.ny; ++j)
        for (int i = 0; i < g.nx; ++i) {
            const int id = g.indexC(g.gi(i), g.gj(j));
            const int d = j * g.nx + i;
            vx[d] = g.vx[id]; vy[d] = g.vy[id]; p[d] = g.p[id]; bxc[d] = g.bxc[id]; byc[d] = g.byc[id];
        }
}

double ref_cfl(void* h) { return CFL_condition_checker(static_cast<RefSim*>(h)->state); }

void ref_set_alpha(void* h, double alpha) {
    RefSim* s = static_cast<RefSim*>(h);
    generate_A_matrix(s->state, s->mem, alpha);
    s->solver.compute(s->mem.A_matrix);
    s->have_matrix = true;
}

// One IMEX step; returns the matrix-vector products of its two implicit solves.
void ref_step(void* h, double dt, long* cg_products2) {
    RefSim* s = static_cast<RefSim*>(h);
    s->solver.product_log.clear();
    IMEX(s->state, s->g1, s->g2, s->mem, s->rv, s->tab, s->solver, dt);
    if (cg_products2) {
        cg_products2[0] = s->solver.product_log.size() > 0 ? static_cast<long>(s->solver.product_log[0]) : -1;
        cg_products2[1] = s->solver.product_log.size() > 1 ? static_cast<long>(s->solver.product_log[1]) : -1;
    }
}

void ref_write_snapshot(void* h, int frame_index, int snapshot_rate, double dt) {
    RefSim* s = static_cast<RefSim*>(h);
    s->state.fillGhostPeriodic();
    s->state.computePrimitives();
    write_data_to_binary_file(s->state, frame_index, snapshot_rate, dt);
}

void ref_divb(void* h, double* rms, double* maxabs) {
    divergence_checker_values v = calculate_current_div_B(static_cast<RefSim*>(h)->state);
    *rms = v.root_mean_square_div;
    *maxabs = v.max_norm_divergence;
}

// Explicit right-hand side of the current state, computed on a copy (state left untouched).
void ref_explicit_rhs(void* h, double* frho, double* fmx, double* fmy, double* fE, double* fbx,
                      double* fby) {
    RefSim* s = static_cast<RefSim*>(h);
    Grid work = s->state;
    global_state_dot f(s->mem.f1_rho, s->mem.f1_m_x, s->mem.f1_m_y, s->mem.f1_b_x_f,
                       s->mem.f1_b_y_f, s->mem.f1_E);
    explicit_rhs(work, f, s->rv, s->mem);
    for (int j = 0; j < work.ny; ++j)
        for (int i = 0; i < work.nx; ++i) {
            const int id = work.indexC(work.gi(i), work.gj(j));
            const int d = j * work.nx + i;
            frho[d] = s->mem.f1_rho[id]; fmx[d] = s->mem.f1_m_x[id]; fmy[d] = s->mem.f1_m_y[id];
            fE[d] = s->mem.f1_E[id]; fbx[d] = s->mem.f1_b_x_f[id]; fby[d] = s->mem.f1_b_y_f[id];
        }
}

// Implicit resistive rate of the current state's face B (solvers.hpp:445-489 with
// solve_implicitly = true); the matrix must have been set with ref_set_alpha.
void ref_implicit_rate(void* h, double* bx_rate, double* by_rate, double* ez_out) {
    RefSim* s = static_cast<RefSim*>(h);
    const Grid& g = s->state;
    resistive_B_term(g, s->mem.b_x_f_solved_1, s->mem.b_y_f_solved_1, s->solver, s->mem, true);
    for (int j = 0; j < g.ny; ++j)
        for (int i = 0; i < g.nx; ++i) {
            const int id = g.indexC(g.gi(i), g.gj(j));
            const int d = j * g.nx + i;
            bx_rate[d] = s->mem.b_x_f_solved_1[id];
            by_rate[d] = s->mem.b_y_f_solved_1[id];
        }
    if (ez_out) {
        // the right-hand side the solve saw (eta * J_z at corners), for inspection
        for (int k = 0; k < g.nx * g.ny; ++k) ez_out[k] = s->mem.Ez_corner_no_padding[k];
    }
}

long ref_last_cg_iterations(void* h) {
    return static_cast<long>(static_cast<RefSim*>(h)->solver.iterations());
}

// Driver loop of integrator_main.cpp:76-112 without I/O. dt_fixed == 0 selects the dynamic CFL
// step; dts_in (if non-null) supplies every step's dt instead. The realised dts are written to
// dts_out (if non-null). The matrix is regenerated only when dt moved by more than 1e-10
// relative, as the reference driver does.
void ref_run(void* h, int nsteps, double dt_fixed, const double* dts_in, double* dts_out,
             long* cg_products_out) {
    RefSim* s = static_cast<RefSim*>(h);
    Grid& g = s->state;
    const double gamma_im = s->tab.A_im[4];
    double first = dts_in ? dts_in[0] : ((dt_fixed == 0.0) ? CFL_condition_checker(g) : dt_fixed);
    double previous = first;
    ref_set_alpha(h, first * g.resistivity * gamma_im);
    for (int n = 0; n < nsteps; ++n) {
        double dt = dts_in ? dts_in[n] : ((dt_fixed == 0.0) ? CFL_condition_checker(g) : dt_fixed);
        if (g.resistivity > 0.0) {
            if (std::abs(dt - previous) > 1e-10 * dt) {
                ref_set_alpha(h, dt * g.resistivity * gamma_im);
            }
        }
        previous = dt;
        s->solver.product_log.clear();
        IMEX(g, s->g1, s->g2, s->mem, s->rv, s->tab, s->solver, dt);
        if (dts_out) dts_out[n] = dt;
        if (cg_products_out) {
            const auto& log = s->solver.product_log;
            cg_products_out[2 * n] = log.size() > 0 ? static_cast<long>(log[0]) : -1;
            cg_products_out[2 * n + 1] = log.size() > 1 ? static_cast<long>(log[1]) : -1;
        }
    }
}

}  // extern "C"
