// C++ drop-in call surface over the C ABI of mhd_b200.h, shaped like the reference's own functions
// so that RikibabManos/Magnetohydrodynamics_Simulator's driver (src/integrator_main.cpp) switches
// its hot path to the GPU by qualifying three calls with `mhd_b200::`:
//
//   generate_A_matrix(grid, workspace, alpha)        solvers.hpp:404-443 (+ solver.compute)
//   IMEX(grid, g1, g2, workspace, rv, tableau, solver, dt)   solvers.hpp:491-613
//   CFL_condition_checker(grid)                      diagnostics.hpp:44-88
//   write_data_to_binary_file(grid, frame, rate, dt) diagnostics.hpp:90-131
//
// The functions are templates over the caller's types, so this header needs none of the
// reference's headers; GridT must provide the members of the reference's Grid (Grid.hpp:9-26):
// nx, ny, ng, cell_width, cell_height, resistivity and the std::vector<double> fields rho, mx,
// my, E, bxf, byf, bxc, byc, vx, vy, p. The workspace, reconstruction, tableau and solver
// arguments are accepted and ignored: the GPU keeps its own workspace, and the matrix-free solver
// needs only alpha.
//
// Semantics match the reference call for call: IMEX advances the grid in place and leaves the
// ghost layers and the primitives (vx, vy, p, bxc, byc, floored rho) filled, as the reference's
// closing fillGhostPeriodic + computePrimitives do (solvers.hpp:610-611). Grid::Ez, the
// reference's internal corner-field scratch, is not written. Every call moves the state between
// host and device; for a device-resident run use mhd_run() of mhd_b200.h.
#pragma once

#include <cstdio>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>

#include "mhd_b200.h"

namespace mhd_b200 {

class Error : public std::runtime_error {
public:
    Error(mhd_status s, const char* where)
        : std::runtime_error(std::string(where) + ": " + mhd_status_string(s)), status(s) {}
    mhd_status status;
};

inline void check(mhd_status s, const char* where) {
    if (s != MHD_OK) throw Error(s, where);
}

// One device context per host Grid object (keyed by its address and shape).
class Session {
public:
    template <class GridT>
    static Session& of(const GridT& g) {
        static std::map<const void*, std::unique_ptr<Session>> sessions;
        auto& slot = sessions[static_cast<const void*>(&g)];
        if (!slot || slot->nx_ != g.nx || slot->ny_ != g.ny || slot->dx_ != g.cell_width ||
            slot->dy_ != g.cell_height || slot->eta_ != g.resistivity)
            slot.reset(new Session(g.nx, g.ny, g.cell_width, g.cell_height, g.resistivity));
        return *slot;
    }

    ~Session() {
        if (ctx_) mhd_destroy(ctx_);
    }

    mhd_context* ctx() { return ctx_; }

private:
    Session(int nx, int ny, double dx, double dy, double eta)
        : nx_(nx), ny_(ny), dx_(dx), dy_(dy), eta_(eta) {
        mhd_params p;
        check(mhd_default_params(&p, nx, ny, dx, dy, eta), "mhd_default_params");
        check(mhd_create(&p, nullptr, &ctx_), "mhd_create");
    }
    mhd_context* ctx_ = nullptr;
    int nx_, ny_;
    double dx_, dy_, eta_;
};

template <class GridT>
inline void upload(mhd_context* c, const GridT& g) {
    const double* f[6] = {g.rho.data(), g.mx.data(), g.my.data(), g.E.data(), g.bxf.data(),
                          g.byf.data()};
    check(mhd_set_state(c, f, MHD_LAYOUT_PADDED, g.ng), "mhd_set_state");
}

template <class GridT>
inline void download(mhd_context* c, GridT& g) {
    double* f[6] = {g.rho.data(), g.mx.data(), g.my.data(), g.E.data(), g.bxf.data(), g.byf.data()};
    check(mhd_get_state(c, f, MHD_LAYOUT_PADDED, g.ng), "mhd_get_state");
    double* prim[6] = {nullptr, g.vx.data(), g.vy.data(), g.p.data(), g.bxc.data(), g.byc.data()};
    check(mhd_get_primitives(c, prim, MHD_LAYOUT_PADDED, g.ng), "mhd_get_primitives");
}

// generate_A_matrix(grid, workspace, alpha) + ConjugateGradient::compute(A)
template <class GridT, class WorkspaceT>
void generate_A_matrix(const GridT& g, WorkspaceT&, double alpha) {
    check(mhd_set_implicit_coefficient(Session::of(g).ctx(), alpha), "mhd_set_implicit_coefficient");
}

// IMEX(grid_imex, grid_intermediary, grid_whole_step, workspace, MUSCL_values, coefficients,
//      solver, dt): one ARS(2,2,2) step of grid_imex in place.
template <class GridT, class WorkspaceT, class RVT, class TableauT, class SolverT>
void IMEX(GridT& g, GridT&, GridT&, WorkspaceT&, RVT&, TableauT&, SolverT&, double dt) {
    mhd_context* c = Session::of(g).ctx();
    upload(c, g);
    check(mhd_step(c, dt), "mhd_step");
    const mhd_status s = mhd_synchronize(c);
    if (s != MHD_OK && s != MHD_ERR_CG_NOT_CONVERGED)  // the reference carries on silently there
        throw Error(s, "IMEX");
    download(c, g);
}

// CFL_condition_checker(grid): the time step of the grid's current state.
template <class GridT>
double CFL_condition_checker(const GridT& g) {
    mhd_context* c = Session::of(g).ctx();
    upload(c, g);
    double dt = 0.0;
    check(mhd_cfl_dt(c, &dt), "mhd_cfl_dt");
    return dt;
}

// write_data_to_binary_file(grid, frame_index, snapshot_rate, dt): the snapshot file
// output/snapshot_NNNNNN.dat of the grid's state, in the reference's format; on disk when the call
// returns, as in the reference. (A device-resident run overlaps its files with stepping through
// mhd_snapshot_write of mhd_b200.h.)
template <class GridT>
void write_data_to_binary_file(GridT& g, int frame_index, int snapshot_rate, double dt) {
    mhd_context* c = Session::of(g).ctx();
    upload(c, g);
    char path[64];
    snprintf(path, sizeof(path), "output/snapshot_%06d.dat", frame_index);
    check(mhd_snapshot_write(c, path, g.ng, snapshot_rate, dt), "mhd_snapshot_write");
    check(mhd_snapshot_wait(c), "write_data_to_binary_file");
}

}  // namespace mhd_b200
