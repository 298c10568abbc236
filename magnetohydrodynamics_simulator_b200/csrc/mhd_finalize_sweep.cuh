// Finalize of the step as a warp column sweep (solvers.hpp:571-611, diagnostics.hpp:44-88):
//   B2      = U2*_B + dt*g * rate(E2)                      (solvers.hpp:573-574)
//   E3      = eta * J_z(B2) at the corners                 (solvers.hpp:450-461, explicit)
//   B^{n+1} = U2*_B + dt*g * rate(E3)                      (solvers.hpp:607-608)
//   density floor of U^{n+1} in place                      (solvers.hpp:610-611, Grid.hpp:115)
//   max CFL signal speed of U^{n+1}                        (diagnostics.hpp:60-78)
//   non-finite check of U^{n+1}
// Lane l holds column c0 - 1 + l; outputs are lanes 1..28 (FS_OUT columns). At sweep row c the
// warp receives E2 of row c+3 and U2*_B of row c+2, forms B2 and E3 of row c+2, B^{n+1} of row c+1
// and writes B^{n+1} and the CFL speed of row c. x neighbours come from shuffles.
#pragma once

#include "mhd_kernels.cuh"

namespace mhd {

constexpr int FS_OUT = 28;
constexpr int FS_WARPS = 8;
constexpr int FS_PRE = 3;  // rows swept before the first output row

// A finalize sweep reaches its grid through an accessor FA: acc(q) the accumulator planes (U2*),
// x() the second solve's corner field E2, bx() / by() the face planes of U^{n+1}, and nx(), ny(),
// dx(), dy(), eta() as the stage sweeps' accessors.
//
// FinParams: everything in kernel parameters.
struct FinParams {
    Planes acc_;
    const double* x_;
    double* bx_;
    double* by_;
    Domain D_;
    __device__ __forceinline__ double* acc(int q) const { return acc_.f[q]; }
    __device__ __forceinline__ const double* x() const { return x_; }
    __device__ __forceinline__ double* bx() const { return bx_; }
    __device__ __forceinline__ double* by() const { return by_; }
    __device__ __forceinline__ int nx() const { return D_.nx; }
    __device__ __forceinline__ int ny() const { return D_.ny; }
    __device__ __forceinline__ double dx() const { return D_.dx; }
    __device__ __forceinline__ double dy() const { return D_.dy; }
    __device__ __forceinline__ double eta() const { return D_.eta; }
};

// The sweep of one warp over rows [r0, r1) of column strip sx of one grid.
template <class FA>
__device__ __forceinline__ void finalize_sweep_warp(const FA& f, const StepCoeffs* __restrict__ C,
                                                    DeviceStatus* st, int sx, int r0, int r1) {
    const int lane = threadIdx.x & 31;
    const int nx = f.nx();  // setup only: the loop reads the grid through f
    const int c0 = sx * FS_OUT;
    if (r0 >= r1) return;
    const int i = c0 - 1 + lane;
    const int iw = wrap(i, nx);
    const bool out_lane = lane >= 1 && lane <= FS_OUT && i < nx;
    const double cg = C->c_g;
    // quotients by dx, dy as products with the hoisted reciprocals (within 1 ulp)
    const double idx = 1.0 / f.dx(), idy = 1.0 / f.dy();
    auto rowp = [&](int j) -> size_t { return (size_t)wrap(j, f.ny()) * f.nx(); };
    auto sdn = [](double v) { return __shfl_down_sync(0xffffffffu, v, 1); };
    auto sup = [](double v) { return __shfl_up_sync(0xffffffffu, v, 1); };

    const int cstart = r0 - FS_PRE;
    // pipelines
    double x_cur = __ldg(&f.x()[rowp(cstart + 2) + iw]);  // E2 row c+2
    double x_in = __ldg(&f.x()[rowp(cstart + 3) + iw]);   // E2 row c+3 (arriving)
    double b0x_in = f.acc(4)[rowp(cstart + 2) + iw];      // U2*_B row c+2 (arriving)
    double b0y_in = f.acc(5)[rowp(cstart + 2) + iw];
    double b0x[2] = {0.0, 0.0}, b0y[2] = {0.0, 0.0};       // U2*_B rows c, c+1
    double bx2_prev = 0.0;                                 // B2_x row c+1
    double e3_prev = 0.0;                                  // E3 row c+1
    double bnx_prev = 0.0, bny_prev = 0.0;                 // B^{n+1} row c
    double h_cur[4] = {0.0, 0.0, 0.0, 0.0};                // U2* hydro of row c (prefetched)
    double vmax = 0.0;
    bool bad = false;

    for (int c = cstart; c < r1; ++c) {
        const double xa = x_in, xb = x_cur;  // rows c+3, c+2
        const double ux = b0x_in, uy = b0y_in;  // U2*_B row c+2
        // issue the next row's loads
        x_cur = xa;
        x_in = __ldg(&f.x()[rowp(c + 4) + iw]);
        b0x_in = f.acc(4)[rowp(c + 3) + iw];
        b0y_in = f.acc(5)[rowp(c + 3) + iw];
        double h_nx[4] = {0.0, 0.0, 0.0, 0.0};
        if (out_lane && c + 1 >= r0 && c + 1 < r1) {
            const size_t g = (size_t)(c + 1) * f.nx() + i;
#pragma unroll
            for (int q = 0; q < 4; ++q) h_nx[q] = f.acc(q)[g];
        }
        // B2 of row c+2 (x neighbour of E2 from the next lane)
        const double bx2 = ux + (-(xa - xb) * idy) * cg;
        const double by2 = uy + ((sdn(xb) - xb) * idx) * cg;
        // E3 of row c+2
        const double e3 = f.eta() * ((by2 - sup(by2)) * idx - (bx2 - bx2_prev) * idy);
        // B^{n+1} of row c+1
        const double bnx = b0x[1] + (-(e3 - e3_prev) * idy) * cg;
        const double bny = b0y[1] + ((sdn(e3_prev) - e3_prev) * idx) * cg;
        // outputs of row c: B^{n+1}, density floor, CFL speed
        const double bnx_right = sdn(bnx_prev);
        if (out_lane && c >= r0 && c < r1) {
            const size_t g = (size_t)c * f.nx() + i;
            f.bx()[g] = bnx_prev;
            f.by()[g] = bny_prev;
            double rho = h_cur[0];
            if (rho < kRhoFloor) f.acc(0)[g] = kRhoFloor;
            const double bxc = (bnx_prev + bnx_right) / 2.0;
            const double byc = (bny_prev + bny) / 2.0;
            double vx, vy;
            const double p = primitives(rho, h_cur[1], h_cur[2], h_cur[3], bxc, byc, vx, vy);
            const double sp = cfl_speed(rho, vx, vy, p, bxc, byc);
            if (sp > vmax) vmax = sp;
            bad |= !(isfinite(rho) && isfinite(h_cur[1]) && isfinite(h_cur[2]) && isfinite(h_cur[3]) &&
                     isfinite(bnx_prev) && isfinite(bny_prev));
        }
        // shift
        b0x[0] = b0x[1]; b0x[1] = ux;
        b0y[0] = b0y[1]; b0y[1] = uy;
        bx2_prev = bx2;
        e3_prev = e3;
        bnx_prev = bnx;
        bny_prev = bny;
#pragma unroll
        for (int q = 0; q < 4; ++q) h_cur[q] = h_nx[q];
    }
    for (int o = 16; o > 0; o >>= 1) vmax = smax(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
    const bool any_bad = __any_sync(0xffffffffu, bad);
    if (lane == 0) {
        atomicMax(&st->smax_bits, (unsigned long long)__double_as_longlong(vmax));
        if (any_bad) atomicOr(&st->flags, (unsigned)kStatusNonFinite);
    }
}

static __global__ void __launch_bounds__(32 * FS_WARPS)
k_finalize_sweep(Domain D, const StepCoeffs* __restrict__ C, Planes acc,
                 const double* __restrict__ xsolve, double* __restrict__ bx_out,
                 double* __restrict__ by_out, DeviceStatus* st, SweepGeom G) {
    const int w = blockIdx.x * FS_WARPS + (threadIdx.x >> 5);
    if (w >= G.nwarps) return;
    const int sx = w % G.strips_x, sy = w / G.strips_x;
    const int r0 = sy * G.seg_h;
    const FinParams f{acc, xsolve, bx_out, by_out, D};
    finalize_sweep_warp(f, C, st, sx, r0, min(r0 + G.seg_h, D.ny));
}

}  // namespace mhd
