// Per-cell and per-face FP64 physics of the reference solver, as device functions.
//
// Each function keeps the reference's arithmetic order (operand order of every sum and product),
// so that the GPU path differs from the reference's CPU path only by FMA contraction and the
// summation order of global reductions. References are to RikibabManos/Magnetohydrodynamics_Simulator.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace mhd {

constexpr double kGammaGas = 5.0 / 3.0;  // Grid.hpp:104, HLL.hpp:31,62,85,108, diagnostics.hpp:48
// p / (gamma - 1) of the ideal-gas energy (HLL.hpp:43, 69, 92) as a product with the folded
// reciprocal: what the reference's -ffast-math build computes (CMakeLists.txt:21), within 1 ulp of
// the quotient, and one FP64 multiply instead of a division sequence.
constexpr double kInvGm1 = 1.0 / (kGammaGas - 1.0);
constexpr double kRhoFloor = 1e-8;       // Grid.hpp:115, diagnostics.hpp:64
constexpr double kPFloor = 1e-8;         // Grid.hpp:124, diagnostics.hpp:65

struct Prim {
    double rho, vx, vy, p, bx, by;
};

struct Flux {
    double rho, mx, my, E, bt;  // bt: the tangential induction flux (F^By in x, F^Bx in y)
};

// std::min / std::max semantics (b < a ? b : a), not fmin/fmax.
__device__ __forceinline__ double smin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double smax(double a, double b) { return (a < b) ? b : a; }

// MUSCL.hpp:11-17
__device__ __forceinline__ double minmod(double a, double b) {
    if (a * b > 0.0) return (fabs(a) < fabs(b)) ? a : b;
    return 0.0;
}

// MUSCL.hpp:26-47, lower (c - s/2) face value of a cell from (left, centre, right)
__device__ __forceinline__ double recon_lo(double fm, double f0, double fp) {
    return f0 - 0.5 * minmod(f0 - fm, fp - f0);
}
// upper (c + s/2) face value
__device__ __forceinline__ double recon_hi(double fm, double f0, double fp) {
    return f0 + 0.5 * minmod(f0 - fm, fp - f0);
}

// Grid.hpp:100-136 computePrimitives for one cell. `rho` is replaced by the floored density;
// velocities divide by the density as stored (before the floor), as the reference does.
// Returns the (floored) pressure.
__device__ __forceinline__ double primitives(double& rho, double mx, double my, double E,
                                             double bxc, double byc, double& vx, double& vy) {
    // one reciprocal instead of two divisions (<= 1 ulp from m/rho; the reference's fast-math
    // build is free to do the same)
    const double ir = 1.0 / rho;
    vx = mx * ir;
    vy = my * ir;
    if (rho < kRhoFloor) rho = kRhoFloor;
    const double kin = 0.5 * rho * (vx * vx + vy * vy);
    const double mag = (bxc * bxc + byc * byc) / 2;
    const double eint = E - kin - mag;
    double p = (kGammaGas - 1) * eint;
    if (p < kPFloor) p = kPFloor;
    return p;
}

// HLL.hpp:107-122 fast magnetosonic speed
__device__ __forceinline__ double fast_speed(const Prim& w, double bn) {
    const double b2 = w.bx * w.bx + w.by * w.by;
    const double ir = 1.0 / w.rho;  // one reciprocal for the three quotients by rho
    const double a2 = kGammaGas * w.p * ir;
    const double t2 = b2 * ir;
    const double n2 = bn * bn * ir;
    const double sum = t2 + a2;
    const double term = sum * sum - 4.0 * a2 * n2;
    return sqrt(0.5 * (sum + sqrt(term > 0.0 ? term : 0.0)));
}

// HLL.hpp:61-104 physical flux normal to direction DIR (0 = x, 1 = y), together with the
// conserved energy of HLL.hpp:31-47 (needed by the HLL average).
template <int DIR>
__device__ __forceinline__ Flux phys_flux(const Prim& w) {
    const double v2 = w.vx * w.vx + w.vy * w.vy;
    const double b2 = w.bx * w.bx + w.by * w.by;
    const double pt = w.p + 0.5 * b2;
    const double vb = w.vx * w.bx + w.vy * w.by;
    const double E = w.p * kInvGm1 + 0.5 * (w.rho * v2 + b2);
    Flux F;
    if (DIR == 0) {
        F.rho = w.rho * w.vx;
        F.mx = w.rho * w.vx * w.vx + pt - w.bx * w.bx;
        F.my = w.rho * w.vx * w.vy - w.bx * w.by;
        F.E = (E + pt) * w.vx - w.bx * vb;
        F.bt = w.vx * w.by - w.vy * w.bx;
    } else {
        F.rho = w.rho * w.vy;
        F.my = w.rho * w.vy * w.vy + pt - w.by * w.by;
        F.mx = w.rho * w.vx * w.vy - w.bx * w.by;
        F.E = (E + pt) * w.vy - w.by * vb;
        F.bt = w.vy * w.bx - w.vx * w.by;
    }
    return F;
}

// HLL.hpp:31-47 ConservedState::fromPrimitive (the components the HLL average uses).
template <int DIR>
__device__ __forceinline__ Flux conserved(const Prim& w) {
    Flux U;
    U.rho = w.rho;
    U.mx = w.rho * w.vx;
    U.my = w.rho * w.vy;
    const double v2 = w.vx * w.vx + w.vy * w.vy;
    const double b2 = w.bx * w.bx + w.by * w.by;
    U.E = w.p * kInvGm1 + 0.5 * w.rho * v2 + 0.5 * b2;
    U.bt = (DIR == 0) ? w.by : w.bx;
    return U;
}

// HLL.hpp:126-172 (DIR = 0) and :177-218 (DIR = 1). L is the lower/left state. SELECT: form the
// HLL average for every face and select the case afterwards instead of returning early (the same
// values; straight-line code that schedules better where registers allow it, measured on B200:
// stage 1 1.030 -> 1.010 ms at 4096^2; stage 2 uses it once its carried values live in shared
// memory; in the batch's stage 2 it fits without spills too but gains nothing, 6.97-6.99 against
// 6.98 ms per batched step, so the batch keeps the branches).
template <int DIR, bool SELECT = false>
__device__ __forceinline__ Flux hll(const Prim& L, const Prim& R) {
    const Flux FL = phys_flux<DIR>(L);
    const Flux FR = phys_flux<DIR>(R);
    const double cL = fast_speed(L, DIR == 0 ? L.bx : L.by);
    const double cR = fast_speed(R, DIR == 0 ? R.bx : R.by);
    const double vL = DIR == 0 ? L.vx : L.vy;
    const double vR = DIR == 0 ? R.vx : R.vy;
    const double sL = smin(vL - cL, vR - cR);
    const double sR = smax(vL + cL, vR + cR);
    if constexpr (SELECT) {
        // sR = sL only where the selection takes F_L or F_R
        const Flux UL = conserved<DIR>(L);
        const Flux UR = conserved<DIR>(R);
        const double inv = 1.0 / (sR - sL);
        const double sLR = sL * sR;
        const bool left = sL >= 0, right = !left && sR <= 0;
        auto pick = [&](double fl, double fr, double ul, double ur) {
            const double avg = (sR * fl - sL * fr + sLR * (ur - ul)) * inv;
            return left ? fl : (right ? fr : avg);
        };
        Flux F;
        F.rho = pick(FL.rho, FR.rho, UL.rho, UR.rho);
        F.mx = pick(FL.mx, FR.mx, UL.mx, UR.mx);
        F.my = pick(FL.my, FR.my, UL.my, UR.my);
        F.E = pick(FL.E, FR.E, UL.E, UR.E);
        F.bt = pick(FL.bt, FR.bt, UL.bt, UR.bt);
        return F;
    } else {
        if (sL >= 0) return FL;
        if (sR <= 0) return FR;
        const Flux UL = conserved<DIR>(L);
        const Flux UR = conserved<DIR>(R);
        const double inv = 1.0 / (sR - sL);
        const double sLR = sL * sR;
        Flux F;
        F.rho = (sR * FL.rho - sL * FR.rho + sLR * (UR.rho - UL.rho)) * inv;
        F.mx = (sR * FL.mx - sL * FR.mx + sLR * (UR.mx - UL.mx)) * inv;
        F.my = (sR * FL.my - sL * FR.my + sLR * (UR.my - UL.my)) * inv;
        F.E = (sR * FL.E - sL * FR.E + sLR * (UR.E - UL.E)) * inv;
        F.bt = (sR * FL.bt - sL * FR.bt + sLR * (UR.bt - UL.bt)) * inv;
        return F;
    }
}

// solvers.hpp:326,333 corner-velocity test. GCC resolves the unqualified abs(double) there to
// int abs(int), so the reference averages whenever (int)v == 0, i.e. |v| < 1 (and, as x86
// converts NaN / out-of-range values to INT_MIN, also for those). mode 1 is the literal
// |v| < 1e-12 test, for physics studies.
__device__ __forceinline__ bool ct_average(double v, int mode) {
    if (mode == 1) return fabs(v) < 1e-12;
    return !(fabs(v) >= 1.0 && fabs(v) < 2147483648.0);
}

// solvers.hpp:314-340 corner electric field from the four face fluxes and the corner velocity.
__device__ __forceinline__ double corner_ez(double eN, double eS, double eE, double eW, double vxc,
                                            double vyc, int mode) {
    double ezy, ezx;
    if (ct_average(vyc, mode)) ezy = 0.5 * (eS + eN);
    else ezy = (vyc > 0.0) ? eS : eN;
    if (ct_average(vxc, mode)) ezx = 0.5 * (eE + eW);
    else ezx = (vxc > 0.0) ? eW : eE;
    return 0.5 * (ezx + ezy);
}

// diagnostics.hpp:60-77 fastest signal speed of one cell from its stored primitives.
__device__ __forceinline__ double cfl_speed(double rho_f, double vx, double vy, double p,
                                            double bxc, double byc) {
    const double r = smax(rho_f, 1e-8);
    const double pr = smax(p, 1e-8);
    const double ir = 1.0 / r;
    const double a2 = kGammaGas * pr * ir;
    const double b2 = (bxc * bxc + byc * byc) * ir;
    return sqrt(a2 + b2) + sqrt(vx * vx + vy * vy);
}

}  // namespace mhd
