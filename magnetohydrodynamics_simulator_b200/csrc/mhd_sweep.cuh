// Explicit stage as a warp column sweep.
//
// A warp owns a strip of SW_OUT = 28 output columns [c0, c0+28): lane l holds column
// i = c0 - 2 + l (the 2-cell MUSCL halo on each side is covered by lanes 0-1 and 30-31). The warp
// sweeps the rows of its strip upwards; every quantity that the reference computes on whole
// planes (solvers.hpp:393-402) is computed here one row at a time, with
//   * the input rows (and stage 2's E1) copied by cp.async into a per-warp ring of 8 row slots in
//     shared memory, four rows ahead of their first use, so that no register holds raw input,
//   * the y-direction stencil of the primitives (rows c-1 .. c+2) held in registers as a rolling
//     window,
//   * the x-direction stencil (columns i-1 .. i+2) read from neighbouring lanes by shuffles.
// Every lane reads back only the ring entries it copied or wrote itself (x neighbours come by
// shuffle), so cp.async.wait_group alone orders the accesses; there is no block-level barrier.
//
// Pipeline at sweep row c (all rows periodic):
//   arrive  row c+3 of the input (stage 2: B1 = U1*_B + dt*g*rate(E1) of row c+3)
//   PRIM    row c+2      (Grid.hpp:82-136)
//   YFACE   top face of row c: HLL of the y-reconstructions of rows c-1..c+2 (solvers.hpp:238-250)
//   XFACE   right face of column i in row c (solvers.hpp:224-236)
//   CORNER  corner Ez at the bottom-left of cell (i, c) (solvers.hpp:294-346)
//   OUT     hydro rates of row c, B rates of row c-1 (solvers.hpp:253-292) + Butcher weights
// Lane validity: PRIM lanes 0-31, XFACE lanes 1-29, YFACE lanes 0-30, CORNER lanes 2-30, outputs
// lanes 2-29; other lanes compute values that are never used.
#pragma once

#include "mhd_kernels.cuh"

namespace mhd {

constexpr int SW_OUT = 28;       // output columns per warp
// The input rows are kept in a per-warp shared-memory ring filled by cp.async, not in registers.
// Slot layout: rho, mx, my, E, bxf, byf of the warp's 32 columns at q*32 + lane, lane 31's
// right-hand neighbour bxf(i+1) at 192; stage 2 adds E1 at SW_E1 + lane and lane 31's right-hand
// E1 at SW_E1 + 32.
constexpr int SW_RING = 8;       // row slots per warp (power of two): rows c-1 .. c+6
constexpr int SW_E1 = 196;       // offset of E1 in a stage-2 slot
constexpr int SW_SLOT = 230;     // doubles per slot (1840 bytes, 16-byte multiple)
// Stage 2 keeps the values it carries from row to row -- the y slopes and the y-face fluxes of the
// previous row, 10 per lane -- in shared memory after its ring, not in registers. The registers it
// frees let stage 2 evaluate HLL branch-free as stage 1 does (measured on B200 at 4096^2: stage 2
// 1.001 -> 0.954 ms; stage 1, whose carried values fit its registers, is 1.7% slower this way).
constexpr int SW_CARRY = 10 * 32;
// doubles of shared memory per warp of an explicit-stage kernel
constexpr int sweep_warp_doubles(int mode) { return SW_RING * SW_SLOT + (mode == 2 ? SW_CARRY : 0); }
// One warp (an independent strip segment) per block: blocks retire warp by warp, so the tail of
// a launch and the persistent batch kernels balance at warp granularity (measured on B200 against
// 4-warp blocks at the same registers: stage 1 1.29 -> 1.25 ms, stage 2 1.24 -> 1.15 ms at 4096^2).
#ifndef MHD_SW_WARPS
#define MHD_SW_WARPS 1
#endif
constexpr int SW_WARPS = MHD_SW_WARPS;  // warps (independent strips) per block
constexpr int SW_PRE = 5;        // rows swept before the first output row of a strip

__device__ __forceinline__ double shup(double v, int d) { return __shfl_up_sync(0xffffffffu, v, d); }
__device__ __forceinline__ double shdn(double v, int d) { return __shfl_down_sync(0xffffffffu, v, d); }

// Resident warps per SM: 12 for both stages, i.e. 3 per SM sub-partition, whose 16K registers
// allow at most 168 per thread (the next step, 16 warps, allows 128 and spills). With the input
// rows in the shared-memory ring both stages fit 168 registers without spilling.
#ifndef MHD_SWEEP_MIN_BLOCKS_1
#define MHD_SWEEP_MIN_BLOCKS_1 (12 / MHD_SW_WARPS)
#endif
#ifndef MHD_SWEEP_MIN_BLOCKS_2
#define MHD_SWEEP_MIN_BLOCKS_2 (12 / MHD_SW_WARPS)
#endif
// Limited slopes formed once per cell (both stages; with the input rows in the shared-memory ring
// the carried slopes fit the 168 registers: stage 1 at 164, measured on B200 at 4096^2: stage 1
// 0.966 -> 0.891 ms against forming them per face).
#ifndef MHD_SWEEP_YREUSE_1
#define MHD_SWEEP_YREUSE_1 1
#endif
#ifndef MHD_SWEEP_XREUSE_1
#define MHD_SWEEP_XREUSE_1 1
#endif
#ifndef MHD_SWEEP_YREUSE_2
#define MHD_SWEEP_YREUSE_2 1
#endif
#ifndef MHD_SWEEP_XREUSE_2
#define MHD_SWEEP_XREUSE_2 1
#endif

// Where a sweep finds its planes: in(q) the six input planes, x() the corner field E1 (stage 2),
// a(q) / b(q) the two output plane sets (stage 1: predictor / accumulator; stage 2: - /
// accumulator, read and written).
// A sweep reaches its grid through an accessor PL:
//   in(q) the six input planes, x() the corner field E1 (stage 2), a(q) / b(q) the two output
//   plane sets (stage 1: predictor / accumulator; stage 2: - / accumulator, read and written);
//   nx(), ny(), dx(), dy(), eta(), ct_mode() the grid's size, spacing, resistivity and CT mode.
//
// ParamPlanes: everything in kernel parameters (constant bank; nothing has to stay in registers).
struct ParamPlanes {
    CPlanes in_;
    const double* x_;
    Planes a_, b_;
    Domain D_;
    __device__ __forceinline__ const double* in(int q) const { return in_.f[q]; }
    __device__ __forceinline__ const double* x() const { return x_; }
    __device__ __forceinline__ double* a(int q) const { return a_.f[q]; }
    __device__ __forceinline__ double* b(int q) const { return b_.f[q]; }
    __device__ __forceinline__ int nx() const { return D_.nx; }
    __device__ __forceinline__ int ny() const { return D_.ny; }
    __device__ __forceinline__ double dx() const { return D_.dx; }
    __device__ __forceinline__ double dy() const { return D_.dy; }
    __device__ __forceinline__ double eta() const { return D_.eta; }
    __device__ __forceinline__ int ct_mode() const { return D_.ct_mode; }
};

// Per-warp record of the instance a batch warp is sweeping (shared memory).
struct SweepInstRec {
    Domain D;
    long long off;  // zone offset of the instance in every plane arena
};
// RecPlanes: one instance of a batch whose planes are arenas holding every instance at the same
// zone offset. The arena bases are kernel parameters; the instance's offset and grid live in the
// warp's shared record and are read (volatile) where they are used, so that a persistent kernel
// stepping many instances holds none of them in registers across its sweep.
struct RecPlanes {
    ParamPlanes base;
    const SweepInstRec* rec;
    template <class T>
    __device__ __forceinline__ static T vload(T const* p) {
        return *static_cast<T const volatile*>(p);
    }
    __device__ __forceinline__ size_t off() const { return (size_t)vload(&rec->off); }
    __device__ __forceinline__ const double* in(int q) const { return base.in_.f[q] + off(); }
    __device__ __forceinline__ const double* x() const { return base.x_ + off(); }
    __device__ __forceinline__ double* a(int q) const { return base.a_.f[q] + off(); }
    __device__ __forceinline__ double* b(int q) const { return base.b_.f[q] + off(); }
    __device__ __forceinline__ int nx() const { return vload(&rec->D.nx); }
    __device__ __forceinline__ int ny() const { return vload(&rec->D.ny); }
    __device__ __forceinline__ double dx() const { return vload(&rec->D.dx); }
    __device__ __forceinline__ double dy() const { return vload(&rec->D.dy); }
    __device__ __forceinline__ double eta() const { return vload(&rec->D.eta); }
    __device__ __forceinline__ int ct_mode() const { return vload(&rec->D.ct_mode); }
};

// The sweep of one warp over rows [r0, r1) of column strip sx of one grid.
template <int MODE, class PL, bool kYReuse = (MODE == 1) ? MHD_SWEEP_YREUSE_1 : MHD_SWEEP_YREUSE_2,
          bool kXReuse = (MODE == 1) ? MHD_SWEEP_XREUSE_1 : MHD_SWEEP_XREUSE_2, bool kSelect = true>
__device__ __forceinline__ void stage_sweep_warp(const StepCoeffs* __restrict__ C, const PL& pl,
                                                 int sx, int r0, int r1, double* ring) {
    const int lane = threadIdx.x & 31;
    const int nx = pl.nx();  // setup only: the loop reads the grid through pl
    const int c0 = sx * SW_OUT;
    if (r0 >= r1) return;
    // kYReuse / kXReuse: limited slopes formed once per cell (y: carried to the next row; x: shared
    // with the lane on the left), or per face as the reference writes them -- the same operands
    // either way
    const int i = c0 - 2 + lane;
    const int iw = wrap(i, nx);
    const bool out_lane = lane >= 2 && lane < 2 + SW_OUT && i < nx;
    const double idx = 1.0 / pl.dx(), idy = 1.0 / pl.dy();
    const double cg = C->c_g;
    const double cA = (MODE == 1) ? C->c_g : C->c_1md;   // outA weight (stage 1: predictor)
    const double cB = (MODE == 1) ? C->c_d : C->c_1md;   // outB weight
    const double c1mg = C->c_1mg;
    // column of the lane to the right (for stage 2's B1 of lane 31)
    const int iw_r = wrap(i + 1, nx);

    auto rowp = [&](int j) -> size_t { return (size_t)wrap(j, pl.ny()) * pl.nx(); };

    // ---- windows (index 0 = oldest row)
    double Prho[4], Pvx[4], Pvy[4], Pp[4], Pbxc[4];  // rows c-1 .. c+2
    double Pbyc[3];                                   // rows c .. c+2
    // y slopes of row c (when carried) and the y-face flux of row c-1: registers in stage 1,
    // shared memory after the ring in stage 2
    double Sy_r[5], fy_r[5];
    double* const carry = ring + SW_RING * SW_SLOT;
    auto Sy = [&](int k) -> double& {
        if constexpr (MODE == 2) return carry[(5 + k) * 32 + lane];
        else return Sy_r[k];
    };
    auto fy_prev = [&](int k) -> double& {
        if constexpr (MODE == 2) return carry[k * 32 + lane];
        else return fy_r[k];
    };
    double fxbt_prev = 0.0, ez_prev = 0.0, jz_prev = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) { Prho[k] = 1.0; Pvx[k] = 0.0; Pvy[k] = 0.0; Pp[k] = 1.0; Pbxc[k] = 0.0; }
#pragma unroll
    for (int k = 0; k < 3; ++k) Pbyc[k] = 0.0;
#pragma unroll
    for (int k = 0; k < 5; ++k) { Sy(k) = 0.0; fy_prev(k) = 0.0; }

    const int cstart = r0 - SW_PRE;
    // The input rows live in the ring: sweep row r sits in slot (r - cstart + 1) % SW_RING; it is
    // copied while the warp works on row r - 7 and read up to row r + 1. Stage 2 also copies E1 and
    // turns the row's faces into B1 when the row arrives (B1 is what every later read of the row
    // needs).
    auto slot = [&](int r) -> double* {
        return ring + (unsigned)((r - cstart + 1) & (SW_RING - 1)) * SW_SLOT;
    };
    auto issue_row = [&](int r) {
        if (r <= r1 + (MODE == 1 ? 3 : 4)) {
            double* sl = slot(r);
            const size_t rp = rowp(r);
#pragma unroll
            for (int q = 0; q < 6; ++q) cp_async8(&sl[q * 32 + lane], &pl.in(q)[rp + iw]);
            if (lane == 31) cp_async8(&sl[192], &pl.in(4)[rp + iw_r]);
            if constexpr (MODE == 2) {
                cp_async8(&sl[SW_E1 + lane], &pl.x()[rp + iw]);
                if (lane == 31) cp_async8(&sl[SW_E1 + 32], &pl.x()[rp + iw_r]);
            }
        }
        cp_async_commit();
    };
#pragma unroll
    for (int r = 0; r < SW_RING; ++r) issue_row(cstart - 1 + r);

    for (int c = cstart; c <= r1; ++c) {
        if constexpr (MODE == 1) cp_async_wait<SW_RING - 5>();  // rows up to c+3 have landed
        else cp_async_wait<SW_RING - 6>();                       // rows up to c+4 have landed
        // stage 2: the accumulator values this row's outputs add to (hydro row c, faces row c-1),
        // loaded here and used at the end of the row
        double accH[4] = {0.0, 0.0, 0.0, 0.0}, accB[2] = {0.0, 0.0};
        if constexpr (MODE == 2) {
            // B1 = U1*_B + dt*g*(rate of E1) of row c+3 (solvers.hpp:484-485, 528-529), written
            // over the row's faces in the ring (lane 31 also converts its right-hand bxf)
            double* s3 = slot(c + 3);
            const double* s4 = slot(c + 4);
            const double ax0 = s3[SW_E1 + lane], ax1 = s4[SW_E1 + lane];
            double axr = shdn(ax0, 1);
            if (lane == 31) axr = s3[SW_E1 + 32];
            const double rbx = -(ax1 - ax0) * idy;
            const double rby = (axr - ax0) * idx;
            s3[4 * 32 + lane] = s3[4 * 32 + lane] + rbx * cg;
            s3[5 * 32 + lane] = s3[5 * 32 + lane] + rby * cg;
            if (lane == 31) s3[192] = s3[192] + (-(s4[SW_E1 + 32] - s3[SW_E1 + 32]) * idy) * cg;
            if (out_lane) {
                if (c >= r0 && c < r1) {
                    const size_t g = (size_t)c * pl.nx() + i;
#pragma unroll
                    for (int q = 0; q < 4; ++q) accH[q] = pl.b(q)[g];
                }
                if (c - 1 >= r0 && c - 1 < r1) {
                    const size_t g = (size_t)(c - 1) * pl.nx() + i;
                    accB[0] = pl.b(4)[g];
                    accB[1] = pl.b(5)[g];
                }
            }
        }
        // ---- PRIM row c+2 (Grid.hpp:82-136): conserved hydro and bxf of row c+2, byf of rows c+2
        //      and c+3; bxf one column to the right from the next lane (lane 31: its own copy)
        double nrho, nvx, nvy, np, nbxc, nbyc;
        {
            const double* s2 = slot(c + 2);
            const double bxf2 = s2[4 * 32 + lane];
            double bxr2 = shdn(bxf2, 1);
            if (lane == 31) bxr2 = s2[192];
            nbxc = (bxf2 + bxr2) / 2.0;
            nbyc = (s2[5 * 32 + lane] + slot(c + 3)[5 * 32 + lane]) / 2.0;
            double rho = s2[lane];
            if (MODE == 2 && rho < kRhoFloor) rho = kRhoFloor;  // floored in place (solvers.hpp:522-523)
            np = primitives(rho, s2[32 + lane], s2[64 + lane], s2[96 + lane], nbxc, nbyc, nvx, nvy);
            nrho = rho;
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            Prho[k] = Prho[k + 1]; Pvx[k] = Pvx[k + 1]; Pvy[k] = Pvy[k + 1];
            Pp[k] = Pp[k + 1]; Pbxc[k] = Pbxc[k + 1];
        }
        Prho[3] = nrho; Pvx[3] = nvx; Pvy[3] = nvy; Pp[3] = np; Pbxc[3] = nbxc;
        Pbyc[0] = Pbyc[1]; Pbyc[1] = Pbyc[2]; Pbyc[2] = nbyc;
        // window rows now: P*[0..3] = c-1 .. c+2, Pbyc[0..2] = c .. c+2; ring rows c-1 .. c+3
        //                  (stage 2: their faces hold B1)

        // ---- YFACE: top face of (i, c); D = upper y-extrapolation of row c, U = lower of c+1
        //      (MUSCL.hpp:26-47). With kYReuse each row's limited slope is formed once, when the
        //      row is c+1, and carried to the next row for its upper extrapolation.
        Flux fy;
        {
            Prim Dn, Up;
            if constexpr (kYReuse) {
                const double s_rho = minmod(Prho[2] - Prho[1], Prho[3] - Prho[2]);
                const double s_vx = minmod(Pvx[2] - Pvx[1], Pvx[3] - Pvx[2]);
                const double s_vy = minmod(Pvy[2] - Pvy[1], Pvy[3] - Pvy[2]);
                const double s_p = minmod(Pp[2] - Pp[1], Pp[3] - Pp[2]);
                const double s_bx = minmod(Pbxc[2] - Pbxc[1], Pbxc[3] - Pbxc[2]);
                Dn.rho = Prho[1] + 0.5 * Sy(0);
                Dn.vx = Pvx[1] + 0.5 * Sy(1);
                Dn.vy = Pvy[1] + 0.5 * Sy(2);
                Dn.p = Pp[1] + 0.5 * Sy(3);
                Dn.bx = Pbxc[1] + 0.5 * Sy(4);
                Up.rho = Prho[2] - 0.5 * s_rho;
                Up.vx = Pvx[2] - 0.5 * s_vx;
                Up.vy = Pvy[2] - 0.5 * s_vy;
                Up.p = Pp[2] - 0.5 * s_p;
                Up.bx = Pbxc[2] - 0.5 * s_bx;
                Sy(0) = s_rho; Sy(1) = s_vx; Sy(2) = s_vy; Sy(3) = s_p; Sy(4) = s_bx;
            } else {
                Dn.rho = recon_hi(Prho[0], Prho[1], Prho[2]);
                Dn.vx = recon_hi(Pvx[0], Pvx[1], Pvx[2]);
                Dn.vy = recon_hi(Pvy[0], Pvy[1], Pvy[2]);
                Dn.p = recon_hi(Pp[0], Pp[1], Pp[2]);
                Dn.bx = recon_hi(Pbxc[0], Pbxc[1], Pbxc[2]);
                Up.rho = recon_lo(Prho[1], Prho[2], Prho[3]);
                Up.vx = recon_lo(Pvx[1], Pvx[2], Pvx[3]);
                Up.vy = recon_lo(Pvy[1], Pvy[2], Pvy[3]);
                Up.p = recon_lo(Pp[1], Pp[2], Pp[3]);
                Up.bx = recon_lo(Pbxc[1], Pbxc[2], Pbxc[3]);
            }
            Dn.by = Up.by = slot(c + 1)[5 * 32 + lane];  // byf of row c+1
            fy = hll<1, kSelect>(Dn, Up);
        }
        // ---- XFACE: right face of (i, c); L = upper x-extrapolation of column i, R = lower of
        //      i+1. With kXReuse every lane limits its own column's slope once and hands its lower
        //      extrapolation to the lane on its left; otherwise each lane forms both from shuffled
        //      neighbours (no shuffle waits on arithmetic).
        Flux fx;
        {
            Prim L, R;
            auto xrecon = [&](double q, double& hi, double& lo_right) {
                if constexpr (kXReuse) {
                    const double s = minmod(q - shup(q, 1), shdn(q, 1) - q);
                    hi = q + 0.5 * s;
                    lo_right = shdn(q - 0.5 * s, 1);
                } else {
                    const double qm = shup(q, 1), qp = shdn(q, 1), qpp = shdn(q, 2);
                    hi = recon_hi(qm, q, qp);
                    lo_right = recon_lo(q, qp, qpp);
                }
            };
            xrecon(Prho[1], L.rho, R.rho);
            xrecon(Pvx[1], L.vx, R.vx);
            xrecon(Pvy[1], L.vy, R.vy);
            xrecon(Pp[1], L.p, R.p);
            xrecon(Pbyc[0], L.by, R.by);
            L.bx = R.bx = shdn(slot(c)[4 * 32 + lane], 1);  // bxf(i+1, c)
            fx = hll<0, kSelect>(L, R);
        }
        // ---- CORNER (i, c): eN = -Fx^By(i-1, c), eS = -Fx^By(i-1, c-1), eE = Fy^Bx(i, c-1),
        //      eW = Fy^Bx(i-1, c-1); corner velocity = mean of the 4 cells
        double ez;
        {
            const double eN = -shup(fx.bt, 1);
            const double eS = -shup(fxbt_prev, 1);
            const double eE = fy_prev(4);
            const double eW = shup(fy_prev(4), 1);
            const double vxc = 0.25 * (Pvx[1] + shup(Pvx[1], 1) + Pvx[0] + shup(Pvx[0], 1));
            const double vyc = 0.25 * (Pvy[1] + shup(Pvy[1], 1) + Pvy[0] + shup(Pvy[0], 1));
            ez = corner_ez(eN, eS, eE, eW, vxc, vyc, pl.ct_mode());
        }
        double jz = 0.0;
        if (MODE == 2) {  // eta*J_z(B1) at corner (i, c) (solvers.hpp:450-461)
            const double by1 = slot(c)[5 * 32 + lane];
            const double dBy_dx = (by1 - shup(by1, 1)) * idx;
            const double dBx_dy = (slot(c)[4 * 32 + lane] - slot(c - 1)[4 * 32 + lane]) * idy;
            jz = pl.eta() * (dBy_dx - dBx_dy);
        }
        // ---- hydro rates of row c
        {
            double f[4];
            f[0] = -((fx.rho - shup(fx.rho, 1)) * idx + (fy.rho - fy_prev(0)) * idy);
            f[1] = -((fx.mx - shup(fx.mx, 1)) * idx + (fy.mx - fy_prev(1)) * idy);
            f[2] = -((fx.my - shup(fx.my, 1)) * idx + (fy.my - fy_prev(2)) * idy);
            f[3] = -((fx.E - shup(fx.E, 1)) * idx + (fy.E - fy_prev(3)) * idy);
            if (out_lane && c >= r0 && c < r1) {
                const size_t g = (size_t)c * pl.nx() + i;
                if constexpr (MODE == 1) {
                    const double* sc = slot(c);
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const double u = sc[q * 32 + lane];
                        pl.a(q)[g] = u + f[q] * cA;                       // predictor
                        const double ua = (q == 0 && u < kRhoFloor) ? kRhoFloor : u;
                        pl.b(q)[g] = ua + f[q] * cB;                      // accumulator
                    }
                } else {
#pragma unroll
                    for (int q = 0; q < 4; ++q) pl.b(q)[g] = accH[q] + f[q] * cB;
                }
            }
        }
        // ---- B rates of row c-1: -(Ez(i, c) - Ez(i, c-1))/dy, (Ez(i+1, c-1) - Ez(i, c-1))/dx
        {
            const double fbx = -(ez - ez_prev) * idy;
            const double fby = (shdn(ez_prev, 1) - ez_prev) * idx;
            double g2x = 0.0, g2y = 0.0;
            if (MODE == 2) {
                g2x = -(jz - jz_prev) * idy;
                g2y = (shdn(jz_prev, 1) - jz_prev) * idx;
            }
            if (out_lane && c - 1 >= r0 && c - 1 < r1) {
                const size_t g = (size_t)(c - 1) * pl.nx() + i;
                if constexpr (MODE == 1) {
                    const double* sp = slot(c - 1);
                    const double ubx = sp[4 * 32 + lane], uby = sp[5 * 32 + lane];  // U^n faces, row c-1
                    pl.a(4)[g] = ubx + fbx * cA;
                    pl.a(5)[g] = uby + fby * cA;
                    pl.b(4)[g] = ubx + fbx * cB;
                    pl.b(5)[g] = uby + fby * cB;
                } else {
                    double ax = accB[0] + fbx * cB;
                    double ay = accB[1] + fby * cB;
                    ax += g2x * c1mg;
                    ay += g2y * c1mg;
                    pl.b(4)[g] = ax;
                    pl.b(5)[g] = ay;
                }
            }
        }
        // ---- carry to the next row
        fy_prev(0) = fy.rho; fy_prev(1) = fy.mx; fy_prev(2) = fy.my; fy_prev(3) = fy.E; fy_prev(4) = fy.bt;
        fxbt_prev = fx.bt;
        ez_prev = ez;
        jz_prev = jz;
        issue_row(c + 7);  // into the slot of row c-1, no longer read
    }
    cp_async_wait<0>();  // leave no copy in flight into the ring
}

// Dynamic shared memory of a block of the explicit-stage kernels (their warps' row rings).
constexpr size_t sweep_smem_bytes(int mode) {
    return (size_t)SW_WARPS * sweep_warp_doubles(mode) * sizeof(double);
}

template <int MODE>
__global__ void __launch_bounds__(32 * SW_WARPS, MODE == 1 ? MHD_SWEEP_MIN_BLOCKS_1 : MHD_SWEEP_MIN_BLOCKS_2)
k_stage_sweep(Domain D, const StepCoeffs* __restrict__ C, CPlanes in,
              const double* __restrict__ xsolve, Planes outA, Planes outB, SweepGeom G) {
#if defined(__CUDA_ARCH__)
    extern __shared__ __align__(16) double sw_ring_mem[];
#else
    static double sw_ring_mem[SW_WARPS * (SW_RING * SW_SLOT + SW_CARRY)];  // host compilation: one copy
#endif
    double* const ring = sw_ring_mem + (size_t)(threadIdx.x >> 5) * sweep_warp_doubles(MODE);
    const int w = blockIdx.x * SW_WARPS + (threadIdx.x >> 5);
    if (w >= G.nwarps) return;
    const ParamPlanes pl{in, xsolve, outA, outB, D};
    const int sx = w % G.strips_x, sy = w / G.strips_x;
    const int r0 = sy * G.seg_h;
    stage_sweep_warp<MODE>(C, pl, sx, r0, min(r0 + G.seg_h, D.ny), ring);
}

}  // namespace mhd
