// Device kernels of one ARS(2,2,2) IMEX step (reference: solvers.hpp:491-613 of
// RikibabManos/Magnetohydrodynamics_Simulator), for sm_100a, FP64.
//
// HBM layout: every field is a dense, row-major nx*ny plane of doubles (index j*nx + i), periodic in
// both directions; there are no ghost cells in device memory -- halos are gathered into shared
// memory with periodic index wrap (the reference's ghost fill, Grid.hpp:143-161, is a periodic
// copy). bxf(i,j) lives on the left face of cell (i,j), byf(i,j) on its bottom face, and the corner
// field of the implicit solve at the bottom-left corner.
//
// One step is five kernels:
//   stage<1>   U^n            -> predictor U1* = U^n + dt*g*f1 and accumulator U^n + dt*d*f1
//   cg         U1*_B          -> corner field E1 of (I - alpha L) E1 = eta J_z(U1*_B)
//   stage<2>   U1*, E1, acc   -> U2* = acc + dt(1-d) f2(U1) + dt(1-g) g2(B1)   (in place on acc)
//   cg         U2*_B          -> E2
//   finalize   U2*, E2        -> B^{n+1} = U2*_B + dt*g*g3(B2), density floor, CFL max speed
// (g = 1 - 1/sqrt(2), d = 1 - 1/(2g): solvers.hpp:39-66).
#pragma once

#include <cstdint>

#include "mhd_physics.cuh"

namespace mhd {

// ------------------------------------------------------------------------------------------
// Shared parameter blocks

struct Domain {
    int nx, ny;
    double dx, dy, eta;
    int ct_mode;  // 0: reference as compiled (int-truncating abs), 1: |v| < 1e-12
};

// Stage weights of one step, all multiplied by dt (solvers.hpp:503, 509-510, 543-546, 585-588).
// A_ex[3] = A_im[4] = b_im[2] = g; A_ex[6] = b_ex[0] = d; A_ex[7] = b_ex[1] = 1 - d;
// A_im[7] = b_im[1] = 1 - g; A_im[3] = A_im[6] = b_im[0] = 0 (the g1 terms vanish).
struct StepCoeffs {
    double dt;
    double c_g;     // dt * g        predictor, implicit diagonal, final g3 weight
    double c_d;     // dt * d        accumulator f1 weight
    double c_1md;   // dt * (1 - d)  f2 weight
    double c_1mg;   // dt * (1 - g)  g2 weight
    double alpha;   // coefficient of the implicit matrix (I - alpha L)
    // driver-loop state (src/integrator_main.cpp:55-60, 76-95)
    double t;        // simulated time
    double prev_dt;  // dt of the previous step
    long long step;  // steps taken since the driver was reset
    long long cur;   // index of the step being taken
    int first;       // no step taken yet: the matrix is set from the first dt
    int pad;
};

struct Planes {
    double* f[6];  // rho, mx, my, E, bxf, byf
};
struct CPlanes {
    const double* f[6];
};

// Device-side status of a context, read back by the host only when it synchronises.
enum StatusBits : unsigned int {
    kStatusNonFinite = 1u << 0,
    kStatusCgNotConverged = 1u << 1,
    kStatusTimeout = 1u << 2,
    kStatusCgBreakdown = 1u << 3,
};

struct DeviceStatus {
    unsigned int flags;
    unsigned int pad;
    unsigned long long smax_bits;  // max CFL signal speed of the current state (as double bits)
    long long cg_products[2];      // matrix-vector products of the last step's two solves
    long long cg_products_total;
    double cg_last_rr[2];          // final recursive |r|^2 / |b|^2 of each solve
};

struct CgSync {
    unsigned long long count;  // zeroed before each launch of the solver
    unsigned int error;
    unsigned int pad;
};

// ------------------------------------------------------------------------------------------
// Small helpers

__device__ __forceinline__ int wrap(int i, int n) {
    if ((unsigned)i < (unsigned)n) return i;
    i %= n;
    return i < 0 ? i + n : i;
}

__device__ __forceinline__ unsigned long long global_timer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

template <int NT>
__device__ __forceinline__ double block_max(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v = smax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    if (w == 0) {
        v = (l < NT / 32) ? red[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v = smax(v, __shfl_xor_sync(0xffffffffu, v, o));
    }
    return v;  // valid in thread 0
}

// Deterministic block sum of K values per thread (fixed shuffle tree, fixed warp order).
template <int NT, int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double* red) {
#pragma unroll
    for (int k = 0; k < K; ++k)
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) red[w * K + k] = v[k];
    }
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double s = (l < NT / 32) ? red[l * K + k] : 0.0;
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            v[k] = s;
        }
    }
}

// ------------------------------------------------------------------------------------------
// Step coefficients (one thread). dt > 0 is taken as given; dt <= 0 selects the CFL step of the
// current state from the max signal speed found by the previous finalize / cfl-scan kernel
// (diagnostics.hpp:82-84 with courant and safety as parameters).
// alpha_mode: 0 = the given alpha (mhd_set_implicit_coefficient); 1 = (dt*eta)*g every step;
// 2 = the reference driver's rule: the matrix is built from the first dt and rebuilt only when
// eta > 0 and dt moved by more than 1e-10 relative to the previous step (integrator_main.cpp:55-60,
// 87-95). t_end > 0 clips dt so the time does not pass it (integrator_main.cpp:83).

__global__ void k_driver_reset(StepCoeffs* C) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    C->t = 0.0;
    C->prev_dt = 0.0;
    C->step = 0;
    C->cur = 0;
    C->first = 1;
}

__global__ void k_step_coeffs(StepCoeffs* C, const DeviceStatus* st, double dt, double alpha,
                              int alpha_mode, double eta, double hmin, double courant,
                              double safety, double g, double d, double t_end, double* dts_out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (dt <= 0.0) {
        const double smaxv = smax(__longlong_as_double((long long)st->smax_bits), 1e-8);
        double dt_res = __longlong_as_double(0x7ff0000000000000LL);  // +inf
        if (eta != 0.0) dt_res = hmin * hmin / (4.0 * eta);
        const double dt_hyp = courant * hmin / smaxv;
        dt = smin(dt_hyp, dt_res) * safety;
    }
    if (alpha_mode == 2) {
        if (C->first) {
            C->alpha = (dt * eta) * g;
            C->prev_dt = dt;
            C->first = 0;
        }
        if (t_end > 0.0 && C->t + dt > t_end) dt = t_end - C->t;
        if (eta > 0.0 && fabs(dt - C->prev_dt) > 1e-10 * dt) C->alpha = (dt * eta) * g;
        C->prev_dt = dt;
    } else {
        if (t_end > 0.0 && C->t + dt > t_end) dt = t_end - C->t;
        C->alpha = (alpha_mode == 1) ? (dt * eta) * g : alpha;
    }
    C->dt = dt;
    C->c_g = dt * g;
    C->c_d = dt * d;
    C->c_1md = dt * (1.0 - d);
    C->c_1mg = dt * (1.0 - g);
    C->cur = C->step;
    if (dts_out) dts_out[C->step] = dt;
    C->step += 1;
    C->t += dt;
}

// ------------------------------------------------------------------------------------------
// Explicit stage: fused halo gather -> primitives -> MUSCL x/y -> HLL x/y -> upwind-CT corner
// Ez -> flux divergence + curl Ez -> Butcher combination.
//
// Tile: TX x TY cells, halo 2 (MUSCL needs cells i-2..i+2 for the faces of a 1-cell ring).

constexpr int ST_TX = 32;
constexpr int ST_TY = 16;
constexpr int ST_NT = 256;
constexpr int ST_RW = ST_TX + 4;           // region width (cells)
constexpr int ST_RH = ST_TY + 4;           // region height
constexpr int ST_R = ST_RW * ST_RH;        // region cells
constexpr int ST_BXW = ST_RW + 1;          // bxf region: one extra face column on the right
constexpr int ST_BX = ST_BXW * ST_RH;
constexpr int ST_BYH = ST_RH + 1;          // byf region: one extra face row on top
constexpr int ST_BY = ST_RW * ST_BYH;
constexpr int ST_FXW = ST_TX + 1, ST_FXH = ST_TY + 2;  // x faces: right faces of cells -1..TX-1
constexpr int ST_FX = ST_FXW * ST_FXH;
constexpr int ST_FYW = ST_TX + 2, ST_FYH = ST_TY + 1;  // y faces: top faces of rows -1..TY-1
constexpr int ST_FY = ST_FYW * ST_FYH;
constexpr int ST_CW = ST_TX + 1, ST_CH = ST_TY + 1;    // corners 0..TX x 0..TY
constexpr int ST_C = ST_CW * ST_CH;
constexpr int ST_XW = ST_RW + 1, ST_XH = ST_RH + 1;    // solved corner field for B1 (stage 2)
constexpr int ST_X = ST_XW * ST_XH;

struct StageSmem {
    double rho[ST_R], vx[ST_R], vy[ST_R], p[ST_R], bxc[ST_R], byc[ST_R];
    double bxf[ST_BX], byf[ST_BY];
    union {
        double x[ST_X];  // stage 2: corner field of the first solve (gather phase only)
        double fx[5][ST_FX];
    } u;
    double fy[5][ST_FY];
    double ez[ST_C];
    double jz[ST_C];  // stage 2: eta*J_z(B1) at the corners (explicit resistive rate g2)
};

template <int MODE>
__global__ void __launch_bounds__(ST_NT, 2)
k_explicit_stage(Domain D, const StepCoeffs* __restrict__ C, CPlanes in,
                 const double* __restrict__ xsolve, Planes outA, Planes outB, int tiles_x) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    StageSmem& s = *reinterpret_cast<StageSmem*>(smem_raw);
    const int tid = threadIdx.x;
    const int tile = blockIdx.x;
    const int i0 = (tile % tiles_x) * ST_TX;
    const int j0 = (tile / tiles_x) * ST_TY;
    const int nx = D.nx, ny = D.ny;

    // ---- gather: hydro and faces over the halo region (periodic wrap)
    for (int k = tid; k < ST_R; k += ST_NT) {
        const int jj = k / ST_RW, ii = k - jj * ST_RW;
        const size_t g = (size_t)wrap(j0 - 2 + jj, ny) * nx + wrap(i0 - 2 + ii, nx);
        s.rho[k] = in.f[0][g];
        s.vx[k] = in.f[1][g];  // momenta / energy until the primitives overwrite them
        s.vy[k] = in.f[2][g];
        s.p[k] = in.f[3][g];
    }
    for (int k = tid; k < ST_BX; k += ST_NT) {
        const int jj = k / ST_BXW, ii = k - jj * ST_BXW;
        s.bxf[k] = in.f[4][(size_t)wrap(j0 - 2 + jj, ny) * nx + wrap(i0 - 2 + ii, nx)];
    }
    for (int k = tid; k < ST_BY; k += ST_NT) {
        const int jj = k / ST_RW, ii = k - jj * ST_RW;
        s.byf[k] = in.f[5][(size_t)wrap(j0 - 2 + jj, ny) * nx + wrap(i0 - 2 + ii, nx)];
    }
    if (MODE == 2) {
        // B1 = U1*_B + dt*g * (rate of the solved corner field), solvers.hpp:484-485, 528-529
        for (int k = tid; k < ST_X; k += ST_NT) {
            const int jj = k / ST_XW, ii = k - jj * ST_XW;
            s.u.x[k] = xsolve[(size_t)wrap(j0 - 2 + jj, ny) * nx + wrap(i0 - 2 + ii, nx)];
        }
        __syncthreads();
        const double cg = C->c_g;
        for (int k = tid; k < ST_BX; k += ST_NT) {
            const int jj = k / ST_BXW, ii = k - jj * ST_BXW;
            const double rate = -(s.u.x[(jj + 1) * ST_XW + ii] - s.u.x[jj * ST_XW + ii]) / D.dy;
            s.bxf[k] += rate * cg;
        }
        for (int k = tid; k < ST_BY; k += ST_NT) {
            const int jj = k / ST_RW, ii = k - jj * ST_RW;
            const double rate = (s.u.x[jj * ST_XW + ii + 1] - s.u.x[jj * ST_XW + ii]) / D.dx;
            s.byf[k] += rate * cg;
        }
    }
    __syncthreads();

    // ---- primitives on the region (Grid.hpp:82-136)
    for (int k = tid; k < ST_R; k += ST_NT) {
        const int jj = k / ST_RW, ii = k - jj * ST_RW;
        const double bx = (s.bxf[jj * ST_BXW + ii] + s.bxf[jj * ST_BXW + ii + 1]) / 2.0;
        const double by = (s.byf[jj * ST_RW + ii] + s.byf[(jj + 1) * ST_RW + ii]) / 2.0;
        double rho = s.rho[k];
        // Stage 2 sees the predictor after its density was floored in place (solvers.hpp:522-523)
        if (MODE == 2 && rho < kRhoFloor) rho = kRhoFloor;
        double vx, vy;
        const double p = primitives(rho, s.vx[k], s.vy[k], s.p[k], bx, by, vx, vy);
        s.rho[k] = rho;
        s.vx[k] = vx;
        s.vy[k] = vy;
        s.p[k] = p;
        s.bxc[k] = bx;
        s.byc[k] = by;
    }
    __syncthreads();

    // ---- x faces (solvers.hpp:224-236, 372): L = upper x-extrapolation of cell ii,
    //      R = lower x-extrapolation of cell ii+1, normal B = bxf of cell ii+1
    for (int k = tid; k < ST_FX; k += ST_NT) {
        const int fj = k / ST_FXW, fi = k - fj * ST_FXW;
        const int jj = fj + 1, ii = fi + 1;
        const int c = jj * ST_RW + ii;
        Prim L, R;
        L.rho = recon_hi(s.rho[c - 1], s.rho[c], s.rho[c + 1]);
        L.vx = recon_hi(s.vx[c - 1], s.vx[c], s.vx[c + 1]);
        L.vy = recon_hi(s.vy[c - 1], s.vy[c], s.vy[c + 1]);
        L.p = recon_hi(s.p[c - 1], s.p[c], s.p[c + 1]);
        L.by = recon_hi(s.byc[c - 1], s.byc[c], s.byc[c + 1]);
        R.rho = recon_lo(s.rho[c], s.rho[c + 1], s.rho[c + 2]);
        R.vx = recon_lo(s.vx[c], s.vx[c + 1], s.vx[c + 2]);
        R.vy = recon_lo(s.vy[c], s.vy[c + 1], s.vy[c + 2]);
        R.p = recon_lo(s.p[c], s.p[c + 1], s.p[c + 2]);
        R.by = recon_lo(s.byc[c], s.byc[c + 1], s.byc[c + 2]);
        L.bx = R.bx = s.bxf[jj * ST_BXW + ii + 1];
        const Flux F = hll<0>(L, R);
        s.u.fx[0][k] = F.rho;
        s.u.fx[1][k] = F.mx;
        s.u.fx[2][k] = F.my;
        s.u.fx[3][k] = F.E;
        s.u.fx[4][k] = F.bt;
    }
    // ---- y faces (solvers.hpp:238-250, 373): D = upper y-extrapolation of cell jj,
    //      U = lower y-extrapolation of cell jj+1, normal B = byf of cell jj+1
    for (int k = tid; k < ST_FY; k += ST_NT) {
        const int fj = k / ST_FYW, fi = k - fj * ST_FYW;
        const int jj = fj + 1, ii = fi + 1;
        const int c = jj * ST_RW + ii;
        const int W = ST_RW;
        Prim Dn, Up;
        Dn.rho = recon_hi(s.rho[c - W], s.rho[c], s.rho[c + W]);
        Dn.vx = recon_hi(s.vx[c - W], s.vx[c], s.vx[c + W]);
        Dn.vy = recon_hi(s.vy[c - W], s.vy[c], s.vy[c + W]);
        Dn.p = recon_hi(s.p[c - W], s.p[c], s.p[c + W]);
        Dn.bx = recon_hi(s.bxc[c - W], s.bxc[c], s.bxc[c + W]);
        Up.rho = recon_lo(s.rho[c], s.rho[c + W], s.rho[c + 2 * W]);
        Up.vx = recon_lo(s.vx[c], s.vx[c + W], s.vx[c + 2 * W]);
        Up.vy = recon_lo(s.vy[c], s.vy[c + W], s.vy[c + 2 * W]);
        Up.p = recon_lo(s.p[c], s.p[c + W], s.p[c + 2 * W]);
        Up.bx = recon_lo(s.bxc[c], s.bxc[c + W], s.bxc[c + 2 * W]);
        Dn.by = Up.by = s.byf[(jj + 1) * ST_RW + ii];
        const Flux F = hll<1>(Dn, Up);
        s.fy[0][k] = F.rho;
        s.fy[1][k] = F.mx;
        s.fy[2][k] = F.my;
        s.fy[3][k] = F.E;
        s.fy[4][k] = F.bt;
    }
    __syncthreads();

    // ---- corners (solvers.hpp:294-346); stage 2 also forms eta*J_z(B1) (solvers.hpp:450-461)
    for (int k = tid; k < ST_C; k += ST_NT) {
        const int tj = k / ST_CW, ti = k - tj * ST_CW;
        const double eN = -s.u.fx[4][(tj + 1) * ST_FXW + ti];
        const double eS = -s.u.fx[4][tj * ST_FXW + ti];
        const double eE = s.fy[4][tj * ST_FYW + ti + 1];
        const double eW = s.fy[4][tj * ST_FYW + ti];
        const int c = (tj + 2) * ST_RW + ti + 2;
        const double vxc = 0.25 * (s.vx[c] + s.vx[c - 1] + s.vx[c - ST_RW] + s.vx[c - ST_RW - 1]);
        const double vyc = 0.25 * (s.vy[c] + s.vy[c - 1] + s.vy[c - ST_RW] + s.vy[c - ST_RW - 1]);
        s.ez[k] = corner_ez(eN, eS, eE, eW, vxc, vyc, D.ct_mode);
        if (MODE == 2) {
            const int cb = (tj + 2) * ST_BXW + ti + 2;
            const int cy = (tj + 2) * ST_RW + ti + 2;
            const double dBy_dx = (s.byf[cy] - s.byf[cy - 1]) / D.dx;
            const double dBx_dy = (s.bxf[cb] - s.bxf[cb - ST_BXW]) / D.dy;
            s.jz[k] = D.eta * (dBy_dx - dBx_dy);
        }
    }
    __syncthreads();

    // ---- cells: rates (solvers.hpp:253-292) and the Butcher combination
    for (int k = tid; k < ST_TX * ST_TY; k += ST_NT) {
        const int tj = k / ST_TX, ti = k - tj * ST_TX;
        const int i = i0 + ti, j = j0 + tj;
        if (i >= nx || j >= ny) continue;
        const size_t g = (size_t)j * nx + i;
        const int xr = (tj + 1) * ST_FXW + ti + 1, xl = xr - 1;
        const int yt = (tj + 1) * ST_FYW + ti + 1, yb = yt - ST_FYW;
        double f[6];
#pragma unroll
        for (int q = 0; q < 4; ++q)
            f[q] = -((s.u.fx[q][xr] - s.u.fx[q][xl]) / D.dx + (s.fy[q][yt] - s.fy[q][yb]) / D.dy);
        const int e = tj * ST_CW + ti;
        f[4] = -(s.ez[e + ST_CW] - s.ez[e]) / D.dy;
        f[5] = (s.ez[e + 1] - s.ez[e]) / D.dx;
        if (MODE == 1) {
            const double cg = C->c_g, cd = C->c_d;
#pragma unroll
            for (int q = 0; q < 6; ++q) {
                const double u = in.f[q][g];
                outA.f[q][g] = u + f[q] * cg;  // predictor (solvers.hpp:512-517)
                // accumulator from the density-floored U^n (explicit_rhs floors it in place)
                const double ua = (q == 0 && u < kRhoFloor) ? kRhoFloor : u;
                outB.f[q][g] = ua + f[q] * cd;  // (solvers.hpp:548-553 / 590-595)
            }
        } else {
            const double c1md = C->c_1md, c1mg = C->c_1mg;
            double a[6];
#pragma unroll
            for (int q = 0; q < 6; ++q) a[q] = outB.f[q][g] + f[q] * c1md;  // :555-560 / :597-602
            // explicit resistive rate of B1 (solvers.hpp:484-485 with Ez = eta J_z)
            const double g2x = -(s.jz[e + ST_CW] - s.jz[e]) / D.dy;
            const double g2y = (s.jz[e + 1] - s.jz[e]) / D.dx;
            a[4] += g2x * c1mg;  // :565-566 / :604-605
            a[5] += g2y * c1mg;
#pragma unroll
            for (int q = 0; q < 6; ++q) outB.f[q][g] = a[q];
        }
    }
}

// ------------------------------------------------------------------------------------------
// Finalize: B2 = U2*_B + dt*g*rate(E2); g3 = explicit resistive rate of B2;
// B^{n+1} = U2*_B + dt*g*g3 (solvers.hpp:571-608); density floor of the new state in place
// (solvers.hpp:610-611); max CFL signal speed (diagnostics.hpp:60-78); non-finite check.

constexpr int FN_TX = 32, FN_TY = 16, FN_NT = 256;
constexpr int FN_XW = FN_TX + 4, FN_XH = FN_TY + 4;   // E2 over [i0-1, i0+TX+2] x [j0-1, j0+TY+2]
constexpr int FN_BXW = FN_TX + 2, FN_BXH = FN_TY + 3;  // bxf over [i0, i0+TX+1] x [j0-1, j0+TY+1]
constexpr int FN_BYW = FN_TX + 3, FN_BYH = FN_TY + 2;  // byf over [i0-1, i0+TX+1] x [j0, j0+TY+1]
constexpr int FN_EW = FN_TX + 2, FN_EH = FN_TY + 2;    // E3 corners [i0, i0+TX+1] x [j0, j0+TY+1]
constexpr int FN_NW = FN_TX + 1, FN_NH = FN_TY + 1;    // B^{n+1} on cells [i0, i0+TX] x [j0, j0+TY]

struct FinalSmem {
    double x[FN_XW * FN_XH];
    double bx0[FN_BXW * FN_BXH], by0[FN_BYW * FN_BYH];  // U2*_B
    double bx2[FN_BXW * FN_BXH], by2[FN_BYW * FN_BYH];  // B2
    double e3[FN_EW * FN_EH];
    double bxn[FN_NW * FN_NH], byn[FN_NW * FN_NH];
    double red[32];
};

__global__ void __launch_bounds__(FN_NT)
k_finalize(Domain D, const StepCoeffs* __restrict__ C, Planes acc, const double* __restrict__ xsolve,
           double* __restrict__ bx_out, double* __restrict__ by_out, DeviceStatus* st, int tiles_x) {
    __shared__ FinalSmem s;
    const int tid = threadIdx.x;
    const int i0 = (blockIdx.x % tiles_x) * FN_TX;
    const int j0 = (blockIdx.x / tiles_x) * FN_TY;
    const int nx = D.nx, ny = D.ny;
    for (int k = tid; k < FN_XW * FN_XH; k += FN_NT) {
        const int jj = k / FN_XW, ii = k - jj * FN_XW;
        s.x[k] = xsolve[(size_t)wrap(j0 - 1 + jj, ny) * nx + wrap(i0 - 1 + ii, nx)];
    }
    for (int k = tid; k < FN_BXW * FN_BXH; k += FN_NT) {
        const int jj = k / FN_BXW, ii = k - jj * FN_BXW;
        s.bx0[k] = acc.f[4][(size_t)wrap(j0 - 1 + jj, ny) * nx + wrap(i0 + ii, nx)];
    }
    for (int k = tid; k < FN_BYW * FN_BYH; k += FN_NT) {
        const int jj = k / FN_BYW, ii = k - jj * FN_BYW;
        s.by0[k] = acc.f[5][(size_t)wrap(j0 + jj, ny) * nx + wrap(i0 - 1 + ii, nx)];
    }
    __syncthreads();
    const double cg = C->c_g;
    // B2 (solvers.hpp:573-574); x index of corner (i,j) = (j - j0 + 1) * XW + (i - i0 + 1)
    for (int k = tid; k < FN_BXW * FN_BXH; k += FN_NT) {
        const int jj = k / FN_BXW, ii = k - jj * FN_BXW;  // face (i0+ii, j0-1+jj)
        const int xc = jj * FN_XW + ii + 1;
        const double rate = -(s.x[xc + FN_XW] - s.x[xc]) / D.dy;
        s.bx2[k] = s.bx0[k] + rate * cg;
    }
    for (int k = tid; k < FN_BYW * FN_BYH; k += FN_NT) {
        const int jj = k / FN_BYW, ii = k - jj * FN_BYW;  // face (i0-1+ii, j0+jj)
        const int xc = (jj + 1) * FN_XW + ii;
        const double rate = (s.x[xc + 1] - s.x[xc]) / D.dx;
        s.by2[k] = s.by0[k] + rate * cg;
    }
    __syncthreads();
    // E3 = eta J_z(B2) at corners (i0+ei, j0+ej) (solvers.hpp:450-461)
    for (int k = tid; k < FN_EW * FN_EH; k += FN_NT) {
        const int ej = k / FN_EW, ei = k - ej * FN_EW;
        const int cyy = ej * FN_BYW + ei + 1;        // byf(i, j): col i-(i0-1), row j-j0
        const int cxx = (ej + 1) * FN_BXW + ei;      // bxf(i, j): col i-i0, row j-(j0-1)
        const double dBy_dx = (s.by2[cyy] - s.by2[cyy - 1]) / D.dx;
        const double dBx_dy = (s.bx2[cxx] - s.bx2[cxx - FN_BXW]) / D.dy;
        s.e3[k] = D.eta * (dBy_dx - dBx_dy);
    }
    __syncthreads();
    // B^{n+1} = U2*_B + dt*g * g3 on cells [i0, i0+TX] x [j0, j0+TY] (solvers.hpp:607-608)
    for (int k = tid; k < FN_NW * FN_NH; k += FN_NT) {
        const int nj = k / FN_NW, ni = k - nj * FN_NW;
        const int e = nj * FN_EW + ni;
        const double g3x = -(s.e3[e + FN_EW] - s.e3[e]) / D.dy;
        const double g3y = (s.e3[e + 1] - s.e3[e]) / D.dx;
        s.bxn[k] = s.bx0[(nj + 1) * FN_BXW + ni] + g3x * cg;
        s.byn[k] = s.by0[nj * FN_BYW + ni + 1] + g3y * cg;
    }
    __syncthreads();
    double vmax = 0.0;
    bool bad = false;
    for (int k = tid; k < FN_TX * FN_TY; k += FN_NT) {
        const int tj = k / FN_TX, ti = k - tj * FN_TX;
        const int i = i0 + ti, j = j0 + tj;
        if (i >= nx || j >= ny) continue;
        const size_t g = (size_t)j * nx + i;
        const int n = tj * FN_NW + ti;
        const double bx = s.bxn[n], by = s.byn[n];
        bx_out[g] = bx;
        by_out[g] = by;
        // primitives of the new state (Grid.hpp:100-136), then the CFL speed of the cell
        double rho = acc.f[0][g];
        const double mx = acc.f[1][g], my = acc.f[2][g], E = acc.f[3][g];
        if (rho < kRhoFloor) acc.f[0][g] = kRhoFloor;
        const double bxc = (bx + s.bxn[n + 1]) / 2.0;
        const double byc = (by + s.byn[n + FN_NW]) / 2.0;
        double vx, vy;
        const double p = primitives(rho, mx, my, E, bxc, byc, vx, vy);
        const double sp = cfl_speed(rho, vx, vy, p, bxc, byc);
        if (sp > vmax) vmax = sp;
        bad |= !(isfinite(rho) && isfinite(mx) && isfinite(my) && isfinite(E) && isfinite(bx) &&
                 isfinite(by));
    }
    vmax = block_max<FN_NT>(vmax, s.red);
    if (__syncthreads_or(bad) && tid == 0) atomicOr(&st->flags, (unsigned)kStatusNonFinite);
    if (tid == 0) atomicMax(&st->smax_bits, (unsigned long long)__double_as_longlong(vmax));
}

// ------------------------------------------------------------------------------------------
// CFL speed of a state that did not come out of a step (diagnostics.hpp:44-88 scan only).

__global__ void __launch_bounds__(256)
k_cfl_scan(Domain D, CPlanes u, DeviceStatus* st) {
    __shared__ double red[32];
    const int nx = D.nx, ny = D.ny;
    const size_t n = (size_t)nx * ny;
    double vmax = 0.0;
    for (size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x; g < n;
         g += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(g / nx), i = (int)(g - (size_t)j * nx);
        const double bxc = (u.f[4][g] + u.f[4][(size_t)j * nx + wrap(i + 1, nx)]) / 2.0;
        const double byc = (u.f[5][g] + u.f[5][(size_t)wrap(j + 1, ny) * nx + i]) / 2.0;
        double rho = u.f[0][g], vx, vy;
        const double p = primitives(rho, u.f[1][g], u.f[2][g], u.f[3][g], bxc, byc, vx, vy);
        vmax = smax(vmax, cfl_speed(rho, vx, vy, p, bxc, byc));
    }
    vmax = block_max<256>(vmax, red);
    if (threadIdx.x == 0) atomicMax(&st->smax_bits, (unsigned long long)__double_as_longlong(vmax));
}

// ------------------------------------------------------------------------------------------
// Matrix-free conjugate gradient for (I - alpha L) E = eta J_z(B) on the corner nodes
// (solvers.hpp:404-489), with Eigen's ConjugateGradient defaults: x0 = 0, Jacobi scaling by the
// (constant) diagonal, stop when |r|^2 < max(tol^2 |b|^2, DBL_MIN), at most max_iters products.
//
// One persistent, cooperatively launched kernel runs the whole solve; its grid-wide barriers spin
// with a wall-clock limit and report a timeout instead of waiting forever. Each iteration has two
// phases separated by a barrier:
//   A: p_k = z_k + beta p_{k-1} on the tile and its 1-ring, q = A p_k, partial p.q   (reads r, p)
//   B: same p_k, q; x += alpha p_k; r_{k+1} = r_k - alpha q; partial r.r, r.z; writes x, r, p
// r and p are double-buffered (a phase reads the halo of one copy and writes the other).
// Partial sums go to per-block slots and every block reduces all slots in the same fixed order,
// so every block takes the same decisions and the result is deterministic.

constexpr int CG_TX = 64, CG_TY = 8, CG_NT = 256;
constexpr int CG_HW = CG_TX + 2, CG_HH = CG_TY + 2;  // tile + 1-ring
constexpr int CG_H = CG_HW * CG_HH;
constexpr int CG_BXW = CG_TX + 2, CG_BXH = CG_TY + 3;  // bxf over [i0-1, i0+TX] x [j0-2, j0+TY]
constexpr int CG_BYW = CG_TX + 3, CG_BYH = CG_TY + 2;  // byf over [i0-2, i0+TX] x [j0-1, j0+TY]

struct CgSmem {
    double r[CG_H];
    double p[CG_H];
    double bx[CG_BXW * CG_BXH];
    double by[CG_BYW * CG_BYH];
    double red[CG_NT / 32 * 4];
    double scal[8];
    int flag;
};

struct CgArgs {
    Domain D;
    const StepCoeffs* C;
    const double* bxf;  // the B* whose corner current forms the right-hand side
    const double* byf;
    double* x;
    double* r[2];
    double* p[2];
    double* partials;  // [2][gridDim.x][4]
    CgSync* sync;
    DeviceStatus* st;
    int solve_index;    // 0 or 1 within the step (for reporting)
    int tiles_x, ntiles;
    long long max_iters;
    double tol;
    double timeout_s;
    long long* prods_out;  // optional per-step record [step][2], indexed by C->cur
};

// Grid barrier with a wall-clock limit. Returns false when the solve must stop (timeout here or
// in another block); the caller then returns without touching memory again.
__device__ __forceinline__ bool grid_barrier(CgSync* sync, unsigned long long& target,
                                             unsigned long long deadline, int* sflag) {
    __syncthreads();
    target += gridDim.x;
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(&sync->count, 1ULL);
        int ok = 1;
        while (true) {
            const unsigned long long c = atomicAdd(&sync->count, 0ULL);
            if (c >= target) break;
            if (*(volatile unsigned int*)&sync->error) { ok = 0; break; }
            if (global_timer_ns() > deadline) {
                atomicExch(&sync->error, 1u);
                ok = 0;
                break;
            }
            __nanosleep(32);
        }
        __threadfence();
        *sflag = ok;
    }
    __syncthreads();
    return *sflag != 0;
}

// Sum the K partial slots of every block in a fixed order (all blocks get identical sums).
template <int K>
__device__ __forceinline__ void reduce_partials(const double* part, int nblocks, double* out,
                                                double* scal) {
    if (threadIdx.x < 32) {
        const int l = threadIdx.x;
        double v[K];
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] = 0.0;
        for (int b = l; b < nblocks; b += 32) {
#pragma unroll
            for (int k = 0; k < K; ++k) v[k] += __ldcg(&part[(size_t)b * 4 + k]);
        }
#pragma unroll
        for (int k = 0; k < K; ++k)
            for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
        if (l == 0) {
#pragma unroll
            for (int k = 0; k < K; ++k) scal[k] = v[k];
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) out[k] = scal[k];
    __syncthreads();
}

// (A p)_c with the row's entries summed in increasing column order for interior rows
// (bottom, left, centre, right, top), as the reference's compressed matrix product does.
__device__ __forceinline__ double apply_row(const double* p, int c, int W, double cx, double cy,
                                            double diag) {
    double acc = 0.0;
    acc += (-cy) * p[c - W];
    acc += (-cx) * p[c - 1];
    acc += diag * p[c];
    acc += (-cx) * p[c + 1];
    acc += (-cy) * p[c + W];
    return acc;
}

// p_k = z_k + beta p_{k-1} with z_k = r_k / diag, rounded step by step (no contraction) so that
// phases A and B form bit-identical directions.
__device__ __forceinline__ double next_direction(double invdiag, double r, double beta, double p) {
    return __dadd_rn(__dmul_rn(invdiag, r), __dmul_rn(beta, p));
}

__global__ void __launch_bounds__(CG_NT)
k_cg_solve(CgArgs a) {
    __shared__ CgSmem s;
    const int tid = threadIdx.x;
    const Domain D = a.D;
    const int nx = D.nx, ny = D.ny;
    const double alpha_m = a.C->alpha;
    const double cx = alpha_m / (D.dx * D.dx), cy = alpha_m / (D.dy * D.dy);
    const double diag = 1 + 2 * (cx + cy);
    const double invdiag = (diag == 0.0) ? 1.0 : 1.0 / diag;
    unsigned long long target = 0;
    const unsigned long long deadline =
        global_timer_ns() + (unsigned long long)(a.timeout_s * 1e9);
    const int G = gridDim.x;
    double* part[2] = {a.partials, a.partials + (size_t)G * 4};
    int phase = 0;

    // ---- phase A0: b = eta J_z(B*) on the tile + ring; r0 = b; p0 = b/d; q0 = A p0
    double acc3[3] = {0.0, 0.0, 0.0};  // b.b, b.z, p.q
    for (int t = blockIdx.x; t < a.ntiles; t += G) {
        const int i0 = (t % a.tiles_x) * CG_TX, j0 = (t / a.tiles_x) * CG_TY;
        for (int k = tid; k < CG_BXW * CG_BXH; k += CG_NT) {
            const int jj = k / CG_BXW, ii = k - jj * CG_BXW;
            s.bx[k] = a.bxf[(size_t)wrap(j0 - 2 + jj, ny) * nx + wrap(i0 - 1 + ii, nx)];
        }
        for (int k = tid; k < CG_BYW * CG_BYH; k += CG_NT) {
            const int jj = k / CG_BYW, ii = k - jj * CG_BYW;
            s.by[k] = a.byf[(size_t)wrap(j0 - 1 + jj, ny) * nx + wrap(i0 - 2 + ii, nx)];
        }
        __syncthreads();
        for (int k = tid; k < CG_H; k += CG_NT) {  // corner (i0-1+hi, j0-1+hj)
            const int hj = k / CG_HW, hi = k - hj * CG_HW;
            const int cyy = hj * CG_BYW + hi + 1;          // byf(i, j)
            const int cxx = (hj + 1) * CG_BXW + hi;        // bxf(i, j)
            const double dBy_dx = (s.by[cyy] - s.by[cyy - 1]) / D.dx;
            const double dBx_dy = (s.bx[cxx] - s.bx[cxx - CG_BXW]) / D.dy;
            const double b = D.eta * (dBy_dx - dBx_dy);
            s.r[k] = b;
            s.p[k] = __dmul_rn(invdiag, b);
        }
        __syncthreads();
        for (int k = tid; k < CG_TX * CG_TY; k += CG_NT) {
            const int tj = k / CG_TX, ti = k - tj * CG_TX;
            if (i0 + ti >= nx || j0 + tj >= ny) continue;
            const int c = (tj + 1) * CG_HW + ti + 1;
            const double b = s.r[c], pz = s.p[c];
            const double q = apply_row(s.p, c, CG_HW, cx, cy, diag);
            acc3[0] += b * b;
            acc3[1] += b * pz;
            acc3[2] += pz * q;
            a.r[0][(size_t)(j0 + tj) * nx + i0 + ti] = b;
        }
        __syncthreads();
    }
    block_sum<CG_NT, 3>(acc3, s.red);
    if (tid == 0) {
        part[phase & 1][(size_t)blockIdx.x * 4 + 0] = acc3[0];
        part[phase & 1][(size_t)blockIdx.x * 4 + 1] = acc3[1];
        part[phase & 1][(size_t)blockIdx.x * 4 + 2] = acc3[2];
    }
    if (!grid_barrier(a.sync, target, deadline, &s.flag)) {
        if (tid == 0 && blockIdx.x == 0) atomicOr(&a.st->flags, (unsigned)kStatusTimeout);
        return;
    }
    double sums[3];
    reduce_partials<3>(part[phase & 1], G, sums, s.scal);
    ++phase;
    const double bb = sums[0];
    double absNew = sums[1];
    double pq = sums[2];
    const double tol = a.tol;
    const double threshold = smax(tol * tol * bb, 2.2250738585072014e-308);
    long long products = 0;
    bool zero_solution = (bb == 0.0) || (bb < threshold);
    bool breakdown = !isfinite(bb);
    double rr_final = 0.0;
    bool converged = zero_solution;

    if (!zero_solution && !breakdown) {
        double beta = 0.0;  // beta_{k-1}; phase A of k = 0 already done
        for (long long k = 0; k < a.max_iters; ++k) {
            const double* rk = a.r[k & 1];
            double* rk1 = a.r[(k + 1) & 1];
            const double* pkm1 = a.p[(k + 1) & 1];  // p_{k-1} (unused when k == 0)
            double* pk = a.p[k & 1];
            if (k > 0) {
                // ---- phase A_k: p_k and p.Ap
                double acc1[1] = {0.0};
                for (int t = blockIdx.x; t < a.ntiles; t += G) {
                    const int i0 = (t % a.tiles_x) * CG_TX, j0 = (t / a.tiles_x) * CG_TY;
                    for (int q = tid; q < CG_H; q += CG_NT) {
                        const int hj = q / CG_HW, hi = q - hj * CG_HW;
                        const size_t g = (size_t)wrap(j0 - 1 + hj, ny) * nx + wrap(i0 - 1 + hi, nx);
                        s.p[q] = next_direction(invdiag, __ldcg(&rk[g]), beta, __ldcg(&pkm1[g]));
                    }
                    __syncthreads();
                    for (int q = tid; q < CG_TX * CG_TY; q += CG_NT) {
                        const int tj = q / CG_TX, ti = q - tj * CG_TX;
                        if (i0 + ti >= nx || j0 + tj >= ny) continue;
                        const int c = (tj + 1) * CG_HW + ti + 1;
                        acc1[0] += s.p[c] * apply_row(s.p, c, CG_HW, cx, cy, diag);
                    }
                    __syncthreads();
                }
                block_sum<CG_NT, 1>(acc1, s.red);
                if (tid == 0) part[phase & 1][(size_t)blockIdx.x * 4] = acc1[0];
                if (!grid_barrier(a.sync, target, deadline, &s.flag)) {
                    if (tid == 0 && blockIdx.x == 0) atomicOr(&a.st->flags, (unsigned)kStatusTimeout);
                    return;
                }
                double v[1];
                reduce_partials<1>(part[phase & 1], G, v, s.scal);
                ++phase;
                pq = v[0];
            }
            const double alpha = absNew / pq;
            // ---- phase B_k: updates
            double acc2[2] = {0.0, 0.0};
            for (int t = blockIdx.x; t < a.ntiles; t += G) {
                const int i0 = (t % a.tiles_x) * CG_TX, j0 = (t / a.tiles_x) * CG_TY;
                for (int q = tid; q < CG_H; q += CG_NT) {
                    const int hj = q / CG_HW, hi = q - hj * CG_HW;
                    const size_t g = (size_t)wrap(j0 - 1 + hj, ny) * nx + wrap(i0 - 1 + hi, nx);
                    const double rv = __ldcg(&rk[g]);
                    s.r[q] = rv;
                    s.p[q] = (k == 0) ? __dmul_rn(invdiag, rv)
                                      : next_direction(invdiag, rv, beta, __ldcg(&pkm1[g]));
                }
                __syncthreads();
                for (int q = tid; q < CG_TX * CG_TY; q += CG_NT) {
                    const int tj = q / CG_TX, ti = q - tj * CG_TX;
                    if (i0 + ti >= nx || j0 + tj >= ny) continue;
                    const int c = (tj + 1) * CG_HW + ti + 1;
                    const size_t g = (size_t)(j0 + tj) * nx + i0 + ti;
                    const double pv = s.p[c];
                    const double qv = apply_row(s.p, c, CG_HW, cx, cy, diag);
                    const double xv = (k == 0) ? alpha * pv : __ldcg(&a.x[g]) + alpha * pv;
                    const double rn = s.r[c] - alpha * qv;
                    a.x[g] = xv;
                    rk1[g] = rn;
                    pk[g] = pv;
                    acc2[0] += rn * rn;
                    acc2[1] += rn * (invdiag * rn);
                }
                __syncthreads();
            }
            block_sum<CG_NT, 2>(acc2, s.red);
            if (tid == 0) {
                part[phase & 1][(size_t)blockIdx.x * 4 + 0] = acc2[0];
                part[phase & 1][(size_t)blockIdx.x * 4 + 1] = acc2[1];
            }
            if (!grid_barrier(a.sync, target, deadline, &s.flag)) {
                if (tid == 0 && blockIdx.x == 0) atomicOr(&a.st->flags, (unsigned)kStatusTimeout);
                return;
            }
            double v2[2];
            reduce_partials<2>(part[phase & 1], G, v2, s.scal);
            ++phase;
            ++products;
            const double rr = v2[0];
            rr_final = rr;
            if (!isfinite(rr) || !isfinite(alpha)) { breakdown = true; break; }
            if (rr < threshold) { converged = true; break; }
            const double absOld = absNew;
            absNew = v2[1];
            beta = absNew / absOld;
        }
    }
    if (zero_solution || breakdown) {
        // x = 0 (Eigen returns the zero vector when b == 0); on breakdown the field is zeroed
        // too and the status says so.
        for (int t = blockIdx.x; t < a.ntiles; t += G) {
            const int i0 = (t % a.tiles_x) * CG_TX, j0 = (t / a.tiles_x) * CG_TY;
            for (int q = tid; q < CG_TX * CG_TY; q += CG_NT) {
                const int tj = q / CG_TX, ti = q - tj * CG_TX;
                if (i0 + ti >= nx || j0 + tj >= ny) continue;
                a.x[(size_t)(j0 + tj) * nx + i0 + ti] = 0.0;
            }
        }
    }
    if (blockIdx.x == 0 && tid == 0) {
        a.st->cg_products[a.solve_index] = products;
        if (a.prods_out) a.prods_out[2 * a.C->cur + a.solve_index] = products;
        a.st->cg_products_total += products;
        a.st->cg_last_rr[a.solve_index] = (bb > 0.0) ? rr_final / bb : 0.0;
        if (breakdown) atomicOr(&a.st->flags, (unsigned)(kStatusCgBreakdown | kStatusNonFinite));
        else if (!converged) atomicOr(&a.st->flags, (unsigned)kStatusCgNotConverged);
    }
}

// ------------------------------------------------------------------------------------------
// Diagnostics

// diagnostics.hpp:15-42: per-block sum of div^2 and max |div| over physical cells.
__global__ void __launch_bounds__(256)
k_divb_partial(Domain D, const double* __restrict__ bxf, const double* __restrict__ byf,
               double* partial) {
    __shared__ double red[64];
    const int nx = D.nx, ny = D.ny;
    const size_t n = (size_t)nx * ny;
    double s2[1] = {0.0};
    double mx = 0.0;
    for (size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x; g < n;
         g += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(g / nx), i = (int)(g - (size_t)j * nx);
        const double d = (bxf[(size_t)j * nx + wrap(i + 1, nx)] - bxf[g]) / D.dx +
                         (byf[(size_t)wrap(j + 1, ny) * nx + i] - byf[g]) / D.dy;
        s2[0] += d * d;
        mx = smax(mx, fabs(d));
    }
    block_sum<256, 1>(s2, red);
    __syncthreads();
    mx = block_max<256>(mx, red + 16);
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = s2[0];
        partial[2 * blockIdx.x + 1] = mx;
    }
}

__global__ void k_divb_final(const double* partial, int nblocks, long long ncells, double* out) {
    if (threadIdx.x != 0) return;
    double s2 = 0.0, mx = 0.0;
    for (int b = 0; b < nblocks; ++b) {
        s2 += partial[2 * b];
        mx = smax(mx, partial[2 * b + 1]);
    }
    out[0] = sqrt(s2 / (double)ncells);
    out[1] = mx;
}

// Primitives of the current state (Grid::computeCellB + computePrimitives), dense layout.
__global__ void __launch_bounds__(256)
k_primitives(Domain D, CPlanes u, double* rho_f, double* vx, double* vy, double* p, double* bxc,
             double* byc) {
    const int nx = D.nx, ny = D.ny;
    const size_t n = (size_t)nx * ny;
    for (size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x; g < n;
         g += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(g / nx), i = (int)(g - (size_t)j * nx);
        const double bx = (u.f[4][g] + u.f[4][(size_t)j * nx + wrap(i + 1, nx)]) / 2.0;
        const double by = (u.f[5][g] + u.f[5][(size_t)wrap(j + 1, ny) * nx + i]) / 2.0;
        double rho = u.f[0][g], ux, uy;
        const double pr = primitives(rho, u.f[1][g], u.f[2][g], u.f[3][g], bx, by, ux, uy);
        if (rho_f) rho_f[g] = rho;
        if (vx) vx[g] = ux;
        if (vy) vy[g] = uy;
        if (p) p[g] = pr;
        if (bxc) bxc[g] = bx;
        if (byc) byc[g] = by;
    }
}

// Dense periodic plane -> padded plane with ng periodic ghost layers (Grid.hpp:143-161).
__global__ void __launch_bounds__(256)
k_pad_plane(const double* __restrict__ src, double* __restrict__ dst, int nx, int ny, int ng) {
    const int W = nx + 2 * ng;
    const size_t n = (size_t)W * (ny + 2 * ng);
    for (size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x; g < n;
         g += (size_t)gridDim.x * blockDim.x) {
        const int pj = (int)(g / W), pi = (int)(g - (size_t)pj * W);
        dst[g] = src[(size_t)wrap(pj - ng, ny) * nx + wrap(pi - ng, nx)];
    }
}

// Density floor in place (what Grid::computePrimitives does to the stored state).
__global__ void k_floor_density(double* rho, size_t n) {
    for (size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x; g < n;
         g += (size_t)gridDim.x * blockDim.x)
        if (rho[g] < kRhoFloor) rho[g] = kRhoFloor;
}

}  // namespace mhd
