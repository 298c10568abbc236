// Shared device code of the ARS(2,2,2) IMEX step (reference: solvers.hpp:491-613 of
// RikibabManos/Magnetohydrodynamics_Simulator), for sm_100a, FP64: parameter blocks, helpers,
// the bounded grid barrier, the step-coefficient / driver kernel, the finalize kernel and the
// diagnostics. The explicit stages live in mhd_sweep.cuh, the implicit solve in mhd_cg_sweep.cuh.
//
// HBM layout: every field is a dense, row-major nx*ny plane of doubles (index j*nx + i), periodic in
// both directions; there are no ghost cells in device memory -- halos are read with periodic index
// wrap (the reference's ghost fill, Grid.hpp:143-161, is a periodic copy). bxf(i,j) lives on the
// left face of cell (i,j), byf(i,j) on its bottom face, and the corner field of the implicit solve
// at the bottom-left corner.
//
// One step is six kernels:
//   coeffs     dt (given or CFL), stage weights, matrix coefficient
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
    long long cg_products_sum[2];  // products of each of the step's two solves, summed over steps
    double cg_last_rr[2];          // final recursive |r|^2 / |b|^2 of each solve
};

struct CgSync {
    unsigned long long count;  // zeroed before each launch of the solver
    unsigned int error;
    unsigned int pad;
};

// Work split of a warp column sweep: column strips, each cut into row segments (one per warp).
struct SweepGeom {
    int strips_x;  // column strips
    int seg_h;     // rows per strip segment
    int segs_y;    // segments per column strip
    int nwarps;    // strips_x * segs_y
};

// ------------------------------------------------------------------------------------------
// Small helpers

__device__ __forceinline__ int wrap(int i, int n) {
    if ((unsigned)i < (unsigned)n) return i;
    i %= n;
    return i < 0 ? i + n : i;
}

// Launch shape of the 2-D grid-stride per-cell kernels: columns on x (256-thread blocks), rows on
// y (at most 65535 row blocks).
inline dim3 cell_grid(int nx, int ny) {
    return dim3((unsigned)((nx + 255) / 256), (unsigned)(ny < 65535 ? ny : 65535));
}

__device__ __forceinline__ unsigned long long global_timer_ns() {
#if defined(__CUDA_ARCH__)
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
#else
    return 0;  // host compilation of the kernel sources has no device timer
#endif
}

// Asynchronous 8-byte global -> shared copy (cp.async), its commit and its wait.
__device__ __forceinline__ void cp_async8(double* smem, const double* gmem) {
#if defined(__CUDA_ARCH__)
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
#else
    *smem = *gmem;  // host compilation of the kernel sources: a plain copy
#endif
}
__device__ __forceinline__ void cp_async_commit() {
#if defined(__CUDA_ARCH__)
    asm volatile("cp.async.commit_group;\n" ::: "memory");
#endif
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
#if defined(__CUDA_ARCH__)
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
#endif
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

// Grid barrier of a cooperatively launched kernel, with a wall-clock limit: returns false when the
// caller must stop (time ran out here or in another block); the caller then returns without
// touching shared state again. The counter is zeroed before each launch.
__device__ __forceinline__ bool grid_barrier(CgSync* sync, unsigned long long& target,
                                             unsigned long long deadline, int* sflag) {
    __syncthreads();
    target += gridDim.x;
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(&sync->count, 1ULL);
        int ok = 1;
        while (true) {
            // poll with a plain load: read-modify-writes here would queue in front of the
            // other blocks' arrivals at the same L2 address
            const unsigned long long c = *(volatile unsigned long long*)&sync->count;
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

// This lane's sum of K consecutive doubles of the 4-double partials of blocks lane, lane + 32, ...
// (< nblocks), in that order. The loads of four blocks are issued before they are added, so a lane
// waits for one round trip per four blocks instead of one per block; the sum is the same.
template <int K>
__device__ __forceinline__ void lane_partial_sum(const double* base, int nblocks, double (&v)[K]) {
    const int l = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = 0.0;
    for (int b0 = l; b0 < nblocks; b0 += 128) {
        double t[4][K];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int b = b0 + 32 * u;
#pragma unroll
            for (int k = 0; k < K; ++k) t[u][k] = (b < nblocks) ? __ldcg(&base[(size_t)b * 4 + k]) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (b0 + 32 * u < nblocks) {
#pragma unroll
                for (int k = 0; k < K; ++k) v[k] += t[u][k];
            }
    }
}

// Sum the K partial slots of every block in a fixed order (all blocks get identical sums).
template <int K>
__device__ __forceinline__ void reduce_partials(const double* part, int nblocks, double* out,
                                                double* scal) {
    if (threadIdx.x < 32) {
        const int l = threadIdx.x;
        double v[K];
        lane_partial_sum<K>(part, nblocks, v);
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

// ------------------------------------------------------------------------------------------
// Step coefficients (one thread). dt > 0 is taken as given; dt <= 0 selects the CFL step of the
// current state from the max signal speed found by the previous finalize / cfl-scan kernel
// (diagnostics.hpp:82-84 with courant and safety as parameters).
// alpha_mode: 0 = the given alpha (mhd_set_implicit_coefficient); 1 = (dt*eta)*g every step;
// 2 = the reference driver's rule: the matrix is built from the first dt and rebuilt only when
// eta > 0 and dt moved by more than 1e-10 relative to the previous step (integrator_main.cpp:55-60,
// 87-95). t_end > 0 clips dt so the time does not pass it (integrator_main.cpp:83).

static __global__ void k_driver_reset(StepCoeffs* C) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    C->t = 0.0;
    C->prev_dt = 0.0;
    C->step = 0;
    C->cur = 0;
    C->first = 1;
}

__device__ __forceinline__ void step_coeffs_one(StepCoeffs* C, const DeviceStatus* st, double dt,
                                                double alpha, int alpha_mode, double eta,
                                                double hmin, double courant, double safety,
                                                double g, double d, double t_end, double* dts_out) {
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

static __global__ void k_step_coeffs(StepCoeffs* C, const DeviceStatus* st, double dt, double alpha,
                              int alpha_mode, double eta, double hmin, double courant,
                              double safety, double g, double d, double t_end, double* dts_out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    step_coeffs_one(C, st, dt, alpha, alpha_mode, eta, hmin, courant, safety, g, d, t_end, dts_out);
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

static __global__ void __launch_bounds__(FN_NT)
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

static __global__ void __launch_bounds__(256)
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
// Diagnostics

// diagnostics.hpp:15-42: per-block sum of div^2 and max |div| over physical cells.
static __global__ void __launch_bounds__(256)
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

static __global__ void k_divb_final(const double* partial, int nblocks, long long ncells, double* out) {
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
static __global__ void __launch_bounds__(256)
k_primitives(Domain D, CPlanes u, double* rho_f, double* vx, double* vy, double* p, double* bxc,
             double* byc) {
    // 2-D launch: columns on x, rows on y (grid-stride in both)
    const int nx = D.nx, ny = D.ny;
    for (int j = blockIdx.y; j < ny; j += gridDim.y)
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nx; i += gridDim.x * blockDim.x) {
        const size_t g = (size_t)j * nx + i;
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

// Snapshot in the reference's file layout (write_data_to_binary_file, diagnostics.hpp:90-131, of
// the Grid after fillGhostPeriodic + computePrimitives, Grid.hpp:64-136): out[0..8] = nx, ny, ng,
// snapshot_rate, dx, dy, dt, divB rms, divB max (divb[0..1]), then the padded (nx+2ng) x (ny+2ng)
// planes rho (floored), E, p, vx, vy, bxc, byc. The reference's ghost fill makes every ghost cell
// the periodic image of a physical one (bxc, byc included: they are wrapped after computeCellB),
// so each padded cell is computed from its image.
static __global__ void __launch_bounds__(256)
k_snapshot_pack(Domain D, CPlanes u, int ng, double rate, double dt, const double* divb,
                double* out) {
    const int nx = D.nx, ny = D.ny;
    const int nxt = nx + 2 * ng, nyt = ny + 2 * ng;
    const size_t plane = (size_t)nxt * nyt;
    if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) {
        out[0] = (double)nx;
        out[1] = (double)ny;
        out[2] = (double)ng;
        out[3] = rate;
        out[4] = D.dx;
        out[5] = D.dy;
        out[6] = dt;
        out[7] = divb[0];
        out[8] = divb[1];
    }
    double* const pl = out + 9;
    for (int J = blockIdx.y; J < nyt; J += gridDim.y) {
        const int j = wrap(J - ng, ny);
        const size_t row = (size_t)j * nx, row_up = (size_t)wrap(j + 1, ny) * nx;
        for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < nxt; I += gridDim.x * blockDim.x) {
            const int i = wrap(I - ng, nx);
            const size_t g = row + i;
            const double bx = (u.f[4][g] + u.f[4][row + wrap(i + 1, nx)]) / 2.0;
            const double by = (u.f[5][g] + u.f[5][row_up + i]) / 2.0;
            double rho = u.f[0][g], vx, vy;
            const double E = u.f[3][g];
            const double p = primitives(rho, u.f[1][g], u.f[2][g], E, bx, by, vx, vy);
            const size_t o = (size_t)J * nxt + I;
            pl[o] = rho;
            pl[plane + o] = E;
            pl[2 * plane + o] = p;
            pl[3 * plane + o] = vx;
            pl[4 * plane + o] = vy;
            pl[5 * plane + o] = bx;
            pl[6 * plane + o] = by;
        }
    }
}

// Rate of the face field from a corner field E (solvers.hpp:472-488): bx' = -(E(i,j+1) - E(i,j))/dy,
// by' = (E(i+1,j) - E(i,j))/dx. With E == nullptr the corner field is eta*J_z(bxf, byf) itself
// (the explicit resistive term, solvers.hpp:450-463 and :470).
static __global__ void __launch_bounds__(256)
k_corner_rates(Domain D, const double* __restrict__ E, const double* __restrict__ bxf,
               const double* __restrict__ byf, double* __restrict__ bx_rate,
               double* __restrict__ by_rate) {
    const int nx = D.nx, ny = D.ny;
    const size_t n = (size_t)nx * ny;
    auto ez = [&](int i, int j) -> double {
        const size_t g = (size_t)wrap(j, ny) * nx + wrap(i, nx);
        if (E) return E[g];
        const double dBy_dx = (byf[g] - byf[(size_t)wrap(j, ny) * nx + wrap(i - 1, nx)]) / D.dx;
        const double dBx_dy = (bxf[g] - bxf[(size_t)wrap(j - 1, ny) * nx + wrap(i, nx)]) / D.dy;
        return D.eta * (dBy_dx - dBx_dy);
    };
    for (size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x; g < n;
         g += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(g / nx), i = (int)(g - (size_t)j * nx);
        const double e = ez(i, j);
        bx_rate[g] = -(ez(i, j + 1) - e) / D.dy;
        by_rate[g] = (ez(i + 1, j) - e) / D.dx;
    }
}

static __global__ void k_set_alpha(StepCoeffs* C, double alpha) {
    if (threadIdx.x == 0 && blockIdx.x == 0) C->alpha = alpha;
}

// Dense periodic plane -> padded plane with ng periodic ghost layers (Grid.hpp:143-161).
static __global__ void __launch_bounds__(256)
k_pad_plane(const double* __restrict__ src, double* __restrict__ dst, int nx, int ny, int ng) {
    const int W = nx + 2 * ng;
    const size_t n = (size_t)W * (ny + 2 * ng);
    for (size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x; g < n;
         g += (size_t)gridDim.x * blockDim.x) {
        const int pj = (int)(g / W), pi = (int)(g - (size_t)pj * W);
        dst[g] = src[(size_t)wrap(pj - ng, ny) * nx + wrap(pi - ng, nx)];
    }
}

}  // namespace mhd
