// One subdomain of a 2-D domain decomposition of the IMEX step (mhd_sub_* in include/mhd_b200.h).
//
// The reference advances one Grid on one thread (src/integrator_main.cpp:29-30 set its size); a
// grid beyond one GPU's memory is split into P x Q subdomains, one per GPU. Each subdomain keeps
// its interior nx x ny cells inside extended planes of (nx + 2H) x (ny + 2H) cells, H = MHD_SUB_HALO
// = 4 on every side. The explicit kernels of a single context (k_stage_sweep<1>, <2>,
// k_finalize_sweep) run unchanged on the extended planes as if they were a periodic grid: every
// interior output depends only on inputs within 3 cells (4 faces) of it, so the interior is exact
// when the halo rings hold the neighbours' values, and the wrapped halo outputs are never used. A
// caller (the decomposition driver) refreshes the rings between kernels by packing strips of the
// interior into buffers and unpacking the neighbours' strips into the rings (mhd_sub_pack /
// mhd_sub_unpack; across GPUs the buffers travel over NCCL).
//
// The implicit solve runs on the interior corners only, as a conjugate gradient with one kernel per
// phase: right-hand side eta J_z(B*) (solvers.hpp:450-461), q = A p, x/r/z update, direction. Each
// kernel returns its subdomain's partial sums (block partials added in a fixed order); the driver
// adds the subdomains' partials in a fixed order and takes Eigen's decisions on the host (x0 = 0,
// Jacobi scaling, stop at |r|^2 < max(tol^2 |b|^2, DBL_MIN)), exchanging p's 1-cell ring before
// every product. The CFL speed and the div B sums are interior scans whose maxima and sums the
// driver combines the same way.
//
// The decisions can also stay on the device (mhd_subcg_*): the phases write their subdomain's sums
// into a slot of a group's array, a one-thread kernel adds the slots in subdomain order and takes
// the same decisions into a control block, and the later phases read alpha, beta and "still
// iterating" from it, doing nothing once the solve has ended. The host then only polls the control
// block, a product behind, instead of waiting for the sums of every phase.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <math_constants.h>
#include <cmath>
#include <cstring>
#include <atomic>
#include <new>
#include <vector>

#include "../../include/mhd_b200.h"
#include "mhd_cg_sweep.cuh"
#include "mhd_finalize_sweep.cuh"
#include "mhd_host_util.h"
#include "mhd_kernels.cuh"
#include "mhd_sweep.cuh"

using namespace mhd;

namespace {

constexpr int kH = MHD_SUB_HALO;
constexpr int kSubNT = 256;
constexpr int kSubPlanes = 6 + 6 + 6 + 5;  // S, T, A, x r p q z
constexpr int kSubMaxBlocks = 1024;
constexpr int kSubCgNT = 256;  // threads of the single-sweep solve's blocks (8 warps, one ring each)
constexpr size_t kSubCgRingBytes = (size_t)(kSubCgNT / 32) * CG_RING * CG_SLOT * sizeof(double);

// Interior view of an extended plane: element (i, j) of the interior at base[(j + H) * nxe + i + H].
struct Interior {
    int nx, ny, nxe;
};

__device__ __forceinline__ size_t at(const Interior& v, int i, int j) {
    return (size_t)(j + kH) * v.nxe + (i + kH);
}

struct SubVecs {
    double* x;
    double* r;
    double* p;
    double* q;
    double* z;
};

struct SubScal {
    double cx, cy, diag, invdiag;
};

// Sum block partials (K per block) into out[K] with one warp, in a fixed order: lane l adds blocks
// l, l + 32, ... in turn, then the lanes' sums meet in a butterfly (the same order on every run; a
// single thread walking the blocks in turn took 25-48 us at 592 blocks, bound by load latency).
template <int K>
__global__ void k_sub_final(const double* __restrict__ part, int nblocks, double* out) {
    const int l = threadIdx.x;
    double s[K];
#pragma unroll
    for (int k = 0; k < K; ++k) s[k] = 0.0;
    for (int b = l; b < nblocks; b += 32) {
#pragma unroll
        for (int k = 0; k < K; ++k) s[k] += part[(size_t)b * K + k];
    }
#pragma unroll
    for (int k = 0; k < K; ++k)
        for (int o = 16; o > 0; o >>= 1) s[k] += __shfl_xor_sync(0xffffffffu, s[k], o);
    if (l == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) out[k] = s[k];
    }
}

// The step's coefficients and the implicit matrix (I - alpha L) of the solves: off-diagonal
// cx = alpha/dx^2, cy = alpha/dy^2, diagonal 1 + 2 (cx + cy) (solvers.hpp:404-443), on the device
// so that a captured solve reads this step's matrix.
__device__ __forceinline__ void sub_set_coeffs(StepCoeffs* C, SubScal* sc, double dt, double alpha, double g,
                                               double d, double dx, double dy) {
    C->dt = dt;
    C->c_g = dt * g;
    C->c_d = dt * d;
    C->c_1md = dt * (1.0 - d);
    C->c_1mg = dt * (1.0 - g);
    C->alpha = alpha;
    const double cx = alpha / (dx * dx), cy = alpha / (dy * dy);
    const double diag = 1.0 + 2.0 * (cx + cy);
    sc->cx = cx;
    sc->cy = cy;
    sc->diag = diag;
    sc->invdiag = (diag == 0.0) ? 1.0 : 1.0 / diag;
}

__global__ void k_sub_set_coeffs(StepCoeffs* C, SubScal* sc, double dt, double alpha, double g, double d,
                                 double dx, double dy) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    sub_set_coeffs(C, sc, dt, alpha, g, d, dx, dy);
}

// The CFL step of P x Q subdomains on the device (diagnostics.hpp:82-86 from the largest interior
// signal speed of all of them, as the host driver computes it) and each subdomain's step
// coefficients and matrix for that dt, alpha = (dt eta) g; dt goes to ctl[MHD_SUBCG_DT] and a
// non-finite state to ctl[MHD_SUBCG_CFL_NONFINITE].
constexpr int kSubCflMax = 64;
struct SubCflTargets {
    const unsigned long long* speed[kSubCflMax];  // each subdomain's (max speed bits, non-finite flag)
    StepCoeffs* coeffs[kSubCflMax];
    SubScal* sc[kSubCflMax];
};

__global__ void k_subcg_cfl_step(SubCflTargets t, int count, double dx, double dy, double eta, double courant,
                                 double safety, double g, double d, double* ctl) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    unsigned long long bits = 0, bad = 0;
    for (int i = 0; i < count; ++i) {
        bits = bits > t.speed[i][0] ? bits : t.speed[i][0];  // non-negative doubles order as their bits
        bad |= t.speed[i][1];
    }
    double smaxv = __longlong_as_double((long long)bits);
    if (smaxv < 1e-8) smaxv = 1e-8;
    const double hmin = dx < dy ? dx : dy;
    const double dt_res = (eta == 0.0) ? CUDART_INF : hmin * hmin / (4.0 * eta);
    const double dt_hyp = courant * hmin / smaxv;
    const double dt = (dt_res < dt_hyp ? dt_res : dt_hyp) * safety;
    const double alpha = (dt * eta) * g;
    for (int i = 0; i < count; ++i) sub_set_coeffs(t.coeffs[i], t.sc[i], dt, alpha, g, d, dx, dy);
    ctl[MHD_SUBCG_DT] = dt;
    ctl[MHD_SUBCG_CFL_NONFINITE] = bad ? 1.0 : 0.0;
}

// Copy the rectangle [x0, x0 + w) x [y0, y0 + h) of np extended planes (row pitch nxe) into buf
// (plane by plane, row-major) or back.
template <bool kPack>
__global__ void __launch_bounds__(kSubNT)
k_sub_strip(Planes set, int np, int nxe, int x0, int y0, int w, int h, double* buf) {
    const size_t per = (size_t)w * h;
    const size_t total = per * np;
    for (size_t t = (size_t)blockIdx.x * kSubNT + threadIdx.x; t < total; t += (size_t)gridDim.x * kSubNT) {
        const int k = (int)(t / per);
        const size_t e = t - (size_t)k * per;
        const int jj = (int)(e / w), ii = (int)(e - (size_t)jj * w);
        double* plane = set.f[0];
#pragma unroll
        for (int q = 1; q < 6; ++q)
            if (k == q) plane = set.f[q];
        const size_t g = (size_t)(y0 + jj) * nxe + (x0 + ii);
        if (kPack) buf[t] = plane[g];
        else plane[g] = buf[t];
    }
}

// The ring of one subdomain (cells within `width` of its interior), gathered from the interiors of
// the 3 x 3 subdomains around it (src[a][b]: the one dy = a - 1, dx = b - 1 away, periodic; itself
// at [1][1] when the partition has one subdomain along an axis). A ring cell west of the interior
// lies in the west neighbour's last columns, a corner cell in the diagonal neighbour's corner.
struct RingSources {
    const double* f[3][3][6];
    int nxe[3][3];
    int nx_w, ny_s;  // interior columns of the west neighbours, rows of the south neighbours
};

__global__ void __launch_bounds__(kSubNT)
k_sub_ring_gather(Planes dst, int np, Interior v, int width, RingSources src) {
    const int w = width, rowlen = v.nx + 2 * w;
    const size_t band = (size_t)w * rowlen;         // cells of the south (or north) band
    const size_t total = 2 * band + (size_t)2 * w * v.ny;
    for (size_t t = (size_t)blockIdx.x * kSubNT + threadIdx.x; t < total; t += (size_t)gridDim.x * kSubNT) {
        int ii, jj;  // interior coordinates of the ring cell, in [-w, n + w)
        if (t < 2 * band) {
            const int r = (int)(t / rowlen);
            ii = (int)(t - (size_t)r * rowlen) - w;
            jj = (r < w) ? r - w : v.ny + (r - w);
        } else {
            const size_t u = t - 2 * band;
            const int r = (int)(u / (2 * w)), c = (int)(u - (size_t)r * 2 * w);
            jj = r;
            ii = (c < w) ? c - w : v.nx + (c - w);
        }
        const int b = (ii < 0) ? 0 : (ii >= v.nx ? 2 : 1);
        const int a = (jj < 0) ? 0 : (jj >= v.ny ? 2 : 1);
        const int si = (b == 0) ? src.nx_w + ii : (b == 2 ? ii - v.nx : ii);  // the source's interior column
        const int sj = (a == 0) ? src.ny_s + jj : (a == 2 ? jj - v.ny : jj);
        const size_t gs = (size_t)(sj + kH) * src.nxe[a][b] + (si + kH);
        const size_t gd = at(v, ii, jj);
        for (int k = 0; k < np; ++k) dst.f[k][gd] = src.f[a][b][k][gs];
    }
}

// b = eta J_z(B*) on the interior corners (solvers.hpp:450-461), r = b, z = p = b/d, x = 0;
// block partials |b|^2, r.z.
__global__ void __launch_bounds__(kSubNT)
k_sub_cg_rhs(Interior v, double eta, double idx, double idy, const double* __restrict__ bxf,
             const double* __restrict__ byf, SubVecs V, const SubScal* __restrict__ sp, double* part) {
    const SubScal s = *sp;
    __shared__ double red[kSubNT / 32 * 2];
    double acc[2] = {0.0, 0.0};
    const size_t n = (size_t)v.nx * v.ny;
    const Domain D{v.nx, v.ny, 0.0, 0.0, eta, 0};
    for (size_t t = (size_t)blockIdx.x * kSubNT + threadIdx.x; t < n; t += (size_t)gridDim.x * kSubNT) {
        const int j = (int)(t / v.nx), i = (int)(t - (size_t)j * v.nx);
        const size_t g = at(v, i, j);
        const double b = corner_rhs(D, idx, idy, byf[g], byf[g - 1], bxf[g], bxf[g - v.nxe]);
        const double z = __dmul_rn(s.invdiag, b);
        V.r[g] = b;
        V.z[g] = z;
        V.p[g] = z;
        V.x[g] = 0.0;
        acc[0] += b * b;
        acc[1] += b * z;
    }
    block_sum<kSubNT, 2>(acc, red);
    if (threadIdx.x == 0) {
        part[(size_t)blockIdx.x * 2] = acc[0];
        part[(size_t)blockIdx.x * 2 + 1] = acc[1];
    }
}

// q = A p = (I - alpha L) p on the interior corners (p's 1-cell ring must hold the neighbours'
// values), in the single context's operand order; block partial p.q.
__global__ void __launch_bounds__(kSubNT)
k_sub_cg_matvec(Interior v, SubVecs V, const SubScal* __restrict__ sp, const double* ctl, double* part) {
    const SubScal s = *sp;
    __shared__ double red[kSubNT / 32];
    if (ctl && ctl[MHD_SUBCG_ACTIVE] == 0.0) return;
    double acc[1] = {0.0};
    const size_t n = (size_t)v.nx * v.ny;
    for (size_t t = (size_t)blockIdx.x * kSubNT + threadIdx.x; t < n; t += (size_t)gridDim.x * kSubNT) {
        const int j = (int)(t / v.nx), i = (int)(t - (size_t)j * v.nx);
        const size_t g = at(v, i, j);
        double q = 0.0;
        q += (-s.cy) * V.p[g - v.nxe];
        q += (-s.cx) * V.p[g - 1];
        q += s.diag * V.p[g];
        q += (-s.cx) * V.p[g + 1];
        q += (-s.cy) * V.p[g + v.nxe];
        V.q[g] = q;
        acc[0] += V.p[g] * q;
    }
    block_sum<kSubNT, 1>(acc, red);
    if (threadIdx.x == 0) part[blockIdx.x] = acc[0];
}

// x += alpha p, r -= alpha q, z = r/d on the interior; block partials |r|^2, r.z.
__global__ void __launch_bounds__(kSubNT)
k_sub_cg_update(Interior v, SubVecs V, const SubScal* __restrict__ sp, double alpha, const double* ctl,
                double* part) {
    const SubScal s = *sp;
    __shared__ double red[kSubNT / 32 * 2];
    if (ctl) {
        if (ctl[MHD_SUBCG_ACTIVE] == 0.0) return;
        alpha = ctl[MHD_SUBCG_ALPHA];
    }
    double acc[2] = {0.0, 0.0};
    const size_t n = (size_t)v.nx * v.ny;
    for (size_t t = (size_t)blockIdx.x * kSubNT + threadIdx.x; t < n; t += (size_t)gridDim.x * kSubNT) {
        const int j = (int)(t / v.nx), i = (int)(t - (size_t)j * v.nx);
        const size_t g = at(v, i, j);
        V.x[g] = fma(alpha, V.p[g], V.x[g]);
        const double r = fma(-alpha, V.q[g], V.r[g]);
        V.r[g] = r;
        const double z = __dmul_rn(s.invdiag, r);
        V.z[g] = z;
        acc[0] += r * r;
        acc[1] += r * z;
    }
    block_sum<kSubNT, 2>(acc, red);
    if (threadIdx.x == 0) {
        part[(size_t)blockIdx.x * 2] = acc[0];
        part[(size_t)blockIdx.x * 2 + 1] = acc[1];
    }
}

// p = z + beta p on the interior.
__global__ void __launch_bounds__(kSubNT) k_sub_cg_dir(Interior v, SubVecs V, double beta, const double* ctl) {
    if (ctl) {
        if (ctl[MHD_SUBCG_ACTIVE] == 0.0) return;
        beta = ctl[MHD_SUBCG_BETA];
    }
    const size_t n = (size_t)v.nx * v.ny;
    for (size_t t = (size_t)blockIdx.x * kSubNT + threadIdx.x; t < n; t += (size_t)gridDim.x * kSubNT) {
        const int j = (int)(t / v.nx), i = (int)(t - (size_t)j * v.nx);
        const size_t g = at(v, i, j);
        V.p[g] = __dadd_rn(V.z[g], __dmul_rn(beta, V.p[g]));
    }
}

// x = 0 on the interior (with a control block: only after a solve that met a non-finite value)
__global__ void __launch_bounds__(kSubNT) k_sub_zero_interior(Interior v, double* x, const double* ctl) {
    if (ctl && ctl[MHD_SUBCG_STATUS] != (double)MHD_SUBCG_NONFINITE) return;
    const size_t n = (size_t)v.nx * v.ny;
    for (size_t t = (size_t)blockIdx.x * kSubNT + threadIdx.x; t < n; t += (size_t)gridDim.x * kSubNT) {
        const int j = (int)(t / v.nx), i = (int)(t - (size_t)j * v.nx);
        x[at(v, i, j)] = 0.0;
    }
}

// ---- the single-sweep form of the solve: the single context's sweeps (cg_rhs_segment,
// cg_iter_segment) over the interior of the extended planes. An interior corner's results need the
// rows and columns within 2 of it, so r_k and p_{k-1} are exchanged with a ring of 2 before each
// iteration (the set MHD_SUB_SET_CG_EVEN / _ODD); their wrapped ring values are never used.
// Vectors: r[0] = r, r[1] = z, p[0] = p, p[1] = q of the subdomain.

// Publish this block's 4 partials; the last block to arrive adds every block's partials in the
// fixed order of k_sub_final (lane-strided, then a butterfly) into slot[0..3] and resets the
// arrival counter for the next launch.
__device__ __forceinline__ void sub_sums_to_slot(const double (&acc)[4], double* part, unsigned* arrivals,
                                                 double* slot) {
    __shared__ bool last;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int c = 0; c < 4; ++c) part[(size_t)blockIdx.x * 4 + c] = acc[c];
        __threadfence();
        last = atomicAdd(arrivals, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x >= 32) return;
    __threadfence();
    const int l = threadIdx.x;
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (int b = l; b < (int)gridDim.x; b += 32) {
#pragma unroll
        for (int c = 0; c < 4; ++c) s[c] += __ldcg(&part[(size_t)b * 4 + c]);
    }
#pragma unroll
    for (int c = 0; c < 4; ++c)
        for (int o = 16; o > 0; o >>= 1) s[c] += __shfl_xor_sync(0xffffffffu, s[c], o);
    if (l == 0) {
#pragma unroll
        for (int c = 0; c < 4; ++c) slot[c] = s[c];
        *arrivals = 0u;
    }
}

__device__ __forceinline__ CgScal sub_cg_scal(const SubScal* sp) {
    CgScal s;
    s.cx = sp->cx;
    s.cy = sp->cy;
    s.diag = sp->diag;
    s.invdiag = sp->invdiag;
    s.beta = 0.0;
    s.alpha = 0.0;
    s.alpha_prev = 0.0;
    return s;
}

// b = eta J_z(B*), r0 = b on the interior; block partials |b|^2, b.z0, z0.A z0.
__global__ void __launch_bounds__(kSubCgNT, 2)
k_sub_cg_sweep_rhs(CgSweepArgs a, const SubScal* __restrict__ sp, double* part, unsigned* arrivals,
                   double* slot) {
    extern __shared__ __align__(16) double sub_ring_mem[];
    __shared__ double red[kSubCgNT / 32 * 4];
    double* const ring = sub_ring_mem + (size_t)(threadIdx.x >> 5) * CG_RING * CG_SLOT;
    const CgScal s = sub_cg_scal(sp);
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    const int rend = a.D.ny - kH;
    for (int w = blockIdx.x * (kSubCgNT / 32) + (threadIdx.x >> 5); w < a.nwarps; w += gridDim.x * (kSubCgNT / 32)) {
        const int sx = w % a.strips_x, r0w = kH + (w / a.strips_x) * a.seg_h;
        cg_rhs_segment<true>(a, s, sx, r0w, min(r0w + a.seg_h, rend), 1, a.r[0], ring, acc);
    }
    block_sum<kSubCgNT, 4>(acc, red);
    sub_sums_to_slot(acc, part, arrivals, slot);
}

// Iteration k = products so far (from the control block, which also gives alpha, beta and
// alpha_{k-1}); nothing once the solve has ended. Block partials r.r, r.z, z.Az, z.q_k. kNb: the
// cells around the interior are read from the neighbours' interiors (nb), not from the rings.
template <bool kNb>
__global__ void __launch_bounds__(kSubCgNT, 2)
k_sub_cg_sweep_iter(CgSweepArgs a, const SubScal* __restrict__ sp, const double* ctl, double* part,
                    unsigned* arrivals, double* slot, CgSubNeighbours nb) {
    if (ctl[MHD_SUBCG_ACTIVE] == 0.0) return;
    extern __shared__ __align__(16) double sub_ring_mem[];
    __shared__ double red[kSubCgNT / 32 * 4];
    double* const ring = sub_ring_mem + (size_t)(threadIdx.x >> 5) * CG_RING * CG_SLOT;
    CgScal s = sub_cg_scal(sp);
    s.alpha = ctl[MHD_SUBCG_ALPHA];
    s.beta = ctl[MHD_SUBCG_BETA];
    s.alpha_prev = ctl[MHD_SUBCG_ALPHA_PREV];
    const long long k = (long long)ctl[MHD_SUBCG_PRODUCTS];
    const bool odd = (k & 1) != 0;
    const double* rk = odd ? a.r[1] : a.r[0];
    double* rk1 = odd ? a.r[0] : a.r[1];
    const double* pkm1 = odd ? a.p[0] : a.p[1];
    double* pk = odd ? a.p[1] : a.p[0];
    const int dir = odd ? 1 : -1;  // alternate (the right-hand side runs upwards)
    const int xm = cg_xmode(k);
    const int rsel = odd ? 1 : 0, psel = odd ? 0 : 1;  // the neighbours' r_k and p_{k-1}
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    const int rend = a.D.ny - kH;
    for (int w = blockIdx.x * (kSubCgNT / 32) + (threadIdx.x >> 5); w < a.nwarps; w += gridDim.x * (kSubCgNT / 32)) {
        const int sx = w % a.strips_x, r0w = kH + (w / a.strips_x) * a.seg_h;
        const int r1w = min(r0w + a.seg_h, rend);
        if (k == 0)
            cg_iter_segment<true, kXSkip, true, kNb>(a, s, sx, r0w, r1w, dir, rk, pkm1, rk1, pk, ring, acc,
                                                     &nb, rsel, psel);
        else if (xm == kXSkip)
            cg_iter_segment<false, kXSkip, true, kNb>(a, s, sx, r0w, r1w, dir, rk, pkm1, rk1, pk, ring, acc,
                                                      &nb, rsel, psel);
        else if (xm == kXPairFirst)
            cg_iter_segment<false, kXPairFirst, true, kNb>(a, s, sx, r0w, r1w, dir, rk, pkm1, rk1, pk, ring,
                                                           acc, &nb, rsel, psel);
        else
            cg_iter_segment<false, kXPair, true, kNb>(a, s, sx, r0w, r1w, dir, rk, pkm1, rk1, pk, ring, acc,
                                                      &nb, rsel, psel);
    }
    block_sum<kSubCgNT, 4>(acc, red);
    sub_sums_to_slot(acc, part, arrivals, slot);
}

// The end of a single-sweep solve (as k_cg_sweep's): x = 0 after a zero right-hand side or a
// breakdown; after an even last iteration k, its alpha_k p_k (x_0 = 0 when k = 0).
__global__ void __launch_bounds__(kSubNT)
k_sub_cg_sweep_finish(Interior v, double* x, const double* p0, const double* ctl) {
    const bool zero = ctl[MHD_SUBCG_ZERO] != 0.0;
    const long long kl = (long long)ctl[MHD_SUBCG_K_LAST];
    const double al = ctl[MHD_SUBCG_ALPHA_LAST];
    const bool fix = !zero && kl >= 0 && (kl & 1) == 0;  // the last iteration wrote p_k into p[0]
    if (!zero && !fix) return;
    const size_t n = (size_t)v.nx * v.ny;
    for (size_t t = (size_t)blockIdx.x * kSubNT + threadIdx.x; t < n; t += (size_t)gridDim.x * kSubNT) {
        const int j = (int)(t / v.nx), i = (int)(t - (size_t)j * v.nx);
        const size_t g = at(v, i, j);
        x[g] = zero ? 0.0 : (kl == 0 ? al * p0[g] : fma(al, p0[g], x[g]));
    }
}

// The decisions of a decomposed solve after one of its phases (phase 0 right-hand side, 1 q = A p,
// 2 the x/r/z update; the single-sweep form: 3 right-hand side, 4 an iteration), from the count
// subdomains' sums (slots[4 i + k], added in subdomain order
// from 0.0, as the host driver adds them) into the control block: Eigen's ConjugateGradient rules
// (x0 = 0; stop when |r|^2 < max(tol^2 |b|^2, DBL_MIN); at most max_products products), the
// single-context solver's (solvers.hpp:445-489).
__host__ __device__ inline void subcg_decide(double* ctl, const double* slots, int count, int phase,
                                             double tol, double max_products) {
    double s0 = 0.0, s1 = 0.0;
    for (int i = 0; i < count; ++i) {
        s0 += slots[4 * i];
        s1 += slots[4 * i + 1];
    }
    if (phase == 0) {
        ctl[MHD_SUBCG_PRODUCTS] = 0.0;
        ctl[MHD_SUBCG_BB] = s0;
        ctl[MHD_SUBCG_ABSNEW] = s1;
        const double thr = tol * tol * s0;
        ctl[MHD_SUBCG_THRESHOLD] = thr > DBL_MIN ? thr : DBL_MIN;
        ctl[MHD_SUBCG_STATUS] = MHD_SUBCG_OK;
        if (!isfinite(s0)) {
            ctl[MHD_SUBCG_STATUS] = MHD_SUBCG_NONFINITE;
            ctl[MHD_SUBCG_ACTIVE] = 0.0;
        } else {
            // a zero (or negligible) right-hand side: x = 0, no product
            ctl[MHD_SUBCG_ACTIVE] = (s0 == 0.0 || s0 < ctl[MHD_SUBCG_THRESHOLD]) ? 0.0 : 1.0;
        }
        return;
    }
    if (phase == 3) {
        // the single-sweep form (the single context's k_cg_sweep): |b|^2, b.z0, z0.A z0
        double s2 = 0.0;
        for (int i = 0; i < count; ++i) s2 += slots[4 * i + 2];
        ctl[MHD_SUBCG_PRODUCTS] = 0.0;
        ctl[MHD_SUBCG_BB] = s0;
        ctl[MHD_SUBCG_ABSNEW] = s1;
        ctl[MHD_SUBCG_PQ] = s2;
        const double thr = tol * tol * s0;
        ctl[MHD_SUBCG_THRESHOLD] = thr > DBL_MIN ? thr : DBL_MIN;
        ctl[MHD_SUBCG_STATUS] = MHD_SUBCG_OK;
        ctl[MHD_SUBCG_BETA] = 0.0;
        ctl[MHD_SUBCG_ALPHA_PREV] = 0.0;
        ctl[MHD_SUBCG_K_LAST] = -1.0;
        ctl[MHD_SUBCG_ALPHA_LAST] = 0.0;
        const bool zero = (s0 == 0.0) || (s0 < ctl[MHD_SUBCG_THRESHOLD]);
        const bool breakdown = !isfinite(s0);
        if (breakdown) ctl[MHD_SUBCG_STATUS] = MHD_SUBCG_NONFINITE;
        ctl[MHD_SUBCG_ZERO] = (zero || breakdown) ? 1.0 : 0.0;
        ctl[MHD_SUBCG_ACTIVE] = (zero || breakdown) ? 0.0 : 1.0;
        if (!(zero || breakdown)) ctl[MHD_SUBCG_ALPHA] = s1 / s2;
        return;
    }
    if (ctl[MHD_SUBCG_ACTIVE] == 0.0) return;
    if (phase == 4) {
        // after iteration k of the single-sweep form: r.r, r.z, z.Az, z.q_k
        double s2 = 0.0, s3 = 0.0;
        for (int i = 0; i < count; ++i) {
            s2 += slots[4 * i + 2];
            s3 += slots[4 * i + 3];
        }
        const double k = ctl[MHD_SUBCG_PRODUCTS];
        ctl[MHD_SUBCG_K_LAST] = k;
        ctl[MHD_SUBCG_ALPHA_LAST] = ctl[MHD_SUBCG_ALPHA];
        ctl[MHD_SUBCG_PRODUCTS] = k + 1.0;
        ctl[MHD_SUBCG_RR] = s0;
        if (!isfinite(s0) || !isfinite(ctl[MHD_SUBCG_ALPHA])) {
            ctl[MHD_SUBCG_STATUS] = MHD_SUBCG_NONFINITE;
            ctl[MHD_SUBCG_ZERO] = 1.0;
            ctl[MHD_SUBCG_ACTIVE] = 0.0;
            return;
        }
        if (s0 < ctl[MHD_SUBCG_THRESHOLD]) {
            ctl[MHD_SUBCG_ACTIVE] = 0.0;
            return;
        }
        // beta = r.z / r.z_old; p.Ap = z.Az + 2 beta z.q + beta^2 p.Ap (the previous p.Ap)
        const double abs_old = ctl[MHD_SUBCG_ABSNEW];
        ctl[MHD_SUBCG_ABSNEW] = s1;
        const double beta = s1 / abs_old;
        const double pap = s2 + 2.0 * beta * s3 + beta * beta * ctl[MHD_SUBCG_PQ];
        ctl[MHD_SUBCG_BETA] = beta;
        ctl[MHD_SUBCG_PQ] = pap;
        if (!(pap > 0.0)) {
            ctl[MHD_SUBCG_STATUS] = MHD_SUBCG_NONFINITE;
            ctl[MHD_SUBCG_ZERO] = 1.0;
            ctl[MHD_SUBCG_ACTIVE] = 0.0;
            return;
        }
        ctl[MHD_SUBCG_ALPHA_PREV] = ctl[MHD_SUBCG_ALPHA];
        ctl[MHD_SUBCG_ALPHA] = s1 / pap;
        if (ctl[MHD_SUBCG_PRODUCTS] >= max_products) {
            ctl[MHD_SUBCG_STATUS] = MHD_SUBCG_NOT_CONVERGED;
            ctl[MHD_SUBCG_ACTIVE] = 0.0;
        }
        return;
    }
    if (phase == 1) {
        ctl[MHD_SUBCG_PQ] = s0;
        ctl[MHD_SUBCG_ALPHA] = ctl[MHD_SUBCG_ABSNEW] / s0;
        return;
    }
    ctl[MHD_SUBCG_RR] = s0;
    ctl[MHD_SUBCG_PRODUCTS] += 1.0;
    if (!(isfinite(s0) && isfinite(ctl[MHD_SUBCG_ALPHA]))) {
        ctl[MHD_SUBCG_STATUS] = MHD_SUBCG_NONFINITE;
        ctl[MHD_SUBCG_ACTIVE] = 0.0;
    } else if (s0 < ctl[MHD_SUBCG_THRESHOLD]) {
        ctl[MHD_SUBCG_ACTIVE] = 0.0;
    } else if (ctl[MHD_SUBCG_PRODUCTS] >= max_products) {
        ctl[MHD_SUBCG_STATUS] = MHD_SUBCG_NOT_CONVERGED;
        ctl[MHD_SUBCG_ACTIVE] = 0.0;
    } else {
        ctl[MHD_SUBCG_BETA] = s1 / ctl[MHD_SUBCG_ABSNEW];
        ctl[MHD_SUBCG_ABSNEW] = s1;
    }
}

__global__ void k_subcg_decide(double* ctl, const double* slots, int count, int phase, double tol,
                               double max_products) {
    if (threadIdx.x == 0 && blockIdx.x == 0) subcg_decide(ctl, slots, count, phase, tol, max_products);
}

// Interior scan of the state: max CFL signal speed (diagnostics.hpp:60-78) and a non-finite flag;
// out[0] = max speed (atomicMax on the bits of a non-negative double: exact in any order),
// out[1] = 1 when a value is not finite. The faces one cell beyond the interior (the ring) give
// the cell-centred B of the last column / row.
__global__ void __launch_bounds__(kSubNT)
k_sub_cfl(Interior v, CPlanes u, unsigned long long* out) {
    __shared__ double red[32];
    double vmax = 0.0;
    bool bad = false;
    const size_t n = (size_t)v.nx * v.ny;
    for (size_t t = (size_t)blockIdx.x * kSubNT + threadIdx.x; t < n; t += (size_t)gridDim.x * kSubNT) {
        const int j = (int)(t / v.nx), i = (int)(t - (size_t)j * v.nx);
        const size_t g = at(v, i, j);
        const double bxc = (u.f[4][g] + u.f[4][g + 1]) / 2.0;
        const double byc = (u.f[5][g] + u.f[5][g + v.nxe]) / 2.0;
        double rho = u.f[0][g], vx, vy;
        const double p = primitives(rho, u.f[1][g], u.f[2][g], u.f[3][g], bxc, byc, vx, vy);
        vmax = smax(vmax, cfl_speed(rho, vx, vy, p, bxc, byc));
        bad |= !(isfinite(u.f[0][g]) && isfinite(u.f[1][g]) && isfinite(u.f[2][g]) &&
                 isfinite(u.f[3][g]) && isfinite(u.f[4][g]) && isfinite(u.f[5][g]));
    }
    vmax = block_max<kSubNT>(vmax, red);
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(&out[1], 1ULL);
    if (threadIdx.x == 0) atomicMax(&out[0], (unsigned long long)__double_as_longlong(vmax));
}

// Interior div B (diagnostics.hpp:15-42): block partials sum of div^2 (slot 0) and max |div|
// (slot 1).
__global__ void __launch_bounds__(kSubNT)
k_sub_divb(Interior v, double dx, double dy, const double* __restrict__ bxf,
           const double* __restrict__ byf, double* part) {
    __shared__ double red[kSubNT / 32];
    __shared__ double redm[32];
    double s2[1] = {0.0};
    double m = 0.0;
    const size_t n = (size_t)v.nx * v.ny;
    for (size_t t = (size_t)blockIdx.x * kSubNT + threadIdx.x; t < n; t += (size_t)gridDim.x * kSubNT) {
        const int j = (int)(t / v.nx), i = (int)(t - (size_t)j * v.nx);
        const size_t g = at(v, i, j);
        const double d = (bxf[g + 1] - bxf[g]) / dx + (byf[g + v.nxe] - byf[g]) / dy;
        s2[0] += d * d;
        m = smax(m, fabs(d));
    }
    block_sum<kSubNT, 1>(s2, red);
    m = block_max<kSubNT>(m, redm);
    if (threadIdx.x == 0) {
        part[(size_t)blockIdx.x * 2] = s2[0];
        part[(size_t)blockIdx.x * 2 + 1] = m;
    }
}

__global__ void k_sub_divb_final(const double* part, int nblocks, double* out) {
    if (threadIdx.x != 0) return;
    double s = 0.0, m = 0.0;
    for (int b = 0; b < nblocks; ++b) {
        s += part[(size_t)b * 2];
        m = smax(m, part[(size_t)b * 2 + 1]);
    }
    out[0] = s;
    out[1] = m;
}

}  // namespace

struct mhd_subdomain {
    mhd_params prm{};
    Domain ext{};       // the extended planes as a periodic grid (what the sweep kernels see)
    Interior iv{};
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int device = 0, num_sms = 0;
    size_t ne = 0;      // cells of an extended plane
    double* pool = nullptr;
    double* S[6]{};
    double* T[6]{};
    double* A[6]{};
    SubVecs V{};
    SubScal* sc = nullptr;  // device: the solves' matrix of this step
    double g = 0.0, d = 0.0;
    double dt = 0.0, alpha = 0.0;
    StepCoeffs* coeffs = nullptr;
    DeviceStatus* scratch_status = nullptr;  // finalize's CFL/NaN record over the extended planes (unused)
    double* part = nullptr;
    double* dev_out = nullptr;  // small results (device)
    double* host_out = nullptr; // pinned read-back
    SweepGeom sg[2]{}, fg{};
    int st_blocks[2]{}, fn_blocks = 0;
    int blocks = 0;     // grid of the per-cell interior kernels
    CgSweepArgs cga{};  // the single-sweep solve's sweep: the interior's strips and row segments
    int cg_blocks = 0;
    unsigned* arrivals = nullptr;  // blocks of the running sweep that have published their sums
    unsigned long long* cfl = nullptr;  // the device CFL step's scan: max speed bits, non-finite flag
    int pending_sums = 0;  // sums enqueued by a CG phase without an output pointer
    cudaEvent_t ev_ready = nullptr;  // in-process exchange: this subdomain's strips may be read
    cudaEvent_t ev_done = nullptr;   // in-process exchange: this subdomain's rings are filled
    cudaEvent_t ev_phase = nullptr;  // a decision group waits for this subdomain's work so far
    unsigned long long uid = 0;      // unique per creation (a freed subdomain's address may recur)
};

// Device-resident decisions of one decomposed solve (mhd_subcg_*): the control block, the
// subdomains' sum slots, and four pinned copies of the control block for the host to poll (the
// host may read a copy posted up to three posts earlier).
constexpr int kPostSlots = 4;
struct mhd_subcg {
    int count = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaEvent_t ev_decided = nullptr;  // the subdomains' streams wait for the group's last decision
    // one product of the solve captured as a CUDA graph (mhd_subcg_product), for these arguments
    cudaGraphExec_t product = nullptr;
    cudaGraphExec_t sweep[2]{};  // one iteration of the single-sweep form, even and odd k
    std::vector<unsigned long long> product_subs;  // uids of the subdomains the graphs were captured for
    int product_P = 0, product_Q = 0;
    double product_tol = 0.0;
    long long product_max = 0;
    double* ctl = nullptr;    // device, MHD_SUBCG_CTL doubles
    double* slots = nullptr;  // device, count x 4
    bool own_slots = false;
    double* host = nullptr;   // pinned, kPostSlots x MHD_SUBCG_CTL
    cudaEvent_t ev[4]{};      // one per posted copy (tags modulo kPostSlots)
};

namespace {

using mhd_host::cuda_status;

mhd_status check_sub(mhd_subdomain* s) {
    if (!s) return MHD_ERR_INVALID_ARGUMENT;
    MHD_TRY(cudaSetDevice(s->device));
    return MHD_OK;
}

// The planes of a set and their count.
int set_planes(mhd_subdomain* s, int set, Planes* out) {
    *out = Planes{};
    switch (set) {
        case MHD_SUB_SET_STATE:
            for (int k = 0; k < 6; ++k) out->f[k] = s->S[k];
            return 6;
        case MHD_SUB_SET_PREDICTOR:
            for (int k = 0; k < 6; ++k) out->f[k] = s->T[k];
            return 6;
        case MHD_SUB_SET_ACCUMULATOR_B:
            out->f[0] = s->A[4];
            out->f[1] = s->A[5];
            return 2;
        case MHD_SUB_SET_SOLUTION:
            out->f[0] = s->V.x;
            return 1;
        case MHD_SUB_SET_DIRECTION:
            out->f[0] = s->V.p;
            return 1;
        case MHD_SUB_SET_CG_EVEN:  // r_k = r[0], p_{k-1} = p[1] of the single-sweep form
            out->f[0] = s->V.r;
            out->f[1] = s->V.q;
            return 2;
        case MHD_SUB_SET_CG_ODD:  // r_k = r[1], p_{k-1} = p[0]
            out->f[0] = s->V.z;
            out->f[1] = s->V.p;
            return 2;
        default:
            return 0;
    }
}

// Rectangle of the extended plane that `side` sends (kPack) or receives, for a ring of `width`.
// West/east strips cover the interior rows only; south/north strips span the whole extended width,
// so that exchanging west/east first and south/north second also fills the corners.
bool strip_rect(const mhd_subdomain* s, int side, int width, bool send, int* x0, int* y0, int* w,
                int* h) {
    const int nx = s->iv.nx, ny = s->iv.ny, nxe = s->iv.nxe;
    if (width < 1 || width > kH) return false;
    switch (side) {
        case MHD_SUB_WEST:  // send: the first `width` interior columns; receive: the ring left of them
            *x0 = send ? kH : kH - width;
            *y0 = kH;
            *w = width;
            *h = ny;
            return true;
        case MHD_SUB_EAST:  // send: the last `width` interior columns; receive: the ring right of them
            *x0 = send ? kH + nx - width : kH + nx;
            *y0 = kH;
            *w = width;
            *h = ny;
            return true;
        case MHD_SUB_SOUTH:
            *x0 = 0;
            *y0 = send ? kH : kH - width;
            *w = nxe;
            *h = width;
            return true;
        case MHD_SUB_NORTH:
            *x0 = 0;
            *y0 = send ? kH + ny - width : kH + ny;
            *w = nxe;
            *h = width;
            return true;
        default:
            return false;
    }
}

mhd_status read_small(mhd_subdomain* s, int n, double* out) {
    MHD_TRY(cudaMemcpyAsync(s->host_out, s->dev_out, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost,
                            s->stream));
    MHD_TRY(cudaStreamSynchronize(s->stream));
    for (int k = 0; k < n; ++k) out[k] = s->host_out[k];
    return MHD_OK;
}

// The CG phases' sums: with an output pointer, wait and return them; without, only enqueue their
// copy to pinned host memory (mhd_sub_sums reads them), so that several subdomains' phases run at
// the same time.
mhd_status sums_out(mhd_subdomain* s, int n, double* out) {
    if (out) return read_small(s, n, out);
    MHD_TRY(cudaMemcpyAsync(s->host_out, s->dev_out, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost,
                            s->stream));
    s->pending_sums = n;
    return MHD_OK;
}

// The group's stream waits for every subdomain's work so far, and the subdomains' streams wait for
// the group's (a subdomain on the group's own stream needs neither).
mhd_status group_after_subs(mhd_subcg* g, mhd_subdomain* const* subs) {
    for (int i = 0; i < g->count; ++i) {
        if (subs[i]->stream == g->stream) continue;
        MHD_TRY(cudaEventRecord(subs[i]->ev_phase, subs[i]->stream));
        MHD_TRY(cudaStreamWaitEvent(g->stream, subs[i]->ev_phase, 0));
    }
    return MHD_OK;
}

mhd_status subs_after_group(mhd_subcg* g, mhd_subdomain* const* subs) {
    MHD_TRY(cudaEventRecord(g->ev_decided, g->stream));
    for (int i = 0; i < g->count; ++i)
        if (subs[i]->stream != g->stream) MHD_TRY(cudaStreamWaitEvent(subs[i]->stream, g->ev_decided, 0));
    return MHD_OK;
}

// Work on the subdomains' streams captured from the group's stream as a graph: the subdomains'
// streams join the capture through the group's event, and rejoin it at the end.
template <class Body>
mhd_status capture_graph(mhd_subcg* g, mhd_subdomain* const* subs, Body body, cudaGraphExec_t* out) {
    *out = nullptr;
    MHD_TRY(cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeRelaxed));
    mhd_status st = subs_after_group(g, subs);
    if (st == MHD_OK) st = body();
    if (st == MHD_OK) st = group_after_subs(g, subs);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(g->stream, &graph);
    if (st == MHD_OK && e != cudaSuccess) st = cuda_status(e);
    if (st == MHD_OK) {
        const cudaError_t ei = cudaGraphInstantiate(out, graph, 0);
        if (ei != cudaSuccess) st = cuda_status(ei);
    }
    if (graph) cudaGraphDestroy(graph);
    if (st != MHD_OK) {
        *out = nullptr;
        cudaGetLastError();
    }
    return st;
}

// One product of the two-sweep solve: p's ring, q = A p, decision, update, decision, direction.
mhd_status capture_product(mhd_subcg* g, mhd_subdomain* const* subs, int P, int Q, double tol,
                           long long max_products) {
    return capture_graph(g, subs, [&]() -> mhd_status {
        mhd_status st = mhd_sub_exchange_local(subs, P, Q, MHD_SUB_SET_DIRECTION, 1);
        for (int i = 0; i < g->count && st == MHD_OK; ++i)
            st = mhd_sub_cg_matvec_dev(subs[i], g->ctl, g->slots + 4 * i);
        if (st == MHD_OK) st = mhd_subcg_decide_on(g, subs, 1, tol, max_products);
        for (int i = 0; i < g->count && st == MHD_OK; ++i)
            st = mhd_sub_cg_update_dev(subs[i], g->ctl, g->slots + 4 * i);
        if (st == MHD_OK) st = mhd_subcg_decide_on(g, subs, 2, tol, max_products);
        for (int i = 0; i < g->count && st == MHD_OK; ++i) st = mhd_sub_cg_direction_dev(subs[i], g->ctl);
        return st;
    }, &g->product);
}

// Subdomain i's 3 x 3 neighbourhood among the P x Q subdomains subs[q * P + p].
CgSubNeighbours neighbourhood(mhd_subdomain* const* subs, int P, int Q, int i) {
    CgSubNeighbours nb{};
    const int p = i % P, q = i / P;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            const mhd_subdomain* n = subs[((q + a - 1 + Q) % Q) * P + (p + b - 1 + P) % P];
            const int e = a * 3 + b;
            nb.r[0][e] = n->V.r;
            nb.r[1][e] = n->V.z;
            nb.p[0][e] = n->V.p;
            nb.p[1][e] = n->V.q;
            nb.nxe[e] = n->iv.nxe;
        }
    nb.nx = subs[i]->iv.nx;
    nb.ny = subs[i]->iv.ny;
    nb.nx_w = subs[q * P + (p + P - 1) % P]->iv.nx;
    nb.ny_s = subs[((q + Q - 1) % Q) * P + p]->iv.ny;
    nb.halo = kH;
    return nb;
}

// One iteration of the single-sweep solve of parity `odd`: the sweeps, which read the cells around
// each interior from the neighbours' interiors (the previous decision has ordered every
// subdomain's last sweep before them, and r and p are double-buffered, so nothing they read is
// being written), then the decision.
mhd_status capture_sweep(mhd_subcg* g, mhd_subdomain* const* subs, int P, int Q, double tol,
                         long long max_products, int odd) {
    (void)odd;  // the sweep takes k, and with it the buffers, from the control block
    return capture_graph(g, subs, [&]() -> mhd_status {
        for (int i = 0; i < g->count; ++i) {
            mhd_subdomain* s = subs[i];
            k_sub_cg_sweep_iter<true><<<s->cg_blocks, kSubCgNT, kSubCgRingBytes, s->stream>>>(
                s->cga, s->sc, g->ctl, s->part, s->arrivals, g->slots + 4 * i, neighbourhood(subs, P, Q, i));
            MHD_TRY(cudaGetLastError());
        }
        return mhd_subcg_decide_on(g, subs, 4, tol, max_products);
    }, &g->sweep[odd]);
}

}  // namespace

extern "C" {

int mhd_sub_halo(void) { return kH; }

mhd_status mhd_sub_create(const mhd_params* p, void* stream, mhd_subdomain** out) {
    if (!p || !out) return MHD_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (p->nx < kH || p->ny < kH || !(p->dx > 0) || !(p->dy > 0) || !(p->eta >= 0) ||
        (p->ct_mode != 0 && p->ct_mode != 1) ||
        (long long)(p->nx + 2 * kH) * (p->ny + 2 * kH) > (1LL << 31))
        return MHD_ERR_INVALID_ARGUMENT;
    if (!mhd_device_available()) return MHD_ERR_NO_DEVICE;
    mhd_subdomain* s = new (std::nothrow) mhd_subdomain();
    if (!s) return MHD_ERR_OUT_OF_MEMORY;
    auto fail = [&](mhd_status st) {
        mhd_sub_destroy(s);
        return st;
    };
    static std::atomic<unsigned long long> next_uid{1};
    s->uid = next_uid.fetch_add(1);
    s->prm = *p;
    s->iv.nx = p->nx;
    s->iv.ny = p->ny;
    s->iv.nxe = p->nx + 2 * kH;
    s->ext = Domain{p->nx + 2 * kH, p->ny + 2 * kH, p->dx, p->dy, p->eta, p->ct_mode};
    s->ne = (size_t)s->ext.nx * s->ext.ny;
    s->g = (2.0 - sqrt(2.0)) / 2.0;     // solvers.hpp:41
    s->d = 1.0 - (1.0 / (2.0 * s->g));  // solvers.hpp:42
    if (cudaGetDevice(&s->device) != cudaSuccess) return fail(MHD_ERR_NO_DEVICE);
    if (cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, s->device) != cudaSuccess)
        return fail(MHD_ERR_NO_DEVICE);
    if (stream) {
        s->stream = (cudaStream_t)stream;
    } else {
        if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess)
            return fail(MHD_ERR_CUDA);
        s->own_stream = true;
    }
    // sweep geometry of the explicit kernels on the extended planes (as a single context's)
    for (int mode = 0; mode < 2; ++mode) {
        int occ = 0;
        const cudaError_t e = mode == 0
            ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_stage_sweep<1>, 32 * SW_WARPS, sweep_smem_bytes(1))
            : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_stage_sweep<2>, 32 * SW_WARPS, sweep_smem_bytes(2));
        if (e != cudaSuccess || occ < 1) return fail(MHD_ERR_CUDA);
        const long long resident = (long long)occ * s->num_sms * SW_WARPS;
        SweepGeom& g = s->sg[mode];
        g.strips_x = (s->ext.nx + SW_OUT - 1) / SW_OUT;
        const int segs = (int)std::max(1LL, resident / g.strips_x);
        g.seg_h = std::max(16, (s->ext.ny + segs - 1) / segs);
        g.segs_y = (s->ext.ny + g.seg_h - 1) / g.seg_h;
        g.nwarps = g.strips_x * g.segs_y;
        s->st_blocks[mode] = (g.nwarps + SW_WARPS - 1) / SW_WARPS;
    }
    {
        int occ = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_finalize_sweep, 32 * FS_WARPS, 0) !=
                cudaSuccess || occ < 1)
            return fail(MHD_ERR_CUDA);
        const long long resident = (long long)occ * s->num_sms * FS_WARPS;
        SweepGeom& g = s->fg;
        g.strips_x = (s->ext.nx + FS_OUT - 1) / FS_OUT;
        const int segs = (int)std::max(1LL, resident / g.strips_x);
        g.seg_h = std::max(16, (s->ext.ny + segs - 1) / segs);
        g.segs_y = (s->ext.ny + g.seg_h - 1) / g.seg_h;
        g.nwarps = g.strips_x * g.segs_y;
        s->fn_blocks = (g.nwarps + FS_WARPS - 1) / FS_WARPS;
    }
    const size_t interior = (size_t)p->nx * p->ny;
    s->blocks = (int)std::max<size_t>(1, std::min<size_t>((interior + kSubNT - 1) / kSubNT,
                                                          std::min(kSubMaxBlocks, s->num_sms * 4)));
    if (cudaMalloc(&s->pool, (size_t)kSubPlanes * s->ne * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&s->coeffs, sizeof(StepCoeffs)) != cudaSuccess ||
        cudaMalloc(&s->scratch_status, sizeof(DeviceStatus)) != cudaSuccess ||
        cudaMalloc(&s->sc, sizeof(SubScal)) != cudaSuccess ||
        cudaMalloc(&s->arrivals, sizeof(unsigned)) != cudaSuccess ||
        cudaMalloc(&s->cfl, 2 * sizeof(unsigned long long)) != cudaSuccess ||
        cudaMalloc(&s->part, (size_t)4 * kSubMaxBlocks * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&s->dev_out, 8 * sizeof(double)) != cudaSuccess ||
        cudaMallocHost(&s->host_out, 8 * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        return fail(MHD_ERR_OUT_OF_MEMORY);
    }
    double* q = s->pool;
    for (int k = 0; k < 6; ++k, q += s->ne) s->S[k] = q;
    for (int k = 0; k < 6; ++k, q += s->ne) s->T[k] = q;
    for (int k = 0; k < 6; ++k, q += s->ne) s->A[k] = q;
    s->V.x = q; q += s->ne;
    s->V.r = q; q += s->ne;
    s->V.p = q; q += s->ne;
    s->V.q = q; q += s->ne;
    s->V.z = q;
    {
        // the single-sweep solve: 28-column strips of the interior, row segments of seg_h rows,
        // about half a device's resident warps (the subdomains of one device share it)
        if (cudaFuncSetAttribute(k_sub_cg_sweep_rhs, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kSubCgRingBytes) != cudaSuccess ||
            cudaFuncSetAttribute(k_sub_cg_sweep_iter<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kSubCgRingBytes) != cudaSuccess ||
            cudaFuncSetAttribute(k_sub_cg_sweep_iter<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kSubCgRingBytes) != cudaSuccess)
            return fail(MHD_ERR_CUDA);
        int occ = 0, occ_nb = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_nb, k_sub_cg_sweep_iter<true>, kSubCgNT,
                                                          kSubCgRingBytes) != cudaSuccess)
            return fail(MHD_ERR_CUDA);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_sub_cg_sweep_iter<false>, kSubCgNT, kSubCgRingBytes) !=
                cudaSuccess || occ < 1 || occ_nb < 1)
            return fail(MHD_ERR_CUDA);
        occ = std::min(occ, occ_nb);
        CgSweepArgs& a = s->cga;
        a.D = s->ext;
        a.x = s->V.x;
        a.r[0] = s->V.r;
        a.r[1] = s->V.z;
        a.p[0] = s->V.p;
        a.p[1] = s->V.q;
        a.col0 = kH;
        a.col_end = kH + p->nx;
        a.strips_x = (p->nx + CG_W - 1) / CG_W;
        const int target = std::max(1, occ * s->num_sms * (kSubCgNT / 32) / 2);
        const int segs = std::max(1, target / a.strips_x);
        a.seg_h = std::max(32, (p->ny + segs - 1) / segs);
        a.nwarps = a.strips_x * ((p->ny + a.seg_h - 1) / a.seg_h);
        s->cg_blocks = std::min((a.nwarps + kSubCgNT / 32 - 1) / (kSubCgNT / 32),
                                std::min(kSubMaxBlocks, occ * s->num_sms));
    }
    if (cudaEventCreateWithFlags(&s->ev_ready, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->ev_done, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->ev_phase, cudaEventDisableTiming) != cudaSuccess)
        return fail(MHD_ERR_CUDA);
    if (cudaMemsetAsync(s->pool, 0, (size_t)kSubPlanes * s->ne * sizeof(double), s->stream) != cudaSuccess ||
        cudaMemsetAsync(s->coeffs, 0, sizeof(StepCoeffs), s->stream) != cudaSuccess ||
        cudaMemsetAsync(s->scratch_status, 0, sizeof(DeviceStatus), s->stream) != cudaSuccess ||
        cudaMemsetAsync(s->sc, 0, sizeof(SubScal), s->stream) != cudaSuccess ||
        cudaMemsetAsync(s->arrivals, 0, sizeof(unsigned), s->stream) != cudaSuccess ||
        cudaStreamSynchronize(s->stream) != cudaSuccess)
        return fail(MHD_ERR_CUDA);
    *out = s;
    return MHD_OK;
}

mhd_status mhd_sub_destroy(mhd_subdomain* s) {
    if (!s) return MHD_ERR_INVALID_ARGUMENT;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    cudaFree(s->pool);
    cudaFree(s->coeffs);
    cudaFree(s->scratch_status);
    cudaFree(s->sc);
    cudaFree(s->arrivals);
    cudaFree(s->cfl);
    cudaFree(s->part);
    cudaFree(s->dev_out);
    if (s->host_out) cudaFreeHost(s->host_out);
    if (s->ev_ready) cudaEventDestroy(s->ev_ready);
    if (s->ev_done) cudaEventDestroy(s->ev_done);
    if (s->ev_phase) cudaEventDestroy(s->ev_phase);
    if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
    cudaGetLastError();
    delete s;
    return MHD_OK;
}

void* mhd_sub_stream(mhd_subdomain* s) { return s ? (void*)s->stream : nullptr; }

mhd_status mhd_sub_set_state(mhd_subdomain* s, const double* const fields[6]) {
    mhd_status st = check_sub(s);
    if (st != MHD_OK) return st;
    if (!fields) return MHD_ERR_INVALID_ARGUMENT;
    const int nx = s->iv.nx, ny = s->iv.ny, nxe = s->iv.nxe;
    for (int k = 0; k < 6; ++k) {
        if (!fields[k]) return MHD_ERR_INVALID_ARGUMENT;
        MHD_TRY(cudaMemcpy2DAsync(s->S[k] + (size_t)kH * nxe + kH, (size_t)nxe * sizeof(double), fields[k],
                                  (size_t)nx * sizeof(double), (size_t)nx * sizeof(double), ny,
                                  cudaMemcpyDefault, s->stream));
    }
    MHD_TRY(cudaStreamSynchronize(s->stream));
    return MHD_OK;
}

mhd_status mhd_sub_get_state(mhd_subdomain* s, double* const fields[6]) {
    mhd_status st = check_sub(s);
    if (st != MHD_OK) return st;
    if (!fields) return MHD_ERR_INVALID_ARGUMENT;
    const int nx = s->iv.nx, ny = s->iv.ny, nxe = s->iv.nxe;
    for (int k = 0; k < 6; ++k) {
        if (!fields[k]) return MHD_ERR_INVALID_ARGUMENT;
        MHD_TRY(cudaMemcpy2DAsync(fields[k], (size_t)nx * sizeof(double), s->S[k] + (size_t)kH * nxe + kH,
                                  (size_t)nxe * sizeof(double), (size_t)nx * sizeof(double), ny,
                                  cudaMemcpyDefault, s->stream));
    }
    MHD_TRY(cudaStreamSynchronize(s->stream));
    return MHD_OK;
}

size_t mhd_sub_strip_doubles(mhd_subdomain* s, int set, int side, int width) {
    if (!s) return 0;
    Planes pl;
    const int np = set_planes(s, set, &pl);
    int x0, y0, w, h;
    if (np == 0 || !strip_rect(s, side, width, true, &x0, &y0, &w, &h)) return 0;
    return (size_t)np * w * h;
}

mhd_status mhd_sub_pack(mhd_subdomain* s, int set, int side, int width, double* buf) {
    mhd_status st = check_sub(s);
    if (st != MHD_OK) return st;
    Planes pl;
    const int np = set_planes(s, set, &pl);
    int x0, y0, w, h;
    if (!buf || np == 0 || !strip_rect(s, side, width, true, &x0, &y0, &w, &h)) return MHD_ERR_INVALID_ARGUMENT;
    const size_t total = (size_t)np * w * h;
    const int blocks = (int)std::max<size_t>(1, std::min<size_t>((total + kSubNT - 1) / kSubNT, 4 * s->num_sms));
    k_sub_strip<true><<<blocks, kSubNT, 0, s->stream>>>(pl, np, s->iv.nxe, x0, y0, w, h, buf);
    MHD_TRY(cudaGetLastError());
    return MHD_OK;
}

mhd_status mhd_sub_unpack(mhd_subdomain* s, int set, int side, int width, const double* buf) {
    mhd_status st = check_sub(s);
    if (st != MHD_OK) return st;
    Planes pl;
    const int np = set_planes(s, set, &pl);
    int x0, y0, w, h;
    if (!buf || np == 0 || !strip_rect(s, side, width, false, &x0, &y0, &w, &h)) return MHD_ERR_INVALID_ARGUMENT;
    const size_t total = (size_t)np * w * h;
    const int blocks = (int)std::max<size_t>(1, std::min<size_t>((total + kSubNT - 1) / kSubNT, 4 * s->num_sms));
    k_sub_strip<false><<<blocks, kSubNT, 0, s->stream>>>(pl, np, s->iv.nxe, x0, y0, w, h,
                                                         const_cast<double*>(buf));
    MHD_TRY(cudaGetLastError());
    return MHD_OK;
}

mhd_status mhd_sub_exchange_local(mhd_subdomain* const* subs, int P, int Q, int set, int width) {
    MHD_NVTX_RANGE("mhd_sub_exchange_local");
    if (!subs || P < 1 || Q < 1) return MHD_ERR_INVALID_ARGUMENT;
    const int count = P * Q;
    for (int i = 0; i < count; ++i) {
        if (!subs[i] || subs[i]->device != subs[0]->device) return MHD_ERR_INVALID_ARGUMENT;
        Planes pl;
        int x0, y0, w, h;
        if (set_planes(subs[i], set, &pl) == 0 || !strip_rect(subs[i], MHD_SUB_WEST, width, true, &x0, &y0, &w, &h))
            return MHD_ERR_INVALID_ARGUMENT;
    }
    // neighbours must agree on the strips they exchange: equal rows along x, equal widths along y
    for (int i = 0; i < count; ++i) {
        const int p = i % P, q = i / P;
        const mhd_subdomain* e = subs[q * P + (p + 1) % P];
        const mhd_subdomain* n = subs[((q + 1) % Q) * P + p];
        if (e->iv.ny != subs[i]->iv.ny || n->iv.nx != subs[i]->iv.nx) return MHD_ERR_INVALID_ARGUMENT;
    }
    MHD_TRY(cudaSetDevice(subs[0]->device));
    // subdomains on one stream are ordered by it: no events
    bool one_stream = true;
    for (int i = 1; i < count; ++i) one_stream = one_stream && subs[i]->stream == subs[0]->stream;
    // every subdomain's work so far is done before a neighbour reads its interior
    if (!one_stream)
        for (int i = 0; i < count; ++i) MHD_TRY(cudaEventRecord(subs[i]->ev_ready, subs[i]->stream));
    for (int i = 0; i < count; ++i) {
        mhd_subdomain* me = subs[i];
        const int p = i % P, q = i / P;
        RingSources src{};
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) {
                mhd_subdomain* from = subs[((q + a - 1 + Q) % Q) * P + (p + b - 1 + P) % P];
                if (!one_stream && from != me) {
                    bool seen = false;  // wait once per distinct neighbour
                    for (int a2 = 0; a2 <= a && !seen; ++a2)
                        for (int b2 = 0; b2 < 3 && !seen; ++b2)
                            if ((a2 < a || b2 < b) && subs[((q + a2 - 1 + Q) % Q) * P + (p + b2 - 1 + P) % P] == from)
                                seen = true;
                    if (!seen) MHD_TRY(cudaStreamWaitEvent(me->stream, from->ev_ready, 0));
                }
                Planes sp;
                set_planes(from, set, &sp);
                for (int k = 0; k < 6; ++k) src.f[a][b][k] = sp.f[k];
                src.nxe[a][b] = from->iv.nxe;
            }
        src.nx_w = subs[q * P + (p + P - 1) % P]->iv.nx;
        src.ny_s = subs[((q + Q - 1) % Q) * P + p]->iv.ny;
        Planes dst;
        const int np = set_planes(me, set, &dst);
        const size_t cells = (size_t)2 * width * (me->iv.nx + 2 * width) + (size_t)2 * width * me->iv.ny;
        const int blocks = (int)std::max<size_t>(1, std::min<size_t>((cells + kSubNT - 1) / kSubNT, 4 * me->num_sms));
        k_sub_ring_gather<<<blocks, kSubNT, 0, me->stream>>>(dst, np, me->iv, width, src);
        MHD_TRY(cudaGetLastError());
    }
    // a subdomain changes its interior again only after its neighbours have read from it
    if (!one_stream) {
        for (int i = 0; i < count; ++i) MHD_TRY(cudaEventRecord(subs[i]->ev_done, subs[i]->stream));
        for (int i = 0; i < count; ++i) {
            const int p = i % P, q = i / P;
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) {
                    mhd_subdomain* nb = subs[((q + a - 1 + Q) % Q) * P + (p + b - 1 + P) % P];
                    if (nb != subs[i]) MHD_TRY(cudaStreamWaitEvent(subs[i]->stream, nb->ev_done, 0));
                }
        }
    }
    return MHD_OK;
}

mhd_status mhd_sub_cfl_speed(mhd_subdomain* s, double* smax_out, int* nonfinite) {
    mhd_status st = check_sub(s);
    if (st != MHD_OK) return st;
    if (!smax_out) return MHD_ERR_INVALID_ARGUMENT;
    MHD_TRY(cudaMemsetAsync(s->dev_out, 0, 2 * sizeof(double), s->stream));
    CPlanes u;
    for (int k = 0; k < 6; ++k) u.f[k] = s->S[k];
    k_sub_cfl<<<s->blocks, kSubNT, 0, s->stream>>>(s->iv, u, reinterpret_cast<unsigned long long*>(s->dev_out));
    MHD_TRY(cudaGetLastError());
    MHD_TRY(cudaMemcpyAsync(s->host_out, s->dev_out, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    MHD_TRY(cudaStreamSynchronize(s->stream));
    unsigned long long bits[2];
    memcpy(bits, s->host_out, sizeof(bits));
    double v;
    memcpy(&v, &bits[0], sizeof(v));  // a non-negative double kept as its bits
    *smax_out = v;
    if (nonfinite) *nonfinite = bits[1] != 0;
    return MHD_OK;
}

mhd_status mhd_sub_set_step(mhd_subdomain* s, double dt, double alpha) {
    mhd_status st = check_sub(s);
    if (st != MHD_OK) return st;
    if (!(dt > 0) || !std::isfinite(dt) || !(alpha >= 0) || !std::isfinite(alpha)) return MHD_ERR_INVALID_ARGUMENT;
    s->dt = dt;
    s->alpha = alpha;
    k_sub_set_coeffs<<<1, 1, 0, s->stream>>>(s->coeffs, s->sc, dt, alpha, s->g, s->d, s->prm.dx, s->prm.dy);
    MHD_TRY(cudaGetLastError());
    return MHD_OK;
}

mhd_status mhd_sub_stage(mhd_subdomain* s, int stage) {
    MHD_NVTX_RANGE("mhd_sub_stage");
    mhd_status st = check_sub(s);
    if (st != MHD_OK) return st;
    CPlanes in;
    Planes T, A;
    for (int k = 0; k < 6; ++k) {
        T.f[k] = s->T[k];
        A.f[k] = s->A[k];
    }
    if (stage == 1) {
        for (int k = 0; k < 6; ++k) in.f[k] = s->S[k];
        k_stage_sweep<1><<<s->st_blocks[0], 32 * SW_WARPS, sweep_smem_bytes(1), s->stream>>>(
            s->ext, s->coeffs, in, nullptr, T, A, s->sg[0]);
    } else if (stage == 2) {
        for (int k = 0; k < 6; ++k) in.f[k] = s->T[k];
        k_stage_sweep<2><<<s->st_blocks[1], 32 * SW_WARPS, sweep_smem_bytes(2), s->stream>>>(
            s->ext, s->coeffs, in, s->V.x, T, A, s->sg[1]);
    } else {
        return MHD_ERR_INVALID_ARGUMENT;
    }
    MHD_TRY(cudaGetLastError());
    return MHD_OK;
}

mhd_status mhd_sub_finalize(mhd_subdomain* s) {
    mhd_status st = check_sub(s);
    if (st != MHD_OK) return st;
    Planes A;
    for (int k = 0; k < 6; ++k) A.f[k] = s->A[k];
    k_finalize_sweep<<<s->fn_blocks, 32 * FS_WARPS, 0, s->stream>>>(s->ext, s->coeffs, A, s->V.x, s->S[4],
                                                                    s->S[5], s->scratch_status, s->fg);
    MHD_TRY(cudaGetLastError());
    // the accumulator's hydro planes hold U^{n+1}: they become the state's (pointer swap)
    for (int k = 0; k < 4; ++k) std::swap(s->S[k], s->A[k]);
    return MHD_OK;
}

mhd_status mhd_sub_cg_rhs(mhd_subdomain* s, int solve_index, double out[2]) {
    mhd_status st = check_sub(s);
    if (st != MHD_OK) return st;
    if (solve_index != 0 && solve_index != 1) return MHD_ERR_INVALID_ARGUMENT;
    const double* bx = solve_index == 0 ? s->T[4] : s->A[4];
    const double* by = solve_index == 0 ? s->T[5] : s->A[5];
    k_sub_cg_rhs<<<s->blocks, kSubNT, 0, s->stream>>>(s->iv, s->prm.eta, 1.0 / s->prm.dx, 1.0 / s->prm.dy,
                                                      bx, by, s->V, s->sc, s->part);
    MHD_TRY(cudaGetLastError());
    k_sub_final<2><<<1, 32, 0, s->stream>>>(s->part, s->blocks, s->dev_out);
    MHD_TRY(cudaGetLastError());
    return sums_out(s, 2, out);
}

mhd_status mhd_sub_cg_matvec(mhd_subdomain* s, double* pq) {
    mhd_status st = check_sub(s);
    if (st != MHD_OK) return st;
    k_sub_cg_matvec<<<s->blocks, kSubNT, 0, s->stream>>>(s->iv, s->V, s->sc, nullptr, s->part);
    MHD_TRY(cudaGetLastError());
    k_sub_final<1><<<1, 32, 0, s->stream>>>(s->part, s->blocks, s->dev_out);
    MHD_TRY(cudaGetLastError());
    return sums_out(s, 1, pq);
}

mhd_status mhd_sub_cg_update(mhd_subdomain* s, double alpha, double out[2]) {
    mhd_status st = check_sub(s);
    if (st != MHD_OK) return st;
    k_sub_cg_update<<<s->blocks, kSubNT, 0, s->stream>>>(s->iv, s->V, s->sc, alpha, nullptr, s->part);
    MHD_TRY(cudaGetLastError());
    k_sub_final<2><<<1, 32, 0, s->stream>>>(s->part, s->blocks, s->dev_out);
    MHD_TRY(cudaGetLastError());
    return sums_out(s, 2, out);
}

mhd_status mhd_sub_sums(mhd_subdomain* s, double* out, int n) {
    mhd_status st = check_sub(s);
    if (st != MHD_OK) return st;
    if (!out || n < 1 || n != s->pending_sums) return MHD_ERR_INVALID_ARGUMENT;
    MHD_TRY(cudaStreamSynchronize(s->stream));
    for (int k = 0; k < n; ++k) out[k] = s->host_out[k];
    s->pending_sums = 0;
    return MHD_OK;
}

mhd_status mhd_sub_cg_direction(mhd_subdomain* s, double beta) {
    mhd_status st = check_sub(s);
    if (st != MHD_OK) return st;
    k_sub_cg_dir<<<s->blocks, kSubNT, 0, s->stream>>>(s->iv, s->V, beta, nullptr);
    MHD_TRY(cudaGetLastError());
    return MHD_OK;
}

mhd_status mhd_sub_cg_zero_solution(mhd_subdomain* s) {
    mhd_status st = check_sub(s);
    if (st != MHD_OK) return st;
    k_sub_zero_interior<<<s->blocks, kSubNT, 0, s->stream>>>(s->iv, s->V.x, nullptr);
    MHD_TRY(cudaGetLastError());
    return MHD_OK;
}

mhd_status mhd_sub_cg_rhs_dev(mhd_subdomain* s, int solve_index, double* slot) {
    mhd_status st = check_sub(s);
    if (st != MHD_OK) return st;
    if ((solve_index != 0 && solve_index != 1) || !slot) return MHD_ERR_INVALID_ARGUMENT;
    const double* bx = solve_index == 0 ? s->T[4] : s->A[4];
    const double* by = solve_index == 0 ? s->T[5] : s->A[5];
    k_sub_cg_rhs<<<s->blocks, kSubNT, 0, s->stream>>>(s->iv, s->prm.eta, 1.0 / s->prm.dx, 1.0 / s->prm.dy,
                                                      bx, by, s->V, s->sc, s->part);
    MHD_TRY(cudaGetLastError());
    k_sub_final<2><<<1, 32, 0, s->stream>>>(s->part, s->blocks, slot);
    MHD_TRY(cudaGetLastError());
    return MHD_OK;
}

mhd_status mhd_sub_cg_matvec_dev(mhd_subdomain* s, const double* ctl, double* slot) {
    mhd_status st = check_sub(s);
    if (st != MHD_OK) return st;
    if (!ctl || !slot) return MHD_ERR_INVALID_ARGUMENT;
    k_sub_cg_matvec<<<s->blocks, kSubNT, 0, s->stream>>>(s->iv, s->V, s->sc, ctl, s->part);
    MHD_TRY(cudaGetLastError());
    k_sub_final<1><<<1, 32, 0, s->stream>>>(s->part, s->blocks, slot);
    MHD_TRY(cudaGetLastError());
    return MHD_OK;
}

mhd_status mhd_sub_cg_update_dev(mhd_subdomain* s, const double* ctl, double* slot) {
    mhd_status st = check_sub(s);
    if (st != MHD_OK) return st;
    if (!ctl || !slot) return MHD_ERR_INVALID_ARGUMENT;
    k_sub_cg_update<<<s->blocks, kSubNT, 0, s->stream>>>(s->iv, s->V, s->sc, 0.0, ctl, s->part);
    MHD_TRY(cudaGetLastError());
    k_sub_final<2><<<1, 32, 0, s->stream>>>(s->part, s->blocks, slot);
    MHD_TRY(cudaGetLastError());
    return MHD_OK;
}

mhd_status mhd_sub_cg_direction_dev(mhd_subdomain* s, const double* ctl) {
    mhd_status st = check_sub(s);
    if (st != MHD_OK) return st;
    if (!ctl) return MHD_ERR_INVALID_ARGUMENT;
    k_sub_cg_dir<<<s->blocks, kSubNT, 0, s->stream>>>(s->iv, s->V, 0.0, ctl);
    MHD_TRY(cudaGetLastError());
    return MHD_OK;
}

mhd_status mhd_sub_cg_finish_dev(mhd_subdomain* s, const double* ctl) {
    mhd_status st = check_sub(s);
    if (st != MHD_OK) return st;
    if (!ctl) return MHD_ERR_INVALID_ARGUMENT;
    k_sub_zero_interior<<<s->blocks, kSubNT, 0, s->stream>>>(s->iv, s->V.x, ctl);
    MHD_TRY(cudaGetLastError());
    return MHD_OK;
}

mhd_status mhd_sub_cg_sweep_rhs_dev(mhd_subdomain* s, int solve_index, double* slot) {
    mhd_status st = check_sub(s);
    if (st != MHD_OK) return st;
    if ((solve_index != 0 && solve_index != 1) || !slot) return MHD_ERR_INVALID_ARGUMENT;
    CgSweepArgs a = s->cga;
    a.bxf = solve_index == 0 ? s->T[4] : s->A[4];
    a.byf = solve_index == 0 ? s->T[5] : s->A[5];
    k_sub_cg_sweep_rhs<<<s->cg_blocks, kSubCgNT, kSubCgRingBytes, s->stream>>>(a, s->sc, s->part, s->arrivals,
                                                                                slot);
    MHD_TRY(cudaGetLastError());
    return MHD_OK;
}

mhd_status mhd_sub_cg_sweep_iter_dev(mhd_subdomain* s, const double* ctl, double* slot) {
    mhd_status st = check_sub(s);
    if (st != MHD_OK) return st;
    if (!ctl || !slot) return MHD_ERR_INVALID_ARGUMENT;
    k_sub_cg_sweep_iter<false><<<s->cg_blocks, kSubCgNT, kSubCgRingBytes, s->stream>>>(
        s->cga, s->sc, ctl, s->part, s->arrivals, slot, CgSubNeighbours{});
    MHD_TRY(cudaGetLastError());
    return MHD_OK;
}

mhd_status mhd_sub_cg_sweep_finish_dev(mhd_subdomain* s, const double* ctl) {
    mhd_status st = check_sub(s);
    if (st != MHD_OK) return st;
    if (!ctl) return MHD_ERR_INVALID_ARGUMENT;
    k_sub_cg_sweep_finish<<<s->blocks, kSubNT, 0, s->stream>>>(s->iv, s->V.x, s->V.p, ctl);
    MHD_TRY(cudaGetLastError());
    return MHD_OK;
}

mhd_status mhd_subcg_create(int count, void* stream, double* slots, mhd_subcg** out) {
    if (!out || count < 1 || count > 1 << 20) return MHD_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (!mhd_device_available()) return MHD_ERR_NO_DEVICE;
    mhd_subcg* g = new (std::nothrow) mhd_subcg();
    if (!g) return MHD_ERR_OUT_OF_MEMORY;
    g->count = count;
    if (cudaGetDevice(&g->device) != cudaSuccess) {
        delete g;
        return MHD_ERR_NO_DEVICE;
    }
    if (stream) {
        g->stream = (cudaStream_t)stream;
    } else if (cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking) == cudaSuccess) {
        g->own_stream = true;
    } else {
        cudaGetLastError();
        delete g;
        return MHD_ERR_CUDA;
    }
    g->slots = slots;
    g->own_slots = slots == nullptr;
    if (cudaMalloc(&g->ctl, MHD_SUBCG_CTL * sizeof(double)) != cudaSuccess ||
        (g->own_slots && cudaMalloc(&g->slots, (size_t)4 * count * sizeof(double)) != cudaSuccess) ||
        cudaMallocHost(&g->host, kPostSlots * MHD_SUBCG_CTL * sizeof(double)) != cudaSuccess ||
        cudaEventCreateWithFlags(&g->ev[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&g->ev[1], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&g->ev[2], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&g->ev[3], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&g->ev_decided, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        mhd_subcg_destroy(g);
        return MHD_ERR_OUT_OF_MEMORY;
    }
    if (cudaMemsetAsync(g->ctl, 0, MHD_SUBCG_CTL * sizeof(double), g->stream) != cudaSuccess ||
        cudaMemsetAsync(g->slots, 0, (size_t)4 * count * sizeof(double), g->stream) != cudaSuccess ||
        cudaStreamSynchronize(g->stream) != cudaSuccess) {
        cudaGetLastError();
        mhd_subcg_destroy(g);
        return MHD_ERR_CUDA;
    }
    *out = g;
    return MHD_OK;
}

mhd_status mhd_subcg_destroy(mhd_subcg* g) {
    if (!g) return MHD_ERR_INVALID_ARGUMENT;
    cudaSetDevice(g->device);
    if (g->stream) cudaStreamSynchronize(g->stream);
    if (g->product) cudaGraphExecDestroy(g->product);
    for (cudaGraphExec_t e : g->sweep)
        if (e) cudaGraphExecDestroy(e);
    for (cudaEvent_t e : g->ev)
        if (e) cudaEventDestroy(e);
    if (g->ev_decided) cudaEventDestroy(g->ev_decided);
    if (g->host) cudaFreeHost(g->host);
    if (g->own_slots) cudaFree(g->slots);
    cudaFree(g->ctl);
    if (g->own_stream) cudaStreamDestroy(g->stream);
    delete g;
    return MHD_OK;
}

double* mhd_subcg_slots(mhd_subcg* g) { return g ? g->slots : nullptr; }
const double* mhd_subcg_control(mhd_subcg* g) { return g ? g->ctl : nullptr; }

mhd_status mhd_subcg_decide(mhd_subcg* g, int phase, double tol, long long max_products) {
    if (!g || phase < 0 || phase > 4 || !(tol >= 0) || max_products < 1) return MHD_ERR_INVALID_ARGUMENT;
    MHD_TRY(cudaSetDevice(g->device));
    k_subcg_decide<<<1, 32, 0, g->stream>>>(g->ctl, g->slots, g->count, phase, tol, (double)max_products);
    MHD_TRY(cudaGetLastError());
    return MHD_OK;
}

mhd_status mhd_subcg_post(mhd_subcg* g, int tag) {
    if (!g || tag < 0) return MHD_ERR_INVALID_ARGUMENT;
    MHD_TRY(cudaSetDevice(g->device));
    const int b = tag % kPostSlots;
    MHD_TRY(cudaMemcpyAsync(g->host + b * MHD_SUBCG_CTL, g->ctl, MHD_SUBCG_CTL * sizeof(double),
                            cudaMemcpyDeviceToHost, g->stream));
    MHD_TRY(cudaEventRecord(g->ev[b], g->stream));
    return MHD_OK;
}

mhd_status mhd_subcg_read(mhd_subcg* g, int tag, double* out) {
    if (!g || tag < 0 || !out) return MHD_ERR_INVALID_ARGUMENT;
    MHD_TRY(cudaSetDevice(g->device));
    const int b = tag % kPostSlots;
    MHD_TRY(cudaEventSynchronize(g->ev[b]));
    memcpy(out, g->host + b * MHD_SUBCG_CTL, MHD_SUBCG_CTL * sizeof(double));
    return MHD_OK;
}

mhd_status mhd_subcg_decide_on(mhd_subcg* g, mhd_subdomain* const* subs, int phase, double tol,
                               long long max_products) {
    if (!g || !subs || phase < 0 || phase > 4 || !(tol >= 0) || max_products < 1) return MHD_ERR_INVALID_ARGUMENT;
    for (int i = 0; i < g->count; ++i)
        if (!subs[i] || subs[i]->device != g->device) return MHD_ERR_INVALID_ARGUMENT;
    MHD_TRY(cudaSetDevice(g->device));
    mhd_status st = group_after_subs(g, subs);
    if (st != MHD_OK) return st;
    k_subcg_decide<<<1, 32, 0, g->stream>>>(g->ctl, g->slots, g->count, phase, tol, (double)max_products);
    MHD_TRY(cudaGetLastError());
    return subs_after_group(g, subs);
}

namespace {
// Drop the captured graphs when the arguments they were captured for change.
mhd_status check_graph_args(mhd_subcg* g, mhd_subdomain* const* subs, int P, int Q, double tol,
                            long long max_products) {
    if (!g || !subs || P < 1 || Q < 1 || P * Q != g->count || !(tol >= 0) || max_products < 1)
        return MHD_ERR_INVALID_ARGUMENT;
    // a captured graph joins the subdomains' streams, which the legacy default stream cannot
    for (int i = 0; i < g->count; ++i)
        if (!subs[i] || subs[i]->device != g->device || !subs[i]->stream) return MHD_ERR_INVALID_ARGUMENT;
    MHD_TRY(cudaSetDevice(g->device));
    bool same = !g->product_subs.empty() && g->product_P == P && g->product_Q == Q &&
                g->product_tol == tol && g->product_max == max_products;
    for (int i = 0; i < g->count && same; ++i) same = g->product_subs[i] == subs[i]->uid;
    if (!same) {
        if (g->product) cudaGraphExecDestroy(g->product);
        g->product = nullptr;
        for (cudaGraphExec_t& e : g->sweep) {
            if (e) cudaGraphExecDestroy(e);
            e = nullptr;
        }
        g->product_subs.resize(g->count);
        for (int i = 0; i < g->count; ++i) g->product_subs[i] = subs[i]->uid;
        g->product_P = P;
        g->product_Q = Q;
        g->product_tol = tol;
        g->product_max = max_products;
    }
    return MHD_OK;
}

// Replay a captured graph after the subdomains' work so far, post the control block under `tag`,
// and order the subdomains' later work after both.
mhd_status replay(mhd_subcg* g, mhd_subdomain* const* subs, cudaGraphExec_t exec, int tag) {
    mhd_status st = group_after_subs(g, subs);
    if (st != MHD_OK) return st;
    MHD_TRY(cudaGraphLaunch(exec, g->stream));
    if ((st = mhd_subcg_post(g, tag)) != MHD_OK) return st;
    return subs_after_group(g, subs);
}
}  // namespace

mhd_status mhd_subcg_cfl_step(mhd_subcg* g, mhd_subdomain* const* subs, double courant, double safety) {
    if (!g || !subs || g->count > kSubCflMax || !(courant > 0) || !(safety > 0)) return MHD_ERR_INVALID_ARGUMENT;
    for (int i = 0; i < g->count; ++i) {
        if (!subs[i] || subs[i]->device != g->device) return MHD_ERR_INVALID_ARGUMENT;
        const mhd_params& a = subs[i]->prm;
        const mhd_params& b = subs[0]->prm;
        if (a.dx != b.dx || a.dy != b.dy || a.eta != b.eta) return MHD_ERR_INVALID_ARGUMENT;
    }
    MHD_TRY(cudaSetDevice(g->device));
    SubCflTargets t{};
    for (int i = 0; i < g->count; ++i) {
        mhd_subdomain* s = subs[i];
        MHD_TRY(cudaMemsetAsync(s->cfl, 0, 2 * sizeof(unsigned long long), s->stream));
        CPlanes u;
        for (int k = 0; k < 6; ++k) u.f[k] = s->S[k];
        k_sub_cfl<<<s->blocks, kSubNT, 0, s->stream>>>(s->iv, u, s->cfl);
        MHD_TRY(cudaGetLastError());
        t.speed[i] = s->cfl;
        t.coeffs[i] = s->coeffs;
        t.sc[i] = s->sc;
    }
    mhd_status st = group_after_subs(g, subs);
    if (st != MHD_OK) return st;
    const mhd_subdomain* s0 = subs[0];
    k_subcg_cfl_step<<<1, 32, 0, g->stream>>>(t, g->count, s0->prm.dx, s0->prm.dy, s0->prm.eta, courant, safety,
                                              s0->g, s0->d, g->ctl);
    MHD_TRY(cudaGetLastError());
    return subs_after_group(g, subs);
}

mhd_status mhd_subcg_product(mhd_subcg* g, mhd_subdomain* const* subs, int P, int Q, double tol,
                             long long max_products, int tag) {
    MHD_NVTX_RANGE("mhd_subcg_product");
    if (tag < 0) return MHD_ERR_INVALID_ARGUMENT;
    mhd_status st = check_graph_args(g, subs, P, Q, tol, max_products);
    if (st != MHD_OK) return st;
    if (!g->product && (st = capture_product(g, subs, P, Q, tol, max_products)) != MHD_OK) return st;
    return replay(g, subs, g->product, tag);
}

mhd_status mhd_subcg_sweep_product(mhd_subcg* g, mhd_subdomain* const* subs, int P, int Q, double tol,
                                   long long max_products, int k, int tag) {
    MHD_NVTX_RANGE("mhd_subcg_sweep_product");
    if (tag < 0 || k < 0) return MHD_ERR_INVALID_ARGUMENT;
    mhd_status st = check_graph_args(g, subs, P, Q, tol, max_products);
    if (st != MHD_OK) return st;
    const int odd = k & 1;
    if (!g->sweep[odd] && (st = capture_sweep(g, subs, P, Q, tol, max_products, odd)) != MHD_OK) return st;
    return replay(g, subs, g->sweep[odd], tag);
}

mhd_status mhd_subcg_decide_host(double* ctl, const double* slots, int count, int phase, double tol,
                                 long long max_products) {
    if (!ctl || !slots || count < 1 || phase < 0 || phase > 4 || !(tol >= 0) || max_products < 1)
        return MHD_ERR_INVALID_ARGUMENT;
    subcg_decide(ctl, slots, count, phase, tol, (double)max_products);
    return MHD_OK;
}

mhd_status mhd_sub_divb_sums(mhd_subdomain* s, double out[2]) {
    mhd_status st = check_sub(s);
    if (st != MHD_OK) return st;
    if (!out) return MHD_ERR_INVALID_ARGUMENT;
    k_sub_divb<<<s->blocks, kSubNT, 0, s->stream>>>(s->iv, s->prm.dx, s->prm.dy, s->S[4], s->S[5], s->part);
    MHD_TRY(cudaGetLastError());
    k_sub_divb_final<<<1, 32, 0, s->stream>>>(s->part, s->blocks, s->dev_out);
    MHD_TRY(cudaGetLastError());
    return read_small(s, 2, out);
}

mhd_status mhd_sub_synchronize(mhd_subdomain* s) {
    mhd_status st = check_sub(s);
    if (st != MHD_OK) return st;
    MHD_TRY(cudaStreamSynchronize(s->stream));
    return MHD_OK;
}

}  // extern "C"
