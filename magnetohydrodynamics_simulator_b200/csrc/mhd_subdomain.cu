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
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>

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

// Sum block partials (K per block) in block order into out[K] (one warp).
template <int K>
__global__ void k_sub_final(const double* __restrict__ part, int nblocks, double* out) {
    if (threadIdx.x != 0) return;
    double s[K];
#pragma unroll
    for (int k = 0; k < K; ++k) s[k] = 0.0;
    for (int b = 0; b < nblocks; ++b) {
#pragma unroll
        for (int k = 0; k < K; ++k) s[k] += part[(size_t)b * K + k];
    }
#pragma unroll
    for (int k = 0; k < K; ++k) out[k] = s[k];
}

__global__ void k_sub_set_coeffs(StepCoeffs* C, double dt, double alpha, double g, double d) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    C->dt = dt;
    C->c_g = dt * g;
    C->c_d = dt * d;
    C->c_1md = dt * (1.0 - d);
    C->c_1mg = dt * (1.0 - g);
    C->alpha = alpha;
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

// b = eta J_z(B*) on the interior corners (solvers.hpp:450-461), r = b, z = p = b/d, x = 0;
// block partials |b|^2, r.z.
__global__ void __launch_bounds__(kSubNT)
k_sub_cg_rhs(Interior v, double eta, double idx, double idy, const double* __restrict__ bxf,
             const double* __restrict__ byf, SubVecs V, SubScal s, double* part) {
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
k_sub_cg_matvec(Interior v, SubVecs V, SubScal s, double* part) {
    __shared__ double red[kSubNT / 32];
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
k_sub_cg_update(Interior v, SubVecs V, SubScal s, double alpha, double* part) {
    __shared__ double red[kSubNT / 32 * 2];
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
__global__ void __launch_bounds__(kSubNT) k_sub_cg_dir(Interior v, SubVecs V, double beta) {
    const size_t n = (size_t)v.nx * v.ny;
    for (size_t t = (size_t)blockIdx.x * kSubNT + threadIdx.x; t < n; t += (size_t)gridDim.x * kSubNT) {
        const int j = (int)(t / v.nx), i = (int)(t - (size_t)j * v.nx);
        const size_t g = at(v, i, j);
        V.p[g] = __dadd_rn(V.z[g], __dmul_rn(beta, V.p[g]));
    }
}

__global__ void __launch_bounds__(kSubNT) k_sub_zero_interior(Interior v, double* x) {
    const size_t n = (size_t)v.nx * v.ny;
    for (size_t t = (size_t)blockIdx.x * kSubNT + threadIdx.x; t < n; t += (size_t)gridDim.x * kSubNT) {
        const int j = (int)(t / v.nx), i = (int)(t - (size_t)j * v.nx);
        x[at(v, i, j)] = 0.0;
    }
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
    SubScal sc{};
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
    int pending_sums = 0;  // sums enqueued by a CG phase without an output pointer
    cudaEvent_t ev_ready = nullptr;  // in-process exchange: this subdomain's strips may be read
    cudaEvent_t ev_done = nullptr;   // in-process exchange: this subdomain's rings are filled
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
        cudaMalloc(&s->part, (size_t)2 * kSubMaxBlocks * sizeof(double)) != cudaSuccess ||
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
    if (cudaEventCreateWithFlags(&s->ev_ready, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->ev_done, cudaEventDisableTiming) != cudaSuccess)
        return fail(MHD_ERR_CUDA);
    if (cudaMemsetAsync(s->pool, 0, (size_t)kSubPlanes * s->ne * sizeof(double), s->stream) != cudaSuccess ||
        cudaMemsetAsync(s->coeffs, 0, sizeof(StepCoeffs), s->stream) != cudaSuccess ||
        cudaMemsetAsync(s->scratch_status, 0, sizeof(DeviceStatus), s->stream) != cudaSuccess ||
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
    cudaFree(s->part);
    cudaFree(s->dev_out);
    if (s->host_out) cudaFreeHost(s->host_out);
    if (s->ev_ready) cudaEventDestroy(s->ev_ready);
    if (s->ev_done) cudaEventDestroy(s->ev_done);
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
    const int sides[2][2] = {{MHD_SUB_WEST, MHD_SUB_EAST}, {MHD_SUB_SOUTH, MHD_SUB_NORTH}};
    for (int axis = 0; axis < 2; ++axis) {
        // every subdomain's work so far is done before a neighbour reads its strips
        for (int i = 0; i < count; ++i) MHD_TRY(cudaEventRecord(subs[i]->ev_ready, subs[i]->stream));
        for (int i = 0; i < count; ++i) {
            mhd_subdomain* me = subs[i];
            const int p = i % P, q = i / P;
            for (int k = 0; k < 2; ++k) {
                const int side = sides[axis][k];
                const int opposite = side ^ 1;  // WEST <-> EAST, SOUTH <-> NORTH
                int nb;
                if (side == MHD_SUB_WEST) nb = q * P + (p + P - 1) % P;
                else if (side == MHD_SUB_EAST) nb = q * P + (p + 1) % P;
                else if (side == MHD_SUB_SOUTH) nb = ((q + Q - 1) % Q) * P + p;
                else nb = ((q + 1) % Q) * P + p;
                mhd_subdomain* from = subs[nb];
                if (from != me) MHD_TRY(cudaStreamWaitEvent(me->stream, from->ev_ready, 0));
                // my ring beyond `side` <- the neighbour's strip next to its opposite side
                int dx0 = 0, dy0 = 0, w = 0, h = 0, sx0 = 0, sy0 = 0, sw = 0, sh = 0;
                if (!strip_rect(me, side, width, false, &dx0, &dy0, &w, &h) ||
                    !strip_rect(from, opposite, width, true, &sx0, &sy0, &sw, &sh))
                    return MHD_ERR_INVALID_ARGUMENT;
                Planes dst, src;
                const int np = set_planes(me, set, &dst);
                set_planes(from, set, &src);
                for (int c = 0; c < np; ++c)
                    MHD_TRY(cudaMemcpy2DAsync(dst.f[c] + (size_t)dy0 * me->iv.nxe + dx0,
                                              (size_t)me->iv.nxe * sizeof(double),
                                              src.f[c] + (size_t)sy0 * from->iv.nxe + sx0,
                                              (size_t)from->iv.nxe * sizeof(double), (size_t)w * sizeof(double),
                                              h, cudaMemcpyDeviceToDevice, me->stream));
            }
        }
        // a subdomain changes its interior again only after its neighbours have copied from it
        for (int i = 0; i < count; ++i) MHD_TRY(cudaEventRecord(subs[i]->ev_done, subs[i]->stream));
        for (int i = 0; i < count; ++i)
            for (int j = 0; j < count; ++j)
                if (j != i) MHD_TRY(cudaStreamWaitEvent(subs[i]->stream, subs[j]->ev_done, 0));
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
    k_sub_set_coeffs<<<1, 1, 0, s->stream>>>(s->coeffs, dt, alpha, s->g, s->d);
    MHD_TRY(cudaGetLastError());
    s->sc.cx = alpha / (s->prm.dx * s->prm.dx);
    s->sc.cy = alpha / (s->prm.dy * s->prm.dy);
    s->sc.diag = 1 + 2 * (s->sc.cx + s->sc.cy);
    s->sc.invdiag = (s->sc.diag == 0.0) ? 1.0 : 1.0 / s->sc.diag;
    return MHD_OK;
}

mhd_status mhd_sub_stage(mhd_subdomain* s, int stage) {
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
    k_sub_cg_matvec<<<s->blocks, kSubNT, 0, s->stream>>>(s->iv, s->V, s->sc, s->part);
    MHD_TRY(cudaGetLastError());
    k_sub_final<1><<<1, 32, 0, s->stream>>>(s->part, s->blocks, s->dev_out);
    MHD_TRY(cudaGetLastError());
    return sums_out(s, 1, pq);
}

mhd_status mhd_sub_cg_update(mhd_subdomain* s, double alpha, double out[2]) {
    mhd_status st = check_sub(s);
    if (st != MHD_OK) return st;
    k_sub_cg_update<<<s->blocks, kSubNT, 0, s->stream>>>(s->iv, s->V, s->sc, alpha, s->part);
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
    k_sub_cg_dir<<<s->blocks, kSubNT, 0, s->stream>>>(s->iv, s->V, beta);
    MHD_TRY(cudaGetLastError());
    return MHD_OK;
}

mhd_status mhd_sub_cg_zero_solution(mhd_subdomain* s) {
    mhd_status st = check_sub(s);
    if (st != MHD_OK) return st;
    k_sub_zero_interior<<<s->blocks, kSubNT, 0, s->stream>>>(s->iv, s->V.x);
    MHD_TRY(cudaGetLastError());
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
