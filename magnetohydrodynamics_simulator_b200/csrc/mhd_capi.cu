// Host side of the C ABI declared in include/mhd_b200.h: device memory plan, launch sequence of
// one ARS(2,2,2) step, the CUDA-graph driver loop, diagnostics and status reporting.
//
// Device memory of a context (all dense nx*ny FP64 planes, periodic, row-major):
//   S[6]  current state            (rho, mx, my, E, bxf, byf)
//   T[6]  predictor U1*            (also scratch for primitives read-back between steps)
//   A[6]  accumulator -> U2*       (its hydro planes become the next state's: pointers swap)
//   x, r[2], p[2]                  conjugate-gradient vectors on the corner nodes
// 23 planes, 184 bytes per cell: 3.1 GB at 4096^2.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <mutex>
#include <vector>

#include "../../include/mhd_b200.h"
#include "mhd_cg_sweep.cuh"
#include "mhd_snapshot.h"
#include "mhd_host_util.h"
#include "mhd_kernels.cuh"
#include "mhd_finalize_sweep.cuh"
#include "mhd_sweep.cuh"

using namespace mhd;

namespace {

constexpr int kPlanes = 23;

struct RunRecord {
    double* dts = nullptr;
    long long* prods = nullptr;
    int cap = 0;
};

}  // namespace

struct mhd_context {
    mhd_params prm{};
    Domain dom{};
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int device = 0;
    int num_sms = 0;
    size_t n = 0;
    double* pool = nullptr;
    double* S[6]{};
    double* T[6]{};
    double* A[6]{};
    double* x = nullptr;
    double* r[2]{};
    double* p[2]{};
    double* partials = nullptr;
    CgSync* sync = nullptr;
    DeviceStatus* status = nullptr;
    StepCoeffs* coeffs = nullptr;
    double* divb_partial = nullptr;
    double* divb_out = nullptr;
    double* host_pinned = nullptr;  // small read-back area
    double* padded = nullptr;       // staging for padded-layout transfers
    size_t padded_elems = 0;
    int divb_blocks = 0;
    SweepGeom sg[2]{};       // explicit-stage sweep geometry (stage 1, stage 2)
    int st_blocks[2]{};
    SweepGeom fg{};          // finalize sweep geometry
    int fn_blocks = 0;
    int cg_strips_x = 0, cg_seg_h = 0, cg_nwarps = 0, cg_grid = 0;
    bool have_state = false;
    bool alpha_fixed = false;
    double alpha = 0.0;
    RunRecord run;
    double g = 0.0, d = 0.0;  // ARS(2,2,2) constants
    // kernel timing: 6 events per recorded step (before stage 1, after each of the 5 kernels)
    bool timing = false;
    std::vector<cudaEvent_t> events;
    size_t events_used = 0;
    mhd_host::SnapshotWriter* snap = nullptr;  // created by the first mhd_snapshot_write
    // pipelined host transfers (mhd_set_state_async / mhd_get_state_async), created on first use
    cudaStream_t h2d = nullptr, d2h = nullptr;
    cudaEvent_t ev_ctx = nullptr, ev_h2d = nullptr, ev_join = nullptr;
    // pipelined transfers move each plane in kXferChunks pieces, one event per piece
    static constexpr int kXferChunks = 4;
    cudaEvent_t ev_d2h[6 * kXferChunks]{};
    bool d2h_pending[6 * kXferChunks]{};
    bool join_pending = false;  // state planes still read by mhd_get_state_async's copies
};

namespace {

using mhd_host::cuda_status;
using mhd_host::env_int;

// Request for k_step_coeffs, mirroring the decisions of the reference driver.
mhd_status launch_coeffs(mhd_context* c, double dt, int alpha_mode, double t_end, double* dts_out) {
    const double hmin = std::min(c->prm.dx, c->prm.dy);
    k_step_coeffs<<<1, 1, 0, c->stream>>>(c->coeffs, c->status, dt, c->alpha, alpha_mode, c->prm.eta,
                                           hmin, c->prm.courant, c->prm.safety, c->g, c->d, t_end,
                                           dts_out);
    MHD_TRY(cudaGetLastError());
    return MHD_OK;
}

mhd_status launch_cg(mhd_context* c, const double* bxf, const double* byf, int solve_index,
                     long long* prods_out) {
    MHD_TRY(cudaMemsetAsync(c->sync, 0, sizeof(CgSync), c->stream));
    CgSweepArgs a{};
    a.D = c->dom;
    a.C = c->coeffs;
    a.bxf = bxf;
    a.byf = byf;
    a.x = c->x;
    a.r[0] = c->r[0];
    a.r[1] = c->r[1];
    a.p[0] = c->p[0];
    a.p[1] = c->p[1];
    a.partials = c->partials;
    a.sync = c->sync;
    a.st = c->status;
    a.prods_out = prods_out;
    a.solve_index = solve_index;
    a.strips_x = c->cg_strips_x;
    a.seg_h = c->cg_seg_h;
    a.nwarps = c->cg_nwarps;
    a.max_iters = c->prm.cg_max_iters > 0 ? c->prm.cg_max_iters : 2LL * (long long)c->n;
    a.tol = c->prm.cg_tol > 0 ? c->prm.cg_tol : 2.220446049250313e-16;
    a.timeout_s = c->prm.cg_timeout_s;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(c->cg_grid);
    cfg.blockDim = dim3(CGS_NT);
    cfg.dynamicSmemBytes = kCgRingBytes;
    cfg.stream = c->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    MHD_TRY(cudaLaunchKernelEx(&cfg, k_cg_sweep, a));
    return MHD_OK;
}

CPlanes cplanes(double* const* f) {
    CPlanes p;
    for (int k = 0; k < 6; ++k) p.f[k] = f[k];
    return p;
}
Planes planes(double* const* f) {
    Planes p;
    for (int k = 0; k < 6; ++k) p.f[k] = f[k];
    return p;
}

// Record the next timing event of the current step (no-op unless timing is enabled).
mhd_status mark(mhd_context* c) {
    if (!c->timing) return MHD_OK;
    if (c->events_used == c->events.size()) {
        cudaEvent_t e;
        MHD_TRY(cudaEventCreate(&e));
        c->events.push_back(e);
    }
    MHD_TRY(cudaEventRecord(c->events[c->events_used++], c->stream));
    return MHD_OK;
}

#define MHD_MARK(c)                          \
    do {                                     \
        mhd_status _m = mark(c);             \
        if (_m != MHD_OK) return _m;         \
    } while (0)

// The kernels of one step after the coefficients kernel.
mhd_status enqueue_step_body(mhd_context* c, long long* prods_out) {
    MHD_MARK(c);
    k_stage_sweep<1><<<c->st_blocks[0], 32 * SW_WARPS, sweep_smem_bytes(1), c->stream>>>(
        c->dom, c->coeffs, cplanes(c->S), nullptr, planes(c->T), planes(c->A), c->sg[0]);
    MHD_TRY(cudaGetLastError());
    MHD_MARK(c);
    mhd_status s = launch_cg(c, c->T[4], c->T[5], 0, prods_out);
    if (s != MHD_OK) return s;
    MHD_MARK(c);
    k_stage_sweep<2><<<c->st_blocks[1], 32 * SW_WARPS, sweep_smem_bytes(2), c->stream>>>(
        c->dom, c->coeffs, cplanes(c->T), c->x, planes(c->T), planes(c->A), c->sg[1]);
    MHD_TRY(cudaGetLastError());
    MHD_MARK(c);
    s = launch_cg(c, c->A[4], c->A[5], 1, prods_out);
    if (s != MHD_OK) return s;
    MHD_TRY(cudaMemsetAsync(&c->status->smax_bits, 0, sizeof(unsigned long long), c->stream));
    MHD_MARK(c);
    k_finalize_sweep<<<c->fn_blocks, 32 * FS_WARPS, 0, c->stream>>>(
        c->dom, c->coeffs, planes(c->A), c->x, c->S[4], c->S[5], c->status, c->fg);
    MHD_TRY(cudaGetLastError());
    MHD_MARK(c);
    // the accumulator's hydro planes now hold U^{n+1}; the old state's become scratch
    for (int k = 0; k < 4; ++k) std::swap(c->S[k], c->A[k]);
    return MHD_OK;
}

mhd_status refresh_cfl(mhd_context* c) {
    MHD_TRY(cudaMemsetAsync(&c->status->smax_bits, 0, sizeof(unsigned long long), c->stream));
    const int blocks = std::max(1, std::min((int)((c->n + 255) / 256), c->num_sms * 8));
    k_cfl_scan<<<blocks, 256, 0, c->stream>>>(c->dom, cplanes(c->S), c->status);
    MHD_TRY(cudaGetLastError());
    return MHD_OK;
}

mhd_status ensure_padded(mhd_context* c, int ng) {
    const size_t need = (size_t)(c->dom.nx + 2 * ng) * (size_t)(c->dom.ny + 2 * ng);
    if (need <= c->padded_elems) return MHD_OK;
    if (c->padded) cudaFree(c->padded);
    c->padded = nullptr;
    c->padded_elems = 0;
    MHD_TRY(cudaMalloc(&c->padded, need * sizeof(double)));
    c->padded_elems = need;
    return MHD_OK;
}

// Copy one dense device plane to a host plane in the requested layout.
mhd_status plane_to_host(mhd_context* c, const double* src, double* dst, int layout, int ng) {
    const int nx = c->dom.nx, ny = c->dom.ny;
    if (layout == MHD_LAYOUT_DENSE) {
        MHD_TRY(cudaMemcpyAsync(dst, src, c->n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        return MHD_OK;
    }
    mhd_status s = ensure_padded(c, ng);
    if (s != MHD_OK) return s;
    const size_t np = (size_t)(nx + 2 * ng) * (ny + 2 * ng);
    k_pad_plane<<<std::max(1, std::min((int)((np + 255) / 256), c->num_sms * 8)), 256, 0, c->stream>>>(
        src, c->padded, nx, ny, ng);
    MHD_TRY(cudaGetLastError());
    MHD_TRY(cudaMemcpyAsync(dst, c->padded, np * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    // the staging plane is reused by the next call: finish this copy first
    MHD_TRY(cudaStreamSynchronize(c->stream));
    return MHD_OK;
}

mhd_status check_ctx(mhd_context* c) {
    if (!c) return MHD_ERR_INVALID_ARGUMENT;
    MHD_TRY(cudaSetDevice(c->device));
    return MHD_OK;
}

// Enqueue on the context's stream: divB of the current state, then its snapshot into device
// memory d (k_snapshot_pack).
mhd_status enqueue_snapshot(mhd_context* c, int ng, int snapshot_rate, double dt, double* d) {
    k_divb_partial<<<c->divb_blocks, 256, 0, c->stream>>>(c->dom, c->S[4], c->S[5], c->divb_partial);
    MHD_TRY(cudaGetLastError());
    k_divb_final<<<1, 32, 0, c->stream>>>(c->divb_partial, c->divb_blocks, (long long)c->n, c->divb_out);
    MHD_TRY(cudaGetLastError());
    const int nxt = c->dom.nx + 2 * ng, nyt = c->dom.ny + 2 * ng;
    k_snapshot_pack<<<cell_grid(nxt, nyt), 256, 0, c->stream>>>(c->dom, cplanes(c->S), ng,
                                                                (double)snapshot_rate, dt,
                                                                c->divb_out, d);
    MHD_TRY(cudaGetLastError());
    return MHD_OK;
}

mhd_status status_from_flags(unsigned flags) {
    if (flags & kStatusTimeout) return MHD_ERR_TIMEOUT;
    if (flags & kStatusNonFinite) return MHD_ERR_NONFINITE;
    if (flags & kStatusCgNotConverged) return MHD_ERR_CG_NOT_CONVERGED;
    return MHD_OK;
}

}  // namespace

extern "C" {

const char* mhd_status_string(mhd_status s) {
    switch (s) {
        case MHD_OK: return "ok";
        case MHD_ERR_INVALID_ARGUMENT: return "invalid argument";
        case MHD_ERR_CUDA: return "CUDA error";
        case MHD_ERR_NONFINITE: return "non-finite value in the state or the implicit solve";
        case MHD_ERR_CG_NOT_CONVERGED: return "implicit solve reached its iteration cap";
        case MHD_ERR_TIMEOUT: return "implicit solve exceeded its wall-clock limit";
        case MHD_ERR_NO_DEVICE: return "no sm_100 CUDA device (or library not built for it)";
        case MHD_ERR_OUT_OF_MEMORY: return "out of device memory";
        case MHD_ERR_NO_STATE: return "no state set";
        case MHD_ERR_TOO_LARGE: return "grid exceeds the fixed scratch of the allocation-free call";
        case MHD_ERR_IO: return "a snapshot file could not be written";
    }
    return "unknown status";
}

int mhd_device_available(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return 0;
    }
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, k_finalize) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return 1;
}

mhd_status mhd_default_params(mhd_params* p, int nx, int ny, double dx, double dy, double eta) {
    if (!p) return MHD_ERR_INVALID_ARGUMENT;
    memset(p, 0, sizeof(*p));
    p->nx = nx;
    p->ny = ny;
    p->dx = dx;
    p->dy = dy;
    p->eta = eta;
    p->ct_mode = MHD_CT_REFERENCE;
    p->cg_tol = 0.0;
    p->cg_max_iters = 0;
    p->courant = 0.5;
    p->safety = 0.9;
    p->cg_timeout_s = 30.0;
    return MHD_OK;
}

mhd_status mhd_create(const mhd_params* p, void* stream, mhd_context** out) {
    if (!p || !out) return MHD_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (p->nx < 2 || p->ny < 2 || !(p->dx > 0) || !(p->dy > 0) || !(p->eta >= 0) ||
        (p->ct_mode != 0 && p->ct_mode != 1) || (long long)p->nx * p->ny > (1LL << 31))
        return MHD_ERR_INVALID_ARGUMENT;
    if (!mhd_device_available()) return MHD_ERR_NO_DEVICE;
    mhd_context* c = new (std::nothrow) mhd_context();
    if (!c) return MHD_ERR_OUT_OF_MEMORY;
    c->prm = *p;
    if (!(c->prm.courant > 0)) c->prm.courant = 0.5;
    if (!(c->prm.safety > 0)) c->prm.safety = 0.9;
    if (!(c->prm.cg_timeout_s > 0)) c->prm.cg_timeout_s = 30.0;
    c->dom.nx = p->nx;
    c->dom.ny = p->ny;
    c->dom.dx = p->dx;
    c->dom.dy = p->dy;
    c->dom.eta = p->eta;
    c->dom.ct_mode = p->ct_mode;
    c->n = (size_t)p->nx * (size_t)p->ny;
    c->g = (2.0 - sqrt(2.0)) / 2.0;       // solvers.hpp:41
    c->d = 1.0 - (1.0 / (2.0 * c->g));    // solvers.hpp:42
    auto fail = [&](mhd_status s) {
        mhd_destroy(c);
        return s;
    };
    if (cudaGetDevice(&c->device) != cudaSuccess) return fail(MHD_ERR_NO_DEVICE);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, c->device) != cudaSuccess) return fail(MHD_ERR_NO_DEVICE);
    c->num_sms = prop.multiProcessorCount;
    if (stream) {
        c->stream = (cudaStream_t)stream;
    } else {
        if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
            return fail(MHD_ERR_CUDA);
        c->own_stream = true;
    }
    // Explicit-stage sweep: strips of SW_OUT columns, each split into row segments so that the
    // warps of one wave cover the grid.
    {
        const int carve = env_int("MHD_B200_SWEEP_CARVEOUT", -1);
        if (carve >= 0) {
            cudaFuncSetAttribute(k_stage_sweep<1>, cudaFuncAttributePreferredSharedMemoryCarveout, carve);
            cudaFuncSetAttribute(k_stage_sweep<2>, cudaFuncAttributePreferredSharedMemoryCarveout, carve);
        }
    }
    for (int mode = 0; mode < 2; ++mode) {
        int occ = 0;
        const cudaError_t e = mode == 0
            ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_stage_sweep<1>, 32 * SW_WARPS, sweep_smem_bytes(1))
            : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_stage_sweep<2>, 32 * SW_WARPS, sweep_smem_bytes(2));
        if (e != cudaSuccess || occ < 1) return fail(MHD_ERR_CUDA);
        const long long resident = (long long)occ * c->num_sms * SW_WARPS;
        SweepGeom& g = c->sg[mode];
        g.strips_x = (p->nx + SW_OUT - 1) / SW_OUT;
        const int segs = (int)std::max(1LL, resident / g.strips_x);
        g.seg_h = std::max(env_int("MHD_B200_STAGE_MIN_ROWS", 16), (p->ny + segs - 1) / segs);
        g.segs_y = (p->ny + g.seg_h - 1) / g.seg_h;
        g.nwarps = g.strips_x * g.segs_y;
        c->st_blocks[mode] = (g.nwarps + SW_WARPS - 1) / SW_WARPS;
        if (getenv("MHD_B200_VERBOSE"))
            fprintf(stderr, "mhd_b200: stage %d: %d blocks/SM, rows per warp %d, %d warps\n", mode + 1,
                    occ, g.seg_h, g.nwarps);
    }
    {
        int occ = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_finalize_sweep, 32 * FS_WARPS, 0) !=
                cudaSuccess ||
            occ < 1)
            return fail(MHD_ERR_CUDA);
        const long long resident = (long long)occ * c->num_sms * FS_WARPS;
        SweepGeom& g = c->fg;
        g.strips_x = (p->nx + FS_OUT - 1) / FS_OUT;
        const int segs = (int)std::max(1LL, resident / g.strips_x);
        g.seg_h = std::max(16, (p->ny + segs - 1) / segs);
        g.segs_y = (p->ny + g.seg_h - 1) / g.seg_h;
        g.nwarps = g.strips_x * g.segs_y;
        c->fn_blocks = (g.nwarps + FS_WARPS - 1) / FS_WARPS;
    }
    // Implicit solve: one wave of co-resident blocks; strips of 32 corner columns split into row
    // segments over all of their warps.
    {
        int occ = 0;
        if (cudaFuncSetAttribute(k_cg_sweep, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kCgRingBytes) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_cg_sweep, CGS_NT, kCgRingBytes) !=
                cudaSuccess ||
            occ < 1)
            return fail(MHD_ERR_CUDA);
        const int per_sm = std::max(1, std::min(occ, env_int("MHD_B200_CG_BLOCKS_PER_SM", 1)));
        c->cg_strips_x = (p->nx + CG_W - 1) / CG_W;
        const long long rows_total = (long long)c->cg_strips_x * p->ny;
        // no more blocks than there are rows of work for their warps
        const long long max_blocks = std::max(1LL, (rows_total + (CGS_NT / 32) * 4 - 1) / ((CGS_NT / 32) * 4));
        c->cg_grid = (int)std::max(1LL, std::min((long long)per_sm * c->num_sms, max_blocks));
        const long long warps = (long long)c->cg_grid * (CGS_NT / 32);
        const int segs = (int)std::max(1LL, warps / c->cg_strips_x);
        c->cg_seg_h = std::max(4, (p->ny + segs - 1) / segs);
        c->cg_nwarps = c->cg_strips_x * ((p->ny + c->cg_seg_h - 1) / c->cg_seg_h);
    }
    c->divb_blocks = std::max(1, std::min((int)((c->n + 255) / 256), c->num_sms * 4));
    // memory
    if (cudaMalloc(&c->pool, (size_t)kPlanes * c->n * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        return fail(MHD_ERR_OUT_OF_MEMORY);
    }
    double* q = c->pool;
    for (int k = 0; k < 6; ++k) c->S[k] = q + (size_t)k * c->n;
    q += 6 * c->n;
    for (int k = 0; k < 6; ++k) c->T[k] = q + (size_t)k * c->n;
    q += 6 * c->n;
    for (int k = 0; k < 6; ++k) c->A[k] = q + (size_t)k * c->n;
    q += 6 * c->n;
    c->x = q;
    c->r[0] = q + c->n;
    c->r[1] = q + 2 * c->n;
    c->p[0] = q + 3 * c->n;
    c->p[1] = q + 4 * c->n;
    if (cudaMalloc(&c->partials, (size_t)2 * c->cg_grid * 4 * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&c->sync, sizeof(CgSync)) != cudaSuccess ||
        cudaMalloc(&c->status, sizeof(DeviceStatus)) != cudaSuccess ||
        cudaMalloc(&c->coeffs, sizeof(StepCoeffs)) != cudaSuccess ||
        cudaMalloc(&c->divb_partial, (size_t)2 * c->divb_blocks * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&c->divb_out, 2 * sizeof(double)) != cudaSuccess ||
        cudaMallocHost(&c->host_pinned, 64 * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        return fail(MHD_ERR_OUT_OF_MEMORY);
    }
    if (cudaMemsetAsync(c->status, 0, sizeof(DeviceStatus), c->stream) != cudaSuccess ||
        cudaMemsetAsync(c->coeffs, 0, sizeof(StepCoeffs), c->stream) != cudaSuccess ||
        cudaMemsetAsync(c->pool, 0, (size_t)kPlanes * c->n * sizeof(double), c->stream) != cudaSuccess ||
        cudaStreamSynchronize(c->stream) != cudaSuccess)
        return fail(MHD_ERR_CUDA);
    *out = c;
    return MHD_OK;
}

mhd_status mhd_destroy(mhd_context* c) {
    if (!c) return MHD_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->h2d) cudaStreamSynchronize(c->h2d);
    if (c->d2h) cudaStreamSynchronize(c->d2h);
    delete c->snap;  // waits for the snapshots in flight
    cudaFree(c->pool);
    cudaFree(c->partials);
    cudaFree(c->sync);
    cudaFree(c->status);
    cudaFree(c->coeffs);
    cudaFree(c->divb_partial);
    cudaFree(c->divb_out);
    cudaFree(c->padded);
    cudaFree(c->run.dts);
    cudaFree(c->run.prods);
    if (c->host_pinned) cudaFreeHost(c->host_pinned);
    for (cudaEvent_t e : c->events) cudaEventDestroy(e);
    for (cudaEvent_t e : {c->ev_ctx, c->ev_h2d, c->ev_join})
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : c->ev_d2h)
        if (e) cudaEventDestroy(e);
    if (c->h2d) cudaStreamDestroy(c->h2d);
    if (c->d2h) cudaStreamDestroy(c->d2h);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    cudaGetLastError();
    delete c;
    return MHD_OK;
}

void* mhd_stream(mhd_context* c) { return c ? (void*)c->stream : nullptr; }

int mhd_launches_per_step(mhd_context* c) {
    (void)c;
    return 6;  // coefficients, stage 1, CG, stage 2, CG, finalize
}

// Work about to write the state planes waits for the copies of mhd_get_state_async.
static mhd_status join_transfers(mhd_context* c) {
    if (!c->join_pending) return MHD_OK;
    MHD_TRY(cudaStreamWaitEvent(c->stream, c->ev_join, 0));
    c->join_pending = false;
    return MHD_OK;
}

// Copy streams and events of the pipelined transfers (first use).
static mhd_status ensure_transfer_streams(mhd_context* c) {
    if (c->h2d) return MHD_OK;
    MHD_TRY(cudaStreamCreateWithFlags(&c->h2d, cudaStreamNonBlocking));
    MHD_TRY(cudaStreamCreateWithFlags(&c->d2h, cudaStreamNonBlocking));
    MHD_TRY(cudaEventCreateWithFlags(&c->ev_ctx, cudaEventDisableTiming));
    MHD_TRY(cudaEventCreateWithFlags(&c->ev_h2d, cudaEventDisableTiming));
    MHD_TRY(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
    for (cudaEvent_t& e : c->ev_d2h) MHD_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return MHD_OK;
}

mhd_status mhd_set_state(mhd_context* c, const double* const f[6], int layout, int ng) {
    MHD_NVTX_RANGE("mhd_set_state");
    mhd_status s = check_ctx(c);
    if (s != MHD_OK) return s;
    if ((s = join_transfers(c)) != MHD_OK) return s;
    if (!f || (layout != MHD_LAYOUT_DENSE && layout != MHD_LAYOUT_PADDED) ||
        (layout == MHD_LAYOUT_PADDED && ng < 0))
        return MHD_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < 6; ++k)
        if (!f[k]) return MHD_ERR_INVALID_ARGUMENT;
    const int nx = c->dom.nx, ny = c->dom.ny;
    for (int k = 0; k < 6; ++k) {
        if (layout == MHD_LAYOUT_DENSE) {
            MHD_TRY(cudaMemcpyAsync(c->S[k], f[k], c->n * sizeof(double), cudaMemcpyHostToDevice,
                                    c->stream));
        } else {
            const size_t pitch = (size_t)(nx + 2 * ng) * sizeof(double);
            const double* src = f[k] + (size_t)ng * (nx + 2 * ng) + ng;
            MHD_TRY(cudaMemcpy2DAsync(c->S[k], (size_t)nx * sizeof(double), src, pitch,
                                      (size_t)nx * sizeof(double), ny, cudaMemcpyHostToDevice,
                                      c->stream));
        }
    }
    c->have_state = true;
    return refresh_cfl(c);
}

mhd_status mhd_set_state_async(mhd_context* c, const double* const f[6]) {
    mhd_status s = check_ctx(c);
    if (s != MHD_OK) return s;
    if (!f) return MHD_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < 6; ++k)
        if (!f[k]) return MHD_ERR_INVALID_ARGUMENT;
    if ((s = ensure_transfer_streams(c)) != MHD_OK) return s;
    // the planes are overwritten only after the work queued on the context so far
    MHD_TRY(cudaEventRecord(c->ev_ctx, c->stream));
    MHD_TRY(cudaStreamWaitEvent(c->h2d, c->ev_ctx, 0));
    constexpr int KC = mhd_context::kXferChunks;
    for (int k = 0; k < 6; ++k) {
        for (int q = 0; q < KC; ++q) {
            // this piece's host buffer (and device plane) may still be read by the previous
            // mhd_get_state_async: its copy goes first, the later pieces' copies overlap it
            const size_t b = c->n * q / KC, e = c->n * (q + 1) / KC;
            if (c->d2h_pending[k * KC + q]) MHD_TRY(cudaStreamWaitEvent(c->h2d, c->ev_d2h[k * KC + q], 0));
            MHD_TRY(cudaMemcpyAsync(c->S[k] + b, f[k] + b, (e - b) * sizeof(double), cudaMemcpyHostToDevice,
                                    c->h2d));
        }
    }
    if (c->join_pending) {  // copies of planes the last mhd_get_state_async skipped
        MHD_TRY(cudaStreamWaitEvent(c->h2d, c->ev_join, 0));
        c->join_pending = false;
    }
    MHD_TRY(cudaEventRecord(c->ev_h2d, c->h2d));
    MHD_TRY(cudaStreamWaitEvent(c->stream, c->ev_h2d, 0));
    c->have_state = true;
    return refresh_cfl(c);
}

mhd_status mhd_get_state_async(mhd_context* c, double* const f[6]) {
    mhd_status s = check_ctx(c);
    if (s != MHD_OK) return s;
    if (!f) return MHD_ERR_INVALID_ARGUMENT;
    if (!c->have_state) return MHD_ERR_NO_STATE;
    if ((s = ensure_transfer_streams(c)) != MHD_OK) return s;
    MHD_TRY(cudaEventRecord(c->ev_ctx, c->stream));
    MHD_TRY(cudaStreamWaitEvent(c->d2h, c->ev_ctx, 0));
    constexpr int KC = mhd_context::kXferChunks;
    for (int k = 0; k < 6; ++k) {
        if (!f[k]) continue;
        for (int q = 0; q < KC; ++q) {
            const size_t b = c->n * q / KC, e = c->n * (q + 1) / KC;
            MHD_TRY(cudaMemcpyAsync(f[k] + b, c->S[k] + b, (e - b) * sizeof(double), cudaMemcpyDeviceToHost,
                                    c->d2h));
            MHD_TRY(cudaEventRecord(c->ev_d2h[k * KC + q], c->d2h));
            c->d2h_pending[k * KC + q] = true;
        }
    }
    // work that writes the state planes waits for these copies (join_transfers); a following
    // mhd_set_state_async orders its own copies plane by plane instead, so the copies of two
    // steps overlap
    MHD_TRY(cudaEventRecord(c->ev_join, c->d2h));
    c->join_pending = true;
    return MHD_OK;
}

mhd_status mhd_transfers_wait(mhd_context* c) {
    mhd_status s = check_ctx(c);
    if (s != MHD_OK) return s;
    if (c->h2d) MHD_TRY(cudaStreamSynchronize(c->h2d));
    if (c->d2h) MHD_TRY(cudaStreamSynchronize(c->d2h));
    for (bool& b : c->d2h_pending) b = false;
    return MHD_OK;
}

mhd_status mhd_set_state_device(mhd_context* c, const double* const f[6]) {
    mhd_status s = check_ctx(c);
    if (s != MHD_OK) return s;
    if ((s = join_transfers(c)) != MHD_OK) return s;
    if (!f) return MHD_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < 6; ++k) {
        if (!f[k]) return MHD_ERR_INVALID_ARGUMENT;
        MHD_TRY(cudaMemcpyAsync(c->S[k], f[k], c->n * sizeof(double), cudaMemcpyDeviceToDevice,
                                c->stream));
    }
    c->have_state = true;
    return refresh_cfl(c);
}

mhd_status mhd_get_state(mhd_context* c, double* const f[6], int layout, int ng) {
    MHD_NVTX_RANGE("mhd_get_state");
    mhd_status s = check_ctx(c);
    if (s != MHD_OK) return s;
    if (!f || (layout != MHD_LAYOUT_DENSE && layout != MHD_LAYOUT_PADDED) ||
        (layout == MHD_LAYOUT_PADDED && ng < 0))
        return MHD_ERR_INVALID_ARGUMENT;
    if (!c->have_state) return MHD_ERR_NO_STATE;
    for (int k = 0; k < 6; ++k) {
        if (!f[k]) continue;
        s = plane_to_host(c, c->S[k], f[k], layout, ng);
        if (s != MHD_OK) return s;
    }
    MHD_TRY(cudaStreamSynchronize(c->stream));
    return MHD_OK;
}

mhd_status mhd_get_state_device(mhd_context* c, double* const f[6]) {
    mhd_status s = check_ctx(c);
    if (s != MHD_OK) return s;
    if (!f) return MHD_ERR_INVALID_ARGUMENT;
    if (!c->have_state) return MHD_ERR_NO_STATE;
    for (int k = 0; k < 6; ++k) {
        if (!f[k]) continue;
        MHD_TRY(cudaMemcpyAsync(f[k], c->S[k], c->n * sizeof(double), cudaMemcpyDeviceToDevice,
                                c->stream));
    }
    return MHD_OK;
}

mhd_status mhd_state_device_pointers(mhd_context* c, double* out[6]) {
    if (!c || !out) return MHD_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < 6; ++k) out[k] = c->S[k];
    return MHD_OK;
}

mhd_status mhd_get_primitives(mhd_context* c, double* const prim[6], int layout, int ng) {
    mhd_status s = check_ctx(c);
    if (s != MHD_OK) return s;
    if (!prim || (layout != MHD_LAYOUT_DENSE && layout != MHD_LAYOUT_PADDED) ||
        (layout == MHD_LAYOUT_PADDED && ng < 0))
        return MHD_ERR_INVALID_ARGUMENT;
    if (!c->have_state) return MHD_ERR_NO_STATE;
    k_primitives<<<cell_grid(c->dom.nx, c->dom.ny), 256, 0, c->stream>>>(c->dom, cplanes(c->S), c->T[0], c->T[1], c->T[2],
                                                 c->T[3], c->T[4], c->T[5]);
    MHD_TRY(cudaGetLastError());
    for (int k = 0; k < 6; ++k) {
        if (!prim[k]) continue;
        s = plane_to_host(c, c->T[k], prim[k], layout, ng);
        if (s != MHD_OK) return s;
    }
    MHD_TRY(cudaStreamSynchronize(c->stream));
    return MHD_OK;
}

mhd_status mhd_set_implicit_coefficient(mhd_context* c, double alpha) {
    if (!c || !(alpha >= 0) || !std::isfinite(alpha)) return MHD_ERR_INVALID_ARGUMENT;
    c->alpha = alpha;
    c->alpha_fixed = true;
    return MHD_OK;
}

mhd_status mhd_step(mhd_context* c, double dt) {
    MHD_NVTX_RANGE("mhd_step");
    mhd_status s = check_ctx(c);
    if (s != MHD_OK) return s;
    if ((s = join_transfers(c)) != MHD_OK) return s;
    if (!c->have_state) return MHD_ERR_NO_STATE;
    if (!std::isfinite(dt)) return MHD_ERR_INVALID_ARGUMENT;
    s = launch_coeffs(c, dt, c->alpha_fixed ? 0 : 1, 0.0, nullptr);
    if (s != MHD_OK) return s;
    return enqueue_step_body(c, nullptr);
}

mhd_status mhd_run(mhd_context* c, int nsteps, double dt_fixed, double t_end, double* dts_out,
                   long long* prods_out) {
    MHD_NVTX_RANGE("mhd_run");
    mhd_status s = check_ctx(c);
    if (s != MHD_OK) return s;
    if ((s = join_transfers(c)) != MHD_OK) return s;
    if (!c->have_state) return MHD_ERR_NO_STATE;
    if (nsteps < 0 || !std::isfinite(dt_fixed) || !std::isfinite(t_end)) return MHD_ERR_INVALID_ARGUMENT;
    if (nsteps == 0) return MHD_OK;
    if (nsteps > c->run.cap) {
        cudaFree(c->run.dts);
        cudaFree(c->run.prods);
        c->run.dts = nullptr;
        c->run.prods = nullptr;
        c->run.cap = 0;
        MHD_TRY(cudaMalloc(&c->run.dts, (size_t)nsteps * sizeof(double)));
        MHD_TRY(cudaMalloc(&c->run.prods, (size_t)nsteps * 2 * sizeof(long long)));
        c->run.cap = nsteps;
    }
    // driver state: time, previous dt, step counter (integrator_main.cpp:55-60, 76-95)
    k_driver_reset<<<1, 1, 0, c->stream>>>(c->coeffs);
    MHD_TRY(cudaGetLastError());
    struct TimingOff {  // per-kernel events are recorded by mhd_step only
        mhd_context* c;
        bool saved;
        ~TimingOff() { c->timing = saved; }
    } timing_off{c, c->timing};
    c->timing = false;
    const int mode = c->alpha_fixed ? 0 : 2;
    auto one_step = [&]() -> mhd_status {
        mhd_status r = launch_coeffs(c, dt_fixed, mode, t_end, c->run.dts);
        if (r != MHD_OK) return r;
        return enqueue_step_body(c, c->run.prods);
    };
    // Two consecutive steps form one CUDA graph (the state's hydro planes swap every step, so
    // a pair returns to the same buffer assignment); it is replayed nsteps/2 times.
    int done = 0;
    const bool use_graph = nsteps >= 4 && env_int("MHD_B200_NO_GRAPH", 0) == 0;
    if (use_graph) {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        bool ok = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
        if (ok) {
            mhd_status r1 = one_step();
            mhd_status r2 = (r1 == MHD_OK) ? one_step() : r1;
            ok = cudaStreamEndCapture(c->stream, &graph) == cudaSuccess && r1 == MHD_OK && r2 == MHD_OK;
            // the captured launches did not run: undo the two pointer swaps they made
            if (r1 == MHD_OK) for (int k = 0; k < 4; ++k) std::swap(c->S[k], c->A[k]);
            if (r2 == MHD_OK) for (int k = 0; k < 4; ++k) std::swap(c->S[k], c->A[k]);
        }
        if (ok) ok = cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
        if (ok) {
            for (; done + 2 <= nsteps; done += 2) {
                if (cudaGraphLaunch(exec, c->stream) != cudaSuccess) {
                    ok = false;
                    break;
                }
            }
        }
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        if (!ok && done == 0) {
            // capture not possible here: plain launches below
        } else if (!ok) {
            return MHD_ERR_CUDA;
        }
    }
    for (; done < nsteps; ++done) {
        s = one_step();
        if (s != MHD_OK) return s;
    }
    if (dts_out || prods_out) {
        if (dts_out)
            MHD_TRY(cudaMemcpyAsync(dts_out, c->run.dts, (size_t)nsteps * sizeof(double),
                                    cudaMemcpyDeviceToHost, c->stream));
        if (prods_out)
            MHD_TRY(cudaMemcpyAsync(prods_out, c->run.prods, (size_t)nsteps * 2 * sizeof(long long),
                                    cudaMemcpyDeviceToHost, c->stream));
        MHD_TRY(cudaStreamSynchronize(c->stream));
    }
    return MHD_OK;
}

mhd_status mhd_resistive_rate(mhd_context* c, int solve_implicitly, double alpha,
                              const double* bxf, const double* byf, double* bx_rate,
                              double* by_rate, long long* cg_products) {
    mhd_status s = check_ctx(c);
    if (s != MHD_OK) return s;
    if (!bxf || !byf || !bx_rate || !by_rate || (solve_implicitly && !(alpha >= 0)) ||
        !std::isfinite(alpha))
        return MHD_ERR_INVALID_ARGUMENT;
    const int blocks = std::max(1, std::min((int)((c->n + 255) / 256), c->num_sms * 8));
    if (solve_implicitly) {
        k_set_alpha<<<1, 1, 0, c->stream>>>(c->coeffs, alpha);
        MHD_TRY(cudaGetLastError());
        s = launch_cg(c, bxf, byf, 0, nullptr);
        if (s != MHD_OK) return s;
        k_corner_rates<<<blocks, 256, 0, c->stream>>>(c->dom, c->x, nullptr, nullptr, bx_rate, by_rate);
    } else {
        k_corner_rates<<<blocks, 256, 0, c->stream>>>(c->dom, nullptr, bxf, byf, bx_rate, by_rate);
    }
    MHD_TRY(cudaGetLastError());
    if (cg_products) {
        if (!solve_implicitly) {
            *cg_products = 0;
        } else {
            MHD_TRY(cudaMemcpyAsync(c->host_pinned, c->status, sizeof(DeviceStatus),
                                    cudaMemcpyDeviceToHost, c->stream));
            MHD_TRY(cudaStreamSynchronize(c->stream));
            DeviceStatus st;
            memcpy(&st, c->host_pinned, sizeof(st));
            *cg_products = st.cg_products[0];
        }
    }
    return MHD_OK;
}

mhd_status mhd_cfl_dt(mhd_context* c, double* dt) {
    mhd_status s = check_ctx(c);
    if (s != MHD_OK) return s;
    if (!dt) return MHD_ERR_INVALID_ARGUMENT;
    if (!c->have_state) return MHD_ERR_NO_STATE;
    MHD_TRY(cudaMemcpyAsync(c->host_pinned, &c->status->smax_bits, sizeof(unsigned long long),
                            cudaMemcpyDeviceToHost, c->stream));
    MHD_TRY(cudaStreamSynchronize(c->stream));
    double smaxv;
    memcpy(&smaxv, c->host_pinned, sizeof(double));
    // diagnostics.hpp:52-86
    const double h = std::min(c->prm.dx, c->prm.dy);
    double dt_res = INFINITY;
    if (c->prm.eta != 0.0) dt_res = h * h / (4.0 * c->prm.eta);
    if (!(smaxv > 1e-8)) smaxv = std::max(smaxv, 1e-8);
    const double dt_hyp = c->prm.courant * h / smaxv;
    *dt = std::min(dt_hyp, dt_res) * c->prm.safety;
    return MHD_OK;
}

size_t mhd_snapshot_bytes(mhd_context* c, int ng) {
    if (!c || ng < 0 || ng > std::min(c->dom.nx, c->dom.ny)) return 0;
    return (9 + 7 * (size_t)(c->dom.nx + 2 * ng) * (size_t)(c->dom.ny + 2 * ng)) * sizeof(double);
}

mhd_status mhd_snapshot_write(mhd_context* c, const char* path, int ng, int snapshot_rate,
                              double dt) {
    MHD_NVTX_RANGE("mhd_snapshot_write");
    mhd_status s = check_ctx(c);
    if (s != MHD_OK) return s;
    const size_t bytes = mhd_snapshot_bytes(c, ng);
    if (!path || bytes == 0) return MHD_ERR_INVALID_ARGUMENT;
    if (!c->have_state) return MHD_ERR_NO_STATE;
    if (!c->snap) {
        c->snap = new (std::nothrow) mhd_host::SnapshotWriter(c->device);
        if (!c->snap) return MHD_ERR_OUT_OF_MEMORY;
    }
    int slot = 0;
    double* d = nullptr;
    if ((s = c->snap->acquire(bytes, &slot, &d)) != MHD_OK) return s;
    if ((s = enqueue_snapshot(c, ng, snapshot_rate, dt, d)) != MHD_OK) {
        c->snap->release(slot);
        return s;
    }
    return c->snap->submit(slot, c->stream, path, bytes);
}

mhd_status mhd_snapshot_wait(mhd_context* c) {
    mhd_status s = check_ctx(c);
    if (s != MHD_OK) return s;
    return c->snap ? c->snap->wait() : MHD_OK;
}

mhd_status mhd_snapshot_pack(mhd_context* c, int ng, int snapshot_rate, double dt, void* out) {
    mhd_status s = check_ctx(c);
    if (s != MHD_OK) return s;
    const size_t bytes = mhd_snapshot_bytes(c, ng);
    if (!out || bytes == 0) return MHD_ERR_INVALID_ARGUMENT;
    if (!c->have_state) return MHD_ERR_NO_STATE;
    double* d = nullptr;
    MHD_TRY(cudaMallocAsync(&d, bytes, c->stream));
    s = enqueue_snapshot(c, ng, snapshot_rate, dt, d);
    if (s == MHD_OK) {
        const cudaError_t e = cudaMemcpyAsync(out, d, bytes, cudaMemcpyDeviceToHost, c->stream);
        if (e != cudaSuccess) s = mhd_host::cuda_status(e);
    }
    cudaFreeAsync(d, c->stream);
    const cudaError_t e = cudaStreamSynchronize(c->stream);
    if (s == MHD_OK && e != cudaSuccess) s = mhd_host::cuda_status(e);
    return s;
}

mhd_status mhd_divb(mhd_context* c, double* rms, double* maxabs) {
    mhd_status s = check_ctx(c);
    if (s != MHD_OK) return s;
    if (!c->have_state) return MHD_ERR_NO_STATE;
    k_divb_partial<<<c->divb_blocks, 256, 0, c->stream>>>(c->dom, c->S[4], c->S[5], c->divb_partial);
    MHD_TRY(cudaGetLastError());
    k_divb_final<<<1, 32, 0, c->stream>>>(c->divb_partial, c->divb_blocks, (long long)c->n, c->divb_out);
    MHD_TRY(cudaGetLastError());
    MHD_TRY(cudaMemcpyAsync(c->host_pinned, c->divb_out, 2 * sizeof(double), cudaMemcpyDeviceToHost,
                            c->stream));
    MHD_TRY(cudaStreamSynchronize(c->stream));
    if (rms) *rms = c->host_pinned[0];
    if (maxabs) *maxabs = c->host_pinned[1];
    return MHD_OK;
}

mhd_status mhd_synchronize(mhd_context* c) {
    mhd_status s = check_ctx(c);
    if (s != MHD_OK) return s;
    if ((s = mhd_transfers_wait(c)) != MHD_OK) return s;
    MHD_TRY(cudaMemcpyAsync(c->host_pinned, c->status, sizeof(DeviceStatus), cudaMemcpyDeviceToHost,
                            c->stream));
    MHD_TRY(cudaStreamSynchronize(c->stream));
    DeviceStatus st;
    memcpy(&st, c->host_pinned, sizeof(st));
    if (st.flags) {
        MHD_TRY(cudaMemsetAsync(&c->status->flags, 0, sizeof(unsigned int), c->stream));
        MHD_TRY(cudaStreamSynchronize(c->stream));
    }
    return status_from_flags(st.flags);
}

mhd_status mhd_set_kernel_timing(mhd_context* c, int enable) {
    mhd_status s = check_ctx(c);
    if (s != MHD_OK) return s;
    c->timing = enable != 0;
    c->events_used = 0;
    return MHD_OK;
}

mhd_status mhd_kernel_times(mhd_context* c, double out_ms[5], long long* steps) {
    mhd_status s = check_ctx(c);
    if (s != MHD_OK) return s;
    if (!out_ms) return MHD_ERR_INVALID_ARGUMENT;
    MHD_TRY(cudaStreamSynchronize(c->stream));
    for (int k = 0; k < 5; ++k) out_ms[k] = 0.0;
    const size_t nsteps = c->events_used / 6;
    for (size_t st = 0; st < nsteps; ++st) {
        for (int k = 0; k < 5; ++k) {
            float ms = 0.f;
            MHD_TRY(cudaEventElapsedTime(&ms, c->events[6 * st + k], c->events[6 * st + k + 1]));
            out_ms[k] += ms;
        }
    }
    if (steps) *steps = (long long)nsteps;
    c->events_used = 0;
    return MHD_OK;
}

mhd_status mhd_last_cg_products(mhd_context* c, long long out[2]) {
    mhd_status s = check_ctx(c);
    if (s != MHD_OK) return s;
    if (!out) return MHD_ERR_INVALID_ARGUMENT;
    MHD_TRY(cudaMemcpyAsync(c->host_pinned, c->status, sizeof(DeviceStatus), cudaMemcpyDeviceToHost,
                            c->stream));
    MHD_TRY(cudaStreamSynchronize(c->stream));
    DeviceStatus st;
    memcpy(&st, c->host_pinned, sizeof(st));
    out[0] = st.cg_products[0];
    out[1] = st.cg_products[1];
    return MHD_OK;
}

mhd_status mhd_cg_products_sum(mhd_context* c, long long out[2]) {
    mhd_status s = check_ctx(c);
    if (s != MHD_OK) return s;
    if (!out) return MHD_ERR_INVALID_ARGUMENT;
    MHD_TRY(cudaMemcpyAsync(c->host_pinned, c->status, sizeof(DeviceStatus), cudaMemcpyDeviceToHost,
                            c->stream));
    MHD_TRY(cudaStreamSynchronize(c->stream));
    DeviceStatus st;
    memcpy(&st, c->host_pinned, sizeof(st));
    out[0] = st.cg_products_sum[0];
    out[1] = st.cg_products_sum[1];
    return MHD_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// Allocation-free implicit resistive rate (mhd_resistive_rate_noalloc in mhd_b200.h).
//
// All scratch of the solve -- the CG vectors x, r[2], p[2], the per-block partial sums and the
// small control blocks (barrier counter, status, coefficients) -- is carved out of the one
// file-scope array below. In host code g_noalloc_scratch is only a host-side stand-in for the
// symbol; its device address is obtained per device with cudaGetSymbolAddress and passed to the
// kernels.

namespace {

constexpr size_t kNoAllocCells = MHD_NOALLOC_MAX_CELLS;
constexpr int kNoAllocMaxBlocks = 1024;
constexpr size_t kNoAllocVecDoubles = 5 * kNoAllocCells;             // x, r0, r1, p0, p1
constexpr size_t kNoAllocPartialDoubles = 2 * 4 * (size_t)kNoAllocMaxBlocks;
constexpr size_t kNoAllocControlDoubles = 64;                        // CgSync, DeviceStatus, StepCoeffs
constexpr size_t kNoAllocDoubles = kNoAllocVecDoubles + kNoAllocPartialDoubles + kNoAllocControlDoubles;
static_assert(sizeof(CgSync) + sizeof(DeviceStatus) + sizeof(StepCoeffs) <= 8 * kNoAllocControlDoubles,
              "control blocks exceed their reserved space");

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

struct NoAllocDevice {
    bool ready = false;
    double* scratch = nullptr;  // device address of g_noalloc_scratch on this device
    int grid = 0;               // co-resident blocks of the solver kernel
};
constexpr int kNoAllocMaxDevices = 64;
NoAllocDevice g_noalloc_dev[kNoAllocMaxDevices];
std::mutex g_noalloc_mutex;

// Once per device, with that device current: resolve the array's address, size the solver grid.
mhd_status noalloc_setup(int dev, NoAllocDevice** out) {
    if (dev < 0 || dev >= kNoAllocMaxDevices) return MHD_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    NoAllocDevice& d = g_noalloc_dev[dev];
    if (!d.ready) {
        void* addr = nullptr;
        MHD_TRY(cudaGetSymbolAddress(&addr, g_noalloc_scratch));
        MHD_TRY(cudaFuncSetAttribute(k_cg_sweep, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)kCgRingBytes));
        int occ = 0, sms = 0;
        MHD_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_cg_sweep, CGS_NT, kCgRingBytes));
        MHD_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        if (occ < 1) return MHD_ERR_CUDA;
        d.scratch = static_cast<double*>(addr);
        // one block per SM, as a context launches the solver
        d.grid = std::max(1, std::min(sms, kNoAllocMaxBlocks));
        d.ready = true;
    }
    *out = &d;
    return MHD_OK;
}

}  // namespace

extern "C" mhd_status mhd_resistive_rate_noalloc(const mhd_params* p, int solve_implicitly,
                                                 double alpha, const double* bxf,
                                                 const double* byf, double* bx_rate,
                                                 double* by_rate, long long* cg_products,
                                                 void* stream_ptr) {
    if (!p || !bxf || !byf || !bx_rate || !by_rate) return MHD_ERR_INVALID_ARGUMENT;
    if (p->nx < 2 || p->ny < 2 || !(p->dx > 0) || !(p->dy > 0) || !(p->eta >= 0) ||
        !std::isfinite(alpha) || (solve_implicitly && !(alpha >= 0)))
        return MHD_ERR_INVALID_ARGUMENT;
    const size_t n = (size_t)p->nx * (size_t)p->ny;
    if (n > kNoAllocCells) return MHD_ERR_TOO_LARGE;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    Domain D{p->nx, p->ny, p->dx, p->dy, p->eta, p->ct_mode};
    int dev = 0;
    MHD_TRY(cudaGetDevice(&dev));
    NoAllocDevice* nd = nullptr;
    mhd_status s = noalloc_setup(dev, &nd);
    if (s != MHD_OK) return s;
    int sms = 0;
    MHD_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int blocks = std::max(1, std::min((int)((n + 255) / 256), sms * 8));
    if (!solve_implicitly) {
        k_corner_rates<<<blocks, 256, 0, stream>>>(D, nullptr, bxf, byf, bx_rate, by_rate);
        MHD_TRY(cudaGetLastError());
        if (cg_products) *cg_products = 0;
        return MHD_OK;
    }
    // carve the scratch array
    double* base = nd->scratch;
    double* x = base;
    double* r0 = base + kNoAllocCells;
    double* r1 = base + 2 * kNoAllocCells;
    double* p0 = base + 3 * kNoAllocCells;
    double* p1 = base + 4 * kNoAllocCells;
    double* partials = base + kNoAllocVecDoubles;
    unsigned char* ctrl = reinterpret_cast<unsigned char*>(partials + kNoAllocPartialDoubles);
    CgSync* sync = reinterpret_cast<CgSync*>(ctrl);
    DeviceStatus* st = reinterpret_cast<DeviceStatus*>(ctrl + 64);
    StepCoeffs* coeffs = reinterpret_cast<StepCoeffs*>(ctrl + 64 + 128);
    static_assert(sizeof(CgSync) <= 64 && sizeof(DeviceStatus) <= 128 &&
                      64 + 128 + sizeof(StepCoeffs) <= 8 * kNoAllocControlDoubles,
                  "control block layout");
    // what must start at zero: the barrier counter, the status and the coefficient block (the
    // array keeps the previous call's contents)
    MHD_TRY(cudaMemsetAsync(ctrl, 0, 8 * kNoAllocControlDoubles, stream));
    k_set_alpha<<<1, 1, 0, stream>>>(coeffs, alpha);
    MHD_TRY(cudaGetLastError());
    // solver geometry exactly as a context's (mhd_create): strips of CG_W columns, no more blocks
    // than rows of work for their warps, so both entry points reduce in the same order
    const int strips_x = (p->nx + CG_W - 1) / CG_W;
    const long long rows_total = (long long)strips_x * p->ny;
    const long long max_blocks =
        std::max(1LL, (rows_total + (CGS_NT / 32) * 4 - 1) / ((CGS_NT / 32) * 4));
    const int grid = (int)std::max(1LL, std::min((long long)nd->grid, max_blocks));
    const long long warps = (long long)grid * (CGS_NT / 32);
    const int segs = (int)std::max(1LL, warps / strips_x);
    const int seg_h = std::max(4, (p->ny + segs - 1) / segs);
    CgSweepArgs a{};
    a.D = D;
    a.C = coeffs;
    a.bxf = bxf;
    a.byf = byf;
    a.x = x;
    a.r[0] = r0;
    a.r[1] = r1;
    a.p[0] = p0;
    a.p[1] = p1;
    a.partials = partials;
    a.sync = sync;
    a.st = st;
    a.prods_out = nullptr;
    a.solve_index = 0;
    a.strips_x = strips_x;
    a.seg_h = seg_h;
    a.nwarps = strips_x * ((p->ny + seg_h - 1) / seg_h);
    a.max_iters = p->cg_max_iters > 0 ? p->cg_max_iters : 2LL * (long long)n;
    a.tol = p->cg_tol > 0 ? p->cg_tol : 2.220446049250313e-16;
    a.timeout_s = p->cg_timeout_s > 0 ? p->cg_timeout_s : 30.0;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(CGS_NT);
    cfg.dynamicSmemBytes = kCgRingBytes;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    MHD_TRY(cudaLaunchKernelEx(&cfg, k_cg_sweep, a));
    k_corner_rates<<<blocks, 256, 0, stream>>>(D, x, nullptr, nullptr, bx_rate, by_rate);
    MHD_TRY(cudaGetLastError());
    // The solve's status lives only in the shared array, where the next call clears it, so it is
    // read back here on every call: the implicit path always waits for its result.
    DeviceStatus hs;
    MHD_TRY(cudaMemcpyAsync(&hs, st, sizeof(hs), cudaMemcpyDeviceToHost, stream));
    MHD_TRY(cudaStreamSynchronize(stream));
    if (cg_products) *cg_products = hs.cg_products[0];
    return status_from_flags(hs.flags);
}
