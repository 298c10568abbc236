// Host side of the adjoint C ABI (mhd_adj_* in include/mhd_b200.h).
//
// Forward: the same kernels as a single context (stage 1, implicit solve, stage 2, implicit solve,
// finalize) on a fixed dt, with every intermediate a step produces kept in a slot:
//   T[6]   predictor U1* (stage 1)          A[6]  accumulator -> U2* (stage 2; its hydro planes
//   Bn[2]  B^{n+1} (finalize)                     become U^{n+1}'s after the finalize's floor)
// so U^{n+1} = (A[0..3], Bn). The corner fields x1, x2 of every step's two implicit solves are kept
// for the whole trajectory (2 planes per step). A forward pass alternates two slots and copies every
// checkpoint_every-th state out; the backward pass recomputes the explicit stages of a segment of
// steps into one slot per step (the stored solutions stand in for the solves) and then runs the
// adjoint steps backwards over it. With MHD_ADJ_RECOMPUTE_SOLVES the solutions are kept for one
// segment only (2 * checkpoint_every planes): the backward pass recomputes each segment's steps
// with their solves (bit-identical: the solver is deterministic), so device memory grows with
// nsteps / checkpoint_every + checkpoint_every planes instead of 2 * nsteps.
//
// Adjoint of one step (U^{n+1} = Phi(U^n); notation of mhd_adjoint.cuh, cg = dt*g, cd = dt*d,
// c1md = dt*(1-d), c1mg = dt*(1-g), S the implicit rate, R the explicit resistive rate):
//   lambda_B2 = cg R(lam'_B)                           deta += -cg  Jz(lam'_B).Jz(B2)
//   lambda_A  = lam' ; lambda_A_B += lambda_B2 + cg S(lambda_B2)
//                                                      deta += -y2.(Jz(A_B) + cg L x2)
//   lambda_B1 = c1mg R(lambda_A_B) + c1md [F'(U1)^T lambda_A]_B
//                                                      deta += -c1mg Jz(lambda_A_B).Jz(B1)
//   lambda_T  = ([c1md F'(U1)^T lambda_A]_hydro, lambda_B1 + cg S(lambda_B1))
//                                                      deta += -y1.(Jz(T_B) + cg L x1)
//   lam       = lambda_A + lambda_T + F'(U)^T (cd lambda_A + cg lambda_T)
// where y = (I - alpha L)^-1 Jz(cg lambda) is the adjoint solve (the matrix is symmetric) and
// Jz(B2) = Jz(A_B) + cg L x2, Jz(B1) = Jz(T_B) + cg L x1.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "mhd_adjoint.cuh"
#include "mhd_cg_sweep.cuh"
#include "mhd_finalize_sweep.cuh"
#include "mhd_host_util.h"
#include "mhd_sweep.cuh"

using namespace mhd;

namespace {

constexpr int kSlotPlanes = 14;     // T[6], A[6], Bn[2]
constexpr int kScratchPlanes = 59;  // adjoint-step and solver scratch (see AdjScratch)

struct Slot {
    double* T[6];
    double* A[6];
    double* Bn[2];
};

struct AdjScratch {
    double* lam[6];   // the adjoint being propagated
    double* lamT[6];  // adjoint of the predictor
    double* w[6];     // rate adjoint handed to F'^T
    double* fb[2];    // face-B temporaries
    double* c1;       // corner temporaries
    double* c2;
    double* B1[2];    // B1 = T_B + cg C(x1)
    double* y;        // solver solution / adjoint solve
    double* r[2];
    double* p[2];
    double* P[6];     // primitives of the explicit-rate adjoint
    double* X[11];    // x-face adjoints
    double* Y[11];    // y-face adjoints
    double* bc[2];    // cell-centred B adjoints
};

}  // namespace

struct mhd_adjoint {
    mhd_params prm{};
    Domain dom{};
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int device = 0, num_sms = 0;
    size_t n = 0;
    double dt = 0.0, eta = 0.0;
    int nsteps = 0, every = 1, nseg = 0, nslots = 0;
    bool recompute_solves = false;  // keep one segment's solutions, re-solve in the backward pass
    double g = 0.0, d = 0.0;
    double* pool = nullptr;
    std::vector<double*> ckpt;  // nseg * 6 planes
    std::vector<Slot> slots;
    std::vector<double*> xs;  // 2 * nsteps planes: the corner fields x1, x2 of every step
    AdjScratch s{};
    StepCoeffs* coeffs = nullptr;
    DeviceStatus* status = nullptr;
    CgSync* sync = nullptr;
    double* partials = nullptr;
    double* dot_partial = nullptr;
    double* geta = nullptr;  // device accumulator of dL/deta
    double* host_small = nullptr;
    SweepGeom sg[2]{}, fg{};
    int st_blocks[2]{}, fn_blocks = 0;
    int cg_strips_x = 0, cg_seg_h = 0, cg_nwarps = 0, cg_grid = 0;
    int ew_blocks = 0, dot_blocks = 0;
    bool have_forward = false;
};

namespace {

mhd_status check_adj(mhd_adjoint* a) {
    if (!a) return MHD_ERR_INVALID_ARGUMENT;
    MHD_TRY(cudaSetDevice(a->device));
    return MHD_OK;
}

CPlanes cplanes6(const double* const* f) {
    CPlanes p;
    for (int k = 0; k < 6; ++k) p.f[k] = f[k];
    return p;
}
Planes planes6(double* const* f) {
    Planes p;
    for (int k = 0; k < 6; ++k) p.f[k] = f[k];
    return p;
}

// Fixed-dt step coefficients (the formulas of step_coeffs_one with alpha = (dt*eta)*g).
mhd_status upload_coeffs(mhd_adjoint* a) {
    StepCoeffs C{};
    C.dt = a->dt;
    C.c_g = a->dt * a->g;
    C.c_d = a->dt * a->d;
    C.c_1md = a->dt * (1.0 - a->d);
    C.c_1mg = a->dt * (1.0 - a->g);
    C.alpha = (a->dt * a->eta) * a->g;
    MHD_TRY(cudaMemcpyAsync(a->coeffs, &C, sizeof(C), cudaMemcpyHostToDevice, a->stream));
    MHD_TRY(cudaStreamSynchronize(a->stream));
    a->dom.eta = a->eta;
    return MHD_OK;
}

// (I - alpha L) x = rhs_scale * Jz(bxf, byf) with the step's alpha.
mhd_status solve(mhd_adjoint* a, const double* bxf, const double* byf, double rhs_scale, double* x) {
    MHD_TRY(cudaMemsetAsync(a->sync, 0, sizeof(CgSync), a->stream));
    CgSweepArgs g{};
    g.D = a->dom;
    g.D.eta = rhs_scale;
    g.C = a->coeffs;
    g.bxf = bxf;
    g.byf = byf;
    g.x = x;
    g.r[0] = a->s.r[0];
    g.r[1] = a->s.r[1];
    g.p[0] = a->s.p[0];
    g.p[1] = a->s.p[1];
    g.partials = a->partials;
    g.sync = a->sync;
    g.st = a->status;
    g.prods_out = nullptr;
    g.solve_index = 0;
    g.strips_x = a->cg_strips_x;
    g.seg_h = a->cg_seg_h;
    g.nwarps = a->cg_nwarps;
    g.max_iters = a->prm.cg_max_iters > 0 ? a->prm.cg_max_iters : 2LL * (long long)a->n;
    g.tol = a->prm.cg_tol > 0 ? a->prm.cg_tol : 2.220446049250313e-16;
    g.timeout_s = a->prm.cg_timeout_s;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(a->cg_grid);
    cfg.blockDim = dim3(CGS_NT);
    cfg.dynamicSmemBytes = kCgRingBytes;
    cfg.stream = a->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    MHD_TRY(cudaLaunchKernelEx(&cfg, k_cg_sweep, g));
    return MHD_OK;
}

// One forward step from U into slot sl (U^{n+1} = (sl.A[0..3], sl.Bn)) with the corner fields of
// the two solves in x1, x2: solved when do_solve, else taken as stored by an earlier pass (the
// same inputs give bit-identical stage outputs, so the stored solutions are those of this step).
mhd_status forward_step(mhd_adjoint* a, const double* const U[6], const Slot& sl, double* x1,
                        double* x2, bool do_solve) {
    const Domain& D = a->dom;
    k_stage_sweep<1><<<a->st_blocks[0], 32 * SW_WARPS, sweep_smem_bytes(1), a->stream>>>(
        D, a->coeffs, cplanes6(U), nullptr, planes6(sl.T), planes6(sl.A), a->sg[0]);
    MHD_TRY(cudaGetLastError());
    mhd_status s;
    if (do_solve && (s = solve(a, sl.T[4], sl.T[5], a->eta, x1)) != MHD_OK) return s;
    k_stage_sweep<2><<<a->st_blocks[1], 32 * SW_WARPS, sweep_smem_bytes(2), a->stream>>>(
        D, a->coeffs, cplanes6(sl.T), x1, planes6(sl.T), planes6(sl.A), a->sg[1]);
    MHD_TRY(cudaGetLastError());
    if (do_solve && (s = solve(a, sl.A[4], sl.A[5], a->eta, x2)) != MHD_OK) return s;
    MHD_TRY(cudaMemsetAsync(&a->status->smax_bits, 0, sizeof(unsigned long long), a->stream));
    k_finalize_sweep<<<a->fn_blocks, 32 * FS_WARPS, 0, a->stream>>>(
        D, a->coeffs, planes6(sl.A), x2, sl.Bn[0], sl.Bn[1], a->status, a->fg);
    MHD_TRY(cudaGetLastError());
    return MHD_OK;
}

void next_state(const Slot& sl, const double* out[6]) {
    for (int k = 0; k < 4; ++k) out[k] = sl.A[k];
    out[4] = sl.Bn[0];
    out[5] = sl.Bn[1];
}

mhd_status copy_planes(mhd_adjoint* a, double* const dst[6], const double* const src[6]) {
    for (int k = 0; k < 6; ++k)
        MHD_TRY(cudaMemcpyAsync(dst[k], src[k], a->n * sizeof(double), cudaMemcpyDeviceToDevice,
                                a->stream));
    return MHD_OK;
}

// geta += scale * sum(x * y)
mhd_status dot_acc(mhd_adjoint* a, const double* x, const double* y, double scale) {
    k_adj_dot_partial<<<a->dot_blocks, 256, 0, a->stream>>>(a->n, x, y, a->dot_partial);
    MHD_TRY(cudaGetLastError());
    k_adj_dot_final<<<1, 32, 0, a->stream>>>(a->dot_partial, a->dot_blocks, scale, a->geta);
    MHD_TRY(cudaGetLastError());
    return MHD_OK;
}

// out (+)= scale * F'(U)^T w.
mhd_status rate_vjp(mhd_adjoint* a, const double* const U[6], const double* const w[6], double scale,
                    int accumulate, double* const out[6]) {
    const Domain& D = a->dom;
    AdjScratch& s = a->s;
    k_primitives<<<cell_grid(D.nx, D.ny), 256, 0, a->stream>>>(D, cplanes6(U), s.P[0], s.P[1], s.P[2], s.P[3],
                                                      s.P[4], s.P[5]);
    MHD_TRY(cudaGetLastError());
    PrimPlanes P;
    for (int k = 0; k < 6; ++k) P.f[k] = s.P[k];
    FaceAdjPlanes X, Y;
    CFaceAdjPlanes cX, cY;
    for (int k = 0; k < 11; ++k) {
        X.f[k] = s.X[k];
        Y.f[k] = s.Y[k];
        cX.f[k] = s.X[k];
        cY.f[k] = s.Y[k];
    }
    k_adj_faces<0><<<cell_grid(D.nx, D.ny), 256, 0, a->stream>>>(D, P, U[4], U[5], cplanes6(w), X);
    MHD_TRY(cudaGetLastError());
    k_adj_faces<1><<<cell_grid(D.nx, D.ny), 256, 0, a->stream>>>(D, P, U[4], U[5], cplanes6(w), Y);
    MHD_TRY(cudaGetLastError());
    k_adj_cells<<<cell_grid(D.nx, D.ny), 256, 0, a->stream>>>(D, cplanes6(U), P, cX, cY, scale, accumulate,
                                                     planes6(out), s.bc[0], s.bc[1]);
    MHD_TRY(cudaGetLastError());
    k_adj_bfaces<<<cell_grid(D.nx, D.ny), 256, 0, a->stream>>>(D, s.bc[0], s.bc[1], s.X[10], s.Y[10], scale,
                                                      accumulate, out[4], out[5]);
    MHD_TRY(cudaGetLastError());
    return MHD_OK;
}

mhd_status axpby(mhd_adjoint* a, int nplanes, double ca, const double* const* x, double cb,
                 const double* const* y, double* const* out) {
    Planes6C X{}, Y{};
    Planes O{};
    for (int k = 0; k < nplanes; ++k) {
        X.f[k] = x[k];
        Y.f[k] = y ? y[k] : nullptr;
        O.f[k] = out[k];
    }
    k_adj_axpby<<<a->ew_blocks, 256, 0, a->stream>>>(nplanes, a->n, ca, X, cb, Y, O);
    MHD_TRY(cudaGetLastError());
    return MHD_OK;
}

// The adjoint of the step taken from U with intermediates in sl, x1, x2: s.lam holds lam' on
// entry and lam on return; geta accumulates.
mhd_status adjoint_step(mhd_adjoint* a, const double* const U[6], const Slot& sl, const double* x1,
                        const double* x2) {
    const Domain& D = a->dom;
    AdjScratch& s = a->s;
    const double eta = a->eta;
    const double cg = a->dt * a->g, cd = a->dt * a->d;
    const double c1md = a->dt * (1.0 - a->d), c1mg = a->dt * (1.0 - a->g);
    const int B = a->ew_blocks;
    const dim3 CG2 = cell_grid(D.nx, D.ny);
    cudaStream_t st = a->stream;
    mhd_status r;
    // final combination: B^{n+1} = A_B + cg * eta * C Jz(B2)
    k_adj_jz<<<CG2, 256, 0, st>>>(D, s.lam[4], s.lam[5], 1.0, nullptr, 0.0, s.c1);
    k_adj_jz<<<CG2, 256, 0, st>>>(D, sl.A[4], sl.A[5], 1.0, x2, cg, s.c2);  // Jz(B2)
    MHD_TRY(cudaGetLastError());
    if ((r = dot_acc(a, s.c1, s.c2, -cg)) != MHD_OK) return r;
    k_adj_curl<<<CG2, 256, 0, st>>>(D, s.c1, cg * eta, nullptr, nullptr, 0.0, nullptr, nullptr, 0.0,
                                  s.fb[0], s.fb[1]);  // lambda_B2
    MHD_TRY(cudaGetLastError());
    // B2 = A_B + cg S(A_B)
    if ((r = solve(a, s.fb[0], s.fb[1], cg, s.y)) != MHD_OK) return r;
    k_adj_curl<<<CG2, 256, 0, st>>>(D, s.y, eta, s.lam[4], s.lam[5], 1.0, s.fb[0], s.fb[1], 1.0,
                                  s.lam[4], s.lam[5]);  // lambda_A_B
    MHD_TRY(cudaGetLastError());
    if ((r = dot_acc(a, s.y, s.c2, -1.0)) != MHD_OK) return r;
    // g2 = R(B1) with weight c1mg
    k_adj_jz<<<CG2, 256, 0, st>>>(D, s.lam[4], s.lam[5], 1.0, nullptr, 0.0, s.c1);
    k_adj_jz<<<CG2, 256, 0, st>>>(D, sl.T[4], sl.T[5], 1.0, x1, cg, s.c2);  // Jz(B1)
    MHD_TRY(cudaGetLastError());
    if ((r = dot_acc(a, s.c1, s.c2, -c1mg)) != MHD_OK) return r;
    k_adj_curl<<<CG2, 256, 0, st>>>(D, s.c1, c1mg * eta, nullptr, nullptr, 0.0, nullptr, nullptr, 0.0,
                                  s.fb[0], s.fb[1]);
    // f2 = F(U1), U1 = (T hydro, B1), weight c1md
    k_adj_curl<<<CG2, 256, 0, st>>>(D, x1, cg, sl.T[4], sl.T[5], 1.0, nullptr, nullptr, 0.0,
                                  s.B1[0], s.B1[1]);
    MHD_TRY(cudaGetLastError());
    const double* U1[6] = {sl.T[0], sl.T[1], sl.T[2], sl.T[3], s.B1[0], s.B1[1]};
    if ((r = rate_vjp(a, U1, s.lam, c1md, 0, s.lamT)) != MHD_OK) return r;
    // lambda_B1 = lamT_B + fb; B1 = T_B + cg S(T_B)
    {
        const double* x2p[2] = {s.lamT[4], s.lamT[5]};
        const double* y2p[2] = {s.fb[0], s.fb[1]};
        double* o2p[2] = {s.lamT[4], s.lamT[5]};
        if ((r = axpby(a, 2, 1.0, x2p, 1.0, y2p, o2p)) != MHD_OK) return r;
    }
    if ((r = solve(a, s.lamT[4], s.lamT[5], cg, s.y)) != MHD_OK) return r;
    k_adj_curl<<<CG2, 256, 0, st>>>(D, s.y, eta, s.lamT[4], s.lamT[5], 1.0, nullptr, nullptr, 0.0,
                                  s.lamT[4], s.lamT[5]);
    MHD_TRY(cudaGetLastError());
    if ((r = dot_acc(a, s.y, s.c2, -1.0)) != MHD_OK) return r;
    // stage 1: T = U + cg f1, A = U + cd f1 (+ ...): lam = lambda_A + lambda_T + F'(U)^T w
    {
        Planes6C lt;
        for (int k = 0; k < 6; ++k) lt.f[k] = s.lamT[k];
        k_adj_close<<<B, 256, 0, st>>>(a->n, cd, cg, planes6(s.lam), lt, planes6(s.w));
        MHD_TRY(cudaGetLastError());
    }
    const double* wc[6] = {s.w[0], s.w[1], s.w[2], s.w[3], s.w[4], s.w[5]};
    return rate_vjp(a, U, wc, 1.0, 1, s.lam);
}

mhd_status read_status(mhd_adjoint* a) {
    MHD_TRY(cudaStreamSynchronize(a->stream));
    DeviceStatus st;
    MHD_TRY(cudaMemcpy(&st, a->status, sizeof(st), cudaMemcpyDeviceToHost));
    if (st.flags) MHD_TRY(cudaMemset(&a->status->flags, 0, sizeof(unsigned int)));
    if (st.flags & kStatusTimeout) return MHD_ERR_TIMEOUT;
    if (st.flags & kStatusNonFinite) return MHD_ERR_NONFINITE;
    if (st.flags & kStatusCgNotConverged) return MHD_ERR_CG_NOT_CONVERGED;
    return MHD_OK;
}

// The solution planes of step `step` (x1, x2): the trajectory's own, or the segment's when the
// solves are recomputed.
double* xs_of(mhd_adjoint* a, int step, int which) {
    const size_t k = a->recompute_solves ? (size_t)(step % a->every) : (size_t)step;
    return a->xs[2 * k + which];
}

}  // namespace

extern "C" {

mhd_status mhd_adj_create(const mhd_params* p, double dt, int nsteps, int checkpoint_every,
                          void* stream, mhd_adjoint** out) {
    return mhd_adj_create_ex(p, dt, nsteps, checkpoint_every, 0, stream, out);
}

mhd_status mhd_adj_create_ex(const mhd_params* p, double dt, int nsteps, int checkpoint_every,
                             int flags, void* stream, mhd_adjoint** out) {
    if (!p || !out || !(dt > 0) || !std::isfinite(dt) || nsteps < 1 || checkpoint_every < 1 ||
        (flags & ~MHD_ADJ_RECOMPUTE_SOLVES) != 0)
        return MHD_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (p->nx < 2 || p->ny < 2 || !(p->dx > 0) || !(p->dy > 0) || !(p->eta >= 0) ||
        (p->ct_mode != 0 && p->ct_mode != 1) || (long long)p->nx * p->ny > (1LL << 31))
        return MHD_ERR_INVALID_ARGUMENT;
    if (!mhd_device_available()) return MHD_ERR_NO_DEVICE;
    mhd_adjoint* a = new (std::nothrow) mhd_adjoint();
    if (!a) return MHD_ERR_OUT_OF_MEMORY;
    auto fail = [&](mhd_status s) {
        mhd_adj_destroy(a);
        return s;
    };
    a->prm = *p;
    if (!(a->prm.cg_timeout_s > 0)) a->prm.cg_timeout_s = 30.0;
    a->dom.nx = p->nx;
    a->dom.ny = p->ny;
    a->dom.dx = p->dx;
    a->dom.dy = p->dy;
    a->dom.eta = p->eta;
    a->dom.ct_mode = p->ct_mode;
    a->n = (size_t)p->nx * p->ny;
    a->dt = dt;
    a->eta = p->eta;
    a->nsteps = nsteps;
    a->every = std::min(checkpoint_every, nsteps);
    a->recompute_solves = (flags & MHD_ADJ_RECOMPUTE_SOLVES) != 0;
    a->nseg = (nsteps + a->every - 1) / a->every;
    a->nslots = std::max(2, a->every);
    a->g = (2.0 - sqrt(2.0)) / 2.0;     // solvers.hpp:41
    a->d = 1.0 - (1.0 / (2.0 * a->g));  // solvers.hpp:42
    if (cudaGetDevice(&a->device) != cudaSuccess) return fail(MHD_ERR_NO_DEVICE);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, a->device) != cudaSuccess) return fail(MHD_ERR_NO_DEVICE);
    a->num_sms = prop.multiProcessorCount;
    if (stream) {
        a->stream = (cudaStream_t)stream;
    } else {
        if (cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking) != cudaSuccess)
            return fail(MHD_ERR_CUDA);
        a->own_stream = true;
    }
    // launch geometry (as a single context: one wave of sweep warps, one wave of solver blocks)
    for (int mode = 0; mode < 2; ++mode) {
        int occ = 0;
        const cudaError_t e = mode == 0
            ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_stage_sweep<1>, 32 * SW_WARPS, sweep_smem_bytes(1))
            : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_stage_sweep<2>, 32 * SW_WARPS, sweep_smem_bytes(2));
        if (e != cudaSuccess || occ < 1) return fail(MHD_ERR_CUDA);
        const long long resident = (long long)occ * a->num_sms * SW_WARPS;
        SweepGeom& g = a->sg[mode];
        g.strips_x = (p->nx + SW_OUT - 1) / SW_OUT;
        const int segs = (int)std::max(1LL, resident / g.strips_x);
        g.seg_h = std::max(16, (p->ny + segs - 1) / segs);
        g.segs_y = (p->ny + g.seg_h - 1) / g.seg_h;
        g.nwarps = g.strips_x * g.segs_y;
        a->st_blocks[mode] = (g.nwarps + SW_WARPS - 1) / SW_WARPS;
    }
    {
        int occ = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_finalize_sweep, 32 * FS_WARPS, 0) !=
                cudaSuccess || occ < 1)
            return fail(MHD_ERR_CUDA);
        const long long resident = (long long)occ * a->num_sms * FS_WARPS;
        SweepGeom& g = a->fg;
        g.strips_x = (p->nx + FS_OUT - 1) / FS_OUT;
        const int segs = (int)std::max(1LL, resident / g.strips_x);
        g.seg_h = std::max(16, (p->ny + segs - 1) / segs);
        g.segs_y = (p->ny + g.seg_h - 1) / g.seg_h;
        g.nwarps = g.strips_x * g.segs_y;
        a->fn_blocks = (g.nwarps + FS_WARPS - 1) / FS_WARPS;
    }
    {
        int occ = 0;
        if (cudaFuncSetAttribute(k_cg_sweep, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kCgRingBytes) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_cg_sweep, CGS_NT, kCgRingBytes) !=
                cudaSuccess || occ < 1)
            return fail(MHD_ERR_CUDA);
        a->cg_strips_x = (p->nx + CG_W - 1) / CG_W;
        const long long rows_total = (long long)a->cg_strips_x * p->ny;
        const long long max_blocks =
            std::max(1LL, (rows_total + (CGS_NT / 32) * 4 - 1) / ((CGS_NT / 32) * 4));
        a->cg_grid = (int)std::max(1LL, std::min((long long)a->num_sms, max_blocks));
        const long long warps = (long long)a->cg_grid * (CGS_NT / 32);
        const int segs = (int)std::max(1LL, warps / a->cg_strips_x);
        a->cg_seg_h = std::max(4, (p->ny + segs - 1) / segs);
        a->cg_nwarps = a->cg_strips_x * ((p->ny + a->cg_seg_h - 1) / a->cg_seg_h);
    }
    a->ew_blocks = std::max(1, std::min((int)((a->n + 255) / 256), a->num_sms * 8));
    a->dot_blocks = std::max(1, std::min((int)((a->n + 255) / 256), a->num_sms * 2));
    // memory: checkpoints, slots, scratch
    const size_t xplanes = 2 * (size_t)(a->recompute_solves ? a->every : a->nsteps);
    const size_t planes = (size_t)a->nseg * 6 + (size_t)a->nslots * kSlotPlanes + xplanes +
                          kScratchPlanes;
    if (cudaMalloc(&a->pool, planes * a->n * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&a->coeffs, sizeof(StepCoeffs)) != cudaSuccess ||
        cudaMalloc(&a->status, sizeof(DeviceStatus)) != cudaSuccess ||
        cudaMalloc(&a->sync, sizeof(CgSync)) != cudaSuccess ||
        cudaMalloc(&a->partials, (size_t)2 * a->cg_grid * 4 * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&a->dot_partial, (size_t)a->dot_blocks * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&a->geta, sizeof(double)) != cudaSuccess ||
        cudaMallocHost(&a->host_small, 8 * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        return fail(MHD_ERR_OUT_OF_MEMORY);
    }
    double* q = a->pool;
    auto take = [&]() {
        double* r = q;
        q += a->n;
        return r;
    };
    a->ckpt.resize((size_t)a->nseg * 6);
    for (auto& c : a->ckpt) c = take();
    a->slots.resize(a->nslots);
    for (Slot& sl : a->slots) {
        for (int k = 0; k < 6; ++k) sl.T[k] = take();
        for (int k = 0; k < 6; ++k) sl.A[k] = take();
        sl.Bn[0] = take();
        sl.Bn[1] = take();
    }
    a->xs.resize(xplanes);
    for (auto& x : a->xs) x = take();
    AdjScratch& s = a->s;
    for (int k = 0; k < 6; ++k) s.lam[k] = take();
    for (int k = 0; k < 6; ++k) s.lamT[k] = take();
    for (int k = 0; k < 6; ++k) s.w[k] = take();
    s.fb[0] = take();
    s.fb[1] = take();
    s.c1 = take();
    s.c2 = take();
    s.B1[0] = take();
    s.B1[1] = take();
    s.y = take();
    s.r[0] = take();
    s.r[1] = take();
    s.p[0] = take();
    s.p[1] = take();
    for (int k = 0; k < 6; ++k) s.P[k] = take();
    for (int k = 0; k < 11; ++k) s.X[k] = take();
    for (int k = 0; k < 11; ++k) s.Y[k] = take();
    s.bc[0] = take();
    s.bc[1] = take();
    if (cudaMemsetAsync(a->pool, 0, planes * a->n * sizeof(double), a->stream) != cudaSuccess ||
        cudaMemsetAsync(a->status, 0, sizeof(DeviceStatus), a->stream) != cudaSuccess)
        return fail(MHD_ERR_CUDA);
    const mhd_status st = upload_coeffs(a);
    if (st != MHD_OK) return fail(st);
    *out = a;
    return MHD_OK;
}

mhd_status mhd_adj_destroy(mhd_adjoint* a) {
    if (!a) return MHD_ERR_INVALID_ARGUMENT;
    cudaSetDevice(a->device);
    if (a->stream) cudaStreamSynchronize(a->stream);
    cudaFree(a->pool);
    cudaFree(a->coeffs);
    cudaFree(a->status);
    cudaFree(a->sync);
    cudaFree(a->partials);
    cudaFree(a->dot_partial);
    cudaFree(a->geta);
    if (a->host_small) cudaFreeHost(a->host_small);
    if (a->own_stream && a->stream) cudaStreamDestroy(a->stream);
    cudaGetLastError();
    delete a;
    return MHD_OK;
}

mhd_status mhd_adj_set_eta(mhd_adjoint* a, double eta) {
    mhd_status s = check_adj(a);
    if (s != MHD_OK) return s;
    if (!(eta >= 0) || !std::isfinite(eta)) return MHD_ERR_INVALID_ARGUMENT;
    a->eta = eta;
    a->have_forward = false;
    return upload_coeffs(a);
}

mhd_status mhd_adj_forward(mhd_adjoint* a, const double* const u0[6], double* const uT[6]) {
    MHD_NVTX_RANGE("mhd_adj_forward");
    mhd_status s = check_adj(a);
    if (s != MHD_OK) return s;
    if (!u0 || !uT) return MHD_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < 6; ++k)
        if (!u0[k] || !uT[k]) return MHD_ERR_INVALID_ARGUMENT;
    const double* U[6];
    for (int step = 0; step < a->nsteps; ++step) {
        if (step % a->every == 0) {
            double* const* ck = &a->ckpt[(size_t)(step / a->every) * 6];
            if ((s = copy_planes(a, ck, step == 0 ? u0 : U)) != MHD_OK) return s;
            for (int k = 0; k < 6; ++k) U[k] = ck[k];
        }
        const Slot& sl = a->slots[step % 2];
        if ((s = forward_step(a, U, sl, xs_of(a, step, 0), xs_of(a, step, 1), true)) != MHD_OK) return s;
        next_state(sl, U);
    }
    if ((s = copy_planes(a, uT, U)) != MHD_OK) return s;
    a->have_forward = true;
    return read_status(a);
}

mhd_status mhd_adj_backward(mhd_adjoint* a, const double* const grad_uT[6], double* const grad_u0[6],
                            double* grad_eta) {
    MHD_NVTX_RANGE("mhd_adj_backward");
    mhd_status s = check_adj(a);
    if (s != MHD_OK) return s;
    if (!grad_uT || !grad_u0) return MHD_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < 6; ++k)
        if (!grad_uT[k] || !grad_u0[k]) return MHD_ERR_INVALID_ARGUMENT;
    if (!a->have_forward) return MHD_ERR_NO_STATE;
    if ((s = copy_planes(a, a->s.lam, grad_uT)) != MHD_OK) return s;
    MHD_TRY(cudaMemsetAsync(a->geta, 0, sizeof(double), a->stream));
    for (int seg = a->nseg - 1; seg >= 0; --seg) {
        const int s0 = seg * a->every, s1 = std::min(a->nsteps, s0 + a->every);
        const double* const* ck = &a->ckpt[(size_t)seg * 6];
        // recompute the explicit stages of the segment (and, with recompute_solves, its solves),
        // keeping every step's intermediates
        const double* U[6];
        for (int k = 0; k < 6; ++k) U[k] = ck[k];
        for (int step = s0; step < s1; ++step) {
            const Slot& sl = a->slots[step - s0];
            if ((s = forward_step(a, U, sl, xs_of(a, step, 0), xs_of(a, step, 1), a->recompute_solves)) !=
                MHD_OK)
                return s;
            next_state(sl, U);
        }
        for (int step = s1 - 1; step >= s0; --step) {
            const double* Us[6];
            if (step == s0) {
                for (int k = 0; k < 6; ++k) Us[k] = ck[k];
            } else {
                next_state(a->slots[step - s0 - 1], Us);
            }
            if ((s = adjoint_step(a, Us, a->slots[step - s0], xs_of(a, step, 0), xs_of(a, step, 1))) !=
                MHD_OK)
                return s;
        }
    }
    const double* lamc[6] = {a->s.lam[0], a->s.lam[1], a->s.lam[2], a->s.lam[3], a->s.lam[4], a->s.lam[5]};
    if ((s = copy_planes(a, grad_u0, lamc)) != MHD_OK) return s;
    MHD_TRY(cudaMemcpyAsync(a->host_small, a->geta, sizeof(double), cudaMemcpyDeviceToHost, a->stream));
    s = read_status(a);
    if (grad_eta) *grad_eta = a->host_small[0];
    return s;
}

mhd_status mhd_adj_step_vjp(mhd_adjoint* a, const double* const u[6], const double* const lam_next[6],
                            double* const lam[6], double* grad_eta) {
    mhd_status s = check_adj(a);
    if (s != MHD_OK) return s;
    if (!u || !lam_next || !lam) return MHD_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < 6; ++k)
        if (!u[k] || !lam_next[k] || !lam[k]) return MHD_ERR_INVALID_ARGUMENT;
    a->have_forward = false;  // the slots are reused
    if ((s = forward_step(a, u, a->slots[0], a->xs[0], a->xs[1], true)) != MHD_OK) return s;
    if ((s = copy_planes(a, a->s.lam, lam_next)) != MHD_OK) return s;
    MHD_TRY(cudaMemsetAsync(a->geta, 0, sizeof(double), a->stream));
    if ((s = adjoint_step(a, u, a->slots[0], a->xs[0], a->xs[1])) != MHD_OK) return s;
    const double* lamc[6] = {a->s.lam[0], a->s.lam[1], a->s.lam[2], a->s.lam[3], a->s.lam[4], a->s.lam[5]};
    if ((s = copy_planes(a, lam, lamc)) != MHD_OK) return s;
    MHD_TRY(cudaMemcpyAsync(a->host_small, a->geta, sizeof(double), cudaMemcpyDeviceToHost, a->stream));
    s = read_status(a);
    if (grad_eta) *grad_eta = a->host_small[0];
    return s;
}

mhd_status mhd_adj_rate_vjp(mhd_adjoint* a, const double* const u[6], const double* const w[6],
                            double* const out[6]) {
    mhd_status s = check_adj(a);
    if (s != MHD_OK) return s;
    if (!u || !w || !out) return MHD_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < 6; ++k)
        if (!u[k] || !w[k] || !out[k]) return MHD_ERR_INVALID_ARGUMENT;
    if ((s = rate_vjp(a, u, w, 1.0, 0, out)) != MHD_OK) return s;
    MHD_TRY(cudaStreamSynchronize(a->stream));
    return MHD_OK;
}

void* mhd_adj_stream(mhd_adjoint* a) { return a ? (void*)a->stream : nullptr; }

size_t mhd_adj_device_bytes(mhd_adjoint* a) {
    if (!a) return 0;
    const size_t xplanes = 2 * (size_t)(a->recompute_solves ? a->every : a->nsteps);
    const size_t planes = (size_t)a->nseg * 6 + (size_t)a->nslots * kSlotPlanes + xplanes +
                          kScratchPlanes;
    return planes * a->n * sizeof(double);
}

mhd_status mhd_adj_launch_counts(mhd_adjoint* a, int* forward_step, int* adjoint_step) {
    if (!a) return MHD_ERR_INVALID_ARGUMENT;
    // forward: stage 1, solve, stage 2, solve, finalize
    if (forward_step) *forward_step = 5;
    // adjoint: 4 corner currents, 4 dot products (2 launches each), 5 curls, 2 solves,
    // 2 explicit-rate VJPs (4 kernels + primitives each), 2 plane combinations; plus the
    // recomputation of the step's explicit stages (stage 1, stage 2, finalize)
    if (adjoint_step) *adjoint_step = 4 + 8 + 5 + 2 + 10 + 2 + 3 + (a->recompute_solves ? 2 : 0);
    return MHD_OK;
}

}  // extern "C"
