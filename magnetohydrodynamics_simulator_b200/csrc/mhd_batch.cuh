// Batched IMEX step: many independent periodic simulations of uneven sizes advanced together,
// one persistent fused launch per stage of the step (coefficients, stage 1, implicit solve,
// stage 2, implicit solve, finalize). Every instance keeps its own dt (CFL or fixed), its own
// matrix coefficient and its own convergence, exactly as if it were stepped alone
// (integrator_main.cpp:76-112 per instance).
//
// The explicit stages and the finalize work on flat lists of warp work items (instance, strip,
// rows): 28-column strips cut into row ranges. Their kernels are persistent and pull items from a
// global counter (largest items first). The solver splits the rows of the instances still
// iterating evenly over its warps in every phase, in a fixed order, because its sums must be
// reduced in a fixed order.
//
// The descriptor array exists twice, for even and odd steps: the finalize leaves U^{n+1}'s hydro
// planes in the accumulator, so the state and accumulator hydro pointers trade places every step.
#pragma once

#include "mhd_cg_sweep.cuh"
#include "mhd_finalize_sweep.cuh"
#include "mhd_sweep.cuh"

namespace mhd {

struct BatchInst {
    Domain D;
    StepCoeffs* C;
    DeviceStatus* st;
    double* S[6];
    double* T[6];
    double* A[6];
    double* x;
    double* r[2];
    double* p[2];
    long long off;  // zone offset of the instance in every plane arena
    int cg_strips_x;  // 28-column strips of the solver
    long long max_iters;
    double tol;
    double alpha;  // fixed matrix coefficient when alpha_fixed
    int alpha_fixed;
    int pad;
    double hmin, courant, safety;
};

// Work item of the explicit stages and the finalize: rows [r0, r1) of column strip sx.
struct SweepItem {
    int inst;
    int sx;
    int r0, r1;
};

static_assert(SW_OUT == FS_OUT, "stages and finalize share one work-item list");

// Step coefficients of every instance (one thread each), then the per-step resets: the max
// signal speed (recomputed by the finalize), the explicit kernels' work counters and the
// solver's barrier counters.
static __global__ void k_batch_coeffs(const BatchInst* __restrict__ insts, int n,
                                      const double* __restrict__ dt_in, double dt_fixed,
                                      int run_mode, double t_end, double g, double d,
                                      double* dts_rec, int rec_stride, int* queues, int nqueues,
                                      CgSync* syncs, int nsync) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nqueues) queues[i] = 0;
    if (i < nsync) {
        syncs[i].count = 0ULL;
        syncs[i].error = 0u;
    }
    if (i >= n) return;
    const BatchInst& I = insts[i];
    const double dt = dt_in ? dt_in[i] : dt_fixed;
    const int mode = I.alpha_fixed ? 0 : run_mode;
    step_coeffs_one(I.C, I.st, dt, I.alpha, mode, I.D.eta, I.hmin, I.courant, I.safety, g, d,
                    t_end, dts_rec ? dts_rec + (size_t)i * rec_stride : nullptr);
    I.st->smax_bits = 0ULL;
}

static __global__ void k_batch_driver_reset(const BatchInst* __restrict__ insts, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    StepCoeffs* C = insts[i].C;
    C->t = 0.0;
    C->prev_dt = 0.0;
    C->step = 0;
    C->cur = 0;
    C->first = 1;
}

// Next work item of the warp from a global counter (lane 0 takes it, all lanes get it).
__device__ __forceinline__ int batch_next_item(int* queue) {
    int it = 0;
    if ((threadIdx.x & 31) == 0) it = atomicAdd(queue, 1);
    return __shfl_sync(0xffffffffu, it, 0);
}

// Stage 2 of the batch carries its y slopes in shared memory (as a single context's stage 2 does)
// and keeps the branchy HLL: the persistent kernel holds an item loop around the sweep, which the
// branch-free HLL pushes into spills. (Measured on B200 on the 64-instance mixed batch: with the
// carried values in shared memory, per-face y slopes 7.18 -> 6.97 ms per step, carried slopes
// 6.93 ms.)
#ifndef MHD_BATCH_YREUSE_2
#define MHD_BATCH_YREUSE_2 1
#endif
#ifndef MHD_BATCH_XREUSE_2
#define MHD_BATCH_XREUSE_2 MHD_SWEEP_XREUSE_2
#endif
// Explicit stage MODE of the batch. base: the arenas of this step's parity (stage 1: in = state,
// a = predictor, b = accumulator; stage 2: in = predictor, x = E1, b = accumulator).
template <int MODE>
__global__ void __launch_bounds__(32 * SW_WARPS, MODE == 1 ? MHD_SWEEP_MIN_BLOCKS_1 : MHD_SWEEP_MIN_BLOCKS_2)
k_stage_batch(const BatchInst* __restrict__ insts, const SweepItem* __restrict__ items, int nitems,
              int* queue, ParamPlanes base) {
#if defined(__CUDA_ARCH__)
    extern __shared__ __align__(16) double sw_ring_mem[];
#else
    static double sw_ring_mem[SW_WARPS * (SW_RING * SW_SLOT + SW_CARRY)];
#endif
    __shared__ SweepInstRec rec[SW_WARPS];
    const int wl = threadIdx.x >> 5;
    double* const ring = sw_ring_mem + (size_t)wl * sweep_warp_doubles(MODE);
    const RecPlanes pl{base, &rec[wl]};
    for (;;) {
        const int it = batch_next_item(queue);
        if (it >= nitems) break;
        const SweepItem e = items[it];
        const BatchInst& I = insts[e.inst];
        __syncwarp();  // the previous item's sweep has read the record
        if ((threadIdx.x & 31) == 0) {
            rec[wl].D = I.D;
            rec[wl].off = I.off;
        }
        __syncwarp();
        stage_sweep_warp<MODE, RecPlanes, MODE == 1 ? MHD_SWEEP_YREUSE_1 : MHD_BATCH_YREUSE_2,
                         MODE == 1 ? MHD_SWEEP_XREUSE_1 : MHD_BATCH_XREUSE_2, MODE == 1>(
            I.C, pl, e.sx, e.r0, e.r1, ring);
    }
}

// RecFin: the finalize's view of one batch instance (arena bases in kernel parameters, the
// instance's offset and grid in the warp's shared record; see RecPlanes).
struct RecFin {
    FinParams base;
    const SweepInstRec* rec;
    __device__ __forceinline__ size_t off() const { return (size_t)RecPlanes::vload(&rec->off); }
    __device__ __forceinline__ double* acc(int q) const { return base.acc_.f[q] + off(); }
    __device__ __forceinline__ const double* x() const { return base.x_ + off(); }
    __device__ __forceinline__ double* bx() const { return base.bx_ + off(); }
    __device__ __forceinline__ double* by() const { return base.by_ + off(); }
    __device__ __forceinline__ int nx() const { return RecPlanes::vload(&rec->D.nx); }
    __device__ __forceinline__ int ny() const { return RecPlanes::vload(&rec->D.ny); }
    __device__ __forceinline__ double dx() const { return RecPlanes::vload(&rec->D.dx); }
    __device__ __forceinline__ double dy() const { return RecPlanes::vload(&rec->D.dy); }
    __device__ __forceinline__ double eta() const { return RecPlanes::vload(&rec->D.eta); }
};

// Finalize of the batch. base: the arenas of this step's parity (acc = accumulator, x = E2,
// bx / by = the state's face planes).
static __global__ void __launch_bounds__(32 * FS_WARPS)
k_finalize_batch(const BatchInst* __restrict__ insts, const SweepItem* __restrict__ items, int nitems,
                 int* queue, FinParams base) {
    __shared__ SweepInstRec rec[FS_WARPS];
    const int wl = threadIdx.x >> 5;
    const RecFin f{base, &rec[wl]};
    for (;;) {
        const int it = batch_next_item(queue);
        if (it >= nitems) break;
        const SweepItem e = items[it];
        const BatchInst& I = insts[e.inst];
        __syncwarp();  // the previous item's sweep has read the record
        if ((threadIdx.x & 31) == 0) {
            rec[wl].D = I.D;
            rec[wl].off = I.off;
        }
        __syncwarp();
        finalize_sweep_warp(f, I.C, I.st, e.sx, e.r0, e.r1);
    }
}

// ------------------------------------------------------------------------------------------
// Batched implicit solve: the CGs of up to CGB_MAX_INST instances in one persistent cooperative
// kernel, running their phases in lockstep (solvers.hpp:404-489 per instance, Eigen's
// ConjugateGradient defaults as in k_cg_sweep).
//
// In every phase the work of the instances still iterating is numbered 0 .. T-1 through a prefix
// sum of their counts, which every block rebuilds from the same decisions, and split over the W
// warps of the grid in one of two ways (the autotuner times both):
//   order 0, rows: the strip rows, instance by instance, band of `rows` rows by band, strip by
//     strip within a band, row by row; warp g sweeps rows [T g/W, T (g+1)/W) as one or more
//     (instance, strip, row range) segments, so a block's warps sweep neighbouring strips of a band;
//   order 1, tiles: tiles of 28 columns x `rows` rows, instance by instance, row of tiles by row;
//     warp g sweeps tiles g, g + W, ...
// Either way every warp gets an even share whichever instances remain, and the sums keep a fixed
// order: So the work of a phase is spread
// evenly over all warps whichever instances remain, and the sums keep a fixed order: every warp sums its partials per instance (item order), each block
// sums its warps per instance (warp order) and publishes one partial per (instance, block); after
// the grid barrier every block reduces each instance's block partials in the same fixed order, so
// all blocks hold identical scalars and take identical decisions. The loop ends when no instance
// is active.

constexpr int CGB_MAX_INST = 64;
// Threads per block of the batched solver (its own size: the per-warp partial sums of 64 instances
// live in dynamic shared memory beside the rows' rings).
#ifndef MHD_CGB_NT
#define MHD_CGB_NT 512
#endif
constexpr int CGB_NT = MHD_CGB_NT;
constexpr int CGB_NW = CGB_NT / 32;
// dynamic shared memory of a k_cg_batch block: the warps' row rings, then wsum[CGB_NW][64][4]
constexpr size_t kCgbRingBytes = (size_t)CGB_NW * CG_RING * CG_SLOT * sizeof(double);
constexpr size_t kCgbSmemBytes = kCgbRingBytes + (size_t)CGB_NW * CGB_MAX_INST * 4 * sizeof(double);

enum CgInstStatus : int { kCgActive = 0, kCgConverged = 1, kCgZero = 2, kCgBreakdown = 3, kCgCapped = 4 };

struct CgBInst {
    double cx, cy, diag, invdiag;  // matrix of this solve
    double alpha, beta;            // CG step scalars
    double alpha_prev;             // alpha of the previous iteration (paired updates of x)
    double bb, absNew, thr, rr, pAp;
    long long products;
    int status;
    int ny, strips;   // rows, 28-column strips
};

struct CgBatchArgs {
    const BatchInst* insts;  // descriptors of this step's parity
    int inst0, ninst;        // instances [inst0, inst0 + ninst) of this launch
    int order;               // 0: even row ranges in bands of `rows` rows; 1: tiles of `rows` rows
    int rows;                // order 1 with rows = 0: the tile height is chosen phase by phase
    double* partials;        // [2][CGB_MAX_INST][gridDim.x][4]
    CgSync* sync;
    int solve_index;         // 0: B* = U1*_B (T planes), 1: B* = U2*_B (A planes)
    int rec_stride;
    long long* prods_rec;    // [instance][rec_stride][2] products record, or null
    double timeout_s;
};

__device__ __forceinline__ CgSweepArgs cgb_args(const CgBatchArgs& a, const BatchInst& I) {
    CgSweepArgs g{};
    g.D = I.D;
    g.C = I.C;
    g.bxf = (a.solve_index == 0) ? I.T[4] : I.A[4];
    g.byf = (a.solve_index == 0) ? I.T[5] : I.A[5];
    g.x = I.x;
    g.r[0] = I.r[0];
    g.r[1] = I.r[1];
    g.p[0] = I.p[0];
    g.p[1] = I.p[1];
    g.strips_x = I.cg_strips_x;
    return g;
}

// Tile heights the phase-by-phase choice picks from (order 1 with rows = 0).
constexpr int kCgbNHeights = 16;
__device__ __constant__ const int kCgbHeights[kCgbNHeights] = {16,  20,  24,  28,  32,  40,  48,  56,
                                                               64,  80,  96,  112, 128, 160, 192, 256};

// The phase's decomposition of the instances with pick(instance): the tile height h (order 1) and
// the prefix sum over the chunk's instances (at most 64) of their work units, strip rows (order 0)
// or tiles of h rows (order 1), by the first warp (lane l: instances l and l + 32), then a block
// barrier. With rows = 0 the height is the one among kCgbHeights that minimises the sweep rows of
// the busiest warp, ceil(tiles / warps) x (h + 4): few tall tiles while many instances iterate,
// short ones for the last few. Every block computes the same plan from the same statuses.
template <class Pick>
__device__ __forceinline__ int cgb_prefix(const CgBatchArgs& a, const CgBInst* sh, long long* pref,
                                          int* h_out, Pick pick) {
    static_assert(CGB_MAX_INST <= 64, "two instances per lane");
    const int ninst = a.ninst;
    if (threadIdx.x < 32) {
        const int l = threadIdx.x;
        int h = a.rows;
        if (a.order != 0 && a.rows == 0) {
            const long long W = (long long)gridDim.x * CGB_NW;
            int hl = kCgbHeights[l % kCgbNHeights];
            long long tiles = 0;
            for (int li = 0; li < ninst; ++li)
                if (pick(sh[li])) tiles += (long long)sh[li].strips * ((sh[li].ny + hl - 1) / hl);
            long long cost = ((tiles + W - 1) / W) * (hl + 4);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {  // lowest cost, then the taller tile: one answer in all lanes
                const long long oc = __shfl_xor_sync(0xffffffffu, cost, o);
                const int oh = __shfl_xor_sync(0xffffffffu, hl, o);
                if (oc < cost || (oc == cost && oh > hl)) {
                    cost = oc;
                    hl = oh;
                }
            }
            h = hl;
        }
        auto units = [&](const CgBInst& S) -> long long {
            return (a.order == 0) ? (long long)S.strips * S.ny : (long long)S.strips * ((S.ny + h - 1) / h);
        };
        const long long u0 = (l < ninst && pick(sh[l])) ? units(sh[l]) : 0;
        const long long u1 = (l + 32 < ninst && pick(sh[l + 32])) ? units(sh[l + 32]) : 0;
        long long s0 = u0, s1 = u1;  // inclusive scans over the lanes
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long y0 = __shfl_up_sync(0xffffffffu, s0, o);
            const long long y1 = __shfl_up_sync(0xffffffffu, s1, o);
            if (l >= o) {
                s0 += y0;
                s1 += y1;
            }
        }
        const long long first = __shfl_sync(0xffffffffu, s0, 31);  // instances 0 .. 31
        if (l < ninst) pref[l] = s0 - u0;
        if (l + 32 < ninst) pref[l + 32] = first + s1 - u1;
        if (l == 31) pref[ninst] = first + s1;
        if (l == 0) *h_out = h;
    }
    __syncthreads();
    return *h_out;
}

// This warp's share of the phase as segments f(li, sx, r0, r1), in increasing unit number; h: the
// phase's tile height (order 1).
template <class F>
__device__ __forceinline__ void cgb_segments(const CgBatchArgs& a, const CgBInst* sh,
                                             const long long* pref, int h, F&& f) {
    constexpr int NW = CGB_NW;
    const long long nw = (long long)gridDim.x * NW;
    const long long g = (long long)blockIdx.x * NW + (threadIdx.x >> 5);
    const long long T = pref[a.ninst];
    if (a.order != 0) {
        int li = 0;
        for (long long j = g; j < T; j += nw) {
            while (pref[li + 1] <= j) ++li;
            const int w = (int)(j - pref[li]);
            const int sx = w % sh[li].strips;
            const int r0 = (w / sh[li].strips) * h;
            f(li, sx, r0, min(r0 + h, sh[li].ny));
        }
        return;
    }
    long long p = T * g / nw;
    const long long p1 = T * (g + 1) / nw;
    int li = 0;
    while (p < p1) {
        while (pref[li + 1] <= p) ++li;  // p only grows: li advances over the prefix once
        const int ny = sh[li].ny;
        const long long S = sh[li].strips;
        const long long q = p - pref[li];
        const int H = min(a.rows, ny);
        const long long band = min(q / (S * H), (long long)((ny - 1) / H));  // last band: ny - b0 rows
        const int b0 = (int)band * H;
        const int h = min(H, ny - b0);
        const long long t = q - band * S * H;  // within the band: strip t / h, row b0 + t % h
        const int sx = (int)(t / h);
        const int r0 = b0 + (int)(t - (long long)sx * h);
        long long e = p + (b0 + h - r0);  // end of this strip's piece of the band
        if (e > p1) e = p1;
        f(li, sx, r0, r0 + (int)(e - p));
        p = e;
    }
}

// One sweep over this warp's items: PH 0 the right-hand side (cg_rhs_segment), 1 the first
// iteration, 2 a later one (cg_iter_segment); NV sums per instance. Ends with the block's partials
// of every instance published in part_out.
template <int PH, int NV, int XM = kXSkip>
__device__ __forceinline__ void cgb_phase(const CgBatchArgs& a, const CgBInst* sh, const long long* pref,
                                          int h, double (*wsum)[CGB_MAX_INST][4], double* ring, int k,
                                          int dir, double* part_out) {
    constexpr int NW = CGB_NW;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int li = lane; li < a.ninst; li += 32)
#pragma unroll
        for (int c = 0; c < NV; ++c) wsum[wid][li][c] = 0.0;
    __syncwarp();
    const bool odd = (k & 1) != 0;
    cgb_segments(a, sh, pref, h, [&](int li, int sx, int r0, int r1) {
        const BatchInst& I = a.insts[a.inst0 + li];
        const CgSweepArgs g = cgb_args(a, I);
        CgScal s;
        s.cx = sh[li].cx;
        s.cy = sh[li].cy;
        s.diag = sh[li].diag;
        s.invdiag = sh[li].invdiag;
        s.alpha = sh[li].alpha;
        s.beta = sh[li].beta;
        s.alpha_prev = sh[li].alpha_prev;
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        if constexpr (PH == 0) {
            cg_rhs_segment(g, s, sx, r0, r1, dir, g.r[0], ring, acc);
        } else {
            const double* rk = odd ? g.r[1] : g.r[0];
            double* rk1 = odd ? g.r[0] : g.r[1];
            const double* pkm1 = odd ? g.p[0] : g.p[1];
            double* pk = odd ? g.p[1] : g.p[0];
            cg_iter_segment<PH == 1, XM>(g, s, sx, r0, r1, dir, rk, pkm1, rk1, pk, ring, acc);
        }
#pragma unroll
        for (int c = 0; c < NV; ++c)
            for (int o = 16; o > 0; o >>= 1) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
        if (lane == 0) {
#pragma unroll
            for (int c = 0; c < NV; ++c) wsum[wid][li][c] += acc[c];
        }
        __syncwarp();
    });
    __syncthreads();
    for (int q = threadIdx.x; q < a.ninst * NV; q += CGB_NT) {
        const int li = q / NV, c = q - li * NV;
        double v = 0.0;
        for (int w2 = 0; w2 < NW; ++w2) v += wsum[w2][li][c];
        part_out[((size_t)li * gridDim.x + blockIdx.x) * 4 + c] = v;
    }
}

// Sum of instance li's block partials (all blocks, fixed order); identical in every lane.
template <int NV>
__device__ __forceinline__ void cgb_span_sum(const double* part, int li, double (&v)[NV]) {
    lane_partial_sum<NV>(part + (size_t)li * gridDim.x * 4, (int)gridDim.x, v);
#pragma unroll
    for (int c = 0; c < NV; ++c)
        for (int o = 16; o > 0; o >>= 1) v[c] += __shfl_xor_sync(0xffffffffu, v[c], o);
}

static __global__ void __launch_bounds__(CGB_NT, MHD_CG_MIN_BLOCKS)
k_cg_batch(CgBatchArgs a) {
    constexpr int NW = CGB_NW;
    __shared__ CgBInst sh[CGB_MAX_INST];
    __shared__ long long pref[CGB_MAX_INST + 1];
    __shared__ int tile_h;  // the phase's tile height (order 1)
    __shared__ int sflag;
#if defined(__CUDA_ARCH__)
    extern __shared__ __align__(16) double cg_ring_mem[];
#else
    static double cg_ring_mem[kCgbSmemBytes / sizeof(double)];
#endif
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    double* const ring = cg_ring_mem + (size_t)wid * CG_RING * CG_SLOT;
    double (*const wsum)[CGB_MAX_INST][4] =
        reinterpret_cast<double (*)[CGB_MAX_INST][4]>(cg_ring_mem + kCgbRingBytes / sizeof(double));
    unsigned long long target = 0;
    const unsigned long long deadline = global_timer_ns() + (unsigned long long)(a.timeout_s * 1e9);
    double* const part0 = a.partials;
    double* const part1 = a.partials + (size_t)CGB_MAX_INST * gridDim.x * 4;
    auto part = [&](int ph) { return (ph & 1) ? part1 : part0; };
    int phase = 0;
    int dir = 1;
    auto barrier_or_quit = [&]() -> bool {
        if (grid_barrier(a.sync, target, deadline, &sflag)) return true;
        if (tid == 0 && blockIdx.x == 0)
            for (int li = 0; li < a.ninst; ++li)
                atomicOr(&a.insts[a.inst0 + li].st->flags, (unsigned)kStatusTimeout);
        return false;
    };

    // matrix of each instance's solve (the coefficient was set by this step's coefficients)
    for (int li = tid; li < a.ninst; li += CGB_NT) {
        const BatchInst& I = a.insts[a.inst0 + li];
        const double am = I.C->alpha;
        CgBInst& S = sh[li];
        S.cx = am / (I.D.dx * I.D.dx);
        S.cy = am / (I.D.dy * I.D.dy);
        S.diag = 1 + 2 * (S.cx + S.cy);
        S.invdiag = (S.diag == 0.0) ? 1.0 : 1.0 / S.diag;
        S.alpha = 0.0;
        S.alpha_prev = 0.0;
        S.beta = 0.0;
        S.products = 0;
        S.rr = 0.0;
        S.status = kCgActive;
        S.ny = I.D.ny;
        S.strips = I.cg_strips_x;
    }
    __syncthreads();
    auto is_active = [](const CgBInst& S) { return S.status == kCgActive; };

    // ---- right-hand side: r0 = b, p0 = z0 = b/d; |b|^2, b.z0, p0.A p0
    int h = cgb_prefix(a, sh, pref, &tile_h, is_active);
    cgb_phase<0, 3>(a, sh, pref, h, wsum, ring, 0, dir, part(phase));
    if (!barrier_or_quit()) return;
    for (int li = wid; li < a.ninst; li += NW) {
        double v[3];
        cgb_span_sum<3>(part(phase), li, v);
        if (lane == 0) {
            CgBInst& S = sh[li];
            const BatchInst& I = a.insts[a.inst0 + li];
            S.bb = v[0];
            S.absNew = v[1];
            S.thr = smax(I.tol * I.tol * S.bb, 2.2250738585072014e-308);
            if (!isfinite(S.bb)) S.status = kCgBreakdown;
            else if (S.bb == 0.0 || S.bb < S.thr) S.status = kCgZero;
            else if (I.max_iters <= 0) S.status = kCgCapped;
            S.pAp = v[2];
            S.alpha = (S.status == kCgActive) ? S.absNew / S.pAp : 0.0;
        }
    }
    ++phase;
    dir = -dir;
    __syncthreads();

    for (int k = 0;; ++k) {
        // ---- iteration k: p_k, q_k, x_{k+1}, r_{k+1}; r.r, r.z, z.Az, z.q_k
        h = cgb_prefix(a, sh, pref, &tile_h, is_active);
        // (all instances run iteration k together, so k's x mode is the same for all of them)
        if (k == 0) cgb_phase<1, 4, kXSkip>(a, sh, pref, h, wsum, ring, k, dir, part(phase));
        else if (cg_xmode(k) == kXSkip) cgb_phase<2, 4, kXSkip>(a, sh, pref, h, wsum, ring, k, dir, part(phase));
        else if (cg_xmode(k) == kXPairFirst)
            cgb_phase<2, 4, kXPairFirst>(a, sh, pref, h, wsum, ring, k, dir, part(phase));
        else cgb_phase<2, 4, kXPair>(a, sh, pref, h, wsum, ring, k, dir, part(phase));
        if (!barrier_or_quit()) return;
        int active = 0;
        for (int li = wid; li < a.ninst; li += NW) {
            if (sh[li].status != kCgActive) continue;
            double v[4];
            cgb_span_sum<4>(part(phase), li, v);
            if (lane == 0) {
                CgBInst& S = sh[li];
                S.products += 1;
                S.rr = v[0];
                if (!isfinite(v[0]) || !isfinite(S.alpha)) S.status = kCgBreakdown;
                else if (v[0] < S.thr) S.status = kCgConverged;
                else if (S.products >= a.insts[a.inst0 + li].max_iters) S.status = kCgCapped;
                else {
                    const double absOld = S.absNew;
                    S.absNew = v[1];
                    S.beta = S.absNew / absOld;
                    S.pAp = v[2] + 2.0 * S.beta * v[3] + S.beta * S.beta * S.pAp;
                    if (!(S.pAp > 0.0)) {
                        S.status = kCgBreakdown;
                    } else {
                        S.alpha_prev = S.alpha;
                        S.alpha = S.absNew / S.pAp;
                        active = 1;
                    }
                }
            }
        }
        ++phase;
        dir = -dir;
        if (!__syncthreads_or(active)) break;
    }

    // x = 0 for a vanished right-hand side (Eigen returns the zero vector) and on breakdown
    h = cgb_prefix(a, sh, pref, &tile_h, [](const CgBInst& S) {
        return S.status == kCgZero || S.status == kCgBreakdown || (S.status == kCgCapped && S.products == 0);
    });
    cgb_segments(a, sh, pref, h, [&](int li, int sx, int r0, int r1) {
        const BatchInst& I = a.insts[a.inst0 + li];
        const int nx = I.D.nx;
        const int i = sx * CG_W - CG_HALO + lane;
        if (lane >= CG_HALO && lane < CG_HALO + CG_W && i < nx)
            for (int j = r0; j < r1; ++j) I.x[(size_t)j * nx + i] = 0.0;
    });
    // solutions whose last iteration was even (an odd number of products) still lack that
    // iteration's alpha_k p_k (x moves every second iteration, see mhd_cg_sweep.cuh)
    __syncthreads();  // every warp is done with the prefix above
    h = cgb_prefix(a, sh, pref, &tile_h, [](const CgBInst& S) {
        return (S.status == kCgConverged || S.status == kCgCapped) && (S.products & 1) == 1;
    });
    cgb_segments(a, sh, pref, h, [&](int li, int sx, int r0, int r1) {
        const BatchInst& I = a.insts[a.inst0 + li];
        const CgBInst& S = sh[li];
        const double* pl = ((S.products - 1) & 1) ? I.p[1] : I.p[0];
        const int nx = I.D.nx;
        const int i = sx * CG_W - CG_HALO + lane;
        if (lane >= CG_HALO && lane < CG_HALO + CG_W && i < nx)
            for (int j = r0; j < r1; ++j) {
                const size_t g = (size_t)j * nx + i;
                I.x[g] = (S.products == 1) ? S.alpha * pl[g] : fma(S.alpha, pl[g], I.x[g]);
            }
    });
    if (blockIdx.x == 0) {
        for (int li = tid; li < a.ninst; li += CGB_NT) {
            const BatchInst& I = a.insts[a.inst0 + li];
            const CgBInst& S = sh[li];
            I.st->cg_products[a.solve_index] = S.products;
            I.st->cg_products_sum[a.solve_index] += S.products;
            I.st->cg_last_rr[a.solve_index] = (S.bb > 0.0) ? S.rr / S.bb : 0.0;
            if (a.prods_rec)
                a.prods_rec[((size_t)(a.inst0 + li) * a.rec_stride + I.C->cur) * 2 + a.solve_index] =
                    S.products;
            if (S.status == kCgBreakdown)
                atomicOr(&I.st->flags, (unsigned)(kStatusCgBreakdown | kStatusNonFinite));
            else if (S.status == kCgCapped)
                atomicOr(&I.st->flags, (unsigned)kStatusCgNotConverged);
        }
    }
}

}  // namespace mhd
