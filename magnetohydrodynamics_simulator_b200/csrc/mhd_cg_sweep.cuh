// Matrix-free conjugate gradient on the corner nodes as a persistent, cooperatively launched warp
// sweep (reference: solvers.hpp:404-489 with Eigen's ConjugateGradient defaults -- x0 = 0, Jacobi
// scaling by the constant diagonal, stop when |r|^2 < max(tol^2 |b|^2, DBL_MIN), at most max_iters
// matrix-vector products).
//
// Each warp owns a strip of 30 corner columns and a segment of rows; its 32 lanes hold the strip and
// one halo column on each side. The 5-point product is formed from a 3-row register window
// (y neighbours) and shuffles (x neighbours); rows are prefetched 8 deep into shared memory with
// cp.async. Per iteration:
//   phase A: p_k = r_k/d + beta p_{k-1} (rows j-1..j+1), q = A p_k, partial p.q          reads r, p
//   phase B: the same p_k and q; x += alpha p_k; r_{k+1} = r_k - alpha q; partial r.r, r.z;
//            writes x, r_{k+1}, p_k                                              reads r, p, x
// r and p are double-buffered (a phase reads one copy's halo and writes the other). Phases A and B
// sweep their rows in opposite directions, so each phase starts on the rows the previous phase
// touched last (still in L2). Partial sums are reduced in a fixed order (lane tree, warp order,
// block order), identically in every block, so every block takes the same decisions and the
// result is deterministic. Grid-wide waits spin with a wall-clock limit (grid_barrier).
#pragma once

#include "mhd_kernels.cuh"

namespace mhd {

constexpr int CGS_NT = 512;  // threads per block (16 warps)
#ifndef MHD_CG_MIN_BLOCKS
#define MHD_CG_MIN_BLOCKS 1      // blocks per SM (the prefetch lives in shared memory)
#endif

struct CgSweepArgs {
    Domain D;
    const StepCoeffs* C;
    const double* bxf;
    const double* byf;
    double* x;
    double* r[2];
    double* p[2];
    double* partials;  // [2][gridDim.x][4]
    CgSync* sync;
    DeviceStatus* st;
    long long* prods_out;
    int solve_index;
    int strips_x, seg_h, nwarps;
    long long max_iters;
    double tol;
    double timeout_s;
};

struct CgScal {
    double invdiag, beta, alpha;
    double cx, cy, diag;
};

// (A p) at a corner from its column window and x neighbours, summed in increasing column order
// for interior rows (bottom, left, centre, right, top) as the reference's compressed product.
__device__ __forceinline__ double stencil(double pb, double pl, double pc, double pr, double pt,
                                          const CgScal& s) {
    double acc = 0.0;
    acc += (-s.cy) * pb;
    acc += (-s.cx) * pl;
    acc += s.diag * pc;
    acc += (-s.cx) * pr;
    acc += (-s.cy) * pt;
    return acc;
}

__device__ __forceinline__ double cg_dir(double invdiag, double r, double beta, double p) {
    return __dadd_rn(__dmul_rn(invdiag, r), __dmul_rn(beta, p));
}

// eta * J_z(B*) at corner (col, j) (solvers.hpp:450-461); byl = byf(col-1, j); idx = 1/dx,
// idy = 1/dy (a multiplication by the hoisted reciprocal is within 1 ulp of the quotient).
__device__ __forceinline__ double corner_rhs(const Domain& D, double idx, double idy, double by,
                                             double byl, double bx, double bxb) {
    const double dBy_dx = (by - byl) * idx;
    const double dBx_dy = (bx - bxb) * idy;
    return D.eta * (dBy_dx - dBx_dy);
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

// Per-warp ring of prefetched rows in shared memory. A slot holds, for one row, up to 3 vectors at
// the warp's 32 columns (lane l's element at v*32 + l) and, in the right-hand-side phase, lane 0's
// extra face value at 96. Every lane reads back only what it copied itself, so
// cp.async.wait_group alone orders the accesses.
constexpr int CG_RING = 8;    // rows in flight per warp (power of two)
constexpr int CG_SLOT = 104;  // doubles per slot (832 bytes, 16-byte multiple)
constexpr int CG_W = 30;      // output columns per warp: lanes 1..30; lanes 0 and 31 are halo
constexpr size_t kCgRingBytes = (size_t)(CGS_NT / 32) * CG_RING * CG_SLOT * sizeof(double);

// One sweep over the warp's segment. PH: 0 = A0 (right-hand side, r0 = b, p0 = b/d),
// 1 = A_k (k >= 1), 2 = B_0, 3 = B_k. acc[] receives this lane's partial sums. Lane l holds corner
// column c0 - 1 + l; every lane does the same work and lanes 1..30 own the results. Row k of the
// sweep (k = 0 is the row behind the first one) is copied into slot k % CG_RING, CG_RING - 3 rows
// before it enters the 3-row stencil window.
template <int PH>
__device__ __forceinline__ void cg_sweep_segment(const CgSweepArgs& a, const CgScal& s, int w,
                                                 int dir, const double* rk, const double* pkm1,
                                                 double* rk1, double* pk, double* ring,
                                                 double (&acc)[3]) {
    const int lane = threadIdx.x & 31;
    const int nx = a.D.nx, ny = a.D.ny;
    const int sx = w % a.strips_x, sy = w / a.strips_x;
    const int c0 = sx * CG_W;
    const int r0 = sy * a.seg_h;
    const int r1 = min(r0 + a.seg_h, ny);
    if (r0 >= r1) return;
    const int i = c0 - 1 + lane;
    const bool owner = lane >= 1 && lane <= CG_W && i < nx;
    const int iw = wrap(i, nx);
    const int iwl = wrap(i - 1, nx);  // lane 0's left neighbour (right-hand-side phase)
    const double idx = 1.0 / a.D.dx, idy = 1.0 / a.D.dy;
    const int jfirst = (dir > 0) ? r0 : r1 - 1;
    const int jlast = (dir > 0) ? r1 - 1 : r0;
    const int nrows = r1 - r0;
    auto rowp = [&](int j) -> size_t { return (size_t)wrap(j, ny) * nx; };
    auto slot = [&](int k) { return ring + (unsigned)(k & (CG_RING - 1)) * CG_SLOT; };

    // copy sweep row k (grid row jfirst + (k-1) dir) into its slot and commit one group
    auto issue = [&](int k) {
        if (k <= nrows + 1) {
            double* sl = slot(k);
            const int j = jfirst + (k - 1) * dir;
            const size_t rp = rowp(j);
            if constexpr (PH == 0) {
                const size_t rb = rowp(j - 1);
                cp_async8(&sl[lane], &a.byf[rp + iw]);
                cp_async8(&sl[32 + lane], &a.bxf[rp + iw]);
                cp_async8(&sl[64 + lane], &a.bxf[rb + iw]);
                if (lane == 0) cp_async8(&sl[96], &a.byf[rp + iwl]);
            } else {
                cp_async8(&sl[lane], &rk[rp + iw]);
                if constexpr (PH != 2) cp_async8(&sl[32 + lane], &pkm1[rp + iw]);
                if constexpr (PH == 3) cp_async8(&sl[64 + lane], &a.x[rp + iw]);
            }
        }
        cp_async_commit();
    };
    // p, r and x at this lane's column of sweep row k, from its slot
    auto compute = [&](int k, double& p_own, double& r_own, double& x_own) {
        const double* sl = slot(k);
        if constexpr (PH == 0) {
            const double by = sl[lane];
            double byl = __shfl_up_sync(0xffffffffu, by, 1);
            if (lane == 0) byl = sl[96];
            const double b = corner_rhs(a.D, idx, idy, by, byl, sl[32 + lane], sl[64 + lane]);
            r_own = b;
            p_own = __dmul_rn(s.invdiag, b);
        } else if constexpr (PH == 2) {
            r_own = sl[lane];
            p_own = __dmul_rn(s.invdiag, r_own);
        } else {
            r_own = sl[lane];
            p_own = cg_dir(s.invdiag, r_own, s.beta, sl[32 + lane]);
        }
        if constexpr (PH == 3) x_own = sl[64 + lane];
        else x_own = 0.0;
    };

#pragma unroll
    for (int k = 0; k < CG_RING; ++k) issue(k);
    cp_async_wait<CG_RING - 3>();  // rows 0, 1, 2 have landed
    // window: p at rows j - dir (behind), j (current), j + dir (ahead)
    double pb, pc, pa, rc, ra, xc, xa, dr, dx_;
    compute(0, pb, dr, dx_);
    compute(1, pc, rc, xc);
    compute(2, pa, ra, xa);
    (void)dr;
    (void)dx_;
    size_t g = (size_t)jfirst * nx + i;  // owner lanes' element of the current row
    const long long gstep = (long long)dir * nx;
    for (int t = 0;; ++t) {
        issue(t + CG_RING);  // slot of row t, which entered the window three rows ago
        const double pl = __shfl_up_sync(0xffffffffu, pc, 1);
        const double pr = __shfl_down_sync(0xffffffffu, pc, 1);
        const double p_lo = (dir > 0) ? pb : pa;  // row j-1
        const double p_hi = (dir > 0) ? pa : pb;  // row j+1
        const double q = stencil(p_lo, pl, pc, pr, p_hi, s);
        if (owner) {
            if constexpr (PH == 0) {
                acc[0] += rc * rc;
                acc[1] += rc * pc;
                acc[2] += pc * q;
                rk1[g] = rc;  // r0 = b
            } else if constexpr (PH == 1) {
                acc[0] += pc * q;
            } else {
                const double xv = (PH == 2) ? s.alpha * pc : xc + s.alpha * pc;
                const double rnew = rc - s.alpha * q;
                a.x[g] = xv;
                rk1[g] = rnew;
                pk[g] = pc;
                acc[0] += rnew * rnew;
                acc[1] += rnew * __dmul_rn(s.invdiag, rnew);
            }
        }
        if (t == nrows - 1) break;
        g += gstep;
        // row t+3 (j + 2dir) enters the window
        cp_async_wait<CG_RING - 3>();
        double pn, rn, xn;
        compute(t + 3, pn, rn, xn);
        pb = pc; pc = pa; pa = pn;
        rc = ra; ra = rn;
        xc = xa; xa = xn;
    }
    (void)jlast;
    cp_async_wait<0>();  // leave no copy in flight into the ring
}

// Block-reduce NV partial sums (fixed order) and publish them in this block's slot.
template <int NV>
__device__ __forceinline__ void publish(double (&acc)[3], double* slot, double* red) {
#pragma unroll
    for (int k = 0; k < NV; ++k)
        for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
    const int wi = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) red[wi * 4 + k] = acc[k];
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double sum = 0.0;
        for (int q = 0; q < CGS_NT / 32; ++q) sum += red[q * 4 + threadIdx.x];
        slot[threadIdx.x] = sum;
    }
}

static __global__ void __launch_bounds__(CGS_NT, MHD_CG_MIN_BLOCKS)
k_cg_sweep(CgSweepArgs a) {
    __shared__ double red[CGS_NT / 32 * 4];
    __shared__ double scal[8];
    __shared__ int sflag;
#if defined(__CUDA_ARCH__)
    extern __shared__ __align__(16) double cg_ring_mem[];
#else
    // host compilation of the kernel sources (single-block logic tests): one shared copy
    static double cg_ring_mem[(CGS_NT / 32) * CG_RING * CG_SLOT];
#endif
    double* const ring = cg_ring_mem + (size_t)(threadIdx.x >> 5) * CG_RING * CG_SLOT;
    const int tid = threadIdx.x;
    const int G = gridDim.x;
    const int warps_per_block = CGS_NT / 32;
    const int wfirst = blockIdx.x * warps_per_block + (tid >> 5);
    const int wstride = G * warps_per_block;
    CgScal s;
    const double alpha_m = a.C->alpha;
    s.cx = alpha_m / (a.D.dx * a.D.dx);
    s.cy = alpha_m / (a.D.dy * a.D.dy);
    s.diag = 1 + 2 * (s.cx + s.cy);
    s.invdiag = (s.diag == 0.0) ? 1.0 : 1.0 / s.diag;
    s.beta = 0.0;
    s.alpha = 0.0;
    unsigned long long target = 0;
    const unsigned long long deadline =
        global_timer_ns() + (unsigned long long)(a.timeout_s * 1e9);
    double* const part0 = a.partials;
    double* const part1 = a.partials + (size_t)G * 4;
    // (conditional selects instead of indexing small arrays by a runtime value, which would put
    // them in local memory)
    auto part = [&](int ph) { return (ph & 1) ? part1 : part0; };
    int phase = 0;
    int dir = 1;

    auto barrier_or_quit = [&]() -> bool {
        if (grid_barrier(a.sync, target, deadline, &sflag)) return true;
        if (tid == 0 && blockIdx.x == 0) atomicOr(&a.st->flags, (unsigned)kStatusTimeout);
        return false;
    };

    // ---- phase A0
    {
        double acc[3] = {0.0, 0.0, 0.0};
        for (int w = wfirst; w < a.nwarps; w += wstride)
            cg_sweep_segment<0>(a, s, w, dir, nullptr, nullptr, a.r[0], nullptr, ring, acc);
        publish<3>(acc, part(phase) + (size_t)blockIdx.x * 4, red);
    }
    if (!barrier_or_quit()) return;
    double sums[3];
    reduce_partials<3>(part(phase), G, sums, scal);
    ++phase;
    dir = -dir;
    const double bb = sums[0];
    double absNew = sums[1];
    double pq = sums[2];
    const double threshold = smax(a.tol * a.tol * bb, 2.2250738585072014e-308);
    long long products = 0;
    const bool zero_solution = (bb == 0.0) || (bb < threshold);
    bool breakdown = !isfinite(bb);
    bool converged = zero_solution;
    double rr_final = 0.0;

    if (!zero_solution && !breakdown) {
        for (long long k = 0; k < a.max_iters; ++k) {
            const bool odd = (k & 1) != 0;
            const double* rk = odd ? a.r[1] : a.r[0];
            double* rk1 = odd ? a.r[0] : a.r[1];
            const double* pkm1 = odd ? a.p[0] : a.p[1];
            double* pk = odd ? a.p[1] : a.p[0];
            if (k > 0) {
                double acc[3] = {0.0, 0.0, 0.0};
                for (int w = wfirst; w < a.nwarps; w += wstride)
                    cg_sweep_segment<1>(a, s, w, dir, rk, pkm1, nullptr, nullptr, ring, acc);
                publish<1>(acc, part(phase) + (size_t)blockIdx.x * 4, red);
                if (!barrier_or_quit()) return;
                double v[1];
                reduce_partials<1>(part(phase), G, v, scal);
                ++phase;
                dir = -dir;
                pq = v[0];
            }
            s.alpha = absNew / pq;
            {
                double acc[3] = {0.0, 0.0, 0.0};
                for (int w = wfirst; w < a.nwarps; w += wstride) {
                    if (k == 0) cg_sweep_segment<2>(a, s, w, dir, rk, pkm1, rk1, pk, ring, acc);
                    else cg_sweep_segment<3>(a, s, w, dir, rk, pkm1, rk1, pk, ring, acc);
                }
                publish<2>(acc, part(phase) + (size_t)blockIdx.x * 4, red);
            }
            if (!barrier_or_quit()) return;
            double v2[2];
            reduce_partials<2>(part(phase), G, v2, scal);
            ++phase;
            dir = -dir;
            ++products;
            const double rr = v2[0];
            rr_final = rr;
            if (!isfinite(rr) || !isfinite(s.alpha)) { breakdown = true; break; }
            if (rr < threshold) { converged = true; break; }
            const double absOld = absNew;
            absNew = v2[1];
            s.beta = absNew / absOld;
        }
    }
    if (zero_solution || breakdown) {
        // x = 0 (Eigen returns the zero vector when b == 0); on breakdown the status says so
        const int nx = a.D.nx, ny = a.D.ny;
        const size_t n = (size_t)nx * ny;
        for (size_t g = (size_t)blockIdx.x * CGS_NT + tid; g < n; g += (size_t)G * CGS_NT) a.x[g] = 0.0;
    }
    if (blockIdx.x == 0 && tid == 0) {
        a.st->cg_products[a.solve_index] = products;
        a.st->cg_products_total += products;
        a.st->cg_last_rr[a.solve_index] = (bb > 0.0) ? rr_final / bb : 0.0;
        if (a.prods_out) a.prods_out[2 * a.C->cur + a.solve_index] = products;
        if (breakdown) atomicOr(&a.st->flags, (unsigned)(kStatusCgBreakdown | kStatusNonFinite));
        else if (!converged) atomicOr(&a.st->flags, (unsigned)kStatusCgNotConverged);
    }
}

}  // namespace mhd
