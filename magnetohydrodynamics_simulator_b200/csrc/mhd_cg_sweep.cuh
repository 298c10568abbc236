// Matrix-free conjugate gradient on the corner nodes as a persistent, cooperatively launched warp
// sweep (reference: solvers.hpp:404-489 with Eigen's ConjugateGradient defaults -- x0 = 0, Jacobi
// scaling by the constant diagonal d, stop when |r|^2 < max(tol^2 |b|^2, DBL_MIN), at most
// max_iters matrix-vector products).
//
// Each warp owns a strip of CG_W = 28 corner columns and a segment of rows; its 32 lanes hold the
// strip and two halo columns on each side. 5-point products are formed from register windows over
// rows (y neighbours) and shuffles (x neighbours); rows are prefetched into a per-warp shared-memory
// ring with cp.async. One sweep per iteration (after the right-hand-side sweep):
//   p_k = z_k + beta_k p_{k-1}; q_k = A p_k; r_{k+1} = r_k - alpha_k q_k; z_{k+1} = r_{k+1}/d;
//   partials r.r, r.z, z.Az, z.q_k (reads r_k, p_{k-1}; writes r_{k+1}, p_k).
// The solution moves every second iteration: odd k also forms
//   x_{k+1} = (x_{k-1} + alpha_{k-1} p_{k-1}) + alpha_k p_k
// from the p_{k-1} the sweep reads anyway -- the two updates of a one-per-iteration CG, in the same
// order -- so even iterations neither read nor write x (32 instead of 48 bytes per cell). A solve
// that stops after an even iteration adds its last alpha_k p_k in one elementwise pass.
// The next step length needs p_{k+1}.A p_{k+1}; with p_{k+1} = z_{k+1} + beta p_k and A symmetric
// it is z.Az + 2 beta z.q_k + beta^2 p_k.q_k, all known after this sweep, so no second sweep over
// the vectors is needed. In exact arithmetic these are Eigen's iterates; the step lengths differ
// from a two-sweep CG by rounding only. r and p are double-buffered (a sweep reads one copy's halo
// rows and writes the other). Consecutive sweeps run their rows in opposite directions, so each
// starts on the rows the previous one touched last (still in L2). Partial sums are reduced in a
// fixed order (lane tree, warp order, block order), identically in every block, so every block
// takes the same decisions and the result is deterministic. Grid-wide waits spin with a
// wall-clock limit (grid_barrier).
#pragma once

#include "mhd_kernels.cuh"

namespace mhd {

#ifndef MHD_CGS_NT
#define MHD_CGS_NT 512
#endif
constexpr int CGS_NT = MHD_CGS_NT;  // threads per block (16 warps)
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
    // a subdomain's interior inside extended planes (the kSub forms of the segment sweeps): strips
    // start at column col0, and columns from col_end on are not owned
    int col0, col_end;
};

struct CgScal {
    double invdiag, beta, alpha;
    double cx, cy, diag;
    double alpha_prev;  // alpha_{k-1} (odd iterations fold its update of x into theirs)
};

// How an iteration's sweep treats the solution x (see the header comment).
enum CgXMode : int {
    kXSkip = 0,      // even k: x neither read nor written
    kXPairFirst = 1, // k = 1: x_2 = alpha_0 p_0 + alpha_1 p_1 (x_0 = 0 is not read)
    kXPair = 2,      // odd k >= 3: x_{k+1} = (x_{k-1} + alpha_{k-1} p_{k-1}) + alpha_k p_k
};
__device__ __forceinline__ int cg_xmode(long long k) {
    return (k & 1) == 0 ? kXSkip : (k == 1 ? kXPairFirst : kXPair);
}

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

// Per-warp ring of prefetched rows in shared memory. A slot holds, for one row, up to 3 vectors at
// the warp's 32 columns (lane l's element at v*32 + l). Every lane reads back only what it copied
// itself, so cp.async.wait_group alone orders the accesses.
constexpr int CG_RING = 8;    // row slots per warp (power of two)
constexpr int CG_SLOT = 96;   // doubles per slot (768 bytes, 16-byte multiple)
constexpr int CG_HALO = 2;    // halo lanes on each side
constexpr int CG_W = 32 - 2 * CG_HALO;  // output columns per warp: lanes 2..29
constexpr size_t kCgRingBytes = (size_t)(CGS_NT / 32) * CG_RING * CG_SLOT * sizeof(double);

// Right-hand-side sweep over rows [r0w, r1w) of column strip sx: r0 = b = eta J_z(B) (written to
// r0), p0 = z0 = b/d, partials |b|^2, b.z0, p0.A p0 (acc[0..2]). Lane l holds corner column
// c0 - 2 + l; lanes 2..29 own the results. Sweep row k (k = 0 is the row behind the first one) sits
// in slot k % CG_RING.
template <bool kSub = false>
__device__ __forceinline__ void cg_rhs_segment(const CgSweepArgs& a, const CgScal& s, int sx, int r0w,
                                               int r1w, int dir, double* r0, double* ring,
                                               double (&acc)[4]) {
    const int lane = threadIdx.x & 31;
    const int nx = a.D.nx, ny = a.D.ny;
    const int c0 = (kSub ? a.col0 : 0) + sx * CG_W;
    if (r0w >= r1w) return;
    const int i = c0 - CG_HALO + lane;
    const bool owner = lane >= CG_HALO && lane < CG_HALO + CG_W && i < (kSub ? a.col_end : nx);
    const int iw = wrap(i, nx);
    const double idx = 1.0 / a.D.dx, idy = 1.0 / a.D.dy;
    const int jfirst = (dir > 0) ? r0w : r1w - 1;
    const int nrows = r1w - r0w;
    auto rowp = [&](int j) -> size_t { return (size_t)wrap(j, ny) * nx; };
    auto slot = [&](int k) { return ring + (unsigned)(k & (CG_RING - 1)) * CG_SLOT; };
    // copy sweep row k (grid row jfirst + (k-1) dir) into its slot and commit one group
    auto issue = [&](int k) {
        if (k <= nrows + 1) {
            double* sl = slot(k);
            const int j = jfirst + (k - 1) * dir;
            const size_t rp = rowp(j);
            const size_t rb = rowp(j - 1);
            cp_async8(&sl[lane], &a.byf[rp + iw]);
            cp_async8(&sl[32 + lane], &a.bxf[rp + iw]);
            cp_async8(&sl[64 + lane], &a.bxf[rb + iw]);
        }
        cp_async_commit();
    };
    // b and p = b/d of sweep row k (lane 0's b is never used: its left neighbour is not loaded)
    auto compute = [&](int k, double& p_own, double& r_own) {
        const double* sl = slot(k);
        const double by = sl[lane];
        const double byl = __shfl_up_sync(0xffffffffu, by, 1);
        const double b = corner_rhs(a.D, idx, idy, by, byl, sl[32 + lane], sl[64 + lane]);
        r_own = b;
        p_own = __dmul_rn(s.invdiag, b);
    };
#pragma unroll
    for (int k = 0; k < CG_RING; ++k) issue(k);
    cp_async_wait<CG_RING - 3>();  // rows 0, 1, 2 have landed
    double pb, pc, pa, rc, ra, dr;
    compute(0, pb, dr);
    compute(1, pc, rc);
    compute(2, pa, ra);
    (void)dr;
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
            acc[0] += rc * rc;
            acc[1] += rc * pc;
            acc[2] += pc * q;
            r0[g] = rc;
        }
        if (t == nrows - 1) break;
        g += gstep;
        // row t+3 (j + 2dir) enters the window
        cp_async_wait<CG_RING - 3>();
        double pn, rn;
        compute(t + 3, pn, rn);
        pb = pc; pc = pa; pa = pn;
        rc = ra; ra = rn;
    }
    cp_async_wait<0>();  // leave no copy in flight into the ring
}

// A subdomain's 3 x 3 neighbourhood for sweeps that read the cells around its interior straight
// from the neighbours' interiors instead of its own halo ring (subdomains of one process, on one
// device): entry a * 3 + b is the subdomain dy = a - 1, dx = b - 1 away (periodic; 4 is itself).
// A cell west of the interior lies in the west neighbour's last columns, a corner cell in the
// diagonal neighbour's corner; cells more than `halo` away are clamped to the ring (never used).
struct CgSubNeighbours {
    const double* r[2][9];  // the neighbours' r[0], r[1] of the single-sweep solve
    const double* p[2][9];  // ... and p[0], p[1]
    int nxe[9];             // their extended row pitch
    int nx, ny;             // this subdomain's interior
    int nx_w, ny_s;         // interior columns of the west neighbours, rows of the south ones
    int halo;               // ring width of the extended planes
};

// One CG iteration k over rows [r0w, r1w) of column strip sx (the sweep of the header comment).
// FIRST: k = 0, p_0 = z_0 (p_{-1} is not read). XM: the iteration's CgXMode. acc[0..3] receive r.r, r.z, z.Az, z.q_k of
// the owned cells. Sweep row t holds grid row jfirst + (t - 2) dir, t = 0 .. nrows + 3; at sweep
// row t the warp forms p_k of row t, q_k, r_{k+1}, z_{k+1} of row t-1 and A z_{k+1} and the outputs
// of row t-2. Row t is copied into slot t % CG_RING by the end of sweep row t - 6.
// kNb (with kSub): r_k and p_{k-1} are read from the neighbourhood nb (buffers rsel and psel of
// each neighbour) rather than from this subdomain's rings; the results are the same.
template <bool FIRST, int XM, bool kSub = false, bool kNb = false>
__device__ __forceinline__ void cg_iter_segment(const CgSweepArgs& a, const CgScal& s, int sx, int r0w,
                                                int r1w, int dir, const double* rk, const double* pkm1,
                                                double* rk1, double* pk, double* ring,
                                                double (&acc)[4], const CgSubNeighbours* nb = nullptr,
                                                int rsel = 0, int psel = 0) {
    const int lane = threadIdx.x & 31;
    const int nx = a.D.nx, ny = a.D.ny;
    const int c0 = (kSub ? a.col0 : 0) + sx * CG_W;
    if (r0w >= r1w) return;
    const int i = c0 - CG_HALO + lane;
    const bool owner = lane >= CG_HALO && lane < CG_HALO + CG_W && i < (kSub ? a.col_end : nx);
    const int iw = wrap(i, nx);
    const int jfirst = (dir > 0) ? r0w : r1w - 1;
    const int total = (r1w - r0w) + 4;
    auto slot = [&](int t) { return ring + (unsigned)(t & (CG_RING - 1)) * CG_SLOT; };
    // kNb: this lane's column in the neighbourhood (clamped to the ring), fixed for the strip
    int nb_b = 1, nb_si = 0;
    if constexpr (kNb) {
        const int ii = min(max(i - nb->halo, -nb->halo), nb->nx + nb->halo - 1);
        nb_b = (ii < 0) ? 0 : (ii >= nb->nx ? 2 : 1);
        nb_si = (nb_b == 0) ? nb->nx_w + ii : (nb_b == 2 ? ii - nb->nx : ii);
    }
    auto issue = [&](int t) {
        if (t < total) {
            double* sl = slot(t);
            const int j = jfirst + (t - 2) * dir;
            const size_t rp = (size_t)wrap(j, ny) * nx + iw;
            if constexpr (kNb) {
                const int jj = min(max(j - nb->halo, -nb->halo), nb->ny + nb->halo - 1);
                const int na = (jj < 0) ? 0 : (jj >= nb->ny ? 2 : 1);
                const int sj = (na == 0) ? nb->ny_s + jj : (na == 2 ? jj - nb->ny : jj);
                const int e = na * 3 + nb_b;
                const size_t q = (size_t)(sj + nb->halo) * nb->nxe[e] + (nb_si + nb->halo);
                cp_async8(&sl[lane], &nb->r[rsel][e][q]);
                if constexpr (!FIRST) cp_async8(&sl[32 + lane], &nb->p[psel][e][q]);
            } else {
                cp_async8(&sl[lane], &rk[rp]);
                if constexpr (!FIRST) cp_async8(&sl[32 + lane], &pkm1[rp]);
            }
            if constexpr (XM == kXPair) cp_async8(&sl[64 + lane], &a.x[rp]);  // read by owner lanes only
        }
        cp_async_commit();
    };
#pragma unroll
    for (int t = 0; t < CG_RING - 2; ++t) issue(t);
    double p_a = 0.0, p_b = 0.0;       // p_k of rows t-2, t-1
    double q_o = 0.0;                  // q_k of row t-2
    double r_o = 0.0, z_o = 0.0;       // r_{k+1}, z_{k+1} of row t-2
    double z_a = 0.0;                  // z_{k+1} of row t-3
    size_t g = (size_t)jfirst * nx + i;  // owner lanes' element of the output row
    const long long gstep = (long long)dir * nx;
    for (int t = 0; t < total; ++t) {
        cp_async_wait<CG_RING - 3>();  // row t has landed (rows t+1 .. t+5 may be in flight)
        const double* sl = slot(t);
        double p_c;
        if constexpr (FIRST) p_c = __dmul_rn(s.invdiag, sl[lane]);
        else p_c = cg_dir(s.invdiag, sl[lane], s.beta, sl[32 + lane]);
        double q_b = 0.0, r_b = 0.0, z_b = 0.0;
        if (t >= 2) {
            // q_k, r_{k+1}, z_{k+1} of row t-1
            const double pl = __shfl_up_sync(0xffffffffu, p_b, 1);
            const double pr = __shfl_down_sync(0xffffffffu, p_b, 1);
            const double p_lo = (dir > 0) ? p_a : p_c;
            const double p_hi = (dir > 0) ? p_c : p_a;
            q_b = stencil(p_lo, pl, p_b, pr, p_hi, s);
            r_b = slot(t - 1)[lane] - s.alpha * q_b;
            z_b = __dmul_rn(s.invdiag, r_b);
        }
        if (t >= 4) {
            // A z_{k+1} and the outputs of row t-2
            const double zl = __shfl_up_sync(0xffffffffu, z_o, 1);
            const double zr = __shfl_down_sync(0xffffffffu, z_o, 1);
            const double z_lo = (dir > 0) ? z_a : z_b;
            const double z_hi = (dir > 0) ? z_b : z_a;
            const double az = stencil(z_lo, zl, z_o, zr, z_hi, s);
            if (owner) {
                if constexpr (XM != kXSkip) {
                    const double* so = slot(t - 2);  // p_{k-1} (and x_{k-1}) of the output row
                    const double xm = (XM == kXPairFirst)
                                          ? s.alpha_prev * so[32 + lane]
                                          : fma(s.alpha_prev, so[32 + lane], so[64 + lane]);
                    a.x[g] = fma(s.alpha, p_a, xm);
                }
                rk1[g] = r_o;
                pk[g] = p_a;
                acc[0] += r_o * r_o;
                acc[1] += r_o * z_o;
                acc[2] += z_o * az;
                acc[3] += z_o * q_o;
            }
            g += gstep;
        }
        p_a = p_b; p_b = p_c;
        q_o = q_b;
        z_a = z_o;
        r_o = r_b; z_o = z_b;
        issue(t + CG_RING - 2);  // into the slot of row t-2, no longer read
    }
    cp_async_wait<0>();  // leave no copy in flight into the ring
}

// Block-reduce NV partial sums (fixed order) and publish them in this block's slot.
template <int NV>
__device__ __forceinline__ void publish(double (&acc)[4], double* slot, double* red) {
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
    s.alpha_prev = 0.0;
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

    // ---- right-hand side: r0 = b, p0 = z0 = b/d; |b|^2, b.z0, p0.A p0
    {
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        for (int w = wfirst; w < a.nwarps; w += wstride) {
            const int sx = w % a.strips_x, r0w = (w / a.strips_x) * a.seg_h;
            cg_rhs_segment(a, s, sx, r0w, min(r0w + a.seg_h, a.D.ny), dir, a.r[0], ring, acc);
        }
        publish<3>(acc, part(phase) + (size_t)blockIdx.x * 4, red);
    }
    if (!barrier_or_quit()) return;
    double sums[4];
    reduce_partials<3>(part(phase), G, sums, scal);
    ++phase;
    dir = -dir;
    const double bb = sums[0];
    double absNew = sums[1];
    double pAp = sums[2];
    const double threshold = smax(a.tol * a.tol * bb, 2.2250738585072014e-308);
    long long products = 0;
    const bool zero_solution = (bb == 0.0) || (bb < threshold);
    bool breakdown = !isfinite(bb);
    bool converged = zero_solution;
    double rr_final = 0.0;
    long long k_last = -1;     // the last iteration swept
    double alpha_last = 0.0;   // its step length

    if (!zero_solution && !breakdown) {
        s.alpha = absNew / pAp;
        for (long long k = 0; k < a.max_iters; ++k) {
            k_last = k;
            alpha_last = s.alpha;
            const bool odd = (k & 1) != 0;
            const double* rk = odd ? a.r[1] : a.r[0];
            double* rk1 = odd ? a.r[0] : a.r[1];
            const double* pkm1 = odd ? a.p[0] : a.p[1];
            double* pk = odd ? a.p[1] : a.p[0];
            {
                double acc[4] = {0.0, 0.0, 0.0, 0.0};
                for (int w = wfirst; w < a.nwarps; w += wstride) {
                    const int sx = w % a.strips_x, r0w = (w / a.strips_x) * a.seg_h;
                    const int r1w = min(r0w + a.seg_h, a.D.ny);
                    switch (cg_xmode(k)) {
                        case kXSkip:
                            if (k == 0)
                                cg_iter_segment<true, kXSkip>(a, s, sx, r0w, r1w, dir, rk, pkm1, rk1, pk, ring, acc);
                            else
                                cg_iter_segment<false, kXSkip>(a, s, sx, r0w, r1w, dir, rk, pkm1, rk1, pk, ring, acc);
                            break;
                        case kXPairFirst:
                            cg_iter_segment<false, kXPairFirst>(a, s, sx, r0w, r1w, dir, rk, pkm1, rk1, pk, ring, acc);
                            break;
                        default:
                            cg_iter_segment<false, kXPair>(a, s, sx, r0w, r1w, dir, rk, pkm1, rk1, pk, ring, acc);
                    }
                }
                publish<4>(acc, part(phase) + (size_t)blockIdx.x * 4, red);
            }
            if (!barrier_or_quit()) return;
            double v[4];
            reduce_partials<4>(part(phase), G, v, scal);
            ++phase;
            dir = -dir;
            ++products;
            const double rr = v[0];
            rr_final = rr;
            if (!isfinite(rr) || !isfinite(s.alpha)) { breakdown = true; break; }
            if (rr < threshold) { converged = true; break; }
            // next step: beta = r.z / r.z_old, p.Ap = z.Az + 2 beta z.q + beta^2 p.Ap
            const double absOld = absNew;
            absNew = v[1];
            s.beta = absNew / absOld;
            pAp = v[2] + 2.0 * s.beta * v[3] + s.beta * s.beta * pAp;
            if (!(pAp > 0.0)) { breakdown = true; break; }
            s.alpha_prev = s.alpha;
            s.alpha = absNew / pAp;
        }
    }
    if (!zero_solution && !breakdown && k_last >= 0 && cg_xmode(k_last) == kXSkip) {
        // the last iteration was even: add its alpha_k p_k (x_0 = 0 when it was the first)
        const double* pl = (k_last & 1) ? a.p[1] : a.p[0];
        const size_t n = (size_t)a.D.nx * a.D.ny;
        for (size_t g = (size_t)blockIdx.x * CGS_NT + tid; g < n; g += (size_t)G * CGS_NT)
            a.x[g] = (k_last == 0) ? alpha_last * pl[g] : fma(alpha_last, pl[g], a.x[g]);
    }
    if (zero_solution || breakdown || k_last < 0) {
        // x = 0 (Eigen returns the zero vector when b == 0, and x0 = 0 when no iteration may run);
        // on breakdown the status says so
        const int nx = a.D.nx, ny = a.D.ny;
        const size_t n = (size_t)nx * ny;
        for (size_t g = (size_t)blockIdx.x * CGS_NT + tid; g < n; g += (size_t)G * CGS_NT) a.x[g] = 0.0;
    }
    if (blockIdx.x == 0 && tid == 0) {
        a.st->cg_products[a.solve_index] = products;
        a.st->cg_products_sum[a.solve_index] += products;
        a.st->cg_last_rr[a.solve_index] = (bb > 0.0) ? rr_final / bb : 0.0;
        if (a.prods_out) a.prods_out[2 * a.C->cur + a.solve_index] = products;
        if (breakdown) atomicOr(&a.st->flags, (unsigned)(kStatusCgBreakdown | kStatusNonFinite));
        else if (!converged) atomicOr(&a.st->flags, (unsigned)kStatusCgNotConverged);
    }
}

}  // namespace mhd
