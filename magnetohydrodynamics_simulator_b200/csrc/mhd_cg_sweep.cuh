// Matrix-free conjugate gradient on the corner nodes as a persistent, cooperatively launched warp
// sweep (reference: solvers.hpp:404-489 with Eigen's ConjugateGradient defaults -- x0 = 0, Jacobi
// scaling by the constant diagonal, stop when |r|^2 < max(tol^2 |b|^2, DBL_MIN), at most max_iters
// matrix-vector products).
//
// Each warp owns a strip of 32 corner columns and a segment of rows; lane l holds column c0 + l and
// lanes 0 / 31 also evaluate the halo column on their side. The 5-point product is formed from a
// 3-row register window (y neighbours) and shuffles (x neighbours). Per iteration:
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

constexpr int CGS_NT = 512;  // threads per block (16 warps); one block per SM

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

// Raw loads of one row for the value of p at this lane's column and (edge lanes) the halo column:
// A0 reads 8 face values, A_k reads r and p (own + halo), B_0 reads r, B_k also reads x.
template <int N>
struct CgRaw {
    double v[N];
};
template <int PH>
constexpr int cg_raw_n() { return PH == 0 ? 8 : (PH == 3 ? 5 : 4); }

// One sweep over the warp's segment. PH: 0 = A0 (right-hand side, r0 = b, p0 = b/d),
// 1 = A_k (k >= 1), 2 = B_0, 3 = B_k. acc[] receives this lane's partial sums. The loads of a row
// are issued DEPTH rows before the row enters the stencil window.
template <int PH>
__device__ __forceinline__ void cg_sweep_segment(const CgSweepArgs& a, const CgScal& s, int w,
                                                 int dir, const double* rk, const double* pkm1,
                                                 double* rk1, double* pk, double (&acc)[3]) {
    constexpr int DEPTH = (PH == 0) ? 2 : 4;
    const int lane = threadIdx.x & 31;
    const int nx = a.D.nx, ny = a.D.ny;
    const int sx = w % a.strips_x, sy = w / a.strips_x;
    const int c0 = sx * 32;
    const int r0 = sy * a.seg_h;
    const int r1 = min(r0 + a.seg_h, ny);
    if (r0 >= r1) return;
    const int i = c0 + lane;
    const bool valid = i < nx;
    const int iw = wrap(i, nx);
    // halo column of the edge lanes: c0-1 for lane 0, c0+32 for lane 31
    const bool edge = (lane == 0) || (lane == 31);
    const int ih = wrap(lane == 0 ? c0 - 1 : c0 + 32, nx);
    const int ihl = wrap(lane == 0 ? c0 - 2 : c0 + 31, nx);  // left of the halo column (A0)
    const int il0 = wrap(c0 - 1, nx);                         // left of lane 0 (A0)
    const double idx = 1.0 / a.D.dx, idy = 1.0 / a.D.dy;
    auto rowp = [&](int j) -> size_t { return (size_t)wrap(j, ny) * nx; };

    using Raw = CgRaw<cg_raw_n<PH>()>;
    auto load_raw = [&](int j) {
        Raw q{};
        const size_t rp = rowp(j);
        if constexpr (PH == 0) {
            const size_t rb = rowp(j - 1);
            q.v[0] = __ldg(&a.byf[rp + iw]);
            q.v[1] = __ldg(&a.bxf[rp + iw]);
            q.v[2] = __ldg(&a.bxf[rb + iw]);
            q.v[3] = (lane == 0) ? __ldg(&a.byf[rp + il0]) : 0.0;
            q.v[4] = edge ? __ldg(&a.byf[rp + ih]) : 0.0;
            q.v[5] = edge ? __ldg(&a.byf[rp + ihl]) : 0.0;
            q.v[6] = edge ? __ldg(&a.bxf[rp + ih]) : 0.0;
            q.v[7] = edge ? __ldg(&a.bxf[rb + ih]) : 0.0;
        } else {
            q.v[0] = __ldcg(&rk[rp + iw]);
            q.v[2] = edge ? __ldcg(&rk[rp + ih]) : 0.0;
            if (PH != 2) {
                q.v[1] = __ldcg(&pkm1[rp + iw]);
                q.v[3] = edge ? __ldcg(&pkm1[rp + ih]) : 0.0;
            }
            if constexpr (PH == 3) q.v[4] = __ldcg(&a.x[rp + iw]);
        }
        return q;
    };
    // p (own column), p (halo column) and r (own column) of a row from its raw loads
    auto compute = [&](const Raw& q, double& p_own, double& p_halo, double& r_own) {
        if constexpr (PH == 0) {
            double byl = __shfl_up_sync(0xffffffffu, q.v[0], 1);
            if (lane == 0) byl = q.v[3];
            const double b = corner_rhs(a.D, idx, idy, q.v[0], byl, q.v[1], q.v[2]);
            r_own = b;
            p_own = __dmul_rn(s.invdiag, b);
            p_halo = edge ? __dmul_rn(s.invdiag, corner_rhs(a.D, idx, idy, q.v[4], q.v[5], q.v[6], q.v[7])) : 0.0;
        } else if (PH == 2) {
            r_own = q.v[0];
            p_own = __dmul_rn(s.invdiag, q.v[0]);
            p_halo = __dmul_rn(s.invdiag, q.v[2]);
        } else {
            r_own = q.v[0];
            p_own = cg_dir(s.invdiag, q.v[0], s.beta, q.v[1]);
            p_halo = cg_dir(s.invdiag, q.v[2], s.beta, q.v[3]);
        }
    };

    const int jfirst = (dir > 0) ? r0 : r1 - 1;
    const int jlast = (dir > 0) ? r1 - 1 : r0;
    const int nrows = r1 - r0;
    // window: p at rows j - dir (behind), j (current), j + dir (ahead); x of the current row
    double pb, pc, pa, hc, ha, rc, ra, xc = 0.0, xa = 0.0, dummy_h, dummy_r;
    {
        const Raw q0 = load_raw(jfirst - dir);
        const Raw q1 = load_raw(jfirst);
        const Raw q2 = load_raw(jfirst + dir);
        compute(q0, pb, dummy_h, dummy_r);
        compute(q1, pc, hc, rc);
        compute(q2, pa, ha, ra);
        if constexpr (PH == 3) {
            xc = q1.v[4];
            xa = q2.v[4];
        }
    }
    (void)dummy_h;
    (void)dummy_r;
    Raw fifo[DEPTH];  // rows j + 2dir .. j + (DEPTH+1) dir
#pragma unroll
    for (int d = 0; d < DEPTH; ++d)
        fifo[d] = (d + 2 <= nrows) ? load_raw(jfirst + (d + 2) * dir) : Raw{};
    // The row loop is unrolled by DEPTH so that FIFO slot u is a fixed register set: a slot is
    // consumed and refilled in the same unrolled step, and its load has DEPTH steps to arrive
    // (a rotating copy would wait on the load at the first move).
    bool done = false;
    for (int t0 = 0; !done; t0 += DEPTH) {
#pragma unroll
        for (int u = 0; u < DEPTH; ++u) {
            if (done) break;
            const int t = t0 + u;
            const int j = jfirst + t * dir;
            // x neighbours of the current row
            double pl = __shfl_up_sync(0xffffffffu, pc, 1);
            double pr = __shfl_down_sync(0xffffffffu, pc, 1);
            if (lane == 0) pl = hc;
            if (lane == 31) pr = hc;
            const double p_lo = (dir > 0) ? pb : pa;  // row j-1
            const double p_hi = (dir > 0) ? pa : pb;  // row j+1
            const double q = stencil(p_lo, pl, pc, pr, p_hi, s);
            if (valid) {
                const size_t g = (size_t)j * nx + i;
                if (PH == 0) {
                    acc[0] += rc * rc;
                    acc[1] += rc * pc;
                    acc[2] += pc * q;
                    rk1[g] = rc;  // r0 = b
                } else if (PH == 1) {
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
            if (j == jlast) {
                done = true;
                break;
            }
            // advance: row j + 2dir (slot u) enters the window; slot u is refilled
            double pn, hn, rn;
            compute(fifo[u], pn, hn, rn);
            double xn = 0.0;
            if constexpr (PH == 3) xn = fifo[u].v[4];
            fifo[u] = (t + DEPTH + 2 <= nrows) ? load_raw(j + (DEPTH + 2) * dir) : Raw{};
            pb = pc; pc = pa; pa = pn;
            hc = ha; ha = hn;
            rc = ra; ra = rn;
            xc = xa; xa = xn;
        }
    }
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

__global__ void __launch_bounds__(CGS_NT, 1)
k_cg_sweep(CgSweepArgs a) {
    __shared__ double red[CGS_NT / 32 * 4];
    __shared__ double scal[8];
    __shared__ int sflag;
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
            cg_sweep_segment<0>(a, s, w, dir, nullptr, nullptr, a.r[0], nullptr, acc);
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
                    cg_sweep_segment<1>(a, s, w, dir, rk, pkm1, nullptr, nullptr, acc);
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
                    if (k == 0) cg_sweep_segment<2>(a, s, w, dir, rk, pkm1, rk1, pk, acc);
                    else cg_sweep_segment<3>(a, s, w, dir, rk, pkm1, rk1, pk, acc);
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
