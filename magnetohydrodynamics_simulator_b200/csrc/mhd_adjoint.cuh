// Discrete adjoint of the ARS(2,2,2) IMEX step (FP64): hand-written vector-Jacobian products of
// the explicit rate (MUSCL-minmod reconstruction, HLL flux, upwind CT, flux divergence) and the
// linear stencils of the resistive term.
//
// Notation. F(U) is the explicit rate of solvers.hpp:393-402 (six planes). For a given adjoint
// w of the rate, F'(U)^T w is computed in four deterministic passes (no atomics):
//   k_adj_xface   per x face: flux adjoint from w (divergence and CT transposed), HLL VJP ->
//                 adjoints of the face's left/right reconstructed states and of its normal B
//   k_adj_yface   the same for y faces
//   k_adj_cells   per cell: gather of the reconstruction adjoints (minmod branches recomputed),
//                 primitive -> conserved VJP; hydro adjoint out, cell-centred B adjoint to scratch
//   k_adj_bfaces  per face: face-B adjoint from the cell-centred averages and the normal-B uses
// The branches of minmod, of the HLL wave-speed min/max and of the CT corner test are those of
// the forward evaluation (the derivative of a selection is that of the selected operand); floors
// contribute zero derivative where they are active.
//
// The resistive operators are symmetric: with Jz the corner current of face B
// (solvers.hpp:450-461 without eta) and C the face rate of a corner field (solvers.hpp:478-486),
// Jz^T = -C and C^T = -Jz, so the explicit rate eta*C*Jz and the implicit rate
// eta*C*(I - alpha L)^-1*Jz are both self-adjoint (Jz*C = L, the corner Laplacian of the matrix).
#pragma once

#include "mhd_kernels.cuh"

namespace mhd {

// ------------------------------------------------------------------------------------------
// Per-face vector-Jacobian products (HLL.hpp:31-218). Adjoints accumulate (+=).

struct PrimAdj {
    double rho, vx, vy, p, bx, by;
};


// fast_speed (HLL.hpp:107-122): given the adjoint of c_f, accumulate into w's adjoint and bn's.
__device__ __forceinline__ void fast_speed_vjp(const Prim& w, double bn, double ac, PrimAdj& aw,
                                               double& abn) {
    const double b2 = w.bx * w.bx + w.by * w.by;
    const double ir = 1.0 / w.rho;
    const double a2 = kGammaGas * w.p * ir;
    const double t2 = b2 * ir;
    const double n2 = bn * bn * ir;
    const double sum = t2 + a2;
    const double term = sum * sum - 4.0 * a2 * n2;
    const double sq = term > 0.0 ? sqrt(term) : 0.0;
    const double c = sqrt(0.5 * (sum + sq));
    // c = sqrt(h), h = (sum + sq) / 2
    const double ah = c > 0.0 ? ac * 0.5 / c : 0.0;
    double asum = 0.5 * ah;
    const double aterm = sq > 0.0 ? 0.5 * ah * 0.5 / sq : 0.0;
    asum += aterm * 2.0 * sum;
    double aa2 = -4.0 * n2 * aterm + asum;
    const double an2 = -4.0 * a2 * aterm;
    const double at2 = asum;
    const double air = aa2 * kGammaGas * w.p + at2 * b2 + an2 * bn * bn;
    aw.p += aa2 * kGammaGas * ir;
    const double ab2 = at2 * ir;
    abn += an2 * 2.0 * bn * ir;
    aw.rho += -air * ir * ir;
    aw.bx += ab2 * 2.0 * w.bx;
    aw.by += ab2 * 2.0 * w.by;
}

// phys_flux<DIR> (HLL.hpp:61-104).
template <int DIR>
__device__ __forceinline__ void phys_flux_vjp(const Prim& w, const Flux& aF, PrimAdj& a) {
    const double v2 = w.vx * w.vx + w.vy * w.vy;
    const double b2 = w.bx * w.bx + w.by * w.by;
    const double pt = w.p + 0.5 * b2;
    const double vb = w.vx * w.bx + w.vy * w.by;
    const double E = w.p * kInvGm1 + 0.5 * (w.rho * v2 + b2);
    double apt, aE, avb;
    if (DIR == 0) {
        // rho vx | rho vx vx + pt - bx bx | rho vx vy - bx by | (E + pt) vx - bx vb | vx by - vy bx
        a.rho += aF.rho * w.vx + aF.mx * w.vx * w.vx + aF.my * w.vx * w.vy;
        a.vx += aF.rho * w.rho + aF.mx * 2.0 * w.rho * w.vx + aF.my * w.rho * w.vy +
                aF.E * (E + pt) + aF.bt * w.by;
        a.vy += aF.my * w.rho * w.vx - aF.bt * w.bx;
        apt = aF.mx + aF.E * w.vx;
        aE = aF.E * w.vx;
        a.bx += -2.0 * w.bx * aF.mx - w.by * aF.my - aF.E * vb - aF.bt * w.vy;
        a.by += -w.bx * aF.my + aF.bt * w.vx;
        avb = -aF.E * w.bx;
    } else {
        // rho vy | rho vx vy - bx by | rho vy vy + pt - by by | (E + pt) vy - by vb | vy bx - vx by
        a.rho += aF.rho * w.vy + aF.my * w.vy * w.vy + aF.mx * w.vx * w.vy;
        a.vy += aF.rho * w.rho + aF.my * 2.0 * w.rho * w.vy + aF.mx * w.rho * w.vx +
                aF.E * (E + pt) + aF.bt * w.bx;
        a.vx += aF.mx * w.rho * w.vy - aF.bt * w.by;
        apt = aF.my + aF.E * w.vy;
        aE = aF.E * w.vy;
        a.by += -2.0 * w.by * aF.my - w.bx * aF.mx - aF.E * vb - aF.bt * w.vx;
        a.bx += -w.by * aF.mx + aF.bt * w.vy;
        avb = -aF.E * w.by;
    }
    a.vx += avb * w.bx;
    a.vy += avb * w.by;
    a.bx += avb * w.vx;
    a.by += avb * w.vy;
    // E = p/(gamma-1) + (rho v2 + b2)/2 ; pt = p + b2/2
    a.p += aE * kInvGm1 + apt;
    a.rho += aE * 0.5 * v2;
    const double av2 = aE * 0.5 * w.rho;
    const double ab2 = aE * 0.5 + 0.5 * apt;
    a.vx += av2 * 2.0 * w.vx;
    a.vy += av2 * 2.0 * w.vy;
    a.bx += ab2 * 2.0 * w.bx;
    a.by += ab2 * 2.0 * w.by;
}

// conserved<DIR> (HLL.hpp:31-47).
template <int DIR>
__device__ __forceinline__ void conserved_vjp(const Prim& w, const Flux& aU, PrimAdj& a) {
    const double v2 = w.vx * w.vx + w.vy * w.vy;
    a.rho += aU.rho + aU.mx * w.vx + aU.my * w.vy + aU.E * 0.5 * v2;
    a.vx += aU.mx * w.rho + aU.E * w.rho * w.vx;
    a.vy += aU.my * w.rho + aU.E * w.rho * w.vy;
    a.p += aU.E * kInvGm1;
    a.bx += aU.E * w.bx;
    a.by += aU.E * w.by;
    if (DIR == 0) a.by += aU.bt;
    else a.bx += aU.bt;
}

// hll<DIR> (HLL.hpp:126-218). The normal field enters both states (L.bx = R.bx in x); its
// adjoint is accumulated in aL.bx / aR.bx (x) or aL.by / aR.by (y) like the other components.
template <int DIR>
__device__ __forceinline__ void hll_vjp(const Prim& L, const Prim& R, const Flux& aF, PrimAdj& aL,
                                        PrimAdj& aR) {
    const Flux FL = phys_flux<DIR>(L);
    const Flux FR = phys_flux<DIR>(R);
    const double bnL = DIR == 0 ? L.bx : L.by;
    const double bnR = DIR == 0 ? R.bx : R.by;
    const double cL = fast_speed(L, bnL);
    const double cR = fast_speed(R, bnR);
    const double vL = DIR == 0 ? L.vx : L.vy;
    const double vR = DIR == 0 ? R.vx : R.vy;
    const double sL = smin(vL - cL, vR - cR);
    const double sR = smax(vL + cL, vR + cR);
    if (sL >= 0) {
        phys_flux_vjp<DIR>(L, aF, aL);
        return;
    }
    if (sR <= 0) {
        phys_flux_vjp<DIR>(R, aF, aR);
        return;
    }
    const Flux UL = conserved<DIR>(L);
    const Flux UR = conserved<DIR>(R);
    const double inv = 1.0 / (sR - sL);
    const double sLR = sL * sR;
    Flux F, aFL, aFR, aUR, aUL;
    F.rho = (sR * FL.rho - sL * FR.rho + sLR * (UR.rho - UL.rho)) * inv;
    F.mx = (sR * FL.mx - sL * FR.mx + sLR * (UR.mx - UL.mx)) * inv;
    F.my = (sR * FL.my - sL * FR.my + sLR * (UR.my - UL.my)) * inv;
    F.E = (sR * FL.E - sL * FR.E + sLR * (UR.E - UL.E)) * inv;
    F.bt = (sR * FL.bt - sL * FR.bt + sLR * (UR.bt - UL.bt)) * inv;
    double asR = 0.0, asL = 0.0;
#define MHD_HLL_ADJ(q)                                                   \
    {                                                                    \
        const double d = UR.q - UL.q;                                    \
        asR += aF.q * (FL.q + sL * d - F.q) * inv;                       \
        asL += aF.q * (-FR.q + sR * d + F.q) * inv;                      \
        aFL.q = aF.q * sR * inv;                                         \
        aFR.q = -aF.q * sL * inv;                                        \
        aUR.q = aF.q * sLR * inv;                                        \
        aUL.q = -aUR.q;                                                  \
    }
    MHD_HLL_ADJ(rho)
    MHD_HLL_ADJ(mx)
    MHD_HLL_ADJ(my)
    MHD_HLL_ADJ(E)
    MHD_HLL_ADJ(bt)
#undef MHD_HLL_ADJ
    phys_flux_vjp<DIR>(L, aFL, aL);
    phys_flux_vjp<DIR>(R, aFR, aR);
    conserved_vjp<DIR>(L, aUL, aL);
    conserved_vjp<DIR>(R, aUR, aR);
    double avL = 0.0, avR = 0.0, acL = 0.0, acR = 0.0;
    // sL = std::min(vL - cL, vR - cR)
    if ((vR - cR) < (vL - cL)) { avR += asL; acR -= asL; }
    else { avL += asL; acL -= asL; }
    // sR = std::max(vL + cL, vR + cR)
    if ((vL + cL) < (vR + cR)) { avR += asR; acR += asR; }
    else { avL += asR; acL += asR; }
    double abnL = 0.0, abnR = 0.0;
    fast_speed_vjp(L, bnL, acL, aL, abnL);
    fast_speed_vjp(R, bnR, acR, aR, abnR);
    if (DIR == 0) {
        aL.vx += avL; aR.vx += avR;
        aL.bx += abnL; aR.bx += abnR;
    } else {
        aL.vy += avL; aR.vy += avR;
        aL.by += abnL; aR.by += abnR;
    }
}

// Which operand minmod(a, b) returned (MUSCL.hpp:11-17): 1 = a, 2 = b, 0 = none.
__device__ __forceinline__ int minmod_branch(double a, double b) {
    if (a * b > 0.0) return (fabs(a) < fabs(b)) ? 1 : 2;
    return 0;
}

// Weight of the north (sel = 0) or south (sel = 1) face value in the corner field for a corner
// velocity v (solvers.hpp:314-340): the corner field is (ezx + ezy) / 2.
__device__ __forceinline__ double ct_weight(double v, int mode, int second) {
    if (ct_average(v, mode)) return 0.25;
    // upwind: v > 0 takes the second operand (eS for ezy, eW for ezx)
    return ((v > 0.0) == (second != 0)) ? 0.5 : 0.0;
}

// Adjoint of the corner field at corner (ic, jc) from the adjoint w of the face-B rates:
// rate_bx(i,j) = -(ez(i,j+1) - ez(i,j))/dy, rate_by(i,j) = (ez(i+1,j) - ez(i,j))/dx.
__device__ __forceinline__ double corner_field_adj(const Domain& D, double idx, double idy,
                                                   const double* __restrict__ wbx,
                                                   const double* __restrict__ wby, int ic, int jc) {
    const int nx = D.nx, ny = D.ny;
    const int i = wrap(ic, nx), j = wrap(jc, ny), im = wrap(ic - 1, nx), jm = wrap(jc - 1, ny);
    return (wbx[(size_t)j * nx + i] - wbx[(size_t)jm * nx + i]) * idy +
           (wby[(size_t)j * nx + im] - wby[(size_t)j * nx + i]) * idx;
}

// Corner velocity component (solvers.hpp:294-346; the order of the sum as in the oracle).
__device__ __forceinline__ double corner_velocity(const double* __restrict__ v, int nx, int ny,
                                                  int ic, int jc) {
    const int i = wrap(ic, nx), j = wrap(jc, ny), im = wrap(ic - 1, nx), jm = wrap(jc - 1, ny);
    return 0.25 * (v[(size_t)j * nx + i] + v[(size_t)j * nx + im] + v[(size_t)jm * nx + i] +
                   v[(size_t)jm * nx + im]);
}

// Primitive planes of the explicit-rate adjoint: rho (floored), vx, vy, p, bxc, byc.
struct PrimPlanes {
    const double* f[6];
};
// Adjoint planes of the reconstructed face states: [0..4] = rho, vx, vy, p, tangential B of the
// lower (left / down) state, [5..9] the same for the upper (right / up) state, [10] normal B.
struct FaceAdjPlanes {
    double* f[11];
};
struct CFaceAdjPlanes {
    const double* f[11];
};

// ------------------------------------------------------------------------------------------
// Pass 1 and 2: faces. Face (i, j) of direction DIR is the right face of cell (i, j) (x) or its
// top face (y). w: the adjoint of the six rates.

template <int DIR>
static __global__ void __launch_bounds__(256, 2)
k_adj_faces(Domain D, PrimPlanes P, const double* __restrict__ bxf, const double* __restrict__ byf,
            CPlanes w, FaceAdjPlanes out) {
    const int nx = D.nx, ny = D.ny;
    for (int j = blockIdx.y; j < ny; j += gridDim.y)
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nx; i += gridDim.x * blockDim.x) {
        const size_t g = (size_t)j * nx + i;
        // cells along the normal: c-1, c, c+1, c+2 (c = this cell)
        auto cell = [&](int k) -> size_t {
            return DIR == 0 ? (size_t)j * nx + wrap(i + k, nx) : (size_t)wrap(j + k, ny) * nx + i;
        };
        const size_t cm = cell(-1), c0 = g, c1 = cell(1), c2 = cell(2);
        // reconstructed states (MUSCL.hpp:26-47): lower state = upper extrapolation of c,
        // upper state = lower extrapolation of c+1; tangential B from the cell averages
        const int qv[5] = {0, 1, 2, 3, DIR == 0 ? 5 : 4};
        double lo[5], hi[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            const double* q = P.f[qv[k]];
            lo[k] = recon_hi(q[cm], q[c0], q[c1]);
            hi[k] = recon_lo(q[c0], q[c1], q[c2]);
        }
        const double bn = DIR == 0 ? bxf[c1] : byf[c1];
        Prim L, R;
        L.rho = lo[0]; L.vx = lo[1]; L.vy = lo[2]; L.p = lo[3];
        R.rho = hi[0]; R.vx = hi[1]; R.vy = hi[2]; R.p = hi[3];
        if (DIR == 0) { L.bx = R.bx = bn; L.by = lo[4]; R.by = hi[4]; }
        else { L.by = R.by = bn; L.bx = lo[4]; R.bx = hi[4]; }
        // flux adjoint: rate_q(c) = -(F(c) - F(c-1))/h  =>  aF(c) = (w(c+1) - w(c))/h
        const double idx = 1.0 / D.dx, idy = 1.0 / D.dy;
        const double ih = DIR == 0 ? idx : idy;
        Flux aF;
        aF.rho = (w.f[0][c1] - w.f[0][c0]) * ih;
        aF.mx = (w.f[1][c1] - w.f[1][c0]) * ih;
        aF.my = (w.f[2][c1] - w.f[2][c0]) * ih;
        aF.E = (w.f[3][c1] - w.f[3][c0]) * ih;
        // tangential-B flux through the corner fields (solvers.hpp:314-340)
        if (DIR == 0) {
            // Fx.bt(i,j) = -eN of corner (i+1, j) = -eS of corner (i+1, j+1)
            const double vyc0 = corner_velocity(P.f[2], nx, ny, i + 1, j);
            const double vyc1 = corner_velocity(P.f[2], nx, ny, i + 1, j + 1);
            aF.bt = -(corner_field_adj(D, idx, idy, w.f[4], w.f[5], i + 1, j) * ct_weight(vyc0, D.ct_mode, 0) +
                      corner_field_adj(D, idx, idy, w.f[4], w.f[5], i + 1, j + 1) * ct_weight(vyc1, D.ct_mode, 1));
        } else {
            // Fy.bt(i,j) = eE of corner (i, j+1) = eW of corner (i+1, j+1)
            const double vxc0 = corner_velocity(P.f[1], nx, ny, i, j + 1);
            const double vxc1 = corner_velocity(P.f[1], nx, ny, i + 1, j + 1);
            aF.bt = corner_field_adj(D, idx, idy, w.f[4], w.f[5], i, j + 1) * ct_weight(vxc0, D.ct_mode, 0) +
                    corner_field_adj(D, idx, idy, w.f[4], w.f[5], i + 1, j + 1) * ct_weight(vxc1, D.ct_mode, 1);
        }
        PrimAdj aL = {0, 0, 0, 0, 0, 0}, aR = {0, 0, 0, 0, 0, 0};
        hll_vjp<DIR>(L, R, aF, aL, aR);
        out.f[0][g] = aL.rho; out.f[1][g] = aL.vx; out.f[2][g] = aL.vy; out.f[3][g] = aL.p;
        out.f[5][g] = aR.rho; out.f[6][g] = aR.vx; out.f[7][g] = aR.vy; out.f[8][g] = aR.p;
        if (DIR == 0) {
            out.f[4][g] = aL.by; out.f[9][g] = aR.by; out.f[10][g] = aL.bx + aR.bx;
        } else {
            out.f[4][g] = aL.bx; out.f[9][g] = aR.bx; out.f[10][g] = aL.by + aR.by;
        }
    }
}

// Adjoint of one primitive of cell c along one direction, gathered from the reconstruction
// adjoints of cells c-1, c, c+1: hi(k) is the adjoint of cell k's upper extrapolation (the
// lower state of face k), lo(k) that of its lower extrapolation (the upper state of face k-1).
// q holds the primitive at cells c-2 .. c+2.
__device__ __forceinline__ double recon_gather(const double (&q)[5], const double (&hi)[3],
                                               const double (&lo)[3]) {
    double as[3];
    int br[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        as[k] = 0.5 * (hi[k] - lo[k]);  // adjoint of cell (c-1+k)'s limited slope
        br[k] = minmod_branch(q[k + 1] - q[k], q[k + 2] - q[k + 1]);
    }
    double a = hi[1] + lo[1];
    if (br[1] == 1) a += as[1];        // slope = q(c) - q(c-1)
    else if (br[1] == 2) a -= as[1];   // slope = q(c+1) - q(c)
    if (br[2] == 1) a -= as[2];        // slope of c+1 = q(c+1) - q(c)
    if (br[0] == 2) a += as[0];        // slope of c-1 = q(c) - q(c-1)
    return a;
}

// Pass 3: cells. Writes scale * (adjoint of rho, mx, my, E) into out (accumulating when
// accumulate != 0) and the adjoint of the cell-centred bxc, byc into bc_adj[0], bc_adj[1].
static __global__ void __launch_bounds__(256)
k_adj_cells(Domain D, CPlanes U, PrimPlanes P, CFaceAdjPlanes X, CFaceAdjPlanes Y, double scale,
            int accumulate, Planes out, double* __restrict__ bxc_adj, double* __restrict__ byc_adj) {
    const int nx = D.nx, ny = D.ny;
    for (int j = blockIdx.y; j < ny; j += gridDim.y)
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nx; i += gridDim.x * blockDim.x) {
        const size_t g = (size_t)j * nx + i;
        double ax[5], ay[5];
        const int qx[5] = {0, 1, 2, 3, 5}, qy[5] = {0, 1, 2, 3, 4};
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            double q[5], hi[3], lo[3];
#pragma unroll
            for (int d = 0; d < 5; ++d) q[d] = P.f[qx[k]][(size_t)j * nx + wrap(i - 2 + d, nx)];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                hi[d] = X.f[k][(size_t)j * nx + wrap(i - 1 + d, nx)];
                lo[d] = X.f[5 + k][(size_t)j * nx + wrap(i - 2 + d, nx)];
            }
            ax[k] = recon_gather(q, hi, lo);
#pragma unroll
            for (int d = 0; d < 5; ++d) q[d] = P.f[qy[k]][(size_t)wrap(j - 2 + d, ny) * nx + i];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                hi[d] = Y.f[k][(size_t)wrap(j - 1 + d, ny) * nx + i];
                lo[d] = Y.f[5 + k][(size_t)wrap(j - 2 + d, ny) * nx + i];
            }
            ay[k] = recon_gather(q, hi, lo);
        }
        double arho_f = ax[0] + ay[0];
        double avx = ax[1] + ay[1];
        double avy = ax[2] + ay[2];
        double ap = ax[3] + ay[3];
        double abyc = ax[4];
        double abxc = ay[4];
        // primitive -> conserved (Grid.hpp:100-136): vx = mx/rho, vy = my/rho (density as
        // stored), rho_f = max(rho, floor), p = max((gamma-1)(E - rho_f v^2/2 - |Bc|^2/2), floor)
        const double rho = U.f[0][g];
        const double vx = P.f[1][g], vy = P.f[2][g], rho_f = P.f[0][g];
        const double bxc = P.f[4][g], byc = P.f[5][g];
        const double eint = U.f[3][g] - 0.5 * rho_f * (vx * vx + vy * vy) - (bxc * bxc + byc * byc) / 2;
        if ((kGammaGas - 1) * eint < kPFloor) ap = 0.0;
        const double gm1ap = (kGammaGas - 1) * ap;
        const double aE = gm1ap;
        arho_f += -gm1ap * 0.5 * (vx * vx + vy * vy);
        avx += -gm1ap * rho_f * vx;
        avy += -gm1ap * rho_f * vy;
        abxc += -gm1ap * bxc;
        abyc += -gm1ap * byc;
        const double ir = 1.0 / rho;
        const double amx = avx * ir;
        const double amy = avy * ir;
        double arho = -(avx * vx + avy * vy) * ir;
        if (!(rho < kRhoFloor)) arho += arho_f;
        const double o[4] = {arho, amx, amy, aE};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const double v = scale * o[k];
            out.f[k][g] = accumulate ? out.f[k][g] + v : v;
        }
        bxc_adj[g] = abxc;
        byc_adj[g] = abyc;
    }
}

// Pass 4: face B. bxc(i) = (bxf(i) + bxf(i+1))/2 and the x face i-1 uses bxf(i) as normal field.
static __global__ void __launch_bounds__(256)
k_adj_bfaces(Domain D, const double* __restrict__ bxc_adj, const double* __restrict__ byc_adj,
             const double* __restrict__ xbn, const double* __restrict__ ybn, double scale,
             int accumulate, double* __restrict__ out_bx, double* __restrict__ out_by) {
    const int nx = D.nx, ny = D.ny;
    for (int j = blockIdx.y; j < ny; j += gridDim.y)
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nx; i += gridDim.x * blockDim.x) {
        const size_t g = (size_t)j * nx + i;
        const size_t gxm = (size_t)j * nx + wrap(i - 1, nx);
        const size_t gym = (size_t)wrap(j - 1, ny) * nx + i;
        const double abx = 0.5 * (bxc_adj[g] + bxc_adj[gxm]) + xbn[gxm];
        const double aby = 0.5 * (byc_adj[g] + byc_adj[gym]) + ybn[gym];
        out_bx[g] = accumulate ? out_bx[g] + scale * abx : scale * abx;
        out_by[g] = accumulate ? out_by[g] + scale * aby : scale * aby;
    }
}

// ------------------------------------------------------------------------------------------
// Linear stencils of the resistive term and plane algebra.

// out = s * Jz(bx, by) + t * L x  (corner plane; x may be null when t == 0).
static __global__ void __launch_bounds__(256)
k_adj_jz(Domain D, const double* __restrict__ bx, const double* __restrict__ by, double s,
         const double* __restrict__ x, double t, double* __restrict__ out) {
    const int nx = D.nx, ny = D.ny;
    const double idx = 1.0 / D.dx, idy = 1.0 / D.dy;
    for (int j = blockIdx.y; j < ny; j += gridDim.y)
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nx; i += gridDim.x * blockDim.x) {
        const size_t g = (size_t)j * nx + i;
        const size_t gxm = (size_t)j * nx + wrap(i - 1, nx);
        const size_t gym = (size_t)wrap(j - 1, ny) * nx + i;
        double v = s * ((by[g] - by[gxm]) * idx - (bx[g] - bx[gym]) * idy);
        if (x) {
            const size_t gxp = (size_t)j * nx + wrap(i + 1, nx);
            const size_t gyp = (size_t)wrap(j + 1, ny) * nx + i;
            const double lap = (x[gxp] + x[gxm] - 2.0 * x[g]) * (idx * idx) +
                               (x[gyp] + x[gym] - 2.0 * x[g]) * (idy * idy);
            v += t * lap;
        }
        out[g] = v;
    }
}

// (out_bx, out_by) = a * (base_bx, base_by) + b * (extra_bx, extra_by) + s * C(E) with
// C(E) = (-(E(i,j+1) - E(i,j))/dy, (E(i+1,j) - E(i,j))/dx). Null base / extra planes count as 0;
// out may alias base.
static __global__ void __launch_bounds__(256)
k_adj_curl(Domain D, const double* __restrict__ E, double s, const double* base_bx,
           const double* base_by, double a, const double* extra_bx, const double* extra_by,
           double b, double* out_bx, double* out_by) {
    const int nx = D.nx, ny = D.ny;
    const double idx = 1.0 / D.dx, idy = 1.0 / D.dy;
    for (int j = blockIdx.y; j < ny; j += gridDim.y)
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nx; i += gridDim.x * blockDim.x) {
        const size_t g = (size_t)j * nx + i;
        const size_t gxp = (size_t)j * nx + wrap(i + 1, nx);
        const size_t gyp = (size_t)wrap(j + 1, ny) * nx + i;
        double rbx = E ? s * (-(E[gyp] - E[g]) * idy) : 0.0;
        double rby = E ? s * ((E[gxp] - E[g]) * idx) : 0.0;
        if (base_bx) { rbx += a * base_bx[g]; rby += a * base_by[g]; }
        if (extra_bx) { rbx += b * extra_bx[g]; rby += b * extra_by[g]; }
        out_bx[g] = rbx;
        out_by[g] = rby;
    }
}

// out[k] = a * x[k] + b * y[k] for the planes k < nplanes (y may be null; out may alias x or y).
struct Planes6C {
    const double* f[6];
};
static __global__ void __launch_bounds__(256)
k_adj_axpby(int nplanes, size_t n, double a, Planes6C x, double b, Planes6C y, Planes out) {
    for (size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x; g < n;
         g += (size_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            if (k < nplanes) {
                double v = a * x.f[k][g];
                if (y.f[k]) v += b * y.f[k][g];
                out.f[k][g] = v;
            }
        }
    }
}

// The two plane combinations that close the adjoint step, in one pass over six planes:
// w = cd * lam + cg * lamT (the explicit-rate adjoint of stage 1) and lam += lamT.
static __global__ void __launch_bounds__(256)
k_adj_close(size_t n, double cd, double cg, Planes lam, Planes6C lamT, Planes w) {
    for (size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x; g < n;
         g += (size_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const double a = lam.f[k][g], t = lamT.f[k][g];
            w.f[k][g] = cd * a + cg * t;
            lam.f[k][g] = a + t;
        }
    }
}

// Deterministic dot product: per-block partial sums of a*b, then one block sums them in order
// and adds scale * total to *acc.
static __global__ void __launch_bounds__(256)
k_adj_dot_partial(size_t n, const double* __restrict__ a, const double* __restrict__ b,
                  double* __restrict__ partial) {
    __shared__ double red[64];
    double s[1] = {0.0};
    for (size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x; g < n;
         g += (size_t)gridDim.x * blockDim.x)
        s[0] += a[g] * b[g];
    block_sum<256, 1>(s, red);
    if (threadIdx.x == 0) partial[blockIdx.x] = s[0];
}

// One warp: lane l sums partials l, l+32, ... in order, then a fixed shuffle tree.
static __global__ void k_adj_dot_final(const double* __restrict__ partial, int nblocks, double scale,
                                       double* acc) {
    if (blockIdx.x != 0 || threadIdx.x >= 32) return;
    double s = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += 32) s += partial[b];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) *acc += scale * s;
}

}  // namespace mhd
