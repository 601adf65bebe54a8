// kernels.cu -- FP64 stage kernels of the hosono-2DMHD time step for sm_100a.
//
// Compiled twice: with -DHOSONO_FAST=0 --fmad=false (strict: every operation
// rounded on its own, bit-identical to the oracle) and with -DHOSONO_FAST=1
// --fmad=true (FMA contraction allowed).  Each object exports one KernelTable.
//
// Data layout in HBM: structure of arrays, one plane per conserved variable
// (and per primitive variable for V), rows of `pitch` doubles (a multiple of
// 32, i.e. 256-byte rows), guard cells included.  Cell (i,j) 0-based at
// j*pitch+i; the interior is [g, g+nx) x [g, g+ny), g = NGC = R+2.
// MOOD state is one byte per cell per flag.
//
// Index ranges (0-based) of the reference loops:
//   reconstruct  [strt-2, stop+2]  -> [g-2, g+n+1]   (reconstruct.f90:81-82)
//   getFluxes    [strt-1, stop+2]  -> [g-1, g+n+1]   (getFluxes.f90:204-205)
//   FLICD        [strt,   stop+1]  -> [g,   g+n]     (FLICDdivB.f90:301-302)
//   update/detect [strt,  stop]    -> [g,   g+n-1]   (timeStep.f90:108-109, detect.f90:81-82)

#include "kernels.h"

#include <cstdio>

#ifndef HOSONO_FAST
#error "HOSONO_FAST must be defined (0 strict, 1 fast)"
#endif

#if HOSONO_FAST
#define KNS kfast
#else
#define KNS kstrict
#endif

namespace hosono {
namespace KNS {

constexpr int BX = 32, BY = 8;

__device__ __forceinline__ int iabs_c(int a) { return a < 0 ? -a : a; }

// GP prediction at quadrature point q of face f of cell (i,j), radius RR:
// sum_k pv(k,q,f,RR) * U(:, stencil_k)  in stencil order k=1..ns
// (reconstruct.f90:109-124; stencil order of GP.f90:85-95).
template <int RR>
__device__ __forceinline__ void gp_face(const double* __restrict__ U, long long plane, int pitch, int i, int j,
                                        const double* __restrict__ pvq, double out[NCONS]) {
#pragma unroll
    for (int v = 0; v < NCONS; v++) out[v] = 0.0;
    int k = 0;
#pragma unroll
    for (int a = -RR; a <= RR; a++) {
#pragma unroll
        for (int b = -RR; b <= RR; b++) {
            if (iabs_c(a) + iabs_c(b) <= RR) {
                const double p = __ldg(pvq + k);
                const long long idx = (long long)(j + b) * pitch + (i + a);
#pragma unroll
                for (int v = 0; v < NCONS; v++) out[v] = out[v] + p * __ldg(U + v * plane + idx);
                k++;
            }
        }
    }
}

__device__ __forceinline__ const double* pv_ptr(const StageArgs& a, int rr, int f, int q) {
    return a.pv + (long long)a.geo.nsMax * (q + a.geo.nqMax * (f + 4 * (rr - 1)));
}

__device__ __forceinline__ double qw_at(const StageArgs& a, int rr, int q) { return __ldg(a.qw + q + a.geo.nqMax * (rr - 1)); }

// face value with a run-time radius; rr == 0 is the first-order copy of U
__device__ __forceinline__ void face_value(const StageArgs& a, int rr, int i, int j, int f, int q, double out[NCONS]) {
    const Geo& G = a.geo;
    if (rr == 0) {
        const long long idx = (long long)j * G.pitch + i;
#pragma unroll
        for (int v = 0; v < NCONS; v++) out[v] = __ldg(a.Uin + v * G.plane + idx);
        return;
    }
    const double* pvq = pv_ptr(a, rr, f, q);
    if (rr == 1)
        gp_face<1>(a.Uin, G.plane, G.pitch, i, j, pvq, out);
    else if (rr == 2)
        gp_face<2>(a.Uin, G.plane, G.pitch, i, j, pvq, out);
    else
        gp_face<3>(a.Uin, G.plane, G.pitch, i, j, pvq, out);
}

__device__ __forceinline__ void warp_flag(int* counter, bool flag) {
    const unsigned m = __ballot_sync(0xffffffffu, flag);
    if (m && (threadIdx.x & 31) == 0) atomicOr(counter, 1);
}

__device__ __forceinline__ void warp_count(int* counter, bool flag) {
    const unsigned m = __ballot_sync(0xffffffffu, flag);
    if (m && (threadIdx.x & 31) == 0) atomicAdd(counter, __popc(m));
}

// ------------------------------------------------------------------------
// MOOD pass 1 (every scheme == R): reconstruct_faceValsWithGP + face CAD/PAD
// + getFluxes_ fused.  One thread per cell (i,j) owns the x-face between
// (i-1,j) and (i,j) and the y-face between (i,j-1) and (i,j).  Face values are
// recomputed per quadrature point and never stored.  A cell fails when any of
// its four faces fails; the four verdicts are kept per face side in failX /
// failY and combined by cascade_lower.  Fluxes of faces next to a failing
// cell are recomputed after the cascade (flux, FLUX_DIRTY).
template <int R>
__global__ void __launch_bounds__(BX* BY) k_face_pass1(StageArgs a) {
    const Geo& G = a.geo;
    const int g = G.g;
    const int i = g - 2 + blockIdx.x * BX + threadIdx.x;
    const int j = g - 2 + blockIdx.y * BY + threadIdx.y;
    const int clo = g - 2, cxhi = g + G.nx + 1, cyhi = g + G.ny + 1;  // reconstruct range
    const int flo = g - 1, fxhi = g + G.nx + 1, fyhi = g + G.ny + 1;  // flux range
    const long long c = (long long)j * G.pitch + i;
    constexpr int NQ = R + 1;
    bool bad = false;

    // x-face
    if (i >= clo && i <= cxhi + 1 && j >= clo && j <= cyhi) {
        const bool needL = (i - 1 >= clo);
        const bool needR = (i <= cxhi);
        const bool doFlux = (i >= flo && i <= fxhi && j >= flo && j <= fyhi);
        uint8_t bits = 0;
        double acc[NCONS];
#pragma unroll
        for (int v = 0; v < NCONS; v++) acc[v] = 0.0;
#pragma unroll 1
        for (int q = 0; q < NQ; q++) {
            double uL[NCONS], uR[NCONS];
            if (needL) {
                gp_face<R>(a.Uin, G.plane, G.pitch, i - 1, j, pv_ptr(a, R, EAST, q), uL);
                if (!admissible(uL[DENS], cons2pres(a.phys, uL))) bits |= 1;
            }
            if (needR) {
                gp_face<R>(a.Uin, G.plane, G.pitch, i, j, pv_ptr(a, R, WEST, q), uR);
                if (!admissible(uR[DENS], cons2pres(a.phys, uR))) bits |= 2;
            }
            if (doFlux) {
                double F[NCONS];
                hllc(a.phys, uL, uR, XDIR, F);
                const double w = qw_at(a, R, q);
#pragma unroll
                for (int v = 0; v < NCONS; v++) acc[v] = acc[v] + w * F[v];
            }
        }
        a.failX[c] = bits;
        bad |= bits != 0;
        if (doFlux) {
#pragma unroll
            for (int v = 0; v < NCONS; v++) a.FX[v * G.plane + c] = acc[v];
            a.CTX[c] = acc[MAGY];
        }
    }
    // y-face
    if (i >= clo && i <= cxhi && j >= clo && j <= cyhi + 1) {
        const bool needB = (j - 1 >= clo);
        const bool needT = (j <= cyhi);
        const bool doFlux = (i >= flo && i <= fxhi && j >= flo && j <= fyhi);
        uint8_t bits = 0;
        double acc[NCONS];
#pragma unroll
        for (int v = 0; v < NCONS; v++) acc[v] = 0.0;
#pragma unroll 1
        for (int q = 0; q < NQ; q++) {
            double uL[NCONS], uR[NCONS];
            if (needB) {
                gp_face<R>(a.Uin, G.plane, G.pitch, i, j - 1, pv_ptr(a, R, NORTH, q), uL);
                if (!admissible(uL[DENS], cons2pres(a.phys, uL))) bits |= 1;
            }
            if (needT) {
                gp_face<R>(a.Uin, G.plane, G.pitch, i, j, pv_ptr(a, R, SOUTH, q), uR);
                if (!admissible(uR[DENS], cons2pres(a.phys, uR))) bits |= 2;
            }
            if (doFlux) {
                double F[NCONS];
                hllc(a.phys, uL, uR, YDIR, F);
                const double w = qw_at(a, R, q);
#pragma unroll
                for (int v = 0; v < NCONS; v++) acc[v] = acc[v] + w * F[v];
            }
        }
        a.failY[c] = bits;
        bad |= bits != 0;
        if (doFlux) {
#pragma unroll
            for (int v = 0; v < NCONS; v++) a.FY[v * G.plane + c] = acc[v];
            a.CTY[c] = acc[MAGX];
        }
    }
    warp_flag(a.counters + CNT_ANYFAIL, bad);
}

// ------------------------------------------------------------------------
// Serial lowering pass of reconstruct.f90:146-169 (order independent: a cell
// only lowers its own scheme; every flag write is a set): for each failing
// cell in [g-2, g+n+1]^2, gridBlock_lowerOrder (gridBlock.f90:194-235) and
// mark the cross for the next inner pass.
__global__ void __launch_bounds__(BX* BY) k_cascade_lower(StageArgs a, int mode) {
    const Geo& G = a.geo;
    const int g = G.g;
    const int i = g - 2 + blockIdx.x * BX + threadIdx.x;
    const int j = g - 2 + blockIdx.y * BY + threadIdx.y;
    bool f = false;
    if (i <= g + G.nx + 1 && j <= g + G.ny + 1) {
        const long long c = (long long)j * G.pitch + i;
        if (mode == CASCADE_FROM_FACES)
            f = ((a.failX[c] & 2) | (a.failX[c + 1] & 1) | (a.failY[c] & 2) | (a.failY[c + G.pitch] & 1)) != 0;
        else
            f = a.fail[c] != 0;
        if (f) {
            const int s = a.scheme[c];
            a.scheme[c] = (int8_t)(s - 1 > 0 ? s - 1 : 0);
            a.rec[c] = 1;
            a.rec[c + 1] = 1;
            a.rec[c - 1] = 1;
            a.rec[c + G.pitch] = 1;
            a.rec[c - G.pitch] = 1;
            for (int jj = j - 2; jj <= j + 2; jj++) {
                if (jj < 0 || jj >= G.nyt) continue;
                for (int ii = i - 2; ii <= i + 2; ii++) {
                    if (ii < 0 || ii >= G.nxt) continue;
                    if (iabs_c(ii - i) + iabs_c(jj - j) <= 2) a.recF[(long long)jj * G.pitch + ii] = 1;
                }
            }
            a.nextPass[c] = 1;
            a.nextPass[c + 1] = 1;
            a.nextPass[c - 1] = 1;
            a.nextPass[c + G.pitch] = 1;
            a.nextPass[c - G.pitch] = 1;
            if (a.trace) a.innerCount[c] = (uint8_t)(a.innerCount[c] + 1);
        }
    }
    warp_count(a.counters + CNT_INNER, f);
}

// ------------------------------------------------------------------------
// One inner pass of reconstruct_faceValsWithGP on the cells flagged in mask:
// all four faces at rr = min(scheme(c), scheme(nbr)) (EDP1), CAD/PAD on every
// quadrature point.  The radius used per face is recorded in rrRec so the
// flux kernel can rebuild exactly these face values later.
__global__ void __launch_bounds__(BX* BY) k_recon_check(StageArgs a, const uint8_t* __restrict__ mask) {
    const Geo& G = a.geo;
    const int g = G.g;
    const int i = g - 2 + blockIdx.x * BX + threadIdx.x;
    const int j = g - 2 + blockIdx.y * BY + threadIdx.y;
    bool bad = false;
    if (i <= g + G.nx + 1 && j <= g + G.ny + 1) {
        const long long c = (long long)j * G.pitch + i;
        if (mask[c]) {
            a.dirty[c] = 1;
            const int s = a.scheme[c];
            int rr[4];
            rr[NORTH] = min(s, (int)a.scheme[c + G.pitch]);
            rr[SOUTH] = min(s, (int)a.scheme[c - G.pitch]);
            rr[EAST] = min(s, (int)a.scheme[c + 1]);
            rr[WEST] = min(s, (int)a.scheme[c - 1]);
            a.rrRec[c] = (uint8_t)(rr[0] | (rr[1] << 2) | (rr[2] << 4) | (rr[3] << 6));
#pragma unroll 1
            for (int f = 0; f < 4 && !bad; f++) {
                if (rr[f] == 0) continue;
#pragma unroll 1
                for (int q = 0; q <= rr[f] && !bad; q++) {
                    double u[NCONS];
                    face_value(a, rr[f], i, j, f, q, u);
                    if (!admissible(u[DENS], cons2pres(a.phys, u))) bad = true;
                }
            }
            if (bad) a.fail[c] = 1;
        }
    }
    warp_flag(a.counters + CNT_ANYFAIL, bad);
}

// ------------------------------------------------------------------------
// getFluxes_ (getFluxes.f90:16-90) on flagged faces.  Face values are rebuilt
// from U at the radius each side was last reconstructed with (rrRec); the
// quadrature uses the face's current radius (riemannSolver.f90:23-47).
__device__ __forceinline__ void face_flux(const StageArgs& a, int dir, int iL, int jL, int fL, int rrL, int iR, int jR,
                                          int fR, int rrR, int rr, double flux[NCONS]) {
    double uL[NCONS], uR[NCONS];
    if (rr == 0) {
        face_value(a, rrL, iL, jL, fL, 0, uL);
        face_value(a, rrR, iR, jR, fR, 0, uR);
        hllc(a.phys, uL, uR, dir, flux);
        return;
    }
#pragma unroll
    for (int v = 0; v < NCONS; v++) flux[v] = 0.0;
#pragma unroll 1
    for (int q = 0; q <= rr; q++) {
        face_value(a, rrL, iL, jL, fL, q, uL);
        face_value(a, rrR, iR, jR, fR, q, uR);
        double F[NCONS];
        hllc(a.phys, uL, uR, dir, F);
        const double w = qw_at(a, rr, q);
#pragma unroll
        for (int v = 0; v < NCONS; v++) flux[v] = flux[v] + w * F[v];
    }
}

__global__ void __launch_bounds__(BX* BY) k_flux(StageArgs a, int mode) {
    const Geo& G = a.geo;
    const int g = G.g;
    const int i = g - 1 + blockIdx.x * BX + threadIdx.x;
    const int j = g - 1 + blockIdx.y * BY + threadIdx.y;
    if (i > g + G.nx + 1 || j > g + G.ny + 1) return;
    const long long c = (long long)j * G.pitch + i;
    const long long cw = c - 1, cs = c - G.pitch;
    const bool doX = mode == FLUX_DIRTY ? (a.dirty[c] | a.dirty[cw]) != 0 : (a.rec[c] | a.rec[cw]) != 0;
    const bool doY = mode == FLUX_DIRTY ? (a.dirty[c] | a.dirty[cs]) != 0 : (a.rec[c] | a.rec[cs]) != 0;
    if (doX) {
        const int rr = min((int)a.scheme[c], (int)a.scheme[cw]);
        const int rrL = (a.rrRec[cw] >> (2 * EAST)) & 3;
        const int rrR = (a.rrRec[c] >> (2 * WEST)) & 3;
        double F[NCONS];
        face_flux(a, XDIR, i - 1, j, EAST, rrL, i, j, WEST, rrR, rr, F);
#pragma unroll
        for (int v = 0; v < NCONS; v++) a.FX[v * G.plane + c] = F[v];
        a.CTX[c] = F[MAGY];
    }
    if (doY) {
        const int rr = min((int)a.scheme[c], (int)a.scheme[cs]);
        const int rrL = (a.rrRec[cs] >> (2 * NORTH)) & 3;
        const int rrR = (a.rrRec[c] >> (2 * SOUTH)) & 3;
        double F[NCONS];
        face_flux(a, YDIR, i, j - 1, NORTH, rrL, i, j, SOUTH, rrR, rr, F);
#pragma unroll
        for (int v = 0; v < NCONS; v++) a.FY[v * G.plane + c] = F[v];
        a.CTY[c] = F[MAGX];
    }
}

// ------------------------------------------------------------------------
// FLICDdivB_fluxCorrections (FLICDdivB.f90:13-70) from fluxRaw.
__device__ __forceinline__ double flicd_x(const StageArgs& a, long long c) {
    const Geo& G = a.geo;
    const double* fxy = a.FX + MAGY * G.plane;
    const double* fyx = a.FY + MAGX * G.plane;
    const long long p = G.pitch;
    return (2 * fxy[c] + fxy[c + 1] + fxy[c - 1] - fyx[c + p] - fyx[c] - fyx[c - 1] - fyx[c - 1 + p]) / 8.0;
}
__device__ __forceinline__ double flicd_y(const StageArgs& a, long long c) {
    const Geo& G = a.geo;
    const double* fxy = a.FX + MAGY * G.plane;
    const double* fyx = a.FY + MAGX * G.plane;
    const long long p = G.pitch;
    return (2 * fyx[c] + fyx[c + p] + fyx[c - p] - fxy[c + 1] - fxy[c] - fxy[c - p] - fxy[c + 1 - p]) / 8.0;
}

// detect_ALL's per-cell test (detect.f90:84-213): true when the cell must be lowered.
__device__ __forceinline__ bool detect_cell(const StageArgs& a, long long c, const double un[NCONS]) {
    const Geo& G = a.geo;
    const Phys& s = a.phys;
    const double* U = a.Uin;
    const long long P = G.plane, p = G.pitch;
    const double presNew = cons2pres(s, un);
    if (!admissible(un[DENS], presNew)) return true;
    double u[NCONS], V[NPRIM], Vip[NPRIM], Vim[NPRIM], Vjp[NPRIM], Vjm[NPRIM];
#pragma unroll
    for (int v = 0; v < NCONS; v++) u[v] = U[v * P + c];
    cons2prim(s, u, V);
#pragma unroll
    for (int v = 0; v < NCONS; v++) u[v] = U[v * P + c + 1];
    cons2prim(s, u, Vip);
#pragma unroll
    for (int v = 0; v < NCONS; v++) u[v] = U[v * P + c - 1];
    cons2prim(s, u, Vim);
#pragma unroll
    for (int v = 0; v < NCONS; v++) u[v] = U[v * P + c + p];
    cons2prim(s, u, Vjp);
#pragma unroll
    for (int v = 0; v < NCONS; v++) u[v] = U[v * P + c - p];
    cons2prim(s, u, Vjm);
    const double dx = G.dx, dy = G.dy;
    double div_vel = (Vip[VELX] - Vim[VELX]) / (2 * dx);
    div_vel = div_vel + (Vjp[VELY] - Vjm[VELY]) / (2 * dy);
    const bool shock1 = div_vel < -(1.0 * (G.maxdxdy * G.maxdxdy));
    double mach = V[VELX] * V[VELX] + V[VELY] * V[VELY];
    mach = V[DENS] * mach / (V[GAMM] * V[PRES]);
    mach = sqrt(mach);
    const bool shock2 = mach > 0.2;
    double pg = fabs(Vip[PRES] - Vim[PRES]) / (fmin(Vip[PRES], Vim[PRES]));
    pg = pg + fabs(Vjp[PRES] - Vjm[PRES]) / (fmin(Vjp[PRES], Vjm[PRES]));
    const bool shock3 = pg > 10.0 * G.maxdxdy;
    if (!(shock1 && shock2 && shock3)) return false;
    const double* rho = U + DENS * P;
    const double d1 = rho[c], d2 = rho[c + 1], d3 = rho[c - 1], d4 = rho[c + p], d5 = rho[c - p];
    const double mn = fmin(fmin(fmin(fmin(d1, d2), d3), d4), d5);
    const double mx = fmax(fmax(fmax(fmax(d1, d2), d3), d4), d5);
    if (mx - mn < G.mindxdy * G.mindxdy * G.mindxdy) return false;
    const double dn = un[DENS];
    if ((mn <= dn) && (dn <= mx)) return false;
    // u2 smoothness (detect.f90:177-213, option 3)
    double mnx = 0, mxx = 0, mny = 0, mxy = 0;
    int k = 0;
#pragma unroll
    for (int ii = -1; ii <= 1; ii++) {
#pragma unroll
        for (int jj = -1; jj <= 1; jj++) {
            if (iabs_c(ii) + iabs_c(jj) <= 1) {
                const long long cc = c + ii + jj * p;
                const double ddx = (rho[cc + 1] - 2 * rho[cc] + rho[cc - 1]) / (dx * dx);
                const double ddy = (rho[cc + p] - 2 * rho[cc] + rho[cc - p]) / (dy * dy);
                if (k == 0) {
                    mnx = mxx = ddx;
                    mny = mxy = ddy;
                } else {
                    mnx = fmin(mnx, ddx);
                    mxx = fmax(mxx, ddx);
                    mny = fmin(mny, ddy);
                    mxy = fmax(mxy, ddy);
                }
                k++;
            }
        }
    }
    const double m = G.mindxdy;
    const bool sx1 = (mnx * mxx > -m);
    const bool sy1 = (mny * mxy > -m);
    const bool sx2 = (fmax(fabs(mnx), fabs(mxx)) < m);
    const bool sy2 = (fmax(fabs(mny), fabs(mxy)) < m);
    const bool sx3 = (fmin(fabs(mnx), fabs(mxx)) >= 0.5 * fmax(fabs(mnx), fabs(mxx)));
    const bool sy3 = (fmin(fabs(mny), fabs(mxy)) >= 0.5 * fmax(fabs(mny), fabs(mxy)));
    const bool smooth1 = sx1 && sx2 && sy1 && sy2;
    const bool smooth2 = sx1 && sx3 && sy1 && sy3;
    return !(smooth1 || smooth2);
}

// FLICD on [g, g+n]^2 where recomputeFLICD; then, on the interior, the
// unsplit update of timeStep.f90:107-118 and detect_ALL.  A corrected flux a
// neighbour needs is recomputed locally when the neighbour is flagged (it
// writes the same value) and read from memory otherwise (nobody writes it).
__global__ void __launch_bounds__(BX* BY) k_ct_update_detect(StageArgs a) {
    const Geo& G = a.geo;
    const int g = G.g;
    const int i = g + blockIdx.x * BX + threadIdx.x;
    const int j = g + blockIdx.y * BY + threadIdx.y;
    bool low = false;
    if (i <= g + G.nx && j <= g + G.ny) {
        const long long c = (long long)j * G.pitch + i;
        if (a.recF[c]) {
            const double ctx = flicd_x(a, c);
            const double cty = flicd_y(a, c);
            a.CTX[c] = ctx;
            a.CTY[c] = cty;
            if (i < g + G.nx && j < g + G.ny) {
                const long long ce = c + 1, cn = c + G.pitch;
                const double ctx_e = a.recF[ce] ? flicd_x(a, ce) : a.CTX[ce];
                const double cty_n = a.recF[cn] ? flicd_y(a, cn) : a.CTY[cn];
                const double dtdx = a.dt / G.dx, dtdy = a.dt / G.dy;
                double un[NCONS];
#pragma unroll
                for (int v = 0; v < NCONS; v++) {
                    double f0, f1, g0, g1;
                    if (v == MAGX) {
                        f0 = 0.0;
                        f1 = 0.0;
                        g0 = cty;
                        g1 = cty_n;
                    } else if (v == MAGY) {
                        f0 = ctx;
                        f1 = ctx_e;
                        g0 = 0.0;
                        g1 = 0.0;
                    } else {
                        f0 = a.FX[v * G.plane + c];
                        f1 = a.FX[v * G.plane + ce];
                        g0 = a.FY[v * G.plane + c];
                        g1 = a.FY[v * G.plane + cn];
                    }
                    un[v] = a.Uin[v * G.plane + c] - dtdx * (f1 - f0) - dtdy * (g1 - g0);
                    a.Uout[v * G.plane + c] = un[v];
                }
                if (a.scheme[c] > 0) {
                    low = detect_cell(a, c, un);
                    if (low) a.lowered[c] = 1;
                }
            }
        }
    }
    warp_count(a.counters + CNT_DETECT, low);
}

// ------------------------------------------------------------------------
// After detect: recompute = cross of lowered cells, recomputeFLICD = radius-2
// diamond (gridBlock_lowerOrder), scheme lowered by one where lowered; then
// boundaryConditions_applyMOOD's periodic sync, which (x sweep over all rows,
// then y sweep over all columns, N >= 2*NGC) makes every cell the OR (flags) /
// MIN (scheme) over its translates by multiples of N that lie in the array.
__device__ __forceinline__ bool lowered_at(const StageArgs& a, int i, int j) {
    const Geo& G = a.geo;
    if (i < 0 || j < 0 || i >= G.nxt || j >= G.nyt) return false;
    return a.lowered[(long long)j * G.pitch + i] != 0;
}

__global__ void __launch_bounds__(BX* BY) k_mood_flags(StageArgs a) {
    const Geo& G = a.geo;
    const int i = blockIdx.x * BX + threadIdx.x;
    const int j = blockIdx.y * BY + threadIdx.y;
    if (i >= G.nxt || j >= G.nyt) return;
    const int reach = G.bc == 1 ? 1 : 0;
    bool rec = false, recF = false;
    int sch = 127;
    for (int b = -reach; b <= reach; b++) {
        const int jo = j + b * G.ny;
        if (jo < 0 || jo >= G.nyt) continue;
        for (int t = -reach; t <= reach; t++) {
            const int io = i + t * G.nx;
            if (io < 0 || io >= G.nxt) continue;
            const long long co = (long long)jo * G.pitch + io;
            const int lo = a.lowered[co];
            const int so = a.scheme[co] - lo;
            sch = min(sch, so > 0 ? so : 0);
            for (int dj = -2; dj <= 2; dj++) {
                for (int di = -2; di <= 2; di++) {
                    const int d = iabs_c(di) + iabs_c(dj);
                    if (d > 2) continue;
                    if (lowered_at(a, io + di, jo + dj)) {
                        recF = true;
                        if (d <= 1) rec = true;
                    }
                }
            }
        }
    }
    const long long c = (long long)j * G.pitch + i;
    a.rec[c] = rec;
    a.recF[c] = recF;
    a.scheme_next[c] = (int8_t)sch;
}

// ------------------------------------------------------------------------
// boundary conditions (boundaryConditions.f90:291-360) as a gather
__device__ __forceinline__ int bc_src(int i, int n, int g, int bc) {
    if (i < g) return bc == 1 ? i + n : g;
    if (i >= g + n) return bc == 1 ? i - n : g + n - 1;
    return i;
}

__global__ void k_bc_fill(Geo G, double* A, int nvar) {
    const int i = blockIdx.x * BX + threadIdx.x;
    const int j = blockIdx.y * BY + threadIdx.y;
    if (i >= G.nxt || j >= G.nyt) return;
    const int si = bc_src(i, G.nx, G.g, G.bc), sj = bc_src(j, G.ny, G.g, G.bc);
    if (si == i && sj == j) return;
    const long long c = (long long)j * G.pitch + i, s = (long long)sj * G.pitch + si;
    for (int v = 0; v < nvar; v++) A[v * G.plane + c] = A[v * G.plane + s];
}

// timeStep.f90:165 over every cell (guards from their images)
__global__ void k_rk_combine2(Geo G, const double* __restrict__ Un, const double* __restrict__ B, double* __restrict__ out) {
    const int i = blockIdx.x * BX + threadIdx.x;
    const int j = blockIdx.y * BY + threadIdx.y;
    if (i >= G.nxt || j >= G.nyt) return;
    const int si = bc_src(i, G.nx, G.g, G.bc), sj = bc_src(j, G.ny, G.g, G.bc);
    const long long c = (long long)j * G.pitch + i, s = (long long)sj * G.pitch + si;
#pragma unroll
    for (int v = 0; v < NCONS; v++) out[v * G.plane + c] = (3 * Un[v * G.plane + s] + B[v * G.plane + s]) / 4.0;
}

// timeStep.f90:169 and :32-41 (V = cons2prim(U), boundary conditions on U and V)
__global__ void k_rk_final(Geo G, Phys P, const double* __restrict__ Un, const double* __restrict__ B,
                           double* __restrict__ outU, double* __restrict__ outV) {
    const int i = blockIdx.x * BX + threadIdx.x;
    const int j = blockIdx.y * BY + threadIdx.y;
    if (i >= G.nxt || j >= G.nyt) return;
    const int si = bc_src(i, G.nx, G.g, G.bc), sj = bc_src(j, G.ny, G.g, G.bc);
    const long long c = (long long)j * G.pitch + i, s = (long long)sj * G.pitch + si;
    double u[NCONS], V[NPRIM];
#pragma unroll
    for (int v = 0; v < NCONS; v++) {
        u[v] = (Un[v * G.plane + s] + 2 * B[v * G.plane + s]) / 3.0;
        outU[v * G.plane + c] = u[v];
    }
    cons2prim(P, u, V);
#pragma unroll
    for (int v = 0; v < NPRIM; v++) outV[v * G.plane + c] = V[v];
}

__global__ void k_cons2prim_all(Geo G, Phys P, const double* __restrict__ U, double* __restrict__ V) {
    const int i = blockIdx.x * BX + threadIdx.x;
    const int j = blockIdx.y * BY + threadIdx.y;
    if (i >= G.nxt || j >= G.nyt) return;
    const long long c = (long long)j * G.pitch + i;
    double u[NCONS], w[NPRIM];
#pragma unroll
    for (int v = 0; v < NCONS; v++) u[v] = U[v * G.plane + c];
    cons2prim(P, u, w);
#pragma unroll
    for (int v = 0; v < NPRIM; v++) V[v * G.plane + c] = w[v];
}

// cfl_computedt (cfl.f90:14-52): max over the interior of |u|+c and |v|+c.
// Non-negative doubles order like their bit patterns, so the block maxima
// are combined with an integer atomicMax.
__global__ void __launch_bounds__(256) k_cfl_max(Geo G, Phys P, const double* __restrict__ V, unsigned long long* out) {
    double xm = 0.0, ym = 0.0;
    const long long n = (long long)G.nx * G.ny;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int ii = (int)(t % G.nx), jj = (int)(t / G.nx);
        const long long c = (long long)(jj + G.g) * G.pitch + (ii + G.g);
        const double rho = V[DENS * G.plane + c], pr = V[PRES * G.plane + c], gam = V[GAMM * G.plane + c];
        double cs;
        if (P.force_hydro) {
            cs = sqrt(gam * pr / rho);
        } else {
            const double bx = V[MAGX * G.plane + c], by = V[MAGY * G.plane + c], bz = V[MAGZ * G.plane + c];
            const double BB = bx * bx + by * by + bz * bz;
            const double bmin = fmin(fmin(fabs(bx), fabs(by)), fabs(bz));
            cs = c_fs(gam, rho, pr, BB, bmin, +1.0);
        }
        xm = fmax(xm, fabs(V[VELX * G.plane + c]) + cs);
        ym = fmax(ym, fabs(V[VELY * G.plane + c]) + cs);
    }
    for (int o = 16; o > 0; o >>= 1) {
        xm = fmax(xm, __shfl_xor_sync(0xffffffffu, xm, o));
        ym = fmax(ym, __shfl_xor_sync(0xffffffffu, ym, o));
    }
    __shared__ double sx[8], sy[8];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        sx[w] = xm;
        sy[w] = ym;
    }
    __syncthreads();
    if (w == 0) {
        xm = l < (int)(blockDim.x >> 5) ? sx[l] : 0.0;
        ym = l < (int)(blockDim.x >> 5) ? sy[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            xm = fmax(xm, __shfl_xor_sync(0xffffffffu, xm, o));
            ym = fmax(ym, __shfl_xor_sync(0xffffffffu, ym, o));
        }
        if (l == 0) {
            atomicMax(out + 0, (unsigned long long)__double_as_longlong(xm));
            atomicMax(out + 1, (unsigned long long)__double_as_longlong(ym));
        }
    }
}

// ------------------------------------------------------------------------
inline dim3 grid2(int nx, int ny) { return dim3((nx + BX - 1) / BX, (ny + BY - 1) / BY); }
const dim3 kBlock(BX, BY);

void face_pass1(const StageArgs& a, cudaStream_t s) {
    const dim3 grd = grid2(a.geo.nx + 5, a.geo.ny + 5);
    switch (a.geo.R) {
        case 1: k_face_pass1<1><<<grd, kBlock, 0, s>>>(a); break;
        case 2: k_face_pass1<2><<<grd, kBlock, 0, s>>>(a); break;
        default: k_face_pass1<3><<<grd, kBlock, 0, s>>>(a); break;
    }
}
void cascade_lower(const StageArgs& a, int mode, cudaStream_t s) {
    k_cascade_lower<<<grid2(a.geo.nx + 4, a.geo.ny + 4), kBlock, 0, s>>>(a, mode);
}
void recon_check(const StageArgs& a, const uint8_t* mask, cudaStream_t s) {
    k_recon_check<<<grid2(a.geo.nx + 4, a.geo.ny + 4), kBlock, 0, s>>>(a, mask);
}
void flux(const StageArgs& a, int mode, cudaStream_t s) {
    k_flux<<<grid2(a.geo.nx + 3, a.geo.ny + 3), kBlock, 0, s>>>(a, mode);
}
void ct_update_detect(const StageArgs& a, cudaStream_t s) {
    k_ct_update_detect<<<grid2(a.geo.nx + 1, a.geo.ny + 1), kBlock, 0, s>>>(a);
}
void mood_flags(const StageArgs& a, cudaStream_t s) { k_mood_flags<<<grid2(a.geo.nxt, a.geo.nyt), kBlock, 0, s>>>(a); }
void bc_fill(const Geo& G, double* A, int nvar, cudaStream_t s) {
    k_bc_fill<<<grid2(G.nxt, G.nyt), kBlock, 0, s>>>(G, A, nvar);
}
void rk_combine2(const Geo& G, const double* Un, const double* B, double* out, cudaStream_t s) {
    k_rk_combine2<<<grid2(G.nxt, G.nyt), kBlock, 0, s>>>(G, Un, B, out);
}
void rk_final(const Geo& G, const Phys& P, const double* Un, const double* B, double* outU, double* outV,
              cudaStream_t s) {
    k_rk_final<<<grid2(G.nxt, G.nyt), kBlock, 0, s>>>(G, P, Un, B, outU, outV);
}
void cons2prim_all(const Geo& G, const Phys& P, const double* U, double* V, cudaStream_t s) {
    k_cons2prim_all<<<grid2(G.nxt, G.nyt), kBlock, 0, s>>>(G, P, U, V);
}
void cfl_max(const Geo& G, const Phys& P, const double* V, unsigned long long* out2, cudaStream_t s) {
    long long n = (long long)G.nx * G.ny;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    k_cfl_max<<<blocks, 256, 0, s>>>(G, P, V, out2);
}

const KernelTable table = {
#if HOSONO_FAST
    "fast",
#else
    "strict",
#endif
    face_pass1, cascade_lower, recon_check, flux, ct_update_detect, mood_flags,
    bc_fill, rk_combine2, rk_final, cons2prim_all, cfl_max};

}  // namespace KNS

#if HOSONO_FAST
const KernelTable* kernels_fast() { return &kfast::table; }
#else
const KernelTable* kernels_strict() { return &kstrict::table; }
#endif

}  // namespace hosono
