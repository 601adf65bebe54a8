// physics.cuh -- pointwise ideal-MHD physics on the device (FP64).
//
// Each function keeps the operation order of the reference Fortran routine
// it cites, so that a build without FMA contraction (--fmad=false) rounds
// exactly like the reference's arithmetic statement by statement.  Fortran
// MAX/MIN become fmax/fmin (the non-NaN argument wins).
#pragma once

#include <cstdint>

namespace hosono {

// variable indices, src/definitions.f90:18-35 (0-based)
enum : int { DENS = 0, MOMX = 1, MOMY = 2, MOMZ = 3, ENER = 4, MAGX = 5, MAGY = 6, MAGZ = 7 };
enum : int { VELX = 1, VELY = 2, VELZ = 3, PRES = 4, EINT = 8, GAMM = 9 };
enum : int { XDIR = 0, YDIR = 1 };
enum : int { NORTH = 0, SOUTH = 1, EAST = 2, WEST = 3 };
constexpr int NCONS = 8;
constexpr int NPRIM = 10;

struct Phys {
    double gamma;
    double small_pressure;
    double small_density;
    double small_b;  // sim_smallB (eigen_beta_T only)
    int force_hydro;
};

// sim_forceHydro as a run-time flag (FH = -1) or as a compile-time constant
// (FH = 0: MHD, 1: hydro), for kernels instantiated per mode.  The
// expressions are the same either way; with a constant the compiler drops
// the other mode's branch and keeps the magnetic field of an MHD state in
// the registers of the conserved variables.
template <int FH>
__device__ __forceinline__ bool hydro(const Phys& s) {
    return FH < 0 ? s.force_hydro != 0 : FH != 0;
}

// src/eos.f90:9-26 (pressure floor)
__device__ __forceinline__ double eos_pres(const Phys& s, double dens, double eint) {
    double pres = (s.gamma - 1.0) * dens * eint;
    if (pres < s.small_pressure) pres = s.small_pressure;
    return pres;
}

// src/convert.f90:198-234
__device__ __forceinline__ void cons2prim(const Phys& s, const double* U, double* V) {
    double Bp;
    if (s.force_hydro)
        Bp = 0.0;
    else
        Bp = 0.5 * (U[MAGX] * U[MAGX] + U[MAGY] * U[MAGY] + U[MAGZ] * U[MAGZ]);
    const double density = U[DENS];
    const double velx = U[MOMX] / density;
    const double vely = U[MOMY] / density;
    const double velz = U[MOMZ] / density;
    const double eint = (U[ENER] - Bp) / density - 0.5 * (velx * velx + vely * vely + velz * velz);
    V[DENS] = density;
    V[VELX] = velx;
    V[VELY] = vely;
    V[VELZ] = velz;
    if (s.force_hydro) {
        V[MAGX] = 0.0;
        V[MAGY] = 0.0;
        V[MAGZ] = 0.0;
    } else {
        V[MAGX] = U[MAGX];
        V[MAGY] = U[MAGY];
        V[MAGZ] = U[MAGZ];
    }
    V[PRES] = eos_pres(s, density, eint);
    V[EINT] = eint;
    V[GAMM] = s.gamma;
}

// src/convert.f90:236-254 (not floored; SUM starts from zero)
template <int FH = -1>
__device__ __forceinline__ double cons2pres(const Phys& s, const double* U) {
    double Bp;
    if (hydro<FH>(s))
        Bp = 0.0;
    else
        Bp = 0.5 * ((0.0 + U[MAGX] * U[MAGX]) + U[MAGY] * U[MAGY] + U[MAGZ] * U[MAGZ]);
    const double msq = (0.0 + U[MOMX] * U[MOMX]) + U[MOMY] * U[MOMY] + U[MOMZ] * U[MOMZ];
    return (s.gamma - 1.0) * (U[ENER] - Bp - 0.5 * msq / U[DENS]);
}

// src/eigen.f90:305-321 (Ryu & Jones 1995, eqs. 2.18-2.19)
__device__ __forceinline__ double c_fs(double gam, double rho, double p, double BB, double B_N, double pm) {
    double c = (gam * p + BB) / rho;
    c = 0.5 * (c + pm * sqrt(c * c - 4.0 * gam * p * (B_N * B_N) / (rho * rho)));
    return sqrt(fmax(1.0e-14, c));
}

__device__ __forceinline__ double dot3(double a0, double a1, double a2, double b0, double b1, double b2) {
    return (0.0 + a0 * b0) + a1 * b1 + a2 * b2;
}

// Division policies for the Riemann solver.  Most of its quotients come in
// groups with one denominator (the density of a side, sR - sL, the HLL
// density, sK - sStar).
//
// IeeeDiv divides each one ('/': IEEE, correctly rounded).
//
// SharedRecipDiv takes y = RN(1/b) once per group (__drcp_rn, correctly
// rounded) and each quotient by Markstein's theorem (P. Markstein, "Computation
// of elementary functions on the IBM RISC System/6000 processor", IBM J. Res.
// Dev. 34(1), 1990): when y = RN(1/b) and q is within one ulp of a/b, the
// remainder r = a - b*q is exact and RN(q + r*y) = RN(a/b).  q0 = RN(a*y) is
// within two ulps of a/b; one correction q1 = RN(q0 + y*RN(a - b*q0)) brings
// it within one ulp, and a second gives the correctly rounded quotient -- the
// same bits as '/' (tests/div_check.cu compares the two on the GPU).  The
// proof assumes no overflow, underflow or subnormal in a, b, a*y and the
// remainders; every operand outside [2^-500, 2^501) (zero
// numerators excepted) clears `ok`, and the caller then recomputes the whole
// solve with IeeeDiv.  Cost per quotient: one multiply and four FMAs, no
// branch.
struct IeeeDiv {
    struct R {
        double b;
    };
    bool ok = true;
    __device__ __forceinline__ R recip(double b) { return R{b}; }
    __device__ __forceinline__ double div(double a, const R& r) { return a / r.b; }
};
struct SharedRecipDiv {
    struct R {
        double b, y;
    };
    bool ok = true;
    // |x| in [2^-500, 2^501), from the exponent bits (integer pipes)
    __device__ __forceinline__ static bool in_range(unsigned long long mag) {
        return (unsigned)((int)(mag >> 52) - (1023 - 500)) <= 1000u;
    }
    __device__ __forceinline__ R recip(double b) {
        ok = ok && in_range((unsigned long long)__double_as_longlong(b) & 0x7fffffffffffffffull);
        return R{b, __drcp_rn(b)};
    }
    __device__ __forceinline__ double div(double a, const R& r) {
        const unsigned long long mag = (unsigned long long)__double_as_longlong(a) & 0x7fffffffffffffffull;
        ok = ok && (mag == 0 || in_range(mag));
        const double q0 = a * r.y;
        const double q1 = fma(fma(-r.b, q0, a), r.y, q0);
        const double q2 = fma(fma(-r.b, q1, a), r.y, q1);
        return mag == 0 ? q0 : q2;  // a = +-0: q0 carries the sign of the IEEE quotient
    }
};

// The primitive variables HLLC reads from one side: cons2prim
// (convert.f90:198-234) without eint; b* are zero for a hydro run.
template <class D>
struct Side {
    double rho, vx, vy, vz, p, bx, by, bz;
    typename D::R rrho;  // the density as a shared denominator
};
template <int FH, class D>
__device__ __forceinline__ void side_prim(const Phys& s, const double* U, Side<D>& V, D& dv) {
    double Bp;
    if (hydro<FH>(s))
        Bp = 0.0;
    else
        Bp = 0.5 * (U[MAGX] * U[MAGX] + U[MAGY] * U[MAGY] + U[MAGZ] * U[MAGZ]);
    const double density = U[DENS];
    V.rho = density;
    V.rrho = dv.recip(density);
    V.vx = dv.div(U[MOMX], V.rrho);
    V.vy = dv.div(U[MOMY], V.rrho);
    V.vz = dv.div(U[MOMZ], V.rrho);
    const double eint = dv.div(U[ENER] - Bp, V.rrho) - 0.5 * (V.vx * V.vx + V.vy * V.vy + V.vz * V.vz);
    V.p = eos_pres(s, density, eint);
    V.bx = hydro<FH>(s) ? 0.0 : U[MAGX];
    V.by = hydro<FH>(s) ? 0.0 : U[MAGY];
    V.bz = hydro<FH>(s) ? 0.0 : U[MAGZ];
}
template <class D>
__device__ __forceinline__ double side_vel(const Side<D>& V, int c) {
    return c == 0 ? V.vx : c == 1 ? V.vy : V.vz;
}
template <class D>
__device__ __forceinline__ double side_mag(const Side<D>& V, int c) {
    return c == 0 ? V.bx : c == 1 ? V.by : V.bz;
}

// fast magnetosonic speed of one side or of the average state (eigen.f90:257-303)
__device__ __forceinline__ double side_cf(const Phys& s, double rho0, double p0, double bx, double by, double bz,
                                          double bN) {
    const double rho = fmax(rho0, s.small_density);
    const double p = fmax(p0, s.small_pressure);
    const double BB = bx * bx + by * by + bz * bz;
    return c_fs(s.gamma, rho, p, BB, bN, +1.0);
}

// cons2flux (convert.f90:28-92) of one side
template <int FH, class D>
__device__ __forceinline__ void side_flux(const Phys& s, const double* U, const Side<D>& V, int dir, double* F,
                                          D& dv) {
    double Bp = 0.0;
    if (!hydro<FH>(s)) Bp = 0.5 * (U[MAGX] * U[MAGX] + U[MAGY] * U[MAGY] + U[MAGZ] * U[MAGZ]);
    const double E = U[ENER];
    const double Ptot = V.p + Bp;
    // normal (N) and tangential (T1, T2 = z) components; the array slots are
    // chosen by selects, so a run-time dir keeps F and U in registers
    const bool x = dir == XDIR;
    const double vN = side_vel(V, dir), vT1 = side_vel(V, 1 - dir), vT2 = V.vz;
    const double BN = side_mag(V, dir), BT1 = side_mag(V, 1 - dir), BT2 = V.bz;
    const double mN = x ? U[MOMX] : U[MOMY];
    double fN = dv.div(mN * mN, V.rrho) + Ptot;
    double fT1 = mN * vT1;
    double fT2 = mN * vT2;
    double fE = (E + Ptot) * vN;
    double gT1 = 0.0, gT2 = 0.0;  // induction fluxes; the normal one is 0
    if (!hydro<FH>(s)) {
        fN = fN - BN * BN;
        fT1 = fT1 - BT1 * BN;
        fT2 = fT2 - BT2 * BN;
        gT1 = vN * BT1 - vT1 * BN;
        gT2 = vN * BT2 - vT2 * BN;
        fE = fE - BN * (V.vx * V.bx + V.vy * V.by + V.vz * V.bz);
    }
    F[DENS] = mN;
    F[MOMX] = x ? fN : fT1;
    F[MOMY] = x ? fT1 : fN;
    F[MOMZ] = fT2;
    F[ENER] = fE;
    F[MAGX] = x ? 0.0 : gT1;
    F[MAGY] = x ? gT1 : 0.0;
    F[MAGZ] = gT2;
}

// src/riemannSolver.f90:68-221 (HLLC for MHD, Li 2005).  Every value keeps
// the reference's expression; what the chosen branch does not read is not
// computed: a supersonic face (flux = fL or fR) evaluates one physical flux
// and no HLL or star state, and the star state is evaluated once, on the
// operands of the chosen side.
template <int FH, class D>
__device__ __forceinline__ void hllc_t(const Phys& s, const double* uL, const double* uR, int dir, double* flux,
                                       D& dv) {
    Side<D> L, R;
    side_prim<FH>(s, uL, L, dv);
    side_prim<FH>(s, uR, R, dv);
    // array slots of the normal / first tangential components are chosen by
    // selects, so a run-time dir keeps every array in registers
    const bool x = dir == XDIR;
    const double velNL = side_vel(L, dir), velNR = side_vel(R, dir);
    const double magNL = side_mag(L, dir), magNR = side_mag(R, dir);
    // eigenvalues 1 and 7 of L, R and the arithmetic average (riemannSolver.f90:84-96)
    const double eL1 = velNL - side_cf(s, L.rho, L.p, L.bx, L.by, L.bz, magNL);
    const double eR7 = velNR + side_cf(s, R.rho, R.p, R.bx, R.by, R.bz, magNR);
    double sL, sR;
    {
        const double vNA = (velNL + velNR) / 2.0;
        const double cfA = side_cf(s, (L.rho + R.rho) / 2.0, (L.p + R.p) / 2.0, (L.bx + R.bx) / 2.0,
                                   (L.by + R.by) / 2.0, (L.bz + R.bz) / 2.0, (magNL + magNR) / 2.0);
        sL = fmin(eL1, vNA - cfA);
        sR = fmax(vNA + cfA, eR7);
    }
    const double rhoL = L.rho, rhoR = R.rho;
    const double pTotL = L.p + 0.5 * dot3(L.bx, L.by, L.bz, L.bx, L.by, L.bz);
    const double pTotR = R.p + 0.5 * dot3(R.bx, R.by, R.bz, R.bx, R.by, R.bz);
    const double dL = sL - velNL, dR = sR - velNR;
    const double mNL = x ? uL[MOMX] : uL[MOMY], mNR = x ? uR[MOMX] : uR[MOMY];
    const double sStr = (mNR * dR - mNL * dL + pTotL - pTotR - magNL * magNL + magNR * magNR) /
                        (rhoR * dR - rhoL * dL);
    // final choice (riemannSolver.f90:189-219): fL if 0 < sL; left star state
    // if sL <= 0 < sStr; right star state if sStr <= 0 <= sR; fR otherwise.
    int side;
    if (0.0 < sL)
        side = 0;
    else if ((sL <= 0.0) && (0.0 < sStr))
        side = 1;
    else if ((sStr <= 0.0) && (0.0 <= sR))
        side = 2;
    else
        side = 3;
    if (side == 0 || side == 3) {
        if (side == 0)
            side_flux<FH>(s, uL, L, dir, flux, dv);
        else
            side_flux<FH>(s, uR, R, dir, flux, dv);
        return;
    }
    double fL[NCONS], fR[NCONS];
    side_flux<FH>(s, uL, L, dir, fL, dv);
    side_flux<FH>(s, uR, R, dir, fR, dv);
    double uHLL[NCONS];
    const typename D::R rS = dv.recip(sR - sL);
#pragma unroll
    for (int v = 0; v < NCONS; v++)
        if (v != ENER) uHLL[v] = dv.div(sR * uR[v] - sL * uL[v] + fL[v] - fR[v], rS);
    const typename D::R rH = dv.recip(uHLL[DENS]);
    const double velHx = dv.div(uHLL[MOMX], rH);
    const double velHy = dv.div(uHLL[MOMY], rH);
    const double velHz = dv.div(uHLL[MOMZ], rH);
    const double magDotVelHLL = dot3(uHLL[MAGX], uHLL[MAGY], uHLL[MAGZ], velHx, velHy, velHz);
    const double magNHLL = x ? uHLL[MAGX] : uHLL[MAGY];
    const double magT1HLL = x ? uHLL[MAGY] : uHLL[MAGX];
    const double pStr = rhoL * dL * (sStr - velNL) + pTotL - magNL * magNL + magNHLL * magNHLL;
    const bool left = side == 1;
    const Side<D>& K = left ? L : R;
    const double sK = left ? sL : sR;
    const double dK = left ? dL : dR;
    const double velNK = left ? velNL : velNR;
    const double pTotK = left ? pTotL : pTotR;
    const double magNK = left ? magNL : magNR;
    const double magDotVelK = dot3(K.bx, K.by, K.bz, K.vx, K.vy, K.vz);
    const double vT1K = side_vel(K, 1 - dir), vT2K = K.vz;
    const double bT1K = side_mag(K, 1 - dir), bT2K = K.bz;
    const double eK = left ? uL[ENER] : uR[ENER];
    const typename D::R rK = dv.recip(sK - sStr);
    double uStr[NCONS];
    uStr[DENS] = dv.div(K.rho * dK, rK);
    const double sN = uStr[DENS] * sStr;
    const double sT1 = uStr[DENS] * vT1K - dv.div(magNHLL * magT1HLL - magNK * bT1K, rK);
    const double sT2 = uStr[DENS] * vT2K - dv.div(magNHLL * uHLL[MAGZ] - magNK * bT2K, rK);
    uStr[MOMX] = x ? sN : sT1;
    uStr[MOMY] = x ? sT1 : sN;
    uStr[MOMZ] = sT2;
    uStr[MAGX] = x ? magNHLL : magT1HLL;
    uStr[MAGY] = x ? magT1HLL : magNHLL;
    uStr[MAGZ] = uHLL[MAGZ];
    uStr[ENER] = eK * dK + pStr * sStr - pTotK * velNK - magNHLL * magDotVelHLL + magNK * magDotVelK;
    uStr[ENER] = dv.div(uStr[ENER], rK);
#pragma unroll
    for (int v = 0; v < NCONS; v++) flux[v] = (left ? fL[v] : fR[v]) + sK * (uStr[v] - (left ? uL[v] : uR[v]));
}

// the Riemann solver with IEEE division throughout (the rare fallback)
template <int FH>
static __device__ __noinline__ void hllc_ieee(const Phys& s, const double* uL, const double* uR, int dir, double* flux) {
    IeeeDiv dv;
    hllc_t<FH>(s, uL, uR, dir, flux, dv);
}

// HLLC with shared reciprocals; any operand outside their proven range sends
// the whole solve through IEEE division instead (same result bits either way)
template <int FH = -1>
__device__ __forceinline__ void hllc(const Phys& s, const double* uL, const double* uR, int dir, double* flux) {
    SharedRecipDiv dv;
    hllc_t<FH>(s, uL, uR, dir, flux, dv);
    if (!dv.ok) hllc_ieee<FH>(s, uL, uR, dir, flux);
}


// ----------------------------------------------------------------------
// eigen_vecsFromPrim (src/eigen.f90:20-255) with eigen_alpha_fs (:323-349)
// and eigen_beta_T (:351-371): the left and right eigenvectors of the 7 MHD
// waves, in primitive or (cons) conserved variables.  Not on the time-step
// path (no .par option of the reference uses it); exposed by
// hosono_gpu_eigenvecs.  Statement order of the reference; MATMUL as sums
// over k ascending from zero.
// alpha_f for pm = +1, alpha_s for pm = -1
__device__ __forceinline__ double eigen_alpha_fs(double c_f, double c_s, double a, double BB, double B_N, double pm) {
    double BB_T = BB - B_N * B_N;
    (void)BB_T;  // computed by the reference, unused
    double cf2_minus_cs2 = c_f * c_f - c_s * c_s;
    double alpha;
    if (cf2_minus_cs2 > 1.0e-14) {
        alpha = 0.5 * (cf2_minus_cs2) + pm * (a * a - 0.5 * (c_f * c_f + c_s * c_s));
        alpha = alpha / (cf2_minus_cs2);
    } else if (pm > 0) {
        alpha = 1.0;
    } else {
        alpha = 0.0;
    }
    alpha = fmin(1.0, fmax(0.0, alpha));
    return sqrt(alpha);
}
// src/eigen.f90:351-371
__device__ __forceinline__ double eigen_beta_T(double B_T1, double B_T2, double smallB) {
    double BB_T = B_T1 * B_T1 + B_T2 * B_T2;
    if (BB_T < smallB * smallB) return copysign(1.0, B_T1) / sqrt(2.0);
    return B_T1 / sqrt(fmax(BB_T, 1.0e-30));
}
// src/eigen.f90:20-255: right eigenvectors (columns of R) and left
// eigenvectors (columns of L) of the 7 MHD waves in direction dir, 8x8
// column-major with the variable index as the row; cons: converted to
// conserved variables by dU/dV and dV/dU (MATMUL as k-ascending sums from 0)
__device__ inline void eigen_vecs(const Phys& s, const double* V, int dir, bool cons, double* Lm, double* Rm) {
    const int vN = dir == XDIR ? VELX : VELY, vT1 = dir == XDIR ? VELY : VELX, vT2 = VELZ;
    const int bN = dir == XDIR ? MAGX : MAGY, bT1 = dir == XDIR ? MAGY : MAGX, bT2 = MAGZ;
#define R(r, c) Rm[(r) + NCONS * ((c) - 1)]
#define L(r, c) Lm[(r) + NCONS * ((c) - 1)]
    const double rho = fmax(V[DENS], s.small_density);
    const double velN = V[vN], velT1 = V[vT1], velT2 = V[vT2];
    const double B_N = V[bN], B_T1 = V[bT1], B_T2 = V[bT2];
    const double p = fmax(V[PRES], s.small_pressure);
    const double gam = V[GAMM];
    const double BB = B_N * B_N + B_T1 * B_T1 + B_T2 * B_T2;
    const double c_f = c_fs(gam, rho, p, BB, B_N, +1.0);
    const double c_s = c_fs(gam, rho, p, BB, B_N, -1.0);
    const double a = sqrt(gam * p / rho);
    const double alpha_f = eigen_alpha_fs(c_f, c_s, a, BB, B_N, +1.0);
    const double alpha_s = eigen_alpha_fs(c_f, c_s, a, BB, B_N, -1.0);
    const double beta_T1 = eigen_beta_T(B_T1, B_T2, s.small_b);
    const double beta_T2 = eigen_beta_T(B_T2, B_T1, s.small_b);
    const double sgnBn = copysign(1.0, B_N);
    const double sr = sqrt(rho);
    for (int k = 0; k < NCONS * NCONS; k++) Rm[k] = Lm[k] = 0.0;
    R(DENS, 1) = alpha_f * rho;
    R(vN, 1) = -alpha_f * c_f;
    R(vT1, 1) = alpha_s * c_s * beta_T1 * sgnBn;
    R(vT2, 1) = alpha_s * c_s * beta_T2 * sgnBn;
    R(bT1, 1) = alpha_s * sr * a * beta_T1;
    R(bT2, 1) = alpha_s * sr * a * beta_T2;
    R(PRES, 1) = alpha_f * rho * (a * a);
    R(vT1, 2) = -beta_T2;
    R(vT2, 2) = beta_T1;
    R(bT1, 2) = -sr * beta_T2 * sgnBn;
    R(bT2, 2) = sr * beta_T1 * sgnBn;
    R(DENS, 3) = alpha_s * rho;
    R(vN, 3) = -alpha_s * c_s;
    R(vT1, 3) = -alpha_f * c_f * beta_T1 * sgnBn;
    R(vT2, 3) = -alpha_f * c_f * beta_T2 * sgnBn;
    R(bT1, 3) = -alpha_f * sr * a * beta_T1;
    R(bT2, 3) = -alpha_f * sr * a * beta_T2;
    R(PRES, 3) = alpha_s * rho * (a * a);
    R(DENS, 4) = 1.0;
    R(DENS, 5) = alpha_s * rho;
    R(vN, 5) = alpha_s * c_s;
    R(vT1, 5) = alpha_f * c_f * beta_T1 * sgnBn;
    R(vT2, 5) = alpha_f * c_f * beta_T2 * sgnBn;
    R(bT1, 5) = -alpha_f * sr * a * beta_T1;
    R(bT2, 5) = -alpha_f * sr * a * beta_T2;
    R(PRES, 5) = alpha_s * rho * (a * a);
    R(vT1, 6) = beta_T2;
    R(vT2, 6) = -beta_T1;
    R(bT1, 6) = -sr * beta_T2 * sgnBn;
    R(bT2, 6) = sr * beta_T1 * sgnBn;
    R(DENS, 7) = alpha_f * rho;
    R(vN, 7) = alpha_f * c_f;
    R(vT1, 7) = -alpha_s * c_s * beta_T1 * sgnBn;
    R(vT2, 7) = -alpha_s * c_s * beta_T2 * sgnBn;
    R(bT1, 7) = alpha_s * sr * a * beta_T1;
    R(bT2, 7) = alpha_s * sr * a * beta_T2;
    R(PRES, 7) = alpha_f * rho * (a * a);
    const double h = 1 / (2 * (a * a));
    L(vN, 1) = h * (-alpha_f * c_f);
    L(vT1, 1) = h * (alpha_s * c_s * beta_T1 * sgnBn);
    L(vT2, 1) = h * (alpha_s * c_s * beta_T2 * sgnBn);
    L(bT1, 1) = h * (alpha_s * a * beta_T1 / sr);
    L(bT2, 1) = h * (alpha_s * a * beta_T2 / sr);
    L(PRES, 1) = h * (alpha_f / rho);
    L(vT1, 2) = 0.5 * (-beta_T2);
    L(vT2, 2) = 0.5 * (beta_T1);
    L(bT1, 2) = 0.5 * (-beta_T2 * sgnBn / sr);
    L(bT2, 2) = 0.5 * (beta_T1 * sgnBn / sr);
    L(vN, 3) = h * (-alpha_s * c_s);
    L(vT1, 3) = h * (-alpha_f * c_f * beta_T1 * sgnBn);
    L(vT2, 3) = h * (-alpha_f * c_f * beta_T2 * sgnBn);
    L(bT1, 3) = h * (-alpha_f * a * beta_T1 / sr);
    L(bT2, 3) = h * (-alpha_f * a * beta_T2 / sr);
    L(PRES, 3) = h * (alpha_s / rho);
    L(DENS, 4) = 1.0;
    L(PRES, 4) = -1 / (a * a);
    L(vN, 5) = h * (alpha_s * c_s);
    L(vT1, 5) = h * (alpha_f * c_f * beta_T1 * sgnBn);
    L(vT2, 5) = h * (alpha_f * c_f * beta_T2 * sgnBn);
    L(bT1, 5) = h * (-alpha_f * a * beta_T1 / sr);
    L(bT2, 5) = h * (-alpha_f * a * beta_T2 / sr);
    L(PRES, 5) = h * (alpha_s / rho);
    L(vT1, 6) = 0.5 * (beta_T2);
    L(vT2, 6) = 0.5 * (-beta_T1);
    L(bT1, 6) = 0.5 * (-beta_T2 * sgnBn / sr);
    L(bT2, 6) = 0.5 * (beta_T1 * sgnBn / sr);
    L(vN, 7) = h * (alpha_f * c_f);
    L(vT1, 7) = h * (-alpha_s * c_s * beta_T1 * sgnBn);
    L(vT2, 7) = h * (-alpha_s * c_s * beta_T2 * sgnBn);
    L(bT1, 7) = h * (alpha_s * a * beta_T1 / sr);
    L(bT2, 7) = h * (alpha_s * a * beta_T2 / sr);
    L(PRES, 7) = h * (alpha_f / rho);
    if (!cons) {
#undef R
#undef L
        return;
    }
#undef R
#undef L
    const double k = 1.0 - gam;
    double dUdV[NCONS * NCONS] = {}, dVdU[NCONS * NCONS] = {};
#define A(r, c) dUdV[(r) + NCONS * (c)]
#define Bm(r, c) dVdU[(r) + NCONS * (c)]
    A(DENS, DENS) = 1.0;
    A(VELX, DENS) = V[VELX];
    A(VELY, DENS) = V[VELY];
    A(VELZ, DENS) = V[VELZ];
    A(PRES, DENS) = 0.5 * (velN * velN + velT1 * velT1 + velT2 * velT2);
    A(VELX, VELX) = rho;
    A(PRES, VELX) = rho * V[VELX];
    A(VELY, VELY) = rho;
    A(PRES, VELY) = rho * V[VELY];
    A(VELZ, VELZ) = rho;
    A(PRES, VELZ) = rho * V[VELZ];
    A(MAGX, MAGX) = 1.0;
    A(PRES, MAGX) = V[MAGX];
    A(MAGY, MAGY) = 1.0;
    A(PRES, MAGY) = V[MAGY];
    A(MAGZ, MAGZ) = 1.0;
    A(PRES, MAGZ) = V[MAGZ];
    A(PRES, PRES) = -1 / k;
    Bm(DENS, DENS) = 1.0;
    Bm(VELX, DENS) = -V[VELX] / rho;
    Bm(VELY, DENS) = -V[VELY] / rho;
    Bm(VELZ, DENS) = -V[VELZ] / rho;
    Bm(PRES, DENS) = -k * A(PRES, DENS);
    Bm(VELX, VELX) = 1 / rho;
    Bm(PRES, VELX) = k * V[VELX];
    Bm(VELY, VELY) = 1 / rho;
    Bm(PRES, VELY) = k * V[VELY];
    Bm(VELZ, VELZ) = 1 / rho;
    Bm(PRES, VELZ) = k * V[VELZ];
    Bm(MAGX, MAGX) = 1.0;
    Bm(PRES, MAGX) = k * V[MAGX];
    Bm(MAGY, MAGY) = 1.0;
    Bm(PRES, MAGY) = k * V[MAGY];
    Bm(MAGZ, MAGZ) = 1.0;
    Bm(PRES, MAGZ) = k * V[MAGZ];
    Bm(PRES, PRES) = -k;
    double Rc[NCONS * NCONS], Lc[NCONS * NCONS];
    for (int j = 0; j < NCONS; j++)
        for (int i = 0; i < NCONS; i++) {
            double r = 0.0, l = 0.0;
            for (int q = 0; q < NCONS; q++) {
                r = r + A(i, q) * Rm[q + NCONS * j];
                l = l + Bm(q, i) * Lm[q + NCONS * j];
            }
            Rc[i + NCONS * j] = r;
            Lc[i + NCONS * j] = l;
        }
#undef A
#undef Bm
    for (int q = 0; q < NCONS * NCONS; q++) {
        Rm[q] = Rc[q];
        Lm[q] = Lc[q];
    }
}

// src/detect.f90:250-265 (CAD) and :238-248 (PAD): both finite (not NaN,
// not infinite) and both > 0, i.e. each bit pattern is a positive, nonzero,
// finite double (tested on the integer pipes)
__device__ __forceinline__ bool positive_finite(double x) {
    const unsigned long long u = (unsigned long long)__double_as_longlong(x);
    return u - 1ull < 0x7fefffffffffffffull;  // u in [1, 0x7fefffffffffffff]
}
__device__ __forceinline__ bool admissible(double dens, double pres) {
    return positive_finite(dens) && positive_finite(pres);
}

}  // namespace hosono
