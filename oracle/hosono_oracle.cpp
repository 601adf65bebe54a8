// hosono_oracle.cpp -- CPU oracle for the hosono-2DMHD time-step path.
//
// TEST INFRASTRUCTURE ONLY: this file is the checker the CUDA path is
// compared against.  It restates the reference's Fortran line by line, in
// the reference's own data layout (AoS, var fastest, guard cells included,
// 1-based indices emulated), with the same loop ranges, the same serial
// lowering passes and the same arithmetic order.  It is compiled twice:
//   * strict  (-ffp-contract=off): every +,-,*,/ rounded on its own.  This is
//     the parity build; the CUDA strict path matches it bit for bit.
//   * fast    (-ffp-contract=fast, -march): the closest stand-in for the
//     reference's `make release` flags; used only to time the CPU baseline.
// Each function cites the Fortran file:line it follows (paths relative to
// the reference project's root).
//
// Fortran MAX/MIN with a NaN argument are unspecified (gfortran >= 9); this
// restatement uses fmax/fmin (the non-NaN argument wins), the same rule the
// CUDA path uses.

#include "hosono_oracle.h"

#include <quadmath.h>
#include <omp.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <fstream>
#include <sstream>
#include <algorithm>

// phase markers for the operation-counting build (flopcount.h); no-ops here
#ifndef FC_PHASE
#define FC_PHASE(p) ((void)0)
#endif

namespace {

// ---------------------------------------------------------------- constants
// src/definitions.f90:6-35 (0-based here)
enum { DENS = 0, MOMX = 1, MOMY = 2, MOMZ = 3, ENER = 4, MAGX = 5, MAGY = 6, MAGZ = 7 };
enum { VELX = 1, VELY = 2, VELZ = 3, PRES = 4, EINT = 8, GAMM = 9 };
enum { XDIR = 0, YDIR = 1 };
enum { NORTH = 0, SOUTH = 1, EAST = 2, WEST = 3 };
constexpr int NCONS = 8;
constexpr int NPRIM = 10;
const double PI = 3.14159265358979323846;  // ACOS(-1.0), definitions.f90:39

typedef __float128 qp;

// ---------------------------------------------------------------- settings
// src/simulation.f90:9-31
struct Sim {
    double gamma = 0, smallB = 0, smallPressure = 0, smallDensity = 0, smallEnergy = 0;
    double cfl = 0, tmax = 0, outputFreqTime = 0;
    int nstepmax = 0, outputFreqStep = 0;
    bool forceHydro = false;
    int bc = 0;  // 0 outflow, 1 periodic (sim_BC)
    int riemannID = 1;
};

// ---------------------------------------------------------------- GP tables
// src/GP.f90:28-33
struct GPTab {
    int R = 0, nsMax = 0, nqMax = 0;
    std::vector<int> nStenc, nQuad;   // [rr-1]
    std::vector<int> stenc;           // (2, nsMax, R)
    std::vector<double> pv;           // (nsMax, nqMax, 4, R)
    std::vector<double> qw;           // (nqMax, R)
    std::vector<double> qpts;         // (nqMax, R)
    int sx(int k, int rr) const { return stenc[0 + 2 * ((k - 1) + nsMax * (rr - 1))]; }
    int sy(int k, int rr) const { return stenc[1 + 2 * ((k - 1) + nsMax * (rr - 1))]; }
    double p(int k, int q, int f, int rr) const {  // f 0-based face, k,q,rr 1-based
        return pv[(k - 1) + nsMax * ((q - 1) + nqMax * (f + 4 * (rr - 1)))];
    }
    double w(int q, int rr) const { return qw[(q - 1) + nqMax * (rr - 1)]; }
};

// ---------------------------------------------------------------- the block
// src/gridBlock.f90:33-90, src/gridState.f90:34-41
struct Block {
    int NGC = 0, N[2] = {0, 0}, minIdx[2] = {1, 1}, maxIdx[2] = {0, 0}, strt[2] = {0, 0}, stop[2] = {0, 0};
    int nTot[2] = {0, 0};
    double domBeg[2] = {0, 0}, domEnd[2] = {0, 0}, dl[2] = {0, 0}, mindxdy = 0, maxdxdy = 0;
    std::vector<double> x, y;  // index i-1
    int nqMax = 0;
    std::vector<double> faceVals;  // (8, nqMax, 4, nx, ny)
    std::vector<double> flux, fluxRaw;  // (8, 2, nx, ny)
    std::vector<int> scheme;
    std::vector<char> recompute, recomputeFLICD;

    size_t ncell() const { return (size_t)nTot[0] * nTot[1]; }
    size_t c(int i, int j) const { return (size_t)(i - 1) + (size_t)nTot[0] * (size_t)(j - 1); }
    double* fv(int q, int f, int i, int j) { return &faceVals[NCONS * ((q - 1) + nqMax * (f + 4 * c(i, j)))]; }
    double* fl(int d, int i, int j) { return &flux[NCONS * (d + 2 * c(i, j))]; }
    double* flr(int d, int i, int j) { return &fluxRaw[NCONS * (d + 2 * c(i, j))]; }
};

struct Trace {
    int stage, pass, nInner, nDetect;
    std::vector<unsigned char> inner, detect;
};

}  // namespace

struct orc_handle {
    Sim sim;
    GPTab gp;
    Block blk;
    std::vector<double> U, V;  // (8|10, nx, ny)
    std::vector<double> Unew;  // stage output of the per-module entry points
    double ellOverDelta = 0;
    bool trace = false;
    int stageCounter = 0;
    std::vector<Trace> traces;
};

namespace {

// ================================================================ .par reader
// src/readParamFile.f90:131-182: the first non-comment line whose text before
// '=' (trailing blanks trimmed, leading blanks kept) equals the key; the text
// after '#' is dropped; the value is what follows '='.
bool read_value_string(const std::string& file, const std::string& key, std::string& out) {
    std::ifstream in(file);
    if (!in) return false;
    std::string line;
    while (std::getline(in, line)) {
        if (!line.empty() && line[0] == '#') continue;
        size_t h = line.find('#');
        if (h != std::string::npos) line = line.substr(0, h);
        size_t e = line.find('=');
        if (e == std::string::npos) continue;
        std::string name = line.substr(0, e);
        while (!name.empty() && (name.back() == ' ' || name.back() == '\t' || name.back() == '\r')) name.pop_back();
        if (name == key) {
            out = line.substr(e + 1);
            return true;
        }
    }
    return false;
}

// list-directed read of the first item of a value string
std::string first_token(const std::string& s) {
    size_t a = s.find_first_not_of(" \t\r");
    if (a == std::string::npos) return "";
    if (s[a] == '\'' || s[a] == '"') {
        char qch = s[a];
        size_t b = s.find(qch, a + 1);
        return s.substr(a + 1, b == std::string::npos ? std::string::npos : b - a - 1);
    }
    size_t b = s.find_first_of(" \t\r,/", a);
    return s.substr(a, b == std::string::npos ? std::string::npos : b - a);
}

std::string fortran_real_text(std::string t) {
    for (auto& ch : t)
        if (ch == 'd' || ch == 'D') ch = 'e';
    return t;
}

struct ParError {
    std::string msg;
};

std::string par_str(const std::string& f, const std::string& k) {
    std::string v;
    if (!read_value_string(f, k, v)) throw ParError{"parameter '" + k + "' was not found inside of '" + f + "'"};
    return first_token(v);
}
double par_real(const std::string& f, const std::string& k) {
    return std::strtod(fortran_real_text(par_str(f, k)).c_str(), nullptr);
}
double par_real_opt(const std::string& f, const std::string& k, double dflt) {
    std::string v;
    if (!read_value_string(f, k, v)) return dflt;
    return std::strtod(fortran_real_text(first_token(v)).c_str(), nullptr);
}
int par_int(const std::string& f, const std::string& k) { return std::atoi(par_str(f, k).c_str()); }
bool par_logical(const std::string& f, const std::string& k) {
    std::string t = par_str(f, k);
    size_t i = 0;
    if (i < t.size() && t[i] == '.') i++;
    return i < t.size() && (t[i] == 't' || t[i] == 'T');
}

// ================================================================ GP set-up
// src/GP.f90:216-280  GP_volAvgToVolAvgSqExpKernel
qp gp_kernel_vv(const qp p1[2], const qp p2[2], const qp dl[2], qp ell) {
    const qp sqrt_two = sqrtq((qp)2);
    const qp qpi = M_PIq;
    qp sqrt2_ell = sqrt_two * ell;
    qp two_ell_sq = (qp)2 * (ell * ell);
    qp sqrt_pi_ell_sq = sqrtq(qpi) * (ell * ell);
    qp kernel = (qp)1;
    for (int i = 0; i < 2; i++) {
        qp sep = p1[i] - p2[i];
        qp r1 = (sep + dl[i]) / sqrt2_ell;
        qp r2 = (sep - dl[i]) / sqrt2_ell;
        qp r3 = -(((sep + dl[i]) * (sep + dl[i])) / two_ell_sq);
        qp r4 = -(((sep - dl[i]) * (sep - dl[i])) / two_ell_sq);
        qp r5 = sep / sqrt2_ell;
        qp r6 = -((sep * sep) / two_ell_sq);
        qp bracket = ((r1 * erfq(r1) + r2 * erfq(r2)) + (expq(r3) + expq(r4)) / sqrtq(qpi))
                     - (qp)2 * (r5 * erfq(r5) + expq(r6) / sqrtq(qpi));
        kernel = ((kernel * sqrt_pi_ell_sq) / (dl[i] * dl[i])) * bracket;
    }
    return kernel;
}

// src/GP.f90:282-335  GP_volAvgToPointSqExpKernel
qp gp_kernel_vp(const qp p1[2], const qp p2[2], const qp dl[2], qp ell) {
    const qp sqrt_two = sqrtq((qp)2);
    const qp sqrt_half_pi = sqrtq(M_PIq / (qp)2);
    qp sqrt2_ell = sqrt_two * ell;
    qp kernel = (qp)1;
    for (int i = 0; i < 2; i++) {
        qp half_delta = dl[i] / (qp)2;
        qp sep = p1[i] - p2[i];
        qp r1 = (sep + half_delta) / sqrt2_ell;
        qp r2 = (sep - half_delta) / sqrt2_ell;
        kernel = ((kernel * sqrt_half_pi) * (ell / dl[i])) * (erfq(r1) - erfq(r2));
    }
    return kernel;
}

// src/linAlgQuadPrecision.f90:107-144 (Cholesky, A = R^T R), :146-175
// (forward substitution), :206-235 (back substitution), :336-365 (solveSPD).
// A is m x m (row-major a[i*m+j]), b is m x n; returns x (m x n).
bool solve_spd(int m, int n, const std::vector<qp>& A, const std::vector<qp>& b, std::vector<qp>& x) {
    std::vector<qp> R(A);
    for (int k = 0; k < m - 1; k++)
        for (int i = k + 1; i < m; i++) R[i * m + k] = 0;
    for (int k = 0; k < m; k++) {
        if (!(R[k * m + k] > 0)) return false;  // "A is not positive definite"
        for (int j = k + 1; j < m; j++)
            for (int l = j; l < m; l++) R[j * m + l] = R[j * m + l] - (R[k * m + l] * R[k * m + j]) / R[k * m + k];
        qp s = sqrtq(R[k * m + k]);
        for (int l = k; l < m; l++) R[k * m + l] = R[k * m + l] / s;
    }
    // forward substitution with L = R^T: L(i,j) = R(j,i)
    std::vector<qp> y((size_t)m * n), ss(n);
    for (int c = 0; c < n; c++) y[0 * n + c] = b[0 * n + c] / R[0];
    for (int i = 1; i < m; i++) {
        for (int c = 0; c < n; c++) ss[c] = 0;
        for (int j = 0; j < i; j++)
            for (int c = 0; c < n; c++) ss[c] = ss[c] + R[j * m + i] * y[j * n + c];
        for (int c = 0; c < n; c++) y[i * n + c] = (b[i * n + c] - ss[c]) / R[i * m + i];
    }
    // back substitution with U = R
    x.assign((size_t)m * n, 0);
    for (int c = 0; c < n; c++) x[(m - 1) * n + c] = y[(m - 1) * n + c] / R[(m - 1) * m + (m - 1)];
    for (int i = m - 2; i >= 0; i--) {
        for (int c = 0; c < n; c++) ss[c] = 0;
        for (int j = i + 1; j < m; j++)
            for (int c = 0; c < n; c++) ss[c] = ss[c] + R[i * m + j] * x[j * n + c];
        for (int c = 0; c < n; c++) x[i * n + c] = (y[i * n + c] - ss[c]) / R[i * m + i];
    }
    return true;
}

// src/GP.f90:37-200  GP_init
bool gp_build(int R, qp dl[2], qp ellOverDelta, GPTab& gp, std::string& err) {
    if (R < 1 || R > 3) {
        err = "GP radius must be 1, 2 or 3";
        return false;
    }
    qp ell = ellOverDelta * (dl[0] < dl[1] ? dl[0] : dl[1]);  // :66 (MINVAL(dl))
    gp.R = R;
    gp.nStenc.resize(R);
    gp.nQuad.resize(R);
    for (int rr = 1; rr <= R; rr++) {  // :73-77
        gp.nStenc[rr - 1] = 1 + 2 * rr * (rr + 1);
        gp.nQuad[rr - 1] = rr + 1;
    }
    gp.nsMax = gp.nStenc[R - 1];
    gp.nqMax = gp.nQuad[R - 1];
    gp.stenc.assign((size_t)2 * gp.nsMax * R, 0);
    for (int rr = 1; rr <= R; rr++) {  // :85-95
        int counter = 0;
        for (int i = -rr; i <= rr; i++)
            for (int j = -rr; j <= rr; j++)
                if (std::abs(i) + std::abs(j) <= rr) {
                    counter++;
                    gp.stenc[0 + 2 * ((counter - 1) + gp.nsMax * (rr - 1))] = i;
                    gp.stenc[1 + 2 * ((counter - 1) + gp.nsMax * (rr - 1))] = j;
                }
    }
    gp.pv.assign((size_t)gp.nsMax * gp.nqMax * 4 * R, 0.0);
    gp.qw.assign((size_t)gp.nqMax * R, 0.0);
    gp.qpts.assign((size_t)gp.nqMax * R, 0.0);
    for (int rr = 1; rr <= R; rr++) {
        int nq = gp.nQuad[rr - 1], ns = gp.nStenc[rr - 1], np = 4 * nq;
        std::vector<qp> XX(2 * ns), XXs(2 * np), qpt(nq);
        for (int k = 0; k < ns; k++) {  // :114-115
            XX[0 + 2 * k] = (qp)gp.stenc[0 + 2 * (k + gp.nsMax * (rr - 1))] * dl[0];
            XX[1 + 2 * k] = (qp)gp.stenc[1 + 2 * (k + gp.nsMax * (rr - 1))] * dl[1];
        }
        double* w = &gp.qw[gp.nqMax * (rr - 1)];
        if (rr == 1) {  // :119-126
            qpt[0] = (qp)1 / (qp)2 / sqrtq((qp)3);
            qpt[1] = -qpt[0];
            w[0] = 1.0 / 2.0;
            w[1] = w[0];
        } else if (rr == 2) {  // :127-136
            qpt[0] = (qp)1 / (qp)2 * sqrtq((qp)3 / (qp)5);
            qpt[1] = 0;
            qpt[2] = -qpt[0];
            w[0] = 5.0 / 18.0;
            w[1] = 8.0 / 18.0;
            w[2] = w[0];
        } else {  // :137-148
            qpt[0] = (qp)1 / (qp)2 * sqrtq((qp)3 / (qp)7 + (qp)2 / (qp)7 * sqrtq((qp)6 / (qp)5));
            qpt[1] = (qp)1 / (qp)2 * sqrtq((qp)3 / (qp)7 - (qp)2 / (qp)7 * sqrtq((qp)6 / (qp)5));
            qpt[2] = -qpt[1];
            qpt[3] = -qpt[0];
            w[0] = (18.0 - std::sqrt(30.0)) / 72.0;
            w[1] = (18.0 + std::sqrt(30.0)) / 72.0;
            w[2] = w[1];
            w[3] = w[0];
        }
        for (int q = 0; q < nq; q++) {  // :155-165
            XXs[0 + 2 * (NORTH * nq + q)] = qpt[q] * dl[0];
            XXs[1 + 2 * (NORTH * nq + q)] = dl[1] / (qp)2;
            XXs[0 + 2 * (SOUTH * nq + q)] = qpt[q] * dl[0];
            XXs[1 + 2 * (SOUTH * nq + q)] = -(dl[1] / (qp)2);
            XXs[0 + 2 * (EAST * nq + q)] = dl[0] / (qp)2;
            XXs[1 + 2 * (EAST * nq + q)] = qpt[q] * dl[1];
            XXs[0 + 2 * (WEST * nq + q)] = -(dl[0] / (qp)2);
            XXs[1 + 2 * (WEST * nq + q)] = qpt[q] * dl[1];
        }
        // :337-381 GP_volAvgToPointPredVect
        std::vector<qp> Kcov((size_t)ns * ns), Kstr((size_t)ns * np), pred;
        for (int i = 0; i < ns; i++)
            for (int j = 0; j < ns; j++) Kcov[i * ns + j] = gp_kernel_vv(&XX[2 * i], &XX[2 * j], dl, ell);
        for (int i = 0; i < ns; i++)
            for (int j = 0; j < np; j++) Kstr[i * np + j] = gp_kernel_vp(&XX[2 * i], &XXs[2 * j], dl, ell);
        if (!solve_spd(ns, np, Kcov, Kstr, pred)) {
            err = "linAlgQuadPrecision_choleskyDecomp: A is not positive definite";
            return false;
        }
        for (int i = 0; i < np; i++) {  // :171-173
            qp s = 0;
            for (int k = 0; k < ns; k++) s = s + pred[k * np + i];
            for (int k = 0; k < ns; k++) pred[k * np + i] = pred[k * np + i] / s;
        }
        for (int f = 0; f < 4; f++)  // :176-186
            for (int q = 0; q < nq; q++)
                for (int k = 0; k < ns; k++)
                    gp.pv[k + gp.nsMax * (q + gp.nqMax * (f + 4 * (rr - 1)))] = (double)pred[k * np + f * nq + q];
        for (int q = 0; q < nq; q++) gp.qpts[q + gp.nqMax * (rr - 1)] = (double)qpt[q];
    }
    return true;
}

qp parse_qp(const std::string& s) { return strtoflt128(fortran_real_text(s).c_str(), nullptr); }

// ================================================================ physics
// src/eos.f90:9-26
inline double eos_presIdealGas(const Sim& s, double dens, double eint, double gama) {
    double pres = (gama - 1.0) * dens * eint;
    if (pres < s.smallPressure) pres = s.smallPressure;
    return pres;
}

// src/convert.f90:198-234
inline void cons2prim(const Sim& s, const double* U, double* V) {
    double Bp;
    if (s.forceHydro)
        Bp = 0.0;
    else
        Bp = 0.5 * (U[MAGX] * U[MAGX] + U[MAGY] * U[MAGY] + U[MAGZ] * U[MAGZ]);
    double density = U[DENS];
    double velx = U[MOMX] / density;
    double vely = U[MOMY] / density;
    double velz = U[MOMZ] / density;
    double internalEnergy = (U[ENER] - Bp) / density - 0.5 * (velx * velx + vely * vely + velz * velz);
    double pressure = eos_presIdealGas(s, density, internalEnergy, s.gamma);
    V[DENS] = density;
    V[VELX] = velx;
    V[VELY] = vely;
    V[VELZ] = velz;
    if (s.forceHydro) {
        V[MAGX] = 0.0;
        V[MAGY] = 0.0;
        V[MAGZ] = 0.0;
    } else {
        V[MAGX] = U[MAGX];
        V[MAGY] = U[MAGY];
        V[MAGZ] = U[MAGZ];
    }
    V[PRES] = pressure;
    V[EINT] = internalEnergy;
    V[GAMM] = s.gamma;
}

// src/convert.f90:236-254 (pressure not floored)
inline double cons2pres(const Sim& s, const double* U) {
    double Bp;
    if (s.forceHydro)
        Bp = 0.0;
    else
        Bp = 0.5 * ((0.0 + U[MAGX] * U[MAGX]) + U[MAGY] * U[MAGY] + U[MAGZ] * U[MAGZ]);
    double msq = (0.0 + U[MOMX] * U[MOMX]) + U[MOMY] * U[MOMY] + U[MOMZ] * U[MOMZ];
    return (s.gamma - 1.0) * (U[ENER] - Bp - 0.5 * msq / U[DENS]);
}

// src/convert.f90:159-196
inline void prim2cons(const Sim& s, const double* V, double* U) {
    double Bp;
    if (s.forceHydro)
        Bp = 0.0;
    else
        Bp = 0.5 * (V[MAGX] * V[MAGX] + V[MAGY] * V[MAGY] + V[MAGZ] * V[MAGZ]);
    double rhoEint = V[PRES] / (s.gamma - 1.0);
    double E = rhoEint + V[DENS] * (0.5 * (V[VELX] * V[VELX] + V[VELY] * V[VELY] + V[VELZ] * V[VELZ])) + Bp;
    U[DENS] = V[DENS];
    U[MOMX] = V[DENS] * V[VELX];
    U[MOMY] = V[DENS] * V[VELY];
    U[MOMZ] = V[DENS] * V[VELZ];
    if (s.forceHydro) {
        U[MAGX] = U[MAGY] = U[MAGZ] = 0.0;
    } else {
        U[MAGX] = V[MAGX];
        U[MAGY] = V[MAGY];
        U[MAGZ] = V[MAGZ];
    }
    U[ENER] = E;
}

// src/convert.f90:28-92
inline void cons2flux(const Sim& s, const double* U, int dir, double* Flux) {
    double V[NPRIM];
    double Bp = 0.0;
    if (!s.forceHydro) Bp = 0.5 * (U[MAGX] * U[MAGX] + U[MAGY] * U[MAGY] + U[MAGZ] * U[MAGZ]);
    double E = U[ENER];
    cons2prim(s, U, V);
    double Ptot = V[PRES] + Bp;
    int mN, mT1, mT2, vN, vT1, vT2, bN, bT1, bT2;
    if (dir == XDIR) {
        mN = MOMX; vN = VELX; mT1 = MOMY; vT1 = VELY; mT2 = MOMZ; vT2 = VELZ;
        bN = MAGX; bT1 = MAGY; bT2 = MAGZ;
    } else {
        mN = MOMY; vN = VELY; mT1 = MOMX; vT1 = VELX; mT2 = MOMZ; vT2 = VELZ;
        bN = MAGY; bT1 = MAGX; bT2 = MAGZ;
    }
    for (int v = 0; v < NCONS; v++) Flux[v] = 0.0;
    Flux[DENS] = U[mN];
    Flux[mN] = U[mN] * U[mN] / U[DENS] + Ptot;
    Flux[mT1] = U[mN] * V[vT1];
    Flux[mT2] = U[mN] * V[vT2];
    Flux[ENER] = (E + Ptot) * V[vN];
    if (!s.forceHydro) {
        Flux[mN] = Flux[mN] - V[bN] * V[bN];
        Flux[mT1] = Flux[mT1] - V[bT1] * V[bN];
        Flux[mT2] = Flux[mT2] - V[bT2] * V[bN];
        Flux[bT1] = V[vN] * V[bT1] - V[vT1] * V[bN];
        Flux[bT2] = V[vN] * V[bT2] - V[vT2] * V[bN];
        Flux[ENER] = Flux[ENER] - V[bN] * (V[VELX] * V[MAGX] + V[VELY] * V[MAGY] + V[VELZ] * V[MAGZ]);
    }
}

// src/eigen.f90:305-321 (Ryu & Jones 1995 eqs. 2.18-2.19)
inline double eigen_c_fs(double gam, double rho, double p, double BB, double B_N, double pm) {
    double c_fs = (gam * p + BB) / rho;
    c_fs = 0.5 * (c_fs + pm * std::sqrt(c_fs * c_fs - 4.0 * gam * p * (B_N * B_N) / (rho * rho)));
    c_fs = std::sqrt(std::fmax(1.0e-14, c_fs));
    return c_fs;
}

// src/eigen.f90:257-303; only eigenvalues 1 (velN - c_f) and 7 (velN + c_f)
// are used by the HLLC solver, so only c_f is evaluated.
inline void eigen_fast(const Sim& s, const double* V, int dir, double& lam1, double& lam7) {
    int dirN = (dir == XDIR) ? 0 : 1;
    double rho = std::fmax(V[DENS], s.smallDensity);
    double velN = V[VELX + dirN];
    double B_N = V[MAGX + dirN];
    double p = std::fmax(V[PRES], s.smallPressure);
    double gam = V[GAMM];
    double BB = V[MAGX] * V[MAGX] + V[MAGY] * V[MAGY] + V[MAGZ] * V[MAGZ];
    double c_f = eigen_c_fs(gam, rho, p, BB, B_N, +1.0);
    lam1 = velN - c_f;
    lam7 = velN + c_f;
}

inline double dot3(const double* a, const double* b) { return (0.0 + a[0] * b[0]) + a[1] * b[1] + a[2] * b[2]; }

// src/riemannSolver.f90:68-221 (HLLC for MHD, Li 2005)
inline void hllc(const Sim& s, const double* uL, const double* uR, int dir, double* flux) {
    double vL[NPRIM], vR[NPRIM], vA[NPRIM];
    cons2prim(s, uL, vL);
    cons2prim(s, uR, vR);
    int vN, vT1, vT2, bN, bT1, bT2, mN, mT1, mT2;
    if (dir == XDIR) {
        vN = VELX; bN = MAGX; mN = MOMX; vT1 = VELY; bT1 = MAGY; mT1 = MOMY; vT2 = VELZ; bT2 = MAGZ; mT2 = MOMZ;
    } else {
        vN = VELY; bN = MAGY; mN = MOMY; vT1 = VELX; bT1 = MAGX; mT1 = MOMX; vT2 = VELZ; bT2 = MAGZ; mT2 = MOMZ;
    }
    double eL1, eL7, eR1, eR7, eA1, eA7;
    eigen_fast(s, vL, dir, eL1, eL7);
    eigen_fast(s, vR, dir, eR1, eR7);
    for (int v = 0; v < NPRIM; v++) vA[v] = (vL[v] + vR[v]) / 2.0;
    eigen_fast(s, vA, dir, eA1, eA7);
    double sL = std::fmin(eL1, eA1);
    double sR = std::fmax(eA7, eR7);
    double fL[NCONS], fR[NCONS], uHLL[NCONS], uStr[NCONS];
    cons2flux(s, uL, dir, fL);
    cons2flux(s, uR, dir, fR);
    for (int v = 0; v < NCONS; v++) uHLL[v] = (sR * uR[v] - sL * uL[v] + fL[v] - fR[v]) / (sR - sL);
    double velHLL[3] = {uHLL[MOMX] / uHLL[DENS], uHLL[MOMY] / uHLL[DENS], uHLL[MOMZ] / uHLL[DENS]};
    double magHLL[3] = {uHLL[MAGX], uHLL[MAGY], uHLL[MAGZ]};
    double magDotVelHLL = dot3(magHLL, velHLL);
    double magDotVelL = dot3(&vL[MAGX], &vL[VELX]);
    double magDotVelR = dot3(&vR[MAGX], &vR[VELX]);
    double velNL = vL[vN], velNR = vR[vN];
    double velT1L = vL[vT1], velT1R = vR[vT1];
    double velT2L = vL[vT2], velT2R = vR[vT2];
    double momNL = uL[mN], momNR = uR[mN];
    double magNL = vL[bN], magNR = vR[bN], magNHLL = uHLL[bN];
    double magT1L = vL[bT1], magT1R = vR[bT1], magT1HLL = uHLL[bT1];
    double magT2L = vL[bT2], magT2R = vR[bT2], magT2HLL = uHLL[bT2];
    double rhoL = vL[DENS], rhoR = vR[DENS];
    double pL = vL[PRES], pR = vR[PRES];
    double pTotL = pL + 0.5 * dot3(&vL[MAGX], &vL[MAGX]);
    double pTotR = pR + 0.5 * dot3(&vR[MAGX], &vR[MAGX]);
    double dL = sL - velNL, dR = sR - velNR;
    double sStr = (momNR * dR - momNL * dL + pTotL - pTotR - magNL * magNL + magNR * magNR) / (rhoR * dR - rhoL * dL);
    double pStr = rhoL * dL * (sStr - velNL) + pTotL - magNL * magNL + magNHLL * magNHLL;
    if (0.0 < sL) {
        for (int v = 0; v < NCONS; v++) flux[v] = fL[v];
    } else if ((sL <= 0.0) && (0.0 < sStr)) {
        uStr[DENS] = rhoL * dL / (sL - sStr);
        uStr[mN] = uStr[DENS] * sStr;
        uStr[mT1] = uStr[DENS] * velT1L - (magNHLL * magT1HLL - magNL * magT1L) / (sL - sStr);
        uStr[mT2] = uStr[DENS] * velT2L - (magNHLL * magT2HLL - magNL * magT2L) / (sL - sStr);
        uStr[bN] = magNHLL;
        uStr[bT1] = magT1HLL;
        uStr[bT2] = magT2HLL;
        uStr[ENER] = uL[ENER] * dL + pStr * sStr - pTotL * velNL - magNHLL * magDotVelHLL + magNL * magDotVelL;
        uStr[ENER] = uStr[ENER] / (sL - sStr);
        for (int v = 0; v < NCONS; v++) flux[v] = fL[v] + sL * (uStr[v] - uL[v]);
    } else if ((sStr <= 0.0) && (0.0 <= sR)) {
        uStr[DENS] = rhoR * dR / (sR - sStr);
        uStr[mN] = uStr[DENS] * sStr;
        uStr[mT1] = uStr[DENS] * velT1R - (magNHLL * magT1HLL - magNR * magT1R) / (sR - sStr);
        uStr[mT2] = uStr[DENS] * velT2R - (magNHLL * magT2HLL - magNR * magT2R) / (sR - sStr);
        uStr[bN] = magNHLL;
        uStr[bT1] = magT1HLL;
        uStr[bT2] = magT2HLL;
        uStr[ENER] = uR[ENER] * dR + pStr * sStr - pTotR * velNR - magNHLL * magDotVelHLL + magNR * magDotVelR;
        uStr[ENER] = uStr[ENER] / (sR - sStr);
        for (int v = 0; v < NCONS; v++) flux[v] = fR[v] + sR * (uStr[v] - uR[v]);
    } else {
        for (int v = 0; v < NCONS; v++) flux[v] = fR[v];
    }
}

// src/riemannSolver.f90:23-47
inline void face_flux(const Sim& s, const GPTab& gp, const double* uL, const double* uR, int dir, int rr,
                      double* flux) {
    // uL, uR are (8, nqMax)
    if (rr == 0) {
        hllc(s, uL, uR, dir, flux);
    } else {
        int nq = gp.nQuad[rr - 1];
        for (int v = 0; v < NCONS; v++) flux[v] = 0.0;
        double f[NCONS];
        for (int q = 1; q <= nq; q++) {
            hllc(s, uL + NCONS * (q - 1), uR + NCONS * (q - 1), dir, f);
            double w = gp.w(q, rr);
            for (int v = 0; v < NCONS; v++) flux[v] = flux[v] + w * f[v];
        }
    }
}

// src/eigen.f90:323-349 (alpha_f for pm = +1, alpha_s for pm = -1)
inline double eigen_alpha_fs(double c_f, double c_s, double a, double BB, double B_N, double pm) {
    double BB_T = BB - B_N * B_N;
    (void)BB_T;
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
    alpha = std::fmin(1.0, std::fmax(0.0, alpha));
    return std::sqrt(alpha);
}
// src/eigen.f90:351-371
inline double eigen_beta_T(double B_T1, double B_T2, double smallB) {
    double BB_T = B_T1 * B_T1 + B_T2 * B_T2;
    if (BB_T < smallB * smallB) return std::copysign(1.0, B_T1) / std::sqrt(2.0);
    return B_T1 / std::sqrt(std::fmax(BB_T, 1.0e-30));
}
// src/eigen.f90:20-255: right eigenvectors (columns of R) and left
// eigenvectors (columns of L) of the 7 MHD waves in direction dir, 8x8
// column-major with the variable index as the row; cons: converted to
// conserved variables by dU/dV and dV/dU (MATMUL as k-ascending sums from 0)
void eigen_vecs(const Sim& s, const double* V, int dir, bool cons, double* Lm, double* Rm) {
    const int vN = dir == XDIR ? VELX : VELY, vT1 = dir == XDIR ? VELY : VELX, vT2 = VELZ;
    const int bN = dir == XDIR ? MAGX : MAGY, bT1 = dir == XDIR ? MAGY : MAGX, bT2 = MAGZ;
    auto R = [&](int r, int c) -> double& { return Rm[r + NCONS * (c - 1)]; };
    auto L = [&](int r, int c) -> double& { return Lm[r + NCONS * (c - 1)]; };
    const double rho = std::fmax(V[DENS], s.smallDensity);
    const double velN = V[vN], velT1 = V[vT1], velT2 = V[vT2];
    const double B_N = V[bN], B_T1 = V[bT1], B_T2 = V[bT2];
    const double p = std::fmax(V[PRES], s.smallPressure);
    const double gam = V[GAMM];
    const double BB = B_N * B_N + B_T1 * B_T1 + B_T2 * B_T2;
    const double c_f = eigen_c_fs(gam, rho, p, BB, B_N, +1.0);
    const double c_s = eigen_c_fs(gam, rho, p, BB, B_N, -1.0);
    const double a = std::sqrt(gam * p / rho);
    const double alpha_f = eigen_alpha_fs(c_f, c_s, a, BB, B_N, +1.0);
    const double alpha_s = eigen_alpha_fs(c_f, c_s, a, BB, B_N, -1.0);
    const double beta_T1 = eigen_beta_T(B_T1, B_T2, s.smallB);
    const double beta_T2 = eigen_beta_T(B_T2, B_T1, s.smallB);
    const double sgnBn = std::copysign(1.0, B_N);
    const double sr = std::sqrt(rho);
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
    if (!cons) return;
    const double k = 1.0 - gam;
    double dUdV[NCONS * NCONS] = {}, dVdU[NCONS * NCONS] = {};
    auto A = [&](int r, int c) -> double& { return dUdV[r + NCONS * c]; };
    auto Bm = [&](int r, int c) -> double& { return dVdU[r + NCONS * c]; };
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
    for (int q = 0; q < NCONS * NCONS; q++) {
        Rm[q] = Rc[q];
        Lm[q] = Lc[q];
    }
}

// src/detect.f90:250-265, :238-248
inline bool detect_CAD(double dens, double pres) {
    return !(std::isnan(dens) || std::isnan(pres) || !std::isfinite(dens) || !std::isfinite(pres));
}
inline bool detect_PAD(double dens, double pres) { return (dens > 0.0) && (pres > 0.0); }

// ================================================================ block ops
inline const double* Uc(const Block& b, const std::vector<double>& U, int i, int j) { return &U[NCONS * b.c(i, j)]; }
inline double* Uc(const Block& b, std::vector<double>& U, int i, int j) { return &U[NCONS * b.c(i, j)]; }

// src/gridBlock.f90:194-235
void lowerOrder(Block& b, int i, int j) {
    b.scheme[b.c(i, j)] = std::max(b.scheme[b.c(i, j)] - 1, 0);
    b.recompute[b.c(i, j)] = 1;
    b.recompute[b.c(i + 1, j)] = 1;
    b.recompute[b.c(i - 1, j)] = 1;
    b.recompute[b.c(i, j + 1)] = 1;
    b.recompute[b.c(i, j - 1)] = 1;
    for (int jj = std::max(j - 2, b.minIdx[1]); jj <= std::min(j + 2, b.maxIdx[1]); jj++)
        for (int ii = std::max(i - 2, b.minIdx[0]); ii <= std::min(i + 2, b.maxIdx[0]); ii++)
            if (std::abs(ii - i) + std::abs(jj - j) <= 2) b.recomputeFLICD[b.c(ii, jj)] = 1;
}

// src/reconstruct.f90:18-175
void reconstruct(orc_handle* h, const std::vector<double>& U, std::vector<unsigned char>* innerMask, int* nInner) {
    Block& b = h->blk;
    const GPTab& gp = h->gp;
    const Sim& s = h->sim;
    std::vector<char> reconstructCell(b.recompute), cellIsAdmissible(b.ncell()), nextPass(b.ncell());
    bool admissibleAll = false;
    const int i0 = b.strt[0] - 2, i1 = b.stop[0] + 2, j0 = b.strt[1] - 2, j1 = b.stop[1] + 2;
    while (!admissibleAll) {
        std::fill(cellIsAdmissible.begin(), cellIsAdmissible.end(), 1);
#pragma omp parallel for collapse(2) schedule(static)
        for (int j = j0; j <= j1; j++) {
            for (int i = i0; i <= i1; i++) {
                if (!reconstructCell[b.c(i, j)]) continue;
                double stencil[NCONS * 25];
                for (int f = 0; f < 4; f++) {
                    int ia = 0, ja = 0;
                    if (f == NORTH) { ia = 0; ja = 1; }
                    else if (f == SOUTH) { ia = 0; ja = -1; }
                    else if (f == EAST) { ia = 1; ja = 0; }
                    else { ia = -1; ja = 0; }
                    int rr = std::min(b.scheme[b.c(i, j)], b.scheme[b.c(i + ia, j + ja)]);
                    if (rr == 0) {
                        const double* u = Uc(b, U, i, j);
                        double* fv = b.fv(1, f, i, j);
                        for (int v = 0; v < NCONS; v++) fv[v] = u[v];
                    } else {
                        int ns = gp.nStenc[rr - 1], nq = gp.nQuad[rr - 1];
                        for (int k = 1; k <= ns; k++) {
                            const double* u = Uc(b, U, gp.sx(k, rr) + i, gp.sy(k, rr) + j);
                            for (int v = 0; v < NCONS; v++) stencil[NCONS * (k - 1) + v] = u[v];
                        }
                        for (int q = 1; q <= nq; q++) {
                            double* fv = b.fv(q, f, i, j);
                            for (int v = 0; v < NCONS; v++) fv[v] = 0.0;
                            for (int k = 1; k <= ns; k++) {
                                double p = gp.p(k, q, f, rr);
                                for (int v = 0; v < NCONS; v++) fv[v] = fv[v] + p * stencil[NCONS * (k - 1) + v];
                            }
                        }
                        for (int q = 1; q <= nq; q++) {
                            double* fv = b.fv(q, f, i, j);
                            double pres = cons2pres(s, fv);
                            if (!(detect_CAD(fv[DENS], pres) && detect_PAD(fv[DENS], pres)))
                                cellIsAdmissible[b.c(i, j)] = 0;
                        }
                    }
                }
            }
        }
        admissibleAll = true;
        std::fill(nextPass.begin(), nextPass.end(), 0);
        for (int j = j0; j <= j1; j++) {
            for (int i = i0; i <= i1; i++) {
                if (!cellIsAdmissible[b.c(i, j)]) {
                    lowerOrder(b, i, j);
                    nextPass[b.c(i - 1, j)] = 1;
                    nextPass[b.c(i, j)] = 1;
                    nextPass[b.c(i + 1, j)] = 1;
                    nextPass[b.c(i, j - 1)] = 1;
                    nextPass[b.c(i, j + 1)] = 1;
                    admissibleAll = false;
                    if (innerMask) (*innerMask)[b.c(i, j)]++;
                    if (nInner) (*nInner)++;
                }
            }
        }
        reconstructCell = nextPass;
    }
}

// src/getFluxes.f90:16-90
void getFluxes(orc_handle* h) {
    Block& b = h->blk;
    const GPTab& gp = h->gp;
    const Sim& s = h->sim;
    const int nqm = b.nqMax;
#pragma omp parallel for collapse(2) schedule(static)
    for (int j = b.strt[1] - 1; j <= b.stop[1] + 2; j++) {
        for (int i = b.strt[0] - 1; i <= b.stop[0] + 2; i++) {
            double uL[NCONS * 4], uR[NCONS * 4];
            if (b.recompute[b.c(i, j)] || b.recompute[b.c(i - 1, j)]) {
                for (int q = 1; q <= nqm; q++)
                    for (int v = 0; v < NCONS; v++) {
                        uR[NCONS * (q - 1) + v] = b.fv(q, WEST, i, j)[v];
                        uL[NCONS * (q - 1) + v] = b.fv(q, EAST, i - 1, j)[v];
                    }
                int rr = std::min(b.scheme[b.c(i, j)], b.scheme[b.c(i - 1, j)]);
                face_flux(s, gp, uL, uR, XDIR, rr, b.flr(XDIR, i, j));
                for (int v = 0; v < NCONS; v++) b.fl(XDIR, i, j)[v] = b.flr(XDIR, i, j)[v];
            }
            if (b.recompute[b.c(i, j)] || b.recompute[b.c(i, j - 1)]) {
                for (int q = 1; q <= nqm; q++)
                    for (int v = 0; v < NCONS; v++) {
                        uR[NCONS * (q - 1) + v] = b.fv(q, SOUTH, i, j)[v];
                        uL[NCONS * (q - 1) + v] = b.fv(q, NORTH, i, j - 1)[v];
                    }
                int rr = std::min(b.scheme[b.c(i, j)], b.scheme[b.c(i, j - 1)]);
                face_flux(s, gp, uL, uR, YDIR, rr, b.flr(YDIR, i, j));
                for (int v = 0; v < NCONS; v++) b.fl(YDIR, i, j)[v] = b.flr(YDIR, i, j)[v];
            }
        }
    }
}

// src/FLICDdivB.f90:13-70
void flicd(orc_handle* h) {
    Block& b = h->blk;
#pragma omp parallel for collapse(2) schedule(static)
    for (int j = b.strt[1]; j <= b.stop[1] + 1; j++) {
        for (int i = b.strt[0]; i <= b.stop[0] + 1; i++) {
            if (b.recomputeFLICD[b.c(i, j)]) {
                b.fl(XDIR, i, j)[MAGY] = (2 * b.flr(XDIR, i, j)[MAGY] + b.flr(XDIR, i + 1, j)[MAGY] +
                                          b.flr(XDIR, i - 1, j)[MAGY] - b.flr(YDIR, i, j + 1)[MAGX] -
                                          b.flr(YDIR, i, j)[MAGX] - b.flr(YDIR, i - 1, j)[MAGX] -
                                          b.flr(YDIR, i - 1, j + 1)[MAGX]) / 8.0;
                b.fl(YDIR, i, j)[MAGX] = (2 * b.flr(YDIR, i, j)[MAGX] + b.flr(YDIR, i, j + 1)[MAGX] +
                                          b.flr(YDIR, i, j - 1)[MAGX] - b.flr(XDIR, i + 1, j)[MAGY] -
                                          b.flr(XDIR, i, j)[MAGY] - b.flr(XDIR, i, j - 1)[MAGY] -
                                          b.flr(XDIR, i + 1, j - 1)[MAGY]) / 8.0;
            }
        }
    }
    const size_t n = b.ncell();
    for (size_t c = 0; c < n; c++) {
        b.flux[NCONS * (XDIR + 2 * c) + MAGX] = 0.0;
        b.flux[NCONS * (YDIR + 2 * c) + MAGY] = 0.0;
    }
}

// src/detect.f90:18-236
bool detect_all(orc_handle* h, const std::vector<double>& U, std::vector<double>& Unew,
                std::vector<unsigned char>* detMask, int* nDet) {
    Block& b = h->blk;
    const Sim& s = h->sim;
    bool exit_mood_loop = true;
    std::vector<char> checkCell(b.recomputeFLICD), lowerCell(b.ncell(), 0);
    std::fill(b.recompute.begin(), b.recompute.end(), 0);
    std::fill(b.recomputeFLICD.begin(), b.recomputeFLICD.end(), 0);
    const double dx = b.dl[0], dy = b.dl[1];
#pragma omp parallel for collapse(2) schedule(static)
    for (int j = b.strt[1]; j <= b.stop[1]; j++) {
        for (int i = b.strt[0]; i <= b.stop[0]; i++) {
            if (!checkCell[b.c(i, j)]) continue;
            if (b.scheme[b.c(i, j)] <= 0) continue;
            const double* un = Uc(b, Unew, i, j);
            double presNew = cons2pres(s, un);
            if (!detect_CAD(un[DENS], presNew)) { lowerCell[b.c(i, j)] = 1; continue; }
            if (!detect_PAD(un[DENS], presNew)) { lowerCell[b.c(i, j)] = 1; continue; }
            double V[NPRIM], Vip[NPRIM], Vim[NPRIM], Vjp[NPRIM], Vjm[NPRIM];
            cons2prim(s, Uc(b, U, i, j), V);
            cons2prim(s, Uc(b, U, i + 1, j), Vip);
            cons2prim(s, Uc(b, U, i - 1, j), Vim);
            cons2prim(s, Uc(b, U, i, j + 1), Vjp);
            cons2prim(s, Uc(b, U, i, j - 1), Vjm);
            bool shock1 = false, shock2 = false, shock3 = false;
            double div_vel = (Vip[VELX] - Vim[VELX]) / (2 * dx);
            div_vel = div_vel + (Vjp[VELY] - Vjm[VELY]) / (2 * dy);
            double sigma_v = 1.0;
            if (div_vel < -(sigma_v * (b.maxdxdy * b.maxdxdy))) shock1 = true;
            double mach = V[VELX] * V[VELX] + V[VELY] * V[VELY];
            mach = V[DENS] * mach / (V[GAMM] * V[PRES]);
            mach = std::sqrt(mach);
            double sigma_M = 0.2;
            if (mach > sigma_M) shock2 = true;
            double pg = std::fabs(Vip[PRES] - Vim[PRES]) / (std::fmin(Vip[PRES], Vim[PRES]));
            pg = pg + std::fabs(Vjp[PRES] - Vjm[PRES]) / (std::fmin(Vjp[PRES], Vjm[PRES]));
            double sigma_p = 10.0;
            if (pg > sigma_p * b.maxdxdy) shock3 = true;
            if (!(shock1 && shock2 && shock3)) continue;
            double densNew = un[DENS];
            double d1 = Uc(b, U, i, j)[DENS], d2 = Uc(b, U, i + 1, j)[DENS], d3 = Uc(b, U, i - 1, j)[DENS];
            double d4 = Uc(b, U, i, j + 1)[DENS], d5 = Uc(b, U, i, j - 1)[DENS];
            double min_d = std::fmin(std::fmin(std::fmin(std::fmin(d1, d2), d3), d4), d5);
            double max_d = std::fmax(std::fmax(std::fmax(std::fmax(d1, d2), d3), d4), d5);
            if (max_d - min_d < b.mindxdy * b.mindxdy * b.mindxdy) continue;
            if ((min_d <= densNew) && (densNew <= max_d)) continue;
            double dd[5][2];
            int counter = 0;
            for (int ii = -1; ii <= 1; ii++)
                for (int jj = -1; jj <= 1; jj++)
                    if (std::abs(ii) + std::abs(jj) <= 1) {
                        dd[counter][0] = (Uc(b, U, i + ii + 1, j + jj)[DENS] - 2 * Uc(b, U, i + ii, j + jj)[DENS] +
                                          Uc(b, U, i + ii - 1, j + jj)[DENS]) / (dx * dx);
                        dd[counter][1] = (Uc(b, U, i + ii, j + jj + 1)[DENS] - 2 * Uc(b, U, i + ii, j + jj)[DENS] +
                                          Uc(b, U, i + ii, j + jj - 1)[DENS]) / (dy * dy);
                        counter++;
                    }
            double mn[2], mx[2];
            for (int d = 0; d < 2; d++) {
                mn[d] = dd[0][d];
                mx[d] = dd[0][d];
                for (int k = 1; k < 5; k++) {
                    mn[d] = std::fmin(mn[d], dd[k][d]);
                    mx[d] = std::fmax(mx[d], dd[k][d]);
                }
            }
            bool sx1 = (mn[0] * mx[0] > -b.mindxdy);
            bool sy1 = (mn[1] * mx[1] > -b.mindxdy);
            bool sx2 = (std::fmax(std::fabs(mn[0]), std::fabs(mx[0])) < b.mindxdy);
            bool sy2 = (std::fmax(std::fabs(mn[1]), std::fabs(mx[1])) < b.mindxdy);
            bool sx3 = (std::fmin(std::fabs(mn[0]), std::fabs(mx[0])) >= 0.5 * std::fmax(std::fabs(mn[0]), std::fabs(mx[0])));
            bool sy3 = (std::fmin(std::fabs(mn[1]), std::fabs(mx[1])) >= 0.5 * std::fmax(std::fabs(mn[1]), std::fabs(mx[1])));
            bool smooth1 = sx1 && sx2 && sy1 && sy2;
            bool smooth2 = sx1 && sx3 && sy1 && sy3;
            if (!(smooth1 || smooth2)) lowerCell[b.c(i, j)] = 1;
        }
    }
    for (int j = b.strt[1]; j <= b.stop[1]; j++)
        for (int i = b.strt[0]; i <= b.stop[0]; i++)
            if (lowerCell[b.c(i, j)]) {
                lowerOrder(b, i, j);
                exit_mood_loop = false;
                if (detMask) (*detMask)[b.c(i, j)]++;
                if (nDet) (*nDet)++;
            }
    return exit_mood_loop;
}

// src/boundaryConditions.f90:79-116 (dispatch), :118-152 (outflow), :154-187 (periodic)
void bc_apply(const Block& b, int bc, std::vector<double>& A, int nv) {
    const int nx = b.nTot[0], ny = b.nTot[1];
    auto at = [&](int i, int j) { return &A[(size_t)nv * ((size_t)(i - 1) + (size_t)nx * (j - 1))]; };
    if (bc == 0) {
        for (int i = b.minIdx[0]; i <= b.NGC; i++)
            for (int j = 1; j <= ny; j++) std::memcpy(at(i, j), at(b.strt[0], j), sizeof(double) * nv);
        for (int i = b.stop[0] + 1; i <= b.maxIdx[0]; i++)
            for (int j = 1; j <= ny; j++) std::memcpy(at(i, j), at(b.stop[0], j), sizeof(double) * nv);
        for (int j = b.minIdx[1]; j <= b.NGC; j++)
            for (int i = 1; i <= nx; i++) std::memcpy(at(i, j), at(i, b.strt[1]), sizeof(double) * nv);
        for (int j = b.stop[1] + 1; j <= b.maxIdx[1]; j++)
            for (int i = 1; i <= nx; i++) std::memcpy(at(i, j), at(i, b.stop[1]), sizeof(double) * nv);
    } else {
        for (int g = 1; g <= b.NGC; g++)
            for (int j = 1; j <= ny; j++) std::memcpy(at(b.strt[0] - g, j), at(b.stop[0] - g + 1, j), sizeof(double) * nv);
        for (int g = 1; g <= b.NGC; g++)
            for (int j = 1; j <= ny; j++) std::memcpy(at(b.stop[0] + g, j), at(b.strt[0] + g - 1, j), sizeof(double) * nv);
        for (int g = 1; g <= b.NGC; g++)
            for (int i = 1; i <= nx; i++) std::memcpy(at(i, b.strt[1] - g), at(i, b.stop[1] - g + 1), sizeof(double) * nv);
        for (int g = 1; g <= b.NGC; g++)
            for (int i = 1; i <= nx; i++) std::memcpy(at(i, b.stop[1] + g), at(i, b.strt[1] + g - 1), sizeof(double) * nv);
    }
}

// src/boundaryConditions.f90:16-51, :189-254
void bc_apply_mood(Block& b, int bc) {
    if (bc == 0) return;
    auto sync = [&](size_t a, size_t c) {
        char e = b.recomputeFLICD[a] || b.recomputeFLICD[c];
        b.recomputeFLICD[a] = e;
        b.recomputeFLICD[c] = e;
        e = b.recompute[a] || b.recompute[c];
        b.recompute[a] = e;
        b.recompute[c] = e;
        int lo = std::min(b.scheme[a], b.scheme[c]);
        b.scheme[a] = lo;
        b.scheme[c] = lo;
    };
    for (int j = b.minIdx[1]; j <= b.maxIdx[1]; j++)
        for (int i = b.minIdx[0]; i <= b.maxIdx[0]; i++) {
            int ip;
            if (i < b.strt[0]) ip = i + b.N[0];
            else if (i > b.stop[0]) ip = i - b.N[0];
            else continue;
            sync(b.c(i, j), b.c(ip, j));
        }
    for (int j = b.minIdx[1]; j <= b.maxIdx[1]; j++) {
        int jp;
        if (j < b.strt[1]) jp = j + b.N[1];
        else if (j > b.stop[1]) jp = j - b.N[1];
        else continue;
        for (int i = b.minIdx[0]; i <= b.maxIdx[0]; i++) sync(b.c(i, j), b.c(i, jp));
    }
}

// the unsplit finite-volume update where recomputeFLICD (src/timeStep.f90:105-118)
void update(orc_handle* h, double dt, const std::vector<double>& U, std::vector<double>& Unew) {
    Block& b = h->blk;
    const double dx = b.dl[0], dy = b.dl[1];
#pragma omp parallel for collapse(2) schedule(static)
    for (int j = b.strt[1]; j <= b.stop[1]; j++) {
        for (int i = b.strt[0]; i <= b.stop[0]; i++) {
            if (b.recomputeFLICD[b.c(i, j)]) {
                const double* u = Uc(b, U, i, j);
                double* un = Uc(b, Unew, i, j);
                const double* fxp = b.fl(XDIR, i + 1, j);
                const double* fx = b.fl(XDIR, i, j);
                const double* fyp = b.fl(YDIR, i, j + 1);
                const double* fy = b.fl(YDIR, i, j);
                for (int v = 0; v < NCONS; v++)
                    un[v] = u[v] - (dt / dx) * (fxp[v] - fx[v]) - (dt / dy) * (fyp[v] - fy[v]);
            }
        }
    }
}

// src/timeStep.f90:45-130
void forward_euler(orc_handle* h, double dt, const std::vector<double>& U, std::vector<double>& Unew) {
    Block& b = h->blk;
    std::fill(b.scheme.begin(), b.scheme.end(), h->gp.R);
    std::fill(b.recompute.begin(), b.recompute.end(), 1);
    std::fill(b.recomputeFLICD.begin(), b.recomputeFLICD.end(), 1);
    bool exit_mood_loop = false;
    int pass = 0;
    const int stage = h->stageCounter++;
    while (!exit_mood_loop) {
        Trace tr;
        tr.stage = stage;
        tr.pass = pass;
        tr.nInner = 0;
        tr.nDetect = 0;
        if (h->trace) {
            tr.inner.assign(b.ncell(), 0);
            tr.detect.assign(b.ncell(), 0);
        }
        FC_PHASE(pass == 0 ? 1 : 2);
        reconstruct(h, U, h->trace ? &tr.inner : nullptr, &tr.nInner);
        getFluxes(h);
        FC_PHASE(3);
        flicd(h);
        update(h, dt, U, Unew);
        exit_mood_loop = detect_all(h, U, Unew, h->trace ? &tr.detect : nullptr, &tr.nDetect);
        bc_apply_mood(b, h->sim.bc);
        if (h->trace) h->traces.push_back(std::move(tr));
        pass++;
    }
    FC_PHASE(0);
}

// src/timeStep.f90:132-171
void rk3(orc_handle* h, double dt, std::vector<double>& U) {
    const Block& b = h->blk;
    const size_t n = U.size();
    std::vector<double> U1(n, 0.0), U2(n, 0.0), U3(n, 0.0);
    forward_euler(h, dt, U, U1);
    bc_apply(b, h->sim.bc, U1, NCONS);
    forward_euler(h, dt, U1, U2);
    bc_apply(b, h->sim.bc, U2, NCONS);
    for (size_t k = 0; k < n; k++) U2[k] = (3 * U[k] + U2[k]) / 4.0;
    bc_apply(b, h->sim.bc, U2, NCONS);
    forward_euler(h, dt, U2, U3);
    bc_apply(b, h->sim.bc, U3, NCONS);
    for (size_t k = 0; k < n; k++) U[k] = (U[k] + 2 * U3[k]) / 3.0;
}

// src/timeStep.f90:22-43
void advance(orc_handle* h, double dt) {
    Block& b = h->blk;
    rk3(h, dt, h->U);
#pragma omp parallel for collapse(2) schedule(static)
    for (int j = b.strt[1]; j <= b.stop[1]; j++)
        for (int i = b.strt[0]; i <= b.stop[0]; i++) cons2prim(h->sim, Uc(b, h->U, i, j), &h->V[NPRIM * b.c(i, j)]);
    bc_apply(b, h->sim.bc, h->U, NCONS);
    bc_apply(b, h->sim.bc, h->V, NPRIM);
}

// src/cfl.f90:14-52
double cfl_dt(const orc_handle* h) {
    const Block& b = h->blk;
    const Sim& s = h->sim;
    double xMax = 0.0, yMax = 0.0;
#pragma omp parallel for collapse(2) reduction(max : xMax, yMax) schedule(static)
    for (int j = b.strt[1]; j <= b.stop[1]; j++) {
        for (int i = b.strt[0]; i <= b.stop[0]; i++) {
            const double* V = &h->V[NPRIM * b.c(i, j)];
            double c;
            if (s.forceHydro) {
                c = std::sqrt(V[GAMM] * V[PRES] / V[DENS]);
            } else {
                double BB = V[MAGX] * V[MAGX] + V[MAGY] * V[MAGY] + V[MAGZ] * V[MAGZ];
                double bmin = std::fmin(std::fmin(std::fabs(V[MAGX]), std::fabs(V[MAGY])), std::fabs(V[MAGZ]));
                c = eigen_c_fs(V[GAMM], V[DENS], V[PRES], BB, bmin, +1.0);
            }
            double xl = std::fabs(V[VELX]) + c;
            double yl = std::fabs(V[VELY]) + c;
            xMax = std::fmax(xMax, xl);
            yMax = std::fmax(yMax, yl);
        }
    }
    return s.cfl * std::fmin(b.dl[0] / xMax, b.dl[1] / yMax);
}

// ================================================================ set-up
// src/grid.f90:31-103
void grid_init(Block& b, int nx, int ny, double xb, double xe, double yb, double ye, int R, int nqMax) {
    b.N[0] = nx;
    b.N[1] = ny;
    b.domBeg[0] = xb;
    b.domEnd[0] = xe;
    b.domBeg[1] = yb;
    b.domEnd[1] = ye;
    b.NGC = R + 2;
    for (int d = 0; d < 2; d++) {
        b.minIdx[d] = 1;
        b.maxIdx[d] = b.N[d] + 2 * b.NGC;
        b.strt[d] = b.minIdx[d] + b.NGC;
        b.stop[d] = b.maxIdx[d] - b.NGC;
        b.dl[d] = (b.domEnd[d] - b.domBeg[d]) / b.N[d];
        b.nTot[d] = b.maxIdx[d];
    }
    b.mindxdy = std::min(b.dl[0], b.dl[1]);
    b.maxdxdy = std::max(b.dl[0], b.dl[1]);
    b.nqMax = nqMax;
    size_t n = b.ncell();
    b.faceVals.assign(n * NCONS * nqMax * 4, 0.0);
    b.flux.assign(n * NCONS * 2, 0.0);
    b.fluxRaw.assign(n * NCONS * 2, 0.0);
    b.scheme.assign(n, 0);
    b.recompute.assign(n, 0);
    b.recomputeFLICD.assign(n, 0);
    b.x.resize(b.nTot[0]);
    b.y.resize(b.nTot[1]);
    for (int i = 1; i <= b.maxIdx[0]; i++) b.x[i - 1] = (i - b.NGC - 0.5) * b.dl[0] + b.domBeg[0];
    for (int j = 1; j <= b.maxIdx[1]; j++) b.y[j - 1] = (j - b.NGC - 0.5) * b.dl[1] + b.domBeg[1];
}

// src/initialCondition.f90:23-226.  Optional keys (not in the reference;
// their defaults reproduce it): IC_B0 and IC_pres for OrszagTang2d
// (default 1/gamma, :206-207), IC_magx/IC_magy/IC_magz for explosion2d
// (default 0).
void initial_condition(orc_handle* h, const std::string& par) {
    Block& b = h->blk;
    const Sim& s = h->sim;
    std::string type = par_str(par, "IC_type");
    std::vector<double>& V = h->V;
    auto Vc = [&](int i, int j) { return &V[NPRIM * b.c(i, j)]; };
    if (type == "explosion2d") {
        double cx = par_real(par, "IC_shockCenter_x"), cy = par_real(par, "IC_shockCenter_y");
        double rad = par_real(par, "IC_shockRad");
        double dIn = par_real(par, "IC_densIns"), dOut = par_real(par, "IC_densOut");
        double vxIn = par_real(par, "IC_velxIns"), vyIn = par_real(par, "IC_velyIns"), vzIn = par_real(par, "IC_velzIns");
        double vxOut = par_real(par, "IC_velxOut"), vyOut = par_real(par, "IC_velyOut"), vzOut = par_real(par, "IC_velzOut");
        double pIn = par_real(par, "IC_presIns"), pOut = par_real(par, "IC_presOut");
        double bx = par_real_opt(par, "IC_magx", 0.0), by = par_real_opt(par, "IC_magy", 0.0), bz = par_real_opt(par, "IC_magz", 0.0);
        std::fill(V.begin(), V.end(), 0.0);
        for (int j = b.strt[1]; j <= b.stop[1]; j++)
            for (int i = b.strt[0]; i <= b.stop[0]; i++) {
                double* v = Vc(i, j);
                double ddx = b.x[i - 1] - cx, ddy = b.y[j - 1] - cy;
                if (std::sqrt(ddx * ddx + ddy * ddy) <= rad) {
                    v[DENS] = dIn; v[VELX] = vxIn; v[VELY] = vyIn; v[VELZ] = vzIn; v[PRES] = pIn;
                } else {
                    v[DENS] = dOut; v[VELX] = vxOut; v[VELY] = vyOut; v[VELZ] = vzOut; v[PRES] = pOut;
                }
                v[MAGX] = bx; v[MAGY] = by; v[MAGZ] = bz;
            }
    } else if (type == "sedov2d") {
        double cx = par_real(par, "IC_shockCenter_x"), cy = par_real(par, "IC_shockCenter_y");
        double rad = 3.5 * std::min(b.dl[0], b.dl[1]);
        int nn = 2;
        double Vin[NPRIM] = {0}, Vout[NPRIM] = {0};
        Vin[DENS] = 1.0;
        Vin[PRES] = 3 * (s.gamma - 1) * 1.0 / ((nn + 1) * PI * (rad * rad));
        Vout[DENS] = 1.0;
        Vout[PRES] = 1e-5;
        std::fill(V.begin(), V.end(), 0.0);
        for (int j = b.strt[1]; j <= b.stop[1]; j++)
            for (int i = b.strt[0]; i <= b.stop[0]; i++) {
                double ddx = b.x[i - 1] - cx, ddy = b.y[j - 1] - cy;
                const double* src = (std::sqrt(ddx * ddx + ddy * ddy) <= rad) ? Vin : Vout;
                std::memcpy(Vc(i, j), src, sizeof(double) * NPRIM);
            }
    } else if (type == "OrszagTang2d") {
        double U0 = par_real(par, "IC_U0");
        double dens = par_real(par, "IC_dens");
        double B0 = par_real_opt(par, "IC_B0", 1 / s.gamma);
        double pres = par_real_opt(par, "IC_pres", 1 / s.gamma);
        for (int j = b.strt[1]; j <= b.stop[1]; j++)
            for (int i = b.strt[0]; i <= b.stop[0]; i++) {
                double xx = b.x[i - 1], yy = b.y[j - 1];
                double* v = Vc(i, j);
                v[DENS] = dens;
                v[VELX] = -U0 * std::sin(PI * yy * 2.0);
                v[VELY] = U0 * std::sin(PI * xx * 2.0);
                v[VELZ] = 0.0;
                v[MAGX] = -B0 * std::sin(PI * yy * 2.0);
                v[MAGY] = B0 * std::sin(PI * xx * 4.0);
                v[MAGZ] = 0.0;
                v[PRES] = pres;
            }
    } else {
        throw ParError{"Unrecognized choice of initial condition: " + type};
    }
    for (int j = b.strt[1]; j <= b.stop[1]; j++)
        for (int i = b.strt[0]; i <= b.stop[0]; i++) {
            double* v = Vc(i, j);
            v[EINT] = v[PRES] / (s.gamma - 1.0) / v[DENS];  // eos_eintIdealGas
            v[GAMM] = s.gamma;
            prim2cons(s, v, Uc(b, h->U, i, j));
        }
    bc_apply(b, s.bc, h->U, NCONS);
    bc_apply(b, s.bc, h->V, NPRIM);
}

}  // namespace

// ================================================================ C API
extern "C" {

orc_handle* orc_create_from_par(const char* parfile, char* err, int errlen) {
    std::string par(parfile);
    orc_handle* h = new orc_handle();
    try {
        Sim& s = h->sim;  // simulation.f90:35-78
        s.smallB = par_real(par, "sim_smallB");
        s.smallPressure = par_real(par, "sim_smallPressure");
        s.smallDensity = par_real(par, "sim_smallDensity");
        s.smallEnergy = par_real(par, "sim_smallEnergy");
        s.gamma = par_real(par, "sim_gamma");
        std::string rs = par_str(par, "sim_riemannSolver");
        s.cfl = par_real(par, "sim_cfl");
        s.tmax = par_real(par, "sim_tmax");
        s.nstepmax = par_int(par, "sim_nstepmax");
        std::string bcs = par_str(par, "sim_BC");
        s.outputFreqTime = par_real(par, "sim_outputFreqTime");
        s.outputFreqStep = par_int(par, "sim_outputFreqStep");
        s.forceHydro = par_logical(par, "sim_forceHydro");
        if (rs != "hllc" && rs != "hllcmhd") throw ParError{"Unrecognized choice of riemann solver: " + rs};
        if (bcs == "outflow") s.bc = 0;
        else if (bcs == "periodic") s.bc = 1;
        else throw ParError{"Unrecognized choice of boundary condition: " + bcs};
        // GP_init (GP.f90:58-69): grid values read in quad precision
        qp xb = parse_qp(par_str(par, "grid_xBeg")), xe = parse_qp(par_str(par, "grid_xEnd"));
        qp yb = parse_qp(par_str(par, "grid_yBeg")), ye = parse_qp(par_str(par, "grid_yEnd"));
        int nx = par_int(par, "grid_Nx"), ny = par_int(par, "grid_Ny");
        qp dlq[2] = {(xe - xb) / (qp)nx, (ye - yb) / (qp)ny};
        std::string eod = par_str(par, "GP_ellOverDelta");
        h->ellOverDelta = std::strtod(fortran_real_text(eod).c_str(), nullptr);
        int R = par_int(par, "GP_maxRadius");
        std::string gerr;
        if (!gp_build(R, dlq, parse_qp(eod), h->gp, gerr)) throw ParError{gerr};
        grid_init(h->blk, nx, ny, par_real(par, "grid_xBeg"), par_real(par, "grid_xEnd"), par_real(par, "grid_yBeg"),
                  par_real(par, "grid_yEnd"), R, h->gp.nqMax);
        h->U.assign(h->blk.ncell() * NCONS, 0.0);
        h->V.assign(h->blk.ncell() * NPRIM, 0.0);
        initial_condition(h, par);
    } catch (const ParError& e) {
        if (err && errlen > 0) std::snprintf(err, errlen, "%s", e.msg.c_str());
        delete h;
        return nullptr;
    }
    return h;
}

void orc_destroy(orc_handle* h) { delete h; }

int orc_info(const orc_handle* h, int* ints, double* dbls) {
    const Block& b = h->blk;
    if (ints) {
        ints[0] = b.N[0]; ints[1] = b.N[1]; ints[2] = b.NGC; ints[3] = h->gp.R;
        ints[4] = b.nTot[0]; ints[5] = b.nTot[1]; ints[6] = h->gp.nqMax; ints[7] = h->gp.nsMax;
        ints[8] = h->sim.bc; ints[9] = h->sim.forceHydro ? 1 : 0;
    }
    if (dbls) {
        dbls[0] = b.dl[0]; dbls[1] = b.dl[1]; dbls[2] = b.mindxdy; dbls[3] = b.maxdxdy;
        dbls[4] = h->sim.gamma; dbls[5] = h->sim.cfl; dbls[6] = h->sim.tmax; dbls[7] = h->sim.smallPressure;
        dbls[8] = h->sim.smallDensity; dbls[9] = h->ellOverDelta;
    }
    return 0;
}

int orc_get_gp(const orc_handle* h, double* pv, double* qw, int* stenc) {
    if (pv) std::memcpy(pv, h->gp.pv.data(), sizeof(double) * h->gp.pv.size());
    if (qw) std::memcpy(qw, h->gp.qw.data(), sizeof(double) * h->gp.qw.size());
    if (stenc) std::memcpy(stenc, h->gp.stenc.data(), sizeof(int) * h->gp.stenc.size());
    return 0;
}

int orc_get_U(const orc_handle* h, double* U) { std::memcpy(U, h->U.data(), sizeof(double) * h->U.size()); return 0; }
int orc_get_V(const orc_handle* h, double* V) { std::memcpy(V, h->V.data(), sizeof(double) * h->V.size()); return 0; }
int orc_set_U(orc_handle* h, const double* U) { std::memcpy(h->U.data(), U, sizeof(double) * h->U.size()); return 0; }
int orc_set_V(orc_handle* h, const double* V) { std::memcpy(h->V.data(), V, sizeof(double) * h->V.size()); return 0; }
int orc_get_scheme(const orc_handle* h, int* scheme) {
    std::memcpy(scheme, h->blk.scheme.data(), sizeof(int) * h->blk.scheme.size());
    return 0;
}

double orc_cfl(const orc_handle* h) { return cfl_dt(h); }

int orc_advance(orc_handle* h, double dt) {
    advance(h, dt);
    return 0;
}

// src/mhd_driver.f90:64-95 with validTimeStep :117-144 (status instead of stop)
int orc_run(orc_handle* h, int max_steps, double* t_out, int* nstep_out) {
    int nStep = 0;
    double t = 0.0;
    int rc = 0;
    while ((t < h->sim.tmax) && (nStep < h->sim.nstepmax)) {
        if (max_steps > 0 && nStep >= max_steps) break;
        double dt = cfl_dt(h);
        if (t + dt > h->sim.tmax) dt = h->sim.tmax - t;
        else if (dt < 0.0) { rc = 3; break; }
        else if (std::isnan(dt)) { rc = 3; break; }
        else if (!std::isfinite(dt)) { rc = 3; break; }
        advance(h, dt);
        t = t + dt;
        nStep = nStep + 1;
    }
    if (t_out) *t_out = t;
    if (nstep_out) *nstep_out = nStep;
    return rc;
}

int orc_reconstruct_all(orc_handle* h, int radius, double* faceVals) {
    Block& b = h->blk;
    std::fill(b.scheme.begin(), b.scheme.end(), radius);
    std::fill(b.recompute.begin(), b.recompute.end(), 1);
    reconstruct(h, h->U, nullptr, nullptr);
    if (faceVals) std::memcpy(faceVals, b.faceVals.data(), sizeof(double) * b.faceVals.size());
    return 0;
}

// ---------------------------------------------------------------- modules
// The stage modules one at a time on the handle's block and state, in the
// reference's arrays (the per-module form of the CUDA library is checked
// against these).  Unew is the handle's stage output (zero until written).
static std::vector<double>& unew_of(orc_handle* h) {
    if (h->Unew.size() != h->U.size()) h->Unew.assign(h->U.size(), 0.0);
    return h->Unew;
}
int orc_mod_set(orc_handle* h, const int* scheme, const int* recompute, const int* recomputeFLICD) {
    Block& b = h->blk;
    const size_t n = b.ncell();
    for (size_t c = 0; c < n; c++) {
        if (scheme) b.scheme[c] = scheme[c];
        if (recompute) b.recompute[c] = recompute[c] ? 1 : 0;
        if (recomputeFLICD) b.recomputeFLICD[c] = recomputeFLICD[c] ? 1 : 0;
    }
    return 0;
}
int orc_mod_get(orc_handle* h, double* faceVals, double* fluxRaw, double* flux, double* Unew, int* scheme,
                int* recompute, int* recomputeFLICD) {
    Block& b = h->blk;
    if (faceVals) std::memcpy(faceVals, b.faceVals.data(), sizeof(double) * b.faceVals.size());
    if (fluxRaw) std::memcpy(fluxRaw, b.fluxRaw.data(), sizeof(double) * b.fluxRaw.size());
    if (flux) std::memcpy(flux, b.flux.data(), sizeof(double) * b.flux.size());
    if (Unew) std::memcpy(Unew, unew_of(h).data(), sizeof(double) * h->U.size());
    const size_t n = b.ncell();
    for (size_t c = 0; c < n; c++) {
        if (scheme) scheme[c] = b.scheme[c];
        if (recompute) recompute[c] = b.recompute[c];
        if (recomputeFLICD) recomputeFLICD[c] = b.recomputeFLICD[c];
    }
    return 0;
}
int orc_mod_reconstruct(orc_handle* h) {
    reconstruct(h, h->U, nullptr, nullptr);
    return 0;
}
int orc_mod_getfluxes(orc_handle* h) {
    getFluxes(h);
    return 0;
}
int orc_mod_flicd(orc_handle* h) {
    flicd(h);
    return 0;
}
int orc_mod_update(orc_handle* h, double dt) {
    update(h, dt, h->U, unew_of(h));
    return 0;
}
int orc_mod_detect(orc_handle* h) { return detect_all(h, h->U, unew_of(h), nullptr, nullptr) ? 1 : 0; }
int orc_mod_bc(orc_handle* h, int which) {
    if (which == 0) bc_apply(h->blk, h->sim.bc, h->U, NCONS);
    else if (which == 1) bc_apply(h->blk, h->sim.bc, h->V, NPRIM);
    else bc_apply(h->blk, h->sim.bc, unew_of(h), NCONS);
    return 0;
}
int orc_mod_bc_mood(orc_handle* h) {
    bc_apply_mood(h->blk, h->sim.bc);
    return 0;
}

int orc_trace_enable(orc_handle* h, int on) {
    h->trace = on != 0;
    return 0;
}
int orc_trace_count(const orc_handle* h) { return (int)h->traces.size(); }
int orc_trace_get(const orc_handle* h, int k, int* meta, unsigned char* inner, unsigned char* detect) {
    if (k < 0 || k >= (int)h->traces.size()) return 1;
    const Trace& t = h->traces[k];
    if (meta) { meta[0] = t.stage; meta[1] = t.pass; meta[2] = t.nInner; meta[3] = t.nDetect; }
    if (inner && !t.inner.empty()) std::memcpy(inner, t.inner.data(), t.inner.size());
    if (detect && !t.detect.empty()) std::memcpy(detect, t.detect.data(), t.detect.size());
    return 0;
}
void orc_trace_clear(orc_handle* h) {
    h->traces.clear();
    h->stageCounter = 0;
}

void orc_cons2prim(const orc_handle* h, const double* U, double* V) { cons2prim(h->sim, U, V); }
double orc_cons2pres(const orc_handle* h, const double* U) { return cons2pres(h->sim, U); }
void orc_cons2flux(const orc_handle* h, const double* U, int dir, double* F) { cons2flux(h->sim, U, dir, F); }
void orc_hllc(const orc_handle* h, const double* uL, const double* uR, int dir, double* F) { hllc(h->sim, uL, uR, dir, F); }
void orc_eigenvecs(const orc_handle* h, const double* V, int dir, int cons, double* L, double* R) {
    eigen_vecs(h->sim, V, dir, cons != 0, L, R);
}
double orc_c_fs(double gam, double rho, double p, double BB, double BN, double pm) {
    return eigen_c_fs(gam, rho, p, BB, BN, pm);
}

int orc_gp_build(int R, const char* x_beg, const char* x_end, int nx, const char* y_beg, const char* y_end, int ny,
                 const char* ell_over_delta, double* pv, double* qw, int* stenc) {
    GPTab gp;
    qp dl[2] = {(parse_qp(x_end) - parse_qp(x_beg)) / (qp)nx, (parse_qp(y_end) - parse_qp(y_beg)) / (qp)ny};
    std::string err;
    if (!gp_build(R, dl, parse_qp(ell_over_delta), gp, err)) return 1;
    if (pv) std::memcpy(pv, gp.pv.data(), sizeof(double) * gp.pv.size());
    if (qw) std::memcpy(qw, gp.qw.data(), sizeof(double) * gp.qw.size());
    if (stenc) std::memcpy(stenc, gp.stenc.data(), sizeof(int) * gp.stenc.size());
    return 0;
}

void orc_set_threads(int n) {
    if (n > 0) omp_set_num_threads(n);
}
int orc_get_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
