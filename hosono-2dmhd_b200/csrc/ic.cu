// ic.cu -- initialCondition_set (src/initialCondition.f90:86-226) on the
// device, from hosono_ic_describe's constants and per-column / per-row
// tables, with the expressions and order of hosono_ic_set (built without FMA
// contraction, so U and V have the same bits).  Guard cells take the value
// of their boundary source cell (boundaryConditions_apply: periodic wrap or
// outflow edge copy), so no separate boundary fill is needed.
#include "engine.h"
#include "hosono_gpu.h"

namespace hosono {

namespace {
constexpr int TX = 32, TY = 8;

__device__ __forceinline__ int src_cell(int i, int n, int g, int bc) {
    if (i < g) return bc == HOSONO_BC_PERIODIC ? i + n : g;
    if (i >= g + n) return bc == HOSONO_BC_PERIODIC ? i - n : g + n - 1;
    return i;
}

__global__ void k_ic(Geo G, int force_hydro, double gam, hosono_ic_desc ic, const double* __restrict__ xtab,
                     const double* __restrict__ ytab, double* __restrict__ U, double* __restrict__ V) {
    const int i = blockIdx.x * TX + threadIdx.x, j = blockIdx.y * TY + threadIdx.y;
    if (i >= G.nxt || j >= G.nyt) return;
    const int si = src_cell(i, G.nx, G.g, G.bc), sj = src_cell(j, G.ny, G.g, G.bc);
    const double* c = ic.c;
    double v[NPRIM] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (ic.type == HOSONO_IC_EXPLOSION) {  // :86-136
        const double ddx = xtab[si] - c[0], ddy = ytab[sj] - c[1];
        const bool in = sqrt(ddx * ddx + ddy * ddy) <= c[2];
        v[0] = in ? c[3] : c[4];
        v[1] = in ? c[5] : c[8];
        v[2] = in ? c[6] : c[9];
        v[3] = in ? c[7] : c[10];
        v[4] = in ? c[11] : c[12];
        v[5] = c[13];
        v[6] = c[14];
        v[7] = c[15];
    } else if (ic.type == HOSONO_IC_SEDOV) {  // :138-187
        const double ddx = xtab[si] - c[0], ddy = ytab[sj] - c[1];
        v[0] = 1.0;
        v[4] = sqrt(ddx * ddx + ddy * ddy) <= c[2] ? c[3] : 1e-5;
    } else {  // Orszag-Tang :189-226; the sines come from the tables
        const double U0 = c[0], B0 = c[2];
        v[0] = c[1];
        v[1] = -U0 * ytab[G.nyt + sj];
        v[2] = U0 * xtab[G.nxt + si];
        v[3] = 0.0;
        v[5] = -B0 * ytab[G.nyt + sj];
        v[6] = B0 * xtab[2 * G.nxt + si];
        v[7] = 0.0;
        v[4] = c[3];
    }
    // :65-74 eint, gamma and convert_prim2cons (src/convert.f90:159-196)
    v[EINT] = v[4] / (gam - 1.0) / v[0];
    v[GAMM] = gam;
    const double Bp = force_hydro ? 0.0 : 0.5 * (v[5] * v[5] + v[6] * v[6] + v[7] * v[7]);
    const double rhoEint = v[4] / (gam - 1.0);
    double u[NCONS];
    u[0] = v[0];
    u[1] = v[0] * v[1];
    u[2] = v[0] * v[2];
    u[3] = v[0] * v[3];
    u[4] = rhoEint + v[0] * (0.5 * (v[1] * v[1] + v[2] * v[2] + v[3] * v[3])) + Bp;
    u[5] = force_hydro ? 0.0 : v[5];
    u[6] = force_hydro ? 0.0 : v[6];
    u[7] = force_hydro ? 0.0 : v[7];
    const long long cc = (long long)j * G.pitch + i;
#pragma unroll
    for (int k = 0; k < NCONS; k++) U[k * G.plane + cc] = u[k];
#pragma unroll
    for (int k = 0; k < NPRIM; k++) V[k * G.plane + cc] = v[k];
}
}  // namespace

void launch_ic(const Geo& G, int force_hydro, double gamma, const hosono_ic_desc& ic, const double* xtab,
               const double* ytab, double* U, double* V, cudaStream_t s) {
    k_ic<<<dim3((G.nxt + TX - 1) / TX, (G.nyt + TY - 1) / TY), dim3(TX, TY), 0, s>>>(G, force_hydro, gamma, ic, xtab,
                                                                                   ytab, U, V);
}

}  // namespace hosono
