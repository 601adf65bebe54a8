// modules.cuh -- the reference's stage modules one at a time, on one
// instance, for a host that drives its own forward-Euler MOOD loop and for
// unit parity of each module.  Included by kernels.cu inside its arithmetic
// namespace (strict or fast), so these kernels share the device physics and
// the arithmetic mode of the fused path.
//
// Unlike the fused path, these kernels keep the reference's block arrays:
// faceVals (gridBlock.f90:51) and flux (:53) live in the module buffers
// (ModBuf), fluxRaw in the instance's FX/FY planes; the MOOD flags are the
// instance's scheme / recompute / recomputeFLICD planes.  One thread per
// cell of the instance's array (2D grid of 32x8 blocks); each kernel tests
// the index range of the reference loop it restates.

__device__ __forceinline__ long long mod_fv(const Geo& G, int f, int q, int v) {
    return ((long long)(f * G.nqMax + q) * NCONS + v) * G.plane;
}

struct ModCell {
    int i, j;
    long long cc;
    bool in;
};
__device__ __forceinline__ ModCell mod_cell(const Geo& G) {
    ModCell c;
    c.i = blockIdx.x * TILE_X + threadIdx.x;
    c.j = blockIdx.y * TILE_Y + threadIdx.y;
    c.in = c.i < G.nxt && c.j < G.nyt;
    c.cc = (long long)c.j * G.pitch + c.i;
    return c;
}
__device__ __forceinline__ bool mod_in(const ModCell& c, int lo, int xhi, int yhi) {
    return c.i >= lo && c.j >= lo && c.i <= xhi && c.j <= yhi;
}

// gridBlock_lowerOrder (gridBlock.f90:194-235): scheme - 1, recompute on the
// cross, recomputeFLICD on the taxicab diamond of radius 2 (clipped to the
// array).  Every flag write sets, so lowerings of several cells commute.
__device__ __forceinline__ void mod_lower_order(const InstDev& d, int8_t* sch, int i, int j, long long cc) {
    const Geo& G = d.geo;
    const int s = sch[cc];
    sch[cc] = (int8_t)(s - 1 > 0 ? s - 1 : 0);
    d.rec[cc] = 1;
    d.rec[cc + 1] = 1;
    d.rec[cc - 1] = 1;
    d.rec[cc + G.pitch] = 1;
    d.rec[cc - G.pitch] = 1;
    for (int jj = j - 2; jj <= j + 2; jj++) {
        if (jj < 0 || jj >= G.nyt) continue;
        for (int ii = i - 2; ii <= i + 2; ii++) {
            if (ii < 0 || ii >= G.nxt) continue;
            if (iabs_c(ii - i) + iabs_c(jj - j) <= 2) d.recF[(long long)jj * G.pitch + ii] = 1;
        }
    }
}

// reconstruct_faceValsWithGP, one inner pass (reconstruct.f90:80-139): every
// cell of [g-2, g+n+1]^2 marked in reconstructCell gets its four faces at
// rr = min(scheme(c), scheme(nbr)) (EDP1): the first-order copy at rr = 0,
// else the GP sums at the rr+1 quadrature points, each tested by CAD/PAD.
__global__ void __launch_bounds__(NTHREADS) k_mod_recon(Batch B, int slot, ModBuf M) {
    const InstDev& d = B.dev[slot];
    const InstState& S = B.st[slot];
    const Geo& G = d.geo;
    const ModCell c = mod_cell(G);
    const int g = G.g;
    if (!c.in || !mod_in(c, g - 2, g + G.nx + 1, g + G.ny + 1) || !M.recon[c.cc]) return;
    const int8_t* sch = d.scheme[S.schemeSel];
    const double* U = role_ptr(d, S.parity, ROLE_STATE);
    bool ok = true;
    for (int f = NORTH; f <= WEST; f++) {
        const long long nb = f == NORTH ? c.cc + G.pitch : f == SOUTH ? c.cc - G.pitch : f == EAST ? c.cc + 1 : c.cc - 1;
        const int s0 = sch[c.cc], s1 = sch[nb];
        const int rr = s0 < s1 ? s0 : s1;
        if (rr == 0) {
#pragma unroll
            for (int v = 0; v < NCONS; v++) M.fv[mod_fv(G, f, 0, v) + c.cc] = U[v * G.plane + c.cc];
            continue;
        }
        for (int q = 0; q <= rr; q++) {
            double u[NCONS];
            face_value(d, U, rr, c.i, c.j, f, q, u);
#pragma unroll
            for (int v = 0; v < NCONS; v++) M.fv[mod_fv(G, f, q, v) + c.cc] = u[v];
            if (!admissible(u[DENS], cons2pres(d.phys, u))) ok = false;
        }
    }
    if (!ok) M.adm[c.cc] = 0;
}

// the serial lowering loop after an inner pass (reconstruct.f90:144-169):
// each inadmissible cell is lowered and its cross marked for the next pass
__global__ void __launch_bounds__(NTHREADS) k_mod_recon_lower(Batch B, int slot, ModBuf M) {
    const InstDev& d = B.dev[slot];
    const InstState& S = B.st[slot];
    const Geo& G = d.geo;
    const ModCell c = mod_cell(G);
    const int g = G.g;
    if (!c.in || !mod_in(c, g - 2, g + G.nx + 1, g + G.ny + 1) || M.adm[c.cc]) return;
    mod_lower_order(d, d.scheme[S.schemeSel], c.i, c.j, c.cc);
    M.next[c.cc] = 1;
    M.next[c.cc + 1] = 1;
    M.next[c.cc - 1] = 1;
    M.next[c.cc + G.pitch] = 1;
    M.next[c.cc - G.pitch] = 1;
    atomicAdd(M.flag, 1);
}

// getFluxes_ (getFluxes.f90:16-90) with riemannSolver_getFaceFlux
// (riemannSolver.f90:23-47): on [g-1, g+n+1]^2, the x-face of (i,j) when
// recompute(i,j) or recompute(i-1,j), the y-face when recompute(i,j) or
// recompute(i,j-1); fluxRaw and flux both take the new value.
__device__ __forceinline__ void mod_face_flux(const InstDev& d, const ModBuf& M, int dir, long long cc, int rr) {
    const Geo& G = d.geo;
    const long long cn = dir == XDIR ? cc - 1 : cc - G.pitch;
    const int fL = dir == XDIR ? EAST : NORTH, fR = dir == XDIR ? WEST : SOUTH;
    double acc[NCONS];
    const int nq = rr == 0 ? 1 : rr + 1;
    for (int q = 0; q < nq; q++) {
        double uL[NCONS], uR[NCONS], F[NCONS];
#pragma unroll
        for (int v = 0; v < NCONS; v++) {
            uL[v] = M.fv[mod_fv(G, fL, q, v) + cn];
            uR[v] = M.fv[mod_fv(G, fR, q, v) + cc];
        }
        hllc(d.phys, uL, uR, dir, F);
        if (rr == 0) {
#pragma unroll
            for (int v = 0; v < NCONS; v++) acc[v] = F[v];
        } else {
            if (q == 0) {
#pragma unroll
                for (int v = 0; v < NCONS; v++) acc[v] = 0.0;
            }
            const double w = qw_at(d, rr, q);
#pragma unroll
            for (int v = 0; v < NCONS; v++) acc[v] = acc[v] + w * F[v];
        }
    }
    double* raw = dir == XDIR ? d.FX : d.FY;
#pragma unroll
    for (int v = 0; v < NCONS; v++) {
        raw[v * G.plane + cc] = acc[v];
        M.flux[(dir * NCONS + v) * G.plane + cc] = acc[v];
    }
}
__global__ void __launch_bounds__(NTHREADS) k_mod_getfluxes(Batch B, int slot, ModBuf M) {
    const InstDev& d = B.dev[slot];
    const InstState& S = B.st[slot];
    const Geo& G = d.geo;
    const ModCell c = mod_cell(G);
    const int g = G.g;
    if (!c.in || !mod_in(c, g - 1, g + G.nx + 1, g + G.ny + 1)) return;
    const int8_t* sch = d.scheme[S.schemeSel];
    const int s0 = sch[c.cc];
    if (d.rec[c.cc] || d.rec[c.cc - 1]) {
        const int s1 = sch[c.cc - 1];
        mod_face_flux(d, M, XDIR, c.cc, s0 < s1 ? s0 : s1);
    }
    if (d.rec[c.cc] || d.rec[c.cc - G.pitch]) {
        const int s1 = sch[c.cc - G.pitch];
        mod_face_flux(d, M, YDIR, c.cc, s0 < s1 ? s0 : s1);
    }
}

// FLICDdivB_fluxCorrections (FLICDdivB.f90:13-70): on [g, g+n]^2 where
// recomputeFLICD, flux(magy, x) and flux(magx, y) from fluxRaw; the host
// then zeroes flux(magx, x) and flux(magy, y) over the whole array.
__global__ void __launch_bounds__(NTHREADS) k_mod_flicd(Batch B, int slot, ModBuf M) {
    const InstDev& d = B.dev[slot];
    const Geo& G = d.geo;
    const ModCell c = mod_cell(G);
    const int g = G.g;
    if (!c.in || !mod_in(c, g, g + G.nx, g + G.ny) || !d.recF[c.cc]) return;
    M.flux[(XDIR * NCONS + MAGY) * G.plane + c.cc] = flicd_x(d, c.cc);
    M.flux[(YDIR * NCONS + MAGX) * G.plane + c.cc] = flicd_y(d, c.cc);
}

// the unsplit update where recomputeFLICD (timeStep.f90:105-118):
// Unew = U - dt/dx (F(i+1) - F(i)) - dt/dy (G(j+1) - G(j)) on the interior
__global__ void __launch_bounds__(NTHREADS) k_mod_update(Batch B, int slot, ModBuf M, double dt) {
    const InstDev& d = B.dev[slot];
    const InstState& S = B.st[slot];
    const Geo& G = d.geo;
    const ModCell c = mod_cell(G);
    const int g = G.g;
    if (!c.in || !mod_in(c, g, g + G.nx - 1, g + G.ny - 1) || !d.recF[c.cc]) return;
    const double* U = role_ptr(d, S.parity, ROLE_STATE);
    double* Un = role_ptr(d, S.parity, ROLE_A);
    const double dtdx = dt / G.dx, dtdy = dt / G.dy;
    const double* FXm = M.flux + (long long)(XDIR * NCONS) * G.plane;
    const double* FYm = M.flux + (long long)(YDIR * NCONS) * G.plane;
#pragma unroll
    for (int v = 0; v < NCONS; v++) {
        const long long o = v * G.plane;
        Un[o + c.cc] = U[o + c.cc] - dtdx * (FXm[o + c.cc + 1] - FXm[o + c.cc]) -
                       dtdy * (FYm[o + c.cc + G.pitch] - FYm[o + c.cc]);
    }
}

// detect_ALL (detect.f90:18-236) on one checked interior cell, in the
// reference's order of decisions: CAD, PAD on Unew; the three shock sensors
// on U; plateau, DMP and the u2 smoothness test
__device__ bool mod_detect_cell(const InstDev& d, const double* __restrict__ U, const double* __restrict__ Un,
                                long long cc) {
    const Geo& G = d.geo;
    const Phys& P = d.phys;
    const long long pl = G.plane, p = G.pitch;
    double un[NCONS];
#pragma unroll
    for (int v = 0; v < NCONS; v++) un[v] = Un[v * pl + cc];
    const double presNew = cons2pres(P, un);
    if (!admissible(un[DENS], presNew)) return true;
    double V[NPRIM], Vip[NPRIM], Vim[NPRIM], Vjp[NPRIM], Vjm[NPRIM];
    {
        double u[NCONS];
        const long long at[5] = {cc, cc + 1, cc - 1, cc + p, cc - p};
        double* out[5] = {V, Vip, Vim, Vjp, Vjm};
        for (int k = 0; k < 5; k++) {
#pragma unroll
            for (int v = 0; v < NCONS; v++) u[v] = U[v * pl + at[k]];
            cons2prim(P, u, out[k]);
        }
    }
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
    const double* rho = U + DENS * pl;
    const double d1 = rho[cc], d2 = rho[cc + 1], d3 = rho[cc - 1], d4 = rho[cc + p], d5 = rho[cc - p];
    const double mn = fmin(fmin(fmin(fmin(d1, d2), d3), d4), d5);
    const double mx = fmax(fmax(fmax(fmax(d1, d2), d3), d4), d5);
    if (mx - mn < G.mindxdy * G.mindxdy * G.mindxdy) return false;  // plateau
    const double dn = un[DENS];
    if ((mn <= dn) && (dn <= mx)) return false;  // DMP
    double mnx = 0, mxx = 0, mny = 0, mxy = 0;
    int k = 0;
    for (int ii = -1; ii <= 1; ii++) {
        for (int jj = -1; jj <= 1; jj++) {
            if (iabs_c(ii) + iabs_c(jj) > 1) continue;
            const long long q = cc + ii + jj * p;
            const double ddx = (rho[q + 1] - 2 * rho[q] + rho[q - 1]) / (dx * dx);
            const double ddy = (rho[q + p] - 2 * rho[q] + rho[q - p]) / (dy * dy);
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
    const double mm = G.mindxdy;
    const bool sx1 = (mnx * mxx > -mm);
    const bool sy1 = (mny * mxy > -mm);
    const bool sx2 = (fmax(fabs(mnx), fabs(mxx)) < mm);
    const bool sy2 = (fmax(fabs(mny), fabs(mxy)) < mm);
    const bool sx3 = (fmin(fabs(mnx), fabs(mxx)) >= 0.5 * fmax(fabs(mnx), fabs(mxx)));
    const bool sy3 = (fmin(fabs(mny), fabs(mxy)) >= 0.5 * fmax(fabs(mny), fabs(mxy)));
    return !((sx1 && sx2 && sy1 && sy2) || (sx1 && sx3 && sy1 && sy3));
}
// the checks (the host copied recomputeFLICD into M.check and cleared both
// flag planes first): lowerCell of every checked interior cell with scheme > 0
__global__ void __launch_bounds__(NTHREADS) k_mod_detect(Batch B, int slot, ModBuf M) {
    const InstDev& d = B.dev[slot];
    const InstState& S = B.st[slot];
    const Geo& G = d.geo;
    const ModCell c = mod_cell(G);
    const int g = G.g;
    if (!c.in || !mod_in(c, g, g + G.nx - 1, g + G.ny - 1) || !M.check[c.cc]) return;
    if (d.scheme[S.schemeSel][c.cc] <= 0) return;
    if (mod_detect_cell(d, role_ptr(d, S.parity, ROLE_STATE), role_ptr(d, S.parity, ROLE_A), c.cc))
        M.lower[c.cc] = 1;
}
// the serial lowering loop of detect_ALL (detect.f90:218-234)
__global__ void __launch_bounds__(NTHREADS) k_mod_detect_lower(Batch B, int slot, ModBuf M) {
    const InstDev& d = B.dev[slot];
    const InstState& S = B.st[slot];
    const Geo& G = d.geo;
    const ModCell c = mod_cell(G);
    const int g = G.g;
    if (!c.in || !mod_in(c, g, g + G.nx - 1, g + G.ny - 1) || !M.lower[c.cc]) return;
    mod_lower_order(d, d.scheme[S.schemeSel], c.i, c.j, c.cc);
    atomicAdd(M.flag, 1);
}

// boundaryConditions_applyMOOD / periodicMOOD (boundaryConditions.f90:16-51,
// :189-254): the x sweep then the y sweep leave every cell with the MIN
// (scheme) and OR (flags) over its translates by the period that lie in the
// array (N >= 2*NGC: one translate each way at most).  Gathered into the
// scratch planes first, copied back by the host, so no cell is read after
// it was written.
__global__ void __launch_bounds__(NTHREADS) k_mod_bc_mood(Batch B, int slot, ModBuf M) {
    const InstDev& d = B.dev[slot];
    const InstState& S = B.st[slot];
    const Geo& G = d.geo;
    const ModCell c = mod_cell(G);
    if (!c.in) return;
    const int8_t* sch = d.scheme[S.schemeSel];
    int s = 127;
    bool r = false, rf = false;
    for (int b = -1; b <= 1; b++) {
        const int jo = c.j + b * G.ny;
        if (jo < 0 || jo >= G.nyt) continue;
        for (int t = -1; t <= 1; t++) {
            const int io = c.i + t * G.nx;
            if (io < 0 || io >= G.nxt) continue;
            const long long co = (long long)jo * G.pitch + io;
            s = min(s, (int)sch[co]);
            r = r || d.rec[co];
            rf = rf || d.recF[co];
        }
    }
    M.tSch[c.cc] = (int8_t)s;
    M.tRec[c.cc] = r;
    M.tRecF[c.cc] = rf;
}

// boundaryConditions_applyBlk (boundaryConditions.f90:53-187) on nv planes as
// a gather from each guard cell's source cell
__global__ void __launch_bounds__(NTHREADS) k_mod_bc(Batch B, int slot, double* A, int nv) {
    const InstDev& d = B.dev[slot];
    const Geo& G = d.geo;
    const ModCell c = mod_cell(G);
    if (!c.in) return;
    const int si = bc_src(c.i, G.nx, G.g, G.bc), sj = bc_src(c.j, G.ny, G.g, G.bc);
    if (si == c.i && sj == c.j) return;
    const long long s = (long long)sj * G.pitch + si;
    for (int v = 0; v < nv; v++) A[v * G.plane + c.cc] = A[v * G.plane + s];
}

// riemannSolver_fromConsHllcMHD (riemannSolver.f90:68-221) on n faces:
// uL, uR, flux are (8, n) arrays, the 8 conserved variables of a face together
__global__ void __launch_bounds__(256) k_mod_riemann(Phys P, int n, const double* __restrict__ uL,
                                                     const double* __restrict__ uR, int dir, double* __restrict__ F) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        double a[NCONS], b[NCONS], f[NCONS];
#pragma unroll
        for (int v = 0; v < NCONS; v++) {
            a[v] = uL[NCONS * e + v];
            b[v] = uR[NCONS * e + v];
        }
        hllc(P, a, b, dir, f);
#pragma unroll
        for (int v = 0; v < NCONS; v++) F[NCONS * e + v] = f[v];
    }
}

// eigen_vecsFromPrim (eigen.f90:20-255) on n primitive states: V is (10, n),
// L and R are (8, 8, n), each 8x8 column-major with one wave per column
__global__ void __launch_bounds__(128) k_mod_eigen(Phys P, int n, const double* __restrict__ V, int dir, int cons,
                                                   double* __restrict__ L, double* __restrict__ R) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        double v[NPRIM], l[NCONS * NCONS], r[NCONS * NCONS];
        for (int k = 0; k < NPRIM; k++) v[k] = V[NPRIM * e + k];
        eigen_vecs(P, v, dir, cons != 0, l, r);
        for (int k = 0; k < NCONS * NCONS; k++) {
            L[NCONS * NCONS * e + k] = l[k];
            R[NCONS * NCONS * e + k] = r[k];
        }
    }
}

dim3 mod_grid(const Geo& G) { return dim3((unsigned)((G.nxt + TILE_X - 1) / TILE_X), (unsigned)((G.nyt + TILE_Y - 1) / TILE_Y)); }
void m_recon(const Batch& B, int slot, const Geo& G, const ModBuf& M, cudaStream_t s) {
    k_mod_recon<<<mod_grid(G), kTile, 0, s>>>(B, slot, M);
}
void m_recon_lower(const Batch& B, int slot, const Geo& G, const ModBuf& M, cudaStream_t s) {
    k_mod_recon_lower<<<mod_grid(G), kTile, 0, s>>>(B, slot, M);
}
void m_getfluxes(const Batch& B, int slot, const Geo& G, const ModBuf& M, cudaStream_t s) {
    k_mod_getfluxes<<<mod_grid(G), kTile, 0, s>>>(B, slot, M);
}
void m_flicd(const Batch& B, int slot, const Geo& G, const ModBuf& M, cudaStream_t s) {
    k_mod_flicd<<<mod_grid(G), kTile, 0, s>>>(B, slot, M);
}
void m_update(const Batch& B, int slot, const Geo& G, const ModBuf& M, double dt, cudaStream_t s) {
    k_mod_update<<<mod_grid(G), kTile, 0, s>>>(B, slot, M, dt);
}
void m_detect(const Batch& B, int slot, const Geo& G, const ModBuf& M, cudaStream_t s) {
    k_mod_detect<<<mod_grid(G), kTile, 0, s>>>(B, slot, M);
}
void m_detect_lower(const Batch& B, int slot, const Geo& G, const ModBuf& M, cudaStream_t s) {
    k_mod_detect_lower<<<mod_grid(G), kTile, 0, s>>>(B, slot, M);
}
void m_bc_mood(const Batch& B, int slot, const Geo& G, const ModBuf& M, cudaStream_t s) {
    k_mod_bc_mood<<<mod_grid(G), kTile, 0, s>>>(B, slot, M);
}
void m_bc(const Batch& B, int slot, const Geo& G, double* A, int nv, cudaStream_t s) {
    k_mod_bc<<<mod_grid(G), kTile, 0, s>>>(B, slot, A, nv);
}
void m_riemann(const Phys& P, int n, const double* uL, const double* uR, int dir, double* F, cudaStream_t s) {
    if (n <= 0) return;
    const int blocks = (n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096;
    k_mod_riemann<<<blocks, 256, 0, s>>>(P, n, uL, uR, dir, F);
}

void m_eigen(const Phys& P, int n, const double* V, int dir, int cons, double* L, double* R, cudaStream_t s) {
    if (n <= 0) return;
    const int blocks = (n + 127) / 128 < 4096 ? (n + 127) / 128 : 4096;
    k_mod_eigen<<<blocks, 128, 0, s>>>(P, n, V, dir, cons, L, R);
}

const ModuleOps mops = {m_recon,  m_recon_lower,  m_getfluxes, m_flicd, m_update, m_detect,
                        m_detect_lower, m_bc_mood, m_bc, m_riemann, m_eigen};
