// diagnostics.cu -- the derived output fields of output_writeHdf5
// (src/output.f90:230-274) computed on the device from the resident V and
// scheme, for the interior cells, plus div(B) norms.  Statement order as the
// reference (Fortran left to right, x**2 as x*x); built without FMA
// contraction, so the fields equal the reference's arithmetic bit for bit.
//
// Field planes (nx*ny doubles each, x fastest -- the HDF5 datasets' order):
//   0 dens  1 velx  2 vely  3 velz  4 pres  5 eint  6 gama  7 ener
//   8 magp  9 divb 10 magx 11 magy 12 magz
// and scheme, ordr = 2*scheme + 1 as ints.
#include "engine.h"

namespace hosono {

namespace {
constexpr int TX = 32, TY = 8;

__global__ void k_diag_fields(Geo G, const double* __restrict__ V, const int8_t* __restrict__ sch,
                              double* __restrict__ out, int* __restrict__ schOut, int* __restrict__ ordr) {
    const int ii = blockIdx.x * TX + threadIdx.x, jj = blockIdx.y * TY + threadIdx.y;
    if (ii >= G.nx || jj >= G.ny) return;
    const long long P = G.plane, p = G.pitch;
    const long long c = (long long)(jj + G.g) * p + (ii + G.g);
    const long long n = (long long)G.nx * G.ny, o = (long long)jj * G.nx + ii;
    const double dens = V[c], velx = V[VELX * P + c], vely = V[VELY * P + c], velz = V[VELZ * P + c];
    const double pres = V[PRES * P + c], eint = V[EINT * P + c], gama = V[GAMM * P + c];
    const double magx = V[MAGX * P + c], magy = V[MAGY * P + c], magz = V[MAGZ * P + c];
    // output.f90:256-262
    double ener = dens * (velx * velx + vely * vely + velz * velz) / 2 + dens * eint;
    const double magp = (magx * magx + magy * magy + magz * magz) / 2;
    ener = ener + magp;
    // output.f90:263-274: central differences of B along each direction
    double divb = 0.0;
    divb = divb + 1 / (2 * G.dx) * (V[MAGX * P + c + 1] - V[MAGX * P + c - 1]);
    divb = divb + 1 / (2 * G.dy) * (V[MAGY * P + c + p] - V[MAGY * P + c - p]);
    const double f[13] = {dens, velx, vely, velz, pres, eint, gama, ener, magp, divb, magx, magy, magz};
#pragma unroll
    for (int k = 0; k < 13; k++) out[k * n + o] = f[k];
    const int s = sch[c];
    schOut[o] = s;
    ordr[o] = 2 * s + 1;
}

// Deterministic norms of divb: each row reduced by one block in a fixed
// order, then the rows by one block; the same bits on every call.
constexpr int RT = 256;
__device__ __forceinline__ void block_sum_max(double& s, double& m) {
    __shared__ double ss[RT], sm[RT];
    ss[threadIdx.x] = s;
    sm[threadIdx.x] = m;
    __syncthreads();
    for (int w = RT / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            ss[threadIdx.x] = ss[threadIdx.x] + ss[threadIdx.x + w];
            sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + w]);
        }
        __syncthreads();
    }
    s = ss[0];
    m = sm[0];
}
__global__ void __launch_bounds__(RT) k_divb_rows(const double* __restrict__ divb, int nx, double* rowSum,
                                                  double* rowMax) {
    const double* r = divb + (long long)blockIdx.x * nx;
    double s = 0.0, m = 0.0;
    for (int i = threadIdx.x; i < nx; i += RT) {
        const double a = fabs(r[i]);
        s = s + a;
        m = fmax(m, a);
    }
    block_sum_max(s, m);
    if (threadIdx.x == 0) {
        rowSum[blockIdx.x] = s;
        rowMax[blockIdx.x] = m;
    }
}
__global__ void __launch_bounds__(RT) k_divb_total(const double* rowSum, const double* rowMax, int ny,
                                                   double* res) {
    double s = 0.0, m = 0.0;
    for (int j = threadIdx.x; j < ny; j += RT) {
        s = s + rowSum[j];
        m = fmax(m, rowMax[j]);
    }
    block_sum_max(s, m);
    if (threadIdx.x == 0) {
        res[0] = s;
        res[1] = m;
    }
}
}  // namespace

// fields: 13 planes + 2 int planes of nx*ny on the device; rows: 2*ny
// doubles; res: 2 doubles (sum |divb|, max |divb|)
void launch_diagnostics(const Geo& G, const double* V, const int8_t* scheme, double* fields, int* schOut,
                        int* ordr, double* rows, double* res, cudaStream_t s) {
    k_diag_fields<<<dim3((G.nx + TX - 1) / TX, (G.ny + TY - 1) / TY), dim3(TX, TY), 0, s>>>(G, V, scheme, fields,
                                                                                         schOut, ordr);
    const long long n = (long long)G.nx * G.ny;
    k_divb_rows<<<G.ny, RT, 0, s>>>(fields + 9 * n, G.nx, rows, rows + G.ny);
    k_divb_total<<<1, RT, 0, s>>>(rows, rows + G.ny, G.ny, res);
}

}  // namespace hosono
