// layout.cu -- conversions between the reference's Fortran-order AoS host
// arrays (var fastest, then i, then j; guards included) and the device SoA
// planes.  Pure data movement: no arithmetic, one build.
#include "engine.h"

namespace hosono {

namespace {
constexpr int TX = 32, TY = 8;

// rows [j0, j1) of the array (the whole array: 0, nyt)
__global__ void k_aos_to_soa(Geo G, const double* __restrict__ aos, double* __restrict__ soa, int nvar, int j0,
                             int j1) {
    const int i = blockIdx.x * TX + threadIdx.x, j = j0 + blockIdx.y * TY + threadIdx.y;
    if (i >= G.nxt || j >= j1) return;
    const long long f = ((long long)j * G.nxt + i) * nvar;
    const long long c = (long long)j * G.pitch + i;
    for (int v = 0; v < nvar; v++) soa[v * G.plane + c] = aos[f + v];
}

__global__ void k_soa_to_aos(Geo G, const double* __restrict__ soa, double* __restrict__ aos, int nvar) {
    const int i = blockIdx.x * TX + threadIdx.x, j = blockIdx.y * TY + threadIdx.y;
    if (i >= G.nxt || j >= G.nyt) return;
    const long long f = ((long long)j * G.nxt + i) * nvar;
    const long long c = (long long)j * G.pitch + i;
    for (int v = 0; v < nvar; v++) aos[f + v] = soa[v * G.plane + c];
}

__global__ void k_scheme_to_int(Geo G, const int8_t* __restrict__ s, int* __restrict__ out) {
    const int i = blockIdx.x * TX + threadIdx.x, j = blockIdx.y * TY + threadIdx.y;
    if (i >= G.nxt || j >= G.nyt) return;
    out[(long long)j * G.nxt + i] = s[(long long)j * G.pitch + i];
}

dim3 grid_of(const Geo& G) { return dim3((G.nxt + TX - 1) / TX, (G.nyt + TY - 1) / TY); }
}  // namespace

void launch_aos_to_soa(const Geo& G, const double* aos, double* soa, int nvar, cudaStream_t s) {
    k_aos_to_soa<<<grid_of(G), dim3(TX, TY), 0, s>>>(G, aos, soa, nvar, 0, G.nyt);
}
void launch_aos_to_soa_rows(const Geo& G, const double* aos, double* soa, int nvar, int j0, int j1, cudaStream_t s) {
    if (j1 <= j0) return;
    const dim3 grid((G.nxt + TX - 1) / TX, (j1 - j0 + TY - 1) / TY);
    k_aos_to_soa<<<grid, dim3(TX, TY), 0, s>>>(G, aos, soa, nvar, j0, j1);
}
void launch_soa_to_aos(const Geo& G, const double* soa, double* aos, int nvar, cudaStream_t s) {
    k_soa_to_aos<<<grid_of(G), dim3(TX, TY), 0, s>>>(G, soa, aos, nvar);
}
void launch_scheme_to_int(const Geo& G, const int8_t* scheme, int* out, cudaStream_t s) {
    k_scheme_to_int<<<grid_of(G), dim3(TX, TY), 0, s>>>(G, scheme, out);
}

}  // namespace hosono
