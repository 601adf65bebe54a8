// noalloc.cu -- CFL time step on caller-owned device memory, allocating
// nothing.
//
// Who needs this: a caller that must not (or cannot) call cudaMalloc at the
// point where it wants dt -- for instance code that is inside a CUDA stream
// capture (allocation calls fail there), a host program whose device memory
// is entirely owned by its own pool allocator (a Fortran/OpenACC driver that
// reserved HBM up front), or a time-critical loop that must not hit the
// driver's allocator, which can synchronise the device.  The regular
// hosono_gpu_cfl keeps its reduction scratch in a buffer that
// hosono_gpu_create allocates; this entry point instead keeps it in a
// file-scope device array that exists, per GPU, for the life of the process.
//
// Limits and rules:
//   * at most HOSONO_NOALLOC_MAX_ROWS interior rows (ny); larger grids are
//     rejected with HOSONO_EINVAL before any GPU work;
//   * the scratch array is shared by every call on a device and keeps the
//     last call's contents; each call writes every slot it later reads, so no
//     clearing is needed -- but calls whose kernels overlap on the GPU (two
//     streams, two threads) race on it and must be serialised by the caller;
//   * the array's device address comes from cudaGetSymbolAddress with the
//     device current (the host-side symbol is only a stand-in and must never
//     be handed to a kernel).  A call on a stream that is not capturing looks
//     it up afresh, so the address stays right after a cudaDeviceReset or a
//     context re-creation reloads the module; a call on a capturing stream
//     uses the address the last such call found.  So the first call on each
//     device must come before any stream capture begins (a capturing first
//     call returns HOSONO_EINVAL);
//   * errors: the kernels are launched with cudaLaunchKernel and only its own
//     return codes are reported, so an earlier, unrelated error pending on the
//     calling thread is neither returned nor cleared.

#include "hosono_gpu.h"
#include "physics.cuh"

#include <cuda_runtime.h>

#include <mutex>

namespace {

constexpr int kMaxDevices = 64;
constexpr int kThreads = 256;

// per interior row: max(|u|+c) at [2*row], max(|v|+c) at [2*row+1]
static __device__ __align__(256) double g_cfl_row_max[2 * HOSONO_NOALLOC_MAX_ROWS];

std::mutex g_mutex;
double* g_scratch[kMaxDevices] = {};

// same per-cell speed as cfl.f90:28-44 (and the library's k_cfl_max)
__device__ __forceinline__ void cell_speeds(const double* __restrict__ V, long long plane, long long c, int force_hydro,
                                            double& lx, double& ly) {
    using namespace hosono;
    const double rho = V[DENS * plane + c], pr = V[PRES * plane + c], gam = V[GAMM * plane + c];
    double cs;
    if (force_hydro) {
        cs = sqrt(gam * pr / rho);
    } else {
        const double bx = V[MAGX * plane + c], by = V[MAGY * plane + c], bz = V[MAGZ * plane + c];
        const double BB = bx * bx + by * by + bz * bz;
        const double bmin = fmin(fmin(fabs(bx), fabs(by)), fabs(bz));
        cs = c_fs(gam, rho, pr, BB, bmin, +1.0);
    }
    lx = fabs(V[VELX * plane + c]) + cs;
    ly = fabs(V[VELY * plane + c]) + cs;
}

__device__ __forceinline__ void block_max2(double& a, double& b) {
    __shared__ double sa[kThreads / 32], sb[kThreads / 32];
    for (int o = 16; o > 0; o >>= 1) {
        a = fmax(a, __shfl_xor_sync(0xffffffffu, a, o));
        b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        sa[w] = a;
        sb[w] = b;
    }
    __syncthreads();
    a = l < (int)(blockDim.x >> 5) ? sa[l] : 0.0;
    b = l < (int)(blockDim.x >> 5) ? sb[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) {
        a = fmax(a, __shfl_xor_sync(0xffffffffu, a, o));
        b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
    }
}

// one block per interior row: row maxima into the scratch array
__global__ void __launch_bounds__(kThreads) k_cfl_rows(const double* __restrict__ V, int nx, int ngc, int pitch,
                                                       long long plane, int force_hydro, double* __restrict__ rows) {
    const int r = blockIdx.x;
    double xm = 0.0, ym = 0.0;
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        const long long c = (long long)(r + ngc) * pitch + (i + ngc);
        double lx, ly;
        cell_speeds(V, plane, c, force_hydro, lx, ly);
        xm = fmax(xm, lx);
        ym = fmax(ym, ly);
    }
    block_max2(xm, ym);
    if (threadIdx.x == 0) {
        rows[2 * r] = xm;
        rows[2 * r + 1] = ym;
    }
}

// one block: reduce the row maxima, dt = cfl * min(dx/xmax, dy/ymax) (cfl.f90:50)
__global__ void __launch_bounds__(kThreads) k_cfl_final(const double* __restrict__ rows, int ny, double dx, double dy,
                                                        double cfl, double* __restrict__ dt) {
    double xm = 0.0, ym = 0.0;
    for (int r = threadIdx.x; r < ny; r += blockDim.x) {
        xm = fmax(xm, rows[2 * r]);
        ym = fmax(ym, rows[2 * r + 1]);
    }
    block_max2(xm, ym);
    if (threadIdx.x == 0) *dt = cfl * fmin(dx / xm, dy / ym);
}

// device address of the scratch array on the current device: looked up
// afresh outside a stream capture (a device reset reloads the module at a new
// address), taken from the last lookup inside one
int scratch_for_current_device(cudaStream_t s, double** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();  // this call's own failure
        return HOSONO_ECUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) return HOSONO_EINVAL;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) {
        cudaGetLastError();  // e.g. the legacy stream while another stream captures
        cap = cudaStreamCaptureStatusActive;
    }
    std::lock_guard<std::mutex> lock(g_mutex);
    if (cap == cudaStreamCaptureStatusNone) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_cfl_row_max) != cudaSuccess || !p) {
            cudaGetLastError();
            return HOSONO_ECUDA;
        }
        g_scratch[dev] = static_cast<double*>(p);
    }
    if (!g_scratch[dev]) return HOSONO_EINVAL;  // first call on this device inside a capture
    *out = g_scratch[dev];
    return HOSONO_OK;
}

}  // namespace

extern "C" int hosono_cfl_noalloc(const double* V_dev, int nx, int ny, int ngc, int pitch, long long plane, double dx,
                                  double dy, double cfl, int force_hydro, double* dt_dev, void* stream) {
    if (!V_dev || !dt_dev || nx < 1 || ny < 1 || ngc < 0 || pitch < nx + 2 * ngc ||
        plane < (long long)pitch * (ny + 2 * ngc) || !(dx > 0) || !(dy > 0))
        return HOSONO_EINVAL;
    if (ny > HOSONO_NOALLOC_MAX_ROWS) return HOSONO_EINVAL;  // scratch holds one slot pair per row
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double* rows = nullptr;
    const int rc = scratch_for_current_device(s, &rows);
    if (rc) return rc;
    int fh = force_hydro ? 1 : 0;
    void* rowArgs[] = {(void*)&V_dev, (void*)&nx, (void*)&ngc, (void*)&pitch, (void*)&plane, (void*)&fh, (void*)&rows};
    cudaError_t e = cudaLaunchKernel((const void*)k_cfl_rows, dim3((unsigned)ny), dim3(kThreads), rowArgs, 0, s);
    if (e == cudaSuccess) {
        const double* rowsIn = rows;
        void* finArgs[] = {(void*)&rowsIn, (void*)&ny, (void*)&dx, (void*)&dy, (void*)&cfl, (void*)&dt_dev};
        e = cudaLaunchKernel((const void*)k_cfl_final, dim3(1), dim3(kThreads), finArgs, 0, s);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();  // the launch's own error, reported by the return value
        return HOSONO_ECUDA;
    }
    return HOSONO_OK;
}
