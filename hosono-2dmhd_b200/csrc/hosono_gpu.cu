// hosono_gpu.cu -- device instance, MOOD-loop orchestration and the C ABI of
// include/hosono_gpu.h.
//
// One handle = one block (gridBlock_t + gridState_t of the reference) resident
// in HBM.  The forward-Euler stage follows timeStep.f90:45-130: every pass
// reconstructs, fluxes, corrects (FLICD), updates and detects the flagged
// cells until detect lowers nothing; the face cascade of reconstruct.f90:73-173
// runs inside each pass until every high-order face state is admissible.

#include "hosono_gpu.h"
#include "kernels.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdlib>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <utility>
#include <vector>

using namespace hosono;

namespace {

struct TraceRec {
    int stage, pass, nInner, nDetect;
    std::vector<unsigned char> inner, detect;  // Fortran order (i fastest), nxt*nyt
};

}  // namespace

struct hosono_handle {
    hosono_params p{};
    Geo geo{};
    Phys phys{};
    const KernelTable* kt = nullptr;
    cudaStream_t stream = nullptr;
    int device = 0;
    size_t ncellp = 0;  // pitch * nyt
    // state and stage buffers (SoA planes)
    double *Un = nullptr, *A = nullptr, *B = nullptr, *V = nullptr;
    double *FX = nullptr, *FY = nullptr, *CTX = nullptr, *CTY = nullptr;
    double *pv = nullptr, *qw = nullptr;
    double* staging = nullptr;  // AoS <-> SoA conversions
    int* scheme_int = nullptr;
    int8_t *scheme = nullptr, *scheme_next = nullptr;
    uint8_t *rec = nullptr, *recF = nullptr, *rrRec = nullptr, *fail = nullptr, *failX = nullptr, *failY = nullptr;
    uint8_t *nextPass = nullptr, *dirty = nullptr, *lowered = nullptr, *innerCount = nullptr;
    int* counters = nullptr;
    int* h_counters = nullptr;  // pinned
    unsigned long long* cflbits = nullptr;
    unsigned long long* h_cflbits = nullptr;  // pinned
    std::vector<void*> allocations;
    hosono_stats stats{};
    // launch accounting / pass-1 timing
    long long launches = 0;
    bool profile = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    bool evPending = false;
    double pass1Ms = 0.0;
    long long pass1Count = 0;
    bool trace = false;
    int traceStage = 0;
    std::vector<TraceRec> traces;
    int err = HOSONO_OK;
    std::string msg;
};

namespace {

int set_err(hosono_handle* h, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (h) {
        h->err = code;
        h->msg = buf;
    }
    return code;
}

#define CU(h, call)                                                                                   \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess)                                                                        \
            return set_err((h), HOSONO_ECUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                           __FILE__, __LINE__);                                                       \
    } while (0)

template <typename T>
int dalloc(hosono_handle* h, T** p, size_t count) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, count * sizeof(T));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_err(h, HOSONO_ENOMEM, "cudaMalloc of %zu bytes failed: %s", count * sizeof(T),
                       cudaGetErrorString(e));
    }
    h->allocations.push_back(q);
    *p = static_cast<T*>(q);
    return HOSONO_OK;
}

StageArgs stage_args(hosono_handle* h, const double* Uin, double* Uout, double dt) {
    StageArgs a{};
    a.geo = h->geo;
    a.phys = h->phys;
    a.pv = h->pv;
    a.qw = h->qw;
    a.Uin = Uin;
    a.Uout = Uout;
    a.FX = h->FX;
    a.FY = h->FY;
    a.CTX = h->CTX;
    a.CTY = h->CTY;
    a.scheme = h->scheme;
    a.scheme_next = h->scheme_next;
    a.rec = h->rec;
    a.recF = h->recF;
    a.rrRec = h->rrRec;
    a.fail = h->fail;
    a.failX = h->failX;
    a.failY = h->failY;
    a.nextPass = h->nextPass;
    a.dirty = h->dirty;
    a.lowered = h->lowered;
    a.innerCount = h->innerCount;
    a.counters = h->counters;
    a.dt = dt;
    a.trace = h->trace ? 1 : 0;
    return a;
}

int read_counters(hosono_handle* h) {
    CU(h, cudaMemcpyAsync(h->h_counters, h->counters, sizeof(int) * CNT_N, cudaMemcpyDeviceToHost, h->stream));
    CU(h, cudaStreamSynchronize(h->stream));
    return HOSONO_OK;
}

int check_launch(hosono_handle* h, const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_err(h, HOSONO_ECUDA, "launch of %s failed: %s", what, cudaGetErrorString(e));
    return HOSONO_OK;
}

#define LAUNCH(h, what, stmt)                  \
    do {                                       \
        stmt;                                  \
        (h)->launches++;                       \
        int rc_ = check_launch((h), (what));   \
        if (rc_) return rc_;                   \
    } while (0)

// accumulate the pass-1 kernel time once its bracketing events completed
int harvest_profile(hosono_handle* h) {
    if (!h->evPending) return HOSONO_OK;
    float ms = 0.f;
    CU(h, cudaEventSynchronize(h->ev1));
    CU(h, cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    h->pass1Ms += ms;
    h->pass1Count++;
    h->evPending = false;
    return HOSONO_OK;
}

#define TRY(x)              \
    do {                    \
        int rc_ = (x);      \
        if (rc_) return rc_; \
    } while (0)

int record_trace(hosono_handle* h, int stage, int pass, int nInner, int nDetect) {
    const Geo& G = h->geo;
    TraceRec t;
    t.stage = stage;
    t.pass = pass;
    t.nInner = nInner;
    t.nDetect = nDetect;
    std::vector<unsigned char> a(h->ncellp), b(h->ncellp);
    CU(h, cudaMemcpyAsync(a.data(), h->innerCount, h->ncellp, cudaMemcpyDeviceToHost, h->stream));
    CU(h, cudaMemcpyAsync(b.data(), h->lowered, h->ncellp, cudaMemcpyDeviceToHost, h->stream));
    CU(h, cudaStreamSynchronize(h->stream));
    t.inner.resize((size_t)G.nxt * G.nyt);
    t.detect.resize((size_t)G.nxt * G.nyt);
    for (int j = 0; j < G.nyt; j++)
        for (int i = 0; i < G.nxt; i++) {
            t.inner[(size_t)j * G.nxt + i] = a[(size_t)j * G.pitch + i];
            t.detect[(size_t)j * G.nxt + i] = b[(size_t)j * G.pitch + i];
        }
    h->traces.push_back(std::move(t));
    return HOSONO_OK;
}

// timeStep_forwardEuler (timeStep.f90:45-130): Uin (guards filled) -> Uout (interior)
int forward_euler(hosono_handle* h, const double* Uin, double* Uout, double dt) {
    const Geo& G = h->geo;
    const KernelTable* K = h->kt;
    cudaStream_t s = h->stream;
    const size_t n = h->ncellp;
    const uint8_t rrAll = (uint8_t)(G.R | (G.R << 2) | (G.R << 4) | (G.R << 6));
    // scheme = R, recompute = recomputeFLICD = .true. on every cell (:79-81)
    CU(h, cudaMemsetAsync(h->scheme, G.R, n, s));
    CU(h, cudaMemsetAsync(h->rec, 1, n, s));
    CU(h, cudaMemsetAsync(h->recF, 1, n, s));
    CU(h, cudaMemsetAsync(h->rrRec, rrAll, n, s));
    CU(h, cudaMemsetAsync(h->dirty, 0, n, s));
    const int stage = h->traceStage++;
    const long long passCap = (long long)G.R * G.nx * G.ny + 2;
    const long long innerCap = (long long)G.R * (G.nx + 4) * (G.ny + 4) + 2;
    int pass = 0;
    for (;;) {
        if (pass >= passCap) return set_err(h, HOSONO_EMOODCAP, "MOOD loop exceeded %lld passes", passCap);
        CU(h, cudaMemsetAsync(h->counters, 0, sizeof(int) * CNT_N, s));
        if (h->trace) CU(h, cudaMemsetAsync(h->innerCount, 0, n, s));
        StageArgs a = stage_args(h, Uin, Uout, dt);
        // reconstruct_faceValsWithGP, first inner pass
        if (pass == 0) {
            if (h->profile) CU(h, cudaEventRecord(h->ev0, s));
            LAUNCH(h, "face_pass1", K->face_pass1(a, s));
            if (h->profile) {
                CU(h, cudaEventRecord(h->ev1, s));
                h->evPending = true;
            }
        } else {
            CU(h, cudaMemsetAsync(h->fail, 0, n, s));
            LAUNCH(h, "recon_check", K->recon_check(a, h->rec, s));
        }
        TRY(read_counters(h));
        TRY(harvest_profile(h));
        // inner cascade (reconstruct.f90:146-171)
        bool cascaded = false;
        int mode = pass == 0 ? CASCADE_FROM_FACES : CASCADE_FROM_CELLS;
        long long iters = 0;
        while (h->h_counters[CNT_ANYFAIL]) {
            if (++iters > innerCap) return set_err(h, HOSONO_EMOODCAP, "face cascade exceeded %lld passes", innerCap);
            cascaded = true;
            CU(h, cudaMemsetAsync(h->nextPass, 0, n, s));
            LAUNCH(h, "cascade_lower", K->cascade_lower(a, mode, s));
            CU(h, cudaMemsetAsync(h->fail, 0, n, s));
            CU(h, cudaMemsetAsync(h->counters + CNT_ANYFAIL, 0, sizeof(int), s));
            LAUNCH(h, "recon_check", K->recon_check(a, h->nextPass, s));
            TRY(read_counters(h));
            mode = CASCADE_FROM_CELLS;
            h->stats.cascade_iters++;
        }
        // getFluxes_
        if (pass == 0) {
            if (cascaded) LAUNCH(h, "flux", K->flux(a, FLUX_DIRTY, s));
        } else {
            LAUNCH(h, "flux", K->flux(a, FLUX_REC, s));
        }
        // FLICD + update + detect_ALL + applyMOOD
        CU(h, cudaMemsetAsync(h->lowered, 0, n, s));
        LAUNCH(h, "ct_update_detect", K->ct_update_detect(a, s));
        LAUNCH(h, "mood_flags", K->mood_flags(a, s));
        std::swap(h->scheme, h->scheme_next);
        TRY(read_counters(h));
        const int nInner = h->h_counters[CNT_INNER], nDetect = h->h_counters[CNT_DETECT];
        h->stats.inner_lowered += nInner;
        h->stats.detect_lowered += nDetect;
        if (h->trace) TRY(record_trace(h, stage, pass, nInner, nDetect));
        pass++;
        if (nDetect == 0) break;
    }
    h->stats.stages++;
    h->stats.mood_passes += pass;
    if (pass > h->stats.max_passes) h->stats.max_passes = pass;
    return HOSONO_OK;
}

// timeStep_advanceSolution + timeStep_RK3 (timeStep.f90:22-43, :132-171)
int advance(hosono_handle* h, double dt) {
    const Geo& G = h->geo;
    const KernelTable* K = h->kt;
    cudaStream_t s = h->stream;
    h->stats = hosono_stats{};
    TRY(forward_euler(h, h->Un, h->A, dt));                     // U1 = FE(U)
    LAUNCH(h, "bc_fill", K->bc_fill(G, h->A, NCONS, s));        // BC(U1)
    TRY(forward_euler(h, h->A, h->B, dt));                      // U2 = FE(U1)
    LAUNCH(h, "rk_combine2", K->rk_combine2(G, h->Un, h->B, h->A, s));  // U2 = (3U+U2)/4, BC
    TRY(forward_euler(h, h->A, h->B, dt));                      // U3 = FE(U2)
    LAUNCH(h, "rk_final", K->rk_final(G, h->phys, h->Un, h->B, h->A, h->V, s));  // (U+2U3)/3, V, BC
    std::swap(h->Un, h->A);
    return HOSONO_OK;
}

int cfl(hosono_handle* h, double* dt) {
    CU(h, cudaMemsetAsync(h->cflbits, 0, 2 * sizeof(unsigned long long), h->stream));
    LAUNCH(h, "cfl_max", h->kt->cfl_max(h->geo, h->phys, h->V, h->cflbits, h->stream));
    CU(h, cudaMemcpyAsync(h->h_cflbits, h->cflbits, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                          h->stream));
    CU(h, cudaStreamSynchronize(h->stream));
    double xm, ym;
    std::memcpy(&xm, &h->h_cflbits[0], sizeof(double));
    std::memcpy(&ym, &h->h_cflbits[1], sizeof(double));
    // cfl.f90:50
    *dt = h->p.cfl * std::fmin(h->geo.dx / xm, h->geo.dy / ym);
    return HOSONO_OK;
}

int upload(hosono_handle* h, const double* U, const double* V) {
    const Geo& G = h->geo;
    const size_t cells = (size_t)G.nxt * G.nyt;
    CU(h, cudaMemcpyAsync(h->staging, U, cells * NCONS * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    LAUNCH(h, "aos_to_soa", launch_aos_to_soa(G, h->staging, h->Un, NCONS, h->stream));
    if (V) {
        CU(h, cudaMemcpyAsync(h->staging, V, cells * NPRIM * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        LAUNCH(h, "aos_to_soa", launch_aos_to_soa(G, h->staging, h->V, NPRIM, h->stream));
    } else {
        LAUNCH(h, "cons2prim_all", h->kt->cons2prim_all(G, h->phys, h->Un, h->V, h->stream));
    }
    CU(h, cudaStreamSynchronize(h->stream));
    return HOSONO_OK;
}

int download(hosono_handle* h, double* U, double* V, int* scheme) {
    const Geo& G = h->geo;
    const size_t cells = (size_t)G.nxt * G.nyt;
    if (U) {
        LAUNCH(h, "soa_to_aos", launch_soa_to_aos(G, h->Un, h->staging, NCONS, h->stream));
        CU(h, cudaMemcpyAsync(U, h->staging, cells * NCONS * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CU(h, cudaStreamSynchronize(h->stream));
    }
    if (V) {
        LAUNCH(h, "soa_to_aos", launch_soa_to_aos(G, h->V, h->staging, NPRIM, h->stream));
        CU(h, cudaMemcpyAsync(V, h->staging, cells * NPRIM * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CU(h, cudaStreamSynchronize(h->stream));
    }
    if (scheme) {
        LAUNCH(h, "scheme_to_int", launch_scheme_to_int(G, h->scheme, h->scheme_int, h->stream));
        CU(h, cudaMemcpyAsync(scheme, h->scheme_int, cells * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
        CU(h, cudaStreamSynchronize(h->stream));
    }
    return HOSONO_OK;
}

void release(hosono_handle* h) {
    for (void* p : h->allocations) cudaFree(p);
    h->allocations.clear();
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->h_counters) cudaFreeHost(h->h_counters);
    if (h->h_cflbits) cudaFreeHost(h->h_cflbits);
    if (h->stream) cudaStreamDestroy(h->stream);
}

}  // namespace

extern "C" {

int hosono_gpu_create(const hosono_params* p, const double* pv, const double* qw, const int* stenc,
                      hosono_handle** out) {
    if (!p || !pv || !qw || !out) return HOSONO_EINVAL;
    *out = nullptr;
    const int R = p->max_radius;
    if (R < 1 || R > 3) return HOSONO_EINVAL;
    if (p->ngc != R + 2) return HOSONO_EINVAL;
    if (p->nx < 2 * p->ngc || p->ny < 2 * p->ngc) return HOSONO_EINVAL;  // periodic images must not overlap
    if (p->bc != HOSONO_BC_OUTFLOW && p->bc != HOSONO_BC_PERIODIC) return HOSONO_EINVAL;
    if (p->riemann_solver != 1) return HOSONO_EINVAL;
    if (!(p->dx > 0) || !(p->dy > 0)) return HOSONO_EINVAL;
    if (stenc) {  // the kernels hard-code the stencil order of GP.f90:85-95; check it
        const int nsMax = 1 + 2 * R * (R + 1);
        for (int rr = 1; rr <= R; rr++) {
            int k = 0;
            for (int a = -rr; a <= rr; a++)
                for (int b = -rr; b <= rr; b++)
                    if (std::abs(a) + std::abs(b) <= rr) {
                        if (stenc[0 + 2 * (k + nsMax * (rr - 1))] != a || stenc[1 + 2 * (k + nsMax * (rr - 1))] != b)
                            return HOSONO_EINVAL;
                        k++;
                    }
        }
    }
    hosono_handle* h = new (std::nothrow) hosono_handle();
    if (!h) return HOSONO_ENOMEM;
    h->p = *p;
    h->kt = p->fp_mode == HOSONO_FP_FAST ? kernels_fast() : kernels_strict();
    Geo& G = h->geo;
    G.nx = p->nx;
    G.ny = p->ny;
    G.g = p->ngc;
    G.nxt = p->nx + 2 * p->ngc;
    G.nyt = p->ny + 2 * p->ngc;
    G.pitch = (G.nxt + 31) / 32 * 32;
    G.plane = (long long)G.pitch * G.nyt;
    G.R = R;
    G.bc = p->bc;
    G.nsMax = 1 + 2 * R * (R + 1);
    G.nqMax = R + 1;
    G.dx = p->dx;
    G.dy = p->dy;
    G.mindxdy = p->mindxdy;
    G.maxdxdy = p->maxdxdy;
    h->phys.gamma = p->gamma;
    h->phys.small_pressure = p->small_pressure;
    h->phys.small_density = p->small_density;
    h->phys.force_hydro = p->force_hydro ? 1 : 0;
    h->ncellp = (size_t)G.plane;
    const size_t n = h->ncellp;
    const size_t cells = (size_t)G.nxt * G.nyt;
    int rc = HOSONO_OK;
    auto fail = [&](int code) {
        release(h);
        delete h;
        return code;
    };
    if (cudaGetDevice(&h->device) != cudaSuccess) return fail(HOSONO_ECUDA);
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(HOSONO_ECUDA);
    if ((rc = dalloc(h, &h->Un, n * NCONS)) || (rc = dalloc(h, &h->A, n * NCONS)) ||
        (rc = dalloc(h, &h->B, n * NCONS)) || (rc = dalloc(h, &h->V, n * NPRIM)) ||
        (rc = dalloc(h, &h->FX, n * NCONS)) || (rc = dalloc(h, &h->FY, n * NCONS)) ||
        (rc = dalloc(h, &h->CTX, n)) || (rc = dalloc(h, &h->CTY, n)) ||
        (rc = dalloc(h, &h->pv, (size_t)G.nsMax * G.nqMax * 4 * R)) || (rc = dalloc(h, &h->qw, (size_t)G.nqMax * R)) ||
        (rc = dalloc(h, &h->staging, cells * NPRIM)) || (rc = dalloc(h, &h->scheme_int, cells)) ||
        (rc = dalloc(h, &h->scheme, n)) || (rc = dalloc(h, &h->scheme_next, n)) || (rc = dalloc(h, &h->rec, n)) ||
        (rc = dalloc(h, &h->recF, n)) || (rc = dalloc(h, &h->rrRec, n)) || (rc = dalloc(h, &h->fail, n)) ||
        (rc = dalloc(h, &h->failX, n)) || (rc = dalloc(h, &h->failY, n)) || (rc = dalloc(h, &h->nextPass, n)) ||
        (rc = dalloc(h, &h->dirty, n)) || (rc = dalloc(h, &h->lowered, n)) || (rc = dalloc(h, &h->innerCount, n)) ||
        (rc = dalloc(h, &h->counters, CNT_N)) || (rc = dalloc(h, &h->cflbits, 2)))
        return fail(rc);
    if (cudaMallocHost(&h->h_counters, sizeof(int) * CNT_N) != cudaSuccess) return fail(HOSONO_ENOMEM);
    if (cudaMallocHost(&h->h_cflbits, sizeof(unsigned long long) * 2) != cudaSuccess) return fail(HOSONO_ENOMEM);
    // every plane starts zeroed, like gridBlock_alloc / gridState_alloc
    for (void* q : {(void*)h->Un, (void*)h->A, (void*)h->B, (void*)h->FX, (void*)h->FY})
        if (cudaMemsetAsync(q, 0, n * NCONS * sizeof(double), h->stream) != cudaSuccess) return fail(HOSONO_ECUDA);
    if (cudaMemsetAsync(h->V, 0, n * NPRIM * sizeof(double), h->stream) != cudaSuccess) return fail(HOSONO_ECUDA);
    if (cudaMemsetAsync(h->CTX, 0, n * sizeof(double), h->stream) != cudaSuccess) return fail(HOSONO_ECUDA);
    if (cudaMemsetAsync(h->CTY, 0, n * sizeof(double), h->stream) != cudaSuccess) return fail(HOSONO_ECUDA);
    for (uint8_t* q : {(uint8_t*)h->scheme, (uint8_t*)h->scheme_next, h->rec, h->recF, h->rrRec, h->fail, h->failX,
                       h->failY, h->nextPass, h->dirty, h->lowered, h->innerCount})
        if (cudaMemsetAsync(q, 0, n, h->stream) != cudaSuccess) return fail(HOSONO_ECUDA);
    if (cudaMemcpyAsync(h->pv, pv, sizeof(double) * G.nsMax * G.nqMax * 4 * R, cudaMemcpyHostToDevice, h->stream) !=
            cudaSuccess ||
        cudaMemcpyAsync(h->qw, qw, sizeof(double) * G.nqMax * R, cudaMemcpyHostToDevice, h->stream) != cudaSuccess)
        return fail(HOSONO_ECUDA);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return fail(HOSONO_ECUDA);
    *out = h;
    return HOSONO_OK;
}

int hosono_gpu_destroy(hosono_handle* h) {
    if (!h) return HOSONO_OK;
    cudaStreamSynchronize(h->stream);
    release(h);
    delete h;
    return HOSONO_OK;
}

int hosono_gpu_upload(hosono_handle* h, const double* U, const double* V) {
    if (!h || !U) return HOSONO_EINVAL;
    return upload(h, U, V);
}

int hosono_gpu_download(hosono_handle* h, double* U, double* V, int* scheme) {
    if (!h) return HOSONO_EINVAL;
    return download(h, U, V, scheme);
}

int hosono_gpu_cfl(hosono_handle* h, double* dt) {
    if (!h || !dt) return HOSONO_EINVAL;
    return cfl(h, dt);
}

int hosono_gpu_advance(hosono_handle* h, double dt) {
    if (!h) return HOSONO_EINVAL;
    if (!(dt >= 0.0) || !std::isfinite(dt)) return set_err(h, HOSONO_ENANDT, "dt = %g is not a valid time step", dt);
    TRY(advance(h, dt));
    CU(h, cudaStreamSynchronize(h->stream));
    return HOSONO_OK;
}

int hosono_gpu_run(hosono_handle* h, double tmax, int nstepmax, int max_steps, double* t_out, int* nstep_out) {
    if (!h) return HOSONO_EINVAL;
    int nStep = 0;
    double t = 0.0;
    int rc = HOSONO_OK;
    while ((t < tmax) && (nStep < nstepmax)) {
        if (max_steps > 0 && nStep >= max_steps) break;
        double dt = 0;
        if ((rc = cfl(h, &dt))) break;
        // validTimeStep (mhd_driver.f90:239-266): clamp first, then check
        if (t + dt > tmax)
            dt = tmax - t;
        else if (dt < 0.0 || std::isnan(dt) || !std::isfinite(dt)) {
            rc = set_err(h, HOSONO_ENANDT, "dt = %g is not a valid time step", dt);
            break;
        }
        if ((rc = advance(h, dt))) break;
        t = t + dt;
        nStep = nStep + 1;
    }
    if (!rc && cudaStreamSynchronize(h->stream) != cudaSuccess) rc = set_err(h, HOSONO_ECUDA, "stream sync failed");
    if (t_out) *t_out = t;
    if (nstep_out) *nstep_out = nStep;
    return rc;
}

int hosono_gpu_advance_host(hosono_handle* h, double dt, double* U, double* V) {
    if (!h || !U) return HOSONO_EINVAL;
    TRY(upload(h, U, V));
    TRY(hosono_gpu_advance(h, dt));
    return download(h, U, V, nullptr);
}

int hosono_gpu_stats(hosono_handle* h, hosono_stats* s) {
    if (!h || !s) return HOSONO_EINVAL;
    *s = h->stats;
    return HOSONO_OK;
}

int hosono_gpu_last_error(hosono_handle* h, char* buf, int len) {
    if (!h) return HOSONO_EINVAL;
    if (buf && len > 0) std::snprintf(buf, (size_t)len, "%s", h->msg.c_str());
    return h->err;
}

int hosono_gpu_trace_enable(hosono_handle* h, int on) {
    if (!h) return HOSONO_EINVAL;
    h->trace = on != 0;
    return HOSONO_OK;
}
int hosono_gpu_trace_count(hosono_handle* h) { return h ? (int)h->traces.size() : 0; }
int hosono_gpu_trace_get(hosono_handle* h, int k, int* meta, unsigned char* inner, unsigned char* detect) {
    if (!h || k < 0 || k >= (int)h->traces.size()) return HOSONO_EINVAL;
    const TraceRec& t = h->traces[k];
    if (meta) {
        meta[0] = t.stage;
        meta[1] = t.pass;
        meta[2] = t.nInner;
        meta[3] = t.nDetect;
    }
    if (inner) std::memcpy(inner, t.inner.data(), t.inner.size());
    if (detect) std::memcpy(detect, t.detect.data(), t.detect.size());
    return HOSONO_OK;
}
int hosono_gpu_trace_clear(hosono_handle* h) {
    if (!h) return HOSONO_EINVAL;
    h->traces.clear();
    h->traceStage = 0;
    return HOSONO_OK;
}

int hosono_gpu_state_layout(hosono_handle* h, double** U_dev, int* pitch, long long* plane) {
    if (!h) return HOSONO_EINVAL;
    if (U_dev) *U_dev = h->Un;
    if (pitch) *pitch = h->geo.pitch;
    if (plane) *plane = h->geo.plane;
    return HOSONO_OK;
}

int hosono_gpu_build_info(int* sm_arch, int* has_fast_mode) {
    if (sm_arch) *sm_arch = 100;
    if (has_fast_mode) *has_fast_mode = 1;
    return HOSONO_OK;
}

int hosono_gpu_set_device(int device) {
    return cudaSetDevice(device) == cudaSuccess ? HOSONO_OK : HOSONO_ECUDA;
}

int hosono_gpu_stream(hosono_handle* h, void** stream) {
    if (!h || !stream) return HOSONO_EINVAL;
    *stream = (void*)h->stream;
    return HOSONO_OK;
}

int hosono_gpu_profile(hosono_handle* h, int on) {
    if (!h) return HOSONO_EINVAL;
    if (on && !h->ev0) {
        CU(h, cudaEventCreate(&h->ev0));
        CU(h, cudaEventCreate(&h->ev1));
    }
    h->profile = on != 0;
    return HOSONO_OK;
}

int hosono_gpu_profile_read(hosono_handle* h, double* pass1_ms, long long* pass1_launches, long long* launches,
                            int reset) {
    if (!h) return HOSONO_EINVAL;
    TRY(harvest_profile(h));
    if (pass1_ms) *pass1_ms = h->pass1Ms;
    if (pass1_launches) *pass1_launches = h->pass1Count;
    if (launches) *launches = h->launches;
    if (reset) {
        h->pass1Ms = 0.0;
        h->pass1Count = 0;
        h->launches = 0;
    }
    return HOSONO_OK;
}

}  // extern "C"
