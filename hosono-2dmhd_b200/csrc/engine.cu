// engine.cu -- host side of the batched engine: instance slots, device
// tables, and the time-step structure (timeStep.f90:22-171 with the driver
// loop of mhd_driver.f90:198-217) recorded either as eager launches driven by
// host loops, or as one CUDA graph whose loops are conditional WHILE nodes:
//
//   run:   WHILE(any instance stepping) {
//            step_prepare, cfl_reduce, step_begin (dt, validTimeStep)
//            stage(U->A), bc(A), stage(A->B), A=(3U+B)/4, stage(A->B), A=(U+2B)/3 + V
//            step_end (t += dt, state = A) }
//   stage: init, pass-1 kernel, WHILE(cascade) {lower, re-reconstruct}, fluxes,
//          FLICD+update+detect, flags, pass_end,
//          WHILE(MOOD) { re-reconstruct flagged, WHILE(cascade) {...}, fluxes,
//                        FLICD+update+detect, flags, pass_end }
//
// Each loop condition is set on the device by the kernel that ends the loop
// body (cudaGraphSetConditional), so a whole run is one graph launch.

#include "engine_host.h"

#include <cmath>
#include <climits>
#include <cstdarg>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <utility>

namespace hosono {

#define CUE(call)                                                                                               \
    do {                                                                                                        \
        cudaError_t e_ = (call);                                                                                \
        if (e_ != cudaSuccess) return fail(HOSONO_ECUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                                           __LINE__);                                                           \
    } while (0)

#define TRYE(x)              \
    do {                     \
        int rc_ = (x);       \
        if (rc_) return rc_; \
    } while (0)

int Engine::fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    err = code;
    msg = buf;
    return code;
}

// ----------------------------------------------------------------------
// Recorder: eager launches, or capture into a graph with conditional nodes.
class Engine::Rec {
  public:
    Rec(Engine* e, cudaGraph_t g) : e_(e), g_(g) {}
    bool graph() const { return g_ != nullptr; }

    int begin() {
        if (g_ && !open_) {
            cudaError_t r = cudaStreamBeginCaptureToGraph(e_->s_, g_, deps_.empty() ? nullptr : deps_.data(), nullptr,
                                                          deps_.size(), cudaStreamCaptureModeThreadLocal);
            if (r != cudaSuccess) return e_->fail(HOSONO_ECUDA, "begin capture: %s", cudaGetErrorString(r));
            open_ = true;
        }
        return HOSONO_OK;
    }
    int end() {
        if (g_ && open_) {
            cudaStreamCaptureStatus st;
            const cudaGraphNode_t* d = nullptr;
            size_t n = 0;
            cudaError_t r = cudaStreamGetCaptureInfo(e_->s_, &st, nullptr, nullptr, &d, &n);
            if (r != cudaSuccess) return e_->fail(HOSONO_ECUDA, "capture info: %s", cudaGetErrorString(r));
            std::vector<cudaGraphNode_t> tail(d, d + n);
            cudaGraph_t out = nullptr;
            r = cudaStreamEndCapture(e_->s_, &out);
            if (r != cudaSuccess) return e_->fail(HOSONO_ECUDA, "end capture: %s", cudaGetErrorString(r));
            deps_ = tail;
            open_ = false;
        }
        return HOSONO_OK;
    }
    template <class F>
    int k(F&& f) {
        TRYE(begin());
        f(e_->s_);
        if (!g_) e_->launches++;
        cudaError_t r = cudaGetLastError();
        if (r != cudaSuccess) return e_->fail(HOSONO_ECUDA, "kernel launch: %s", cudaGetErrorString(r));
        return HOSONO_OK;
    }
    int event(cudaEvent_t ev) {
        TRYE(begin());
        // External: under capture this becomes an event-record node of the graph
        cudaError_t r = g_ ? cudaEventRecordWithFlags(ev, e_->s_, cudaEventRecordExternal) : cudaEventRecord(ev, e_->s_);
        if (r != cudaSuccess) return e_->fail(HOSONO_ECUDA, "event record: %s", cudaGetErrorString(r));
        return HOSONO_OK;
    }
    int cond(cudaGraphConditionalHandle* h, unsigned dflt) {
        *h = 0;
        if (!g_) return HOSONO_OK;
        TRYE(end());
        cudaError_t r = cudaGraphConditionalHandleCreate(h, g_, dflt, cudaGraphCondAssignDefault);
        if (r != cudaSuccess) return e_->fail(HOSONO_ECUDA, "conditional handle: %s", cudaGetErrorString(r));
        return HOSONO_OK;
    }
    // WHILE(flag) body.  Eager: the host reads the flag the preceding
    // condition kernel wrote.  Graph: a conditional WHILE node.
    template <class Body>
    int loop(cudaGraphConditionalHandle h, int BatchFlags::*field, long long cap, Body&& body) {
        if (!g_) {
            TRYE(e_->sync());
            long long it = 0;
            while (e_->h_flags_->*field) {
                if (++it > cap) return e_->fail(HOSONO_EMOODCAP, "loop exceeded %lld iterations", cap);
                TRYE(body(*this));
                TRYE(e_->sync());
            }
            return HOSONO_OK;
        }
        TRYE(end());
        cudaGraphNodeParams p = {};
        p.type = cudaGraphNodeTypeConditional;
        p.conditional.handle = h;
        p.conditional.type = cudaGraphCondTypeWhile;
        p.conditional.size = 1;
        cudaGraphNode_t node;
        cudaError_t r = cudaGraphAddNode(&node, g_, deps_.empty() ? nullptr : deps_.data(), deps_.size(), &p);
        if (r != cudaSuccess) return e_->fail(HOSONO_ECUDA, "conditional node: %s", cudaGetErrorString(r));
        Rec sub(e_, p.conditional.phGraph_out[0]);
        TRYE(body(sub));
        TRYE(sub.end());
        deps_.assign(1, node);
        return HOSONO_OK;
    }
    template <class H>
    int host(H&& h) {
        if (g_) return HOSONO_OK;
        TRYE(e_->sync());
        return h();
    }

  private:
    Engine* e_;
    cudaGraph_t g_;
    std::vector<cudaGraphNode_t> deps_;
    bool open_ = false;
};

// ----------------------------------------------------------------------
Engine::~Engine() {
    if (s_) cudaStreamSynchronize(s_);
    for (auto& sl : slots_)
        for (void* p : sl.allocs) dfree(p);
    for (cudaGraphExec_t g : {gAdvance_, gRun_, gProf_})
        if (g) cudaGraphExecDestroy(g);
    for (cudaEvent_t ev : profEv_)
        if (ev) cudaEventDestroy(ev);
    for (void* p : {(void*)d_instTiles_, (void*)d_actRange_, (void*)d_actInfo_, (void*)d_casRange_,
                    (void*)d_casInfo_})
        if (p) cudaFree(p);
    for (void* p : {(void*)d_dev_, (void*)d_st_, (void*)d_tiles_, (void*)d_ntiles_, (void*)d_flags_, (void*)staging_,
                    (void*)schemeInt_, (void*)lists_.rec, (void*)lists_.face, (void*)lists_.recF, (void*)lists_.low,
                    (void*)lists_.next, (void*)lists_.casc, (void*)lists_.sync, (void*)lists_.rec2,
                    (void*)lists_.counts})
        if (p) cudaFree(p);
    if (h_flags_) cudaFreeHost(h_flags_);
    if (h_st_) cudaFreeHost(h_st_);
    if (s_) cudaStreamDestroy(s_);
}

int Engine::init(int max_inst, int max_tiles, int fp_mode) {
    if (max_inst < 1 || max_tiles < 1) return fail(HOSONO_EINVAL, "engine capacity must be positive");
    maxInst_ = max_inst;
    maxTiles_ = max_tiles;
    K_ = fp_mode == HOSONO_FP_FAST ? kernelset_fast() : kernelset_strict();
    CUE(cudaStreamCreateWithFlags(&s_, cudaStreamNonBlocking));
    CUE(cudaMalloc(&d_dev_, sizeof(InstDev) * maxInst_));
    CUE(cudaMalloc(&d_st_, sizeof(InstState) * maxInst_));
    CUE(cudaMalloc(&d_tiles_, sizeof(int4) * maxTiles_));
    CUE(cudaMalloc(&d_instTiles_, sizeof(int2) * maxInst_));
    CUE(cudaMalloc(&d_actRange_, sizeof(int2) * maxInst_));
    CUE(cudaMalloc(&d_actInfo_, sizeof(int) * 2));
    CUE(cudaMalloc(&d_casRange_, sizeof(int2) * maxInst_));
    CUE(cudaMalloc(&d_casInfo_, sizeof(int) * 2));
    CUE(cudaMemsetAsync(d_casInfo_, 0, sizeof(int) * 2, s_));
    CUE(cudaMemsetAsync(d_instTiles_, 0, sizeof(int2) * maxInst_, s_));
    CUE(cudaMemsetAsync(d_actInfo_, 0, sizeof(int) * 2, s_));
    instTiles_.assign(maxInst_, make_int2(0, 0));
    CUE(cudaMalloc(&d_ntiles_, sizeof(int)));
    CUE(cudaMalloc(&d_flags_, sizeof(BatchFlags)));
    lists_.cap = (long long)maxTiles_ * TILE_X * TILE_Y;
    CUE(cudaMalloc(&lists_.rec, sizeof(int2) * lists_.cap));
    CUE(cudaMalloc(&lists_.rec2, sizeof(int2) * lists_.cap));
    CUE(cudaMalloc(&lists_.face, sizeof(int2) * 2 * lists_.cap));
    CUE(cudaMalloc(&lists_.recF, sizeof(int2) * lists_.cap));
    CUE(cudaMalloc(&lists_.low, sizeof(int2) * lists_.cap));
    CUE(cudaMalloc(&lists_.next, sizeof(int2) * lists_.cap));
    CUE(cudaMalloc(&lists_.casc, sizeof(int2) * lists_.cap));
    CUE(cudaMalloc(&lists_.sync, sizeof(int8_t) * 2 * lists_.cap));
    CUE(cudaMalloc(&lists_.counts, sizeof(int) * (LIST_N + 1)));
    CUE(cudaMemsetAsync(lists_.counts, 0, sizeof(int) * (LIST_N + 1), s_));
    CUE(cudaMallocHost(&h_flags_, sizeof(BatchFlags)));
    CUE(cudaMallocHost(&h_st_, sizeof(InstState) * maxInst_));
    CUE(cudaMemsetAsync(d_dev_, 0, sizeof(InstDev) * maxInst_, s_));
    CUE(cudaMemsetAsync(d_st_, 0, sizeof(InstState) * maxInst_, s_));
    CUE(cudaMemsetAsync(d_ntiles_, 0, sizeof(int), s_));
    CUE(cudaMemsetAsync(d_flags_, 0, sizeof(BatchFlags), s_));
    std::memset(h_flags_, 0, sizeof(BatchFlags));
    slots_.assign(maxInst_, Slot{});
    traceStageBase.assign(maxInst_, 0);
    tracePassesSeen_.assign(maxInst_, 0);
    for (cudaEvent_t& ev : profEv_) CUE(cudaEventCreate(&ev));
    CUE(cudaStreamSynchronize(s_));
    return HOSONO_OK;
}

Batch Engine::batch() const {
    Batch B;
    B.dev = d_dev_;
    B.st = d_st_;
    B.tiles = d_tiles_;
    B.ntiles = d_ntiles_;
    B.flags = d_flags_;
    B.L = lists_;
    B.maxTiles = maxTiles_;
    B.maxInst = maxInst_;
    B.instTiles = d_instTiles_;
    B.actRange = d_actRange_;
    B.actInfo = d_actInfo_;
    B.casRange = d_casRange_;
    B.casInfo = d_casInfo_;
    return B;
}

int Engine::sync() {
    CUE(cudaMemcpyAsync(h_flags_, d_flags_, sizeof(BatchFlags), cudaMemcpyDeviceToHost, s_));
    CUE(cudaStreamSynchronize(s_));
    return HOSONO_OK;
}

int Engine::tiles_of(const hosono_params& p) const {
    const int nxt = p.nx + 2 * p.ngc, nyt = p.ny + 2 * p.ngc;
    return ((nxt + TILE_X - 1) / TILE_X) * ((nyt + TILE_Y - 1) / TILE_Y);
}

int Engine::live_count() const {
    int n = 0;
    for (const auto& s : slots_) n += s.live ? 1 : 0;
    return n;
}

namespace {
constexpr int kDoublePlanes = 3 * NCONS + NPRIM + 2 * NCONS + 2;  // U x3, V, FX, FY, CTX, CTY
constexpr int kBytePlanes = 13;
size_t plane_of(const hosono_params& p) {
    const size_t nxt = p.nx + 2 * p.ngc, nyt = p.ny + 2 * p.ngc;
    const size_t pitch = (nxt + 31) / 32 * 32;
    return pitch * nyt;
}
}  // namespace

size_t Engine::instance_bytes(const hosono_params& p) const {
    const int R = p.max_radius;
    const size_t nsMax = 1 + 2 * R * (R + 1), nqMax = R + 1;
    return plane_of(p) * (kDoublePlanes * sizeof(double) + kBytePlanes) + (nsMax * nqMax * 4 * R + nqMax * R) * 8 + 512;
}

int Engine::upload_tables() {
    tiles_.clear();
    radii_ = 0;
    for (int k = 0; k < maxInst_; k++) {
        instTiles_[k] = make_int2((int)tiles_.size(), 0);
        if (!slots_[k].live) continue;
        const Geo& G = slots_[k].dev.geo;
        radii_ |= 1 << G.R;
        for (int y = 0; y < G.nyt; y += TILE_Y)
            for (int x = 0; x < G.nxt; x += TILE_X) tiles_.push_back(make_int4(k, x, y, 0));
        instTiles_[k].y = (int)tiles_.size() - instTiles_[k].x;
    }
    if ((int)tiles_.size() > maxTiles_) return fail(HOSONO_EINVAL, "tile capacity exceeded");
    const int n = (int)tiles_.size();
    if (n) CUE(cudaMemcpyAsync(d_tiles_, tiles_.data(), sizeof(int4) * n, cudaMemcpyHostToDevice, s_));
    CUE(cudaMemcpyAsync(d_ntiles_, &n, sizeof(int), cudaMemcpyHostToDevice, s_));
    CUE(cudaMemcpyAsync(&d_flags_->radii, &radii_, sizeof(int), cudaMemcpyHostToDevice, s_));
    CUE(cudaMemcpyAsync(d_instTiles_, instTiles_.data(), sizeof(int2) * maxInst_, cudaMemcpyHostToDevice, s_));
    CUE(cudaStreamSynchronize(s_));
    return HOSONO_OK;
}

int Engine::write_state_field(int slot, size_t offset, const void* src, size_t n) {
    CUE(cudaMemcpyAsync((char*)(d_st_ + slot) + offset, src, n, cudaMemcpyHostToDevice, s_));
    CUE(cudaStreamSynchronize(s_));
    return HOSONO_OK;
}

int Engine::state(int slot, InstState* out) {
    if (slot < 0 || slot >= maxInst_) return fail(HOSONO_EINVAL, "bad slot %d", slot);
    CUE(cudaMemcpyAsync(out, d_st_ + slot, sizeof(InstState), cudaMemcpyDeviceToHost, s_));
    CUE(cudaStreamSynchronize(s_));
    return HOSONO_OK;
}

void* Engine::dalloc(size_t bytes) {
    if (alloc_) return alloc_->alloc(bytes);
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return p;
}

void Engine::dfree(void* p) {
    if (!p) return;
    if (alloc_)
        alloc_->release(p);
    else
        cudaFree(p);
}

int Engine::reserve_staging(size_t cells) {
    if (cells <= stagingCells_) return HOSONO_OK;
    CUE(cudaStreamSynchronize(s_));
    if (staging_) cudaFree(staging_);
    if (schemeInt_) cudaFree(schemeInt_);
    staging_ = nullptr;
    schemeInt_ = nullptr;
    stagingCells_ = 0;
    CUE(cudaMalloc(&staging_, sizeof(double) * cells * NPRIM));
    CUE(cudaMalloc(&schemeInt_, sizeof(int) * cells));
    stagingCells_ = cells;
    return HOSONO_OK;
}

int Engine::add(const hosono_params& p, const double* pv, const double* qw, int* slot_out, bool commit) {
    const int R = p.max_radius;
    if (R < 1 || R > 3 || p.ngc != R + 2 || p.nx < 2 * p.ngc || p.ny < 2 * p.ngc ||
        (p.bc != HOSONO_BC_OUTFLOW && p.bc != HOSONO_BC_PERIODIC) || p.riemann_solver != 1 || !(p.dx > 0) ||
        !(p.dy > 0) || !pv || !qw)
        return fail(HOSONO_EINVAL, "invalid instance parameters");
    int k = -1;
    for (int t = 0; t < maxInst_; t++)
        if (!slots_[t].live) {
            k = t;
            break;
        }
    if (k < 0) return fail(HOSONO_EINVAL, "no free instance slot");
    if (used_tiles() + tiles_of(p) > maxTiles_) return fail(HOSONO_EINVAL, "tile capacity exceeded");
    Slot sl;
    sl.p = p;
    Geo& G = sl.dev.geo;
    G.nx = p.nx;
    G.ny = p.ny;
    G.g = p.ngc;
    G.nxt = p.nx + 2 * p.ngc;
    G.nyt = p.ny + 2 * p.ngc;
    G.pitch = (G.nxt + 31) / 32 * 32;
    G.plane = (long long)G.pitch * G.nyt;
    G.R = R;
    G.bc = p.bc;
    G.nsMax = 1 + 2 * R * (R + 1);
    G.nqMax = R + 1;
    G.dx = p.dx;
    G.dy = p.dy;
    G.mindxdy = p.mindxdy;
    G.maxdxdy = p.maxdxdy;
    sl.dev.phys.gamma = p.gamma;
    sl.dev.phys.small_pressure = p.small_pressure;
    sl.dev.phys.small_density = p.small_density;
    sl.dev.phys.force_hydro = p.force_hydro ? 1 : 0;
    sl.dev.cfl = p.cfl;
    const size_t plane = (size_t)G.plane;
    const size_t npv = (size_t)G.nsMax * G.nqMax * 4 * R, nqw = (size_t)G.nqMax * R;
    double* dbl = (double*)dalloc(sizeof(double) * (plane * kDoublePlanes + npv + nqw));
    if (!dbl) return fail(HOSONO_ENOMEM, "no device memory for the instance state");
    sl.allocs.push_back(dbl);
    uint8_t* byt = (uint8_t*)dalloc(plane * kBytePlanes);
    if (!byt) {
        dfree(dbl);
        return fail(HOSONO_ENOMEM, "no device memory for the instance flags");
    }
    sl.allocs.push_back(byt);
    double* q = dbl;
    for (int r = 0; r < 3; r++, q += plane * NCONS) sl.dev.U[r] = q;
    sl.dev.V = q;
    q += plane * NPRIM;
    sl.dev.FX = q;
    q += plane * NCONS;
    sl.dev.FY = q;
    q += plane * NCONS;
    sl.dev.CTX = q;
    q += plane;
    sl.dev.CTY = q;
    q += plane;
    double* dpv = q;
    double* dqw = q + npv;
    sl.dev.pv = dpv;
    sl.dev.qw = dqw;
    uint8_t* b = byt;
    sl.dev.scheme[0] = (int8_t*)b;
    sl.dev.scheme[1] = (int8_t*)(b + plane);
    b += 2 * plane;
    uint8_t** bp[] = {&sl.dev.rec, &sl.dev.recF, &sl.dev.rrRec, &sl.dev.fail, &sl.dev.failX,
                      &sl.dev.failY, &sl.dev.nextPass, &sl.dev.dirty, &sl.dev.lowered, &sl.dev.innerCount,
                      &sl.dev.detMask};
    for (uint8_t** pp : bp) {
        *pp = b;
        b += plane;
    }
    CUE(cudaMemsetAsync(dbl, 0, sizeof(double) * plane * kDoublePlanes, s_));
    CUE(cudaMemsetAsync(byt, 0, plane * kBytePlanes, s_));
    CUE(cudaMemcpyAsync(dpv, pv, sizeof(double) * npv, cudaMemcpyHostToDevice, s_));
    CUE(cudaMemcpyAsync(dqw, qw, sizeof(double) * nqw, cudaMemcpyHostToDevice, s_));
    CUE(cudaMemcpyAsync(d_dev_ + k, &sl.dev, sizeof(InstDev), cudaMemcpyHostToDevice, s_));
    InstState st{};
    st.live = 1;
    st.tmax = HUGE_VAL;
    st.nstepmax = INT_MAX;
    st.passCap = (int)std::min<long long>((long long)R * p.nx * p.ny + 2, INT_MAX);
    CUE(cudaMemcpyAsync(d_st_ + k, &st, sizeof(InstState), cudaMemcpyHostToDevice, s_));
    sl.live = true;
    sl.ntiles = tiles_of(p);
    slots_[k] = sl;
    traceStageBase[k] = 0;
    tracePassesSeen_[k] = 0;
    if (commit) TRYE(upload_tables());
    TRYE(reserve_staging((size_t)G.nxt * G.nyt));
    *slot_out = k;
    return HOSONO_OK;
}

int Engine::remove(int slot, bool commit) {
    if (slot < 0 || slot >= maxInst_ || !slots_[slot].live) return fail(HOSONO_EINVAL, "bad slot %d", slot);
    CUE(cudaStreamSynchronize(s_));
    InstState st{};
    CUE(cudaMemcpyAsync(d_st_ + slot, &st, sizeof(InstState), cudaMemcpyHostToDevice, s_));
    slots_[slot].live = false;
    if (commit) TRYE(upload_tables());
    CUE(cudaStreamSynchronize(s_));  // no kernel of this stream still reads the memory
    for (void* p : slots_[slot].allocs) dfree(p);
    slots_[slot] = Slot{};
    return HOSONO_OK;
}

int Engine::upload(int slot, const double* U, const double* V) {
    if (slot < 0 || slot >= maxInst_ || !slots_[slot].live || !U) return fail(HOSONO_EINVAL, "bad upload");
    InstState st;
    TRYE(state(slot, &st));
    const Slot& sl = slots_[slot];
    const Geo& G = sl.dev.geo;
    const size_t cells = (size_t)G.nxt * G.nyt;
    CUE(cudaMemcpyAsync(staging_, U, cells * NCONS * sizeof(double), cudaMemcpyHostToDevice, s_));
    launch_aos_to_soa(G, staging_, sl.dev.U[st.parity], NCONS, s_);
    launches++;
    if (V) {
        CUE(cudaMemcpyAsync(staging_, V, cells * NPRIM * sizeof(double), cudaMemcpyHostToDevice, s_));
        launch_aos_to_soa(G, staging_, sl.dev.V, NPRIM, s_);
        launches++;
        CUE(cudaGetLastError());
        CUE(cudaStreamSynchronize(s_));
    } else {
        TRYE(write_field(slot, &InstState::stepping, 1));
        K_->cons2prim_all(batch(), s_);
        launches++;
        CUE(cudaGetLastError());
        TRYE(write_field(slot, &InstState::stepping, 0));
    }
    return HOSONO_OK;
}

int Engine::ic(int slot, const hosono_ic_desc& d, const double* xtab, const double* ytab) {
    if (slot < 0 || slot >= maxInst_ || !slots_[slot].live || !xtab || !ytab) return fail(HOSONO_EINVAL, "bad ic");
    if (d.type != HOSONO_IC_EXPLOSION && d.type != HOSONO_IC_SEDOV && d.type != HOSONO_IC_ORSZAG_TANG)
        return fail(HOSONO_EINVAL, "unknown initial-condition type %d", d.type);
    InstState st;
    TRYE(state(slot, &st));
    const Slot& sl = slots_[slot];
    const Geo& G = sl.dev.geo;
    // the tables go through the staging buffer (cells*10 doubles >= 3*nxt + 2*nyt)
    CUE(cudaMemcpyAsync(staging_, xtab, sizeof(double) * 3 * G.nxt, cudaMemcpyHostToDevice, s_));
    CUE(cudaMemcpyAsync(staging_ + 3 * G.nxt, ytab, sizeof(double) * 2 * G.nyt, cudaMemcpyHostToDevice, s_));
    launch_ic(G, sl.dev.phys.force_hydro, sl.dev.phys.gamma, d, staging_, staging_ + 3 * G.nxt, sl.dev.U[st.parity],
              sl.dev.V, s_);
    launches++;
    CUE(cudaGetLastError());
    CUE(cudaStreamSynchronize(s_));
    return HOSONO_OK;
}

int Engine::diagnostics(int slot, double* fields, int* scheme, int* ordr, double* divb_l1, double* divb_linf) {
    if (slot < 0 || slot >= maxInst_ || !slots_[slot].live) return fail(HOSONO_EINVAL, "bad diagnostics slot");
    InstState st;
    TRYE(state(slot, &st));
    const Slot& sl = slots_[slot];
    const Geo& G = sl.dev.geo;
    const size_t n = (size_t)G.nx * G.ny;
    char* buf = nullptr;
    const size_t bytes = n * (13 * sizeof(double) + 2 * sizeof(int)) + (2 * (size_t)G.ny + 2) * sizeof(double);
    cudaError_t e = cudaMalloc(&buf, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(HOSONO_ENOMEM, "no device memory for the diagnostics: %s", cudaGetErrorString(e));
    }
    double* f = (double*)buf;
    double* rows = f + 13 * n;
    double* res = rows + 2 * G.ny;
    int* si = (int*)(res + 2);
    int* oi = si + n;
    launch_diagnostics(G, sl.dev.V, sl.dev.scheme[st.schemeSel], f, si, oi, rows, res, s_);
    launches += 3;
    double r[2] = {0, 0};
    int rc = HOSONO_OK;
    if (cudaGetLastError() != cudaSuccess) rc = fail(HOSONO_ECUDA, "diagnostics launch failed");
    if (!rc && fields && cudaMemcpyAsync(fields, f, n * 13 * sizeof(double), cudaMemcpyDeviceToHost, s_))
        rc = fail(HOSONO_ECUDA, "diagnostics copy failed");
    if (!rc && scheme && cudaMemcpyAsync(scheme, si, n * sizeof(int), cudaMemcpyDeviceToHost, s_))
        rc = fail(HOSONO_ECUDA, "diagnostics copy failed");
    if (!rc && ordr && cudaMemcpyAsync(ordr, oi, n * sizeof(int), cudaMemcpyDeviceToHost, s_))
        rc = fail(HOSONO_ECUDA, "diagnostics copy failed");
    if (!rc && cudaMemcpyAsync(r, res, sizeof r, cudaMemcpyDeviceToHost, s_)) rc = fail(HOSONO_ECUDA, "copy failed");
    if (cudaStreamSynchronize(s_) != cudaSuccess && !rc) rc = fail(HOSONO_ECUDA, "diagnostics failed");
    cudaFree(buf);
    if (rc) return rc;
    if (divb_l1) *divb_l1 = r[0] / (double)n;
    if (divb_linf) *divb_linf = r[1];
    return HOSONO_OK;
}

int Engine::download(int slot, double* U, double* V, int* scheme) {
    if (slot < 0 || slot >= maxInst_ || !slots_[slot].live) return fail(HOSONO_EINVAL, "bad download");
    InstState st;
    TRYE(state(slot, &st));
    const Slot& sl = slots_[slot];
    const Geo& G = sl.dev.geo;
    const size_t cells = (size_t)G.nxt * G.nyt;
    if (U) {
        launch_soa_to_aos(G, sl.dev.U[st.parity], staging_, NCONS, s_);
        launches++;
        CUE(cudaMemcpyAsync(U, staging_, cells * NCONS * sizeof(double), cudaMemcpyDeviceToHost, s_));
        CUE(cudaStreamSynchronize(s_));
    }
    if (V) {
        launch_soa_to_aos(G, sl.dev.V, staging_, NPRIM, s_);
        launches++;
        CUE(cudaMemcpyAsync(V, staging_, cells * NPRIM * sizeof(double), cudaMemcpyDeviceToHost, s_));
        CUE(cudaStreamSynchronize(s_));
    }
    if (scheme) {
        launch_scheme_to_int(G, sl.dev.scheme[st.schemeSel], schemeInt_, s_);
        launches++;
        CUE(cudaMemcpyAsync(scheme, schemeInt_, cells * sizeof(int), cudaMemcpyDeviceToHost, s_));
        CUE(cudaStreamSynchronize(s_));
    }
    CUE(cudaGetLastError());
    return HOSONO_OK;
}

int Engine::set_time(int slot, double t, double tmax, int nstep, int nstepmax) {
    if (slot < 0 || slot >= maxInst_ || !slots_[slot].live) return fail(HOSONO_EINVAL, "bad slot %d", slot);
    InstState st;
    TRYE(state(slot, &st));
    st.t = t;
    st.tmax = tmax;
    st.nstep = nstep;
    st.nstepmax = nstepmax;
    st.done = (t < tmax && nstep < nstepmax) ? 0 : 1;
    st.error = 0;
    st.stepping = 0;
    CUE(cudaMemcpyAsync(d_st_ + slot, &st, sizeof(InstState), cudaMemcpyHostToDevice, s_));
    CUE(cudaStreamSynchronize(s_));
    return HOSONO_OK;
}

// ----------------------------------------------------------------------
// The forward-Euler stage (timeStep.f90:45-130).
int Engine::record_stage(Rec& r, int uin, int uout, cudaEvent_t ev0, cudaEvent_t ev1) {
    const Batch B = batch();
    const KernelSet* K = K_;
    const long long cap = (long long)INT_MAX;
    TRYE(r.k([&](cudaStream_t s) { K->stage_init(B, s); }));
    if (ev0) TRYE(r.event(ev0));
    TRYE(r.k([&](cudaStream_t s) { K->face_pass1(B, uin, s); }));
    if (ev1) TRYE(r.event(ev1));
    cudaGraphConditionalHandle hc1, hm;
    TRYE(r.cond(&hc1, 0));
    TRYE(r.k([&](cudaStream_t s) { K->cascade_cond(B, hc1, s); }));
    auto cascade_body = [&](cudaGraphConditionalHandle hc, int later) {
        return [&, hc, later](Rec& c) -> int {
            TRYE(c.k([&](cudaStream_t s) { K->cascade_lower(B, later, s); }));
            TRYE(c.k([&](cudaStream_t s) { K->recon_check(B, uin, later, s); }));
            if (!c.graph()) launches += 2;  // both launch two kernels
            TRYE(c.k([&](cudaStream_t s) { K->cascade_cond(B, hc, s); }));
            return HOSONO_OK;
        };
    };
    TRYE(r.loop(hc1, &BatchFlags::anyFail, cap, cascade_body(hc1, 0)));
    TRYE(r.k([&](cudaStream_t s) { K->compact_dirty(B, s); }));
    TRYE(r.k([&](cudaStream_t s) { K->flux_list(B, uin, s); }));
    TRYE(r.k([&](cudaStream_t s) { K->ct_update_detect(B, uin, uout, s); }));
    TRYE(r.k([&](cudaStream_t s) { K->mood_flags(B, MOOD_FLAGS_DENSE, s); }));
    if (trace) TRYE(r.host([&] { return trace_snapshot(); }));
    TRYE(r.k([&](cudaStream_t s) { K->clear_low(B, s); }));
    TRYE(r.cond(&hm, 0));
    TRYE(r.k([&](cudaStream_t s) { K->pass_end(B, hm, 1, s); }));
    if (trace) TRYE(r.host([&] { return trace_after_pass(); }));
    // later MOOD passes touch the flagged cells only: each step builds a work
    // list (warp ballot + one atomic per warp) and a list kernel consumes it
    TRYE(r.loop(hm, &BatchFlags::anyActive, cap, [&](Rec& b) -> int {
        if (trace) TRYE(b.host([&] { return trace_before_pass(); }));
        TRYE(b.k([&](cudaStream_t s) { K->recon_list(B, uin, s); }));
        cudaGraphConditionalHandle hc2;
        TRYE(b.cond(&hc2, 0));
        TRYE(b.k([&](cudaStream_t s) { K->cascade_cond(B, hc2, s); }));
        TRYE(b.loop(hc2, &BatchFlags::anyFail, cap, cascade_body(hc2, 1)));
        TRYE(b.k([&](cudaStream_t s) { K->compact_post(B, s); }));
        TRYE(b.k([&](cudaStream_t s) { K->flux_list(B, uin, s); }));
        TRYE(b.k([&](cudaStream_t s) { K->ct_list(B, uin, uout, s); }));
        if (trace) {  // the trace reads `lowered` before it is cleared
            TRYE(b.k([&](cudaStream_t s) { K->mood_flags(B, MOOD_FLAGS_LISTS, s); }));
            TRYE(b.host([&] { return trace_snapshot(); }));
            TRYE(b.k([&](cudaStream_t s) { K->clear_low(B, s); }));
        } else {
            TRYE(b.k([&](cudaStream_t s) { K->mood_flags(B, MOOD_FLAGS_LISTS_CLEAR, s); }));
        }
        if (!b.graph()) launches += 2;  // three kernels
        TRYE(b.k([&](cudaStream_t s) { K->pass_end(B, hm, 0, s); }));
        if (trace) TRYE(b.host([&] { return trace_after_pass(); }));
        return HOSONO_OK;
    }));
    return HOSONO_OK;
}

// One time step (timeStep_RK3 + advanceSolution; with the driver's cfl and
// validTimeStep unless the host supplies dt).  With profile, CUDA events
// bracket the pass-1 kernel of each stage.
int Engine::record_step(Rec& r, bool host_dt, cudaGraphConditionalHandle run_cond, bool profile) {
    const Batch B = batch();
    const KernelSet* K = K_;
    if (!host_dt) {
        TRYE(r.k([&](cudaStream_t s) { K->step_prepare(B, 0, s); }));
        TRYE(r.k([&](cudaStream_t s) { K->cfl_reduce(B, s); }));
        TRYE(r.k([&](cudaStream_t s) { K->step_begin(B, 0, s); }));
    }
    // U1 = FE(U), BC; U2 = FE(U1); U2 = (3U+U2)/4, BC; U3 = FE(U2); Unew = (U+2U3)/3
    const int uin[3] = {ROLE_STATE, ROLE_A, ROLE_A};
    const int uout[3] = {ROLE_A, ROLE_B, ROLE_B};
    for (int st = 0; st < 3; st++) {
        TRYE(record_stage(r, uin[st], uout[st], profile ? profEv_[2 * st] : nullptr,
                          profile ? profEv_[2 * st + 1] : nullptr));
        if (st == 0) TRYE(r.k([&](cudaStream_t s) { K->bc_fill(B, ROLE_A, s); }));
        if (st == 1) TRYE(r.k([&](cudaStream_t s) { K->rk_combine2(B, s); }));
        if (st == 2) TRYE(r.k([&](cudaStream_t s) { K->rk_final(B, s); }));
    }
    TRYE(r.k([&](cudaStream_t s) { K->step_end(B, run_cond, s); }));
    return HOSONO_OK;
}

int Engine::build_graphs() {
    if (gAdvance_) return HOSONO_OK;
    for (int which = 0; which < 3; which++) {
        cudaGraph_t g;
        CUE(cudaGraphCreate(&g, 0));
        Rec r(this, g);
        int rc;
        if (which == 0) {
            rc = record_step(r, true, 0, false);
        } else if (which == 2) {
            // one step at the graph's top level: event records are not allowed
            // inside conditional bodies, and pass 1 sits outside the MOOD loops
            rc = record_step(r, false, 0, true);
        } else {
            cudaGraphConditionalHandle hr;
            rc = r.cond(&hr, 1);
            if (!rc)
                rc = r.loop(hr, &BatchFlags::anyLive, INT_MAX,
                            [&](Rec& b) -> int { return record_step(b, false, hr, which == 2); });
        }
        if (!rc) rc = r.end();
        if (rc) {
            cudaGraphDestroy(g);
            return rc;
        }
        cudaGraphExec_t ex;
        cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail(HOSONO_ECUDA, "graph instantiate: %s", cudaGetErrorString(e));
        (which == 0 ? gAdvance_ : which == 1 ? gRun_ : gProf_) = ex;
    }
    return HOSONO_OK;
}

int Engine::launch(cudaGraphExec_t g) {
    CUE(cudaGraphLaunch(g, s_));
    CUE(cudaStreamSynchronize(s_));
    return HOSONO_OK;
}

int Engine::check_errors() {
    CUE(cudaMemcpyAsync(h_st_, d_st_, sizeof(InstState) * maxInst_, cudaMemcpyDeviceToHost, s_));
    CUE(cudaMemcpyAsync(h_flags_, d_flags_, sizeof(BatchFlags), cudaMemcpyDeviceToHost, s_));
    CUE(cudaStreamSynchronize(s_));
    if (h_flags_->error) return fail(h_flags_->error, "a MOOD work list overflowed its capacity");
    if (!instance_errors_fatal) return HOSONO_OK;
    for (int k = 0; k < maxInst_; k++)
        if (slots_[k].live && h_st_[k].error)
            return fail(h_st_[k].error, "instance %d stopped: %s", k,
                        h_st_[k].error == HOSONO_ENANDT ? "dt is NaN, infinite or negative" : "MOOD pass cap reached");
    return HOSONO_OK;
}

int Engine::cfl(int slot, double* dt) {
    if (slot < 0 || slot >= maxInst_ || !slots_[slot].live) return fail(HOSONO_EINVAL, "bad slot %d", slot);
    InstState st;
    TRYE(state(slot, &st));
    st.stepping = 1;
    st.cflbits[0] = st.cflbits[1] = 0;
    CUE(cudaMemcpyAsync(d_st_ + slot, &st, sizeof(InstState), cudaMemcpyHostToDevice, s_));
    K_->cfl_reduce(batch(), s_);
    launches++;
    CUE(cudaGetLastError());
    TRYE(state(slot, &st));
    const unsigned long long bits[2] = {st.cflbits[0], st.cflbits[1]};
    TRYE(write_field(slot, &InstState::stepping, 0));
    double xm, ym;
    std::memcpy(&xm, &bits[0], sizeof xm);
    std::memcpy(&ym, &bits[1], sizeof ym);
    const Slot& sl = slots_[slot];
    *dt = sl.p.cfl * std::fmin(sl.dev.geo.dx / xm, sl.dev.geo.dy / ym);  // cfl.f90:50
    return HOSONO_OK;
}

int Engine::advance(int slot, double dt) {
    if (slot < 0 || slot >= maxInst_ || !slots_[slot].live) return fail(HOSONO_EINVAL, "bad slot %d", slot);
    if (!(dt >= 0.0) || !std::isfinite(dt)) return fail(HOSONO_ENANDT, "dt = %g is not a valid time step", dt);
    InstState st;
    TRYE(state(slot, &st));
    st.dt = dt;
    st.stepping = 1;
    st.error = 0;
    CUE(cudaMemcpyAsync(d_st_ + slot, &st, sizeof(InstState), cudaMemcpyHostToDevice, s_));
    if (use_graphs && !trace) {
        TRYE(build_graphs());
        TRYE(launch(gAdvance_));
    } else {
        Rec r(this, nullptr);
        TRYE(record_step(r, true, 0, false));
        CUE(cudaStreamSynchronize(s_));
    }
    return check_errors();
}

int Engine::run(int max_steps) {
    BatchFlags f{};
    f.anyLive = 1;
    f.radii = radii_;
    f.stepsLeft = max_steps > 0 ? max_steps : INT_MAX;
    CUE(cudaMemcpyAsync(d_flags_, &f, sizeof f, cudaMemcpyHostToDevice, s_));
    if (use_graphs && !trace) {
        TRYE(build_graphs());
        TRYE(launch(gRun_));
    } else {
        Rec r(this, nullptr);
        CUE(cudaStreamSynchronize(s_));
        *h_flags_ = f;
        long long it = 0;
        while (h_flags_->anyLive) {
            if (++it > (long long)INT_MAX) break;
            TRYE(record_step(r, false, 0, false));
            TRYE(sync());
        }
    }
    return check_errors();
}

int Engine::run_profiled_step(double* pass1_ms, int* pass1_launches) {
    BatchFlags f{};
    f.anyLive = 1;
    f.radii = radii_;
    f.stepsLeft = 1;
    CUE(cudaMemcpyAsync(d_flags_, &f, sizeof f, cudaMemcpyHostToDevice, s_));
    TRYE(build_graphs());
    TRYE(launch(gProf_));
    double ms = 0;
    for (int st = 0; st < 3; st++) {
        float t = 0.f;
        CUE(cudaEventElapsedTime(&t, profEv_[2 * st], profEv_[2 * st + 1]));
        ms += t;
    }
    *pass1_ms = ms;
    *pass1_launches = 3;
    return check_errors();
}

// ----------------------------------------------------------------------
// MOOD trace (eager execution only): per pass and instance, the per-cell
// lowering counts of the face cascade and of detect.
int Engine::trace_before_pass() {
    for (int k = 0; k < maxInst_; k++)
        if (slots_[k].live)
            CUE(cudaMemsetAsync(slots_[k].dev.innerCount, 0, (size_t)slots_[k].dev.geo.plane, s_));
    return HOSONO_OK;
}

int Engine::trace_snapshot() {
    snapInner_.assign(maxInst_, {});
    snapLow_.assign(maxInst_, {});
    for (int k = 0; k < maxInst_; k++) {
        if (!slots_[k].live) continue;
        const Geo& G = slots_[k].dev.geo;
        snapInner_[k].resize((size_t)G.plane);
        snapLow_[k].resize((size_t)G.plane);
        CUE(cudaMemcpyAsync(snapInner_[k].data(), slots_[k].dev.innerCount, (size_t)G.plane, cudaMemcpyDeviceToHost,
                            s_));
        CUE(cudaMemcpyAsync(snapLow_[k].data(), slots_[k].dev.lowered, (size_t)G.plane, cudaMemcpyDeviceToHost, s_));
    }
    CUE(cudaStreamSynchronize(s_));
    return HOSONO_OK;
}

int Engine::trace_after_pass() {
    CUE(cudaMemcpyAsync(h_st_, d_st_, sizeof(InstState) * maxInst_, cudaMemcpyDeviceToHost, s_));
    CUE(cudaStreamSynchronize(s_));
    for (int k = 0; k < maxInst_; k++) {
        if (!slots_[k].live) continue;
        const InstState& S = h_st_[k];
        if (S.passesTotal == tracePassesSeen_[k]) continue;
        tracePassesSeen_[k] = S.passesTotal;
        const Geo& G = slots_[k].dev.geo;
        TraceRec t;
        t.slot = k;
        t.stage = S.stages - 1 - traceStageBase[k];
        t.pass = S.passes - 1;
        t.nInner = S.lastInner;
        t.nDetect = S.lastDetect;
        const std::vector<unsigned char>& a = snapInner_[k];
        const std::vector<unsigned char>& b = snapLow_[k];
        t.inner.resize((size_t)G.nxt * G.nyt);
        t.detect.resize((size_t)G.nxt * G.nyt);
        for (int j = 0; j < G.nyt; j++)
            for (int i = 0; i < G.nxt; i++) {
                t.inner[(size_t)j * G.nxt + i] = a[(size_t)j * G.pitch + i];
                t.detect[(size_t)j * G.nxt + i] = b[(size_t)j * G.pitch + i];
            }
        traces.push_back(std::move(t));
    }
    return HOSONO_OK;
}

}  // namespace hosono
