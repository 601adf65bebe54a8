// engine.cu -- host side of the batched engine: instance slots, device
// tables, and the time-step structure (timeStep.f90:22-171 with the driver
// loop of mhd_driver.f90:76-95) recorded either as eager launches driven by
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
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
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

namespace {
thread_local bool tl_pdl_next = false, tl_pdl_chain = false;
}  // namespace
void pdl_arm(bool first, bool chain) {
    tl_pdl_next = first;
    tl_pdl_chain = chain;
}
bool pdl_take() {
    const bool r = tl_pdl_next;
    tl_pdl_next = tl_pdl_chain;
    return r;
}

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
            afterKernel_ = false;  // the segment's first launch depends on nodes of an earlier segment
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
    // a kernel launch (or a few in a row): programmatic when the tuning asks
    // for it and the previous operation recorded was a kernel launch too
    template <class F>
    int k(F&& f) {
        TRYE(begin());
        const bool pdl = e_->tune_.pdl != 0;
        pdl_arm(pdl && afterKernel_, pdl);
        f(e_->s_);
        pdl_arm(false, false);
        afterKernel_ = true;
        if (!g_) e_->launches++;
        cudaError_t r = cudaGetLastError();
        if (r != cudaSuccess) return e_->fail(HOSONO_ECUDA, "kernel launch: %s", cudaGetErrorString(r));
        return HOSONO_OK;
    }
    int event(cudaEvent_t ev) {
        TRYE(begin());
        afterKernel_ = false;
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
            afterKernel_ = false;
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
        afterKernel_ = false;
        return HOSONO_OK;
    }
    template <class H>
    int host(H&& h) {
        if (g_) return HOSONO_OK;
        TRYE(e_->sync());
        afterKernel_ = false;  // h may queue copies
        return h();
    }

  private:
    Engine* e_;
    cudaGraph_t g_;
    std::vector<cudaGraphNode_t> deps_;
    bool open_ = false;
    bool afterKernel_ = false;  // the last operation recorded was a kernel launch
};

// ----------------------------------------------------------------------
Engine::~Engine() {
    if (s_) cudaStreamSynchronize(s_);
    for (auto& sl : slots_) {
        for (void* p : sl.allocs) dfree(p);
        if (sl.modAlloc) cudaFree(sl.modAlloc);
    }
    if (sCopy_) cudaStreamSynchronize(sCopy_);
    for (cudaGraphExec_t g : {gAdvance_, gRun_, gProf_, gAdvRest_})
        if (g) cudaGraphExecDestroy(g);
    for (cudaEvent_t ev : profEv_)
        if (ev) cudaEventDestroy(ev);
    for (cudaEvent_t ev : bandEv_)
        if (ev) cudaEventDestroy(ev);
    if (sCopy_) cudaStreamDestroy(sCopy_);
    for (void* p : {(void*)d_instTiles_, (void*)d_actRange_, (void*)d_actInfo_, (void*)d_casRange_,
                    (void*)d_casInfo_, (void*)d_hold_, (void*)d_gbar_})
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
    CUE(cudaMalloc(&d_hold_, sizeof(int) * maxInst_));
    CUE(cudaMemsetAsync(d_hold_, 0, sizeof(int) * maxInst_, s_));
    CUE(cudaMalloc(&d_gbar_, sizeof(unsigned) * 2));
    CUE(cudaMemsetAsync(d_gbar_, 0, sizeof(unsigned) * 2, s_));
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

namespace {
// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library links no libcuda of its own)
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
    static const EncodeTiledFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return (EncodeTiledFn) nullptr;
        }
        return (EncodeTiledFn)p;
    }();
    return fn;
}
}  // namespace

// TMA descriptors of the three U buffers: a 3D tensor (x: pitch doubles,
// y: nyt rows, var: 8 planes) read in boxes of the pass-1 stencil box
int Engine::encode_tmaps(InstDev& dev) {
    const EncodeTiledFn enc = encode_tiled();
    if (!enc) return fail(HOSONO_ECUDA, "cuTensorMapEncodeTiled is not available from the driver");
    const Geo& G = dev.geo;
    const cuuint64_t dims[3] = {(cuuint64_t)G.pitch, (cuuint64_t)G.nyt, (cuuint64_t)NCONS};
    const cuuint64_t strides[2] = {(cuuint64_t)G.pitch * sizeof(double), (cuuint64_t)G.plane * sizeof(double)};
    const cuuint32_t box[3] = {(cuuint32_t)P1_SX, (cuuint32_t)p1_sy(G.R), (cuuint32_t)NCONS};
    const cuuint32_t es[3] = {1, 1, 1};
    const cuuint32_t boxU[3] = {(cuuint32_t)CT_SX, (cuuint32_t)CT_UY, (cuuint32_t)NCONS};
    const cuuint32_t boxF[3] = {(cuuint32_t)CT_SX, (cuuint32_t)CT_FY, (cuuint32_t)NCONS};
    auto one = [&](CUtensorMap* m, double* base, const cuuint32_t* b) {
        return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, base, dims, strides, b, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    };
    for (int r = 0; r < 3; r++) {
        CUresult e = one(&dev.tmU[r], dev.U[r], box);
        if (e == CUDA_SUCCESS) e = one(&dev.tmCU[r], dev.U[r], boxU);
        if (e != CUDA_SUCCESS) return fail(HOSONO_ECUDA, "cuTensorMapEncodeTiled failed (%d)", (int)e);
    }
    CUresult e = one(&dev.tmFX, dev.FX, boxF);
    if (e == CUDA_SUCCESS) e = one(&dev.tmFY, dev.FY, boxF);
    if (e != CUDA_SUCCESS) return fail(HOSONO_ECUDA, "cuTensorMapEncodeTiled failed (%d)", (int)e);
    return HOSONO_OK;
}

void Engine::drop_graphs() {
    if (s_) cudaStreamSynchronize(s_);
    for (cudaGraphExec_t* g : {&gAdvance_, &gRun_, &gProf_, &gAdvRest_})
        if (*g) {
            cudaGraphExecDestroy(*g);
            *g = nullptr;
        }
}

int Engine::set_tuning(const hosono_tuning& t) {
    if (t.pass1_staging != HOSONO_STAGE_CP_ASYNC && t.pass1_staging != HOSONO_STAGE_TMA)
        return fail(HOSONO_EINVAL, "pass1_staging %d", t.pass1_staging);
    if (t.pass1_schedule != HOSONO_SCHED_STATIC && t.pass1_schedule != HOSONO_SCHED_DYNAMIC)
        return fail(HOSONO_EINVAL, "pass1_schedule %d", t.pass1_schedule);
    if (t.pass1_blocks_per_sm != 0 && (t.pass1_blocks_per_sm < 2 || t.pass1_blocks_per_sm > 4))
        return fail(HOSONO_EINVAL, "pass1_blocks_per_sm %d (0 or 2..4)", t.pass1_blocks_per_sm);
    if (t.pass1_blocks_per_sm > 2 && t.pass1_staging == HOSONO_STAGE_TMA)
        return fail(HOSONO_EINVAL, "TMA staging runs at two pass-1 blocks per SM");
    if (t.later_passes != HOSONO_LATER_KERNELS && t.later_passes != HOSONO_LATER_PERSISTENT)
        return fail(HOSONO_EINVAL, "later_passes %d", t.later_passes);
    if (t.pass1_boxes < 0 || t.pass1_boxes > 2)
        return fail(HOSONO_EINVAL, "pass1_boxes %d (0, 1 or 2)", t.pass1_boxes);
    if (t.pass1_boxes == 2 && t.pass1_blocks_per_sm > 2)
        return fail(HOSONO_EINVAL, "two stencil boxes run at two pass-1 blocks per SM");
    if (t.pdl != 0 && t.pdl != 1) return fail(HOSONO_EINVAL, "pdl %d (0 or 1)", t.pdl);
    if (t.update_staging != HOSONO_STAGE_CP_ASYNC && t.update_staging != HOSONO_STAGE_TMA)
        return fail(HOSONO_EINVAL, "update_staging %d", t.update_staging);
    if (t.upload_bands < 0 || t.upload_bands > HOSONO_UPLOAD_BANDS_MAX)
        return fail(HOSONO_EINVAL, "upload_bands %d (0..%d)", t.upload_bands, HOSONO_UPLOAD_BANDS_MAX);
    tune_ = t;
    drop_graphs();  // the graphs hold the launch choices in their kernel parameters
    return HOSONO_OK;
}

namespace {
// the autotuner's process-wide cache: (fp mode, radii, size class, instance class) -> tuning
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int>, hosono_tuning> g_tune_cache;
}  // namespace

int Engine::autotune(int trials, bool force, hosono_tune_report* rep) {
    if (trials < 1 || trials > 1000) return fail(HOSONO_EINVAL, "autotune: trials %d outside [1, 1000]", trials);
    hosono_tune_report r{};
    long long cells = 0;
    int inst = 0;
    for (const Slot& sl : slots_)
        if (sl.live) {
            cells += (long long)sl.p.nx * sl.p.ny;
            inst++;
        }
    if (!inst) return fail(HOSONO_EINVAL, "autotune: no instance to time");
    int sc = 0, ic = 0;
    while ((2LL << sc) <= cells) sc++;
    while ((2 << ic) <= inst) ic++;
    r.size_class = sc;
    r.instances = inst;
    const auto key = std::make_tuple(K_ == kernelset_fast() ? 1 : 0, radii_, sc, ic);
    if (!force) {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            r.cached = 1;
            r.best = it->second;
            r.best.later_passes = tune_.later_passes;  // the caller's choices stay
            r.best.upload_bands = tune_.upload_bands;
            r.best.pdl = tune_.pdl;
            r.best.update_staging = tune_.update_staging;
            if (rep) *rep = r;
            return set_tuning(r.best);
        }
    }
    CUE(cudaStreamSynchronize(s_));
    const hosono_tuning saved = tune_;
    // candidates: two blocks per SM with cp.async or TMA staging and one or
    // two stencil boxes, three and four blocks per SM with cp.async and one
    // box; each with the static and the dynamic tile schedule
    std::vector<hosono_tuning> cands;
    const int forms[6][3] = {{2, HOSONO_STAGE_CP_ASYNC, 1}, {2, HOSONO_STAGE_TMA, 1}, {2, HOSONO_STAGE_CP_ASYNC, 2},
                             {2, HOSONO_STAGE_TMA, 2},      {3, HOSONO_STAGE_CP_ASYNC, 1}, {4, HOSONO_STAGE_CP_ASYNC, 1}};
    for (const auto& f : forms)
        for (int sched : {HOSONO_SCHED_STATIC, HOSONO_SCHED_DYNAMIC}) {
            hosono_tuning t = tune_;  // the caller's later-pass choice stays
            t.pass1_blocks_per_sm = f[0];
            t.pass1_staging = f[1];
            t.pass1_boxes = f[2];
            t.pass1_schedule = sched;
            cands.push_back(t);
        }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CUE(cudaEventCreate(&e0));
    CUE(cudaEventCreate(&e1));
    int rc = HOSONO_OK;
    K_->tune_mark(batch(), 1, s_);
    for (size_t c = 0; c < cands.size() && c < HOSONO_TUNE_MAX && !rc; c++) {
        {
            const hosono_tuning t = cands[c];
            tune_ = t;
            const Batch B = batch();
            float ms = 0.f;
            for (int k = 0; k <= trials; k++) {
                if (k == 1) cudaEventRecord(e0, s_);
                cudaMemsetAsync(d_flags_->p1Next, 0, sizeof d_flags_->p1Next, s_);
                K_->face_pass1(B, ROLE_STATE, s_);
            }
            cudaEventRecord(e1, s_);
            if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess ||
                cudaGetLastError() != cudaSuccess)
                rc = fail(HOSONO_ECUDA, "autotune: timing launch failed");
            r.tried[r.candidates] = t;
            r.ms[r.candidates] = ms / trials;
            r.candidates++;
        }
    }
    K_->tune_mark(batch(), 0, s_);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    tune_ = saved;
    if (rc) return rc;
    CUE(cudaStreamSynchronize(s_));
    if (h_flags_) {  // a bounded wait of the TMA variant that gave up is an error, not a result
        CUE(cudaMemcpy(h_flags_, d_flags_, sizeof(BatchFlags), cudaMemcpyDeviceToHost));
        if (h_flags_->error) return fail(h_flags_->error, "autotune: a timing launch reported an error");
    }
    int best = 0;
    for (int k = 1; k < r.candidates; k++)
        if (r.ms[k] < r.ms[best]) best = k;
    r.best = r.tried[best];
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune_cache[key] = r.best;
    }
    if (rep) *rep = r;
    return set_tuning(r.best);
}

Batch Engine::batch() const {
    Batch B;
    B.p1Tma = tune_.pass1_staging == HOSONO_STAGE_TMA ? 1 : 0;
    B.p1Dyn = tune_.pass1_schedule == HOSONO_SCHED_DYNAMIC ? 1 : 0;
    B.p1Blocks = tune_.pass1_blocks_per_sm == 0 ? 2 : tune_.pass1_blocks_per_sm;
    B.p1Boxes = tune_.pass1_boxes == 2 ? 2 : 1;
    B.p1Radii = radii_;
    B.p1First = 0;
    B.p1End = INT_MAX;
    B.ctStaged = tune_.update_staging == HOSONO_STAGE_TMA ? 1 : 0;
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
    B.hold = d_hold_;
    B.gbar = d_gbar_;
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
    // the graphs launch pass 1 for the radii held when they were recorded:
    // a new radius needs new graphs
    if (radii_ & ~graphRadii_) drop_graphs();
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
    sl.dev.phys.small_b = p.small_b;
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
    if (int rc = encode_tmaps(sl.dev)) {
        for (void* a : sl.allocs) dfree(a);
        return rc;
    }
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
    st.passCap = HOSONO_MOOD_CAP_DEFAULT(R, p.nx, p.ny);
    CUE(cudaMemcpyAsync(d_st_ + k, &st, sizeof(InstState), cudaMemcpyHostToDevice, s_));
    CUE(cudaMemsetAsync(d_hold_ + k, 0, sizeof(int), s_));
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
    if (slots_[slot].modAlloc) cudaFree(slots_[slot].modAlloc);
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

int Engine::upload_u(int slot, const double* U) {
    if (slot < 0 || slot >= maxInst_ || !slots_[slot].live || !U) return fail(HOSONO_EINVAL, "bad upload");
    InstState st;
    TRYE(state(slot, &st));
    const Slot& sl = slots_[slot];
    const Geo& G = sl.dev.geo;
    CUE(cudaMemcpyAsync(staging_, U, (size_t)G.nxt * G.nyt * NCONS * sizeof(double), cudaMemcpyHostToDevice, s_));
    launch_aos_to_soa(G, staging_, sl.dev.U[st.parity], NCONS, s_);
    launches++;
    CUE(cudaGetLastError());
    return HOSONO_OK;
}

// timeStep_advanceSolution on host arrays (mhd_driver.f90:117-144 with
// grid_state on the host).  Banded form: the band copies go up on sCopy_
// one after another (one DMA stream); the main stream sets up the first
// stage (scheme = R, flags: timeStep.f90:77-81), then per band waits for its
// rows, converts them and runs pass 1 on the band's tile rows -- whose
// stencil boxes reach R + 1 rows past the band, so a band's copy ends that
// far beyond its last tile row -- and finally the step graph without the
// first stage's set-up and pass 1.  Tiles are independent in pass 1, so the
// result bits do not depend on the banding.
int Engine::advance_host(int slot, double dt, double* U, double* V) {
    if (slot < 0 || slot >= maxInst_ || !slots_[slot].live || !U) return fail(HOSONO_EINVAL, "bad advance_host");
    if (!(dt >= 0.0) || !std::isfinite(dt)) return fail(HOSONO_ENANDT, "dt = %g is not a valid time step", dt);
    const Slot& sl = slots_[slot];
    const Geo& G = sl.dev.geo;
    // by size: 16 bands from 2048 array rows, 8 from 1024 (measured on
    // Orszag-Tang 2048^2: 17.44 ms per step with 8, 17.32 with 16)
    int nb = tune_.upload_bands ? tune_.upload_bands : (G.nyt >= 2048 ? 16 : G.nyt >= 1024 ? 8 : 1);
    const int tileRows = (G.nyt + TILE_Y - 1) / TILE_Y, tilesPerRow = (G.nxt + TILE_X - 1) / TILE_X;
    if (nb > tileRows) nb = tileRows;
    // one instance per engine, step graphs in use: otherwise upload, then step
    int liveCount = 0;
    for (const Slot& x : slots_) liveCount += x.live ? 1 : 0;
    // a step that stops with an error leaves U as uploaded: V is rebuilt from
    // it, so the device state stays consistent for the caller's next cfl
    auto restore_v = [&](int rc) -> int {
        const std::string m = msg;
        if (write_field(slot, &InstState::stepping, 1) == HOSONO_OK) {
            K_->cons2prim_all(batch(), s_);
            launches++;
            write_field(slot, &InstState::stepping, 0);
        }
        err = rc;
        msg = m;
        return rc;
    };
    if (nb <= 1 || liveCount != 1 || !use_graphs || trace) {
        TRYE(upload_u(slot, U));
        if (int rc = advance(slot, dt)) return restore_v(rc);
        return download(slot, U, V, nullptr);
    }
    if (!sCopy_) {
        CUE(cudaStreamCreateWithFlags(&sCopy_, cudaStreamNonBlocking));
        for (cudaEvent_t& ev : bandEv_) CUE(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    }
    InstState st;
    TRYE(state(slot, &st));
    st.dt = dt;
    st.stepping = 1;
    st.error = 0;
    CUE(cudaMemcpyAsync(d_st_ + slot, &st, sizeof(InstState), cudaMemcpyHostToDevice, s_));
    TRYE(build_graphs());
    // the copies start once everything before on the main stream is done with the staging buffer
    CUE(cudaEventRecord(bandEv_[HOSONO_UPLOAD_BANDS_MAX], s_));
    CUE(cudaStreamWaitEvent(sCopy_, bandEv_[HOSONO_UPLOAD_BANDS_MAX], 0));
    const size_t rowBytes = (size_t)G.nxt * NCONS * sizeof(double), rowDoubles = (size_t)G.nxt * NCONS;
    const Batch B = batch();
    K_->stage_init(B, s_);
    launches++;
    const int base = instTiles_[slot].x;
    // band by band: the copy on sCopy_, then on the main stream the wait,
    // the conversion and pass 1 on the band's tile rows.  Interleaved, so
    // that with a pageable host U (whose copies return only once the data
    // has left it) a band's pass 1 is queued before the next band's copy.
    for (int b = 0, r0 = 0, tr0 = 0; b < nb; b++) {
        const int tr1 = (int)((long long)tileRows * (b + 1) / nb);
        const int want = b == nb - 1 ? G.nyt : tr1 * TILE_Y + G.R + 1;  // last row the band's boxes read + 1
        const int r1 = want < G.nyt ? (want > r0 ? want : r0) : G.nyt;
        if (r1 > r0)
            CUE(cudaMemcpyAsync(staging_ + (size_t)r0 * rowDoubles, U + (size_t)r0 * rowDoubles,
                                (size_t)(r1 - r0) * rowBytes, cudaMemcpyHostToDevice, sCopy_));
        CUE(cudaEventRecord(bandEv_[b], sCopy_));
        CUE(cudaStreamWaitEvent(s_, bandEv_[b], 0));
        launch_aos_to_soa_rows(G, staging_, sl.dev.U[st.parity], NCONS, r0, r1, s_);
        if (b > 0) CUE(cudaMemsetAsync(d_flags_->p1Next, 0, sizeof d_flags_->p1Next, s_));
        Batch Bb = B;
        Bb.p1First = base + tr0 * tilesPerRow;
        Bb.p1End = base + tr1 * tilesPerRow;
        K_->face_pass1(Bb, ROLE_STATE, s_);
        launches += 1 + radii_held();
        r0 = r1;
        tr0 = tr1;
    }
    CUE(cudaGetLastError());
    CUE(cudaGraphLaunch(gAdvRest_, s_));
    if (int rc = check_errors()) return restore_v(rc);
    return download(slot, U, V, nullptr);
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

int Engine::set_holds(const int* holds) {
    CUE(cudaMemcpyAsync(d_hold_, holds, sizeof(int) * maxInst_, cudaMemcpyHostToDevice, s_));
    CUE(cudaStreamSynchronize(s_));
    return HOSONO_OK;
}

int Engine::set_mood_cap(int slot, int cap) {
    if (slot < 0 || slot >= maxInst_ || !slots_[slot].live) return fail(HOSONO_EINVAL, "bad slot %d", slot);
    const hosono_params& p = slots_[slot].p;
    // every pass that does not end the loop lowers at least one cell by one
    // order, and a cell can be lowered at most R times: R*nx*ny + 1 passes
    // always suffice (guard cells only follow their interior images)
    const long long proven = (long long)p.max_radius * p.nx * p.ny + 1;
    const long long c = cap > 0 ? std::min<long long>(cap, proven) : proven;
    return write_field(slot, &InstState::passCap, (int)std::min<long long>(c, INT_MAX));
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
int Engine::record_stage(Rec& r, int uin, int uout, cudaEvent_t ev0, cudaEvent_t ev1, bool head) {
    const Batch B = batch();
    const KernelSet* K = K_;
    const long long cap = (long long)INT_MAX;
    if (head) {
        TRYE(r.k([&](cudaStream_t s) { K->stage_init(B, s); }));
        if (ev0) TRYE(r.event(ev0));
        TRYE(r.k([&](cudaStream_t s) { K->face_pass1(B, uin, s); }));
        if (!r.graph()) launches += radii_held() - 1;  // one pass-1 kernel per radius held
        if (ev1) TRYE(r.event(ev1));
    }
    cudaGraphConditionalHandle hc1, hm;
    TRYE(r.cond(&hc1, 0));
    TRYE(r.k([&](cudaStream_t s) { K->cascade_cond(B, hc1, s); }));
    auto cascade_body = [&](cudaGraphConditionalHandle hc, int later) {
        return [&, hc, later](Rec& c) -> int {
            TRYE(c.k([&](cudaStream_t s) { K->cascade_lower(B, later, s); }));
            TRYE(c.k([&](cudaStream_t s) { K->recon_check(B, uin, later, s); }));
            if (!c.graph()) launches += 1;  // recon_check launches two kernels
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
    if (tune_.later_passes == HOSONO_LATER_PERSISTENT && !trace) {
        // the later passes as one persistent launch (it reads anyActive itself)
        TRYE(r.k([&](cudaStream_t s) { K->pass_end(B, 0, 1, s); }));
        TRYE(r.k([&](cudaStream_t s) { K->mood_rest(B, uin, uout, s); }));
        return HOSONO_OK;
    }
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
int Engine::record_step(Rec& r, bool host_dt, cudaGraphConditionalHandle run_cond, bool profile,
                        bool first_head) {
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
                          profile ? profEv_[2 * st + 1] : nullptr, st > 0 || first_head));
        if (st == 0) TRYE(r.k([&](cudaStream_t s) { K->bc_fill(B, ROLE_A, s); }));
        if (st == 1) TRYE(r.k([&](cudaStream_t s) { K->rk_combine2(B, s); }));
        if (st == 2) TRYE(r.k([&](cudaStream_t s) { K->rk_final(B, s); }));
    }
    TRYE(r.k([&](cudaStream_t s) { K->step_end(B, run_cond, s); }));
    return HOSONO_OK;
}

int Engine::build_graphs() {
    if (gAdvance_) return HOSONO_OK;
    graphRadii_ = radii_;
    for (int which = 0; which < 4; which++) {
        cudaGraph_t g;
        CUE(cudaGraphCreate(&g, 0));
        Rec r(this, g);
        int rc;
        if (which == 0) {
            rc = record_step(r, true, 0, false);
        } else if (which == 3) {  // the banded upload ran the first stage's set-up and pass 1
            rc = record_step(r, true, 0, false, false);
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
        (which == 0 ? gAdvance_ : which == 1 ? gRun_ : which == 2 ? gProf_ : gAdvRest_) = ex;
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
// Per-module form: reconstruct_faceValsWithGP, getFluxes_, FLICD, the
// update, detect_ALL and the boundary routines one at a time on one
// instance (modules.cuh), for a host that keeps its own MOOD loop.
int Engine::mod_ensure(int slot) {
    if (slot < 0 || slot >= maxInst_ || !slots_[slot].live) return fail(HOSONO_EINVAL, "bad slot %d", slot);
    Slot& sl = slots_[slot];
    if (sl.modAlloc) return HOSONO_OK;
    const Geo& G = sl.dev.geo;
    const size_t plane = (size_t)G.plane;
    const size_t nfv = (size_t)NCONS * G.nqMax * 4, nfl = 2 * NCONS, nbyte = 8;
    const size_t bytes = sizeof(double) * plane * (nfv + nfl) + plane * nbyte + 256;
    char* p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(HOSONO_ENOMEM, "no device memory for the module buffers (%zu bytes): %s", bytes,
                    cudaGetErrorString(e));
    }
    CUE(cudaMemsetAsync(p, 0, bytes, s_));  // faceVals and flux start at zero (gridBlock.f90:160-169)
    ModBuf& M = sl.mod;
    M.fv = (double*)p;
    M.flux = M.fv + plane * nfv;
    uint8_t* b = (uint8_t*)(M.flux + plane * nfl);
    uint8_t** planes[] = {&M.recon, &M.adm, &M.next, &M.check, &M.lower, &M.tRec, &M.tRecF, (uint8_t**)&M.tSch};
    for (uint8_t** pp : planes) {
        *pp = b;
        b += plane;
    }
    M.flag = (int*)(((uintptr_t)b + 15) & ~(uintptr_t)15);
    sl.modAlloc = p;
    CUE(cudaStreamSynchronize(s_));
    return HOSONO_OK;
}

namespace {
// Fortran (i, j) order with guards <-> a device plane (rows `pitch` elements apart)
template <typename T>
cudaError_t plane_copy_down(const Geo& G, const T* d, T* h, cudaStream_t s) {
    return cudaMemcpy2DAsync(h, sizeof(T) * G.nxt, d, sizeof(T) * G.pitch, sizeof(T) * G.nxt, G.nyt,
                             cudaMemcpyDeviceToHost, s);
}
template <typename T>
cudaError_t plane_copy_up(const Geo& G, T* d, const T* h, cudaStream_t s) {
    return cudaMemcpy2DAsync(d, sizeof(T) * G.pitch, h, sizeof(T) * G.nxt, sizeof(T) * G.nxt, G.nyt,
                             cudaMemcpyHostToDevice, s);
}
}  // namespace

int Engine::mod_set(int slot, const int* scheme, const int* rec, const int* recF) {
    TRYE(mod_ensure(slot));
    InstState st;
    TRYE(state(slot, &st));
    const InstDev& d = slots_[slot].dev;
    const Geo& G = d.geo;
    const size_t n = (size_t)G.nxt * G.nyt;
    std::vector<int8_t> sb(scheme ? n : 0);
    std::vector<uint8_t> rb(rec ? n : 0), fb(recF ? n : 0);
    for (size_t c = 0; c < n; c++) {
        if (scheme) {
            if (scheme[c] < 0 || scheme[c] > G.R) return fail(HOSONO_EINVAL, "scheme %d outside [0, R]", scheme[c]);
            sb[c] = (int8_t)scheme[c];
        }
        if (rec) rb[c] = rec[c] ? 1 : 0;
        if (recF) fb[c] = recF[c] ? 1 : 0;
    }
    if (scheme) CUE(plane_copy_up(G, d.scheme[st.schemeSel], sb.data(), s_));
    if (rec) CUE(plane_copy_up(G, d.rec, rb.data(), s_));
    if (recF) CUE(plane_copy_up(G, d.recF, fb.data(), s_));
    CUE(cudaStreamSynchronize(s_));
    return HOSONO_OK;
}

int Engine::mod_get(int slot, double* faceVals, double* fluxRaw, double* flux, double* Unew, int* scheme, int* rec,
                    int* recF) {
    TRYE(mod_ensure(slot));
    InstState st;
    TRYE(state(slot, &st));
    const InstDev& d = slots_[slot].dev;
    const ModBuf& M = slots_[slot].mod;
    const Geo& G = d.geo;
    const size_t n = (size_t)G.nxt * G.nyt;
    std::vector<double> tmp(n);
    // one device plane into every k-th double of a host array starting at `first`
    auto scatter = [&](const double* dplane, double* host, size_t first, size_t k) -> int {
        CUE(plane_copy_down(G, dplane, tmp.data(), s_));
        CUE(cudaStreamSynchronize(s_));
        for (size_t c = 0; c < n; c++) host[first + k * c] = tmp[c];
        return HOSONO_OK;
    };
    if (faceVals) {  // (8, nqMax, 4, nxt, nyt)
        const size_t per = (size_t)NCONS * G.nqMax * 4;
        for (int f = 0; f < 4; f++)
            for (int q = 0; q < G.nqMax; q++)
                for (int v = 0; v < NCONS; v++)
                    TRYE(scatter(M.fv + ((size_t)(f * G.nqMax + q) * NCONS + v) * G.plane, faceVals,
                                 v + (size_t)NCONS * (q + (size_t)G.nqMax * f), per));
    }
    for (int dir = 0; dir < 2; dir++)
        for (int v = 0; v < NCONS; v++) {  // (8, 2, nxt, nyt)
            if (fluxRaw) TRYE(scatter((dir == XDIR ? d.FX : d.FY) + (size_t)v * G.plane, fluxRaw, v + NCONS * dir, 2 * NCONS));
            if (flux) TRYE(scatter(M.flux + (size_t)(dir * NCONS + v) * G.plane, flux, v + NCONS * dir, 2 * NCONS));
        }
    if (Unew) {
        const double* A = role_ptr(d, st.parity, ROLE_A);
        for (int v = 0; v < NCONS; v++) TRYE(scatter(A + (size_t)v * G.plane, Unew, v, NCONS));
    }
    std::vector<uint8_t> b(n);
    auto bytes_to_int = [&](const void* dplane, int* out, bool is_signed) -> int {
        CUE(plane_copy_down(G, (const uint8_t*)dplane, b.data(), s_));
        CUE(cudaStreamSynchronize(s_));
        for (size_t c = 0; c < n; c++) out[c] = is_signed ? (int)(int8_t)b[c] : (int)b[c];
        return HOSONO_OK;
    };
    if (scheme) TRYE(bytes_to_int(d.scheme[st.schemeSel], scheme, true));
    if (rec) TRYE(bytes_to_int(d.rec, rec, false));
    if (recF) TRYE(bytes_to_int(d.recF, recF, false));
    return HOSONO_OK;
}

int Engine::mod_reconstruct(int slot) {
    TRYE(mod_ensure(slot));
    const Slot& sl = slots_[slot];
    const Geo& G = sl.dev.geo;
    const ModBuf& M = sl.mod;
    const Batch B = batch();
    const size_t plane = (size_t)G.plane;
    CUE(cudaMemcpyAsync(M.recon, sl.dev.rec, plane, cudaMemcpyDeviceToDevice, s_));  // reconstructCell = recompute
    // every inner pass that goes on lowers at least one cell of the range by
    // one order, so (R + 1) * cells passes bound the loop
    const long long cap = (long long)(G.R + 1) * G.nxt * G.nyt + 1;
    for (long long it = 0;; it++) {
        if (it > cap) return fail(HOSONO_EMOODCAP, "reconstruct: inner cascade exceeded %lld passes", cap);
        CUE(cudaMemsetAsync(M.adm, 1, plane, s_));
        CUE(cudaMemsetAsync(M.next, 0, plane, s_));
        CUE(cudaMemsetAsync(M.flag, 0, sizeof(int), s_));
        K_->mod->recon(B, slot, G, M, s_);
        K_->mod->recon_lower(B, slot, G, M, s_);
        launches += 2;
        CUE(cudaGetLastError());
        int lowered = 0;
        CUE(cudaMemcpyAsync(&lowered, M.flag, sizeof(int), cudaMemcpyDeviceToHost, s_));
        CUE(cudaStreamSynchronize(s_));
        if (!lowered) break;
        CUE(cudaMemcpyAsync(M.recon, M.next, plane, cudaMemcpyDeviceToDevice, s_));
    }
    return HOSONO_OK;
}

int Engine::mod_getfluxes(int slot) {
    TRYE(mod_ensure(slot));
    K_->mod->getfluxes(batch(), slot, slots_[slot].dev.geo, slots_[slot].mod, s_);
    launches++;
    CUE(cudaGetLastError());
    CUE(cudaStreamSynchronize(s_));
    return HOSONO_OK;
}

int Engine::mod_flicd(int slot) {
    TRYE(mod_ensure(slot));
    const Geo& G = slots_[slot].dev.geo;
    const ModBuf& M = slots_[slot].mod;
    K_->mod->flicd(batch(), slot, G, M, s_);
    launches++;
    CUE(cudaGetLastError());
    // FLICDdivB.f90:67-68: the normal-B fluxes are zero over the whole array
    CUE(cudaMemsetAsync(M.flux + (size_t)(XDIR * NCONS + MAGX) * G.plane, 0, sizeof(double) * G.plane, s_));
    CUE(cudaMemsetAsync(M.flux + (size_t)(YDIR * NCONS + MAGY) * G.plane, 0, sizeof(double) * G.plane, s_));
    CUE(cudaStreamSynchronize(s_));
    return HOSONO_OK;
}

int Engine::mod_update(int slot, double dt) {
    TRYE(mod_ensure(slot));
    K_->mod->update(batch(), slot, slots_[slot].dev.geo, slots_[slot].mod, dt, s_);
    launches++;
    CUE(cudaGetLastError());
    CUE(cudaStreamSynchronize(s_));
    return HOSONO_OK;
}

int Engine::mod_detect(int slot, int* exit_mood_loop) {
    TRYE(mod_ensure(slot));
    const Slot& sl = slots_[slot];
    const Geo& G = sl.dev.geo;
    const ModBuf& M = sl.mod;
    const size_t plane = (size_t)G.plane;
    // checkCell = recomputeFLICD; both flag planes start the pass cleared (detect.f90:65-68)
    CUE(cudaMemcpyAsync(M.check, sl.dev.recF, plane, cudaMemcpyDeviceToDevice, s_));
    CUE(cudaMemsetAsync(sl.dev.rec, 0, plane, s_));
    CUE(cudaMemsetAsync(sl.dev.recF, 0, plane, s_));
    CUE(cudaMemsetAsync(M.lower, 0, plane, s_));
    CUE(cudaMemsetAsync(M.flag, 0, sizeof(int), s_));
    const Batch B = batch();
    K_->mod->detect(B, slot, G, M, s_);
    K_->mod->detect_lower(B, slot, G, M, s_);
    launches += 2;
    CUE(cudaGetLastError());
    int lowered = 0;
    CUE(cudaMemcpyAsync(&lowered, M.flag, sizeof(int), cudaMemcpyDeviceToHost, s_));
    CUE(cudaStreamSynchronize(s_));
    if (exit_mood_loop) *exit_mood_loop = lowered ? 0 : 1;
    return HOSONO_OK;
}

int Engine::mod_bc(int slot, int which) {
    if (which < 0 || which > 2) return fail(HOSONO_EINVAL, "boundary target %d: 0 = U, 1 = V, 2 = Unew", which);
    TRYE(mod_ensure(slot));
    InstState st;
    TRYE(state(slot, &st));
    const InstDev& d = slots_[slot].dev;
    double* A = which == 0 ? d.U[st.parity] : which == 1 ? d.V : role_ptr(d, st.parity, ROLE_A);
    K_->mod->bc(batch(), slot, d.geo, A, which == 1 ? NPRIM : NCONS, s_);
    launches++;
    CUE(cudaGetLastError());
    CUE(cudaStreamSynchronize(s_));
    return HOSONO_OK;
}

int Engine::mod_bc_mood(int slot) {
    TRYE(mod_ensure(slot));
    InstState st;
    TRYE(state(slot, &st));
    const InstDev& d = slots_[slot].dev;
    if (d.geo.bc != HOSONO_BC_PERIODIC) return HOSONO_OK;  // outflow: nothing to do (boundaryConditions.f90:39-48)
    const ModBuf& M = slots_[slot].mod;
    const size_t plane = (size_t)d.geo.plane;
    K_->mod->bc_mood(batch(), slot, d.geo, M, s_);
    launches++;
    CUE(cudaGetLastError());
    CUE(cudaMemcpyAsync(d.scheme[st.schemeSel], M.tSch, plane, cudaMemcpyDeviceToDevice, s_));
    CUE(cudaMemcpyAsync(d.rec, M.tRec, plane, cudaMemcpyDeviceToDevice, s_));
    CUE(cudaMemcpyAsync(d.recF, M.tRecF, plane, cudaMemcpyDeviceToDevice, s_));
    CUE(cudaStreamSynchronize(s_));
    return HOSONO_OK;
}

int Engine::eigenvecs(int slot, int n, const double* V, int dir, int cons, double* L, double* R) {
    if (slot < 0 || slot >= maxInst_ || !slots_[slot].live) return fail(HOSONO_EINVAL, "bad slot %d", slot);
    if (n < 0 || (dir != XDIR && dir != YDIR) || (n > 0 && (!V || !L || !R)))
        return fail(HOSONO_EINVAL, "eigenvecs: bad arguments");
    K_->mod->eigen(slots_[slot].dev.phys, n, V, dir, cons, L, R, s_);
    launches++;
    CUE(cudaGetLastError());
    CUE(cudaStreamSynchronize(s_));
    return HOSONO_OK;
}

int Engine::riemann(int slot, int n, const double* uL, const double* uR, int dir, double* F) {
    if (slot < 0 || slot >= maxInst_ || !slots_[slot].live) return fail(HOSONO_EINVAL, "bad slot %d", slot);
    if (n < 0 || (dir != XDIR && dir != YDIR) || (n > 0 && (!uL || !uR || !F)))
        return fail(HOSONO_EINVAL, "riemann: bad arguments");
    K_->mod->riemann(slots_[slot].dev.phys, n, uL, uR, dir, F, s_);
    launches++;
    CUE(cudaGetLastError());
    CUE(cudaStreamSynchronize(s_));
    return HOSONO_OK;
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
