// engine_host.h -- host side of the batched engine (engine.cu).
#pragma once

#include "engine.h"
#include "hosono_gpu.h"

#include <string>
#include <vector>

namespace hosono {

struct TraceRec {
    int slot, stage, pass, nInner, nDetect;
    std::vector<unsigned char> inner, detect;  // nxt*nyt, i fastest
};

// Where an engine takes instance memory from: cudaMalloc by default, or a
// caller's pool (the server's arena).
struct DeviceAllocator {
    virtual ~DeviceAllocator() = default;
    virtual void* alloc(size_t bytes) = 0;  // nullptr when it does not fit
    virtual void release(void* p) = 0;
};

class Engine {
  public:
    Engine() = default;
    ~Engine();
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    // capacity: instance slots and 32x8 tiles over all instances
    int init(int max_inst, int max_tiles, int fp_mode);
    // commit_tables = false defers the tile-list upload to commit_tables(),
    // so that many admissions or retirements rebuild it once
    int add(const hosono_params& p, const double* pv, const double* qw, int* slot, bool commit_tables = true);
    int remove(int slot, bool commit_tables = true);
    int commit_tables() { return upload_tables(); }
    // staging for upload/download of instances up to `cells` cells
    int reserve_staging(size_t cells);
    void set_allocator(DeviceAllocator* a) { alloc_ = a; }
    int upload(int slot, const double* U, const double* V);
    // U host -> device (Fortran-order AoS with guards), nothing else
    int upload_u(int slot, const double* U);
    // hosono_gpu_advance_host: U up, one step of dt, U (and V) down.  With
    // upload bands, U goes up in row bands on a second stream while the first
    // stage's pass 1 computes the tiles of the bands already landed.
    int advance_host(int slot, double dt, double* U, double* V);
    int download(int slot, double* U, double* V, int* scheme);
    // the initial state built on the device (hosono_ic_describe's output)
    int ic(int slot, const hosono_ic_desc& d, const double* xtab, const double* ytab);
    // output_writeHdf5's fields of the interior (13 double planes + scheme,
    // ordr; any may be null) and mean / max |div B|; allocates device scratch
    int diagnostics(int slot, double* fields, int* scheme, int* ordr, double* divb_l1, double* divb_linf);
    int set_time(int slot, double t, double tmax, int nstep, int nstepmax);
    // per slot (maxInst entries): nonzero holds the instance out of the
    // following run() launches, its state untouched (serving priority)
    int set_holds(const int* holds);
    // MOOD passes a stage may take before the instance stops with
    // HOSONO_EMOODCAP (cap <= 0: the proven bound R*nx*ny + 1)
    int set_mood_cap(int slot, int cap);
    int state(int slot, InstState* out);
    // cfl_computedt of one instance (dt to the host)
    int cfl(int slot, double* dt);
    // timeStep_advanceSolution of one instance with a host dt
    int advance(int slot, double dt);
    // time loop of every live instance: up to max_steps steps (<=0: until done)
    int run(int max_steps);
    // one step of every live instance with the pass-1 kernel bracketed by events
    int run_profiled_step(double* pass1_ms, int* pass1_launches);

    int tiles_of(const hosono_params& p) const;
    // ---- per-module form (the reference's stage modules one at a time on
    // one instance; modules.cuh).  Host arrays in the reference's Fortran
    // order; NULL pointers are skipped.
    int mod_set(int slot, const int* scheme, const int* rec, const int* recF);
    int mod_get(int slot, double* faceVals, double* fluxRaw, double* flux, double* Unew, int* scheme, int* rec,
                int* recF);
    int mod_reconstruct(int slot);
    int mod_getfluxes(int slot);
    int mod_flicd(int slot);
    int mod_update(int slot, double dt);
    int mod_detect(int slot, int* exit_mood_loop);
    int mod_bc(int slot, int which);
    int mod_bc_mood(int slot);
    int riemann(int slot, int n, const double* uL, const double* uR, int dir, double* F);
    int eigenvecs(int slot, int n, const double* V, int dir, int cons, double* L, double* R);

    // launch geometry of the kernels for radius R over this engine's tile capacity
    void launch_info(int R, int* pass1_grid, int* tile_grid_max) const { K_->launch_info(R, maxTiles_, pass1_grid, tile_grid_max); }
    int live_count() const;
    size_t instance_bytes(const hosono_params& p) const;
    const hosono_params& params(int slot) const { return slots_[slot].p; }
    const Geo& geo(int slot) const { return slots_[slot].dev.geo; }
    const InstDev& dev(int slot) const { return slots_[slot].dev; }
    cudaStream_t stream() const { return s_; }
    int max_inst() const { return maxInst_; }
    int max_tiles() const { return maxTiles_; }
    int used_tiles() const {  // of every live slot, committed to the tile list or not
        int n = 0;
        for (const auto& sl : slots_) n += sl.live ? sl.ntiles : 0;
        return n;
    }

    // run() fails when an instance stopped with an error; when false, the
    // instance just ends (done, with its error code) and the others go on
    bool instance_errors_fatal = true;
    // per-slot states as of the end of the last run() (pinned host copy)
    const InstState* host_states() const { return h_st_; }
    // launch choices (hosono_tuning); changing them rebuilds the step graphs
    int set_tuning(const hosono_tuning& t);
    // time the candidate tunings on the live instances, apply the fastest
    int autotune(int trials, bool force, hosono_tune_report* rep);
    const hosono_tuning& tuning() const { return tune_; }
    // GP radii among the held instances (one pass-1 launch each per stage)
    int radii_held() const { return __builtin_popcount((unsigned)radii_); }
    bool use_graphs = true;
    bool trace = false;
    std::vector<TraceRec> traces;
    std::vector<int> traceStageBase;
    long long launches = 0;  // kernels launched (eager) or executed (graph, counted per node)

    int err = HOSONO_OK;
    std::string msg;
    int fail(int code, const char* fmt, ...);

  private:
    struct Slot {
        bool live = false;
        hosono_params p{};
        InstDev dev{};
        std::vector<void*> allocs;
        int ntiles = 0;
        ModBuf mod{};         // per-module buffers, allocated on first use
        void* modAlloc = nullptr;
    };
    int mod_ensure(int slot);
    int encode_tmaps(InstDev& dev);
    void drop_graphs();
    // a new engine's launch choices: the fastest on the benchmarked workloads
    // (TMA staging, dynamic tile schedule, two blocks per SM with one box each)
    hosono_tuning tune_{HOSONO_STAGE_TMA, HOSONO_SCHED_DYNAMIC, 2, HOSONO_LATER_KERNELS, 1, 0, 0, HOSONO_STAGE_CP_ASYNC};
    class Rec;
    friend class Rec;

    Batch batch() const;
    int upload_tables();
    int write_state_field(int slot, size_t offset, const void* src, size_t n);
    template <typename T>
    int write_field(int slot, T InstState::*field, T value) {
        const InstState* z = nullptr;
        return write_state_field(slot, (size_t)((const char*)&(z->*field) - (const char*)z), &value, sizeof(T));
    }
    // head = false leaves out the stage's set-up and pass 1 (run before, by the banded upload)
    int record_stage(Rec& r, int uin, int uout, cudaEvent_t ev0, cudaEvent_t ev1, bool head = true);
    int record_step(Rec& r, bool host_dt, cudaGraphConditionalHandle run_cond, bool profile,
                    bool first_head = true);
    int build_graphs();
    int launch(cudaGraphExec_t g);
    int sync();
    int check_errors();
    int trace_before_pass();
    int trace_snapshot();
    int trace_after_pass();

    void* dalloc(size_t bytes);
    void dfree(void* p);

    DeviceAllocator* alloc_ = nullptr;
    const KernelSet* K_ = nullptr;
    cudaStream_t s_ = nullptr;
    int maxInst_ = 0, maxTiles_ = 0;
    int radii_ = 0;       // BatchFlags::radii of the committed tile list
    int graphRadii_ = 0;  // radii_ when the step graphs were recorded (their pass-1 launches)
    InstDev* d_dev_ = nullptr;
    InstState* d_st_ = nullptr;
    int4* d_tiles_ = nullptr;
    int2* d_instTiles_ = nullptr;
    int2* d_actRange_ = nullptr;
    int* d_actInfo_ = nullptr;
    int2* d_casRange_ = nullptr;
    int* d_casInfo_ = nullptr;
    int* d_hold_ = nullptr;
    unsigned* d_gbar_ = nullptr;
    std::vector<int2> instTiles_;
    int* d_ntiles_ = nullptr;
    BatchFlags* d_flags_ = nullptr;
    Lists lists_{};
    BatchFlags* h_flags_ = nullptr;  // pinned
    InstState* h_st_ = nullptr;      // pinned
    double* staging_ = nullptr;
    size_t stagingCells_ = 0;
    int* schemeInt_ = nullptr;
    std::vector<Slot> slots_;
    std::vector<int4> tiles_;
    cudaGraphExec_t gAdvance_ = nullptr, gRun_ = nullptr, gProf_ = nullptr;
    cudaGraphExec_t gAdvRest_ = nullptr;  // gAdvance_ without the first stage's set-up and pass 1
    cudaStream_t sCopy_ = nullptr;        // the banded upload's copy stream
    cudaEvent_t bandEv_[HOSONO_UPLOAD_BANDS_MAX + 1] = {};
    cudaEvent_t profEv_[6] = {};
    std::vector<long long> tracePassesSeen_;
    std::vector<std::vector<unsigned char>> snapInner_, snapLow_;
};

}  // namespace hosono
