// engine.h -- batched solver engine: any number of independent blocks
// ("instances", each a gridBlock_t + gridState_t of the reference) advanced
// together by one set of kernel launches.  A plain single solve is a batch of
// one.
//
// Kernels read their work from device tables: InstDev (per-instance geometry,
// physics and buffer pointers), InstState (per-instance mutable scalars: t,
// dt, MOOD counters, ...) and a list of 32x8 cell tiles (instance, x0, y0).
// The tile list and its length live in device memory, so instances can be
// added or removed between launches without rebuilding a CUDA graph.
#pragma once

#include <cuda.h>  // CUtensorMap (TMA descriptors; encoded through the runtime's driver entry point)
#include <cuda_runtime.h>
#include <cstdint>

#include "hosono_gpu.h"
#include "physics.cuh"

namespace hosono {

constexpr int TILE_X = 32, TILE_Y = 8;
// the MOOD pass-1 stencil box of a tile: x in [x0-4, x0+36), y in
// [y0-1-R, y0+9+R), all 8 conserved variables (kernels.cu P1Box; the TMA
// descriptors are encoded for this box shape)
constexpr int P1_SX = TILE_X + 8;
constexpr int p1_sy(int R) { return TILE_Y + 2 * R + 1; }

// Index bookkeeping of gridBlock_t (src/gridBlock.f90:36-45), 0-based:
// cells i in [0, nxt), interior [g, g+nx); planes are pitch*nyt doubles.
struct Geo {
    int nx, ny, g, nxt, nyt, pitch;
    long long plane;
    int R;   // GP_maxRadius
    int bc;  // 0 outflow, 1 periodic
    int nsMax, nqMax;
    double dx, dy, mindxdy, maxdxdy;
};

// Per-instance descriptor (device memory; written by the host at admission).
struct InstDev {
    Geo geo;
    Phys phys;
    double cfl;
    const double* pv;  // (nsMax, nqMax, 4, R)
    const double* qw;  // (nqMax, R)
    double* U[3];      // state and two stage buffers; roles rotate, see role_ptr
    double* V;         // 10 planes
    double* FX;        // fluxRaw x (8 planes): face between (i-1,j) and (i,j)
    double* FY;        // fluxRaw y (8 planes): face between (i,j-1) and (i,j)
    double* CTX;       // flux(magy, xdir): FLICD-corrected, or the raw copy
    double* CTY;       // flux(magx, ydir)
    int8_t* scheme[2];  // double-buffered MOOD scheme (GP radius per cell)
    uint8_t* rec;       // blk%recompute
    uint8_t* recF;      // blk%recomputeFLICD
    uint8_t* rrRec;     // radius each face was last reconstructed at (2 bits x 4 faces)
    uint8_t* fail;      // cell failed face CAD/PAD (inner cascade)
    uint8_t* failX;     // bit0: E side of (i-1,j) failed, bit1: W side of (i,j)
    uint8_t* failY;     // bit0: N side of (i,j-1) failed, bit1: S side of (i,j)
    uint8_t* nextPass;  // reconstructNextPass
    uint8_t* dirty;     // re-reconstructed by the pass-1 cascade
    uint8_t* lowered;   // lowered by detect in this pass
    uint8_t* innerCount;  // per-cell inner lowerings of this pass (trace)
    uint8_t* detMask;     // per-stage detect_ALL terms (shock, plateau, u2 smooth)
    // TMA descriptors of U[0..2] as (x: pitch, y: nyt, var: 8) boxes of the
    // pass-1 stencil box shape (zero fill outside the array)
    CUtensorMap tmU[3];
    // the same tensors in the boxes the staged pass-1 update reads: U[0..2]
    // as CT_SX x CT_UY x 8 boxes, fluxRaw FX and FY as CT_SX x CT_FY x 8
    CUtensorMap tmCU[3];
    CUtensorMap tmFX, tmFY;
};
// the staged pass-1 update's boxes around tile (x0, y0): U over
// [x0-4, x0+36) x [y0-2, y0+10), FX and FY over [x0-4, x0+36) x [y0-1, y0+10)
constexpr int CT_SX = TILE_X + 8, CT_UY = TILE_Y + 4, CT_FY = TILE_Y + 3;

// Per-instance mutable scalars (device memory).
struct InstState {
    double dt, t, tmax;
    int nstep, nstepmax;
    int live;        // slot holds an instance
    int done;        // time loop finished (t >= tmax or nstep >= nstepmax) or failed
    int error;       // HOSONO_* status that stopped it
    int parity;      // which of U[0], U[1] holds the state
    int schemeSel;   // which scheme buffer is current
    int stepping;    // takes part in the current step
    int stageActive;  // MOOD loop of the current stage still running
    int anyFail;     // face cascade: some cell failed CAD/PAD since the last check
    int nextIter;    // face cascade: this instance runs the next inner iteration
    int cascaded;    // face cascade ran in the current pass
    int cascadeMode;  // CASCADE_FROM_FACES after pass 1's fused kernel, else FROM_CELLS
    int nInner, nDetect;  // lowerings in the current pass
    int lastInner, lastDetect;  // lowerings of the last finished pass
    int passes;      // MOOD passes in the current stage
    int passCap;     // pass limit of a stage (HOSONO_MOOD_CAP_DEFAULT, or set by the caller)
    int maxPasses, stages, cascadeIters, passesTotal;
    long long innerTotal, detectTotal;
    unsigned long long cflbits[2];
};

// Batch-wide flags the graph's conditional nodes are driven by.
struct BatchFlags {
    int anyActive;   // some instance's MOOD loop still running
    int anyFail;     // some instance is in its face cascade
    int anyLive;     // some instance still stepping (time loop)
    int error;
    int stepsLeft;   // step budget of the current run launch
    int radii;       // bit R set when a live instance has GP radius R (per-radius kernels of absent radii exit)
    int recSel;      // which recompute list the current MOOD pass reads (0: Lists::rec, 1: rec2)
    int p1Next[4];   // pass 1 with the dynamic schedule: next tile index per radius (zeroed by stage_init)
};

// Roles of the three U buffers: the state lives in U[parity]; A in
// U[1-parity]; B in U[2].  The final RK combine writes A and flips parity.
enum : int { ROLE_STATE = 0, ROLE_A = 1, ROLE_B = 2 };

__host__ __device__ inline double* role_ptr(const InstDev& d, int parity, int role) {
    return role == ROLE_STATE ? d.U[parity] : role == ROLE_A ? d.U[1 - parity] : d.U[2];
}

// Work lists of the later MOOD passes (compacted by warp ballot): entries are
// (instance, cell index j*pitch+i); face entries carry 2*cell+dir.
enum : int { LIST_REC = 0, LIST_FACE = 1, LIST_RECF = 2, LIST_LOW = 3, LIST_NEXT = 4, LIST_CASC = 5, LIST_REC2 = 6,
             LIST_N = 7, LIST_OVERFLOW = 7 };
struct Lists {
    int2* rec;    // cells to re-reconstruct (recompute set), two buffers:
    int2* rec2;   // the current pass reads one, the flag rebuild fills the other (BatchFlags::recSel)
    int2* face;   // faces to re-flux
    int2* recF;   // cells to FLICD + update + detect (recomputeFLICD set)
    int2* low;    // cells detect lowered this pass (to clear `lowered` after use)
    int2* next;   // cells an inner cascade iteration re-reconstructs (nextPass set)
    int2* casc;   // cells the inner cascade lowered in this MOOD pass (each once)
    int8_t* sync; // per entry of low then casc: the scheme its translate class takes
    int* counts;  // [LIST_*] entries, [LIST_OVERFLOW] set if a list overflowed
    long long cap;  // entries per list (the face list holds 2*cap)
};

// One kernel launch over the batch: tables and the tile list.
struct Batch {
    const InstDev* dev;
    InstState* st;
    const int4* tiles;   // x: instance, y: x0, z: y0
    const int* ntiles;   // device counter
    BatchFlags* flags;
    Lists L;
    int p1Tma;           // pass 1 stages its stencil box with TMA (1) or cp.async (0)
    int p1Dyn;           // pass-1 blocks take tiles from a shared counter (1) or grid-stride (0)
    int p1Blocks;        // resident pass-1 blocks per SM the variant aims at (2, 3 or 4)
    int p1Boxes;         // stencil boxes per pass-1 block at two blocks per SM (1 or 2)
    int p1Radii;         // bit R: the host launches the radius-R pass-1 kernel (radii held)
    int p1First, p1End;  // pass 1 covers tiles [p1First, min(p1End, ntiles)) of the tile list
    int ctStaged;        // the pass-1 update reads TMA-staged boxes (1) or the planes (0)
    int maxTiles;        // capacity of the tile list
    int maxInst;         // capacity (slots)
    const int2* instTiles;  // per slot: first tile in the tile list, tile count (0: not live)
    const int* hold;        // per slot: nonzero = sits out the run launches (state untouched)
    unsigned* gbar;         // grid barrier of the persistent later-pass launch: {count, generation}
    // instances still in their MOOD loop after the last pass_end, in slot
    // order: (slot, first virtual tile); actInfo = {instances, tiles}.  The
    // dense kernels of the later passes walk only these tiles.
    int2* actRange;
    int* actInfo;
    // the same for the instances in the current face-cascade iteration
    // (built by cascade_cond; the cascade kernels walk only these tiles)
    int2* casRange;
    int* casInfo;
};

enum : int { CASCADE_FROM_FACES = 0, CASCADE_FROM_CELLS = 1 };
enum : int { MOOD_FLAGS_LISTS = 0, MOOD_FLAGS_DENSE = 1, MOOD_FLAGS_LISTS_CLEAR = 2 };

// Buffers of the per-module entry points (the reference's block arrays the
// fused path does not keep), allocated on a handle's first module call.
struct ModBuf {
    double* fv;       // faceVals: plane ((f*nqMax + q)*8 + v), f = NORTH..WEST
    double* flux;     // flux (gridBlock%flux): plane (dir*8 + v)
    uint8_t* recon;   // reconstructCell of the inner cascade
    uint8_t* adm;     // cellIsAdmissible
    uint8_t* next;    // reconstructNextPass
    uint8_t* check;   // detect_ALL's checkCell (recomputeFLICD on entry)
    uint8_t* lower;   // detect_ALL's lowerCell
    uint8_t* tRec;    // applyMOOD gathers (copied back afterwards)
    uint8_t* tRecF;
    int8_t* tSch;
    int* flag;        // cells lowered by the last lowering kernel
};

// Launchers of the per-module kernels (modules.cuh) for one instance.
struct ModuleOps {
    void (*recon)(const Batch&, int slot, const Geo&, const ModBuf&, cudaStream_t);
    void (*recon_lower)(const Batch&, int slot, const Geo&, const ModBuf&, cudaStream_t);
    void (*getfluxes)(const Batch&, int slot, const Geo&, const ModBuf&, cudaStream_t);
    void (*flicd)(const Batch&, int slot, const Geo&, const ModBuf&, cudaStream_t);
    void (*update)(const Batch&, int slot, const Geo&, const ModBuf&, double dt, cudaStream_t);
    void (*detect)(const Batch&, int slot, const Geo&, const ModBuf&, cudaStream_t);
    void (*detect_lower)(const Batch&, int slot, const Geo&, const ModBuf&, cudaStream_t);
    void (*bc_mood)(const Batch&, int slot, const Geo&, const ModBuf&, cudaStream_t);
    void (*bc)(const Batch&, int slot, const Geo&, double* A, int nv, cudaStream_t);
    void (*riemann)(const Phys&, int n, const double* uL, const double* uR, int dir, double* F, cudaStream_t);
    void (*eigen)(const Phys&, int n, const double* V, int dir, int cons, double* L, double* R, cudaStream_t);
};

// Launchers of one arithmetic build (kernels.cu compiled strict or fast).
struct KernelSet {
    const char* name;
    // time loop: per-instance step begin (cfl -> validated dt) and end
    void (*cfl_reduce)(const Batch&, cudaStream_t);
    void (*step_prepare)(const Batch&, int steps, cudaStream_t);
    void (*step_begin)(const Batch&, int use_host_dt, cudaStream_t);
    void (*step_end)(const Batch&, cudaGraphConditionalHandle run_cond, cudaStream_t);
    // forward-Euler stage
    void (*stage_init)(const Batch&, cudaStream_t);
    void (*face_pass1)(const Batch&, int uin, cudaStream_t);
    void (*cascade_cond)(const Batch&, cudaGraphConditionalHandle h, cudaStream_t);
    // face cascade: the kernels walk the tiles of the instances in the
    // current iteration (Batch::casRange); `later` marks a later MOOD pass
    void (*cascade_lower)(const Batch&, int later, cudaStream_t);
    void (*recon_check)(const Batch&, int uin, int later, cudaStream_t);  // compact nextPass, re-reconstruct
    void (*ct_update_detect)(const Batch&, int uin, int uout, cudaStream_t);
    // MOOD_FLAGS_*: dense on every cell (pass 1), or from the work lists
    // (later passes), clearing `lowered` too unless a trace reads it first
    void (*mood_flags)(const Batch&, int mode, cudaStream_t);
    // flip: the dense flag rebuild wrote the other scheme buffer
    void (*pass_end)(const Batch&, cudaGraphConditionalHandle h, int flip, cudaStream_t);
    // later MOOD passes on compacted work lists
    void (*recon_list)(const Batch&, int uin, cudaStream_t);
    void (*compact_post)(const Batch&, cudaStream_t);   // faces and recomputeFLICD cells
    void (*compact_dirty)(const Batch&, cudaStream_t);  // pass-1 faces next to re-reconstructed cells
    void (*flux_list)(const Batch&, int uin, cudaStream_t);
    void (*ct_list)(const Batch&, int uin, int uout, cudaStream_t);
    void (*clear_low)(const Batch&, cudaStream_t);
    // RK3 combines and boundary conditions
    void (*bc_fill)(const Batch&, int role, cudaStream_t);
    void (*rk_combine2)(const Batch&, cudaStream_t);
    void (*rk_final)(const Batch&, cudaStream_t);
    void (*cons2prim_all)(const Batch&, cudaStream_t);
    // autotuner: mark the live, unfinished, not held instances as stepping
    // (on) or at rest (off) so that pass 1 can be timed outside a step
    void (*tune_mark)(const Batch&, int on, cudaStream_t);
    // every later MOOD pass of a stage in one persistent (cooperative) launch
    void (*mood_rest)(const Batch&, int uin, int uout, cudaStream_t);
    // grids the launchers use: the pass-1 kernel of radius R, and the
    // largest grid of the other per-tile kernels (each capped at maxTiles)
    void (*launch_info)(int R, int maxTiles, int* pass1_grid, int* tile_grid_max);
    const ModuleOps* mod;
};

const KernelSet* kernelset_strict();
const KernelSet* kernelset_fast();

// layout conversions for one instance (no arithmetic; one build)
// Programmatic dependent launch of the next kernel launch on this host
// thread: pdl_arm(first, chain) before a step's launches (first: the next
// launch may overlap its predecessor; chain: the launches after it too),
// pdl_take() in each launch helper.  Off outside the step recorder.
void pdl_arm(bool first, bool chain);
bool pdl_take();

void launch_aos_to_soa(const Geo& G, const double* aos, double* soa, int nvar, cudaStream_t s);
void launch_aos_to_soa_rows(const Geo& G, const double* aos, double* soa, int nvar, int j0, int j1, cudaStream_t s);
void launch_soa_to_aos(const Geo& G, const double* soa, double* aos, int nvar, cudaStream_t s);
void launch_scheme_to_int(const Geo& G, const int8_t* scheme, int* out, cudaStream_t s);
// initialCondition_set on the device (ic.cu)
void launch_ic(const Geo& G, int force_hydro, double gamma, const hosono_ic_desc& ic, const double* xtab,
               const double* ytab, double* U, double* V, cudaStream_t s);
// output_writeHdf5's derived fields and div(B) norms (diagnostics.cu)
void launch_diagnostics(const Geo& G, const double* V, const int8_t* scheme, double* fields, int* schOut,
                        int* ordr, double* rows, double* res, cudaStream_t s);

}  // namespace hosono
