// kernels.h -- launch interface between the solver (host orchestration) and
// the stage kernels.  kernels.cu is compiled twice, once per arithmetic mode
// (strict: no FMA contraction; fast: contraction allowed); each object
// exports one KernelTable.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "physics.cuh"

namespace hosono {

// Index bookkeeping of gridBlock_t (src/gridBlock.f90:36-45), 0-based:
// cells i in [0, nxt), interior [g, g+nx); planes are pitch*nyt doubles.
struct Geo {
    int nx, ny, g, nxt, nyt, pitch;
    long long plane;
    int R;       // GP_maxRadius
    int bc;      // 0 outflow, 1 periodic
    int nsMax, nqMax;
    double dx, dy, mindxdy, maxdxdy;
};

// counters[] slots
enum : int { CNT_ANYFAIL = 0, CNT_INNER = 1, CNT_DETECT = 2, CNT_N = 4 };

struct StageArgs {
    Geo geo;
    Phys phys;
    const double* pv;  // (nsMax, nqMax, 4, R)
    const double* qw;  // (nqMax, R)
    const double* Uin;  // stage input U (8 planes, guards filled)
    double* Uout;       // stage candidate Unew (8 planes, interior written)
    double* FX;         // fluxRaw x (8 planes): face between (i-1,j) and (i,j)
    double* FY;         // fluxRaw y (8 planes): face between (i,j-1) and (i,j)
    double* CTX;        // flux(magy, xdir): FLICD-corrected (or raw copy)
    double* CTY;        // flux(magx, ydir)
    int8_t* scheme;     // current MOOD scheme (GP radius) per cell
    int8_t* scheme_next;
    uint8_t* rec;       // blk%recompute
    uint8_t* recF;      // blk%recomputeFLICD
    uint8_t* rrRec;     // radius each face's values were last reconstructed at (2 bits x 4 faces)
    uint8_t* fail;      // cell failed the face CAD/PAD check (inner cascade)
    uint8_t* failX;     // bit0: E side of (i-1,j) failed, bit1: W side of (i,j) failed
    uint8_t* failY;     // bit0: N side of (i,j-1) failed, bit1: S side of (i,j) failed
    uint8_t* nextPass;  // reconstructNextPass
    uint8_t* dirty;     // cell re-reconstructed by the inner cascade in pass 1
    uint8_t* lowered;   // cells lowered by detect in this pass
    uint8_t* innerCount;  // per-cell inner lowerings (trace only)
    int* counters;
    double dt;
    int trace;
};

enum : int { CASCADE_FROM_FACES = 0, CASCADE_FROM_CELLS = 1 };
enum : int { FLUX_DIRTY = 0, FLUX_REC = 1 };

struct KernelTable {
    const char* name;
    // MOOD pass 1: reconstruct + face CAD/PAD + HLLC fluxes, every face at radius R
    void (*face_pass1)(const StageArgs&, cudaStream_t);
    // inner cascade: lower failing cells (gridBlock_lowerOrder) and flag the cross
    void (*cascade_lower)(const StageArgs&, int mode, cudaStream_t);
    // reconstruct + CAD/PAD check of the cells flagged in mask
    void (*recon_check)(const StageArgs&, const uint8_t* mask, cudaStream_t);
    // getFluxes_ on flagged faces
    void (*flux)(const StageArgs&, int mode, cudaStream_t);
    // FLICD + unsplit update + detect_ALL on cells with recomputeFLICD
    void (*ct_update_detect)(const StageArgs&, cudaStream_t);
    // rebuild scheme/recompute/recomputeFLICD from the lowered cells, with the
    // periodic guard/image sync of boundaryConditions_applyMOOD
    void (*mood_flags)(const StageArgs&, cudaStream_t);
    // boundaryConditions_applyBlk on nvar planes (guard gather)
    void (*bc_fill)(const Geo&, double* A, int nvar, cudaStream_t);
    // U2 = (3U + U2)/4 on every cell (guards from their images)
    void (*rk_combine2)(const Geo&, const double* Un, const double* B, double* out, cudaStream_t);
    // Unew = (U + 2 U3)/3 and V = cons2prim(Unew) on every cell
    void (*rk_final)(const Geo&, const Phys&, const double* Un, const double* B, double* outU, double* outV,
                     cudaStream_t);
    // V = cons2prim(U) on every cell
    void (*cons2prim_all)(const Geo&, const Phys&, const double* U, double* V, cudaStream_t);
    // max |u|+c_f, |v|+c_f over the interior (bit patterns of two non-negative doubles)
    void (*cfl_max)(const Geo&, const Phys&, const double* V, unsigned long long* out2, cudaStream_t);
};

const KernelTable* kernels_strict();
const KernelTable* kernels_fast();

// layout conversions (no arithmetic; one variant)
void launch_aos_to_soa(const Geo& G, const double* aos, double* soa, int nvar, cudaStream_t s);
void launch_soa_to_aos(const Geo& G, const double* soa, double* aos, int nvar, cudaStream_t s);
void launch_scheme_to_int(const Geo& G, const int8_t* scheme, int* out, cudaStream_t s);

}  // namespace hosono
