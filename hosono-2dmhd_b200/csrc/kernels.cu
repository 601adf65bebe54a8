// kernels.cu -- FP64 stage kernels of the hosono-2DMHD time step for sm_100a,
// batched: every launch walks a list of 32x8 cell tiles that may belong to
// any number of independent instances (engine.h).
//
// Compiled twice: with -DHOSONO_FAST=0 --fmad=false (strict: every operation
// rounded on its own, bit-identical to the oracle) and with -DHOSONO_FAST=1
// --fmad=true (FMA contraction allowed).  Each object exports one KernelSet.
//
// Data layout in HBM: structure of arrays, one plane per conserved variable
// (and per primitive variable for V), rows of `pitch` doubles (a multiple of
// 32, i.e. 256-byte rows), guard cells included.  Cell (i,j) 0-based at
// j*pitch+i; the interior is [g, g+nx) x [g, g+ny), g = NGC = R+2.  MOOD
// state is one byte per cell per flag.
//
// Index ranges (0-based) of the reference loops:
//   reconstruct   [strt-2, stop+2] -> [g-2, g+n+1]   (reconstruct.f90:81-82)
//   getFluxes     [strt-1, stop+2] -> [g-1, g+n+1]   (getFluxes.f90:27-28)
//   FLICD         [strt,   stop+1] -> [g,   g+n]     (FLICDdivB.f90:34-35)
//   update/detect [strt,   stop]   -> [g,   g+n-1]   (timeStep.f90:108-109, detect.f90:81-82)

#include <algorithm>
#include <mutex>

#include "engine.h"
#include "hosono_gpu.h"

#ifndef HOSONO_FAST
#error "HOSONO_FAST must be defined (0 strict, 1 fast)"
#endif

#if HOSONO_FAST
#define KNS kfast
#else
#define KNS kstrict
#endif


namespace hosono {
namespace KNS {

constexpr int NTHREADS = TILE_X * TILE_Y;

// detMask bits: the per-stage detect_ALL terms (written by k_ct_update_detect),
// and DM_CASC, set while a cell sits on the cascade-lowered list of the
// current MOOD pass
enum : int { DM_SHOCK = 1, DM_PLATEAU = 2, DM_SMOOTH = 4, DM_CASC = 8 };

__device__ __forceinline__ int iabs_c(int a) { return a < 0 ? -a : a; }

// The instance and cell a thread works on in tile t.
struct Cell {
    int k, i, j;
};
__device__ __forceinline__ Cell tile_at(const Batch& B, int t) {
    const int4 v = B.tiles[t];
    Cell c;
    c.k = v.x;
    c.i = v.y + threadIdx.x;
    c.j = v.z + threadIdx.y;
    return c;
}
// Kernels walk the tile list grid-stride: the grid is sized to the GPU, the
// tile count is read from device memory at run time.
#define FOR_TILES(B, t) for (int t = blockIdx.x, n_ = __ldg((B).ntiles); t < n_; t += gridDim.x)

// Tile of virtual index v in the active instances' tiles (binary search over
// the ranges pass_end left); uniform over a block.
__device__ __forceinline__ int range_tile(const Batch& B, const int2* range, const int* info, int v) {
    int lo = 0, hi = info[0] - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (range[mid].y <= v)
            lo = mid;
        else
            hi = mid - 1;
    }
    const int2 r = range[lo];
    return B.instTiles[r.x].x + (v - r.y);
}
__device__ __forceinline__ int active_tile(const Batch& B, int v) { return range_tile(B, B.actRange, B.actInfo, v); }
// The face cascade: only the tiles of instances in the current iteration.
#define FOR_CASCADE_TILES(B, t)                                                              \
    for (int v_ = blockIdx.x, nv_ = (B).casInfo[1], t = 0; v_ < nv_; v_ += gridDim.x)       \
        for (bool once_ = (t = range_tile((B), (B).casRange, (B).casInfo, v_), true); once_; once_ = false)
// Later MOOD passes: only the tiles of instances still in their MOOD loop.
#define FOR_ACTIVE_TILES(B, t)                                                              \
    for (int v_ = blockIdx.x, nv_ = (B).actInfo[1], t = 0; v_ < nv_; v_ += gridDim.x)      \
        for (bool once_ = (t = active_tile((B), v_), true); once_; once_ = false)


// the one thread per instance that owns cell (0,0) (every instance has a tile at its origin)
__device__ __forceinline__ bool first_tile_thread(const Cell& c) { return c.i == 0 && c.j == 0; }

// GP prediction at quadrature point q of face f of cell (i,j), radius RR:
// sum_k pv(k,q,f,RR) * U(:, stencil_k), stencil order k=1..ns
// (reconstruct.f90:109-124; stencil order of GP.f90:85-95).
template <int RR>
__device__ __forceinline__ void gp_face(const double* __restrict__ U, long long plane, int pitch, int i, int j,
                                        const double* __restrict__ pvq, double out[NCONS]) {
#pragma unroll
    for (int v = 0; v < NCONS; v++) out[v] = 0.0;
    int k = 0;
#pragma unroll
    for (int a = -RR; a <= RR; a++) {
#pragma unroll
        for (int b = -RR; b <= RR; b++) {
            if (iabs_c(a) + iabs_c(b) <= RR) {
                const double p = __ldg(pvq + k);
                const long long idx = (long long)(j + b) * pitch + (i + a);
#pragma unroll
                for (int v = 0; v < NCONS; v++) out[v] = out[v] + p * __ldg(U + v * plane + idx);
                k++;
            }
        }
    }
}

__device__ __forceinline__ const double* pv_ptr(const InstDev& d, int rr, int f, int q) {
    return d.pv + (long long)d.geo.nsMax * (q + d.geo.nqMax * (f + 4 * (rr - 1)));
}
__device__ __forceinline__ double qw_at(const InstDev& d, int rr, int q) {
    return __ldg(d.qw + q + d.geo.nqMax * (rr - 1));
}

// face value with a run-time radius; rr == 0 is the first-order copy of U
__device__ __forceinline__ void face_value(const InstDev& d, const double* __restrict__ U, int rr, int i, int j, int f,
                                           int q, double out[NCONS]) {
    const Geo& G = d.geo;
    if (rr == 0) {
        const long long idx = (long long)j * G.pitch + i;
#pragma unroll
        for (int v = 0; v < NCONS; v++) out[v] = __ldg(U + v * G.plane + idx);
        return;
    }
    const double* pvq = pv_ptr(d, rr, f, q);
    if (rr == 1)
        gp_face<1>(U, G.plane, G.pitch, i, j, pvq, out);
    else if (rr == 2)
        gp_face<2>(U, G.plane, G.pitch, i, j, pvq, out);
    else
        gp_face<3>(U, G.plane, G.pitch, i, j, pvq, out);
}

__device__ __forceinline__ void warp_flag(int* flag, bool v) {
    const unsigned m = __ballot_sync(0xffffffffu, v);
    if (m && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}
__device__ __forceinline__ void warp_count(int* counter, bool v) {
    const unsigned m = __ballot_sync(0xffffffffu, v);
    if (m && (threadIdx.x & 31) == 0) atomicAdd(counter, __popc(m));
}

// ----------------------------------------------------------------------
// Work lists of the later MOOD passes.  Appends are warp-aggregated: one
// atomicAdd per warp reserves the slots, each active lane writes at its rank.
__device__ __forceinline__ void warp_append(const Lists& L, int which, int2* list, long long cap, bool pred,
                                            int2 item) {
    const unsigned m = __ballot_sync(0xffffffffu, pred);
    if (!m) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(L.counts + which, __popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    const long long pos = (long long)base + __popc(m & ((1u << lane) - 1));
    if (pred) {
        if (pos < cap)
            list[pos] = item;
        else
            L.counts[LIST_OVERFLOW] = 1;
    }
}

__device__ __forceinline__ int2 entry(int k, long long cc) { return make_int2(k, (int)cc); }

// The two recompute lists: the current MOOD pass reads one (next = false),
// the flag rebuild at its end fills the other (next = true); pass_end swaps.
__device__ __forceinline__ int rec_sel(const Batch& B, bool next) { return B.flags->recSel ^ (next ? 1 : 0); }
__device__ __forceinline__ int2* rec_list(const Batch& B, bool next) { return rec_sel(B, next) ? B.L.rec2 : B.L.rec; }
__device__ __forceinline__ int rec_count(const Batch& B, bool next) { return rec_sel(B, next) ? LIST_REC2 : LIST_REC; }

// Programmatic dependent launch.  A kernel launched with
// cudaLaunchAttributeProgrammaticStreamSerialization may be scheduled while
// its predecessor on the stream still runs: every block first waits here,
// before it touches memory, until the predecessor grid has completed and its
// writes are visible, then lets its own successor be scheduled (whose blocks
// wait here in turn, so at most two grids are resident and the earlier one
// has all its blocks running).  Without the attribute both are no-ops.
#define PDL_ENTRY()                                                     \
    do {                                                                \
        asm volatile("griddepcontrol.wait;\n" ::: "memory");             \
        asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); \
    } while (0)

// ======================================================================
// MOOD pass 1 (every scheme == R): reconstruct_faceValsWithGP + face CAD/PAD
// + getFluxes_ fused.  A thread owns the x-face between (i-1,j) and (i,j) and
// the y-face between (i,j-1) and (i,j).  Face values are recomputed per
// quadrature point and never stored.  A cell fails when any of its four
// faces fails; the verdicts are kept per face side in failX / failY and
// combined by cascade_lower.  Fluxes next to a cell the cascade
// re-reconstructs are recomputed after it (compact_dirty + flux_list).
//
// The block stages its tile's stencil box -- x in [x0-4, x0+36), y in
// [y0-1-R, y0+9+R), all 8 planes -- in shared memory (16-byte vector loads,
// 256-byte rows), so every GP dot product reads shared memory at offsets
// known at compile time.
template <int R>
struct P1Box {
    static constexpr int SX = P1_SX;     // [x0-4, x0+36)
    static constexpr int SY = p1_sy(R);  // [y0-1-R, y0+8+R)
    static constexpr int PLANE = SX * SY;
    static constexpr int DOUBLES = NCONS * PLANE;
    static constexpr int OX = 4, OY = 1 + R;       // shared coordinates of the tile origin
    // the instance's radius-R prediction vectors pv(k, q, face) (the rr = R
    // block of its (nsMax, nqMax, 4, R) table, nsMax = NS, nqMax = NQ)
    static constexpr int NS = 1 + 2 * R * (R + 1), NQ = R + 1;
    static constexpr int PVN = NS * NQ * 4;
};

// GP prediction from the shared box: sum_k pv(k,q,f,RR) * U(:, stencil_k)
// around shared coordinates (sx, sy), stencil order k=1..ns; pvq points at
// the prediction vector in shared memory (one broadcast load per k)
template <int RR, int R>
__device__ __forceinline__ void gp_face_s(const double* __restrict__ sU, int sx, int sy,
                                          const double* __restrict__ pvq, double out[NCONS]) {
    constexpr int SX = P1Box<R>::SX, PL = P1Box<R>::PLANE;
    const double* base = sU + sy * SX + sx;
#pragma unroll
    for (int v = 0; v < NCONS; v++) out[v] = 0.0;
    int k = 0;
#pragma unroll
    for (int a = -RR; a <= RR; a++) {
#pragma unroll
        for (int b = -RR; b <= RR; b++) {
            if (iabs_c(a) + iabs_c(b) <= RR) {
                const double p = pvq[k];
#pragma unroll
                for (int v = 0; v < NCONS; v++) out[v] = out[v] + p * base[v * PL + b * SX + a];
                k++;
            }
        }
    }
}

// one face (both sides, every quadrature point); returns the side verdict bits
// (the Gauss sum of the fluxes accumulates in this thread's column of
// shared memory, acc[v * NTHREADS], which keeps it out of the registers the
// Riemann solver needs).  dir is a run-time value: the kernel holds one copy
// of this code (and of the Riemann solver) for both face directions, which
// halves its instruction footprint.
template <int R, int FH>
__device__ __forceinline__ uint8_t pass1_face(const InstDev& d, const double* __restrict__ sU,
                                              const double* __restrict__ sPv, int sx, int sy, int dir, bool needL,
                                              bool needR, bool doFlux, long long c, double* acc) {
    const Geo& G = d.geo;
    const Phys& P = d.phys;
    constexpr int NQ = R + 1;
    const bool x = dir == XDIR;
    const int FL = x ? EAST : NORTH, FR = x ? WEST : SOUTH;
    const int lx = x ? sx - 1 : sx, ly = x ? sy : sy - 1;
    uint8_t bits = 0;
#pragma unroll
    for (int v = 0; v < NCONS; v++) acc[v * NTHREADS] = 0.0;
#pragma unroll 1
    for (int q = 0; q < NQ; q++) {
        double uL[NCONS], uR[NCONS];
        if (needL) {
            gp_face_s<R, R>(sU, lx, ly, sPv + P1Box<R>::NS * (q + P1Box<R>::NQ * FL), uL);
            if (!admissible(uL[DENS], cons2pres<FH>(P, uL))) bits |= 1;
        }
        if (needR) {
            gp_face_s<R, R>(sU, sx, sy, sPv + P1Box<R>::NS * (q + P1Box<R>::NQ * FR), uR);
            if (!admissible(uR[DENS], cons2pres<FH>(P, uR))) bits |= 2;
        }
        if (doFlux) {
            double F[NCONS];
            hllc<FH>(P, uL, uR, dir, F);
            const double w = qw_at(d, R, q);
#pragma unroll
            for (int v = 0; v < NCONS; v++) acc[v * NTHREADS] = acc[v * NTHREADS] + w * F[v];
        }
    }
    if (doFlux) {
        double* Fo = x ? d.FX : d.FY;
#pragma unroll
        for (int v = 0; v < NCONS; v++) Fo[v * G.plane + c] = acc[v * NTHREADS];
        (x ? d.CTX : d.CTY)[c] = acc[(x ? MAGY : MAGX) * NTHREADS];
    }
    return bits;
}

// the x- and y-faces of one cell of the staged tile (sim_forceHydro fixed at
// compile time); returns whether any face state failed CAD/PAD
template <int R, int FH>
__device__ __forceinline__ bool pass1_tile(const InstDev& d, const double* __restrict__ sU,
                                           const double* __restrict__ sPv, const Cell& c, double* acc) {
    using Box = P1Box<R>;
    const Geo& G = d.geo;
    const int i = c.i, j = c.j;
    const int g = G.g;
    const int clo = g - 2, cxhi = g + G.nx + 1, cyhi = g + G.ny + 1;  // reconstruct range
    const int flo = g - 1, fxhi = g + G.nx + 1, fyhi = g + G.ny + 1;  // flux range
    const int sx = threadIdx.x + Box::OX, sy = threadIdx.y + Box::OY;
    const long long cc = (long long)j * G.pitch + i;
    const bool inF = i >= flo && i <= fxhi && j >= flo && j <= fyhi;
    bool bad = false;
#pragma unroll 1
    for (int dir = XDIR; dir <= YDIR; dir++) {  // the x-face, then the y-face of this cell
        const bool x = dir == XDIR;
        if (i >= clo && i <= cxhi + (x ? 1 : 0) && j >= clo && j <= cyhi + (x ? 0 : 1)) {
            const int a = x ? i : j, ahi = x ? cxhi : cyhi;
            const uint8_t bits = pass1_face<R, FH>(d, sU, sPv, sx, sy, dir, a - 1 >= clo, a <= ahi, inF, cc, acc);
            (x ? d.failX : d.failY)[cc] = bits;
            bad |= bits != 0;
        }
    }
    return bad;
}

// 16-byte asynchronous copy global -> shared (cp.async); src_bytes = 0
// writes zeros and reads nothing
__device__ __forceinline__ void cp_async16(void* dst, const void* src, int src_bytes) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(src_bytes) : "memory");
}
// 8-byte asynchronous copy global -> shared (cp.async.ca: 4, 8 or 16 bytes)
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// ---- TMA staging (cp.async.bulk.tensor with an mbarrier; 1-GPU memory
// only, no multicast).  One thread issues the copies of a box; every thread
// waits on the box's mbarrier.  Waits are bounded: after about two seconds a
// wait gives up and the kernel reports HOSONO_ETIMEOUT instead of hanging.
constexpr long long kWaitCycles = 4000000000LL;
__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
// true once the barrier's phase `parity` has completed; false after kWaitCycles
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
    const unsigned a = smem_addr(bar);
    const long long t0 = clock64();
    for (;;) {
        unsigned done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > kWaitCycles) return false;
    }
}
// a (x, y, var) box of the tensor map into shared memory; x * 8 bytes is a
// multiple of 16 (x = x0 - 4 with x0 a multiple of 32) and may be negative
// (zero fill), as may y
__device__ __forceinline__ void tma_box3(void* dst, const CUtensorMap* tm, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];\n" ::"r"(smem_addr(dst)),
        "l"(tm), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
        : "memory");
}
// contiguous bytes (a multiple of 16, both addresses 16-byte aligned)
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// next tile at or after t (stride gridDim.x) that this launch works on
template <int R>
__device__ __forceinline__ int pass1_next(const Batch& B, int t, int n) {
    for (; t < n; t += gridDim.x) {
        const int k = B.tiles[t].x;
        if (B.st[k].stepping && B.dev[k].geo.R == R) return t;
    }
    return n;
}

// the dynamic schedule: the next tile of this radius from the launch-wide
// counter, counted from the launch's first tile (one atomic per tile taken;
// n when none is left)
template <int R>
__device__ __forceinline__ int pass1_take(const Batch& B, int n) {
    for (;;) {
        const int t = B.p1First + atomicAdd(&B.flags->p1Next[R], 1);
        if (t >= n) return n;
        const int k = B.tiles[t].x;
        if (B.st[k].stepping && B.dev[k].geo.R == R) return t;
    }
}

// stage tile t's stencil box (zeros outside the array) into dst and its
// instance's radius-R prediction vectors into dstPv (one commit group)
template <int R>
__device__ __forceinline__ void pass1_stage(const Batch& B, int uin, int t, double* dst, double* dstPv, int tid) {
    using Box = P1Box<R>;
    const int4 tl = B.tiles[t];
    const InstDev& d = B.dev[tl.x];
    const Geo& G = d.geo;
    const double* U = role_ptr(d, B.st[tl.x].parity, uin);
    const int x0 = tl.y - Box::OX, y0 = tl.z - Box::OY;
    for (int e = tid; e < NCONS * Box::SY * (Box::SX / 2); e += NTHREADS) {
        const int v = e / (Box::SY * (Box::SX / 2));
        const int r = e - v * (Box::SY * (Box::SX / 2));
        const int yy = r / (Box::SX / 2), xx = 2 * (r - yy * (Box::SX / 2));
        const int gx = x0 + xx, gy = y0 + yy;
        const bool in = gx >= 0 && gx < G.pitch && gy >= 0 && gy < G.nyt;
        const double* src = in ? U + v * G.plane + (long long)gy * G.pitch + gx : U;
        cp_async16(dst + v * Box::PLANE + yy * Box::SX + xx, src, in ? 16 : 0);
    }
    const double* pv = d.pv + (long long)Box::PVN * (R - 1);  // geo.R == R: nsMax = NS, nqMax = NQ
    for (int e = tid; e < Box::PVN; e += NTHREADS) cp_async8(dstPv + e, pv + e);
    cp_async_commit();
}

// the same staging by TMA: one (x, y, var) box of the stage input's tensor
// map and one bulk copy of the prediction vectors, both completing on `bar`
template <int R>
__device__ __forceinline__ void pass1_stage_tma(const Batch& B, int uin, int t, double* dst, double* dstPv,
                                                uint64_t* bar) {
    using Box = P1Box<R>;
    const int4 tl = B.tiles[t];
    const InstDev& d = B.dev[tl.x];
    const int par = B.st[tl.x].parity;
    const int u = uin == ROLE_STATE ? par : uin == ROLE_A ? 1 - par : 2;  // role_ptr's buffer index
    mbar_expect_tx(bar, (unsigned)((Box::DOUBLES + Box::PVN) * sizeof(double)));
    tma_box3(dst, &d.tmU[u], tl.y - Box::OX, tl.z - Box::OY, 0, bar);
    bulk_copy(dstPv, d.pv + (long long)Box::PVN * (R - 1), (unsigned)(Box::PVN * sizeof(double)), bar);
}

// One launch per radius: blocks skip tiles of instances with another GP
// radius.  Shared memory: NBUF stencil boxes with their prediction vectors,
// the per-thread flux accumulators and, with TMA staging, the boxes'
// mbarriers.  TMA = false stages with per-thread cp.async copies.
//
// MINB is the number of resident blocks per SM the register budget aims at
// (launch bounds: 128 registers at 2, 80 at 3, 64 at 4).  With two boxes the
// next tile's box loads while the current one is computed; with one box a
// block loads, computes, then loads the next, and relies on the other
// resident blocks to hide the load.  One box takes 36 KB less shared memory
// per block, which the SM gives to L1, where the kernel's register spills
// live: at two blocks per SM that wins over double-buffering on the 2048^2
// workloads.  Three or four blocks per SM keep one box (their shared memory
// would not fit two).
template <int R>
struct P1Smem {  // dynamic shared memory layout (doubles): boxes, accumulators, prediction vectors, mbarriers
    static constexpr int box(int nbuf) { return nbuf * P1Box<R>::DOUBLES; }
    static constexpr int bytes(int nbuf) {
        return (nbuf * P1Box<R>::DOUBLES + NCONS * NTHREADS + nbuf * P1Box<R>::PVN) * (int)sizeof(double) + 2 * 8;
    }
};
template <int R, bool TMA, bool DYN, int MINB, int NBUF>
__global__ void __launch_bounds__(NTHREADS, MINB) k_face_pass1(Batch B, int uin) { PDL_ENTRY();
    static_assert(NBUF == 1 || NBUF == 2, "one or two stencil boxes");
    extern __shared__ __align__(128) double smem[];
    __shared__ int sTile;  // the dynamic schedule's tile, as thread 0 took it
    using Box = P1Box<R>;
    const int tid = threadIdx.y * TILE_X + threadIdx.x;
    double* acc = smem + P1Smem<R>::box(NBUF) + tid;
    double* pvBuf = smem + P1Smem<R>::box(NBUF) + NCONS * NTHREADS;  // NBUF prediction-vector buffers
    uint64_t* bars = reinterpret_cast<uint64_t*>(pvBuf + NBUF * Box::PVN);
    if (!(B.flags->radii & (1 << R))) return;  // no instance of this radius
    if (TMA) {
        if (tid == 0) {
            mbar_init(bars);
            mbar_init(bars + 1);
            mbar_fence_init();
        }
        __syncthreads();
    }
    unsigned phase = 0;  // bit b: parity of buffer b's next completion
    const int n = min(__ldg(B.ntiles), B.p1End);  // the launch covers tiles [p1First, n)
    // the block's next tile: grid-stride (every thread computes it), or
    // taken from the counter by thread 0 and broadcast
    auto next_tile = [&](int after) -> int {
        if (!DYN) return pass1_next<R>(B, after, n);
        __syncthreads();  // every thread has read the previous sTile
        if (tid == 0) sTile = pass1_take<R>(B, n);
        __syncthreads();
        return sTile;
    };
    int t = next_tile(B.p1First + blockIdx.x);
    int buf = 0;
    if constexpr (NBUF == 1) {  // one box: load, compute, next
        while (t < n) {
            if (!TMA) {
                pass1_stage<R>(B, uin, t, smem, pvBuf, tid);
                cp_async_wait<0>();
            } else {
                if (tid == 0) pass1_stage_tma<R>(B, uin, t, smem, pvBuf, bars);
                const bool ok = mbar_wait(bars, phase & 1u);
                phase ^= 1u;
                if (!__syncthreads_and(ok)) {  // a copy that never lands: report it, leave without reading
                    if (tid == 0) atomicExch(&B.flags->error, HOSONO_ETIMEOUT);
                    return;
                }
            }
            __syncthreads();  // tile t's box is in place for every thread
            const Cell c = tile_at(B, t);
            InstState& S = B.st[c.k];
            const InstDev& d = B.dev[c.k];
            if (first_tile_thread(c)) S.cascadeMode = CASCADE_FROM_FACES;
            const bool bad = d.phys.force_hydro ? pass1_tile<R, 1>(d, smem, pvBuf, c, acc)
                                                : pass1_tile<R, 0>(d, smem, pvBuf, c, acc);
            warp_flag(&S.anyFail, bad);
            __syncthreads();  // every read of this box is done before it is refilled
            t = next_tile(t + gridDim.x);
        }
        return;
    }
    if (t < n) {
        if (!TMA)
            pass1_stage<R>(B, uin, t, smem, pvBuf, tid);
        else if (tid == 0)
            pass1_stage_tma<R>(B, uin, t, smem, pvBuf, bars);
    }
    while (t < n) {
        const int tn = next_tile(t + gridDim.x);
        if (!TMA) {
            if (tn < n) {
                pass1_stage<R>(B, uin, tn, smem + (buf ^ 1) * Box::DOUBLES, pvBuf + (buf ^ 1) * Box::PVN, tid);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
        } else {
            if (tn < n && tid == 0)
                pass1_stage_tma<R>(B, uin, tn, smem + (buf ^ 1) * Box::DOUBLES, pvBuf + (buf ^ 1) * Box::PVN,
                                   bars + (buf ^ 1));
            const bool ok = mbar_wait(bars + buf, (phase >> buf) & 1u);
            phase ^= 1u << buf;
            if (!__syncthreads_and(ok)) {
                // a copy that never lands: report it, let the copies in flight
                // finish (bounded), and leave without reading the box
                if (tid == 0) atomicExch(&B.flags->error, HOSONO_ETIMEOUT);
                if (tn < n) mbar_wait(bars + (buf ^ 1), (phase >> (buf ^ 1)) & 1u);
                return;
            }
        }
        __syncthreads();  // tile t's box is in place for every thread
        const double* sU = smem + buf * Box::DOUBLES;
        const double* sPv = pvBuf + buf * Box::PVN;
        const Cell c = tile_at(B, t);
        InstState& S = B.st[c.k];
        const InstDev& d = B.dev[c.k];
        if (first_tile_thread(c)) S.cascadeMode = CASCADE_FROM_FACES;
        // one instance per tile: the branch is uniform over the block
        const bool bad = d.phys.force_hydro ? pass1_tile<R, 1>(d, sU, sPv, c, acc) : pass1_tile<R, 0>(d, sU, sPv, c, acc);
        warp_flag(&S.anyFail, bad);
        __syncthreads();  // every read of this box is done before it is refilled
        buf ^= 1;
        t = tn;
    }
}

constexpr int PASS_END_THREADS = 128;

// (slot, first virtual tile) of every instance with pick(slot) true, in slot
// order, and info = {instances, tiles}: per-thread chunks of slots, a block
// scan of the counts, then each thread writes its chunk.  One block of NT
// threads (thread index tid).
template <int NT, class Pick>
__device__ __forceinline__ void build_ranges(const Batch& B, int tid, Pick pick, int2* range, int* info) {
    __shared__ int sCnt[NT / 32], sTil[NT / 32];
    const int per = (B.maxInst + NT - 1) / NT;
    const int k0 = min(B.maxInst, tid * per), k1 = min(B.maxInst, k0 + per);
    int cnt = 0, til = 0;
    for (int k = k0; k < k1; k++)
        if (pick(k)) {
            cnt++;
            til += B.instTiles[k].y;
        }
    // inclusive scan: within each warp by shuffles, then over the warp totals
    const int lane = tid & 31, wid = tid >> 5;
    int ic = cnt, it = til;
    for (int off = 1; off < 32; off <<= 1) {
        const int a = __shfl_up_sync(0xffffffffu, ic, off), b = __shfl_up_sync(0xffffffffu, it, off);
        if (lane >= off) {
            ic += a;
            it += b;
        }
    }
    if (lane == 31) {
        sCnt[wid] = ic;
        sTil[wid] = it;
    }
    __syncthreads();
    for (int w = 0; w < wid; w++) {
        ic += sCnt[w];
        it += sTil[w];
    }
    int c0 = ic - cnt, t0 = it - til;
    for (int k = k0; k < k1; k++)
        if (pick(k)) {
            range[c0++] = make_int2(k, t0);
            t0 += B.instTiles[k].y;
        }
    if (tid == NT - 1) {
        info[0] = ic;
        info[1] = it;
    }
    __syncthreads();  // sCnt/sTil may be reused by the caller's next call
}

// ======================================================================
// Face cascade (reconstruct.f90:143-171).
// cascade_cond: per instance, whether it entered (or stays in) the cascade;
// sets the batch condition.  Single block, one thread per slot.
template <int NT>
__device__ __forceinline__ void d_cascade_cond(const Batch& B, int tid, cudaGraphConditionalHandle h,
                                               int set_handle) {
    __shared__ int any;
    if (tid == 0) any = 0;
    __syncthreads();
    for (int k = tid; k < B.maxInst; k += NT) {
        InstState& S = B.st[k];
        const int in = (S.stepping && S.stageActive && S.anyFail) ? 1 : 0;
        S.anyFail = 0;
        S.nextIter = in;
        if (in) {
            S.cascaded = 1;
            S.cascadeIters++;
            any = 1;
        }
    }
    __syncthreads();
    build_ranges<NT>(B, tid, [&](int k) { return B.st[k].nextIter != 0; }, B.casRange, B.casInfo);
    if (tid == 0) {
        B.flags->anyFail = any;
        B.L.counts[LIST_NEXT] = 0;  // the next cascade iteration compacts its cells afresh
        if (set_handle) cudaGraphSetConditional(h, any ? 1u : 0u);
    }
}
__global__ void __launch_bounds__(PASS_END_THREADS) k_cascade_cond(Batch B, cudaGraphConditionalHandle h,
                                                                      int set_handle) { PDL_ENTRY();
    d_cascade_cond<PASS_END_THREADS>(B, threadIdx.x, h, set_handle);
}

// the serial lowering loop of reconstruct.f90:146-169 (order independent: a
// cell lowers only its own scheme; every flag write sets): for each failing
// cell in [g-2, g+n+1]^2, gridBlock_lowerOrder (gridBlock.f90:194-235) and
// mark the cross for the next inner pass.  The marks in the reconstruct
// range start the iteration clear: compact_next, their only reader, clears
// each mark of the range as it reads it, in the same iteration.

// gridBlock_lowerOrder (gridBlock.f90:194-235) of cell (i,j) plus the mark of
// its cross for the next inner pass
__device__ __forceinline__ void lower_cell(const InstDev& d, const InstState& S, int i, int j, long long cc) {
    const Geo& G = d.geo;
    int8_t* sch = d.scheme[S.schemeSel];
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
    d.nextPass[cc] = 1;
    d.nextPass[cc + 1] = 1;
    d.nextPass[cc - 1] = 1;
    d.nextPass[cc + G.pitch] = 1;
    d.nextPass[cc - G.pitch] = 1;
    d.innerCount[cc] = (uint8_t)(d.innerCount[cc] + 1);
}

// For each cell of [g-2, g+n+1]^2 that failed (face verdicts of pass 1, or the
// `fail` plane of a re-reconstruction, which is cleared as it is consumed):
// lower it.
__device__ __forceinline__ void t_cascade_lower(const Batch& B, const Cell c) {
    InstState& S = B.st[c.k];
    if (!S.nextIter) return;
    const InstDev& d = B.dev[c.k];
    const Geo& G = d.geo;
    const int g = G.g;
    const int i = c.i, j = c.j;
    bool f = false;
    if (i >= g - 2 && j >= g - 2 && i <= g + G.nx + 1 && j <= g + G.ny + 1) {
        const long long cc = (long long)j * G.pitch + i;
        if (S.cascadeMode == CASCADE_FROM_FACES) {
            f = ((d.failX[cc] & 2) | (d.failX[cc + 1] & 1) | (d.failY[cc] & 2) | (d.failY[cc + G.pitch] & 1)) != 0;
        } else {
            f = d.fail[cc] != 0;
            if (f) d.fail[cc] = 0;
        }
        if (f) lower_cell(d, S, i, j, cc);
    }
    warp_count(&S.nInner, f);
    // the first lowering of a cell in this pass puts it on the list whose
    // translate classes the later-pass flag rebuild brings to one scheme
    const long long cc = (long long)j * G.pitch + i;
    const bool first = f && !(d.detMask[cc] & DM_CASC);
    if (first) d.detMask[cc] |= DM_CASC;
    warp_append(B.L, LIST_CASC, B.L.casc, B.L.cap, first, entry(c.k, cc));
}
__global__ void __launch_bounds__(NTHREADS) k_cascade_lower(Batch B) { PDL_ENTRY();
    FOR_CASCADE_TILES(B, t) t_cascade_lower(B, tile_at(B, t));
}


// Lane groups: list kernels give each item (a cell to re-reconstruct, a face
// to re-flux) a group of GL lanes that split its independent parts (faces x
// quadrature points, or quadrature points), so one item costs the latency of
// one face value instead of a dozen in a row.  The loop runs in whole-warp
// steps so warp collectives see every lane.
// gt, gs: the calling thread's global index and the threads of the launch
// (linear: in a 2D block of 32-wide rows, gt & 31 is still the lane).
#define FOR_GROUPS_G(n, GL, e, sub, act, gt, gs)                                                          \
    for (int wbase_ = ((gt) >> 5) * (32 / (GL)), sub = ((gt) & 31) % (GL), e = wbase_ + ((gt) & 31) / (GL); \
         wbase_ < (n); wbase_ += ((gs) >> 5) * (32 / (GL)), e = wbase_ + ((gt) & 31) / (GL))                 \
        for (bool act = e < (n), once_ = true; once_; once_ = false)
// a 1D launch's global thread index and thread count
#define GT1 ((int)(blockIdx.x * blockDim.x + threadIdx.x))
#define GS1 ((int)(gridDim.x * blockDim.x))

// One cell of an inner pass of reconstruct_faceValsWithGP on 16 lanes: lane
// sub = 4*f + q takes face f at quadrature point q, at rr = min(scheme(c),
// scheme(nbr)) (EDP1), and tests CAD/PAD there.  The radius used per face is
// recorded in rrRec; `fail` is set when any face state is inadmissible (the
// reference's loop stops at the first one; the verdict is the same).
// Returns the cell's verdict on every lane of the group.
constexpr int RECON_GL = 16;
__device__ __forceinline__ bool recon_cell_group(const InstDev& d, const InstState& S, int uin, long long cc,
                                                 int sub, bool act) {
    bool bad = false;
    int i = 0, j = 0;
    if (act) {
        const Geo& G = d.geo;
        j = (int)(cc / G.pitch);
        i = (int)(cc - (long long)j * G.pitch);
        const int8_t* sch = d.scheme[S.schemeSel];
        const int s = sch[cc];
        const int f = sub >> 2, q = sub & 3;
        const long long nb = f == NORTH ? cc + G.pitch : f == SOUTH ? cc - G.pitch : f == EAST ? cc + 1 : cc - 1;
        const int rr = min(s, (int)sch[nb]);
        if (sub == 0) {
            const int rN = min(s, (int)sch[cc + G.pitch]), rS = min(s, (int)sch[cc - G.pitch]);
            const int rE = min(s, (int)sch[cc + 1]), rW = min(s, (int)sch[cc - 1]);
            d.dirty[cc] = 1;
            d.rrRec[cc] = (uint8_t)(rN | (rS << 2) | (rE << 4) | (rW << 6));
        }
        if (rr > 0 && q <= rr) {
            double u[NCONS];
            face_value(d, role_ptr(d, S.parity, uin), rr, i, j, f, q, u);
            bad = !admissible(u[DENS], cons2pres(d.phys, u));
        }
    }
    const unsigned m = __ballot_sync(0xffffffffu, bad);
    const unsigned gm = 0xffffu << ((threadIdx.x & 31) & ~15);
    const bool any = (m & gm) != 0;
    if (act && sub == 0 && any) d.fail[cc] = 1;
    return any;
}

// Inner cascade pass: compact the cells marked in nextPass (dense over the
// tiles of instances in their cascade) ...
__device__ __forceinline__ void t_compact_next(const Batch& B, const Cell c) {
    InstState& S = B.st[c.k];
    if (!S.nextIter) return;
    const InstDev& d = B.dev[c.k];
    const Geo& G = d.geo;
    const int g = G.g;
    if (first_tile_thread(c)) S.cascadeMode = CASCADE_FROM_CELLS;
    bool p = false;
    long long cc = 0;
    if (c.i >= g - 2 && c.j >= g - 2 && c.i <= g + G.nx + 1 && c.j <= g + G.ny + 1) {
        cc = (long long)c.j * G.pitch + c.i;
        p = d.nextPass[cc] != 0;
        if (p) d.nextPass[cc] = 0;  // read and cleared: the next iteration's lowering marks afresh
    }
    warp_append(B.L, LIST_NEXT, B.L.next, B.L.cap, p, entry(c.k, cc));
}
__global__ void __launch_bounds__(NTHREADS) k_compact_next(Batch B) { PDL_ENTRY();
    FOR_CASCADE_TILES(B, t) t_compact_next(B, tile_at(B, t));
}
// ... and re-reconstruct them (list `which`: LIST_NEXT in the cascade,
// LIST_REC at the start of a later MOOD pass)
__device__ __forceinline__ void d_recon_group(const Batch& B, int uin, int which, int gt, int gs) {
    const int2* list = which == LIST_NEXT ? B.L.next : rec_list(B, false);
    const int n = min(B.L.counts[which == LIST_NEXT ? (int)LIST_NEXT : rec_count(B, false)], (int)B.L.cap);
    FOR_GROUPS_G(n, RECON_GL, e, sub, act, gt, gs) {
        int2 it = make_int2(0, 0);
        if (act) it = list[e];
        InstState& S = B.st[it.x];
        const bool bad = recon_cell_group(B.dev[it.x], S, uin, it.y, sub, act);
        if (act && sub == 0 && bad) atomicOr(&S.anyFail, 1);
    }
}
__global__ void __launch_bounds__(256, 2) k_recon_group(Batch B, int uin, int which) { PDL_ENTRY();
    d_recon_group(B, uin, which, GT1, GS1);
}



// After the face cascade of a later MOOD pass: the faces getFluxes_ recomputes
// (x-face (i,j) if recompute(i,j) or (i-1,j), y-face if recompute(i,j) or
// (i,j-1), on [g-1, g+n+1]^2, getFluxes.f90:27-89) and the cells FLICD,
// the update and detect visit (recomputeFLICD on [g, g+n]^2).
__device__ __forceinline__ void t_compact_post(const Batch& B, const Cell c) {
    const InstState& S = B.st[c.k];
    if (!(S.stepping && S.stageActive)) return;
    const InstDev& d = B.dev[c.k];
    const Geo& G = d.geo;
    const int g = G.g;
    bool px = false, py = false, pf = false;
    long long cc = 0;
    if (c.i >= g - 1 && c.j >= g - 1 && c.i <= g + G.nx + 1 && c.j <= g + G.ny + 1) {
        cc = (long long)c.j * G.pitch + c.i;
        const bool r = d.rec[cc] != 0;
        px = r || d.rec[cc - 1] != 0;
        py = r || d.rec[cc - G.pitch] != 0;
        pf = c.i >= g && c.j >= g && c.i <= g + G.nx && c.j <= g + G.ny && d.recF[cc] != 0;
    }
    warp_append(B.L, LIST_FACE, B.L.face, 2 * B.L.cap, px, make_int2(c.k, (int)(2 * cc + XDIR)));
    warp_append(B.L, LIST_FACE, B.L.face, 2 * B.L.cap, py, make_int2(c.k, (int)(2 * cc + YDIR)));
    warp_append(B.L, LIST_RECF, B.L.recF, B.L.cap, pf, entry(c.k, cc));
}
__global__ void __launch_bounds__(NTHREADS) k_compact_post(Batch B) { PDL_ENTRY();
    FOR_ACTIVE_TILES(B, t) t_compact_post(B, tile_at(B, t));
}

// Pass 1 after a face cascade: the faces next to a re-reconstructed cell
// (their pass-1 flux used face values that have since changed).
__device__ __forceinline__ void t_compact_dirty(const Batch& B, const Cell c) {
    const InstState& S = B.st[c.k];
    if (!(S.stepping && S.stageActive && S.cascaded)) return;
    const InstDev& d = B.dev[c.k];
    const Geo& G = d.geo;
    const int g = G.g;
    bool px = false, py = false;
    long long cc = 0;
    if (c.i >= g - 1 && c.j >= g - 1 && c.i <= g + G.nx + 1 && c.j <= g + G.ny + 1) {
        cc = (long long)c.j * G.pitch + c.i;
        const bool r = d.dirty[cc] != 0;
        px = r || d.dirty[cc - 1] != 0;
        py = r || d.dirty[cc - G.pitch] != 0;
    }
    warp_append(B.L, LIST_FACE, B.L.face, 2 * B.L.cap, px, make_int2(c.k, (int)(2 * cc + XDIR)));
    warp_append(B.L, LIST_FACE, B.L.face, 2 * B.L.cap, py, make_int2(c.k, (int)(2 * cc + YDIR)));
}
__global__ void __launch_bounds__(NTHREADS) k_compact_dirty(Batch B) { PDL_ENTRY();
    FOR_TILES(B, t) t_compact_dirty(B, tile_at(B, t));
}

// List kernels walk their list grid-stride in whole-warp steps, so warp
// collectives see every lane.
#define FOR_LIST_G(n, e, act, gt, gs)                                                       \
    for (int base_ = (gt) & ~31, e = base_ + ((gt) & 31); base_ < (n); base_ += (gs), e = base_ + ((gt) & 31)) \
        for (bool act = e < (n), once_ = true; once_; once_ = false)

// ======================================================================
// getFluxes_ (getFluxes.f90:16-90) on flagged faces.  Face values are rebuilt
// from U at the radius each side was last reconstructed with (rrRec); the
// quadrature uses the face's current radius (riemannSolver.f90:23-47).
// getFluxes_ on the face list of a later MOOD pass, 4 lanes per face: lane q
// takes quadrature point q (both face values and the Riemann solve); the
// group's first lane sums w_q * F_q in quadrature order, as
// riemannSolver_getFaceFlux does.
constexpr int FLUX_GL = 4;
__device__ __forceinline__ void d_flux_list(const Batch& B, int uin, int gt, int gs) {
    const int n = min(B.L.counts[LIST_FACE], (int)(2 * B.L.cap));
    FOR_GROUPS_G(n, FLUX_GL, e, sub, act, gt, gs) {
        int2 it = make_int2(0, 0);
        if (act) it = B.L.face[e];
        const InstDev& d = B.dev[it.x];
        const InstState& S = B.st[it.x];
        const Geo& G = d.geo;
        const long long cc = (long long)(it.y >> 1);
        const int dir = it.y & 1;
        double F[NCONS];
#pragma unroll
        for (int v = 0; v < NCONS; v++) F[v] = 0.0;
        int rr = 0;
        if (act) {
            const int j = (int)(cc / G.pitch), i = (int)(cc - (long long)j * G.pitch);
            const long long cn = dir == XDIR ? cc - 1 : cc - G.pitch;
            const int8_t* sch = d.scheme[S.schemeSel];
            rr = min((int)sch[cc], (int)sch[cn]);
            if (sub <= rr) {  // rr == 0: one Riemann solve, on lane 0
                const int fL = dir == XDIR ? EAST : NORTH, fR = dir == XDIR ? WEST : SOUTH;
                const int rrL = (d.rrRec[cn] >> (2 * fL)) & 3;
                const int rrR = (d.rrRec[cc] >> (2 * fR)) & 3;
                const double* U = role_ptr(d, S.parity, uin);
                double uL[NCONS], uR[NCONS];
                face_value(d, U, rrL, dir == XDIR ? i - 1 : i, dir == XDIR ? j : j - 1, fL, sub, uL);
                face_value(d, U, rrR, i, j, fR, sub, uR);
                hllc(d.phys, uL, uR, dir, F);
            }
        }
        const int lane0 = (threadIdx.x & 31) & ~(FLUX_GL - 1);
        double acc[NCONS];
#pragma unroll
        for (int v = 0; v < NCONS; v++) acc[v] = 0.0;
#pragma unroll
        for (int q = 0; q < FLUX_GL; q++) {
            double Fq[NCONS];
#pragma unroll
            for (int v = 0; v < NCONS; v++) Fq[v] = __shfl_sync(0xffffffffu, F[v], lane0 + q);
            if (act && sub == 0 && rr > 0 && q <= rr) {
                const double w = qw_at(d, rr, q);
#pragma unroll
                for (int v = 0; v < NCONS; v++) acc[v] = acc[v] + w * Fq[v];
            }
        }
        if (act && sub == 0) {
            if (rr == 0) {
#pragma unroll
                for (int v = 0; v < NCONS; v++) acc[v] = F[v];
            }
            double* Fo = dir == XDIR ? d.FX : d.FY;
#pragma unroll
            for (int v = 0; v < NCONS; v++) Fo[v * G.plane + cc] = acc[v];
            (dir == XDIR ? d.CTX : d.CTY)[cc] = dir == XDIR ? acc[MAGY] : acc[MAGX];
        }
    }
}
__global__ void __launch_bounds__(256, 2) k_flux_list(Batch B, int uin) { PDL_ENTRY(); d_flux_list(B, uin, GT1, GS1); }

// ======================================================================
// FLICDdivB_fluxCorrections (FLICDdivB.f90:13-70) from fluxRaw: fxy =
// FX(magy), fyx = FY(magx), rows p doubles apart (the instance's planes, or
// a box of them staged in shared memory)
__device__ __forceinline__ double flicd_x_at(const double* fxy, const double* fyx, long long c, long long p) {
    return (2 * fxy[c] + fxy[c + 1] + fxy[c - 1] - fyx[c + p] - fyx[c] - fyx[c - 1] - fyx[c - 1 + p]) / 8.0;
}
__device__ __forceinline__ double flicd_y_at(const double* fxy, const double* fyx, long long c, long long p) {
    return (2 * fyx[c] + fyx[c + p] + fyx[c - p] - fxy[c + 1] - fxy[c] - fxy[c - p] - fxy[c + 1 - p]) / 8.0;
}
__device__ __forceinline__ double flicd_x(const InstDev& d, long long c) {
    const Geo& G = d.geo;
    return flicd_x_at(d.FX + MAGY * G.plane, d.FY + MAGX * G.plane, c, G.pitch);
}
__device__ __forceinline__ double flicd_y(const InstDev& d, long long c) {
    const Geo& G = d.geo;
    return flicd_y_at(d.FX + MAGY * G.plane, d.FY + MAGX * G.plane, c, G.pitch);
}

// detect_ALL (detect.f90:84-213).  Everything but CAD, PAD and the DMP reads
// only the stage input U, so it is the same in every MOOD pass of a stage:
// the pass-1 update kernel evaluates it once per stage into detMask --
//   bit 0: shock1 && shock2 && shock3 (:115-146), bit 1: plateau (:161),
//   bit 2: u2 smoothness accepts (:177-213, option 3) --
// and the per-pass test keeps the reference's order of decisions.


// the per-pass test on the new state un of a cell: its detect terms in
// *mask, the stage input's density at rho[c] (rows p doubles apart)
__device__ __forceinline__ bool detect_cell_at(const Phys& P, const uint8_t* mask, const double* __restrict__ rho,
                                               long long c, long long p, const double un[NCONS]) {
    const double presNew = cons2pres(P, un);
    if (!admissible(un[DENS], presNew)) return true;  // CAD, PAD
    const int m = *mask;
    if (!(m & DM_SHOCK)) return false;
    if (m & DM_PLATEAU) return false;
    const double d1 = rho[c], d2 = rho[c + 1], d3 = rho[c - 1], d4 = rho[c + p], d5 = rho[c - p];
    const double mn = fmin(fmin(fmin(fmin(d1, d2), d3), d4), d5);
    const double mx = fmax(fmax(fmax(fmax(d1, d2), d3), d4), d5);
    const double dn = un[DENS];
    if ((mn <= dn) && (dn <= mx)) return false;  // DMP
    return !(m & DM_SMOOTH);
}

// Per-stage part of detect_ALL on the interior, evaluated once per stage by
// the pass-1 update kernel (it reads only the stage input U).  The primitive
// variables of the tile and a one-cell halo are computed once into shared
// memory.  Called by every thread of the block (it synchronises).
// load(v, gx, gy) gives U(v) of array cell (gx, gy); rho[rc] is the cell's
// stage-input density, rows rp doubles apart (the instance's plane, or a
// staged box).
constexpr int DP_SX = TILE_X + 2, DP_SY = TILE_Y + 2;
template <class LoadU>
__device__ __forceinline__ void detect_prep_tile_t(const InstDev& d, const Cell c, double* sV, LoadU load,
                                                   const double* __restrict__ rho, long long rc, long long rp) {
    const Geo& G = d.geo;
    const Phys& P = d.phys;
    const int x0 = c.i - (int)threadIdx.x - 1, y0 = c.j - (int)threadIdx.y - 1;
    const int tid = threadIdx.y * TILE_X + threadIdx.x;
    __syncthreads();  // the previous tile's reads of sV are done
    for (int e = tid; e < DP_SX * DP_SY; e += TILE_X * TILE_Y) {
        const int ey = e / DP_SX, ex = e - ey * DP_SX;
        const int gx = x0 + ex, gy = y0 + ey;
        double vx = 0.0, vy = 0.0, pr = 1.0, rho = 1.0;
        if (gx >= 0 && gx < G.nxt && gy >= 0 && gy < G.nyt) {
            double u[NCONS], V[NPRIM];
#pragma unroll
            for (int v = 0; v < NCONS; v++) u[v] = load(v, gx, gy);
            cons2prim(P, u, V);
            vx = V[VELX];
            vy = V[VELY];
            pr = V[PRES];
            rho = V[DENS];
        }
        sV[0 * DP_SX * DP_SY + e] = vx;
        sV[1 * DP_SX * DP_SY + e] = vy;
        sV[2 * DP_SX * DP_SY + e] = pr;
        sV[3 * DP_SX * DP_SY + e] = rho;
    }
    __syncthreads();
    const int g = G.g;
    if (!(c.i >= g && c.j >= g && c.i < g + G.nx && c.j < g + G.ny)) return;  // no barrier follows
    const int e = (threadIdx.y + 1) * DP_SX + threadIdx.x + 1;
    const double* svx = sV;
    const double* svy = sV + DP_SX * DP_SY;
    const double* spr = sV + 2 * DP_SX * DP_SY;
    const double* srho = sV + 3 * DP_SX * DP_SY;
    const double dx = G.dx, dy = G.dy;
    double div_vel = (svx[e + 1] - svx[e - 1]) / (2 * dx);
    div_vel = div_vel + (svy[e + DP_SX] - svy[e - DP_SX]) / (2 * dy);
    const bool shock1 = div_vel < -(1.0 * (G.maxdxdy * G.maxdxdy));
    double mach = svx[e] * svx[e] + svy[e] * svy[e];
    mach = srho[e] * mach / (P.gamma * spr[e]);
    mach = sqrt(mach);
    const bool shock2 = mach > 0.2;
    double pg = fabs(spr[e + 1] - spr[e - 1]) / (fmin(spr[e + 1], spr[e - 1]));
    pg = pg + fabs(spr[e + DP_SX] - spr[e - DP_SX]) / (fmin(spr[e + DP_SX], spr[e - DP_SX]));
    const bool shock3 = pg > 10.0 * G.maxdxdy;
    const long long cc = (long long)c.j * G.pitch + c.i;
    int m = 0;
    if (shock1 && shock2 && shock3) {
        m |= DM_SHOCK;
        const long long p = rp;
        const double d1 = rho[rc], d2 = rho[rc + 1], d3 = rho[rc - 1], d4 = rho[rc + p], d5 = rho[rc - p];
        const double mn = fmin(fmin(fmin(fmin(d1, d2), d3), d4), d5);
        const double mx = fmax(fmax(fmax(fmax(d1, d2), d3), d4), d5);
        if (mx - mn < G.mindxdy * G.mindxdy * G.mindxdy) m |= DM_PLATEAU;
        double mnx = 0, mxx = 0, mny = 0, mxy = 0;
        int k = 0;
#pragma unroll
        for (int ii = -1; ii <= 1; ii++) {
#pragma unroll
            for (int jj = -1; jj <= 1; jj++) {
                if (iabs_c(ii) + iabs_c(jj) <= 1) {
                    const long long q = rc + ii + jj * p;
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
        }
        const double mm = G.mindxdy;
        const bool sx1 = (mnx * mxx > -mm);
        const bool sy1 = (mny * mxy > -mm);
        const bool sx2 = (fmax(fabs(mnx), fabs(mxx)) < mm);
        const bool sy2 = (fmax(fabs(mny), fabs(mxy)) < mm);
        const bool sx3 = (fmin(fabs(mnx), fabs(mxx)) >= 0.5 * fmax(fabs(mnx), fabs(mxx)));
        const bool sy3 = (fmin(fabs(mny), fabs(mxy)) >= 0.5 * fmax(fabs(mny), fabs(mxy)));
        if ((sx1 && sx2 && sy1 && sy2) || (sx1 && sx3 && sy1 && sy3)) m |= DM_SMOOTH;
    }
    d.detMask[cc] = (uint8_t)(m | (d.detMask[cc] & DM_CASC));
}
// from the instance's planes
__device__ __forceinline__ void detect_prep_tile(const Batch& B, const InstState& S, int uin, const Cell c,
                                                 double* sV) {
    const InstDev& d = B.dev[c.k];
    const Geo& G = d.geo;
    const double* U = role_ptr(d, S.parity, uin);
    detect_prep_tile_t(
        d, c, sV, [&](int v, int gx, int gy) { return U[v * G.plane + (long long)gy * G.pitch + gx]; },
        U + DENS * G.plane, (long long)c.j * G.pitch + c.i, (long long)G.pitch);
}

// Where a cell's inputs are read: the stage input U around the cell (index
// uc, planes uplane and rows up doubles apart) and fluxRaw FX / FY (index
// fc, planes fplane, rows fp apart) -- the instance's planes, or boxes of
// them staged in shared memory.  Either way the same values in the same
// expressions.
struct CellSrc {
    const double* U;
    long long uc, uplane, up;
    const double* FX;
    const double* FY;
    long long fc, fplane, fp;
};
__device__ __forceinline__ CellSrc global_src(const InstDev& d, const InstState& S, int uin, long long cc) {
    const Geo& G = d.geo;
    return CellSrc{role_ptr(d, S.parity, uin), cc, G.plane, G.pitch, d.FX, d.FY, cc, G.plane, G.pitch};
}

// the unsplit update of timeStep.f90:107-118 and detect_ALL for one interior
// cell cc, given its corrected fluxes and those of its east / north faces
__device__ __forceinline__ bool update_detect_at(const InstDev& d, const InstState& S, int uout, long long cc,
                                                 const CellSrc& src, double ctx, double cty, double ctx_e,
                                                 double cty_n) {
    const Geo& G = d.geo;
    double* Uo = role_ptr(d, S.parity, uout);
    const double dt = S.dt;
    const double dtdx = dt / G.dx, dtdy = dt / G.dy;
    double un[NCONS];
#pragma unroll
    for (int v = 0; v < NCONS; v++) {
        double f0, f1, g0, g1;
        if (v == MAGX) {
            f0 = 0.0;
            f1 = 0.0;
            g0 = cty;
            g1 = cty_n;
        } else if (v == MAGY) {
            f0 = ctx;
            f1 = ctx_e;
            g0 = 0.0;
            g1 = 0.0;
        } else {
            f0 = src.FX[v * src.fplane + src.fc];
            f1 = src.FX[v * src.fplane + src.fc + 1];
            g0 = src.FY[v * src.fplane + src.fc];
            g1 = src.FY[v * src.fplane + src.fc + src.fp];
        }
        un[v] = src.U[v * src.uplane + src.uc] - dtdx * (f1 - f0) - dtdy * (g1 - g0);
        Uo[v * G.plane + cc] = un[v];
    }
    bool low = false;
    if (d.scheme[S.schemeSel][cc] > 0)
        low = detect_cell_at(d.phys, d.detMask + cc, src.U + DENS * src.uplane, src.uc, src.up, un);
    if (low) d.lowered[cc] = 1;
    return low;
}

// FLICD on [g, g+n]^2 where recomputeFLICD; then, on the interior, the
// unsplit update of timeStep.f90:107-118 and detect_ALL.  A corrected flux a
// neighbour needs is recomputed locally when the neighbour is flagged (it
// writes the same value) and read from memory otherwise (nobody writes it).
// A lowered cell sets `lowered` (cleared again after the flags are rebuilt)
// and is appended to the lowered list.
__device__ __forceinline__ bool ct_cell_at(const InstDev& d, const InstState& S, int uout, int i, int j, long long cc,
                                           const CellSrc& src) {
    const Geo& G = d.geo;
    const int g = G.g;
    if (!d.recF[cc]) return false;
    const double* fxy = src.FX + MAGY * src.fplane;
    const double* fyx = src.FY + MAGX * src.fplane;
    const double ctx = flicd_x_at(fxy, fyx, src.fc, src.fp);
    const double cty = flicd_y_at(fxy, fyx, src.fc, src.fp);
    d.CTX[cc] = ctx;
    d.CTY[cc] = cty;
    if (i >= g + G.nx || j >= g + G.ny) return false;  // FLICD-only row and column
    const long long ce = cc + 1, cn = cc + G.pitch;
    const double ctx_e = d.recF[ce] ? flicd_x_at(fxy, fyx, src.fc + 1, src.fp) : d.CTX[ce];
    const double cty_n = d.recF[cn] ? flicd_y_at(fxy, fyx, src.fc + src.fp, src.fp) : d.CTY[cn];
    return update_detect_at(d, S, uout, cc, src, ctx, cty, ctx_e, cty_n);
}
__device__ __forceinline__ bool ct_cell(const InstDev& d, const InstState& S, int uin, int uout, int i, int j,
                                        long long cc) {
    return ct_cell_at(d, S, uout, i, j, cc, global_src(d, S, uin, cc));
}

__device__ __forceinline__ void t_ct_update_detect(const Batch& B, int uin, int uout, const Cell c, double* sV) {
    InstState& S = B.st[c.k];
    if (!(S.stepping && S.stageActive)) return;  // uniform over the block
    detect_prep_tile(B, S, uin, c, sV);
    const InstDev& d = B.dev[c.k];
    const Geo& G = d.geo;
    const int g = G.g;
    bool low = false;
    long long cc = 0;
    if (c.i >= g && c.j >= g && c.i <= g + G.nx && c.j <= g + G.ny) {
        cc = (long long)c.j * G.pitch + c.i;
        low = ct_cell(d, S, uin, uout, c.i, c.j, cc);
    }
    warp_count(&S.nDetect, low);
    warp_append(B.L, LIST_LOW, B.L.low, B.L.cap, low, entry(c.k, cc));
}
// six resident blocks (a 40-register budget, a few hundred bytes of spills):
// the tile's loads wait at two barriers, so more warps in flight keep HBM
// busier.  Per step on Orszag-Tang 2048^2: 3 blocks (80 registers) 11.66 ms,
// 4 blocks 11.23 ms, 5 blocks 11.14 ms, 6 blocks 11.08 ms.  Computing each
// cell's corrected fluxes once into shared memory (instead of a cell also
// evaluating its east and north neighbours' FLICD) made a launch about 5 %
// slower: the extra barrier costs more than the loads it saves, which hit L1.
__global__ void __launch_bounds__(NTHREADS, 6) k_ct_update_detect(Batch B, int uin, int uout) { PDL_ENTRY();
    __shared__ double sV[4 * DP_SX * DP_SY];
    FOR_TILES(B, t) t_ct_update_detect(B, uin, uout, tile_at(B, t), sV);
}

// The same with the tile's inputs staged by TMA: one copy each of the
// stage input U over [x0-4, x0+36) x [y0-2, y0+10) and of fluxRaw FX and FY
// over [x0-4, x0+36) x [y0-1, y0+10), all 8 planes, completing on one
// mbarrier (zero fill outside the array; the x origin x0 - 4 is a multiple of
// 4 doubles), then the per-stage detect terms, FLICD, the update and detect
// read shared memory.  The boxes replace the dependent load chains of the
// cached version by three bulk copies per tile; two blocks per SM, so one
// block's copies overlap the other's arithmetic.  This GPU's own memory
// only, no multicast.  Waits are bounded as in pass 1 (HOSONO_ETIMEOUT).
constexpr int CT_UPL = CT_SX * CT_UY, CT_FPL = CT_SX * CT_FY;
constexpr int CT_SMEM_BYTES = (NCONS * CT_UPL + 2 * NCONS * CT_FPL + 4 * DP_SX * DP_SY) * (int)sizeof(double) + 16;
__global__ void __launch_bounds__(NTHREADS, 2) k_ct_update_detect_tma(Batch B, int uin, int uout) { PDL_ENTRY();
    extern __shared__ __align__(128) double smem[];
    double* sU = smem;
    double* sFX = sU + NCONS * CT_UPL;
    double* sFY = sFX + NCONS * CT_FPL;
    double* sV = sFY + NCONS * CT_FPL;
    uint64_t* bar = reinterpret_cast<uint64_t*>(sV + 4 * DP_SX * DP_SY);
    const int tid = threadIdx.y * TILE_X + threadIdx.x;
    if (tid == 0) {
        mbar_init(bar);
        mbar_fence_init();
    }
    __syncthreads();
    unsigned phase = 0;
    FOR_TILES(B, t) {
        const Cell c = tile_at(B, t);
        InstState& S = B.st[c.k];
        if (!(S.stepping && S.stageActive)) continue;  // uniform over the block
        const InstDev& d = B.dev[c.k];
        const Geo& G = d.geo;
        const int x0 = c.i - (int)threadIdx.x, y0 = c.j - (int)threadIdx.y;  // the tile's origin
        const int ux0 = x0 - 4, uy0 = y0 - 2, fy0 = y0 - 1;              // the boxes' origins
        __syncthreads();  // every read of the previous tile's boxes is done
        if (tid == 0) {
            const int par = S.parity;
            const int u = uin == ROLE_STATE ? par : uin == ROLE_A ? 1 - par : 2;  // role_ptr's buffer index
            mbar_expect_tx(bar, (unsigned)((NCONS * CT_UPL + 2 * NCONS * CT_FPL) * sizeof(double)));
            tma_box3(sU, &d.tmCU[u], ux0, uy0, 0, bar);
            tma_box3(sFX, &d.tmFX, ux0, fy0, 0, bar);
            tma_box3(sFY, &d.tmFY, ux0, fy0, 0, bar);
        }
        const bool ok = mbar_wait(bar, phase & 1u);
        phase ^= 1u;
        if (!__syncthreads_and(ok)) {  // a copy that never lands: report it, leave without reading
            if (tid == 0) atomicExch(&B.flags->error, HOSONO_ETIMEOUT);
            return;
        }
        detect_prep_tile_t(
            d, c, sV, [&](int v, int gx, int gy) { return sU[v * CT_UPL + (gy - uy0) * CT_SX + (gx - ux0)]; },
            sU + DENS * CT_UPL, (long long)(c.j - uy0) * CT_SX + (c.i - ux0), (long long)CT_SX);
        const int g = G.g;
        bool low = false;
        long long cc = 0;
        if (c.i >= g && c.j >= g && c.i <= g + G.nx && c.j <= g + G.ny) {
            cc = (long long)c.j * G.pitch + c.i;
            const CellSrc src{sU,  (long long)(c.j - uy0) * CT_SX + (c.i - ux0), CT_UPL, CT_SX,
                              sFX, sFY, (long long)(c.j - fy0) * CT_SX + (c.i - ux0), CT_FPL, CT_SX};
            low = ct_cell_at(d, S, uout, c.i, c.j, cc, src);
        }
        warp_count(&S.nDetect, low);
        warp_append(B.L, LIST_LOW, B.L.low, B.L.cap, low, entry(c.k, cc));
    }
}

// the same on the recomputeFLICD list of a later MOOD pass
__device__ __forceinline__ void d_ct_list(const Batch& B, int uin, int uout, int gt, int gs) {
    const int n = min(B.L.counts[LIST_RECF], (int)B.L.cap);
    FOR_LIST_G(n, e, act, gt, gs) {
        bool low = false;
        int2 it = make_int2(0, 0);
        if (act) {
            it = B.L.recF[e];
            InstState& S = B.st[it.x];
            const InstDev& d = B.dev[it.x];
            const long long cc = it.y;
            const int j = (int)(cc / d.geo.pitch), i = (int)(cc - (long long)j * d.geo.pitch);
            low = ct_cell(d, S, uin, uout, i, j, cc);
            if (low) atomicAdd(&S.nDetect, 1);
        }
        warp_append(B.L, LIST_LOW, B.L.low, B.L.cap, low, it);
    }
}
__global__ void __launch_bounds__(256) k_ct_list(Batch B, int uin, int uout) { PDL_ENTRY(); d_ct_list(B, uin, uout, GT1, GS1); }

// `lowered` back to zero on the cells this pass lowered
__device__ __forceinline__ void d_clear_low(const Batch& B, int gt, int gs) {
    const int n = min(B.L.counts[LIST_LOW], (int)B.L.cap);
    for (int e = gt; e < n; e += gs) {
        const int2 it = B.L.low[e];
        B.dev[it.x].lowered[it.y] = 0;
    }
}
__global__ void __launch_bounds__(256) k_clear_low(Batch B) { PDL_ENTRY(); d_clear_low(B, GT1, GS1); }

// ======================================================================
// After detect: recompute = cross of lowered cells, recomputeFLICD = radius-2
// diamond (gridBlock_lowerOrder), scheme lowered by one where lowered; then
// boundaryConditions_applyMOOD's periodic sync, which (x sweep over all rows,
// then y sweep over all columns, N >= 2*NGC) makes every cell the OR (flags) /
// MIN (scheme) over its translates by multiples of N that lie in the array.
// one cell of the dense rebuild; returns its new recompute flag
__device__ __forceinline__ bool mood_flags_cell(const InstDev& d, const InstState& S, int i, int j) {
    const Geo& G = d.geo;
    const int8_t* sch = d.scheme[S.schemeSel];
    int8_t* schN = d.scheme[1 - S.schemeSel];
    const int reach = G.bc == 1 ? 1 : 0;
    bool rec = false, recF = false;
    int s = 127;
    for (int b = -reach; b <= reach; b++) {
        const int jo = j + b * G.ny;
        if (jo < 0 || jo >= G.nyt) continue;
        for (int t = -reach; t <= reach; t++) {
            const int io = i + t * G.nx;
            if (io < 0 || io >= G.nxt) continue;
            const long long co = (long long)jo * G.pitch + io;
            const int lo = d.lowered[co];
            const int so = sch[co] - lo;
            s = min(s, so > 0 ? so : 0);
            for (int dj = -2; dj <= 2; dj++) {
                const int jj = jo + dj;
                if (jj < 0 || jj >= G.nyt) continue;
                for (int di = -2; di <= 2; di++) {
                    const int dd = iabs_c(di) + iabs_c(dj);
                    const int ii = io + di;
                    if (dd > 2 || ii < 0 || ii >= G.nxt) continue;
                    if (d.lowered[(long long)jj * G.pitch + ii]) {
                        recF = true;
                        if (dd <= 1) rec = true;
                    }
                }
            }
        }
    }
    const long long cc = (long long)j * G.pitch + i;
    d.rec[cc] = rec;
    d.recF[cc] = recF;
    schN[cc] = (int8_t)s;
    d.detMask[cc] &= (uint8_t)~DM_CASC;
    return rec;
}
// An instance whose pass lowered no cell (neither the face cascade nor
// detect) keeps its scheme, and its MOOD loop ends here: the rebuild is
// skipped, and pass_end leaves its scheme buffer where it is.
__device__ __forceinline__ bool pass_lowered(const InstState& S) { return S.nInner != 0 || S.nDetect != 0; }
__device__ __forceinline__ void t_mood_flags(const Batch& B, const Cell c) {
    const InstState& S = B.st[c.k];
    if (!(S.stepping && S.stageActive) || !pass_lowered(S)) return;
    const InstDev& d = B.dev[c.k];
    const Geo& G = d.geo;
    const int i = c.i, j = c.j;
    const bool inArr = i < G.nxt && j < G.nyt;
    const int g = G.g;
    const bool inRec = inArr && i >= g - 2 && j >= g - 2 && i <= g + G.nx + 1 && j <= g + G.ny + 1;
    const bool newRec = inArr && mood_flags_cell(d, S, i, j);
    // the next pass's recompute list (reconstruct range, reconstruct.f90:83)
    warp_append(B.L, rec_count(B, true), rec_list(B, true), B.L.cap, newRec && inRec,
                entry(c.k, (long long)j * G.pitch + i));
}
// eight resident blocks (32 registers): a latency-bound byte-gather over the
// lowered flags, faster with more warps in flight
__global__ void __launch_bounds__(NTHREADS, 8) k_mood_flags(Batch B) { PDL_ENTRY();
    FOR_TILES(B, t) t_mood_flags(B, tile_at(B, t));
}

// The same result from the work lists in a later MOOD pass, where few cells
// change.  The flags read later (recompute on [g-2, g+n+1]^2, recomputeFLICD
// on [g, g+n]^2) can only be set on cells of this pass's lists -- recompute:
// the pass's starting list, both cells of each re-fluxed face, the cross of
// each cascade lowering; recomputeFLICD: its list -- so clear those, then set
// the cross / diamond of every translate of each cell detect lowered.  The scheme changes only on the translate classes of
// cells lowered in this pass (by detect or by the inner cascade, which does
// not sync): each takes min over its class of (scheme - lowered)^+, computed
// for every listed cell first and written afterwards (two kernels), so no
// class member is read after it was written.
// recompute := 1; the first setter of a cell in the reconstruct range puts
// it on the next pass's list (the byte is set through its 32-bit word so
// that exactly one thread sees it change)
__device__ __forceinline__ void set_rec(const Batch& B, const InstDev& d, long long cn, int ii, int jj, int k) {
    const unsigned sh = 8u * (unsigned)(cn & 3);
    unsigned* w = reinterpret_cast<unsigned*>(d.rec + (cn - (cn & 3)));
    const unsigned old = atomicOr(w, 1u << sh);
    const Geo& G = d.geo;
    const int g = G.g;
    if (((old >> sh) & 0xffu) == 0 && ii >= g - 2 && jj >= g - 2 && ii <= g + G.nx + 1 && jj <= g + G.ny + 1) {
        const int pos = atomicAdd(B.L.counts + rec_count(B, true), 1);
        if (pos < B.L.cap)
            rec_list(B, true)[pos] = entry(k, cn);
        else
            B.L.counts[LIST_OVERFLOW] = 1;
    }
}
__device__ __forceinline__ void sync_cell(const Batch& B, int e, int nLow, int2* it_out, bool* from_low) {
    *from_low = e < nLow;
    *it_out = *from_low ? B.L.low[e] : B.L.casc[e - nLow];
}
__device__ __forceinline__ void d_flags_clear(const Batch& B, int gt, int gs) {
    const int nF = min(B.L.counts[LIST_FACE], (int)(2 * B.L.cap));
    const int nR = min(B.L.counts[LIST_RECF], (int)B.L.cap);
    const int nP = min(B.L.counts[rec_count(B, false)], (int)B.L.cap);
    const int2* recCur = rec_list(B, false);
    const int nC = min(B.L.counts[LIST_CASC], (int)B.L.cap);
    for (int e = gt; e < nF + nR + nP + nC; e += gs) {
        if (e < nF) {  // both cells of a re-fluxed face
            const int2 it = B.L.face[e];
            const InstDev& d = B.dev[it.x];
            const long long cc = (long long)(it.y >> 1);
            d.rec[cc] = 0;
            d.rec[(it.y & 1) == XDIR ? cc - 1 : cc - d.geo.pitch] = 0;
        } else if (e < nF + nR) {
            const int2 it = B.L.recF[e - nF];
            B.dev[it.x].recF[it.y] = 0;
        } else if (e < nF + nR + nP) {  // recompute at the start of the pass
            const int2 it = recCur[e - nF - nR];
            B.dev[it.x].rec[it.y] = 0;
        } else {  // the cross a cascade lowering marked
            const int2 it = B.L.casc[e - nF - nR - nP];
            const InstDev& d = B.dev[it.x];
            const long long cc = it.y, p = d.geo.pitch;
            d.rec[cc] = 0;
            d.rec[cc + 1] = 0;
            d.rec[cc - 1] = 0;
            d.rec[cc + p] = 0;
            d.rec[cc - p] = 0;
        }
    }
}
__global__ void __launch_bounds__(256) k_flags_clear(Batch B) { PDL_ENTRY(); d_flags_clear(B, GT1, GS1); }
__device__ __forceinline__ void d_flags_scatter(const Batch& B, int gt, int gs) {
    const int nL = min(B.L.counts[LIST_LOW], (int)B.L.cap);
    const int nC = min(B.L.counts[LIST_CASC], (int)B.L.cap);
    for (int e = gt; e < nL + nC; e += gs) {
        int2 it;
        bool fromLow;
        sync_cell(B, e, nL, &it, &fromLow);
        const InstDev& d = B.dev[it.x];
        const InstState& S = B.st[it.x];
        const Geo& G = d.geo;
        const int8_t* sch = d.scheme[S.schemeSel];
        const long long c0 = it.y;
        const int j0 = (int)(c0 / G.pitch), i0 = (int)(c0 - (long long)j0 * G.pitch);
        const int reach = G.bc == 1 ? 1 : 0;
        int s = 127;
        for (int b = -reach; b <= reach; b++) {
            const int jo = j0 + b * G.ny;
            if (jo < 0 || jo >= G.nyt) continue;
            for (int t = -reach; t <= reach; t++) {
                const int io = i0 + t * G.nx;
                if (io < 0 || io >= G.nxt) continue;
                const long long co = (long long)jo * G.pitch + io;
                const int so = sch[co] - d.lowered[co];
                s = min(s, so > 0 ? so : 0);
                if (!fromLow) continue;
                for (int dj = -2; dj <= 2; dj++) {
                    const int jj = jo + dj;
                    if (jj < 0 || jj >= G.nyt) continue;
                    for (int di = -2; di <= 2; di++) {
                        const int dd = iabs_c(di) + iabs_c(dj);
                        const int ii = io + di;
                        if (dd > 2 || ii < 0 || ii >= G.nxt) continue;
                        const long long cn = (long long)jj * G.pitch + ii;
                        d.recF[cn] = 1;
                        if (dd <= 1) set_rec(B, d, cn, ii, jj, it.x);
                    }
                }
            }
        }
        B.L.sync[e] = (int8_t)s;
    }
}
__global__ void __launch_bounds__(256) k_flags_scatter(Batch B) { PDL_ENTRY(); d_flags_scatter(B, GT1, GS1); }
__device__ __forceinline__ void d_scheme_sync(const Batch& B, int clear_low, int gt, int gs) {
    const int nL = min(B.L.counts[LIST_LOW], (int)B.L.cap);
    const int nC = min(B.L.counts[LIST_CASC], (int)B.L.cap);
    for (int e = gt; e < nL + nC; e += gs) {
        int2 it;
        bool fromLow;
        sync_cell(B, e, nL, &it, &fromLow);
        const InstDev& d = B.dev[it.x];
        const Geo& G = d.geo;
        int8_t* sch = d.scheme[B.st[it.x].schemeSel];
        const long long c0 = it.y;
        const int j0 = (int)(c0 / G.pitch), i0 = (int)(c0 - (long long)j0 * G.pitch);
        const int reach = G.bc == 1 ? 1 : 0;
        const int8_t s = B.L.sync[e];
        for (int b = -reach; b <= reach; b++) {
            const int jo = j0 + b * G.ny;
            if (jo < 0 || jo >= G.nyt) continue;
            for (int t = -reach; t <= reach; t++) {
                const int io = i0 + t * G.nx;
                if (io < 0 || io >= G.nxt) continue;
                sch[(long long)jo * G.pitch + io] = s;
            }
        }
        if (!fromLow) d.detMask[c0] &= (uint8_t)~DM_CASC;
        if (fromLow && clear_low) d.lowered[c0] = 0;  // k_flags_scatter has read it
    }
}
__global__ void __launch_bounds__(256) k_scheme_sync(Batch B, int clear_low) { PDL_ENTRY();
    d_scheme_sync(B, clear_low, GT1, GS1);
}

// End of a MOOD pass (timeStep.f90:86-128 loop test): an instance whose detect
// lowered nothing leaves the loop.  Single block, one thread per slot.
template <int NT>
__device__ __forceinline__ void d_pass_end(const Batch& B, int tid, cudaGraphConditionalHandle h, int set_handle,
                                           int flip) {
    __shared__ int any;
    if (tid == 0) any = 0;
    __syncthreads();
    for (int k = tid; k < B.maxInst; k += NT) {
        InstState& S = B.st[k];
        if (!(S.stepping && S.stageActive)) continue;
        if (flip && pass_lowered(S)) S.schemeSel = 1 - S.schemeSel;  // k_mood_flags wrote the other buffer
        S.passes++;
        S.passesTotal++;
        S.innerTotal += S.nInner;
        S.detectTotal += S.nDetect;
        S.lastInner = S.nInner;
        S.lastDetect = S.nDetect;
        if (S.nDetect == 0) {
            S.stageActive = 0;
            if (S.passes > S.maxPasses) S.maxPasses = S.passes;
        } else if (S.passes >= S.passCap) {
            S.stageActive = 0;
            S.stepping = 0;
            S.done = 1;
            S.error = HOSONO_EMOODCAP;
        } else {
            any = 1;
            S.cascadeMode = CASCADE_FROM_CELLS;  // later passes' cascades start from re-reconstructions
        }
        S.nInner = 0;
        S.nDetect = 0;
        S.cascaded = 0;
    }
    __syncthreads();
    // the instances still in their MOOD loop and their tiles, for the dense
    // kernels of the next pass
    build_ranges<NT>(B, tid, [&](int k) { return B.st[k].stepping && B.st[k].stageActive; }, B.actRange, B.actInfo);
    if (tid == 0) {
        B.flags->anyActive = any;
        if (B.L.counts[LIST_OVERFLOW]) B.flags->error = HOSONO_EINVAL;
        // the next pass reads the recompute list the flag rebuild just filled
        // and builds every other list afresh
        const int cur = B.flags->recSel ^ 1;
        B.flags->recSel = cur;
        for (int w = 0; w < LIST_N; w++)
            if (w != (cur ? LIST_REC2 : LIST_REC)) B.L.counts[w] = 0;
        if (set_handle) cudaGraphSetConditional(h, any ? 1u : 0u);
    }
}
__global__ void __launch_bounds__(PASS_END_THREADS) k_pass_end(Batch B, cudaGraphConditionalHandle h, int set_handle,
                                                                int flip) { PDL_ENTRY();
    d_pass_end<PASS_END_THREADS>(B, threadIdx.x, h, set_handle, flip);
}

// timeStep_forwardEuler's reset (timeStep.f90:79-81) on every cell:
// scheme = R, recompute = recomputeFLICD = .true.; plus the per-instance
// stage scalars.
__device__ __forceinline__ void t_stage_init(const Batch& B, const Cell c) {
    InstState& S = B.st[c.k];
    if (!S.stepping) return;
    const InstDev& d = B.dev[c.k];
    const Geo& G = d.geo;
    if (first_tile_thread(c)) {
        S.stageActive = 1;
        S.passes = 0;
        S.nInner = 0;
        S.nDetect = 0;
        S.anyFail = 0;
        S.cascaded = 0;
        S.stages++;
    }
    if (c.i >= G.nxt || c.j >= G.nyt) return;
    const long long cc = (long long)c.j * G.pitch + c.i;
    const int R = G.R;
    d.scheme[S.schemeSel][cc] = (int8_t)R;
    d.rec[cc] = 1;
    d.recF[cc] = 1;
    d.rrRec[cc] = (uint8_t)(R | (R << 2) | (R << 4) | (R << 6));
    d.dirty[cc] = 0;
    d.innerCount[cc] = 0;
}
__global__ void __launch_bounds__(NTHREADS) k_stage_init(Batch B) { PDL_ENTRY();
    if (blockIdx.x == 0 && threadIdx.x == 0 && threadIdx.y == 0) {  // the recompute lists start empty
        B.L.counts[LIST_REC] = 0;
        B.L.counts[LIST_REC2] = 0;
        for (int r = 0; r < 4; r++) B.flags->p1Next[r] = 0;  // pass 1's dynamic schedule starts over
        B.gbar[0] = 0;  // the persistent later-pass launch's barrier count (after an aborted launch too)
    }
    FOR_TILES(B, t) t_stage_init(B, tile_at(B, t));
}

// ======================================================================
// boundary conditions (boundaryConditions.f90:79-187) as a gather
__device__ __forceinline__ int bc_src(int i, int n, int g, int bc) {
    if (i < g) return bc == 1 ? i + n : g;
    if (i >= g + n) return bc == 1 ? i - n : g + n - 1;
    return i;
}

__device__ __forceinline__ void t_bc_fill(const Batch& B, int role, const Cell c) {
    const InstState& S = B.st[c.k];
    if (!S.stepping) return;
    const InstDev& d = B.dev[c.k];
    const Geo& G = d.geo;
    if (c.i >= G.nxt || c.j >= G.nyt) return;
    const int si = bc_src(c.i, G.nx, G.g, G.bc), sj = bc_src(c.j, G.ny, G.g, G.bc);
    if (si == c.i && sj == c.j) return;
    double* A = role_ptr(d, S.parity, role);
    const long long cc = (long long)c.j * G.pitch + c.i, s = (long long)sj * G.pitch + si;
#pragma unroll
    for (int v = 0; v < NCONS; v++) A[v * G.plane + cc] = A[v * G.plane + s];
}
__global__ void __launch_bounds__(NTHREADS) k_bc_fill(Batch B, int role) { PDL_ENTRY();
    FOR_TILES(B, t) t_bc_fill(B, role, tile_at(B, t));
}

// timeStep.f90:165-166 over every cell (guards from their images): A = (3 U + B)/4
__device__ __forceinline__ void t_rk_combine2(const Batch& B, const Cell c) {
    const InstState& S = B.st[c.k];
    if (!S.stepping) return;
    const InstDev& d = B.dev[c.k];
    const Geo& G = d.geo;
    if (c.i >= G.nxt || c.j >= G.nyt) return;
    const int si = bc_src(c.i, G.nx, G.g, G.bc), sj = bc_src(c.j, G.ny, G.g, G.bc);
    const long long cc = (long long)c.j * G.pitch + c.i, s = (long long)sj * G.pitch + si;
    const double* Un = role_ptr(d, S.parity, ROLE_STATE);
    const double* Bb = role_ptr(d, S.parity, ROLE_B);
    double* out = role_ptr(d, S.parity, ROLE_A);
#pragma unroll
    for (int v = 0; v < NCONS; v++) out[v * G.plane + cc] = (3 * Un[v * G.plane + s] + Bb[v * G.plane + s]) / 4.0;
}
__global__ void __launch_bounds__(NTHREADS) k_rk_combine2(Batch B) { PDL_ENTRY();
    FOR_TILES(B, t) t_rk_combine2(B, tile_at(B, t));
}

// timeStep.f90:169 and :32-41: A = (U + 2 B)/3, V = cons2prim(A), on every
// cell (guards from their images).  step_end makes A the state.
__device__ __forceinline__ void t_rk_final(const Batch& B, const Cell c) {
    const InstState& S = B.st[c.k];
    if (!S.stepping) return;
    const InstDev& d = B.dev[c.k];
    const Geo& G = d.geo;
    if (c.i >= G.nxt || c.j >= G.nyt) return;
    const int si = bc_src(c.i, G.nx, G.g, G.bc), sj = bc_src(c.j, G.ny, G.g, G.bc);
    const long long cc = (long long)c.j * G.pitch + c.i, s = (long long)sj * G.pitch + si;
    const double* Un = role_ptr(d, S.parity, ROLE_STATE);
    const double* Bb = role_ptr(d, S.parity, ROLE_B);
    double* out = role_ptr(d, S.parity, ROLE_A);
    double u[NCONS], V[NPRIM];
#pragma unroll
    for (int v = 0; v < NCONS; v++) {
        u[v] = (Un[v * G.plane + s] + 2 * Bb[v * G.plane + s]) / 3.0;
        out[v * G.plane + cc] = u[v];
    }
    cons2prim(d.phys, u, V);
#pragma unroll
    for (int v = 0; v < NPRIM; v++) d.V[v * G.plane + cc] = V[v];
}
// six resident blocks (40 registers) for more loads in flight
__global__ void __launch_bounds__(NTHREADS, 6) k_rk_final(Batch B) { PDL_ENTRY();
    FOR_TILES(B, t) t_rk_final(B, tile_at(B, t));
}

// V = cons2prim(state) on every cell (upload without V)
__device__ __forceinline__ void t_cons2prim_all(const Batch& B, const Cell c) {
    const InstState& S = B.st[c.k];
    if (!S.stepping) return;
    const InstDev& d = B.dev[c.k];
    const Geo& G = d.geo;
    if (c.i >= G.nxt || c.j >= G.nyt) return;
    const long long cc = (long long)c.j * G.pitch + c.i;
    const double* U = role_ptr(d, S.parity, ROLE_STATE);
    double u[NCONS], w[NPRIM];
#pragma unroll
    for (int v = 0; v < NCONS; v++) u[v] = U[v * G.plane + cc];
    cons2prim(d.phys, u, w);
#pragma unroll
    for (int v = 0; v < NPRIM; v++) d.V[v * G.plane + cc] = w[v];
}
__global__ void __launch_bounds__(NTHREADS) k_cons2prim_all(Batch B) { PDL_ENTRY();
    FOR_TILES(B, t) t_cons2prim_all(B, tile_at(B, t));
}

// ======================================================================
// cfl_computedt (cfl.f90:14-52): per instance, max of |u|+c and |v|+c over the
// interior.  Non-negative doubles order like their bit patterns, so block
// maxima are combined with an integer atomicMax.
__device__ __forceinline__ void t_cfl_reduce(const Batch& B, const Cell c) {
    InstState& S = B.st[c.k];
    if (!S.stepping) return;
    const InstDev& d = B.dev[c.k];
    const Geo& G = d.geo;
    double xm = 0.0, ym = 0.0;
    if (c.i >= G.g && c.j >= G.g && c.i < G.g + G.nx && c.j < G.g + G.ny) {
        const long long cc = (long long)c.j * G.pitch + c.i;
        const double* V = d.V;
        const double rho = V[DENS * G.plane + cc], pr = V[PRES * G.plane + cc], gam = V[GAMM * G.plane + cc];
        double cs;
        if (d.phys.force_hydro) {
            cs = sqrt(gam * pr / rho);
        } else {
            const double bx = V[MAGX * G.plane + cc], by = V[MAGY * G.plane + cc], bz = V[MAGZ * G.plane + cc];
            const double BB = bx * bx + by * by + bz * bz;
            const double bmin = fmin(fmin(fabs(bx), fabs(by)), fabs(bz));
            cs = c_fs(gam, rho, pr, BB, bmin, +1.0);
        }
        xm = fabs(V[VELX * G.plane + cc]) + cs;
        ym = fabs(V[VELY * G.plane + cc]) + cs;
    }
    for (int o = 16; o > 0; o >>= 1) {
        xm = fmax(xm, __shfl_xor_sync(0xffffffffu, xm, o));
        ym = fmax(ym, __shfl_xor_sync(0xffffffffu, ym, o));
    }
    __shared__ double sx[NTHREADS / 32], sy[NTHREADS / 32];
    const int lane = (threadIdx.y * TILE_X + threadIdx.x) & 31, w = (threadIdx.y * TILE_X + threadIdx.x) >> 5;
    if (lane == 0) {
        sx[w] = xm;
        sy[w] = ym;
    }
    __syncthreads();
    if (w == 0) {
        xm = lane < NTHREADS / 32 ? sx[lane] : 0.0;
        ym = lane < NTHREADS / 32 ? sy[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            xm = fmax(xm, __shfl_xor_sync(0xffffffffu, xm, o));
            ym = fmax(ym, __shfl_xor_sync(0xffffffffu, ym, o));
        }
        if (lane == 0) {
            atomicMax(&S.cflbits[0], (unsigned long long)__double_as_longlong(xm));
            atomicMax(&S.cflbits[1], (unsigned long long)__double_as_longlong(ym));
        }
    }
    __syncthreads();  // sx/sy are reused by the block's next tile
}
__global__ void __launch_bounds__(NTHREADS) k_cfl_reduce(Batch B) { PDL_ENTRY();
    FOR_TILES(B, t) t_cfl_reduce(B, tile_at(B, t));
}

// Step begin: dt = cfl * min(dx/xmax, dy/ymax) (cfl.f90:50) and validTimeStep
// (mhd_driver.f90:117-144: clamp to tmax first, then reject negative, NaN or
// infinite dt).  With use_host_dt the host already stored dt.
__global__ void k_step_begin(Batch B, int use_host_dt) { PDL_ENTRY();
    for (int k = threadIdx.x; k < B.maxInst; k += blockDim.x) {
        InstState& S = B.st[k];
        if (!S.stepping) continue;
        if (use_host_dt) continue;
        const InstDev& d = B.dev[k];
        const double xm = __longlong_as_double((long long)S.cflbits[0]);
        const double ym = __longlong_as_double((long long)S.cflbits[1]);
        double dt = d.cfl * fmin(d.geo.dx / xm, d.geo.dy / ym);
        if (S.t + dt > S.tmax) {
            dt = S.tmax - S.t;
        } else if (dt < 0.0 || isnan(dt) || !isfinite(dt)) {
            S.error = HOSONO_ENANDT;
            S.done = 1;
            S.stepping = 0;
        }
        S.dt = dt;
    }
}

// Step start: which instances take part, fresh CFL accumulators.  (The step
// budget flags->stepsLeft is set by the host before each run launch.)
__global__ void k_step_prepare(Batch B, int /*unused*/) { PDL_ENTRY();
    for (int k = threadIdx.x; k < B.maxInst; k += blockDim.x) {
        InstState& S = B.st[k];
        S.stepping = (S.live && !S.done && !B.hold[k]) ? 1 : 0;
        S.cflbits[0] = 0;
        S.cflbits[1] = 0;
    }
}

// Step end: the new state is buffer A (parity flips), t += dt, nstep += 1,
// and the time-loop test of mhd_driver.f90:76; next step's participants and
// the batch condition.
__global__ void k_step_end(Batch B, cudaGraphConditionalHandle h, int set_handle) { PDL_ENTRY();
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    for (int k = threadIdx.x; k < B.maxInst; k += blockDim.x) {
        InstState& S = B.st[k];
        if (S.stepping) {
            S.parity = 1 - S.parity;
            S.t = S.t + S.dt;
            S.nstep = S.nstep + 1;
            if (!((S.t < S.tmax) && (S.nstep < S.nstepmax))) S.done = 1;
        }
        S.stepping = 0;  // at rest between launches; step_prepare picks the next participants
        S.cflbits[0] = 0;
        S.cflbits[1] = 0;
        if (S.live && !S.done && !B.hold[k]) any = 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int left = --B.flags->stepsLeft;
        B.flags->anyLive = any && left > 0;
        if (set_handle) cudaGraphSetConditional(h, (any && left > 0) ? 1u : 0u);
    }
}

// ======================================================================
// The later MOOD passes of a forward-Euler stage as one persistent launch
// (timeStep.f90:86-128 after the first pass): every phase of a pass -- the
// re-reconstruction of the recompute list, the face cascade, the face and
// FLICD lists, re-flux, FLICD + update + detect, the flag rebuild and the
// pass end -- runs in turn over the whole grid, separated by grid-wide
// barriers instead of kernel boundaries.  The blocks are all resident (a
// cooperative launch sized by occupancy: one 256-thread block per SM, whose
// 255-register budget holds the Riemann solver of the re-flux phase without
// spills).  The single-block steps (cascade_cond, pass_end) run on block 0
// while the others wait.

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int ld_acquire_s32(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Grid-wide barrier: each block's thread 0 publishes its block's writes
// (fence), counts itself in, and waits for the generation counter to move;
// the last block to arrive resets the count and moves the generation.  The
// wait is bounded: after kWaitCycles, or as soon as some block reported an
// error, the block reports HOSONO_ETIMEOUT (the first error stays) and the
// function returns false so that the caller leaves.
__device__ __forceinline__ bool grid_barrier(const Batch& B) {
    __shared__ int sOk;
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        unsigned* cnt = B.gbar;
        unsigned* gen = B.gbar + 1;
        const unsigned g = ld_acquire_u32(gen);
        __threadfence();
        int ok = 1;
        if (atomicAdd(cnt, 1u) + 1u == gridDim.x) {
            atomicExch(cnt, 0u);
            __threadfence();
            atomicAdd(gen, 1u);
        } else {
            const long long t0 = clock64();
            while (ld_acquire_u32(gen) == g) {
                if (ld_acquire_s32(&B.flags->error) || clock64() - t0 > kWaitCycles) {
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        if (!ok) atomicCAS(&B.flags->error, 0, HOSONO_ETIMEOUT);
        sOk = ok;
    }
    __syncthreads();
    return sOk != 0;
}

__global__ void __launch_bounds__(NTHREADS, 1) k_mood_rest(Batch B, int uin, int uout) {
    const int tid = threadIdx.y * TILE_X + threadIdx.x;
    const int gt = blockIdx.x * NTHREADS + tid, gs = gridDim.x * NTHREADS;
#define GSYNC_OR_LEAVE \
    if (!grid_barrier(B)) return
    for (;;) {
        if (!ld_acquire_s32(&B.flags->anyActive)) return;  // the same value in every block (read after a barrier)
        d_recon_group(B, uin, LIST_REC, gt, gs);
        GSYNC_OR_LEAVE;
        if (blockIdx.x == 0) d_cascade_cond<NTHREADS>(B, tid, 0, 0);
        GSYNC_OR_LEAVE;
        while (ld_acquire_s32(&B.flags->anyFail)) {
            FOR_CASCADE_TILES(B, t) t_cascade_lower(B, tile_at(B, t));
            GSYNC_OR_LEAVE;
            FOR_CASCADE_TILES(B, t) t_compact_next(B, tile_at(B, t));
            GSYNC_OR_LEAVE;
            d_recon_group(B, uin, LIST_NEXT, gt, gs);
            GSYNC_OR_LEAVE;
            if (blockIdx.x == 0) d_cascade_cond<NTHREADS>(B, tid, 0, 0);
            GSYNC_OR_LEAVE;
        }
        FOR_ACTIVE_TILES(B, t) t_compact_post(B, tile_at(B, t));
        GSYNC_OR_LEAVE;
        d_flux_list(B, uin, gt, gs);
        GSYNC_OR_LEAVE;
        d_ct_list(B, uin, uout, gt, gs);
        GSYNC_OR_LEAVE;
        d_flags_clear(B, gt, gs);
        GSYNC_OR_LEAVE;
        d_flags_scatter(B, gt, gs);
        GSYNC_OR_LEAVE;
        d_scheme_sync(B, 1, gt, gs);
        GSYNC_OR_LEAVE;
        if (blockIdx.x == 0) d_pass_end<NTHREADS>(B, tid, 0, 0, 0);
        GSYNC_OR_LEAVE;
    }
#undef GSYNC_OR_LEAVE
}

// The autotuner times pass 1 between steps: the instances that would step
// are marked stepping, and put back at rest afterwards (the face-cascade
// flag pass 1 raised is cleared too; every stage starts from stage_init).
__global__ void k_tune_mark(Batch B, int on) { PDL_ENTRY();
    for (int k = threadIdx.x; k < B.maxInst; k += blockDim.x) {
        InstState& S = B.st[k];
        S.stepping = (on && S.live && !S.done && !B.hold[k]) ? 1 : 0;
        S.anyFail = 0;
    }
}

// ======================================================================
const dim3 kTile(TILE_X, TILE_Y);

// Grid of a tile kernel: as many blocks as fit on the GPU at once (the
// kernels loop over the tile list), and never more than the tile capacity.
int resident_blocks(const void* kernel, int smem = 0) {
    static std::mutex mu;  // engines on several host threads launch concurrently
    std::lock_guard<std::mutex> lock(mu);
    static const void* keys[64];
    static int vals[64];
    static int n = 0;
    for (int k = 0; k < n; k++)
        if (keys[k] == kernel) return vals[k];
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, TILE_X * TILE_Y, smem);
    const int v = sms * (per > 0 ? per : 1);
    if (n < 64) {
        keys[n] = kernel;
        vals[n] = v;
        n++;
    }
    return v;
}
template <typename K>
dim3 grid_for(K kernel, const Batch& B) {
    const int r = resident_blocks((const void*)kernel);
    return dim3((unsigned)(r < B.maxTiles ? r : B.maxTiles));
}
// launch kern on s; programmatic (PDL_ENTRY) when the engine asked for it
// for this launch (pdl_take: the recorder's choice for the kernels of a step)
template <typename... KArgs, typename... Args>
void lk(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    if (pdl_take()) {
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
    }
    cudaLaunchKernelEx(&cfg, kern, args...);
}
#define TILE_LAUNCH(kern, B, s, ...) lk(kern, grid_for(kern, B), kTile, 0, s, B, ##__VA_ARGS__)
#define LIST_LAUNCH(kern, B, s, ...) \
    lk(kern, dim3((unsigned)resident_blocks((const void*)kern)), dim3(256), 0, s, B, ##__VA_ARGS__)

void l_cfl_reduce(const Batch& B, cudaStream_t s) { TILE_LAUNCH(k_cfl_reduce, B, s); }
void l_step_prepare(const Batch& B, int steps, cudaStream_t s) { lk(k_step_prepare, dim3(1), dim3(128), 0, s, B, steps); }
void l_step_begin(const Batch& B, int use_host_dt, cudaStream_t s) { lk(k_step_begin, dim3(1), dim3(128), 0, s, B, use_host_dt); }
void l_step_end(const Batch& B, cudaGraphConditionalHandle h, cudaStream_t s) {
    lk(k_step_end, dim3(1), dim3(128), 0, s, B, h, (int)(h != 0));
}
void l_stage_init(const Batch& B, cudaStream_t s) { TILE_LAUNCH(k_stage_init, B, s); }
// dynamic shared memory of a pass-1 kernel variant
template <int R, int NBUF>
constexpr int pass1_smem() {
    return P1Smem<R>::bytes(NBUF);
}
template <int R, bool TMA, bool DYN, int MINB, int NBUF>
int pass1_grid(int maxTiles) {
    static const bool attr =  // once per process (thread-safe static initialisation)
        cudaFuncSetAttribute((const void*)k_face_pass1<R, TMA, DYN, MINB, NBUF>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, pass1_smem<R, NBUF>()) == cudaSuccess;
    (void)attr;
    const int r = resident_blocks((const void*)k_face_pass1<R, TMA, DYN, MINB, NBUF>, pass1_smem<R, NBUF>());
    return r < maxTiles ? r : maxTiles;
}
template <int R, bool TMA, bool DYN, int MINB, int NBUF>
void launch_pass1_v(const Batch& B, int uin, cudaStream_t s) {
    lk(k_face_pass1<R, TMA, DYN, MINB, NBUF>, dim3((unsigned)pass1_grid<R, TMA, DYN, MINB, NBUF>(B.maxTiles)), kTile,
       (size_t)pass1_smem<R, NBUF>(), s, B, uin);
}
template <int R, int MINB, int NBUF>
void launch_pass1_s(const Batch& B, int uin, cudaStream_t s) {  // staging and schedule
    if (B.p1Tma) {
        if (B.p1Dyn)
            launch_pass1_v<R, true, true, MINB, NBUF>(B, uin, s);
        else
            launch_pass1_v<R, true, false, MINB, NBUF>(B, uin, s);
    } else {
        if (B.p1Dyn)
            launch_pass1_v<R, false, true, MINB, NBUF>(B, uin, s);
        else
            launch_pass1_v<R, false, false, MINB, NBUF>(B, uin, s);
    }
}
// the variant the tuning asks for: TMA staging and two boxes only with two
// blocks per SM
template <int R>
void launch_pass1(const Batch& B, int uin, cudaStream_t s) {
    if (B.p1Blocks == 3) {
        if (B.p1Dyn)
            launch_pass1_v<R, false, true, 3, 1>(B, uin, s);
        else
            launch_pass1_v<R, false, false, 3, 1>(B, uin, s);
    } else if (B.p1Blocks == 4) {
        if (B.p1Dyn)
            launch_pass1_v<R, false, true, 4, 1>(B, uin, s);
        else
            launch_pass1_v<R, false, false, 4, 1>(B, uin, s);
    } else if (B.p1Boxes == 1) {
        launch_pass1_s<R, 2, 1>(B, uin, s);
    } else {
        launch_pass1_s<R, 2, 2>(B, uin, s);
    }
}
// one launch per radius held (the kernels also skip radii the device's
// tile list does not hold)
void l_face_pass1(const Batch& B, int uin, cudaStream_t s) {
    if (B.p1Radii & (1 << 2)) launch_pass1<2>(B, uin, s);
    if (B.p1Radii & (1 << 1)) launch_pass1<1>(B, uin, s);
    if (B.p1Radii & (1 << 3)) launch_pass1<3>(B, uin, s);
}
void l_cascade_cond(const Batch& B, cudaGraphConditionalHandle h, cudaStream_t s) {
    lk(k_cascade_cond, dim3(1), dim3(PASS_END_THREADS), 0, s, B, h, (int)(h != 0));
}
void l_cascade_lower(const Batch& B, int /*later*/, cudaStream_t s) { TILE_LAUNCH(k_cascade_lower, B, s); }
void l_recon_check(const Batch& B, int uin, int /*later*/, cudaStream_t s) {
    TILE_LAUNCH(k_compact_next, B, s);
    LIST_LAUNCH(k_recon_group, B, s, uin, (int)LIST_NEXT);
}
void l_ct_update_detect(const Batch& B, int uin, int uout, cudaStream_t s) {
    if (!B.ctStaged) {
        TILE_LAUNCH(k_ct_update_detect, B, s, uin, uout);
        return;
    }
    static const bool attr =  // once per process (thread-safe static initialisation)
        cudaFuncSetAttribute((const void*)k_ct_update_detect_tma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             CT_SMEM_BYTES) == cudaSuccess;
    (void)attr;
    const int r = resident_blocks((const void*)k_ct_update_detect_tma, CT_SMEM_BYTES);
    lk(k_ct_update_detect_tma, dim3((unsigned)(r < B.maxTiles ? r : B.maxTiles)), kTile, (size_t)CT_SMEM_BYTES, s, B,
       uin, uout);
}
void l_mood_flags(const Batch& B, int mode, cudaStream_t s) {
    if (mode == MOOD_FLAGS_DENSE) {
        TILE_LAUNCH(k_mood_flags, B, s);
    } else {
        LIST_LAUNCH(k_flags_clear, B, s);
        LIST_LAUNCH(k_flags_scatter, B, s);
        LIST_LAUNCH(k_scheme_sync, B, s, mode == MOOD_FLAGS_LISTS_CLEAR ? 1 : 0);
    }
}
void l_pass_end(const Batch& B, cudaGraphConditionalHandle h, int flip, cudaStream_t s) {
    lk(k_pass_end, dim3(1), dim3(PASS_END_THREADS), 0, s, B, h, (int)(h != 0), flip);
}
void l_compact_post(const Batch& B, cudaStream_t s) { TILE_LAUNCH(k_compact_post, B, s); }
void l_compact_dirty(const Batch& B, cudaStream_t s) { TILE_LAUNCH(k_compact_dirty, B, s); }
void l_recon_list(const Batch& B, int uin, cudaStream_t s) { LIST_LAUNCH(k_recon_group, B, s, uin, (int)LIST_REC); }
void l_flux_list(const Batch& B, int uin, cudaStream_t s) { LIST_LAUNCH(k_flux_list, B, s, uin); }
void l_ct_list(const Batch& B, int uin, int uout, cudaStream_t s) { LIST_LAUNCH(k_ct_list, B, s, uin, uout); }
void l_clear_low(const Batch& B, cudaStream_t s) { LIST_LAUNCH(k_clear_low, B, s); }
void l_bc_fill(const Batch& B, int role, cudaStream_t s) { TILE_LAUNCH(k_bc_fill, B, s, role); }
void l_rk_combine2(const Batch& B, cudaStream_t s) { TILE_LAUNCH(k_rk_combine2, B, s); }
void l_rk_final(const Batch& B, cudaStream_t s) { TILE_LAUNCH(k_rk_final, B, s); }
void l_cons2prim_all(const Batch& B, cudaStream_t s) { TILE_LAUNCH(k_cons2prim_all, B, s); }
void l_tune_mark(const Batch& B, int on, cudaStream_t s) { lk(k_tune_mark, dim3(1), dim3(128), 0, s, B, on); }
// every block resident at once: a cooperative launch of as many blocks as
// fit on the GPU (never more, or a barrier could not complete)
void l_mood_rest(const Batch& B, int uin, int uout, cudaStream_t s) {
    const int grid = resident_blocks((const void*)k_mood_rest);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = kTile;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_mood_rest, B, uin, uout);
}
void l_launch_info(int R, int maxTiles, int* pass1, int* tile_grid_max) {
    *pass1 = R == 1   ? pass1_grid<1, false, false, 2, 2>(maxTiles)
             : R == 2 ? pass1_grid<2, false, false, 2, 2>(maxTiles)
                      : pass1_grid<3, false, false, 2, 2>(maxTiles);
    const void* tile_kernels[] = {(const void*)k_cfl_reduce,     (const void*)k_stage_init,
                                  (const void*)k_cascade_lower,  (const void*)k_compact_next, (const void*)k_compact_post,
                                  (const void*)k_compact_dirty,  (const void*)k_ct_update_detect, (const void*)k_mood_flags,
                                  (const void*)k_bc_fill,        (const void*)k_rk_combine2,  (const void*)k_rk_final,
                                  (const void*)k_cons2prim_all};
    int mx = 0;
    for (const void* k : tile_kernels) {
        const int r = resident_blocks(k);
        mx = std::max(mx, r < maxTiles ? r : maxTiles);
    }
    *tile_grid_max = mx;
}

#include "modules.cuh"

const KernelSet kset = {
#if HOSONO_FAST
    "fast",
#else
    "strict",
#endif
    l_cfl_reduce, l_step_prepare, l_step_begin, l_step_end, l_stage_init, l_face_pass1, l_cascade_cond, l_cascade_lower,
    l_recon_check, l_ct_update_detect, l_mood_flags, l_pass_end, l_recon_list,
    l_compact_post, l_compact_dirty, l_flux_list, l_ct_list, l_clear_low, l_bc_fill, l_rk_combine2, l_rk_final,
    l_cons2prim_all, l_tune_mark, l_mood_rest, l_launch_info, &mops};

}  // namespace KNS

#if HOSONO_FAST
const KernelSet* kernelset_fast() { return &kfast::kset; }
#else
const KernelSet* kernelset_strict() { return &kstrict::kset; }
#endif

}  // namespace hosono
