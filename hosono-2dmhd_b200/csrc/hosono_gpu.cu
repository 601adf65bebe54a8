// hosono_gpu.cu -- the C ABI of include/hosono_gpu.h over the batched engine.
//
// hosono_gpu_* : one block (the reference's grid_block + grid_state), i.e. an
//                engine holding one instance.
// hosono_batch_*: many independent blocks of any sizes advanced together.

#include "checks.h"
#include "engine_host.h"
#include "hosono_gpu.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>

using namespace hosono;

struct hosono_handle {
    Engine eng;
    int slot = 0;
    hosono_stats stats{};
    bool profile = false;
    double pass1Ms = 0.0;
    long long pass1Count = 0;
};

struct hosono_batch {
    Engine eng;
};

namespace {

hosono_stats stats_delta(const InstState& a, const InstState& b) {
    hosono_stats s{};
    s.stages = b.stages - a.stages;
    s.mood_passes = b.passesTotal - a.passesTotal;
    s.max_passes = b.maxPasses;
    s.detect_lowered = b.detectTotal - a.detectTotal;
    s.inner_lowered = b.innerTotal - a.innerTotal;
    s.cascade_iters = b.cascadeIters - a.cascadeIters;
    return s;
}

// kernels one graph execution launched, from the work counters: per step 4
// time-loop kernels (cfl path) or 1 (host dt), 3 RK kernels; per stage 8
// plus one pass-1 face kernel per GP radius held; per cascade iteration 4;
// per further MOOD pass 9.
long long graph_launches(const hosono_stats& s, int steps, bool host_dt, int radii) {
    return (long long)steps * ((host_dt ? 1 : 4) + 3) + (8LL + radii) * s.stages + 4LL * s.cascade_iters +
           9LL * (s.mood_passes - s.stages);
}

}  // namespace

extern "C" {

int hosono_gpu_create(const hosono_params* p, const double* pv, const double* qw, const int* stenc,
                      hosono_handle** out) {
    if (!p || !pv || !qw || !out) return HOSONO_EINVAL;
    *out = nullptr;
    if (!params_ok(*p) || !stencil_ok(p->max_radius, stenc)) return HOSONO_EINVAL;
    hosono_handle* h = new (std::nothrow) hosono_handle();
    if (!h) return HOSONO_ENOMEM;
    int rc = h->eng.init(1, h->eng.tiles_of(*p), p->fp_mode);
    if (!rc) rc = h->eng.add(*p, pv, qw, &h->slot);
    if (rc) {
        delete h;
        return rc;
    }
    *out = h;
    return HOSONO_OK;
}

int hosono_gpu_destroy(hosono_handle* h) {
    delete h;
    return HOSONO_OK;
}

int hosono_gpu_upload(hosono_handle* h, const double* U, const double* V) {
    if (!h || !U) return HOSONO_EINVAL;
    return h->eng.upload(h->slot, U, V);
}

int hosono_gpu_download(hosono_handle* h, double* U, double* V, int* scheme) {
    if (!h) return HOSONO_EINVAL;
    return h->eng.download(h->slot, U, V, scheme);
}

int hosono_gpu_cfl(hosono_handle* h, double* dt) {
    if (!h || !dt) return HOSONO_EINVAL;
    return h->eng.cfl(h->slot, dt);
}

int hosono_gpu_advance(hosono_handle* h, double dt) {
    if (!h) return HOSONO_EINVAL;
    InstState a, b;
    int rc = h->eng.state(h->slot, &a);
    if (!rc) rc = h->eng.advance(h->slot, dt);
    if (!rc) rc = h->eng.state(h->slot, &b);
    if (!rc) {
        h->stats = stats_delta(a, b);
        if (h->eng.use_graphs && !h->eng.trace) h->eng.launches += graph_launches(h->stats, 1, true, h->eng.radii_held());
    }
    return rc;
}

int hosono_gpu_set_time(hosono_handle* h, double t, double tmax, int nstep, int nstepmax) {
    if (!h) return HOSONO_EINVAL;
    return h->eng.set_time(h->slot, t, tmax, nstep, nstepmax);
}

int hosono_gpu_set_mood_cap(hosono_handle* h, int cap) {
    if (!h) return HOSONO_EINVAL;
    return h->eng.set_mood_cap(h->slot, cap);
}

int hosono_gpu_step(hosono_handle* h, int max_steps, double* t_out, int* nstep_out) {
    if (!h) return HOSONO_EINVAL;
    InstState a, b;
    int rc = h->eng.state(h->slot, &a);
    if (rc) return rc;
    if (h->profile) {
        for (int k = 0; k < (max_steps > 0 ? max_steps : 1) && !rc; k++) {
            InstState c;
            rc = h->eng.state(h->slot, &c);
            if (rc || c.done) break;
            double ms = 0;
            int n = 0;
            rc = h->eng.run_profiled_step(&ms, &n);
            h->pass1Ms += ms;
            h->pass1Count += n;
        }
    } else {
        rc = h->eng.run(max_steps);
    }
    if (rc) return rc;
    rc = h->eng.state(h->slot, &b);
    if (rc) return rc;
    h->stats = stats_delta(a, b);
    if (h->eng.use_graphs && !h->eng.trace) h->eng.launches += graph_launches(h->stats, b.nstep - a.nstep, false, h->eng.radii_held());
    if (t_out) *t_out = b.t;
    if (nstep_out) *nstep_out = b.nstep;
    return HOSONO_OK;
}

int hosono_gpu_run(hosono_handle* h, double tmax, int nstepmax, int max_steps, double* t_out, int* nstep_out) {
    if (!h) return HOSONO_EINVAL;
    int rc = h->eng.set_time(h->slot, 0.0, tmax, 0, nstepmax);
    if (rc) return rc;
    return hosono_gpu_step(h, max_steps, t_out, nstep_out);
}

int hosono_gpu_advance_host(hosono_handle* h, double dt, double* U, double* V) {
    if (!h || !U) return HOSONO_EINVAL;
    InstState a, b;
    int rc = h->eng.state(h->slot, &a);
    if (!rc) rc = h->eng.advance_host(h->slot, dt, U, V);
    if (!rc) rc = h->eng.state(h->slot, &b);
    if (!rc) {
        h->stats = stats_delta(a, b);
        if (h->eng.use_graphs && !h->eng.trace) h->eng.launches += graph_launches(h->stats, 1, true, h->eng.radii_held());
    }
    return rc;
}

int hosono_gpu_stats(hosono_handle* h, hosono_stats* s) {
    if (!h || !s) return HOSONO_EINVAL;
    *s = h->stats;
    return HOSONO_OK;
}

int hosono_gpu_last_error(hosono_handle* h, char* buf, int len) {
    if (!h) return HOSONO_EINVAL;
    if (buf && len > 0) std::snprintf(buf, (size_t)len, "%s", h->eng.msg.c_str());
    return h->eng.err;
}

int hosono_gpu_trace_enable(hosono_handle* h, int on) {
    if (!h) return HOSONO_EINVAL;
    h->eng.trace = on != 0;
    return HOSONO_OK;
}
int hosono_gpu_trace_count(hosono_handle* h) { return h ? (int)h->eng.traces.size() : 0; }
int hosono_gpu_trace_get(hosono_handle* h, int k, int* meta, unsigned char* inner, unsigned char* detect) {
    if (!h || k < 0 || k >= (int)h->eng.traces.size()) return HOSONO_EINVAL;
    const TraceRec& t = h->eng.traces[k];
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
    h->eng.traces.clear();
    InstState st;
    int rc = h->eng.state(h->slot, &st);
    if (!rc) h->eng.traceStageBase[h->slot] = st.stages;
    return rc;
}

int hosono_gpu_module_set(hosono_handle* h, const int* scheme, const int* recompute, const int* recompute_flicd) {
    return h ? h->eng.mod_set(h->slot, scheme, recompute, recompute_flicd) : HOSONO_EINVAL;
}
int hosono_gpu_module_get(hosono_handle* h, double* faceVals, double* fluxRaw, double* flux, double* Unew,
                          int* scheme, int* recompute, int* recompute_flicd) {
    return h ? h->eng.mod_get(h->slot, faceVals, fluxRaw, flux, Unew, scheme, recompute, recompute_flicd)
             : HOSONO_EINVAL;
}
int hosono_gpu_reconstruct(hosono_handle* h) { return h ? h->eng.mod_reconstruct(h->slot) : HOSONO_EINVAL; }
int hosono_gpu_getfluxes(hosono_handle* h) { return h ? h->eng.mod_getfluxes(h->slot) : HOSONO_EINVAL; }
int hosono_gpu_flicd(hosono_handle* h) { return h ? h->eng.mod_flicd(h->slot) : HOSONO_EINVAL; }
int hosono_gpu_update(hosono_handle* h, double dt) { return h ? h->eng.mod_update(h->slot, dt) : HOSONO_EINVAL; }
int hosono_gpu_detect(hosono_handle* h, int* exit_mood_loop) {
    return h ? h->eng.mod_detect(h->slot, exit_mood_loop) : HOSONO_EINVAL;
}
int hosono_gpu_bc(hosono_handle* h, int which) { return h ? h->eng.mod_bc(h->slot, which) : HOSONO_EINVAL; }
int hosono_gpu_bc_mood(hosono_handle* h) { return h ? h->eng.mod_bc_mood(h->slot) : HOSONO_EINVAL; }
int hosono_gpu_mood_pass_stats(hosono_handle* h, int* npasses, long long* ntroubled) {
    if (!h) return HOSONO_EINVAL;
    if (npasses) *npasses = h->stats.mood_passes;
    if (ntroubled) *ntroubled = h->stats.detect_lowered + h->stats.inner_lowered;
    return HOSONO_OK;
}
int hosono_gpu_riemann(hosono_handle* h, int n, const double* uL_dev, const double* uR_dev, int dir,
                       double* flux_dev) {
    return h ? h->eng.riemann(h->slot, n, uL_dev, uR_dev, dir, flux_dev) : HOSONO_EINVAL;
}

int hosono_gpu_eigenvecs(hosono_handle* h, int n, const double* V_dev, int dir, int cons, double* L_dev,
                         double* R_dev) {
    return h ? h->eng.eigenvecs(h->slot, n, V_dev, dir, cons, L_dev, R_dev) : HOSONO_EINVAL;
}

int hosono_gpu_state_layout(hosono_handle* h, double** U_dev, int* pitch, long long* plane) {
    if (!h) return HOSONO_EINVAL;
    InstState st;
    int rc = h->eng.state(h->slot, &st);
    if (rc) return rc;
    const Geo& G = h->eng.geo(h->slot);
    if (pitch) *pitch = G.pitch;
    if (plane) *plane = G.plane;
    if (U_dev) *U_dev = h->eng.dev(h->slot).U[st.parity];
    return HOSONO_OK;
}

int hosono_gpu_build_info(int* sm_arch, int* has_fast_mode) {
    if (sm_arch) *sm_arch = 100;
    if (has_fast_mode) *has_fast_mode = 1;
    return HOSONO_OK;
}

int hosono_gpu_set_device(int device) { return cudaSetDevice(device) == cudaSuccess ? HOSONO_OK : HOSONO_ECUDA; }

int hosono_gpu_stream(hosono_handle* h, void** stream) {
    if (!h || !stream) return HOSONO_EINVAL;
    *stream = (void*)h->eng.stream();
    return HOSONO_OK;
}

int hosono_gpu_set_tuning(hosono_handle* h, const hosono_tuning* t) {
    return h && t ? h->eng.set_tuning(*t) : HOSONO_EINVAL;
}
int hosono_gpu_get_tuning(hosono_handle* h, hosono_tuning* t) {
    if (!h || !t) return HOSONO_EINVAL;
    *t = h->eng.tuning();
    return HOSONO_OK;
}
int hosono_batch_set_tuning(hosono_batch* b, const hosono_tuning* t) {
    return b && t ? b->eng.set_tuning(*t) : HOSONO_EINVAL;
}
int hosono_batch_get_tuning(hosono_batch* b, hosono_tuning* t) {
    if (!b || !t) return HOSONO_EINVAL;
    *t = b->eng.tuning();
    return HOSONO_OK;
}

int hosono_gpu_autotune(hosono_handle* h, int trials, int force, hosono_tune_report* report) {
    return h ? h->eng.autotune(trials, force != 0, report) : HOSONO_EINVAL;
}
int hosono_batch_autotune(hosono_batch* b, int trials, int force, hosono_tune_report* report) {
    return b ? b->eng.autotune(trials, force != 0, report) : HOSONO_EINVAL;
}

int hosono_gpu_launch_info(hosono_handle* h, hosono_launch_info* info) {
    if (!h || !info) return HOSONO_EINVAL;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
                                                  cudaSuccess) {
        cudaGetLastError();
        return HOSONO_ECUDA;
    }
    info->tiles = h->eng.used_tiles();
    info->sms = sms;
    h->eng.launch_info(h->eng.params(h->slot).max_radius, &info->pass1_grid, &info->tile_grid_max);
    return HOSONO_OK;
}

int hosono_gpu_set_graphs(hosono_handle* h, int on) {
    if (!h) return HOSONO_EINVAL;
    h->eng.use_graphs = on != 0;
    return HOSONO_OK;
}

int hosono_gpu_profile(hosono_handle* h, int on) {
    if (!h) return HOSONO_EINVAL;
    h->profile = on != 0;
    return HOSONO_OK;
}

int hosono_gpu_profile_read(hosono_handle* h, double* pass1_ms, long long* pass1_launches, long long* launches,
                            int reset) {
    if (!h) return HOSONO_EINVAL;
    if (pass1_ms) *pass1_ms = h->pass1Ms;
    if (pass1_launches) *pass1_launches = h->pass1Count;
    if (launches) *launches = h->eng.launches;
    if (reset) {
        h->pass1Ms = 0.0;
        h->pass1Count = 0;
        h->eng.launches = 0;
    }
    return HOSONO_OK;
}

// ---------------------------------------------------------------- batches

int hosono_batch_create(int max_instances, int max_tiles, int fp_mode, hosono_batch** out) {
    if (!out || max_instances < 1 || max_tiles < 1) return HOSONO_EINVAL;
    *out = nullptr;
    hosono_batch* b = new (std::nothrow) hosono_batch();
    if (!b) return HOSONO_ENOMEM;
    int rc = b->eng.init(max_instances, max_tiles, fp_mode);
    if (rc) {
        delete b;
        return rc;
    }
    *out = b;
    return HOSONO_OK;
}

int hosono_batch_destroy(hosono_batch* b) {
    delete b;
    return HOSONO_OK;
}

int hosono_batch_tiles_for(const hosono_params* p) {
    if (!p) return -1;
    const int nxt = p->nx + 2 * p->ngc, nyt = p->ny + 2 * p->ngc;
    return ((nxt + TILE_X - 1) / TILE_X) * ((nyt + TILE_Y - 1) / TILE_Y);
}

long long hosono_batch_instance_bytes(const hosono_params* p) {
    if (!p) return -1;
    Engine e;
    return (long long)e.instance_bytes(*p);
}

int hosono_batch_add(hosono_batch* b, const hosono_params* p, const double* pv, const double* qw, const int* stenc,
                     int* slot) {
    if (!b || !p || !slot) return HOSONO_EINVAL;
    if (!params_ok(*p) || !stencil_ok(p->max_radius, stenc)) return HOSONO_EINVAL;
    return b->eng.add(*p, pv, qw, slot);
}

int hosono_batch_remove(hosono_batch* b, int slot) { return b ? b->eng.remove(slot) : HOSONO_EINVAL; }

int hosono_batch_upload(hosono_batch* b, int slot, const double* U, const double* V) {
    return b ? b->eng.upload(slot, U, V) : HOSONO_EINVAL;
}

int hosono_batch_download(hosono_batch* b, int slot, double* U, double* V, int* scheme) {
    return b ? b->eng.download(slot, U, V, scheme) : HOSONO_EINVAL;
}

int hosono_batch_set_time(hosono_batch* b, int slot, double t, double tmax, int nstep, int nstepmax) {
    return b ? b->eng.set_time(slot, t, tmax, nstep, nstepmax) : HOSONO_EINVAL;
}

int hosono_batch_set_mood_cap(hosono_batch* b, int slot, int cap) {
    return b ? b->eng.set_mood_cap(slot, cap) : HOSONO_EINVAL;
}

int hosono_batch_run(hosono_batch* b, int max_steps) { return b ? b->eng.run(max_steps) : HOSONO_EINVAL; }

int hosono_batch_status(hosono_batch* b, int slot, double* t, double* dt, int* nstep, int* done, int* error) {
    if (!b) return HOSONO_EINVAL;
    InstState st;
    int rc = b->eng.state(slot, &st);
    if (rc) return rc;
    if (t) *t = st.t;
    if (dt) *dt = st.dt;
    if (nstep) *nstep = st.nstep;
    if (done) *done = st.done;
    if (error) *error = st.error;
    return HOSONO_OK;
}

int hosono_batch_stats(hosono_batch* b, int slot, hosono_stats* s) {
    if (!b || !s) return HOSONO_EINVAL;
    InstState st;
    int rc = b->eng.state(slot, &st);
    if (rc) return rc;
    s->stages = st.stages;
    s->mood_passes = st.passesTotal;
    s->max_passes = st.maxPasses;
    s->detect_lowered = st.detectTotal;
    s->inner_lowered = st.innerTotal;
    s->cascade_iters = st.cascadeIters;
    return HOSONO_OK;
}

int hosono_batch_stream(hosono_batch* b, void** stream) {
    if (!b || !stream) return HOSONO_EINVAL;
    *stream = (void*)b->eng.stream();
    return HOSONO_OK;
}

int hosono_batch_set_graphs(hosono_batch* b, int on) {
    if (!b) return HOSONO_EINVAL;
    b->eng.use_graphs = on != 0;
    return HOSONO_OK;
}

int hosono_gpu_ic(hosono_handle* h, const hosono_ic_desc* ic, const double* xtab, const double* ytab) {
    return h && ic ? h->eng.ic(h->slot, *ic, xtab, ytab) : HOSONO_EINVAL;
}

int hosono_batch_ic(hosono_batch* b, int slot, const hosono_ic_desc* ic, const double* xtab, const double* ytab) {
    return b && ic ? b->eng.ic(slot, *ic, xtab, ytab) : HOSONO_EINVAL;
}

int hosono_gpu_diagnostics(hosono_handle* h, double* fields, int* scheme, int* ordr, double* divb_l1,
                           double* divb_linf) {
    return h ? h->eng.diagnostics(h->slot, fields, scheme, ordr, divb_l1, divb_linf) : HOSONO_EINVAL;
}

int hosono_batch_diagnostics(hosono_batch* b, int slot, double* fields, int* scheme, int* ordr, double* divb_l1,
                             double* divb_linf) {
    return b ? b->eng.diagnostics(slot, fields, scheme, ordr, divb_l1, divb_linf) : HOSONO_EINVAL;
}

int hosono_batch_last_error(hosono_batch* b, char* buf, int len) {
    if (!b) return HOSONO_EINVAL;
    if (buf && len > 0) std::snprintf(buf, (size_t)len, "%s", b->eng.msg.c_str());
    return b->eng.err;
}

int hosono_batch_capacity(hosono_batch* b, int* max_instances, int* max_tiles, int* used_tiles, int* live) {
    if (!b) return HOSONO_EINVAL;
    if (max_instances) *max_instances = b->eng.max_inst();
    if (max_tiles) *max_tiles = b->eng.max_tiles();
    if (used_tiles) *used_tiles = b->eng.used_tiles();
    if (live) *live = b->eng.live_count();
    return HOSONO_OK;
}

}  // extern "C"
