// server.cu -- the serving layer of include/hosono_gpu.h (no counterpart in
// the reference): a queue of solves, admission by a device-memory budget, and
// continuous batching of the resident solves over one Engine, under one of
// two policies (FIFO; or shortest estimated work first with an aging bound,
// HOSONO_SERVE_SHORTEST).
//
// Threads: callers submit, wait, poll and ask for snapshots under one mutex;
// a scheduler thread owns the Engine, the CUDA stream and the budget arena,
// and is the only thread that makes CUDA calls.  Its loop:
//   admit    -- while the next solve (the queue head, or under SHORTEST the
//               oldest past the aging bound, else the least estimated work)
//               fits (slot, tiles, a free arena range): Engine::add on arena
//               memory, one tile-list upload for all, then upload each
//               initial state and set its time limits;
//   snapshot -- copy out resident solves that callers asked for;
//   launch   -- one batched run of up to `steps` time steps (one graph
//               launch); `steps` follows the measured time per step so that
//               a launch takes about chunk_ms.  Under SHORTEST the residents
//               with the most estimated remaining work sit the launch out
//               (Engine::set_holds) once the others fill fill_tiles tiles;
//   retire   -- solves whose InstState says done: copy the final state to
//               the caller's buffers, free the slot and the arena range.
// Each solve keeps its own t, dt, MOOD loop and limits inside the batch, so
// its arithmetic does not depend on the other residents.

#include "arena.h"
#include "checks.h"
#include "engine_host.h"
#include "hosono_gpu.h"

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

using namespace hosono;

namespace {

double clock_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct Request {
    hosono_params p{};
    std::vector<double> pv, qw, U, V;
    bool devIC = false;  // initial state built on the device from ic + tables
    hosono_ic_desc ic{};
    std::vector<double> xtab, ytab;
    double tmax = 0;
    int nstepmax = 0;
    double* outU = nullptr;
    double* outV = nullptr;
    int* outScheme = nullptr;
    int tiles = 0;
    int baseNstep = 0;
    double work = 0;         // estimated work: interior cells x tmax / min(dx, dy)
    double lastStep_s = 0;   // server clock when it last took part in a launch (or was admitted)
    hosono_request_info info{};
};

struct Snapshot {
    long long id = 0;
    double* U = nullptr;
    double* V = nullptr;
    int* scheme = nullptr;
    double t = 0;
    int nstep = 0;
    int status = -1;  // -1 while pending
};

// Engine memory from the budget arena (one device allocation)
class ArenaAllocator : public DeviceAllocator {
  public:
    char* base = nullptr;
    Arena arena;
    void* alloc(size_t n) override {
        size_t off = 0;
        if (!base || !arena.alloc(n, &off)) return nullptr;
        return base + off;
    }
    void release(void* p) override {
        if (p) arena.release((size_t)((char*)p - base));
    }
};

// device bytes one 32x8 tile of a resident solve takes at least: an instance
// of c allocated cells uses >= c * (38 doubles + 13 flag bytes) and covers
// at most 1.1 c / 256 tiles (rows rounded up to 8, grids of >= 70 rows)
constexpr double kBytesPerTile = 256.0 * (38 * 8 + 13) / 1.1;

}  // namespace

struct hosono_server {
    hosono_serve_config cfg{};
    int device = 0;
    std::thread th;
    std::mutex mu;
    std::condition_variable wake;  // scheduler: new work or stop
    std::condition_variable done;  // callers: a solve or snapshot finished, or start-up ended
    std::deque<Request*> queue;
    std::unordered_map<long long, std::unique_ptr<Request>> reqs;
    std::vector<Request*> resident;
    std::deque<long long> finished;
    std::deque<Snapshot*> snaps;
    long long nextId = 1;
    bool stop = false;
    bool started = false;
    int startRc = HOSONO_OK;
    int fatal = HOSONO_OK;
    int err = HOSONO_OK;
    std::string msg;
    hosono_serve_totals st{};
    int maxTiles = 0;
    long long budget = 0;
    int inflight = 0;  // callers blocked in wait/drain/snapshot (destroy lets them leave first)

    int fail(int code, const std::string& m) {  // caller holds mu
        err = code;
        msg = m;
        return code;
    }
};

namespace {

// caller holds S->mu
void finish_locked(hosono_server* S, Request* r, int status) {
    r->info.state = HOSONO_REQ_DONE;
    r->info.status = status;
    r->info.slot = -1;
    r->info.finish_s = clock_s();
    if (status == HOSONO_OK) {
        S->st.completed++;
        S->st.zone_updates += r->info.zone_updates;
    } else {
        S->st.failed++;
    }
    S->finished.push_back(r->info.id);
    r->pv.clear();
    r->qw.clear();
    r->U = std::vector<double>();
    r->V = std::vector<double>();
}

void fill_mood(hosono_request_info& info, const InstState& s) {
    info.mood.stages = s.stages;
    info.mood.mood_passes = s.passesTotal;
    info.mood.max_passes = s.maxPasses;
    info.mood.detect_lowered = s.detectTotal;
    info.mood.inner_lowered = s.innerTotal;
    info.mood.cascade_iters = s.cascadeIters;
}

class Scheduler {
  public:
    explicit Scheduler(hosono_server* s) : S(s) {}

    void main() {
        int rc = start();
        {
            std::lock_guard<std::mutex> lk(S->mu);
            S->startRc = rc;
            S->started = true;
            if (rc) S->fail(rc, eng ? eng->msg : std::string("server start-up failed"));
        }
        S->done.notify_all();
        if (!rc) loop();
        shutdown();
    }

  private:
    hosono_server* S;
    std::unique_ptr<Engine> eng;
    ArenaAllocator mem;
    double msPerStep = 0.0;

    int start() {
        if (cudaSetDevice(S->device) != cudaSuccess) return HOSONO_ECUDA;
        size_t freeB = 0, totalB = 0;
        if (cudaMemGetInfo(&freeB, &totalB) != cudaSuccess) return HOSONO_ECUDA;
        long long budget = S->cfg.memory_budget > 0 ? S->cfg.memory_budget : (long long)(0.55 * (double)freeB);
        budget = budget / (long long)Arena::kAlign * (long long)Arena::kAlign;
        if (budget <= 0) return HOSONO_EINVAL;
        const int maxTiles = (int)std::min<double>((double)budget / kBytesPerTile + 64.0, (double)INT_MAX / 512);
        if (cudaMalloc(&mem.base, (size_t)budget) != cudaSuccess) {
            cudaGetLastError();
            mem.base = nullptr;
            return HOSONO_ENOMEM;
        }
        mem.arena.reset((size_t)budget);
        eng.reset(new (std::nothrow) Engine());
        if (!eng) return HOSONO_ENOMEM;
        eng->set_allocator(&mem);
        eng->instance_errors_fatal = false;
        const int rc = eng->init(S->cfg.max_resident, maxTiles, S->cfg.fp_mode);
        if (rc) return rc;
        std::lock_guard<std::mutex> lk(S->mu);
        S->maxTiles = maxTiles;
        S->budget = budget;
        S->st.budget_bytes = budget;
        return HOSONO_OK;
    }

    void loop() {
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(S->mu);
                S->wake.wait(lk, [&] { return S->stop || !S->queue.empty() || !S->resident.empty() || !S->snaps.empty(); });
                if (S->stop) return;
            }
            const double t0 = clock_s();
            int rc = admit();
            if (!rc) rc = serve_snapshots();
            const double t1 = clock_s();
            bool ran = false;
            double t2 = t1;
            if (!rc && !resident_empty()) {
                rc = launch();
                ran = true;
                t2 = clock_s();
                if (!rc) rc = retire();
            }
            const double t3 = clock_s();
            {
                std::lock_guard<std::mutex> lk(S->mu);
                S->st.admin_s += (t1 - t0) + (t3 - t2);
                if (ran) S->st.busy_s += t2 - t1;
                if (rc) {
                    S->fatal = rc;
                    S->fail(rc, "server stopped: " + eng->msg);
                }
            }
            if (rc) return;
        }
    }

    bool resident_empty() {
        std::lock_guard<std::mutex> lk(S->mu);
        return S->resident.empty();
    }

    // the queued solve to admit next: the head (FIFO); or the oldest solve
    // past the aging bound, else the one with the least estimated work that
    // was not passed over in this admission round (SHORTEST).  `aged` tells
    // the caller not to pass over it.  Caller holds S->mu.
    Request* pick_locked(const std::vector<Request*>& passed, bool* aged) {
        *aged = true;
        if (S->cfg.policy != HOSONO_SERVE_SHORTEST) return S->queue.front();
        const double now = clock_s();
        for (Request* r : S->queue)  // queue order is arrival order
            if (now - r->info.submit_s >= S->cfg.aging_s) return r;
        *aged = false;
        Request* best = nullptr;
        for (Request* r : S->queue)
            if (std::find(passed.begin(), passed.end(), r) == passed.end() && (!best || r->work < best->work)) best = r;
        return best;
    }

    int admit() {
        std::vector<Request*> added, passed;
        for (;;) {
            Request* r = nullptr;
            bool aged = true;
            {
                std::lock_guard<std::mutex> lk(S->mu);
                if (S->queue.empty() || S->stop) break;
                r = pick_locked(passed, &aged);
                if (!r) break;  // every queued solve was passed over this round
            }
            if (eng->live_count() >= eng->max_inst()) {
                std::lock_guard<std::mutex> lk(S->mu);
                S->st.head_blocked++;
                break;
            }
            if (eng->used_tiles() + r->tiles > eng->max_tiles()) {
                std::lock_guard<std::mutex> lk(S->mu);
                S->st.head_blocked++;
                if (aged) break;
                passed.push_back(r);
                continue;
            }
            const size_t before = mem.arena.used();
            int slot = -1;
            const int rc = eng->add(r->p, r->pv.data(), r->qw.data(), &slot, false);
            if (rc == HOSONO_ENOMEM && eng->live_count() > 0) {  // wait for a retirement
                std::lock_guard<std::mutex> lk(S->mu);
                S->st.head_blocked++;
                if (aged) break;
                passed.push_back(r);
                continue;
            }
            std::lock_guard<std::mutex> lk(S->mu);
            S->queue.erase(std::find(S->queue.begin(), S->queue.end(), r));
            if (rc == HOSONO_ECUDA) return rc;
            if (rc) {  // cannot ever be admitted
                finish_locked(S, r, rc);
                S->done.notify_all();
                continue;
            }
            r->info.state = HOSONO_REQ_RUNNING;
            r->info.slot = slot;
            r->info.admit_s = clock_s();
            r->lastStep_s = r->info.admit_s;
            r->info.device_bytes = (long long)(mem.arena.used() - before);
            S->resident.push_back(r);
            S->st.resident = (long long)S->resident.size();
            S->st.peak_resident = std::max(S->st.peak_resident, S->st.resident);
            S->st.used_bytes = (long long)mem.arena.used();
            S->st.peak_bytes = std::max(S->st.peak_bytes, S->st.used_bytes);
            S->st.queued = (long long)S->queue.size();
            added.push_back(r);
        }
        if (added.empty()) return HOSONO_OK;
        int rc = eng->commit_tables();
        for (Request* r : added) {
            if (!rc)
                rc = r->devIC ? eng->ic(r->info.slot, r->ic, r->xtab.data(), r->ytab.data())
                              : eng->upload(r->info.slot, r->U.data(), r->V.empty() ? nullptr : r->V.data());
            if (!rc) rc = eng->set_time(r->info.slot, 0.0, r->tmax, 0, r->nstepmax);
            r->U = std::vector<double>();
            r->V = std::vector<double>();
            r->xtab = std::vector<double>();
            r->ytab = std::vector<double>();
        }
        return rc;
    }

    int serve_snapshots() {
        for (;;) {
            Snapshot* sn = nullptr;
            int slot = -1;
            {
                std::lock_guard<std::mutex> lk(S->mu);
                if (S->snaps.empty()) return HOSONO_OK;
                sn = S->snaps.front();
                S->snaps.pop_front();
                auto it = S->reqs.find(sn->id);
                if (it != S->reqs.end() && it->second->info.state == HOSONO_REQ_RUNNING) slot = it->second->info.slot;
            }
            int status = HOSONO_EINVAL;
            if (slot >= 0) {
                InstState s{};
                int rc = eng->state(slot, &s);
                if (!rc) rc = eng->download(slot, sn->U, sn->V, sn->scheme);
                if (rc == HOSONO_ECUDA) return rc;
                status = rc;
                sn->t = s.t;
                sn->nstep = s.nstep;
            }
            {
                std::lock_guard<std::mutex> lk(S->mu);
                sn->status = status;
            }
            S->done.notify_all();
        }
    }

    // SHORTEST: which residents step in the next launch.  A solve that has
    // not stepped yet (no dt known) or has sat out aging_s seconds steps;
    // then the least estimated remaining work first until fill_tiles tiles
    // step.  The others hold (state untouched).
    int choose_holds() {
        const InstState* hs = eng->host_states();
        const double now = clock_s();
        std::vector<std::pair<double, Request*>> rest;
        std::vector<int> hold(eng->max_inst(), 1);
        int tiles = 0;
        {
            std::lock_guard<std::mutex> lk(S->mu);
            for (Request* r : S->resident) {
                const InstState& st = hs[r->info.slot];
                if (r->info.nstep == 0 || !(st.dt > 0) || now - r->lastStep_s >= S->cfg.aging_s) {
                    hold[r->info.slot] = 0;
                    tiles += r->tiles;
                } else {
                    const double left = std::max(0.0, r->tmax - st.t) / st.dt;
                    rest.emplace_back((double)r->p.nx * r->p.ny * std::min(left, (double)(r->nstepmax - st.nstep)), r);
                }
            }
        }
        std::sort(rest.begin(), rest.end(),
                  [](const std::pair<double, Request*>& a, const std::pair<double, Request*>& b) {
                      return a.first < b.first;
                  });
        for (const auto& w : rest) {
            if (tiles >= S->cfg.fill_tiles) break;
            hold[w.second->info.slot] = 0;
            tiles += w.second->tiles;
        }
        return eng->set_holds(hold.data());
    }

    int launch() {
        int steps = 1;
        if (msPerStep > 0) {
            const double want = S->cfg.chunk_ms / msPerStep;
            steps = (int)std::max(1.0, std::min((double)S->cfg.max_chunk_steps, std::floor(want)));
        }
        if (S->cfg.policy == HOSONO_SERVE_SHORTEST)
            if (int rc = choose_holds()) return rc;
        {
            std::lock_guard<std::mutex> lk(S->mu);
            for (Request* r : S->resident) r->baseNstep = r->info.nstep;
        }
        const double t0 = clock_s();
        const int rc = eng->run(steps);
        const double el = (clock_s() - t0) * 1e3;
        if (rc) return rc;
        const InstState* hs = eng->host_states();
        int taken = 0;
        const double now = clock_s();
        std::lock_guard<std::mutex> lk(S->mu);
        for (Request* r : S->resident) {
            const InstState& s = hs[r->info.slot];
            r->info.nstep = s.nstep;
            r->info.t = s.t;
            taken = std::max(taken, s.nstep - r->baseNstep);
            if (s.nstep > r->baseNstep) r->lastStep_s = now;
        }
        if (taken > 0) msPerStep = el / taken;
        S->st.chunks++;
        S->st.steps += taken;
        return HOSONO_OK;
    }

    int retire() {
        const InstState* hs = eng->host_states();
        std::vector<Request*> leaving;
        {
            std::lock_guard<std::mutex> lk(S->mu);
            for (Request* r : S->resident)
                if (hs[r->info.slot].done || hs[r->info.slot].error) leaving.push_back(r);
        }
        if (leaving.empty()) return HOSONO_OK;
        std::vector<int> status(leaving.size(), HOSONO_OK);
        for (size_t i = 0; i < leaving.size(); i++) {
            Request* r = leaving[i];
            const InstState s = hs[r->info.slot];
            status[i] = s.error;
            if (r->outU || r->outV || r->outScheme) {
                const int rc = eng->download(r->info.slot, r->outU, r->outV, r->outScheme);
                if (rc) return rc;
            }
            r->info.nstep = s.nstep;
            r->info.t = s.t;
            r->info.zone_updates = (long long)r->p.nx * r->p.ny * s.nstep;
            fill_mood(r->info, s);
            const int rc = eng->remove(r->info.slot, false);
            if (rc) return rc;
        }
        const int rc = eng->commit_tables();
        std::lock_guard<std::mutex> lk(S->mu);
        for (size_t i = 0; i < leaving.size(); i++) {
            Request* r = leaving[i];
            S->resident.erase(std::find(S->resident.begin(), S->resident.end(), r));
            finish_locked(S, r, status[i]);
        }
        S->st.resident = (long long)S->resident.size();
        S->st.used_bytes = (long long)mem.arena.used();
        S->done.notify_all();
        return rc;
    }

    void shutdown() {
        {
            std::lock_guard<std::mutex> lk(S->mu);
            for (Request* r : S->queue) finish_locked(S, r, HOSONO_ECANCELED);
            S->queue.clear();
            for (Request* r : S->resident) finish_locked(S, r, HOSONO_ECANCELED);
            S->resident.clear();
            for (Snapshot* sn : S->snaps) sn->status = HOSONO_ECANCELED;
            S->snaps.clear();
            S->st.queued = S->st.resident = 0;
        }
        S->done.notify_all();
        eng.reset();  // frees instance memory into the arena
        if (mem.base) cudaFree(mem.base);
        mem.base = nullptr;
    }
};

}  // namespace

extern "C" {

double hosono_serve_clock(void) { return clock_s(); }

int hosono_serve_create(const hosono_serve_config* cfg, hosono_server** out) {
    if (!out) return HOSONO_EINVAL;
    *out = nullptr;
    hosono_serve_config c{};
    if (cfg) c = *cfg;
    if (c.max_resident <= 0) c.max_resident = 1024;
    if (!(c.chunk_ms > 0)) c.chunk_ms = 25.0;
    if (c.max_chunk_steps <= 0) c.max_chunk_steps = 64;
    if (c.fp_mode != HOSONO_FP_STRICT && c.fp_mode != HOSONO_FP_FAST) return HOSONO_EINVAL;
    if (c.policy != HOSONO_SERVE_FIFO && c.policy != HOSONO_SERVE_SHORTEST) return HOSONO_EINVAL;
    if (!(c.aging_s > 0)) c.aging_s = 5.0;
    if (c.fill_tiles <= 0) {
        int dev = 0, sms = 148;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
                                                      cudaSuccess) {
            cudaGetLastError();
            sms = 148;
        }
        c.fill_tiles = 40 * sms;
    }
    hosono_server* S = new (std::nothrow) hosono_server();
    if (!S) return HOSONO_ENOMEM;
    S->cfg = c;
    if (cudaGetDevice(&S->device) != cudaSuccess) {
        cudaGetLastError();
        delete S;
        return HOSONO_ECUDA;
    }
    try {
        S->th = std::thread([S] { Scheduler(S).main(); });
    } catch (...) {
        delete S;
        return HOSONO_ENOMEM;
    }
    int rc;
    {
        std::unique_lock<std::mutex> lk(S->mu);
        S->done.wait(lk, [&] { return S->started; });
        rc = S->startRc;
    }
    if (rc) {
        S->th.join();
        delete S;
        return rc;
    }
    *out = S;
    return HOSONO_OK;
}

int hosono_serve_destroy(hosono_server* S) {
    if (!S) return HOSONO_OK;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->wake.notify_all();
    if (S->th.joinable()) S->th.join();
    {  // every solve is done now; blocked callers return before the server goes
        std::unique_lock<std::mutex> lk(S->mu);
        S->done.notify_all();
        S->done.wait(lk, [&] { return S->inflight == 0; });
    }
    delete S;
    return HOSONO_OK;
}

static int submit_common(hosono_server* S, const hosono_params* p, const double* pv, const double* qw,
                         const int* stenc, const double* U, const double* V, const hosono_ic_desc* ic,
                         const double* xtab, const double* ytab, double tmax, int nstepmax, double* U_out,
                         double* V_out, int* scheme_out, long long* id);

int hosono_serve_submit(hosono_server* S, const hosono_params* p, const double* pv, const double* qw, const int* stenc,
                        const double* U, const double* V, double tmax, int nstepmax, double* U_out, double* V_out,
                        int* scheme_out, long long* id) {
    if (!U) return HOSONO_EINVAL;
    return submit_common(S, p, pv, qw, stenc, U, V, nullptr, nullptr, nullptr, tmax, nstepmax, U_out, V_out,
                         scheme_out, id);
}

int hosono_serve_submit_ic(hosono_server* S, const hosono_params* p, const double* pv, const double* qw,
                           const int* stenc, const hosono_ic_desc* ic, const double* xtab, const double* ytab,
                           double tmax, int nstepmax, double* U_out, double* V_out, int* scheme_out, long long* id) {
    if (!ic || !xtab || !ytab) return HOSONO_EINVAL;
    return submit_common(S, p, pv, qw, stenc, nullptr, nullptr, ic, xtab, ytab, tmax, nstepmax, U_out, V_out,
                         scheme_out, id);
}

static int submit_common(hosono_server* S, const hosono_params* p, const double* pv, const double* qw,
                         const int* stenc, const double* U, const double* V, const hosono_ic_desc* ic,
                         const double* xtab, const double* ytab, double tmax, int nstepmax, double* U_out,
                         double* V_out, int* scheme_out, long long* id) {
    if (!S || !p || !pv || !qw || !id) return HOSONO_EINVAL;
    if (!params_ok(*p) || !stencil_ok(p->max_radius, stenc) || std::isnan(tmax) || nstepmax < 0) {
        std::lock_guard<std::mutex> lk(S->mu);
        return S->fail(HOSONO_EINVAL, "invalid solve parameters");
    }
    const int R = p->max_radius;
    const size_t nsMax = 1 + 2 * R * (R + 1), nqMax = R + 1;
    const size_t cells = (size_t)(p->nx + 2 * p->ngc) * (size_t)(p->ny + 2 * p->ngc);
    std::unique_ptr<Request> r(new (std::nothrow) Request());
    if (!r) return HOSONO_ENOMEM;
    try {
        r->pv.assign(pv, pv + nsMax * nqMax * 4 * R);
        r->qw.assign(qw, qw + nqMax * R);
        if (ic) {
            r->devIC = true;
            r->ic = *ic;
            const size_t nxt = (size_t)(p->nx + 2 * p->ngc), nyt = (size_t)(p->ny + 2 * p->ngc);
            r->xtab.assign(xtab, xtab + 3 * nxt);
            r->ytab.assign(ytab, ytab + 2 * nyt);
        } else {
            r->U.assign(U, U + cells * NCONS);
            if (V) r->V.assign(V, V + cells * NPRIM);
        }
    } catch (...) {
        return HOSONO_ENOMEM;
    }
    r->p = *p;
    r->tmax = tmax;
    r->nstepmax = nstepmax > 0 ? nstepmax : INT_MAX;
    r->outU = U_out;
    r->outV = V_out;
    r->outScheme = scheme_out;
    r->tiles = hosono_batch_tiles_for(p);
    r->work = (double)p->nx * p->ny * (std::isfinite(tmax) ? std::max(tmax, 0.0) : 1e30) / std::min(p->dx, p->dy);
    const long long bytes = hosono_batch_instance_bytes(p);
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->fatal) return S->fail(S->fatal, "server stopped after an error; " + S->msg);
    if (bytes > S->budget || r->tiles > S->maxTiles)
        return S->fail(HOSONO_ENOMEM, "solve needs more device memory than the server's whole budget");
    r->info.id = S->nextId++;
    r->info.state = HOSONO_REQ_QUEUED;
    r->info.slot = -1;
    r->info.submit_s = clock_s();
    *id = r->info.id;
    S->queue.push_back(r.get());
    S->reqs[r->info.id] = std::move(r);
    S->st.submitted++;
    S->st.queued = (long long)S->queue.size();
    S->wake.notify_all();
    return HOSONO_OK;
}

int hosono_serve_wait(hosono_server* S, long long id, double timeout_s, hosono_request_info* info) {
    if (!S) return HOSONO_EINVAL;
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return S->fail(HOSONO_EINVAL, "unknown solve id");
    Request* r = it->second.get();
    auto ready = [&] { return r->info.state == HOSONO_REQ_DONE; };
    S->inflight++;
    bool ok = true;
    if (timeout_s < 0)
        S->done.wait(lk, ready);
    else
        ok = S->done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready);
    if (ok && info) *info = r->info;
    S->inflight--;
    S->done.notify_all();
    return ok ? HOSONO_OK : HOSONO_ETIMEOUT;
}

int hosono_serve_release(hosono_server* S, long long id) {
    if (!S) return HOSONO_EINVAL;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return S->fail(HOSONO_EINVAL, "unknown solve id");
    if (it->second->info.state != HOSONO_REQ_DONE) return S->fail(HOSONO_EINVAL, "solve is not done");
    S->reqs.erase(it);
    return HOSONO_OK;
}

int hosono_serve_poll(hosono_server* S, long long* ids, int cap, int* n) {
    if (!S || !n || (cap > 0 && !ids)) return HOSONO_EINVAL;
    std::lock_guard<std::mutex> lk(S->mu);
    int k = 0;
    while (k < cap && !S->finished.empty()) {
        ids[k++] = S->finished.front();
        S->finished.pop_front();
    }
    *n = k;
    return HOSONO_OK;
}

int hosono_serve_info(hosono_server* S, long long id, hosono_request_info* info) {
    if (!S || !info) return HOSONO_EINVAL;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return S->fail(HOSONO_EINVAL, "unknown solve id");
    *info = it->second->info;
    return HOSONO_OK;
}

int hosono_serve_snapshot(hosono_server* S, long long id, double* U, double* V, int* scheme, double* t, int* nstep) {
    if (!S) return HOSONO_EINVAL;
    Snapshot sn;
    sn.id = id;
    sn.U = U;
    sn.V = V;
    sn.scheme = scheme;
    std::unique_lock<std::mutex> lk(S->mu);
    if (S->stop || S->fatal) return S->fail(HOSONO_ECANCELED, "server is stopping");
    S->snaps.push_back(&sn);
    S->wake.notify_all();
    S->inflight++;
    S->done.wait(lk, [&] { return sn.status >= 0; });
    S->inflight--;
    S->done.notify_all();
    if (sn.status == HOSONO_EINVAL) return S->fail(HOSONO_EINVAL, "solve is not resident");
    if (t) *t = sn.t;
    if (nstep) *nstep = sn.nstep;
    return sn.status;
}

int hosono_serve_drain(hosono_server* S, double timeout_s) {
    if (!S) return HOSONO_EINVAL;
    std::unique_lock<std::mutex> lk(S->mu);
    auto idle = [&] { return (S->queue.empty() && S->resident.empty()) || S->fatal || S->stop; };
    S->inflight++;
    bool ok = true;
    if (timeout_s < 0)
        S->done.wait(lk, idle);
    else
        ok = S->done.wait_for(lk, std::chrono::duration<double>(timeout_s), idle);
    S->inflight--;
    S->done.notify_all();
    return ok ? S->fatal : HOSONO_ETIMEOUT;
}

int hosono_serve_stats(hosono_server* S, hosono_serve_totals* st) {
    if (!S || !st) return HOSONO_EINVAL;
    std::lock_guard<std::mutex> lk(S->mu);
    *st = S->st;
    return HOSONO_OK;
}

int hosono_serve_last_error(hosono_server* S, char* buf, int len) {
    if (!S) return HOSONO_EINVAL;
    std::lock_guard<std::mutex> lk(S->mu);
    if (buf && len > 0) std::snprintf(buf, (size_t)len, "%s", S->msg.c_str());
    return S->err;
}

}  // extern "C"
