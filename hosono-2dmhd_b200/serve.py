"""Serving form of the solver: a request loop over ``hosono_serve_*``.

``Server`` wraps the native server (include/hosono_gpu.h): a scheduler thread
in the library owns one batch on the GPU, admits queued solves while an
instance slot and a free range of its device-memory budget are available,
advances every resident solve in the same batched launches (continuous
batching) and hands back each final state.  Nothing here computes physics;
the compute path is the library's CUDA path only.

``run_stream`` drives a seeded request stream (a workload manifest such as
workloads/served2000_seed1.json) as an open loop: request i is submitted at
its arrival time, t0 + sum(gap[:i+1]) / rate, whatever the server is doing.
Solves are prepared (``.par`` -> parameters, GP tables, initial state, all on
the host as the reference's setup does) by a producer thread a few requests
ahead of their arrival.  The report gives latency percentiles (submit to
finish, on the server's clock) beside zone-updates/s.
"""
import ctypes
import os
import queue
import tempfile
import threading
import time

import numpy as np

from . import (ECANCELED, ETIMEOUT, FP_STRICT, SERVE_FIFO, SERVE_SHORTEST, HosonoError, RequestInfo, ServeConfig, ServeTotals,
               _p, ic_describe, ic_set, load_library, par_gp, par_load)
from . import problems


def clock():
    """Seconds on the server clock (the one RequestInfo timestamps use)."""
    return load_library().hosono_serve_clock()


class Server:
    """hosono_serve_*: admission by device-memory budget, continuous batching;
    policy SERVE_FIFO (the queue in order, every resident steps every launch)
    or SERVE_SHORTEST (least estimated work first, long residents sit out
    launches once the short ones fill `fill_tiles` tiles, an aging bound)."""

    def __init__(self, memory_budget=0, max_resident=0, fp_mode=FP_STRICT, chunk_ms=0.0, max_chunk_steps=0,
                 policy=SERVE_FIFO, aging_s=0.0, fill_tiles=0):
        self.lib = load_library()
        cfg = ServeConfig(int(memory_budget), int(max_resident), int(fp_mode), float(chunk_ms),
                          int(max_chunk_steps), int(policy), float(aging_s), int(fill_tiles), 0)
        h = ctypes.c_void_p()
        rc = self.lib.hosono_serve_create(ctypes.byref(cfg), ctypes.byref(h))
        if rc:
            raise HosonoError(rc, "hosono_serve_create")
        self.h = h
        self._outputs = {}  # id -> (U, V, scheme) arrays the library fills at the end
        self._lock = threading.Lock()

    def _check(self, rc, what):
        if rc:
            buf = ctypes.create_string_buffer(512)
            self.lib.hosono_serve_last_error(self.h, buf, 512)
            raise HosonoError(rc, f"{what}: {buf.value.decode()}")

    def close(self):
        if getattr(self, "h", None):
            self.lib.hosono_serve_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def submit(self, params, pv, qw, stenc, U, V, tmax, nstepmax=0, want_state=True, want_V=False,
               want_scheme=False):
        """Queue one solve; returns its id.  U and V (None: cons2prim(U) on
        the device) are copied by the library."""
        nxt, nyt = params.nx + 2 * params.ngc, params.ny + 2 * params.ngc
        U = np.ascontiguousarray(U, dtype=np.float64)
        assert U.size == nxt * nyt * 8
        if V is not None:
            V = np.ascontiguousarray(V, dtype=np.float64)
            assert V.size == nxt * nyt * 10
        pv = np.ascontiguousarray(pv, dtype=np.float64)
        qw = np.ascontiguousarray(qw, dtype=np.float64)
        st = np.ascontiguousarray(stenc, dtype=np.int32)
        Uo = np.empty((nyt, nxt, 8)) if want_state else None
        Vo = np.empty((nyt, nxt, 10)) if want_V else None
        So = np.empty((nyt, nxt), dtype=np.int32) if want_scheme else None
        rid = ctypes.c_longlong()
        self._check(self.lib.hosono_serve_submit(
            self.h, ctypes.byref(params), _p(pv), _p(qw), _p(st, ctypes.c_int), _p(U),
            _p(V) if V is not None else None, float(tmax), int(nstepmax),
            _p(Uo) if Uo is not None else None, _p(Vo) if Vo is not None else None,
            _p(So, ctypes.c_int) if So is not None else None, ctypes.byref(rid)), "submit")
        with self._lock:
            self._outputs[rid.value] = (Uo, Vo, So)
        return rid.value

    def submit_ic(self, params, pv, qw, stenc, desc, xtab, ytab, tmax, nstepmax=0, want_state=True):
        """Queue one solve whose initial state the server builds on the device
        from ic_describe's output (O(nx+ny) host data); returns its id."""
        nxt, nyt = params.nx + 2 * params.ngc, params.ny + 2 * params.ngc
        pv = np.ascontiguousarray(pv, dtype=np.float64)
        qw = np.ascontiguousarray(qw, dtype=np.float64)
        st = np.ascontiguousarray(stenc, dtype=np.int32)
        xt = np.ascontiguousarray(xtab, dtype=np.float64)
        yt = np.ascontiguousarray(ytab, dtype=np.float64)
        assert xt.size == 3 * nxt and yt.size == 2 * nyt
        Uo = np.empty((nyt, nxt, 8)) if want_state else None
        rid = ctypes.c_longlong()
        self._check(self.lib.hosono_serve_submit_ic(
            self.h, ctypes.byref(params), _p(pv), _p(qw), _p(st, ctypes.c_int), ctypes.byref(desc), _p(xt), _p(yt),
            float(tmax), int(nstepmax), _p(Uo) if Uo is not None else None, None, None, ctypes.byref(rid)),
            "submit_ic")
        with self._lock:
            self._outputs[rid.value] = (Uo, None, None)
        return rid.value

    def wait(self, rid, timeout=None, release=True):
        """Block until the solve is done; returns (info dict, U, V, scheme).
        With release (the default) the server then forgets the solve."""
        info = RequestInfo()
        rc = self.lib.hosono_serve_wait(self.h, int(rid), -1.0 if timeout is None else float(timeout),
                                        ctypes.byref(info))
        if rc == ETIMEOUT:
            raise TimeoutError(f"solve {rid} not done after {timeout} s")
        self._check(rc, "wait")
        if release and info.status != ECANCELED:  # a canceled solve: the server is shutting down
            self.release(rid)
        with self._lock:
            out = self._outputs.pop(int(rid), (None, None, None))
        return (info.as_dict(),) + tuple(out)

    def release(self, rid):
        """Forget a finished solve (its id becomes unknown to the server)."""
        self._check(self.lib.hosono_serve_release(self.h, int(rid)), "release")

    def info(self, rid):
        info = RequestInfo()
        self._check(self.lib.hosono_serve_info(self.h, int(rid), ctypes.byref(info)), "info")
        return info.as_dict()

    def poll(self, cap=1024):
        ids = (ctypes.c_longlong * cap)()
        n = ctypes.c_int()
        self._check(self.lib.hosono_serve_poll(self.h, ids, int(cap), ctypes.byref(n)), "poll")
        return list(ids[:n.value])

    def snapshot(self, rid, shape_of):
        """Current state of a resident solve: (t, nstep, U, V, scheme)."""
        nxt, nyt = shape_of.nx + 2 * shape_of.ngc, shape_of.ny + 2 * shape_of.ngc
        U = np.empty((nyt, nxt, 8))
        V = np.empty((nyt, nxt, 10))
        S = np.empty((nyt, nxt), dtype=np.int32)
        t = ctypes.c_double()
        n = ctypes.c_int()
        self._check(self.lib.hosono_serve_snapshot(self.h, int(rid), _p(U), _p(V), _p(S, ctypes.c_int),
                                                   ctypes.byref(t), ctypes.byref(n)), "snapshot")
        return t.value, n.value, U, V, S

    def drain(self, timeout=None):
        rc = self.lib.hosono_serve_drain(self.h, -1.0 if timeout is None else float(timeout))
        if rc == ETIMEOUT:
            raise TimeoutError("server did not drain")
        self._check(rc, "drain")

    def stats(self):
        s = ServeTotals()
        self._check(self.lib.hosono_serve_stats(self.h, ctypes.byref(s)), "stats")
        return s.as_dict()


def prepare(entry, workdir, device_ic=False):
    """Host set-up of one manifest entry, as the reference's mhd_driver init:
    (params, pv, qw, stenc, U, V, tmax); with device_ic, U and V are replaced
    by the (ICDesc, xtab, ytab) the server builds them from on the device."""
    kv = problems.from_entry(entry)
    par = problems.make(workdir, f"req{entry['id']}", kv)
    p, run = par_load(par)
    pv, qw, st = par_gp(par, p.max_radius)
    if device_ic:
        U, V = None, ic_describe(par, p)
    else:
        U, V = ic_set(par, p)
    os.remove(par)
    return p, pv, qw, st, U, V, run.tmax


def percentile(xs, q):
    xs = sorted(xs)
    if not xs:
        return float("nan")
    k = (len(xs) - 1) * q / 100.0
    lo, hi = int(np.floor(k)), int(np.ceil(k))
    return xs[lo] + (xs[hi] - xs[lo]) * (k - lo)


def run_stream(entries, rate, server, keep=(), prefetch=6, fp_mode=FP_STRICT, closed=False, device_ic=False):
    """Submit `entries` with arrival gaps entry['gap'] / rate seconds (open
    loop), or all at once (closed=True); wait for every solve.  Returns the
    report dict and {id in keep: final U}."""
    keep = set(keep)
    work = tempfile.mkdtemp(prefix="hosono_serve_")
    ready = queue.Queue(maxsize=max(1, prefetch))
    errors = []

    def producer():
        try:
            for e in entries:
                p, pv, qw, st, U, V, tmax = prepare(e, work, device_ic)
                p.fp_mode = fp_mode
                ready.put((e, p, pv, qw, st, U, V, tmax))
        except Exception as exc:  # surfaced by the submitter
            errors.append(exc)
            ready.put(None)

    th = threading.Thread(target=producer, daemon=True)
    th.start()
    sched = []
    t0 = clock()
    due = t0
    ids = []
    for _ in entries:
        item = ready.get()
        if item is None:
            raise errors[0]
        e, p, pv, qw, st, U, V, tmax = item
        if not closed:
            due += float(e["gap"]) / rate
            while True:
                wait = due - clock()
                if wait <= 0:
                    break
                time.sleep(min(wait, 0.05))
        if device_ic:
            rid = server.submit_ic(p, pv, qw, st, *V, tmax, want_state=e["id"] in keep)
        else:
            rid = server.submit(p, pv, qw, st, U, V, tmax, want_state=e["id"] in keep)
        ids.append((e, rid, due))
    th.join()
    kept = {}
    infos = []
    for e, rid, due in ids:
        info, Uo, _, _ = server.wait(rid)
        info["entry"] = e["id"]
        info["due"] = due
        infos.append(info)
        if e["id"] in keep:
            kept[e["id"]] = Uo
    ok = [i for i in infos if i["status"] == 0]
    lat = [i["finish_s"] - i["submit_s"] for i in ok]
    qwait = [i["admit_s"] - i["submit_s"] for i in ok]
    lag = [max(0.0, i["submit_s"] - i["due"]) for i in infos] if not closed else [0.0]
    first = min(i["submit_s"] for i in infos)
    last = max(i["finish_s"] for i in infos)
    zu = sum(i["zone_updates"] for i in ok)
    st = server.stats()
    report = dict(
        requests=len(infos), completed=len(ok), failed=len(infos) - len(ok),
        failed_status=sorted({i["status"] for i in infos if i["status"] != 0}),
        zone_updates=zu, makespan_s=last - first, zone_updates_per_s=zu / (last - first),
        latency_p50_s=percentile(lat, 50), latency_p99_s=percentile(lat, 99), latency_max_s=max(lat) if lat else None,
        queue_wait_p50_s=percentile(qwait, 50), queue_wait_p99_s=percentile(qwait, 99),
        submit_lag_max_s=max(lag), rate_per_s=None if closed else rate,
        peak_resident=st["peak_resident"], peak_bytes=st["peak_bytes"], budget_bytes=st["budget_bytes"],
        head_blocked=st["head_blocked"], chunks=st["chunks"], batch_steps=st["steps"],
        gpu_busy_frac=st["busy_s"] / (last - first), admin_s=st["admin_s"])
    return report, kept, infos
