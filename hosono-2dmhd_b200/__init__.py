"""hosono-2DMHD time-step path on B200: Python binding of libhosono_gpu.so.

The native library (include/hosono_gpu.h) replaces the reference's
``cfl_computedt`` (src/cfl.f90:14-52) and ``timeStep_advanceSolution``
(src/timeStep.f90:22-43) with FP64 CUDA kernels for sm_100a.  This module
is a thin ctypes layer over that C ABI; the compute path is the native one
only, and every entry point raises if the library or a GPU is missing.

Host arrays use the reference's layout, shaped (nyTot, nxTot, nvar) in numpy
(Fortran ``U(var, i, j)`` with var fastest), guard cells included.
"""
import ctypes
import os

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libhosono_gpu.so")

OK, EINVAL, ENOMEM, ECUDA, ENANDT, EMOODCAP, ETIMEOUT, EPAR, ENOTBUILT, ECANCELED = range(10)
BC_OUTFLOW, BC_PERIODIC = 0, 1
FP_STRICT, FP_FAST = 0, 1
STATUS_NAMES = {OK: "OK", EINVAL: "EINVAL", ENOMEM: "ENOMEM", ECUDA: "ECUDA", ENANDT: "ENANDT",
                EMOODCAP: "EMOODCAP", ETIMEOUT: "ETIMEOUT", EPAR: "EPAR", ENOTBUILT: "ENOTBUILT",
                ECANCELED: "ECANCELED"}


class HosonoError(RuntimeError):
    def __init__(self, code, msg=""):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


class Params(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("ngc", ctypes.c_int), ("max_radius", ctypes.c_int),
                ("bc", ctypes.c_int), ("force_hydro", ctypes.c_int), ("riemann_solver", ctypes.c_int),
                ("fp_mode", ctypes.c_int), ("dx", ctypes.c_double), ("dy", ctypes.c_double),
                ("mindxdy", ctypes.c_double), ("maxdxdy", ctypes.c_double), ("gamma", ctypes.c_double),
                ("small_pressure", ctypes.c_double), ("small_density", ctypes.c_double),
                ("small_energy", ctypes.c_double), ("small_b", ctypes.c_double), ("cfl", ctypes.c_double)]


class RunInfo(ctypes.Structure):
    _fields_ = [("tmax", ctypes.c_double), ("nstepmax", ctypes.c_int), ("output_freq_step", ctypes.c_int),
                ("output_freq_time", ctypes.c_double), ("ell_over_delta", ctypes.c_double),
                ("x_beg", ctypes.c_double), ("x_end", ctypes.c_double), ("y_beg", ctypes.c_double),
                ("y_end", ctypes.c_double), ("nx_tot", ctypes.c_int), ("ny_tot", ctypes.c_int),
                ("ic_type", ctypes.c_char * 32), ("data_file_base", ctypes.c_char * 256)]


class Stats(ctypes.Structure):
    _fields_ = [("stages", ctypes.c_int), ("mood_passes", ctypes.c_int), ("max_passes", ctypes.c_int),
                ("detect_lowered", ctypes.c_longlong), ("inner_lowered", ctypes.c_longlong),
                ("cascade_iters", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServeConfig(ctypes.Structure):
    _fields_ = [("memory_budget", ctypes.c_longlong), ("max_resident", ctypes.c_int), ("fp_mode", ctypes.c_int),
                ("chunk_ms", ctypes.c_double), ("max_chunk_steps", ctypes.c_int), ("policy", ctypes.c_int),
                ("aging_s", ctypes.c_double), ("fill_tiles", ctypes.c_int), ("pad", ctypes.c_int)]


SERVE_FIFO, SERVE_SHORTEST = 0, 1


class RequestInfo(ctypes.Structure):
    _fields_ = [("id", ctypes.c_longlong), ("state", ctypes.c_int), ("status", ctypes.c_int),
                ("nstep", ctypes.c_int), ("slot", ctypes.c_int), ("t", ctypes.c_double),
                ("zone_updates", ctypes.c_longlong), ("device_bytes", ctypes.c_longlong),
                ("submit_s", ctypes.c_double), ("admit_s", ctypes.c_double), ("finish_s", ctypes.c_double),
                ("mood", Stats)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "mood"}
        d["mood"] = self.mood.as_dict()
        return d


class ServeTotals(ctypes.Structure):
    _fields_ = [(k, ctypes.c_longlong) for k in ("submitted", "completed", "failed", "queued", "resident",
                                                  "zone_updates", "chunks", "steps", "peak_resident",
                                                  "budget_bytes", "used_bytes", "peak_bytes", "head_blocked")] + \
               [("busy_s", ctypes.c_double), ("admin_s", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class LaunchInfo(ctypes.Structure):
    _fields_ = [("tiles", ctypes.c_int), ("sms", ctypes.c_int), ("pass1_grid", ctypes.c_int),
                ("tile_grid_max", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Tuning(ctypes.Structure):
    _fields_ = [("pass1_staging", ctypes.c_int), ("pass1_schedule", ctypes.c_int),
                ("pass1_blocks_per_sm", ctypes.c_int), ("later_passes", ctypes.c_int),
                ("pass1_boxes", ctypes.c_int), ("upload_bands", ctypes.c_int), ("pdl", ctypes.c_int),
                ("update_staging", ctypes.c_int)]
    KEYS = ("pass1_staging", "pass1_schedule", "pass1_blocks_per_sm", "later_passes", "pass1_boxes", "upload_bands",
            "pdl", "update_staging")

    def as_dict(self):
        return {k: getattr(self, k) for k in self.KEYS}

    def update(self, kw):
        for k, v in kw.items():
            if k not in self.KEYS:
                raise TypeError(f"unknown tuning field {k!r} (one of {', '.join(self.KEYS)})")
            setattr(self, k, int(v))


STAGE_CP_ASYNC, STAGE_TMA = 0, 1
SCHED_STATIC, SCHED_DYNAMIC = 0, 1
LATER_KERNELS, LATER_PERSISTENT = 0, 1
TUNE_MAX = 12
UPLOAD_BANDS_MAX = 16


class TuneReport(ctypes.Structure):
    _fields_ = [("candidates", ctypes.c_int), ("cached", ctypes.c_int), ("size_class", ctypes.c_int),
                ("instances", ctypes.c_int), ("tried", Tuning * TUNE_MAX), ("ms", ctypes.c_double * TUNE_MAX),
                ("best", Tuning)]

    def as_dict(self):
        return {"cached": bool(self.cached), "size_class": self.size_class, "instances": self.instances,
                "best": self.best.as_dict(),
                "table": [dict(self.tried[k].as_dict(), pass1_ms=self.ms[k]) for k in range(self.candidates)]}


class ICDesc(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int), ("pad", ctypes.c_int), ("c", ctypes.c_double * 16)]


REQ_QUEUED, REQ_RUNNING, REQ_DONE = 0, 1, 2

# Every symbol the C ABI exports (include/hosono_gpu.h), with its signature.
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p
_cp = ctypes.c_char_p
_i = ctypes.c_int
_d = ctypes.c_double
SIGNATURES = {
    "hosono_gp_build": [_i, _cp, _cp, _i, _cp, _cp, _i, _cp, _dp, _dp, _ip],
    "hosono_par_load": [_cp, ctypes.POINTER(Params), ctypes.POINTER(RunInfo), _cp, _i],
    "hosono_par_gp": [_cp, _dp, _dp, _ip, _cp, _i],
    "hosono_gp_cache_info": [ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong), _ip],
    "hosono_gp_cache_clear": [],
    "hosono_ic_set": [_cp, ctypes.POINTER(Params), _dp, _dp, _cp, _i],
    "hosono_gpu_create": [ctypes.POINTER(Params), _dp, _dp, _ip, ctypes.POINTER(_vp)],
    "hosono_gpu_destroy": [_vp],
    "hosono_gpu_upload": [_vp, _dp, _dp],
    "hosono_gpu_download": [_vp, _dp, _dp, _ip],
    "hosono_gpu_cfl": [_vp, _dp],
    "hosono_gpu_advance": [_vp, _d],
    "hosono_gpu_run": [_vp, _d, _i, _i, _dp, _ip],
    "hosono_gpu_advance_host": [_vp, _d, _dp, _dp],
    "hosono_gpu_stats": [_vp, ctypes.POINTER(Stats)],
    "hosono_gpu_last_error": [_vp, _cp, _i],
    "hosono_gpu_trace_enable": [_vp, _i],
    "hosono_gpu_trace_count": [_vp],
    "hosono_gpu_trace_get": [_vp, _i, _ip, _vp, _vp],
    "hosono_gpu_trace_clear": [_vp],
    "hosono_gpu_module_set": [_vp, _ip, _ip, _ip],
    "hosono_gpu_module_get": [_vp, _dp, _dp, _dp, _dp, _ip, _ip, _ip],
    "hosono_gpu_reconstruct": [_vp],
    "hosono_gpu_getfluxes": [_vp],
    "hosono_gpu_flicd": [_vp],
    "hosono_gpu_update": [_vp, _d],
    "hosono_gpu_detect": [_vp, _ip],
    "hosono_gpu_bc": [_vp, _i],
    "hosono_gpu_bc_mood": [_vp],
    "hosono_gpu_mood_pass_stats": [_vp, _ip, ctypes.POINTER(ctypes.c_longlong)],
    "hosono_gpu_riemann": [_vp, _i, _vp, _vp, _i, _vp],
    "hosono_gpu_eigenvecs": [_vp, _i, _vp, _i, _i, _vp, _vp],
    "hosono_gpu_state_layout": [_vp, ctypes.POINTER(_vp), _ip, ctypes.POINTER(ctypes.c_longlong)],
    "hosono_gpu_build_info": [_ip, _ip],
    "hosono_gpu_set_device": [_i],
    "hosono_gpu_stream": [_vp, ctypes.POINTER(_vp)],
    "hosono_gpu_launch_info": [_vp, ctypes.POINTER(LaunchInfo)],
    "hosono_gpu_set_tuning": [_vp, ctypes.POINTER(Tuning)],
    "hosono_gpu_autotune": [_vp, _i, _i, ctypes.POINTER(TuneReport)],
    "hosono_batch_autotune": [_vp, _i, _i, ctypes.POINTER(TuneReport)],
    "hosono_gpu_get_tuning": [_vp, ctypes.POINTER(Tuning)],
    "hosono_batch_set_tuning": [_vp, ctypes.POINTER(Tuning)],
    "hosono_batch_get_tuning": [_vp, ctypes.POINTER(Tuning)],
    "hosono_gpu_profile": [_vp, _i],
    "hosono_gpu_profile_read": [_vp, _dp, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong), _i],
    "hosono_cfl_noalloc": [_vp, _i, _i, _i, _i, ctypes.c_longlong, _d, _d, _d, _i, _vp, _vp],
    "hosono_gpu_set_time": [_vp, _d, _d, _i, _i],
    "hosono_gpu_set_mood_cap": [_vp, _i],
    "hosono_batch_set_mood_cap": [_vp, _i, _i],
    "hosono_gpu_step": [_vp, _i, _dp, _ip],
    "hosono_gpu_set_graphs": [_vp, _i],
    "hosono_batch_create": [_i, _i, _i, ctypes.POINTER(_vp)],
    "hosono_batch_destroy": [_vp],
    "hosono_batch_tiles_for": [ctypes.POINTER(Params)],
    "hosono_batch_instance_bytes": [ctypes.POINTER(Params)],
    "hosono_batch_add": [_vp, ctypes.POINTER(Params), _dp, _dp, _ip, _ip],
    "hosono_batch_remove": [_vp, _i],
    "hosono_batch_upload": [_vp, _i, _dp, _dp],
    "hosono_batch_download": [_vp, _i, _dp, _dp, _ip],
    "hosono_batch_set_time": [_vp, _i, _d, _d, _i, _i],
    "hosono_batch_run": [_vp, _i],
    "hosono_batch_status": [_vp, _i, _dp, _dp, _ip, _ip, _ip],
    "hosono_batch_stats": [_vp, _i, ctypes.POINTER(Stats)],
    "hosono_batch_stream": [_vp, ctypes.POINTER(_vp)],
    "hosono_batch_set_graphs": [_vp, _i],
    "hosono_batch_last_error": [_vp, _cp, _i],
    "hosono_batch_capacity": [_vp, _ip, _ip, _ip, _ip],
    "hosono_ic_describe": [_cp, ctypes.POINTER(Params), ctypes.POINTER(ICDesc), _dp, _dp, _cp, _i],
    "hosono_gpu_ic": [_vp, ctypes.POINTER(ICDesc), _dp, _dp],
    "hosono_batch_ic": [_vp, _i, ctypes.POINTER(ICDesc), _dp, _dp],
    "hosono_serve_submit_ic": [_vp, ctypes.POINTER(Params), _dp, _dp, _ip, ctypes.POINTER(ICDesc), _dp, _dp, _d, _i,
                               _dp, _dp, _ip, ctypes.POINTER(ctypes.c_longlong)],
    "hosono_gpu_diagnostics": [_vp, _dp, _ip, _ip, _dp, _dp],
    "hosono_batch_diagnostics": [_vp, _i, _dp, _ip, _ip, _dp, _dp],
    "hosono_serve_clock": [],
    "hosono_serve_create": [ctypes.POINTER(ServeConfig), ctypes.POINTER(_vp)],
    "hosono_serve_destroy": [_vp],
    "hosono_serve_submit": [_vp, ctypes.POINTER(Params), _dp, _dp, _ip, _dp, _dp, _d, _i, _dp, _dp, _ip,
                            ctypes.POINTER(ctypes.c_longlong)],
    "hosono_serve_wait": [_vp, ctypes.c_longlong, _d, ctypes.POINTER(RequestInfo)],
    "hosono_serve_release": [_vp, ctypes.c_longlong],
    "hosono_serve_poll": [_vp, ctypes.POINTER(ctypes.c_longlong), _i, _ip],
    "hosono_serve_info": [_vp, ctypes.c_longlong, ctypes.POINTER(RequestInfo)],
    "hosono_serve_snapshot": [_vp, ctypes.c_longlong, _dp, _dp, _ip, _dp, _ip],
    "hosono_serve_drain": [_vp, _d],
    "hosono_serve_stats": [_vp, ctypes.POINTER(ServeTotals)],
    "hosono_serve_last_error": [_vp, _cp, _i],
}
RESTYPES = {"hosono_batch_instance_bytes": ctypes.c_longlong, "hosono_serve_clock": ctypes.c_double}
NOALLOC_MAX_ROWS = 16384  # HOSONO_NOALLOC_MAX_ROWS


def mood_cap_default(radius, nx, ny):
    """HOSONO_MOOD_CAP_DEFAULT(R, nx, ny): MOOD passes per stage before EMOODCAP."""
    return (radius + 1) * (nx + ny)


def set_device(device):
    """Select the CUDA device the library creates its next handles on."""
    rc = load_library().hosono_gpu_set_device(int(device))
    if rc:
        raise HosonoError(rc, f"cudaSetDevice({device})")

_lib = None


def load_library(path=LIB_PATH):
    """Load libhosono_gpu.so; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise HosonoError(ENOTBUILT, f"{path} is missing; run __graft_entry__.build() or "
                                     f"python hosono-2dmhd_b200/build.py")
    lib = ctypes.CDLL(path)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = RESTYPES.get(name, ctypes.c_int)
    _lib = lib
    return lib


def build(verbose=False, force=False):
    import importlib.util
    spec = importlib.util.spec_from_file_location("hosono_build", os.path.join(PKG_DIR, "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.build(verbose=verbose, force=force)


def _p(a, t=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(t))


def gp_build(radius, x_beg, x_end, nx, y_beg, y_end, ny, ell_over_delta):
    """GP_init: (pv, qw, stenc) in Fortran order from .par strings."""
    lib = load_library()
    ns, nq = 1 + 2 * radius * (radius + 1), radius + 1
    pv = np.zeros(ns * nq * 4 * radius)
    qw = np.zeros(nq * radius)
    st = np.zeros(2 * ns * radius, dtype=np.int32)
    rc = lib.hosono_gp_build(radius, str(x_beg).encode(), str(x_end).encode(), nx, str(y_beg).encode(),
                             str(y_end).encode(), ny, str(ell_over_delta).encode(), _p(pv), _p(qw),
                             _p(st, ctypes.c_int))
    if rc:
        raise HosonoError(rc, "hosono_gp_build")
    return pv, qw, st


def par_load(parfile):
    """simulation_init + grid_init: (Params, RunInfo) from a .par file."""
    lib = load_library()
    p, r = Params(), RunInfo()
    err = ctypes.create_string_buffer(512)
    rc = lib.hosono_par_load(os.fsencode(parfile), ctypes.byref(p), ctypes.byref(r), err, 512)
    if rc:
        raise HosonoError(rc, err.value.decode())
    return p, r


def gp_cache_info():
    """Hits, misses and entries of the library's GP table cache."""
    lib = load_library()
    h, m, n = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_int()
    lib.hosono_gp_cache_info(ctypes.byref(h), ctypes.byref(m), ctypes.byref(n))
    return dict(hits=h.value, misses=m.value, entries=n.value)


def gp_cache_clear():
    load_library().hosono_gp_cache_clear()


def par_gp(parfile, radius):
    lib = load_library()
    ns, nq = 1 + 2 * radius * (radius + 1), radius + 1
    pv = np.zeros(ns * nq * 4 * radius)
    qw = np.zeros(nq * radius)
    st = np.zeros(2 * ns * radius, dtype=np.int32)
    err = ctypes.create_string_buffer(512)
    rc = lib.hosono_par_gp(os.fsencode(parfile), _p(pv), _p(qw), _p(st, ctypes.c_int), err, 512)
    if rc:
        raise HosonoError(rc, err.value.decode())
    return pv, qw, st


def ic_set(parfile, params):
    """initialCondition_set: (U, V) host arrays shaped (nyTot, nxTot, 8|10)."""
    lib = load_library()
    nxt, nyt = params.nx + 2 * params.ngc, params.ny + 2 * params.ngc
    U = np.zeros((nyt, nxt, 8))
    V = np.zeros((nyt, nxt, 10))
    err = ctypes.create_string_buffer(512)
    rc = lib.hosono_ic_set(os.fsencode(parfile), ctypes.byref(params), _p(U), _p(V), err, 512)
    if rc:
        raise HosonoError(rc, err.value.decode())
    return U, V


def ic_describe(parfile, params):
    """initialCondition_set for the device: (ICDesc, xtab, ytab) -- a few
    constants and per-column / per-row tables, O(nx+ny)."""
    lib = load_library()
    nxt, nyt = params.nx + 2 * params.ngc, params.ny + 2 * params.ngc
    d = ICDesc()
    xt = np.zeros(3 * nxt)
    yt = np.zeros(2 * nyt)
    err = ctypes.create_string_buffer(512)
    rc = lib.hosono_ic_describe(os.fsencode(parfile), ctypes.byref(params), ctypes.byref(d), _p(xt), _p(yt), err, 512)
    if rc:
        raise HosonoError(rc, err.value.decode())
    return d, xt, yt


class Solver:
    """One block advanced on the GPU (gridBlock_t + gridState_t resident in HBM)."""

    def __init__(self, params, pv, qw, stenc):
        self.lib = load_library()
        self.params = params
        self.nxt = params.nx + 2 * params.ngc
        self.nyt = params.ny + 2 * params.ngc
        self._pv = np.ascontiguousarray(pv, dtype=np.float64)
        self._qw = np.ascontiguousarray(qw, dtype=np.float64)
        self._st = np.ascontiguousarray(stenc, dtype=np.int32)
        h = ctypes.c_void_p()
        rc = self.lib.hosono_gpu_create(ctypes.byref(params), _p(self._pv), _p(self._qw),
                                        _p(self._st, ctypes.c_int), ctypes.byref(h))
        if rc:
            raise HosonoError(rc, "hosono_gpu_create")
        self.h = h

    @classmethod
    def from_par(cls, parfile, fp_mode=FP_STRICT):
        """simulation_init + GP_init + grid_init + initialCondition_set, then upload."""
        p, run = par_load(parfile)
        p.fp_mode = fp_mode
        pv, qw, st = par_gp(parfile, p.max_radius)
        s = cls(p, pv, qw, st)
        s.run_info = run
        U, V = ic_set(parfile, p)
        s.upload(U, V)
        return s

    def _check(self, rc, what):
        if rc:
            buf = ctypes.create_string_buffer(512)
            self.lib.hosono_gpu_last_error(self.h, buf, 512)
            raise HosonoError(rc, f"{what}: {buf.value.decode()}")

    def close(self):
        if getattr(self, "h", None):
            self.lib.hosono_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def upload(self, U, V=None):
        U = np.ascontiguousarray(U, dtype=np.float64)
        assert U.size == self.nxt * self.nyt * 8
        Vp = None
        if V is not None:
            V = np.ascontiguousarray(V, dtype=np.float64)
            assert V.size == self.nxt * self.nyt * 10
            Vp = _p(V)
        self._check(self.lib.hosono_gpu_upload(self.h, _p(U), Vp), "upload")

    def download(self, U=None, V=None, with_scheme=True):
        """(U, V, scheme); pass U/V (C-contiguous float64) to fill them in place."""
        U = np.zeros((self.nyt, self.nxt, 8)) if U is None else U
        V = np.zeros((self.nyt, self.nxt, 10)) if V is None else V
        assert U.flags.c_contiguous and V.flags.c_contiguous
        S = np.zeros((self.nyt, self.nxt), dtype=np.int32) if with_scheme else None
        self._check(self.lib.hosono_gpu_download(self.h, _p(U), _p(V), _p(S, ctypes.c_int) if with_scheme else None),
                    "download")
        return U, V, S

    def upload_ic(self, desc, xtab, ytab):
        """Build the initial state on the device (see ic_describe)."""
        self._check(self.lib.hosono_gpu_ic(self.h, ctypes.byref(desc), _p(np.ascontiguousarray(xtab)),
                                           _p(np.ascontiguousarray(ytab))), "ic")

    def cfl_computedt(self):
        dt = ctypes.c_double()
        self._check(self.lib.hosono_gpu_cfl(self.h, ctypes.byref(dt)), "cfl")
        return dt.value

    def timeStep_advanceSolution(self, dt):
        self._check(self.lib.hosono_gpu_advance(self.h, float(dt)), "advance")

    def advance_host(self, dt, U, V=None):
        """Drop-in on host arrays: U in, advanced U (and V) out, in place."""
        assert U.flags.c_contiguous and U.dtype == np.float64
        self._check(self.lib.hosono_gpu_advance_host(self.h, float(dt), _p(U), _p(V) if V is not None else None),
                    "advance_host")

    def set_graphs(self, on=True):
        """Run the MOOD loops from the captured CUDA graph (default) or host-driven."""
        self._check(self.lib.hosono_gpu_set_graphs(self.h, 1 if on else 0), "set_graphs")

    def set_time(self, t, tmax, nstep=0, nstepmax=1 << 30):
        self._check(self.lib.hosono_gpu_set_time(self.h, float(t), float(tmax), int(nstep), int(nstepmax)),
                    "set_time")

    def set_mood_cap(self, cap):
        """MOOD passes a stage may take before the solve stops with EMOODCAP
        (cap <= 0: the proven bound R*nx*ny + 1)."""
        self._check(self.lib.hosono_gpu_set_mood_cap(self.h, int(cap)), "set_mood_cap")

    def step(self, max_steps=1):
        """Continue the time loop (cfl + validTimeStep + advance on the device) by
        up to max_steps steps; returns (t, nstep)."""
        t = ctypes.c_double()
        n = ctypes.c_int()
        self._check(self.lib.hosono_gpu_step(self.h, int(max_steps), ctypes.byref(t), ctypes.byref(n)), "step")
        return t.value, n.value

    def run(self, tmax=None, nstepmax=None, max_steps=0):
        """mhd_driver's time loop (no output)."""
        ri = getattr(self, "run_info", None)
        tmax = ri.tmax if tmax is None else tmax
        nstepmax = (ri.nstepmax if ri is not None else 1 << 30) if nstepmax is None else nstepmax
        t = ctypes.c_double()
        n = ctypes.c_int()
        self._check(self.lib.hosono_gpu_run(self.h, float(tmax), int(nstepmax), int(max_steps), ctypes.byref(t),
                                            ctypes.byref(n)), "run")
        return t.value, n.value

    def stats(self):
        s = Stats()
        self._check(self.lib.hosono_gpu_stats(self.h, ctypes.byref(s)), "stats")
        return s.as_dict()

    def trace(self, on=True):
        self._check(self.lib.hosono_gpu_trace_enable(self.h, 1 if on else 0), "trace")

    def trace_clear(self):
        self._check(self.lib.hosono_gpu_trace_clear(self.h), "trace_clear")

    def traces(self, masks=True):
        out = []
        n = self.nxt * self.nyt
        for k in range(self.lib.hosono_gpu_trace_count(self.h)):
            meta = np.zeros(4, dtype=np.int32)
            inner = np.zeros(n, dtype=np.uint8)
            det = np.zeros(n, dtype=np.uint8)
            self._check(self.lib.hosono_gpu_trace_get(self.h, k, _p(meta, ctypes.c_int), inner.ctypes.data,
                                                      det.ctypes.data), "trace_get")
            rec = dict(stage=int(meta[0]), mood_pass=int(meta[1]), n_inner=int(meta[2]), n_detect=int(meta[3]))
            if masks:
                rec["inner"] = inner.reshape(self.nyt, self.nxt)
                rec["detect"] = det.reshape(self.nyt, self.nxt)
            out.append(rec)
        return out

    def stream(self):
        """cudaStream_t (as an int) all of this solver's kernels run on."""
        s = ctypes.c_void_p()
        self._check(self.lib.hosono_gpu_stream(self.h, ctypes.byref(s)), "stream")
        return s.value or 0

    # ---- the reference's stage modules one at a time (module state of the
    # handle; host arrays in the reference's layout, numpy-shaped [j, i, ...])
    def module_set(self, scheme=None, recompute=None, recompute_flicd=None):
        keep = []

        def arg(a):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=np.int32).reshape(-1)
            assert a.size == self.nxt * self.nyt
            keep.append(a)
            return _p(a, ctypes.c_int)
        self._check(self.lib.hosono_gpu_module_set(self.h, arg(scheme), arg(recompute), arg(recompute_flicd)),
                    "module_set")

    def module_get(self):
        """dict of faceVals [j, i, face, q, var], fluxRaw / flux [j, i, dir, var],
        Unew [j, i, var], scheme / recompute / recompute_flicd [j, i]."""
        nq = self.params.max_radius + 1
        sh = (self.nyt, self.nxt)
        fv = np.zeros((*sh, 4, nq, 8))
        fr = np.zeros((*sh, 2, 8))
        fl = np.zeros((*sh, 2, 8))
        un = np.zeros((*sh, 8))
        sc, rc, rf = (np.zeros(sh, dtype=np.int32) for _ in range(3))
        self._check(self.lib.hosono_gpu_module_get(self.h, _p(fv), _p(fr), _p(fl), _p(un), _p(sc, ctypes.c_int),
                                                   _p(rc, ctypes.c_int), _p(rf, ctypes.c_int)), "module_get")
        return dict(faceVals=fv, fluxRaw=fr, flux=fl, Unew=un, scheme=sc, recompute=rc, recompute_flicd=rf)

    def reconstruct(self):
        """reconstruct_faceValsWithGP(blk, state%U)"""
        self._check(self.lib.hosono_gpu_reconstruct(self.h), "reconstruct")

    def getfluxes(self):
        self._check(self.lib.hosono_gpu_getfluxes(self.h), "getfluxes")

    def flicd(self):
        self._check(self.lib.hosono_gpu_flicd(self.h), "flicd")

    def update(self, dt):
        self._check(self.lib.hosono_gpu_update(self.h, float(dt)), "update")

    def detect(self):
        """detect_ALL; returns exit_mood_loop."""
        e = ctypes.c_int()
        self._check(self.lib.hosono_gpu_detect(self.h, ctypes.byref(e)), "detect")
        return bool(e.value)

    def bc(self, which):
        """boundaryConditions_applyBlk on U (0), V (1) or Unew (2)."""
        self._check(self.lib.hosono_gpu_bc(self.h, int(which)), "bc")

    def bc_mood(self):
        self._check(self.lib.hosono_gpu_bc_mood(self.h), "bc_mood")

    def mood_pass_stats(self):
        n = ctypes.c_int()
        t = ctypes.c_longlong()
        self._check(self.lib.hosono_gpu_mood_pass_stats(self.h, ctypes.byref(n), ctypes.byref(t)),
                    "mood_pass_stats")
        return n.value, t.value

    def riemann(self, n, uL_dev, uR_dev, direction, flux_dev):
        """riemannSolver_fromConsHllcMHD on n faces of device arrays (8, n)."""
        self._check(self.lib.hosono_gpu_riemann(self.h, int(n), ctypes.c_void_p(uL_dev), ctypes.c_void_p(uR_dev),
                                                int(direction), ctypes.c_void_p(flux_dev)), "riemann")

    def set_tuning(self, **kw):
        """Launch choices (results are the same bits for every choice)."""
        t = Tuning()
        self._check(self.lib.hosono_gpu_get_tuning(self.h, ctypes.byref(t)), "get_tuning")
        t.update(kw)
        self._check(self.lib.hosono_gpu_set_tuning(self.h, ctypes.byref(t)), "set_tuning")

    def tuning(self):
        t = Tuning()
        self._check(self.lib.hosono_gpu_get_tuning(self.h, ctypes.byref(t)), "get_tuning")
        return t.as_dict()

    def autotune(self, trials=5, force=False):
        """Time the candidate launch choices on this solve and apply the fastest."""
        r = TuneReport()
        self._check(self.lib.hosono_gpu_autotune(self.h, int(trials), 1 if force else 0, ctypes.byref(r)),
                    "autotune")
        return r.as_dict()

    def eigenvecs(self, n, V_dev, direction, cons, L_dev, R_dev):
        """eigen_vecsFromPrim on n primitive states of a device array (10, n)."""
        self._check(self.lib.hosono_gpu_eigenvecs(self.h, int(n), ctypes.c_void_p(V_dev), int(direction),
                                                  1 if cons else 0, ctypes.c_void_p(L_dev), ctypes.c_void_p(R_dev)),
                    "eigenvecs")

    def launch_info(self):
        """Launch geometry: tiles, SMs, pass-1 grid, largest other tile-kernel grid."""
        li = LaunchInfo()
        self._check(self.lib.hosono_gpu_launch_info(self.h, ctypes.byref(li)), "launch_info")
        return li.as_dict()

    DIAG_FIELDS = ("dens", "velx", "vely", "velz", "pres", "eint", "gama", "ener", "magp", "divb", "magx",
                   "magy", "magz")

    def diagnostics(self):
        """output_writeHdf5's fields on the device: ({name: (ny, nx) array},
        scheme, ordr, mean |div B|, max |div B|)."""
        nx, ny = self.params.nx, self.params.ny
        f = np.empty((13, ny, nx))
        s = np.empty((ny, nx), dtype=np.int32)
        o = np.empty((ny, nx), dtype=np.int32)
        l1, li = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.hosono_gpu_diagnostics(self.h, _p(f), _p(s, ctypes.c_int), _p(o, ctypes.c_int),
                                                    ctypes.byref(l1), ctypes.byref(li)), "diagnostics")
        return dict(zip(self.DIAG_FIELDS, f)), s, o, l1.value, li.value

    def profile(self, on=True):
        self._check(self.lib.hosono_gpu_profile(self.h, 1 if on else 0), "profile")

    def profile_read(self, reset=True):
        """(pass-1 kernel ms summed, pass-1 launches, all launches) since the last reset."""
        ms = ctypes.c_double()
        n1 = ctypes.c_longlong()
        n = ctypes.c_longlong()
        self._check(self.lib.hosono_gpu_profile_read(self.h, ctypes.byref(ms), ctypes.byref(n1), ctypes.byref(n),
                                                     1 if reset else 0), "profile_read")
        return ms.value, n1.value, n.value

    def state_layout(self):
        ptr = ctypes.c_void_p()
        pitch = ctypes.c_int()
        plane = ctypes.c_longlong()
        self._check(self.lib.hosono_gpu_state_layout(self.h, ctypes.byref(ptr), ctypes.byref(pitch),
                                                     ctypes.byref(plane)), "state_layout")
        return ptr.value, pitch.value, plane.value


class Batch:
    """Many independent blocks advanced together (include/hosono_gpu.h, hosono_batch_*)."""

    def __init__(self, max_instances, max_tiles, fp_mode=FP_STRICT):
        self.lib = load_library()
        h = ctypes.c_void_p()
        rc = self.lib.hosono_batch_create(int(max_instances), int(max_tiles), int(fp_mode), ctypes.byref(h))
        if rc:
            raise HosonoError(rc, "hosono_batch_create")
        self.h = h
        self.shapes = {}
        self.ngcs = {}
        self._keep = {}

    @staticmethod
    def tiles_for(params):
        return load_library().hosono_batch_tiles_for(ctypes.byref(params))

    @staticmethod
    def instance_bytes(params):
        return load_library().hosono_batch_instance_bytes(ctypes.byref(params))

    def _check(self, rc, what):
        if rc:
            buf = ctypes.create_string_buffer(512)
            self.lib.hosono_batch_last_error(self.h, buf, 512)
            raise HosonoError(rc, f"{what}: {buf.value.decode()}")

    def close(self):
        if getattr(self, "h", None):
            self.lib.hosono_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, params, pv, qw, stenc):
        pv = np.ascontiguousarray(pv, dtype=np.float64)
        qw = np.ascontiguousarray(qw, dtype=np.float64)
        st = np.ascontiguousarray(stenc, dtype=np.int32)
        slot = ctypes.c_int()
        self._check(self.lib.hosono_batch_add(self.h, ctypes.byref(params), _p(pv), _p(qw), _p(st, ctypes.c_int),
                                              ctypes.byref(slot)), "add")
        k = slot.value
        self.shapes[k] = (params.ny + 2 * params.ngc, params.nx + 2 * params.ngc)
        self.ngcs[k] = params.ngc
        return k

    def add_par(self, parfile, fp_mode=None):
        """Set up an instance from a .par file (GP tables, IC, time limits) and upload it."""
        p, run = par_load(parfile)
        pv, qw, st = par_gp(parfile, p.max_radius)
        k = self.add(p, pv, qw, st)
        U, V = ic_set(parfile, p)
        self.upload(k, U, V)
        self.set_time(k, 0.0, run.tmax, 0, run.nstepmax)
        return k

    def remove(self, slot):
        self._check(self.lib.hosono_batch_remove(self.h, int(slot)), "remove")
        self.shapes.pop(slot, None)

    def upload(self, slot, U, V=None):
        U = np.ascontiguousarray(U, dtype=np.float64)
        Vp = None
        if V is not None:
            V = np.ascontiguousarray(V, dtype=np.float64)
            Vp = _p(V)
        self._check(self.lib.hosono_batch_upload(self.h, int(slot), _p(U), Vp), "upload")

    def download(self, slot):
        nyt, nxt = self.shapes[slot]
        U = np.zeros((nyt, nxt, 8))
        V = np.zeros((nyt, nxt, 10))
        S = np.zeros((nyt, nxt), dtype=np.int32)
        self._check(self.lib.hosono_batch_download(self.h, int(slot), _p(U), _p(V), _p(S, ctypes.c_int)),
                    "download")
        return U, V, S

    def diagnostics(self, slot):
        """Solver.diagnostics for one instance of the batch."""
        nyt, nxt = self.shapes[slot]
        ngc = self.ngcs[slot]
        nx, ny = nxt - 2 * ngc, nyt - 2 * ngc
        f = np.empty((13, ny, nx))
        s = np.empty((ny, nx), dtype=np.int32)
        o = np.empty((ny, nx), dtype=np.int32)
        l1, li = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.hosono_batch_diagnostics(self.h, int(slot), _p(f), _p(s, ctypes.c_int),
                                                      _p(o, ctypes.c_int), ctypes.byref(l1), ctypes.byref(li)),
                    "diagnostics")
        return dict(zip(Solver.DIAG_FIELDS, f)), s, o, l1.value, li.value

    def set_time(self, slot, t, tmax, nstep=0, nstepmax=1 << 30):
        self._check(self.lib.hosono_batch_set_time(self.h, int(slot), float(t), float(tmax), int(nstep),
                                                   int(nstepmax)), "set_time")

    def set_tuning(self, **kw):
        t = Tuning()
        self._check(self.lib.hosono_batch_get_tuning(self.h, ctypes.byref(t)), "get_tuning")
        t.update(kw)
        self._check(self.lib.hosono_batch_set_tuning(self.h, ctypes.byref(t)), "set_tuning")

    def tuning(self):
        t = Tuning()
        self._check(self.lib.hosono_batch_get_tuning(self.h, ctypes.byref(t)), "get_tuning")
        return t.as_dict()

    def autotune(self, trials=5, force=False):
        """Time the candidate launch choices on the batch's instances; apply the fastest."""
        r = TuneReport()
        self._check(self.lib.hosono_batch_autotune(self.h, int(trials), 1 if force else 0, ctypes.byref(r)),
                    "autotune")
        return r.as_dict()

    def set_mood_cap(self, slot, cap):
        self._check(self.lib.hosono_batch_set_mood_cap(self.h, int(slot), int(cap)), "set_mood_cap")

    def run(self, max_steps=0):
        self._check(self.lib.hosono_batch_run(self.h, int(max_steps)), "run")

    def status(self, slot):
        t = ctypes.c_double()
        dt = ctypes.c_double()
        n = ctypes.c_int()
        done = ctypes.c_int()
        err = ctypes.c_int()
        self._check(self.lib.hosono_batch_status(self.h, int(slot), ctypes.byref(t), ctypes.byref(dt),
                                                 ctypes.byref(n), ctypes.byref(done), ctypes.byref(err)), "status")
        return dict(t=t.value, dt=dt.value, nstep=n.value, done=bool(done.value), error=err.value)

    def stats(self, slot):
        s = Stats()
        self._check(self.lib.hosono_batch_stats(self.h, int(slot), ctypes.byref(s)), "stats")
        return s.as_dict()

    def stream(self):
        s = ctypes.c_void_p()
        self._check(self.lib.hosono_batch_stream(self.h, ctypes.byref(s)), "stream")
        return s.value or 0

    def set_graphs(self, on=True):
        self._check(self.lib.hosono_batch_set_graphs(self.h, 1 if on else 0), "set_graphs")

    def capacity(self):
        a, b, c, d = (ctypes.c_int() for _ in range(4))
        self._check(self.lib.hosono_batch_capacity(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c),
                                                   ctypes.byref(d)), "capacity")
        return dict(max_instances=a.value, max_tiles=b.value, used_tiles=c.value, live=d.value)
