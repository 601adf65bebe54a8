"""ctypes wrapper of the CPU oracle (test infrastructure only).

The oracle restates the reference Fortran time-step path on the CPU; see
hosono_oracle.cpp.  Only tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py import this module.

Arrays are returned as numpy views shaped (nyTot, nxTot, nvar): the
reference's Fortran-order U(var, i, j) read with var fastest.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")

_libs = {}


def build():
    """Compile both oracle libraries (strict parity build and fast baseline build)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _lib(fast=False, count=False):
    key = "count" if count else "fast" if fast else "strict"
    if key in _libs:
        return _libs[key]
    name = dict(count="libhosono_oracle_count.so", fast="libhosono_oracle_fast.so",
                strict="libhosono_oracle.so")[key]
    path = os.path.join(BUILD, name)
    # make rebuilds a library whose sources changed (a no-op otherwise)
    subprocess.run(["make", "-s", "-C", HERE] + (["count"] if count else []), check=True)
    lib = ctypes.CDLL(path)
    d, i, p = ctypes.c_double, ctypes.c_int, ctypes.c_void_p
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)
    lib.orc_create_from_par.restype = p
    lib.orc_create_from_par.argtypes = [ctypes.c_char_p, ctypes.c_char_p, i]
    lib.orc_destroy.argtypes = [p]
    lib.orc_info.argtypes = [p, ip, dp]
    lib.orc_get_gp.argtypes = [p, dp, dp, ip]
    for n in ("orc_get_U", "orc_get_V", "orc_set_U", "orc_set_V"):
        getattr(lib, n).argtypes = [p, dp]
    lib.orc_get_scheme.argtypes = [p, ip]
    lib.orc_cfl.restype = d
    lib.orc_cfl.argtypes = [p]
    lib.orc_advance.argtypes = [p, d]
    lib.orc_run.argtypes = [p, i, dp, ip]
    lib.orc_reconstruct_all.argtypes = [p, i, dp]
    lib.orc_trace_enable.argtypes = [p, i]
    lib.orc_trace_count.argtypes = [p]
    lib.orc_trace_get.argtypes = [p, i, ip, ctypes.c_void_p, ctypes.c_void_p]
    lib.orc_trace_clear.argtypes = [p]
    lib.orc_cons2prim.argtypes = [p, dp, dp]
    lib.orc_cons2pres.restype = d
    lib.orc_cons2pres.argtypes = [p, dp]
    lib.orc_cons2flux.argtypes = [p, dp, i, dp]
    lib.orc_hllc.argtypes = [p, dp, dp, i, dp]
    lib.orc_eigenvecs.argtypes = [p, dp, i, i, dp, dp]
    lib.orc_c_fs.restype = d
    lib.orc_c_fs.argtypes = [d, d, d, d, d, d]
    lib.orc_gp_build.argtypes = [i, ctypes.c_char_p, ctypes.c_char_p, i, ctypes.c_char_p, ctypes.c_char_p, i,
                                 ctypes.c_char_p, dp, dp, ip]
    lib.orc_mod_set.argtypes = [p, ip, ip, ip]
    lib.orc_mod_get.argtypes = [p, dp, dp, dp, dp, ip, ip, ip]
    for n in ("orc_mod_reconstruct", "orc_mod_getfluxes", "orc_mod_flicd", "orc_mod_detect", "orc_mod_bc_mood"):
        getattr(lib, n).argtypes = [p]
    lib.orc_mod_update.argtypes = [p, d]
    lib.orc_mod_bc.argtypes = [p, i]
    lib.orc_set_threads.argtypes = [i]
    lib.orc_get_threads.restype = i
    if count:
        lib.orc_count_get.argtypes = [i, ctypes.POINTER(ctypes.c_ulonglong)]
        lib.orc_count_reset.argtypes = []
    _libs[key] = lib
    return lib


COUNT_CLASSES = ("add", "mul", "div", "sqrt", "cmp", "other")


def count_reset():
    """Zero the operation counters of the counting build (flopcount.h)."""
    _lib(count=True).orc_count_reset()


COUNT_PHASES = ("rest", "pass1", "later_passes", "update_detect")


def count_get():
    """Operations the counting build executed since count_reset(), by phase
    of the time step (COUNT_PHASES) and class; 'flops' = add + mul + div +
    sqrt."""
    out = {}
    for k, name in enumerate(COUNT_PHASES):
        c = (ctypes.c_ulonglong * 6)()
        _lib(count=True).orc_count_get(k, c)
        d = dict(zip(COUNT_CLASSES, (int(v) for v in c)))
        d["flops"] = d["add"] + d["mul"] + d["div"] + d["sqrt"]
        out[name] = d
    return out


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def set_threads(n, fast=False, count=False):
    _lib(fast, count).orc_set_threads(int(n))


def get_threads(fast=False):
    return _lib(fast).orc_get_threads()


def gp_build(R, x_beg, x_end, nx, y_beg, y_end, ny, ell_over_delta):
    """GP tables for the given .par strings: (pv, qw, stenc) in Fortran order."""
    lib = _lib()
    ns = 1 + 2 * R * (R + 1)
    nq = R + 1
    pv = np.zeros(ns * nq * 4 * R)
    qw = np.zeros(nq * R)
    st = np.zeros(2 * ns * R, dtype=np.int32)
    rc = lib.orc_gp_build(R, x_beg.encode(), x_end.encode(), nx, y_beg.encode(), y_end.encode(), ny,
                          ell_over_delta.encode(), _dp(pv), _dp(qw), _ip(st))
    if rc != 0:
        raise RuntimeError("orc_gp_build failed")
    return pv, qw, st


class Oracle:
    """One solver instance built from a .par file."""

    def __init__(self, parfile, fast=False, count=False):
        self.lib = _lib(fast, count)
        err = ctypes.create_string_buffer(512)
        self.h = self.lib.orc_create_from_par(os.fsencode(parfile), err, 512)
        if not self.h:
            raise ValueError(err.value.decode())
        ints = np.zeros(10, dtype=np.int32)
        dbls = np.zeros(10)
        self.lib.orc_info(self.h, _ip(ints), _dp(dbls))
        (self.nx, self.ny, self.ngc, self.R, self.nxTot, self.nyTot, self.nqMax, self.nsMax,
         self.bc, self.force_hydro) = [int(v) for v in ints]
        (self.dx, self.dy, self.mindxdy, self.maxdxdy, self.gamma, self.cfl_number, self.tmax,
         self.small_pressure, self.small_density, self.ell_over_delta) = [float(v) for v in dbls]

    def close(self):
        if self.h:
            self.lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def ncell(self):
        return self.nxTot * self.nyTot

    def gp(self):
        pv = np.zeros(self.nsMax * self.nqMax * 4 * self.R)
        qw = np.zeros(self.nqMax * self.R)
        st = np.zeros(2 * self.nsMax * self.R, dtype=np.int32)
        self.lib.orc_get_gp(self.h, _dp(pv), _dp(qw), _ip(st))
        return pv, qw, st

    def U(self):
        a = np.zeros(self.ncell * 8)
        self.lib.orc_get_U(self.h, _dp(a))
        return a.reshape(self.nyTot, self.nxTot, 8)

    def V(self):
        a = np.zeros(self.ncell * 10)
        self.lib.orc_get_V(self.h, _dp(a))
        return a.reshape(self.nyTot, self.nxTot, 10)

    def set_U(self, U):
        a = np.ascontiguousarray(U, dtype=np.float64).reshape(-1)
        assert a.size == self.ncell * 8
        self.lib.orc_set_U(self.h, _dp(a))

    def set_V(self, V):
        a = np.ascontiguousarray(V, dtype=np.float64).reshape(-1)
        assert a.size == self.ncell * 10
        self.lib.orc_set_V(self.h, _dp(a))

    def scheme(self):
        a = np.zeros(self.ncell, dtype=np.int32)
        self.lib.orc_get_scheme(self.h, _ip(a))
        return a.reshape(self.nyTot, self.nxTot)

    def cfl(self):
        return self.lib.orc_cfl(self.h)

    def advance(self, dt):
        self.lib.orc_advance(self.h, float(dt))

    def run(self, max_steps=0):
        t = ctypes.c_double(0.0)
        n = ctypes.c_int(0)
        rc = self.lib.orc_run(self.h, int(max_steps), ctypes.byref(t), ctypes.byref(n))
        return rc, t.value, n.value

    def reconstruct_all(self, radius):
        fv = np.zeros(self.ncell * 8 * self.nqMax * 4)
        self.lib.orc_reconstruct_all(self.h, int(radius), _dp(fv))
        # Fortran (8, nqMax, 4, nxTot, nyTot) -> [j, i, face, q, var]
        return fv.reshape(self.nyTot, self.nxTot, 4, self.nqMax, 8)

    def trace(self, on=True):
        self.lib.orc_trace_enable(self.h, 1 if on else 0)

    def trace_clear(self):
        self.lib.orc_trace_clear(self.h)

    def traces(self, masks=True):
        out = []
        for k in range(self.lib.orc_trace_count(self.h)):
            meta = np.zeros(4, dtype=np.int32)
            inner = np.zeros(self.ncell, dtype=np.uint8) if masks else None
            det = np.zeros(self.ncell, dtype=np.uint8) if masks else None
            self.lib.orc_trace_get(self.h, k, _ip(meta),
                                   inner.ctypes.data if masks else None,
                                   det.ctypes.data if masks else None)
            rec = dict(stage=int(meta[0]), mood_pass=int(meta[1]), n_inner=int(meta[2]), n_detect=int(meta[3]))
            if masks:
                rec["inner"] = inner.reshape(self.nyTot, self.nxTot)
                rec["detect"] = det.reshape(self.nyTot, self.nxTot)
            out.append(rec)
        return out

    # ---- the stage modules one at a time (reference arrays, Fortran order)
    def mod_set(self, scheme=None, recompute=None, recompute_flicd=None):
        """Set blk%scheme / recompute / recomputeFLICD, each (nyTot, nxTot) or None."""
        def arg(a):
            if a is None:
                return None, None
            a = np.ascontiguousarray(a, dtype=np.int32).reshape(-1)
            assert a.size == self.ncell
            return a, _ip(a)
        keep = [arg(a) for a in (scheme, recompute, recompute_flicd)]
        self.lib.orc_mod_set(self.h, *(k[1] for k in keep))

    def mod_get(self):
        """dict of faceVals [j, i, face, q, var], fluxRaw / flux [j, i, dir, var],
        Unew [j, i, var], scheme / recompute / recompute_flicd [j, i]."""
        nq = self.nqMax
        fv = np.zeros(self.ncell * 8 * nq * 4)
        fr = np.zeros(self.ncell * 16)
        fl = np.zeros(self.ncell * 16)
        un = np.zeros(self.ncell * 8)
        sc, rc, rf = (np.zeros(self.ncell, dtype=np.int32) for _ in range(3))
        self.lib.orc_mod_get(self.h, _dp(fv), _dp(fr), _dp(fl), _dp(un), _ip(sc), _ip(rc), _ip(rf))
        sh = (self.nyTot, self.nxTot)
        return dict(faceVals=fv.reshape(*sh, 4, nq, 8), fluxRaw=fr.reshape(*sh, 2, 8), flux=fl.reshape(*sh, 2, 8),
                    Unew=un.reshape(*sh, 8), scheme=sc.reshape(sh), recompute=rc.reshape(sh),
                    recompute_flicd=rf.reshape(sh))

    def mod_reconstruct(self):
        self.lib.orc_mod_reconstruct(self.h)

    def mod_getfluxes(self):
        self.lib.orc_mod_getfluxes(self.h)

    def mod_flicd(self):
        self.lib.orc_mod_flicd(self.h)

    def mod_update(self, dt):
        self.lib.orc_mod_update(self.h, float(dt))

    def mod_detect(self):
        """detect_ALL; returns exit_mood_loop."""
        return bool(self.lib.orc_mod_detect(self.h))

    def mod_bc(self, which):
        self.lib.orc_mod_bc(self.h, int(which))

    def mod_bc_mood(self):
        self.lib.orc_mod_bc_mood(self.h)

    # pointwise physics
    def cons2prim(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        v = np.zeros(10)
        self.lib.orc_cons2prim(self.h, _dp(u), _dp(v))
        return v

    def cons2pres(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        return self.lib.orc_cons2pres(self.h, _dp(u))

    def cons2flux(self, u, direction):
        u = np.ascontiguousarray(u, dtype=np.float64)
        f = np.zeros(8)
        self.lib.orc_cons2flux(self.h, _dp(u), int(direction), _dp(f))
        return f

    def eigenvecs(self, V, direction, cons=False):
        """eigen_vecsFromPrim: (L, R) as 8x8 arrays [row=variable, col=wave]."""
        V = np.ascontiguousarray(V, dtype=np.float64)
        L = np.zeros(64)
        R = np.zeros(64)
        self.lib.orc_eigenvecs(self.h, _dp(V), int(direction), 1 if cons else 0, _dp(L), _dp(R))
        return L.reshape(8, 8).T, R.reshape(8, 8).T

    def hllc(self, uL, uR, direction):
        uL = np.ascontiguousarray(uL, dtype=np.float64)
        uR = np.ascontiguousarray(uR, dtype=np.float64)
        f = np.zeros(8)
        self.lib.orc_hllc(self.h, _dp(uL), _dp(uR), int(direction), _dp(f))
        return f
