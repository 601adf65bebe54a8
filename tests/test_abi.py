"""The C ABI library loads and exports every symbol include/hosono_gpu.h
declares; host-side set-up entry points run without a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle
import parfiles
import pkg

HEADER = os.path.join(pkg.ROOT, "include", "hosono_gpu.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(hosono_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    m = pkg.load()
    lib = m.load_library()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(m.SIGNATURES), set(names) ^ set(m.SIGNATURES)


@pytest.mark.parametrize("R", [1, 2, 3])
def test_gp_tables_bit_identical_to_oracle(R):
    m = pkg.load()
    for args in (("0.0", "1.0", 128, "0.0", "1.0", 128, "6.0"), ("-0.5", "0.5", 512, "-0.5", "0.5", 256, "12.0")):
        a = m.gp_build(R, *args)
        b = oracle.gp_build(R, *args)
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("name,kv", [
    ("ot", parfiles.orszag_tang(40, 2)),
    ("ot_refic", parfiles.orszag_tang(24, 3, standard=False)),
    ("sedov", parfiles.sedov(36, 2)),
    ("blast", parfiles.blast(48, 2, p_ratio=300.0, theta=0.7)),
])
def test_par_and_initial_condition_match_oracle(name, kv, tmp_par_dir):
    m = pkg.load()
    par = parfiles.make(tmp_par_dir, name, kv)
    p, run = m.par_load(par)
    U, V = m.ic_set(par, p)
    o = oracle.Oracle(par)
    np.testing.assert_array_equal(U, o.U())
    np.testing.assert_array_equal(V, o.V())
    assert (p.nx, p.ny, p.ngc, p.max_radius) == (o.nx, o.ny, o.ngc, o.R)
    assert p.dx == o.dx and p.dy == o.dy and p.mindxdy == o.mindxdy and p.maxdxdy == o.maxdxdy
    assert run.tmax == o.tmax


def test_par_missing_key_is_reported(tmp_par_dir):
    m = pkg.load()
    kv = parfiles.orszag_tang(16, 1)
    del kv["sim_cfl"]
    par = parfiles.make(tmp_par_dir, "missing", kv)
    with pytest.raises(m.HosonoError) as e:
        m.par_load(par)
    assert e.value.code == m.EPAR and "sim_cfl" in str(e.value)


def test_par_every_missing_key_is_reported(tmp_par_dir):
    """The required keys are checked up front: the reference's message names
    the first missing key (in its read order), and the rest follow."""
    m = pkg.load()
    kv = parfiles.orszag_tang(16, 1)
    for k in ("grid_yEnd", "sim_gamma", "GP_ellOverDelta", "GP_maxRadius", "grid_xBeg"):
        del kv[k]
    par = parfiles.make(tmp_par_dir, "missing3", kv)
    with pytest.raises(m.HosonoError) as e:
        m.par_load(par)
    msg = str(e.value)
    assert e.value.code == m.EPAR
    assert "The parameter 'sim_gamma' was not found" in msg
    # GP_init reads grid_xBeg .. grid_Ny, then GP_ellOverDelta, then
    # GP_maxRadius (GP.f90:58-69)
    assert "also missing: grid_xBeg, grid_yEnd, GP_ellOverDelta, GP_maxRadius" in msg


def test_par_first_match_and_comments(tmp_par_dir):
    """readParamFile.f90:150-175: comment lines skipped, text after '#'
    dropped, first matching key wins, leading blanks make a different key."""
    m = pkg.load()
    kv = parfiles.orszag_tang(16, 1)
    par = parfiles.make(tmp_par_dir, "dup", kv)
    with open(par) as f:
        body = f.read()
    body = "# sim_cfl = 0.1\n   sim_cfl = 0.2\n" + body.replace("sim_cfl = 0.8", "sim_cfl = 0.8 # courant") + \
        "sim_cfl = 0.3\n"
    with open(par, "w") as f:
        f.write(body)
    p, _ = m.par_load(par)
    assert p.cfl == 0.8


def test_create_rejects_bad_params():
    m = pkg.load()
    p = m.Params(nx=8, ny=8, ngc=3, max_radius=2, bc=1, riemann_solver=1, dx=0.1, dy=0.1)
    pv, qw, st = m.gp_build(2, "0.0", "1.0", 8, "0.0", "1.0", 8, "6.0")
    h = ctypes.c_void_p()
    lib = m.load_library()
    rc = lib.hosono_gpu_create(ctypes.byref(p), pv.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                               qw.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                               st.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), ctypes.byref(h))
    assert rc == m.EINVAL  # ngc must be R + 2


def test_serve_create_without_gpu_fails_cleanly():
    """hosono_serve_create on a machine without a usable GPU returns an error
    status (the scheduler thread starts, fails its CUDA set-up and exits)."""
    import importlib
    m = pkg.load()
    srv = importlib.import_module("hosono_2dmhd_b200.serve")
    try:
        s = srv.Server(memory_budget=1 << 26)
    except m.HosonoError as e:
        assert e.code in (m.ECUDA, m.ENOMEM)
        return
    s.close()
    pytest.skip("a GPU is present")


STRUCTS = {"hosono_params": "Params", "hosono_run_info": "RunInfo", "hosono_stats": "Stats",
           "hosono_serve_config": "ServeConfig", "hosono_request_info": "RequestInfo",
           "hosono_serve_totals": "ServeTotals", "hosono_launch_info": "LaunchInfo", "hosono_tuning": "Tuning",
           "hosono_tune_report": "TuneReport", "hosono_ic_desc": "ICDesc"}


def test_binding_structs_match_the_header(tmp_path):
    """Every struct the Python binding mirrors has the header's size and the
    header's field offsets (a C program compiled against include/hosono_gpu.h
    prints them)."""
    import subprocess
    m = pkg.load()
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "hosono_gpu.h"', "int main(void) {"]
    for c, py in STRUCTS.items():
        lines.append(f'printf("{c} size %zu\\n", sizeof({c}));')
        for name, _ in getattr(m, py)._fields_:
            lines.append(f'printf("{c} {name} %zu\\n", offsetof({c}, {name}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l}
    for c, py in STRUCTS.items():
        cls = getattr(m, py)
        assert got[(c, "size")] == ctypes.sizeof(cls), c
        for name, _ in cls._fields_:
            assert got[(c, name)] == getattr(cls, name).offset, (c, name)


def test_tuning_rejects_unknown_fields():
    m = pkg.load()
    t = m.Tuning()
    t.update({"pass1_boxes": 2, "pdl": 1})
    assert t.as_dict()["pass1_boxes"] == 2 and t.as_dict()["pdl"] == 1
    with pytest.raises(TypeError):
        t.update({"pass1_box": 1})
