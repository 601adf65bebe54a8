"""The initial state built on the device (hosono_gpu_ic, hosono_serve_submit_ic)
equals the host's hosono_ic_set bit for bit, and a served solve started that
way ends equal to its oracle run."""
import importlib

import numpy as np
import pytest

import oracle
import parfiles
import pkg

CASES = [
    ("ot", parfiles.orszag_tang(40, 2)),
    ("ot_refic", parfiles.orszag_tang(24, 1, standard=False)),
    ("sedov", parfiles.sedov(36, 2)),
    ("blast", parfiles.blast(48, 2, p_ratio=300.0, theta=0.7)),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,kv", CASES)
def test_device_ic_equals_host(name, kv, tmp_par_dir):
    m = pkg.load()
    par = parfiles.make(tmp_par_dir, name, kv)
    p, _ = m.par_load(par)
    pv, qw, st = m.par_gp(par, p.max_radius)
    U, V = m.ic_set(par, p)
    s = m.Solver(p, pv, qw, st)
    s.upload_ic(*m.ic_describe(par, p))
    Ud, Vd, _ = s.download()
    np.testing.assert_array_equal(Ud, U)
    np.testing.assert_array_equal(Vd, V)
    s.close()


@pytest.mark.gpu
def test_served_with_device_ic_equals_oracle(tmp_par_dir):
    pkg.load()
    srv = importlib.import_module("hosono_2dmhd_b200.serve")
    entries = [dict(id=0, problem="OrszagTang2d", n=40, radius=2, tmax=0.04, gap=0.0),
               dict(id=1, problem="sedov2d", n=36, radius=1, tmax=0.003, gap=0.0),
               dict(id=2, problem="explosion2d", n=44, radius=2, tmax=0.002, p_ratio=80.0, theta=0.5, gap=0.0)]
    with srv.Server() as s:
        rep, kept, infos = srv.run_stream(entries, 1.0, s, keep=[0, 1, 2], closed=True, device_ic=True)
    assert rep["completed"] == 3
    for e in entries:
        par = srv.problems.make(tmp_par_dir, f"o{e['id']}", srv.problems.from_entry(e))
        o = oracle.Oracle(par)
        rc, t, n = o.run()
        np.testing.assert_array_equal(kept[e["id"]], o.U())
