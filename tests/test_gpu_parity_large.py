"""Parity on the benchmarked configurations and on the multi-tile path.

Strict arithmetic, bit for bit against the oracle: U, V, the MOOD scheme and
every MOOD pass's troubled-cell masks (timeStep.f90:45-171,
detect.f90:18-236), at the sizes the bench measures:

* Orszag-Tang 2048^2, R=2, ell/Delta=12 (the roofline workload);
* Sedov 2048^2, R=2 (MOOD-heavy, outflow, hydro);
* Orszag-Tang 1024^2, R=2, ell/Delta=12;
* Orszag-Tang 640^2, R=2, ell/Delta=12: more tiles than any per-tile kernel
  keeps resident blocks, so every grid-stride tile loop takes several trips,
  the pass-1 kernel's double-buffered prefetch of the next tile runs, and
  its one-box form reloads its box per tile;
* Orszag-Tang 512^2, R=2, ell/Delta=12 to t_end = 0.5: the accuracy gate at
  t_end (relative L1 <= 1e-8 per conserved variable, div(B) within 2x of the
  oracle's, output.f90:261-274), on top of bitwise equality.

The oracle runs with every host thread; a 2048^2 step takes a few seconds.
"""
import os

import numpy as np
import pytest

import oracle
import parfiles
import pkg
from test_gpu_diagnostics import numpy_fields
from test_gpu_parity import compare_traces, rel_l1

LARGE = {
    "ot2048_r2_l12": (lambda: parfiles.orszag_tang(2048, 2, ell=12.0), 1),
    "sedov2048_r2": (lambda: parfiles.sedov(2048, 2), 1),
    "ot1024_r2_l12": (lambda: parfiles.orszag_tang(1024, 2, ell=12.0), 2),
}


@pytest.fixture(scope="module", autouse=True)
def oracle_threads():
    oracle.set_threads(os.cpu_count() or 1)


def _traced_steps(m, par, nsteps, **tuning):
    """nsteps host-launched, traced steps on both sides, compared after each."""
    o = oracle.Oracle(par)
    s = m.Solver.from_par(par, fp_mode=m.FP_STRICT)
    if tuning:
        s.set_tuning(**tuning)
    o.trace(True)
    s.trace(True)
    for step in range(nsteps):
        dt_o = o.cfl()
        dt_g = s.cfl_computedt()
        assert dt_g == dt_o, (step, dt_g, dt_o)
        o.advance(dt_o)
        s.timeStep_advanceSolution(dt_g)
        U, V, S = s.download()
        np.testing.assert_array_equal(U, o.U())
        np.testing.assert_array_equal(V, o.V())
        np.testing.assert_array_equal(S, o.scheme())
        compare_traces(s.traces(), o.traces())
        s.trace_clear()
        o.trace_clear()
    s.trace(False)
    o.trace(False)
    return o, s


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(LARGE))
def test_benchmarked_config_bitwise(case, tmp_par_dir):
    """One (or two) traced steps, then one step from the CUDA graph with dt
    computed and validated on the device."""
    m = pkg.load()
    make, nsteps = LARGE[case]
    par = parfiles.make(tmp_par_dir, case, make())
    o, s = _traced_steps(m, par, nsteps)
    s.set_graphs(True)
    s.set_time(0.0, o.tmax, nsteps, 1 << 30)
    o.advance(o.cfl())
    s.step(1)
    U, V, S = s.download()
    np.testing.assert_array_equal(U, o.U())
    np.testing.assert_array_equal(V, o.V())
    np.testing.assert_array_equal(S, o.scheme())
    s.close()
    o.close()


@pytest.mark.gpu
@pytest.mark.parametrize("boxes", [1, 2])
@pytest.mark.parametrize("staging", ["cp_async", "tma"])
def test_multi_tile_path_bitwise(staging, boxes, tmp_par_dir):
    """A grid with more tiles than any tile kernel's grid: blocks take
    several tiles each, and pass 1 either stages the next tile while
    computing one (two boxes) or reloads its one box per tile, with
    per-thread cp.async copies or one TMA copy per box."""
    m = pkg.load()
    par = parfiles.make(tmp_par_dir, "ot640", parfiles.orszag_tang(640, 2, ell=12.0))
    o, s = _traced_steps(m, par, 3, pass1_staging=m.STAGE_TMA if staging == "tma" else m.STAGE_CP_ASYNC,
                         pass1_boxes=boxes)
    info = s.launch_info()
    assert info["tiles"] > 2 * info["pass1_grid"], info
    assert info["tiles"] > info["tile_grid_max"], info
    s.set_graphs(True)
    s.set_time(0.0, o.tmax, 3, 1 << 30)
    for _ in range(3):
        o.advance(o.cfl())
    s.step(3)
    U, V, S = s.download()
    np.testing.assert_array_equal(U, o.U())
    np.testing.assert_array_equal(V, o.V())
    np.testing.assert_array_equal(S, o.scheme())
    s.close()
    o.close()


@pytest.mark.gpu
def test_multi_tile_staged_update_bitwise(tmp_par_dir):
    """The pass-1 update from TMA-staged boxes on a grid with more tiles than
    its grid of blocks (each block stages and computes several tiles in
    turn): three traced steps equal the oracle."""
    m = pkg.load()
    par = parfiles.make(tmp_par_dir, "ot640_stu", parfiles.orszag_tang(640, 2, ell=12.0))
    o, s = _traced_steps(m, par, 3, update_staging=m.STAGE_TMA)
    info = s.launch_info()
    assert info["tiles"] > 2 * info["pass1_grid"], info
    s.close()
    o.close()


@pytest.mark.gpu
def test_advance_host_banded_ot1024(tmp_par_dir):
    """The drop-in with host buffers on Orszag-Tang 1024^2, R=2, ell/Delta=12:
    its 1032 array rows take the banded upload by default (8 bands, the
    first stage's pass 1 overlapped with the copies); two steps of
    cfl_computedt + advance_host equal the oracle bit for bit."""
    m = pkg.load()
    par = parfiles.make(tmp_par_dir, "ot1024_host", parfiles.orszag_tang(1024, 2, ell=12.0))
    o = oracle.Oracle(par)
    s = m.Solver.from_par(par, fp_mode=m.FP_STRICT)
    assert s.tuning()["upload_bands"] == 0  # by size: banded from 1024 array rows
    U, _, _ = s.download()
    for _ in range(2):
        dt = o.cfl()
        assert s.cfl_computedt() == dt
        o.advance(dt)
        s.advance_host(dt, U)
        np.testing.assert_array_equal(U, o.U())
    _, V, S = s.download()
    np.testing.assert_array_equal(V, o.V())
    np.testing.assert_array_equal(S, o.scheme())
    s.close()
    o.close()


@pytest.mark.gpu
def test_t_end_gate_ot512_r2(tmp_par_dir):
    """Orszag-Tang 512^2, R=2, ell/Delta=12 to t_end = 0.5 from the CUDA
    graph: the accuracy gate (<= 1e-8 relative L1 on every conserved
    variable, mean |div B| within 2x of the oracle's), and bitwise equality."""
    m = pkg.load()
    par = parfiles.make(tmp_par_dir, "ot512", parfiles.orszag_tang(512, 2, ell=12.0))
    o = oracle.Oracle(par)
    s = m.Solver.from_par(par, fp_mode=m.FP_STRICT)
    t_g, n_g = s.run()
    rc, t_o, n_o = o.run()
    assert rc == 0 and (t_g, n_g) == (t_o, n_o) and t_g == 0.5
    U, V, S = s.download()
    Uo, Vo = o.U(), o.V()
    g = o.ngc
    for v in range(8):
        a, b = U[g:-g, g:-g, v], Uo[g:-g, g:-g, v]
        if np.abs(b).sum() > 0:
            assert rel_l1(a, b) <= 1e-8, (v, rel_l1(a, b))
    _, _, _, l1, _ = s.diagnostics()
    l1_o = np.abs(numpy_fields(Vo, s.params)["divb"]).mean()
    assert l1 <= 2 * l1_o and l1_o <= 2 * l1, (l1, l1_o)
    np.testing.assert_array_equal(U, Uo)
    np.testing.assert_array_equal(V, Vo)
    np.testing.assert_array_equal(S, o.scheme())
    st = s.stats()
    print("Orszag-Tang 512^2 R=2 to t_end: largest MOOD pass count of a stage", st["max_passes"])
    assert st["max_passes"] < m.mood_cap_default(2, 512, 512)
    s.close()
    o.close()
