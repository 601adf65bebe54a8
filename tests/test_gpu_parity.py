"""GPU path (through the C ABI) against the oracle on identical inputs.

Strict arithmetic (no FMA contraction) must reproduce the oracle bit for bit:
U, V, the MOOD scheme and every pass's troubled-cell masks.  The FMA build
must stay within the parity tolerance of 1e-12 relative L1 after one step.
"""
import numpy as np
import pytest

import oracle
import parfiles
import pkg

CASES = {
    "ot32_r1": lambda: parfiles.orszag_tang(32, 1),
    "ot32_r2": lambda: parfiles.orszag_tang(32, 2),
    "ot24_r3_refic": lambda: parfiles.orszag_tang(24, 3, standard=False),
    "sedov32_r2": lambda: parfiles.sedov(32, 2),
    "sedov33x40_r1": lambda: dict(parfiles.sedov(33, 1), grid_Ny="40", grid_yEnd="0.7"),
    "blast40_r2": lambda: parfiles.blast(40, 2, p_ratio=1000.0, theta=0.3),
    "blast36_r3": lambda: parfiles.blast(36, 3, p_ratio=100.0, theta=1.2),
}


def rel_l1(a, b):
    return np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300)


def compare_traces(gt, ot):
    assert len(gt) == len(ot), (len(gt), len(ot))
    for g, o in zip(gt, ot):
        assert (g["stage"], g["mood_pass"], g["n_inner"], g["n_detect"]) == \
               (o["stage"], o["mood_pass"], o["n_inner"], o["n_detect"]), (g, o)
        np.testing.assert_array_equal(g["detect"], o["detect"])
        np.testing.assert_array_equal(g["inner"], o["inner"])


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(CASES))
def test_strict_bitwise_steps(case, tmp_par_dir):
    m = pkg.load()
    par = parfiles.make(tmp_par_dir, case, CASES[case]())
    o = oracle.Oracle(par)
    s = m.Solver.from_par(par, fp_mode=m.FP_STRICT)
    o.trace(True)
    s.trace(True)
    nsteps = 6
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
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["ot32_r1", "ot24_r3_refic", "sedov32_r2", "blast40_r2"])
def test_strict_bitwise_graph_path(case, tmp_par_dir):
    """The production path (whole step from a CUDA graph with conditional MOOD
    loops, dt computed and validated on the device) equals the oracle's
    driver loop bit for bit."""
    m = pkg.load()
    par = parfiles.make(tmp_par_dir, case + "_g", CASES[case]())
    o = oracle.Oracle(par)
    s = m.Solver.from_par(par, fp_mode=m.FP_STRICT)
    s.set_time(0.0, o.tmax, 0, 1 << 30)
    for chunk in (1, 3, 4):
        for _ in range(chunk):
            dt = o.cfl()
            o.advance(dt)
        s.step(chunk)
        U, V, S = s.download()
        np.testing.assert_array_equal(U, o.U())
        np.testing.assert_array_equal(V, o.V())
        np.testing.assert_array_equal(S, o.scheme())
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["ot32_r2", "blast40_r2", "sedov32_r2"])
def test_fast_one_step_tolerance(case, tmp_par_dir):
    """FMA build: one RK3 step within 1e-12 relative L1 on all 8 variables."""
    m = pkg.load()
    par = parfiles.make(tmp_par_dir, case, CASES[case]())
    o = oracle.Oracle(par)
    s = m.Solver.from_par(par, fp_mode=m.FP_FAST)
    dt = o.cfl()
    assert abs(s.cfl_computedt() - dt) <= 1e-14 * dt
    o.advance(dt)
    s.timeStep_advanceSolution(dt)
    U, _, _ = s.download()
    Uo = o.U()
    g = o.ngc
    for v in range(8):
        a, b = U[g:-g, g:-g, v], Uo[g:-g, g:-g, v]
        if np.abs(b).sum() > 0:
            assert rel_l1(a, b) <= 1e-12, (v, rel_l1(a, b))
    s.close()


@pytest.mark.gpu
def test_orszag_tang_128_r1_to_t_end(tmp_par_dir):
    """The reference's own runnable case (OT 128^2, R=1, t_end=0.5): strict
    path bit-identical to the oracle at t_end."""
    m = pkg.load()
    par = parfiles.make(tmp_par_dir, "ot128", parfiles.orszag_tang(128, 1))
    o = oracle.Oracle(par)
    s = m.Solver.from_par(par, fp_mode=m.FP_STRICT)
    rc, t_o, n_o = o.run()
    t_g, n_g = s.run()
    assert rc == 0 and n_g == n_o and t_g == t_o == 0.5
    U, V, S = s.download()
    np.testing.assert_array_equal(U, o.U())
    np.testing.assert_array_equal(V, o.V())
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("staging", ["tma", "cp_async_static"])
@pytest.mark.parametrize("case", ["ot32_r1", "ot24_r3_refic", "sedov33x40_r1", "blast40_r2"])
def test_pass1_staging_bitwise(case, staging, tmp_par_dir):
    """Pass 1 with its stencil box staged by TMA (one cp.async.bulk.tensor per
    box, zero fill beyond the array; the default) or by per-thread cp.async
    copies on the round-robin tile schedule gives the oracle's bits."""
    m = pkg.load()
    par = parfiles.make(tmp_par_dir, f"{case}_{staging}", CASES[case]())
    o = oracle.Oracle(par)
    s = m.Solver.from_par(par, fp_mode=m.FP_STRICT)
    if staging == "tma":
        assert s.tuning()["pass1_staging"] == m.STAGE_TMA  # the default
    else:
        s.set_tuning(pass1_staging=m.STAGE_CP_ASYNC, pass1_schedule=m.SCHED_STATIC)
        assert s.tuning()["pass1_staging"] == m.STAGE_CP_ASYNC
    s.set_time(0.0, o.tmax, 0, 1 << 30)
    for chunk in (1, 3):
        for _ in range(chunk):
            o.advance(o.cfl())
        s.step(chunk)
        U, V, S = s.download()
        np.testing.assert_array_equal(U, o.U())
        np.testing.assert_array_equal(V, o.V())
        np.testing.assert_array_equal(S, o.scheme())
    s.close()


BANDED = {
    "ot96_r2_b4": (lambda: parfiles.orszag_tang(96, 2), 4),
    "sedov100_r2_b3": (lambda: parfiles.sedov(100, 2), 3),
    "blast72_r3_b16": (lambda: parfiles.blast(72, 3, p_ratio=300.0, theta=0.4), 16),
    "ot64_r1_b2": (lambda: parfiles.orszag_tang(64, 1), 2),
}


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(BANDED))
def test_advance_host_banded_upload(case, tmp_par_dir):
    """hosono_gpu_advance_host with the upload in row bands overlapped with the
    first stage's pass 1 (each band's tiles computed once its rows and halo
    have landed): three steps equal the oracle bit for bit, and the same as
    the unbanded call."""
    m = pkg.load()
    make, bands = BANDED[case]
    par = parfiles.make(tmp_par_dir, case, make())
    o = oracle.Oracle(par)
    s = m.Solver.from_par(par, fp_mode=m.FP_STRICT)
    s.set_tuning(upload_bands=bands)
    assert s.tuning()["upload_bands"] == bands
    U, V, _ = s.download()
    for step in range(3):
        dt = o.cfl()
        assert s.cfl_computedt() == dt
        o.advance(dt)
        s.advance_host(dt, U, V)
        np.testing.assert_array_equal(U, o.U())
        np.testing.assert_array_equal(V, o.V())
    _, _, S = s.download()
    np.testing.assert_array_equal(S, o.scheme())
    with pytest.raises(m.HosonoError):
        s.set_tuning(upload_bands=m.UPLOAD_BANDS_MAX + 1)
    s.close()
    o.close()


@pytest.mark.gpu
@pytest.mark.parametrize("bands", [1, 3])
def test_advance_host_failed_step_keeps_state(bands, tmp_par_dir):
    """A host-buffer step that stops with HOSONO_EMOODCAP (MOOD pass cap 1 on
    a blast that needs several passes) leaves the caller's U untouched and
    the device holding the uploaded U with its V: the next cfl_computedt is
    the oracle's on that state."""
    m = pkg.load()
    par = parfiles.make(tmp_par_dir, f"capfail_{bands}", parfiles.blast(40, 2, p_ratio=1000.0, theta=0.3))
    o = oracle.Oracle(par)
    s = m.Solver.from_par(par, fp_mode=m.FP_STRICT)
    s.set_tuning(upload_bands=bands)
    o.advance(o.cfl())  # a state the device has not seen: one oracle step ahead
    U1 = o.U().copy()
    s.set_mood_cap(1)
    U_in = U1.copy()
    with pytest.raises(m.HosonoError) as e:
        s.advance_host(o.cfl(), U_in)
    assert e.value.code == m.EMOODCAP
    np.testing.assert_array_equal(U_in, U1)
    assert s.cfl_computedt() == o.cfl()
    U_dev, V_dev, _ = s.download()
    np.testing.assert_array_equal(U_dev, U1)
    np.testing.assert_array_equal(V_dev, o.V())
    s.close()
    o.close()


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["ot32_r2", "sedov32_r2", "blast40_r2"])
def test_advance_host_drop_in(case, tmp_par_dir):
    """hosono_gpu_advance_host, the form a driver that keeps grid_state on
    the host binds: the host U (and V, or none: then V = cons2prim(U) on the
    device) goes in, the advanced U and V come back in place; three steps of
    cfl_computedt + advance_host equal the oracle bit for bit."""
    m = pkg.load()
    par = parfiles.make(tmp_par_dir, case + "_host", CASES[case]())
    o = oracle.Oracle(par)
    s = m.Solver.from_par(par, fp_mode=m.FP_STRICT)
    U, V, _ = s.download()
    for step in range(3):
        dt = o.cfl()
        assert s.cfl_computedt() == dt
        o.advance(dt)
        if step == 1:
            s.advance_host(dt, U)  # U alone: V rebuilt on the device, V not returned
            _, V, _ = s.download()
        else:
            s.advance_host(dt, U, V)
        np.testing.assert_array_equal(U, o.U())
        np.testing.assert_array_equal(V, o.V())
    s.close()
