"""Launch choices and the autotuner.  Every hosono_tuning gives the same
bits (strict arithmetic: the oracle's); the autotuner times the candidates
on the instances actually held, applies the fastest, caches the choice per
(arithmetic, radii, size class, instance class), and leaves the solution
untouched."""
import numpy as np
import pytest

import oracle
import parfiles
import pkg


@pytest.mark.gpu
@pytest.mark.parametrize("boxes", [1, 2])
@pytest.mark.parametrize("staging", [0, 1])
@pytest.mark.parametrize("case", ["ot96_r2", "blast40_r1", "sedov36_r3"])
def test_every_tuning_is_bitwise(case, staging, boxes, tmp_par_dir):
    """The dynamic tile schedule of pass 1 (blocks take tiles from a shared
    counter) with either staging and one or two stencil boxes per block,
    through the step graph, equals the oracle."""
    m = pkg.load()
    kv = {"ot96_r2": lambda: parfiles.orszag_tang(96, 2), "blast40_r1": lambda: parfiles.blast(40, 1, p_ratio=500.0),
          "sedov36_r3": lambda: parfiles.sedov(36, 3)}[case]()
    par = parfiles.make(tmp_par_dir, f"{case}_{staging}_{boxes}", kv)
    o = oracle.Oracle(par)
    s = m.Solver.from_par(par, fp_mode=m.FP_STRICT)
    s.set_tuning(pass1_staging=staging, pass1_schedule=m.SCHED_DYNAMIC, pass1_boxes=boxes)
    assert s.tuning()["pass1_boxes"] == boxes
    s.set_time(0.0, o.tmax, 0, 1 << 30)
    for _ in range(3):
        o.advance(o.cfl())
    s.step(3)
    U, V, S = s.download()
    np.testing.assert_array_equal(U, o.U())
    np.testing.assert_array_equal(V, o.V())
    np.testing.assert_array_equal(S, o.scheme())
    s.close()


@pytest.mark.gpu
def test_autotune_plain_solve(tmp_par_dir):
    m = pkg.load()
    par = parfiles.make(tmp_par_dir, "tune_ot", parfiles.orszag_tang(400, 2, ell=12.0))
    o = oracle.Oracle(par)
    s = m.Solver.from_par(par, fp_mode=m.FP_STRICT)
    s.set_time(0.0, o.tmax, 0, 1 << 30)
    o.advance(o.cfl())
    s.step(1)
    rep = s.autotune(trials=3, force=True)
    assert not rep["cached"] and len(rep["table"]) == m.TUNE_MAX
    assert all(row["pass1_ms"] > 0 for row in rep["table"])
    best = min(rep["table"], key=lambda r: r["pass1_ms"])
    assert rep["best"] == {k: best[k] for k in rep["best"]}
    assert s.tuning() == rep["best"]
    # the timing launches leave the solution alone: the next steps still match
    for _ in range(2):
        o.advance(o.cfl())
    s.step(2)
    U, V, S = s.download()
    np.testing.assert_array_equal(U, o.U())
    np.testing.assert_array_equal(S, o.scheme())
    # same key: the cached choice, nothing timed
    s2 = m.Solver.from_par(par, fp_mode=m.FP_STRICT)
    rep2 = s2.autotune(trials=3)
    assert rep2["cached"] and rep2["best"] == rep["best"] and s2.tuning() == rep["best"]
    s2.close()
    s.close()


@pytest.mark.gpu
def test_autotune_batch_mix(tmp_par_dir):
    m = pkg.load()
    kvs = [parfiles.blast(64, 2, p_ratio=300.0, theta=0.2), parfiles.orszag_tang(48, 1),
           parfiles.blast(96, 2, p_ratio=30.0, theta=1.1), parfiles.sedov(40, 2)]
    pars = [parfiles.make(tmp_par_dir, f"tb{i}", kv) for i, kv in enumerate(kvs)]
    tiles = sum(m.Batch.tiles_for(m.par_load(p)[0]) for p in pars)
    b = m.Batch(len(pars), tiles, fp_mode=m.FP_STRICT)
    slots = [b.add_par(p) for p in pars]
    for k in slots:
        b.set_time(k, 0.0, 1e30)
    rep = b.autotune(trials=2, force=True)
    assert rep["instances"] == len(pars) and len(rep["table"]) == m.TUNE_MAX
    b.run(max_steps=2)
    for k, p in zip(slots, pars):
        o = oracle.Oracle(p)
        for _ in range(2):
            o.advance(o.cfl())
        U, V, S = b.download(k)
        np.testing.assert_array_equal(U, o.U())
    b.close()


PERSISTENT_CASES = {
    "blast40_r2": lambda: parfiles.blast(40, 2, p_ratio=1000.0, theta=0.3),
    "sedov36_r3": lambda: parfiles.sedov(36, 3),
    "ot128_r1": lambda: parfiles.orszag_tang(128, 1),
    "blast36_r1": lambda: parfiles.blast(36, 1, p_ratio=300.0, theta=1.0),
}


@pytest.mark.gpu
@pytest.mark.parametrize("graphs", [True, False])
@pytest.mark.parametrize("case", sorted(PERSISTENT_CASES))
def test_persistent_later_passes_bitwise(case, graphs, tmp_par_dir):
    """Every later MOOD pass of a stage in one persistent launch (grid-wide
    barriers between the phases) gives the oracle's bits, from the step
    graph and from host launches."""
    m = pkg.load()
    par = parfiles.make(tmp_par_dir, f"pers_{case}_{int(graphs)}", PERSISTENT_CASES[case]())
    o = oracle.Oracle(par)
    s = m.Solver.from_par(par, fp_mode=m.FP_STRICT)
    s.set_tuning(later_passes=m.LATER_PERSISTENT)
    s.set_graphs(graphs)
    s.set_time(0.0, o.tmax, 0, 1 << 30)
    for chunk in (1, 4):
        for _ in range(chunk):
            o.advance(o.cfl())
        s.step(chunk)
        U, V, S = s.download()
        np.testing.assert_array_equal(U, o.U())
        np.testing.assert_array_equal(V, o.V())
        np.testing.assert_array_equal(S, o.scheme())
    if case != "ot128_r1":  # early Orszag-Tang steps converge in one pass per stage
        assert s.stats()["mood_passes"] > s.stats()["stages"]  # later passes did run
    s.close()


@pytest.mark.gpu
def test_persistent_later_passes_batch(tmp_par_dir):
    """The persistent launch over a batch of uneven MOOD-active instances:
    each equals its own oracle run."""
    m = pkg.load()
    kvs = [parfiles.blast(64, 2, p_ratio=300.0, theta=0.2), parfiles.orszag_tang(48, 1),
           parfiles.blast(96, 2, p_ratio=30.0, theta=1.1), parfiles.sedov(40, 2), parfiles.blast(32, 1, p_ratio=50.0)]
    pars = [parfiles.make(tmp_par_dir, f"pb{i}", kv) for i, kv in enumerate(kvs)]
    tiles = sum(m.Batch.tiles_for(m.par_load(p)[0]) for p in pars)
    b = m.Batch(len(pars), tiles, fp_mode=m.FP_STRICT)
    b.set_tuning(later_passes=m.LATER_PERSISTENT)
    slots = [b.add_par(p) for p in pars]
    for k in slots:
        b.set_time(k, 0.0, 1e30)
    b.run(max_steps=3)
    for k, p in zip(slots, pars):
        o = oracle.Oracle(p)
        for _ in range(3):
            o.advance(o.cfl())
        U, V, S = b.download(k)
        np.testing.assert_array_equal(U, o.U())
        np.testing.assert_array_equal(S, o.scheme())
    b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("graphs", [True, False])
@pytest.mark.parametrize("case", sorted(PERSISTENT_CASES))
def test_programmatic_launch_bitwise(case, graphs, tmp_par_dir):
    """The step's kernels as programmatic dependent launches (each waits on
    the GPU for its predecessor before touching memory) give the oracle's
    bits, from the step graph and from host launches."""
    m = pkg.load()
    par = parfiles.make(tmp_par_dir, f"pdl_{case}_{int(graphs)}", PERSISTENT_CASES[case]())
    o = oracle.Oracle(par)
    s = m.Solver.from_par(par, fp_mode=m.FP_STRICT)
    s.set_tuning(pdl=1)
    assert s.tuning()["pdl"] == 1
    s.set_graphs(graphs)
    s.set_time(0.0, o.tmax, 0, 1 << 30)
    for chunk in (1, 4):
        for _ in range(chunk):
            o.advance(o.cfl())
        s.step(chunk)
        U, V, S = s.download()
        np.testing.assert_array_equal(U, o.U())
        np.testing.assert_array_equal(V, o.V())
        np.testing.assert_array_equal(S, o.scheme())
    s.close()


@pytest.mark.gpu
def test_programmatic_launch_batch(tmp_par_dir):
    """Programmatic dependent launches over a batch of uneven MOOD-active
    instances: each equals its own oracle run."""
    m = pkg.load()
    kvs = [parfiles.blast(64, 2, p_ratio=300.0, theta=0.2), parfiles.orszag_tang(48, 1),
           parfiles.blast(96, 2, p_ratio=30.0, theta=1.1), parfiles.sedov(40, 2)]
    pars = [parfiles.make(tmp_par_dir, f"pdlb{i}", kv) for i, kv in enumerate(kvs)]
    tiles = sum(m.Batch.tiles_for(m.par_load(p)[0]) for p in pars)
    b = m.Batch(len(pars), tiles, fp_mode=m.FP_STRICT)
    b.set_tuning(pdl=1)
    slots = [b.add_par(p) for p in pars]
    for k in slots:
        b.set_time(k, 0.0, 1e30)
    b.run(max_steps=3)
    for k, p in zip(slots, pars):
        o = oracle.Oracle(p)
        for _ in range(3):
            o.advance(o.cfl())
        U, V, S = b.download(k)
        np.testing.assert_array_equal(U, o.U())
        np.testing.assert_array_equal(S, o.scheme())
    b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("graphs", [True, False])
@pytest.mark.parametrize("case", sorted(PERSISTENT_CASES) + ["ot96_r2"])
def test_staged_update_bitwise(case, graphs, tmp_par_dir):
    """The pass-1 update (per-stage detect terms, FLICD, update, detect) from
    TMA-staged boxes of U, FX and FY gives the oracle's bits, as the cached
    version does."""
    m = pkg.load()
    kv = parfiles.orszag_tang(96, 2) if case == "ot96_r2" else PERSISTENT_CASES[case]()
    par = parfiles.make(tmp_par_dir, f"stu_{case}_{int(graphs)}", kv)
    o = oracle.Oracle(par)
    s = m.Solver.from_par(par, fp_mode=m.FP_STRICT)
    s.set_tuning(update_staging=m.STAGE_TMA)
    assert s.tuning()["update_staging"] == m.STAGE_TMA
    s.set_graphs(graphs)
    s.set_time(0.0, o.tmax, 0, 1 << 30)
    for chunk in (1, 4):
        for _ in range(chunk):
            o.advance(o.cfl())
        s.step(chunk)
        U, V, S = s.download()
        np.testing.assert_array_equal(U, o.U())
        np.testing.assert_array_equal(V, o.V())
        np.testing.assert_array_equal(S, o.scheme())
    s.close()


@pytest.mark.gpu
def test_staged_update_batch(tmp_par_dir):
    """The staged pass-1 update over a batch of uneven instances (outflow and
    periodic, R = 1 and 2): each equals its own oracle run."""
    m = pkg.load()
    kvs = [parfiles.blast(64, 2, p_ratio=300.0, theta=0.2), parfiles.orszag_tang(48, 1),
           parfiles.blast(96, 2, p_ratio=30.0, theta=1.1), parfiles.sedov(40, 2)]
    pars = [parfiles.make(tmp_par_dir, f"stub{i}", kv) for i, kv in enumerate(kvs)]
    tiles = sum(m.Batch.tiles_for(m.par_load(p)[0]) for p in pars)
    b = m.Batch(len(pars), tiles, fp_mode=m.FP_STRICT)
    b.set_tuning(update_staging=m.STAGE_TMA)
    slots = [b.add_par(p) for p in pars]
    for k in slots:
        b.set_time(k, 0.0, 1e30)
    b.run(max_steps=3)
    for k, p in zip(slots, pars):
        o = oracle.Oracle(p)
        for _ in range(3):
            o.advance(o.cfl())
        U, V, S = b.download(k)
        np.testing.assert_array_equal(U, o.U())
        np.testing.assert_array_equal(S, o.scheme())
    b.close()
