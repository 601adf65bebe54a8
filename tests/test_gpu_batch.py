"""Batched engine: independent instances of different problems, sizes, radii
and boundary conditions advanced together must each equal their own oracle
run bit for bit (strict arithmetic), each with its own dt."""
import os

import numpy as np
import pytest

import oracle
import parfiles
import pkg

MIX = [
    ("ot40_r2", lambda: parfiles.orszag_tang(40, 2)),
    ("sedov36x48_r2", lambda: dict(parfiles.sedov(36, 2), grid_Ny="48", grid_yEnd="0.8333333333333334")),
    ("blast32_r1", lambda: parfiles.blast(32, 1, p_ratio=50.0, theta=0.9)),
    ("blast44_r3", lambda: parfiles.blast(44, 3, p_ratio=800.0, theta=0.2)),
    ("ot24_r1_refic", lambda: parfiles.orszag_tang(24, 1, standard=False)),
]


def _make(tmp_par_dir):
    pars = [parfiles.make(tmp_par_dir, name, f()) for name, f in MIX]
    return pars


@pytest.mark.gpu
@pytest.mark.parametrize("graphs", [True, False])
def test_batch_matches_independent_oracles(graphs, tmp_par_dir):
    m = pkg.load()
    pars = _make(tmp_par_dir)
    tiles = sum(m.Batch.tiles_for(m.par_load(p)[0]) for p in pars)
    b = m.Batch(len(pars) + 2, tiles + 64, fp_mode=m.FP_STRICT)
    b.set_graphs(graphs)
    slots = [b.add_par(p) for p in pars]
    for k in slots:  # no tmax clamp: the oracle loop below steps with the raw CFL dt
        b.set_time(k, 0.0, 1e30)
    refs = [oracle.Oracle(p) for p in pars]
    for chunk in (2, 3):
        b.run(max_steps=chunk)
        for o in refs:
            for _ in range(chunk):
                o.advance(o.cfl())
        for k, o in zip(slots, refs):
            U, V, S = b.download(k)
            np.testing.assert_array_equal(U, o.U())
            np.testing.assert_array_equal(V, o.V())
            np.testing.assert_array_equal(S, o.scheme())
            st = b.status(k)
            assert st["error"] == 0 and st["nstep"] == (2 if chunk == 2 else 5)
    b.close()


@pytest.mark.gpu
def test_batch_runs_each_instance_to_its_own_tmax(tmp_par_dir):
    """Continuous batching: instances with different tmax finish at their own
    time; a finished instance is removed and a new one admitted into the
    running batch; results equal independent oracle runs to t_end."""
    m = pkg.load()
    kvs = [parfiles.orszag_tang(32, 1, tmax=0.05), parfiles.blast(32, 2, p_ratio=100.0, tmax=0.004),
           parfiles.sedov(32, 2, tmax=0.002)]
    pars = [parfiles.make(tmp_par_dir, f"tm{i}", kv) for i, kv in enumerate(kvs)]
    b = m.Batch(4, 4 * 64, fp_mode=m.FP_STRICT)
    slots = [b.add_par(p) for p in pars[:2]]
    b.run(max_steps=3)
    # admit the third while the first two are mid-run
    slots.append(b.add_par(pars[2]))
    b.run()  # until every instance reaches its tmax
    for k, p in zip(slots, pars):
        o = oracle.Oracle(p)
        rc, t, n = o.run()
        st = b.status(k)
        assert st["done"] and st["error"] == 0
        assert st["t"] == t and st["nstep"] == n
        U, V, S = b.download(k)
        np.testing.assert_array_equal(U, o.U())
    # remove one and admit a new instance into its slot
    b.remove(slots[0])
    k = b.add_par(pars[0])
    b.run()
    o = oracle.Oracle(pars[0])
    o.run()
    np.testing.assert_array_equal(b.download(k)[0], o.U())
    b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("graphs", [True, False])
def test_mood_cap_stops_only_its_instance(graphs, tmp_par_dir):
    """A stage that reaches its MOOD pass cap stops its instance with
    HOSONO_EMOODCAP, its state left at the start of the step, while the other
    instances of the batch run on bit-identical to their oracle runs."""
    m = pkg.load()
    kvs = [parfiles.blast(40, 2, p_ratio=1000.0, theta=0.3), parfiles.orszag_tang(32, 2),
           parfiles.blast(32, 1, p_ratio=50.0, theta=0.9)]
    pars = [parfiles.make(tmp_par_dir, f"cap{i}", kv) for i, kv in enumerate(kvs)]
    # precondition: a stage of the capped solve's first step needs more than one MOOD pass
    o0 = oracle.Oracle(pars[0])
    o0.trace(True)
    o0.advance(o0.cfl())
    assert max(t["mood_pass"] for t in o0.traces(masks=False)) >= 1
    o0.close()
    tiles = sum(m.Batch.tiles_for(m.par_load(p)[0]) for p in pars)
    b = m.Batch(len(pars), tiles, fp_mode=m.FP_STRICT)
    b.set_graphs(graphs)
    slots = [b.add_par(p) for p in pars]
    for k in slots:
        b.set_time(k, 0.0, 1e30)
    U0 = b.download(slots[0])[0]
    b.set_mood_cap(slots[0], 1)
    with pytest.raises(m.HosonoError) as e:
        b.run(max_steps=2)
    assert e.value.code == m.EMOODCAP
    st = b.status(slots[0])
    assert st["done"] and st["error"] == m.EMOODCAP and st["nstep"] == 0
    np.testing.assert_array_equal(b.download(slots[0])[0], U0)
    for k, p in zip(slots[1:], pars[1:]):
        o = oracle.Oracle(p)
        for _ in range(2):
            o.advance(o.cfl())
        st = b.status(k)
        assert st["error"] == 0 and st["nstep"] == 2
        U, V, S = b.download(k)
        np.testing.assert_array_equal(U, o.U())
        np.testing.assert_array_equal(S, o.scheme())
    b.close()


def test_mood_cap_default_matches_header():
    m = pkg.load()
    src = open(os.path.join(pkg.ROOT, "include", "hosono_gpu.h")).read()
    assert "#define HOSONO_MOOD_CAP_DEFAULT(R, nx, ny) (((R) + 1) * ((nx) + (ny)))" in src
    assert [m.mood_cap_default(r, 512, 256) for r in (1, 2, 3)] == [1536, 2304, 3072]
