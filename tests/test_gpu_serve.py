"""Serving form: solves of different problems, sizes and radii submitted at
different times share the GPU through continuous batching; each result must
be the same alone and in the mix, and equal to its own oracle run to t_end
(strict arithmetic: bit for bit)."""
import importlib
import threading
import time

import numpy as np
import pytest

import oracle
import pkg

ENTRIES = [
    dict(id=0, problem="OrszagTang2d", n=48, radius=2, tmax=0.05, gap=0.0),
    dict(id=1, problem="sedov2d", n=40, radius=2, tmax=0.004, gap=0.02),
    dict(id=2, problem="explosion2d", n=64, radius=2, tmax=0.003, p_ratio=100.0, theta=0.4, gap=0.01),
    dict(id=3, problem="OrszagTang2d", n=33, radius=1, tmax=0.1, gap=0.03),
    dict(id=4, problem="sedov2d", n=56, radius=1, tmax=0.002, gap=0.0),
    dict(id=5, problem="explosion2d", n=40, radius=1, tmax=0.002, p_ratio=30.0, theta=1.2, gap=0.02),
]


def _serve():
    pkg.load()
    return importlib.import_module("hosono_2dmhd_b200.serve")


def _oracle_final(e, tmp_par_dir):
    srv = _serve()
    par = srv.problems.make(tmp_par_dir, f"o{e['id']}", srv.problems.from_entry(e))
    o = oracle.Oracle(par)
    rc, t, n = o.run()
    assert rc == 0
    return o.U(), t, n


@pytest.mark.gpu
def test_served_mix_equals_alone_and_oracle(tmp_par_dir):
    srv = _serve()
    keep = [e["id"] for e in ENTRIES]
    with srv.Server() as s:
        mix, kept, infos = srv.run_stream(ENTRIES, rate=100.0, server=s, keep=keep)
    assert mix["completed"] == len(ENTRIES) and mix["failed"] == 0
    assert mix["peak_resident"] >= 2  # the solves overlapped on the device
    for e in ENTRIES:
        with srv.Server() as s:
            alone, kept1, inf1 = srv.run_stream([dict(e, gap=0.0)], rate=1.0, server=s, keep=[e["id"]])
        np.testing.assert_array_equal(kept[e["id"]], kept1[e["id"]])
        U, t, n = _oracle_final(e, tmp_par_dir)
        np.testing.assert_array_equal(kept[e["id"]], U)
        info = next(i for i in infos if i["entry"] == e["id"])
        assert info["t"] == t and info["nstep"] == n
        assert info["zone_updates"] == e["n"] * e["n"] * n


@pytest.mark.gpu
def test_admission_waits_for_memory_budget(tmp_par_dir):
    """A budget that holds about two of the solves: the rest wait in the queue
    (head-of-line) and are admitted as memory is freed; results unchanged."""
    m = pkg.load()
    srv = _serve()
    sizes = []
    for e in ENTRIES:
        p, *_ = srv.prepare(e, tmp_par_dir)
        sizes.append(m.Batch.instance_bytes(p))
    budget = sorted(sizes)[-1] + sorted(sizes)[-2] + 4096
    with srv.Server(memory_budget=budget) as s:
        rep, kept, infos = srv.run_stream(ENTRIES, rate=1.0, server=s, keep=[0, 3], closed=True)
        st = s.stats()
    assert rep["completed"] == len(ENTRIES)
    assert st["peak_bytes"] <= budget and st["head_blocked"] > 0
    assert 1 <= st["peak_resident"] < len(ENTRIES)
    for eid in (0, 3):
        U, _, _ = _oracle_final(ENTRIES[eid], tmp_par_dir)
        np.testing.assert_array_equal(kept[eid], U)


@pytest.mark.gpu
def test_snapshot_of_a_resident_solve(tmp_par_dir):
    m = pkg.load()
    srv = _serve()
    e = dict(ENTRIES[0], tmax=0.5, n=64)
    p, pv, qw, st, U0, V0, tmax = srv.prepare(e, tmp_par_dir)
    with srv.Server(chunk_ms=1.0, max_chunk_steps=1) as s:
        rid = s.submit(p, pv, qw, st, U0, V0, tmax)
        deadline = time.time() + 60
        while s.info(rid)["nstep"] < 3 and time.time() < deadline:
            time.sleep(0.005)
        t, n, U, V, S = s.snapshot(rid, p)
        assert 0 < t < tmax and n >= 3
        info, Uf, _, _ = s.wait(rid)
        assert info["status"] == 0 and info["nstep"] > n
    par = srv.problems.make(tmp_par_dir, "snap", srv.problems.from_entry(e))
    o = oracle.Oracle(par)
    for _ in range(n):
        o.advance(o.cfl())
    np.testing.assert_array_equal(U, o.U())


@pytest.mark.gpu
def test_oversized_solve_refused_and_shutdown_cancels(tmp_par_dir):
    m = pkg.load()
    srv = _serve()
    p, pv, qw, st, U0, V0, tmax = srv.prepare(ENTRIES[2], tmp_par_dir)
    with srv.Server(memory_budget=m.Batch.instance_bytes(p) // 2) as s:
        with pytest.raises(m.HosonoError) as ex:
            s.submit(p, pv, qw, st, U0, V0, tmax)
        assert ex.value.code == m.ENOMEM
    s = srv.Server(max_resident=1)
    ids = [s.submit(p, pv, qw, st, U0, V0, 10.0) for _ in range(3)]  # long solves: the first is resident
    out = []
    th = threading.Thread(target=lambda: out.append(s.wait(ids[2])))  # still queued at close
    th.start()
    time.sleep(0.3)
    assert s.info(ids[0])["state"] == m.REQ_RUNNING and s.info(ids[2])["state"] == m.REQ_QUEUED
    s.close()
    th.join(30)
    assert out and out[0][0]["status"] == m.ECANCELED


@pytest.mark.gpu
def test_failed_solve_is_isolated(tmp_par_dir):
    """A solve with a negative CFL number gets a negative first dt, which
    validTimeStep rejects: it leaves with HOSONO_ENANDT at step 0 while the
    solves resident beside it finish unchanged.  (NaN wave speeds would not
    do: the CFL maximum, like the oracle's, is an fmax that drops NaN.)"""
    m = pkg.load()
    srv = _serve()
    good = [ENTRIES[0], ENTRIES[3]]
    prepared = [srv.prepare(e, tmp_par_dir) for e in good]
    p, pv, qw, st, U0, V0, tmax = srv.prepare(dict(ENTRIES[2], id=9), tmp_par_dir)
    p = type(p).from_buffer_copy(p)
    p.cfl = -abs(p.cfl)
    with srv.Server() as s:
        ids = [s.submit(*prep) for prep in prepared]
        bid = s.submit(p, pv, qw, st, U0, V0, tmax)
        infos = [s.wait(i) for i in ids]
        binfo = s.wait(bid)[0]
    assert binfo["status"] == m.ENANDT and binfo["nstep"] == 0
    for e, (info, U, _, _) in zip(good, infos):
        assert info["status"] == 0
        Uo, _, _ = _oracle_final(e, tmp_par_dir)
        np.testing.assert_array_equal(U, Uo)


@pytest.mark.gpu
def test_shortest_first_policy_gives_the_same_results(tmp_par_dir):
    """SERVE_SHORTEST admits the least estimated work first and lets the
    residents with the most remaining work sit launches out (fill_tiles set
    low so that they do): every solve still ends bit-identical to its oracle
    run, and the short ones finish before the long ones that arrived with
    them."""
    m = pkg.load()
    srv = _serve()
    keep = [e["id"] for e in ENTRIES]
    with srv.Server(policy=m.SERVE_SHORTEST, fill_tiles=1, chunk_ms=2.0) as s:
        rep, kept, infos = srv.run_stream(ENTRIES, rate=1.0, server=s, keep=keep, closed=True)
    assert rep["completed"] == len(ENTRIES) and rep["failed"] == 0
    for e in ENTRIES:
        U, t, n = _oracle_final(e, tmp_par_dir)
        np.testing.assert_array_equal(kept[e["id"]], U)
        info = next(i for i in infos if i["entry"] == e["id"])
        assert info["t"] == t and info["nstep"] == n
    work = {i["entry"]: i["zone_updates"] for i in infos}
    fin = {i["entry"]: i["finish_s"] for i in infos}
    small, big = min(work, key=work.get), max(work, key=work.get)
    assert fin[small] < fin[big]


@pytest.mark.gpu
def test_released_solve_is_forgotten(tmp_par_dir):
    m = pkg.load()
    srv = _serve()
    p, pv, qw, st, U0, V0, tmax = srv.prepare(ENTRIES[0], tmp_par_dir)
    with srv.Server() as s:
        rid = s.submit(p, pv, qw, st, U0, V0, tmax)
        info = s.wait(rid, release=False)[0]
        assert info["status"] == 0 and s.info(rid)["state"] == m.REQ_DONE
        s.release(rid)
        with pytest.raises(m.HosonoError) as e:
            s.info(rid)
        assert e.value.code == m.EINVAL
