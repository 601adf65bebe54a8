"""The operation-counting build of the oracle (oracle/flopcount.h; CPU
only): it computes exactly what the strict build computes, attributes its
counts to the phases of the step, and reproduces the pass-1 operation count
per cell that bench.py's FP64 roofline uses."""
import importlib.util
import os

import numpy as np
import pytest

import oracle
import parfiles

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="module", autouse=True)
def one_thread():
    oracle.set_threads(1, count=True)  # the counters are plain globals


@pytest.mark.parametrize("case", ["orszag_tang", "blast"])
def test_counting_build_is_bit_identical(case, tmp_par_dir):
    kv = parfiles.orszag_tang(48, 2) if case == "orszag_tang" else parfiles.blast(48, 2, p_ratio=300.0)
    par = parfiles.make(tmp_par_dir, f"count_{case}", kv)
    a, b = oracle.Oracle(par), oracle.Oracle(par, count=True)
    for _ in range(3):
        dt = a.cfl()
        assert b.cfl() == dt
        a.advance(dt)
        b.advance(dt)
    np.testing.assert_array_equal(a.U(), b.U())
    np.testing.assert_array_equal(a.V(), b.V())
    np.testing.assert_array_equal(a.scheme(), b.scheme())


def test_phases(tmp_par_dir):
    """Early Orszag-Tang converges in one MOOD pass per stage (no later-pass
    work); the blast needs later passes.  Pass 1 dominates either way."""
    for case, kv, later in [("ot", parfiles.orszag_tang(48, 2), False), ("blast", parfiles.blast(48, 2, 300.0), True)]:
        o = oracle.Oracle(parfiles.make(tmp_par_dir, f"phases_{case}", kv), count=True)
        dt = o.cfl()
        oracle.count_reset()
        o.advance(dt)
        c = oracle.count_get()
        assert (c["later_passes"]["flops"] > 0) == later, case
        assert c["pass1"]["flops"] > 10 * c["update_detect"]["flops"] > 0
        assert c["pass1"]["div"] > 0 and c["pass1"]["sqrt"] > 0


def test_pass1_count_matches_bench_constant(tmp_par_dir):
    """Orszag-Tang 512^2, R=2, ell/dx=12: pass-1 flops per zone-update within
    2 % above the 2048^2 count bench.py uses (the reconstruction range is
    N+4 cells wide, so a smaller grid does relatively more halo work)."""
    b = _bench()
    per_launch = b.PASS1_FLOPS[("ot", 2, 12.0)]
    o = oracle.Oracle(parfiles.make(tmp_par_dir, "count_ot512", parfiles.orszag_tang(512, 2, ell=12.0)), count=True)
    dt = o.cfl()
    oracle.count_reset()
    o.advance(dt)
    per_zu = oracle.count_get()["pass1"]["flops"] / 512 ** 2
    assert 1.0 <= per_zu / (3 * per_launch) <= 1.02
