"""The GP table cache of hosono_gp_build (CPU only): a hit returns exactly
the bits of a fresh build (and of the oracle's GP_init), inputs that give
the same quad-precision spacing share an entry, other inputs miss, and
concurrent callers get the same tables."""
import threading

import numpy as np

import oracle
import pkg


def _build(m, R, x0, x1, nx, ell, y0=None, y1=None, ny=None):
    return m.gp_build(R, x0, x1, nx, x0 if y0 is None else y0, x1 if y1 is None else y1, nx if ny is None else ny,
                      ell)


def _same(a, b):
    return all(np.array_equal(x, y) for x, y in zip(a, b))


def test_hit_returns_the_fresh_bits():
    m = pkg.load()
    m.gp_cache_clear()
    fresh = _build(m, 2, "0.0", "1.0", 64, "12.0")
    assert m.gp_cache_info() == dict(hits=0, misses=1, entries=1)
    again = _build(m, 2, "0.0", "1.0", 64, "12.0")
    assert m.gp_cache_info() == dict(hits=1, misses=1, entries=1)
    assert _same(fresh, again)
    pv, qw, st = oracle.gp_build(2, "0.0", "1.0", 64, "0.0", "1.0", 64, "12.0")
    assert _same(again, (pv, qw, st))


def test_equal_spacing_shares_an_entry():
    """[0,1] and [-0.5,0.5] at equal N give the same quad dx, dy and ell."""
    m = pkg.load()
    m.gp_cache_clear()
    a = _build(m, 3, "0.0", "1.0", 128, "6.0")
    b = _build(m, 3, "-0.5", "0.5", 128, "6.0")
    assert m.gp_cache_info()["hits"] == 1 and _same(a, b)
    m.gp_cache_clear()
    assert _same(_build(m, 3, "-0.5", "0.5", 128, "6.0"), a)  # and equals its own fresh build


def test_other_inputs_miss():
    m = pkg.load()
    m.gp_cache_clear()
    base = _build(m, 2, "0.0", "1.0", 64, "12.0")
    for args in [(1, "0.0", "1.0", 64, "12.0"), (2, "0.0", "1.0", 65, "12.0"), (2, "0.0", "1.0", 64, "6.0"),
                 (2, "0.0", "2.0", 64, "12.0")]:
        out = _build(m, *args)
        if args[0] == 2 and args[4] != "12.0":  # another ell/Delta: other vectors
            assert not np.array_equal(out[0], base[0])
    info = m.gp_cache_info()
    assert info["hits"] == 0 and info["misses"] == 5 and info["entries"] == 5
    # rectangular cells: dx != dy is part of the key
    sq = _build(m, 2, "0.0", "1.0", 64, "12.0", ny=32)
    assert not np.array_equal(sq[0], base[0])


def test_concurrent_callers_get_identical_tables():
    m = pkg.load()
    m.gp_cache_clear()
    keys = [(2, "0.0", "1.0", n, "12.0") for n in (48, 64, 96)] + [(1, "0.0", "1.0", 33, "6.0")]
    m.gp_cache_clear()
    expect = {k: _build(m, *k) for k in keys}
    m.gp_cache_clear()
    bad = []

    def worker(seed):
        rng = np.random.default_rng(seed)
        for _ in range(25):
            k = keys[int(rng.integers(len(keys)))]
            if not _same(_build(m, *k), expect[k]):
                bad.append(k)

    threads = [threading.Thread(target=worker, args=(s,)) for s in range(8)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not bad
    info = m.gp_cache_info()
    assert info["entries"] == len(keys) and info["hits"] + info["misses"] == 8 * 25
