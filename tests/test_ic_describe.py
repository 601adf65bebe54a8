"""hosono_ic_describe's constants and tables rebuild hosono_ic_set's initial
state bit for bit (numpy evaluates the device kernel's expressions, src/ic.cu,
one IEEE operation at a time).  Host only."""
import numpy as np
import pytest

import parfiles
import pkg


def rebuild(m, p, d, xt, yt):
    g, nx, ny = p.ngc, p.nx, p.ny
    nxt, nyt = nx + 2 * g, ny + 2 * g
    per = p.bc == m.BC_PERIODIC

    def src(i, n):
        if i < g:
            return i + n if per else g
        if i >= g + n:
            return i - n if per else g + n - 1
        return i

    si = np.array([src(i, nx) for i in range(nxt)])
    sj = np.array([src(j, ny) for j in range(nyt)])
    X = np.broadcast_to(xt[si][None, :], (nyt, nxt))
    Y = np.broadcast_to(yt[sj][:, None], (nyt, nxt))
    c = np.array(d.c)
    v = np.zeros((10, nyt, nxt))
    if d.type == 1:
        ddx, ddy = X - c[0], Y - c[1]
        inside = np.sqrt(ddx * ddx + ddy * ddy) <= c[2]
        for k, (a, b) in enumerate([(3, 4), (5, 8), (6, 9), (7, 10), (11, 12)]):
            v[k] = np.where(inside, c[a], c[b])
        v[5], v[6], v[7] = c[13], c[14], c[15]
    elif d.type == 2:
        ddx, ddy = X - c[0], Y - c[1]
        v[0] = 1.0
        v[4] = np.where(np.sqrt(ddx * ddx + ddy * ddy) <= c[2], c[3], 1e-5)
    else:
        S2y = np.broadcast_to(yt[nyt + sj][:, None], (nyt, nxt))
        S2x = np.broadcast_to(xt[nxt + si][None, :], (nyt, nxt))
        S4x = np.broadcast_to(xt[2 * nxt + si][None, :], (nyt, nxt))
        v[0] = c[1]
        v[1] = -c[0] * S2y
        v[2] = c[0] * S2x
        v[5] = -c[2] * S2y
        v[6] = c[2] * S4x
        v[4] = c[3]
    gam = p.gamma
    v[8] = v[4] / (gam - 1.0) / v[0]
    v[9] = gam
    Bp = 0.0 if p.force_hydro else 0.5 * (v[5] * v[5] + v[6] * v[6] + v[7] * v[7])
    u = np.zeros((8, nyt, nxt))
    u[0] = v[0]
    u[1], u[2], u[3] = v[0] * v[1], v[0] * v[2], v[0] * v[3]
    u[4] = v[4] / (gam - 1.0) + v[0] * (0.5 * (v[1] * v[1] + v[2] * v[2] + v[3] * v[3])) + Bp
    for k in (5, 6, 7):
        u[k] = 0.0 if p.force_hydro else v[k]
    return np.moveaxis(u, 0, -1), np.moveaxis(v, 0, -1)


@pytest.mark.parametrize("name,kv", [
    ("ot", parfiles.orszag_tang(40, 2)),
    ("ot_refic", parfiles.orszag_tang(24, 1, standard=False)),
    ("sedov", parfiles.sedov(36, 2)),
    ("blast", parfiles.blast(48, 2, p_ratio=300.0, theta=0.7)),
])
def test_describe_rebuilds_ic_set(name, kv, tmp_par_dir):
    m = pkg.load()
    par = parfiles.make(tmp_par_dir, name, kv)
    p, _ = m.par_load(par)
    U, V = m.ic_set(par, p)
    d, xt, yt = m.ic_describe(par, p)
    U2, V2 = rebuild(m, p, d, xt, yt)
    np.testing.assert_array_equal(U2, U)
    np.testing.assert_array_equal(V2, V)
