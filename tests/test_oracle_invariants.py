"""Analytic invariants of the oracle's time step (CPU only).  HLLC, FLICD,
detect and RK3 have no golden values in the reference's tests, so besides
the known-answer tests the oracle is held to properties the scheme has by
construction: a uniform state stays uniform, a state that varies along x
only keeps identical rows through MOOD lowerings, the MHD HLLC solver
reduces to the Euler HLLC solver when B = 0, and the flux-interpolated CT
correction (FLICDdivB_fluxCorrections, src/FLICDdivB.f90:13-70) keeps the
central-difference div(B) of src/output.f90:261-274 at round-off."""
import math

import numpy as np
import pytest

import oracle
import parfiles


@pytest.mark.parametrize("R", [1, 2, 3])
def test_uniform_state_is_preserved(R, tmp_par_dir):
    """Every face of a uniform periodic state sees the same two states, so
    every flux difference vanishes: three RK3 steps leave U unchanged (up to
    the rounding of the RK combinations) and no cell is lowered."""
    o = oracle.Oracle(parfiles.make(tmp_par_dir, f"uniform{R}", parfiles.orszag_tang(24, R)))
    g = o.ngc
    u = np.array([1.3, 0.4, -0.7, 0.2, 0.0, 0.3, -0.5, 0.25])
    u[1:4] *= u[0]
    u[4] = 0.5 * (u[1:4] ** 2).sum() / u[0] + 0.5 * (u[5:8] ** 2).sum() + 2.0
    U = np.broadcast_to(u, (o.nyTot, o.nxTot, 8)).copy()
    o.set_U(U)
    o.set_V(np.broadcast_to(o.cons2prim(u), (o.nyTot, o.nxTot, 10)).copy())
    for _ in range(3):
        o.advance(o.cfl())
    np.testing.assert_allclose(o.U(), U, rtol=1e-14, atol=0)
    assert (o.scheme()[g:-g, g:-g] == R).all()


def hllc_euler(uL, uR, d, gam):
    """The HLLC solver for the Euler equations in Toro's form (Riemann Solvers
    and Numerical Methods for Fluid Dynamics, 3rd ed., section 10.4), with the
    wave-speed estimates and the branch order of riemannSolver.f90:84-96 and
    :189-219 (sL = min(uL - cL, uA - cA), sR = max(uA + cA, uR + cR) from the
    arithmetic mean A of the primitive states; the left star state is taken
    whenever sL <= 0 < s*).  Returns (flux, branch)."""
    def prim(u):
        rho = u[0]
        vel = u[1:4] / rho
        return rho, vel, (gam - 1) * (u[4] - 0.5 * rho * (vel ** 2).sum())

    def flux(u, vel, p):
        f = np.zeros(8)
        f[0] = u[1 + d]
        f[1:4] = u[1:4] * vel[d]
        f[1 + d] += p
        f[4] = (u[4] + p) * vel[d]
        return f

    rL, vL, pL = prim(uL)
    rR, vR, pR = prim(uR)
    cL, cR = math.sqrt(gam * pL / rL), math.sqrt(gam * pR / rR)
    rA, vA, pA = (rL + rR) / 2, (vL[d] + vR[d]) / 2, (pL + pR) / 2
    cA = math.sqrt(gam * pA / rA)
    sL, sR = min(vL[d] - cL, vA - cA), max(vA + cA, vR[d] + cR)
    sS = (pR - pL + rL * vL[d] * (sL - vL[d]) - rR * vR[d] * (sR - vR[d])) / (rL * (sL - vL[d]) - rR * (sR - vR[d]))
    if 0 < sL:
        return flux(uL, vL, pL), 0
    if sS > 0:
        u, r, v, p, s, branch = uL, rL, vL, pL, sL, 1
    elif 0 <= sR:
        u, r, v, p, s, branch = uR, rR, vR, pR, sR, 2
    else:
        return flux(uR, vR, pR), 3
    k = r * (s - v[d]) / (s - sS)
    ustar = np.zeros(8)
    ustar[0] = k
    ustar[1:4] = k * v
    ustar[1 + d] = k * sS
    ustar[4] = k * (u[4] / r + (sS - v[d]) * (sS + p / (r * (s - v[d]))))
    return flux(u, v, p) + s * (ustar - u), branch


def test_hllc_at_zero_field_is_the_euler_hllc(tmp_par_dir):
    """With B = 0 the MHD HLLC solver (Li 2005) is the Euler HLLC solver: the
    oracle's flux equals an independent Euler HLLC in Toro's star-state form
    to round-off, over random subsonic and supersonic states that reach all
    four branches."""
    o = oracle.Oracle(parfiles.make(tmp_par_dir, "hllc_euler", parfiles.orszag_tang(8, 1)))
    rng = np.random.default_rng(5)

    def state():
        u = np.zeros(8)
        u[0] = rng.uniform(0.3, 3.0)
        u[1:4] = rng.normal(size=3) * rng.choice([0.3, 1.0, 4.0]) * u[0]
        u[4] = 0.5 * (u[1:4] ** 2).sum() / u[0] + rng.uniform(0.1, 3.0) / (o.gamma - 1)
        return u

    hits = [0, 0, 0, 0]
    for _ in range(1000):
        uL, uR = state(), state()
        for d in (0, 1):
            f, branch = hllc_euler(uL, uR, d, o.gamma)
            hits[branch] += 1
            np.testing.assert_allclose(o.hllc(uL, uR, d), f, rtol=0, atol=1e-12 * np.abs(f).max())
    assert min(hits) >= 50, hits


def central_div_b(o, U):
    """(Bx(i+1,j) - Bx(i-1,j)) / 2dx + (By(i,j+1) - By(i,j-1)) / 2dy on the
    interior (output.f90:261-274)."""
    g = o.ngc
    bx, by = U[..., 5], U[..., 6]
    ny, nx = o.ny, o.nx
    return ((bx[g:g + ny, g + 1:g + nx + 1] - bx[g:g + ny, g - 1:g + nx - 1]) / (2 * o.dx) +
            (by[g + 1:g + ny + 1, g:g + nx] - by[g - 1:g + ny - 1, g:g + nx]) / (2 * o.dy))


@pytest.mark.parametrize("case", ["orszag_tang", "blast"])
def test_flicd_keeps_central_div_b(case, tmp_par_dir):
    """Orszag-Tang (Bx depends on y only, By on x only) and the magnetised
    blast (uniform B) start with a central-difference div(B) of exactly zero.
    FLICD's corrected induction fluxes keep it at round-off through RK3 steps,
    including the blast's MOOD passes, which lower cells to first order and
    update only the recomputeFLICD cells."""
    kv = parfiles.orszag_tang(32, 2) if case == "orszag_tang" else parfiles.blast(48, 2, p_ratio=300.0, theta=0.7)
    o = oracle.Oracle(parfiles.make(tmp_par_dir, f"divb_{case}", kv))
    U0 = o.U()
    scale = np.abs(U0[..., 5:7]).max() / min(o.dx, o.dy)
    assert np.abs(central_div_b(o, U0)).max() == 0.0
    for _ in range(4):
        o.advance(o.cfl())
    assert np.abs(central_div_b(o, o.U())).max() <= 1e-14 * scale
    if case == "blast":
        g = o.ngc
        assert o.scheme()[g:-g, g:-g].min() == 0  # MOOD lowered cells to first order


def _random_prims(rng, n):
    V = np.zeros((n, 10))
    V[:, 0] = rng.uniform(0.1, 3.0, n)
    V[:, 1:4] = rng.normal(size=(n, 3))
    V[:, 4] = rng.uniform(0.05, 3.0, n)
    V[:, 5:8] = rng.normal(size=(n, 3)) * rng.choice([0.0, 1e-3, 1.0, 5.0], size=(n, 1))
    V[::7, 6:8] = 0.0  # no tangential field: the beta_T guard (eigen.f90:364-368)
    V[:, 9] = 5.0 / 3.0
    return V


def test_eigenvectors_are_biorthonormal(tmp_par_dir):
    """eigen_vecsFromPrim (eigen.f90:20-255): the left eigenvectors (columns
    of L) and the right ones (columns of R) of the 7 waves satisfy
    L^T R = I, in primitive and in conserved variables (dV/dU dU/dV = I),
    also where the field or its tangential part vanishes."""
    o = oracle.Oracle(parfiles.make(tmp_par_dir, "eig", parfiles.orszag_tang(8, 1)))
    rng = np.random.default_rng(1)
    for V in _random_prims(rng, 400):
        for d in (0, 1):
            for cons in (False, True):
                L, R = o.eigenvecs(V, d, cons=cons)
                np.testing.assert_allclose(L[:, :7].T @ R[:, :7], np.eye(7), rtol=0, atol=1e-12)
                assert not L[:, 7].any() and not R[:, 7].any()


@pytest.mark.parametrize("R", [1, 2])
def test_planar_state_keeps_identical_rows(R, tmp_par_dir):
    """A periodic state that varies only along x (an MHD shock tube with a
    constant normal field, so div B = 0, and a smooth transverse wave) gives
    every row the same inputs in the same order: after three RK3 steps, with
    the MOOD loop lowering cells at the discontinuities, every row of U and
    of the scheme still equals the first row bit for bit."""
    o = oracle.Oracle(parfiles.make(tmp_par_dir, f"planar{R}", parfiles.orszag_tang(48, R)))
    nx = o.nxTot
    x = (np.arange(nx) + 0.5) / nx
    left = (x > 0.25) & (x < 0.6)
    rho = np.where(left, 1.0, 0.125)
    p = np.where(left, 1.0, 0.1)
    vx = 0.1 * np.sin(2 * np.pi * x)
    vy = 0.2 * np.cos(2 * np.pi * x)
    bx = np.full(nx, 0.75)
    by = np.where(left, 1.0, -1.0)
    bz = 0.1 * np.sin(4 * np.pi * x)
    gam = 5.0 / 3.0
    row = np.zeros((nx, 8))
    row[:, 0] = rho
    row[:, 1] = rho * vx
    row[:, 2] = rho * vy
    row[:, 5], row[:, 6], row[:, 7] = bx, by, bz
    row[:, 4] = p / (gam - 1) + 0.5 * rho * (vx ** 2 + vy ** 2) + 0.5 * (bx ** 2 + by ** 2 + bz ** 2)
    U = np.broadcast_to(row, (o.nyTot, nx, 8)).copy()
    o.set_U(U)
    o.set_V(np.stack([np.broadcast_to(o.cons2prim(row[i]), (o.nyTot, 10)) for i in range(nx)], axis=1).copy())
    lowered = False
    for _ in range(3):
        o.advance(o.cfl())
        S = o.scheme()
        lowered |= bool((S < R).any())
    Uo, S = o.U(), o.scheme()
    assert lowered  # the discontinuities made MOOD lower cells
    for j in range(1, o.nyTot):
        np.testing.assert_array_equal(Uo[j], Uo[0])
        np.testing.assert_array_equal(S[j], S[0])
    o.close()
