"""The stage modules one at a time through the C ABI (hosono_gpu_reconstruct,
_getfluxes, _flicd, _update, _detect, _bc, _bc_mood, _riemann) against the
oracle's restatement of the same reference routines, bit for bit (strict
arithmetic), and the reference's own known-answer values for
reconstruct_faceValsWithGP (test/test_reconstruct_faceValsWithGP.f90:31-34:
scheme = 3 on every cell, then one call)."""
import json
import os

import numpy as np
import pytest

import oracle
import parfiles
import pkg

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FACES = dict(north=0, south=1, east=2, west=3)


def _fresh(tmp_par_dir, name, kv):
    m = pkg.load()
    par = parfiles.make(tmp_par_dir, name, kv)
    return m, oracle.Oracle(par), m.Solver.from_par(par, fp_mode=m.FP_STRICT)


def _same_module_state(s, o, what=("faceVals", "fluxRaw", "flux", "scheme", "recompute", "recompute_flicd"),
                       unew_interior=False):
    a, b = s.module_get(), o.mod_get()
    for k in what:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    if unew_interior:
        g = o.ngc
        np.testing.assert_array_equal(a["Unew"][g:-g, g:-g], b["Unew"][g:-g, g:-g], err_msg="Unew")


@pytest.mark.gpu
def test_reconstruct_known_answers_through_the_gpu(tmp_par_dir):
    """The reference's reconstruct test on the GPU: Orszag-Tang 128^2 with the
    reference's own state, GP radius 3, ell/Delta = 6, every cell at scheme 3:
    the 153 printed face values and cell averages, to the printed 6 digits;
    and every face value of the array equal to the oracle's bit for bit."""
    m = pkg.load()
    d = json.load(open(os.path.join(GOLD, "gp_facevals_r3_kat.json")))
    par = parfiles.write_par(os.path.join(str(tmp_par_dir), "kat_gpu.par"), d["par"])
    s = m.Solver.from_par(par, fp_mode=m.FP_STRICT)
    ones = np.ones((s.nyt, s.nxt), dtype=np.int32)
    s.module_set(scheme=d["radius"] * ones, recompute=ones)
    s.reconstruct()
    st = s.module_get()
    fv = st["faceVals"]
    U, _, _ = s.download()
    g = s.params.ngc
    ic, jc = g + d["center_interior_offset"][0], g + d["center_interior_offset"][1]
    v = d["var"] - 1
    assert len(d["entries"]) == 153
    for e in d["entries"]:
        i, j = ic + e["di"], jc + e["dj"]
        got = U[j, i, v] if e["face"] == "avg" else fv[j, i, FACES[e["face"]], e["q"] - 1, v]
        ref = e["value"]
        tol = 0.5e-5 * 10 ** np.floor(np.log10(abs(ref))) * (1 + 1e-9)
        assert abs(got - ref) <= tol, (e, got)
    o = oracle.Oracle(par)
    np.testing.assert_array_equal(fv, o.reconstruct_all(d["radius"]))
    assert (st["scheme"] == d["radius"]).all()  # smooth state: no face state fails CAD/PAD
    s.close()


CASES = {
    "ot48_r2": lambda: parfiles.orszag_tang(48, 2),
    "blast40_r2": lambda: parfiles.blast(40, 2, p_ratio=1000.0, theta=0.3),
    "sedov36_r3": lambda: parfiles.sedov(36, 3),
    "blast36_r1": lambda: parfiles.blast(36, 1, p_ratio=300.0, theta=1.0),
}


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(CASES))
def test_forward_euler_stage_module_by_module(case, tmp_par_dir):
    """One forward-Euler stage driven from the host through the module entry
    points, as timeStep_forwardEuler does (timeStep.f90:76-128): scheme = R,
    flags set, then {reconstruct, getFluxes, FLICD, update, detect,
    applyMOOD} until detect lowers nothing.  After every module the module
    state equals the oracle's; the stage needs several MOOD passes on the
    blast and Sedov cases.  Then one more stage from the new state."""
    m, o, s = _fresh(tmp_par_dir, case, CASES[case]())
    R = s.params.max_radius
    ones = np.ones((s.nyt, s.nxt), dtype=np.int32)
    dt = o.cfl()
    passes = 0
    for stage in range(2):
        if stage == 1:  # the next stage starts from Unew with its guard cells filled
            s.bc(2)
            o.mod_bc(2)
            un = s.module_get()["Unew"]
            np.testing.assert_array_equal(un, o.mod_get()["Unew"])
            U, V, _ = s.download()
            s.upload(un, V)
            o.set_U(un)
        s.module_set(scheme=R * ones, recompute=ones, recompute_flicd=ones)
        o.mod_set(scheme=R * ones, recompute=ones, recompute_flicd=ones)
        for p in range(64):
            s.reconstruct()
            o.mod_reconstruct()
            _same_module_state(s, o, ("faceVals", "scheme", "recompute", "recompute_flicd"))
            s.getfluxes()
            o.mod_getfluxes()
            _same_module_state(s, o, ("fluxRaw", "flux"))
            s.flicd()
            o.mod_flicd()
            _same_module_state(s, o, ("flux",))
            s.update(dt)
            o.mod_update(dt)
            _same_module_state(s, o, (), unew_interior=True)
            ex_g = s.detect()
            ex_o = o.mod_detect()
            assert ex_g == ex_o, (stage, p)
            _same_module_state(s, o, ("scheme", "recompute", "recompute_flicd"))
            s.bc_mood()
            o.mod_bc_mood()
            _same_module_state(s, o, ("scheme", "recompute", "recompute_flicd"))
            passes += 1
            if ex_g:
                break
        else:
            pytest.fail("MOOD loop did not end in 64 passes")
    if case.startswith(("blast", "sedov")):
        assert passes > 2
    s.close()
    o.close()


@pytest.mark.gpu
def test_boundary_modules_match_oracle(tmp_par_dir):
    """boundaryConditions_applyBlk on U, V and Unew, periodic and outflow."""
    for name, kv in (("bc_ot", parfiles.orszag_tang(36, 2)), ("bc_sedov", parfiles.sedov(36, 2))):
        m, o, s = _fresh(tmp_par_dir, name, kv)
        rng = np.random.default_rng(5)
        U = rng.normal(size=(s.nyt, s.nxt, 8))
        V = rng.normal(size=(s.nyt, s.nxt, 10))
        s.upload(U, V)
        o.set_U(U)
        o.set_V(V)
        s.bc(0)
        s.bc(1)
        o.mod_bc(0)
        o.mod_bc(1)
        Ug, Vg, _ = s.download()
        np.testing.assert_array_equal(Ug, o.U())
        np.testing.assert_array_equal(Vg, o.V())
        s.close()
        o.close()


@pytest.mark.gpu
def test_riemann_solver_matches_oracle(tmp_par_dir):
    """riemannSolver_fromConsHllcMHD on random face states covering the four
    branches (supersonic left/right, both star states), x and y."""
    import torch

    for name, kv in (("rs_mhd", parfiles.orszag_tang(8, 1)), ("rs_hydro", parfiles.sedov(8, 1))):
        m, o, s = _fresh(tmp_par_dir, name, kv)
        rng = np.random.default_rng(11)
        n = 4096

        def states():
            u = np.zeros((n, 8))
            u[:, 0] = rng.uniform(0.05, 3.0, n)
            u[:, 1:4] = rng.normal(size=(n, 3)) * u[:, :1] * rng.choice([0.2, 1.0, 6.0], size=(n, 1))
            u[:, 5:8] = rng.normal(size=(n, 3))
            u[:, 4] = (0.5 * (u[:, 1:4] ** 2).sum(1) / u[:, 0] + 0.5 * (u[:, 5:8] ** 2).sum(1) +
                       rng.uniform(0.01, 3.0, n))
            return u
        uL, uR = states(), states()
        dL, dR = (torch.from_numpy(a).cuda() for a in (uL, uR))
        for direction in (0, 1):
            F = torch.zeros((n, 8), dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            s.riemann(n, dL.data_ptr(), dR.data_ptr(), direction, F.data_ptr())
            got = F.cpu().numpy()
            ref = np.array([o.hllc(uL[k], uR[k], direction) for k in range(n)])
            np.testing.assert_array_equal(got, ref)
        s.close()
        o.close()


@pytest.mark.gpu
def test_mood_pass_stats(tmp_par_dir):
    m, o, s = _fresh(tmp_par_dir, "stats", parfiles.blast(40, 2, p_ratio=1000.0, theta=0.3))
    o.trace(True)
    dt = o.cfl()
    o.advance(dt)
    s.timeStep_advanceSolution(dt)
    tr = o.traces(masks=False)
    npasses, ntroubled = s.mood_pass_stats()
    assert npasses == len(tr)
    assert ntroubled == sum(t["n_inner"] + t["n_detect"] for t in tr)
    s.close()
    o.close()


@pytest.mark.gpu
def test_eigenvectors_match_oracle(tmp_par_dir):
    """eigen_vecsFromPrim through hosono_gpu_eigenvecs on random primitive
    states (some with no tangential field), x and y, primitive and
    conserved forms: the oracle's bits."""
    import torch
    from test_oracle_invariants import _random_prims

    m, o, s = _fresh(tmp_par_dir, "eig", parfiles.orszag_tang(8, 1))
    rng = np.random.default_rng(7)
    n = 2048
    V = _random_prims(rng, n)
    dV = torch.from_numpy(V).cuda()
    for direction in (0, 1):
        for cons in (False, True):
            L = torch.zeros((n, 8, 8), dtype=torch.float64, device="cuda")
            R = torch.zeros_like(L)
            torch.cuda.synchronize()
            s.eigenvecs(n, dV.data_ptr(), direction, cons, L.data_ptr(), R.data_ptr())
            Lg, Rg = L.cpu().numpy(), R.cpu().numpy()
            for k in range(0, n, 7):
                Lo, Ro = o.eigenvecs(V[k], direction, cons=cons)
                np.testing.assert_array_equal(Lg[k].T, Lo)
                np.testing.assert_array_equal(Rg[k].T, Ro)
    s.close()
    o.close()
