"""The oracle against the reference's own known-answer values (CPU only)."""
import json
import os

import numpy as np
import pytest

import oracle
import parfiles

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FACES = dict(north=0, south=1, east=2, west=3)


def test_gp_facevals_r3_match_reference_printout(tmp_par_dir):
    """test/test_reconstruct_faceValsWithGP.f90: 153 printed values (ES12.5)."""
    d = json.load(open(os.path.join(GOLD, "gp_facevals_r3_kat.json")))
    par = parfiles.write_par(os.path.join(str(tmp_par_dir), "kat.par"), d["par"])
    o = oracle.Oracle(par)
    fv = o.reconstruct_all(d["radius"])
    U = o.U()
    ic = o.ngc + d["center_interior_offset"][0]
    jc = o.ngc + d["center_interior_offset"][1]
    v = d["var"] - 1
    assert len(d["entries"]) == 153
    for e in d["entries"]:
        i, j = ic + e["di"], jc + e["dj"]
        got = U[j, i, v] if e["face"] == "avg" else fv[j, i, FACES[e["face"]], e["q"] - 1, v]
        ref = e["value"]
        # 6 significant digits: half a unit in the 6th digit
        tol = 0.5e-5 * 10 ** np.floor(np.log10(abs(ref))) * (1 + 1e-9)
        assert abs(got - ref) <= tol, (e, got)


def test_gp_init_structure():
    """test/test_GP_init.f90:28-48 and test/test_GP_prediction_vectors.f90:20-25."""
    d = json.load(open(os.path.join(GOLD, "gp_init_kat.json")))
    p = d["par"]
    R = d["radius"]
    pv, qw, st = oracle.gp_build(R, p["grid_xBeg"], p["grid_xEnd"], int(p["grid_Nx"]), p["grid_yBeg"],
                                 p["grid_yEnd"], int(p["grid_Ny"]), p["GP_ellOverDelta"])
    ns, nq = d["ns"], d["nq"]
    st = st.reshape(R, ns, 2)
    assert np.sum((st[R - 1, :, 0] == 0) & (st[R - 1, :, 1] == 0)) == 1
    assert not np.isnan(pv).any()
    qw = qw.reshape(R, nq)
    assert abs(qw[R - 1].sum() - d["weight_sum"]) <= d["weight_sum_tol"]
    pv = pv.reshape(R, 4, nq, ns)
    for rr in range(1, R + 1):
        nsr, nqr = 1 + 2 * rr * (rr + 1), rr + 1
        sums = pv[rr - 1, :, :nqr, :nsr].sum(axis=-1)
        assert np.all(np.abs(sums - d["one_norm"]) <= d["one_norm_tol"])


@pytest.mark.parametrize("R", [1, 2, 3])
def test_gp_stencil_order_and_symmetry(R):
    """Stencil order of GP.f90:85-95 and the mirror symmetry of the vectors."""
    pv, qw, st = oracle.gp_build(R, "0.0", "1.0", 64, "0.0", "1.0", 64, "6.0")
    ns, nq = 1 + 2 * R * (R + 1), R + 1
    st = st.reshape(R, ns, 2)[R - 1]
    expect = [(i, j) for i in range(-R, R + 1) for j in range(-R, R + 1) if abs(i) + abs(j) <= R]
    assert [tuple(x) for x in st] == expect
    pv = pv.reshape(R, 4, nq, ns)[R - 1]
    # north/south faces are mirror images in y: pv(k, q, N) = pv(mirror_y(k), q, S)
    idx = {tuple(x): k for k, x in enumerate(st)}
    mir = [idx[(x[0], -x[1])] for x in st]
    np.testing.assert_allclose(pv[0][:, mir], pv[1], rtol=0, atol=1e-14)
    assert np.allclose(pv.sum(axis=-1), 1.0, atol=1e-13)


def test_orszag_tang_conserves_periodic(tmp_par_dir):
    """Periodic boundaries: the interior sums of all conserved variables stay
    constant (the unsplit update telescopes)."""
    par = parfiles.make(tmp_par_dir, "ot32", parfiles.orszag_tang(32, 2))
    o = oracle.Oracle(par)
    g = o.ngc
    s0 = o.U()[g:-g, g:-g].sum(axis=(0, 1))
    rc, t, n = o.run(max_steps=5)
    assert rc == 0 and n == 5
    s1 = o.U()[g:-g, g:-g].sum(axis=(0, 1))
    scale = np.abs(o.U()[g:-g, g:-g]).sum(axis=(0, 1)) + 1e-300
    assert np.all(np.abs(s1 - s0) <= 1e-12 * scale)


def test_hllc_consistency(tmp_par_dir):
    """F_hllc(u, u) equals the physical flux f(u) (consistency)."""
    par = parfiles.make(tmp_par_dir, "ot8", parfiles.orszag_tang(8, 1))
    o = oracle.Oracle(par)
    rng = np.random.default_rng(3)
    for _ in range(50):
        u = np.zeros(8)
        u[0] = rng.uniform(0.1, 2)
        u[1:4] = rng.normal(size=3) * u[0]
        u[5:8] = rng.normal(size=3)
        u[4] = 0.5 * (u[1:4] ** 2).sum() / u[0] + 0.5 * (u[5:8] ** 2).sum() + rng.uniform(0.1, 2)
        for d in (0, 1):
            np.testing.assert_allclose(o.hllc(u, u, d), o.cons2flux(u, d), rtol=1e-12, atol=1e-12)
