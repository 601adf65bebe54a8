"""Device-side output diagnostics (output_writeHdf5's derived fields,
src/output.f90:230-274) against the same expressions evaluated in numpy on
the state V (host copy): every field bit for bit, and the div(B) norms; at
t_end of Orszag-Tang 128^2 R=1 the GPU's divB equals the one of the oracle's
final state (the accuracy gate only asks for within 2x)."""
import numpy as np
import pytest

import oracle
import parfiles
import pkg


def numpy_fields(V, p):
    g, nx, ny = p.ngc, p.nx, p.ny
    I = V[g:g + ny, g:g + nx]
    dens, velx, vely, velz, pres = I[..., 0], I[..., 1], I[..., 2], I[..., 3], I[..., 4]
    magx, magy, magz, eint, gama = I[..., 5], I[..., 6], I[..., 7], I[..., 8], I[..., 9]
    ener = dens * (velx * velx + vely * vely + velz * velz) / 2 + dens * eint
    magp = (magx * magx + magy * magy + magz * magz) / 2
    ener = ener + magp
    divb = 0.0 + 1 / (2 * p.dx) * (V[g:g + ny, g + 1:g + nx + 1, 5] - V[g:g + ny, g - 1:g + nx - 1, 5])
    divb = divb + 1 / (2 * p.dy) * (V[g + 1:g + ny + 1, g:g + nx, 6] - V[g - 1:g + ny - 1, g:g + nx, 6])
    return dict(dens=dens, velx=velx, vely=vely, velz=velz, pres=pres, eint=eint, gama=gama, ener=ener,
                magp=magp, divb=divb, magx=magx, magy=magy, magz=magz)


@pytest.mark.gpu
def test_diagnostic_fields_bitwise(tmp_par_dir):
    m = pkg.load()
    par = parfiles.make(tmp_par_dir, "diag", parfiles.orszag_tang(40, 2))
    s = m.Solver.from_par(par, fp_mode=m.FP_STRICT)
    s.set_time(0.0, 0.5)
    s.step(4)
    U, V, S = s.download()
    f, sch, ordr, l1, linf = s.diagnostics()
    ref = numpy_fields(V, s.params)
    for k, a in ref.items():
        np.testing.assert_array_equal(f[k], a, err_msg=k)
    g = s.params.ngc
    np.testing.assert_array_equal(sch, S[g:-g, g:-g])
    np.testing.assert_array_equal(ordr, 2 * S[g:-g, g:-g] + 1)
    assert linf == np.abs(ref["divb"]).max()
    assert abs(l1 - np.abs(ref["divb"]).mean()) <= 1e-12 * max(l1, 1e-300)
    assert s.diagnostics()[3:] == (l1, linf)  # same bits on every call
    s.close()


@pytest.mark.gpu
def test_divb_at_t_end_matches_oracle(tmp_par_dir):
    m = pkg.load()
    par = parfiles.make(tmp_par_dir, "ot128", parfiles.orszag_tang(128, 1))
    s = m.Solver.from_par(par, fp_mode=m.FP_STRICT)
    s.set_time(0.0, 0.5)
    t, n = s.step(0)
    f, _, _, l1, linf = s.diagnostics()
    o = oracle.Oracle(par)
    rc, to, no = o.run()
    assert (t, n) == (to, no)
    ref = numpy_fields(o.V(), s.params)["divb"]
    np.testing.assert_array_equal(f["divb"], ref)
    assert linf == np.abs(ref).max()
    s.close()


@pytest.mark.gpu
def test_batch_diagnostics_equal_plain(tmp_par_dir):
    m = pkg.load()
    pars = [parfiles.make(tmp_par_dir, "b0", parfiles.orszag_tang(36, 2)),
            parfiles.make(tmp_par_dir, "b1", parfiles.blast(40, 1, p_ratio=100.0, theta=0.3))]
    tiles = sum(m.Batch.tiles_for(m.par_load(p)[0]) for p in pars)
    b = m.Batch(2, tiles, fp_mode=m.FP_STRICT)
    slots = [b.add_par(p) for p in pars]
    for k in slots:
        b.set_time(k, 0.0, 1e30)
    b.run(max_steps=3)
    for k, par in zip(slots, pars):
        s = m.Solver.from_par(par, fp_mode=m.FP_STRICT)
        s.set_time(0.0, 1e30)
        s.step(3)
        fb, sb, ob, l1b, lib_ = b.diagnostics(k)
        fs, ss, os_, l1s, lis = s.diagnostics()
        for name in fs:
            np.testing.assert_array_equal(fb[name], fs[name], err_msg=name)
        np.testing.assert_array_equal(sb, ss)
        assert (l1b, lib_) == (l1s, lis)
        s.close()
    b.close()
