"""Extract the reference's known-answer values into committed fixtures.

Run where the reference project is checked out; its path is the required
first argument:

    python tests/golden/make_golden.py PATH_TO_REFERENCE

Writes:

* gp_facevals_r3_kat.json -- the momentum-x face values and cell averages
  printed by test/test_reconstruct_faceValsWithGP.f90 (output captured in
  test/test_reconstruct_faceValsWithGP/output.txt:59-100): Orszag-Tang IC,
  128x128, GP radius 3, ell/Delta = 6, every face reconstructed at radius 3,
  on the 3x3 cells around interior cell (5,5) (0-based from the first interior
  cell).  Values are ES12.5, i.e. 6 significant digits.
* gp_init_kat.json -- the structural facts test/test_GP_init.f90:28-48
  asserts for test/par/test_GP_init.par (8x8, R=2, ell/Delta=2), plus the
  1-norm check of test/test_GP_prediction_vectors.f90:20-25.

The parameter files the tests use are written from the key/value pairs of
the reference's test .par files (test/par/*.par).
"""
import json
import os
import re
import sys

if len(sys.argv) < 2:
    sys.exit("usage: make_golden.py PATH_TO_REFERENCE (the hosono-2DMHD project root)")
REF = sys.argv[1]
HERE = os.path.dirname(os.path.abspath(__file__))
FLOAT = re.compile(r"[-+]?\d\.\d+E[-+]\d+")


def read_par(path):
    kv = {}
    with open(path) as f:
        for line in f:
            if line.startswith("#"):
                continue
            line = line.split("#", 1)[0]
            if "=" not in line:
                continue
            k, v = line.split("=", 1)
            kv[k.strip()] = v.strip()
    return kv


def facevals_kat():
    txt = open(os.path.join(REF, "test/test_reconstruct_faceValsWithGP/output.txt")).read().splitlines()
    start = next(k for k, l in enumerate(txt) if l.startswith("U(2,:,:) and its face values"))
    header = txt[start]
    nq = int(re.search(r"with (\d+) quadrature points", header).group(1))
    grid = [l for l in txt[start + 4:] if l.startswith("|") or l.startswith("-")]
    seps = [k for k, l in enumerate(grid) if l.startswith("-")]
    assert len(seps) == 4, "expected a 3x3 block of cells"
    entries = []
    for r in range(3):
        dj = 1 - r  # the top block row is j = jc + 1
        block = grid[seps[r] + 1:seps[r + 1]]
        rows = [[FLOAT.findall(seg) for seg in line.split("|")[1:4]] for line in block]
        for c in range(3):
            di = c - 1
            north = rows[0][c]
            south = rows[-1][c]
            assert len(north) == nq and len(south) == nq
            for p in range(nq):  # printed left to right as k = nq..1
                k = nq - p
                entries.append(dict(di=di, dj=dj, face="north", q=k, value=float(north[p])))
                entries.append(dict(di=di, dj=dj, face="south", q=k, value=float(south[p])))
            side_rows = [row[c] for row in rows[2:2 + nq]]  # k = 1..nq from top to bottom
            for k, vals in enumerate(side_rows, start=1):
                if len(vals) == 3:  # west, cell average, east
                    entries.append(dict(di=di, dj=dj, face="avg", q=0, value=float(vals[1])))
                    vals = [vals[0], vals[2]]
                assert len(vals) == 2
                entries.append(dict(di=di, dj=dj, face="west", q=k, value=float(vals[0])))
                entries.append(dict(di=di, dj=dj, face="east", q=k, value=float(vals[1])))
    par = read_par(os.path.join(REF, "test/par/test_reconstruct_faceValsWithGP.par"))
    return dict(
        source="test/test_reconstruct_faceValsWithGP/output.txt:59-100",
        var=2, radius=3, nq=nq, center_interior_offset=[5, 5], significant_digits=6,
        par=par, entries=entries)


def gp_init_kat():
    par = read_par(os.path.join(REF, "test/par/test_GP_init.par"))
    R = int(par["GP_maxRadius"])
    return dict(
        source="test/test_GP_init.f90:28-48; test/test_GP_prediction_vectors.f90:20-25",
        par=par, radius=R, nq=R + 1, ns=1 + 2 * R * (R + 1), npred=4 * (R + 1),
        weight_sum=1.0, weight_sum_tol=1e-5, one_norm=1.0, one_norm_tol=1e-2)


def main():
    for name, obj in (("gp_facevals_r3_kat.json", facevals_kat()), ("gp_init_kat.json", gp_init_kat())):
        with open(os.path.join(HERE, name), "w") as f:
            json.dump(obj, f, indent=1)
        print("wrote", name)


if __name__ == "__main__":
    main()
