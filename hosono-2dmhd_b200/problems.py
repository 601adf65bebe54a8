"""Parameter files (the reference's .par format, src/readParamFile.f90:1-9) for
the three initial conditions the workloads use: Orszag-Tang vortex, Sedov
blast (sedov2d) and MHD blast (explosion2d with a uniform field).

Keys beyond the reference (IC_B0, IC_pres, IC_magx/y/z) have defaults that
reproduce the reference's own initial conditions (src/initialCondition.f90).
"""
import math
import os

COMMON = dict(
    sim_smallPressure="1.0e-12", sim_smallEnergy="1.0e-12", sim_smallDensity="1.0e-12", sim_smallB="1.0e-12",
    sim_riemannSolver="'hllc'", sim_nstepmax="1000000", sim_outputFreqTime="0.02", sim_outputFreqStep="0",
    sim_outputHdf5=".false.", sim_outputAscii=".false.", sim_dataFileBaseName="'data/run'")
GAMMA_MHD = "1.66666666666666666"


def orszag_tang(n, radius, ell=6.0, tmax=0.5, cfl=0.8):
    """[0,1]^2, periodic, rho=25/(36 pi), p=5/(12 pi), v=(-sin 2pi y, sin 2pi x),
    B=B0(-sin 2pi y, sin 4pi x), B0=1/sqrt(4 pi)."""
    kv = dict(COMMON)
    kv.update(sim_gamma=GAMMA_MHD, sim_cfl=repr(cfl), sim_tmax=repr(tmax), sim_forceHydro=".false.",
              grid_Nx=str(n), grid_Ny=str(n), grid_xBeg="0.0", grid_xEnd="1.0", grid_yBeg="0.0", grid_yEnd="1.0",
              GP_maxRadius=str(radius), GP_ellOverDelta=repr(ell), IC_type="'OrszagTang2d'", IC_U0="1.0",
              IC_dens=repr(25 / (36 * math.pi)), IC_pres=repr(5 / (12 * math.pi)),
              IC_B0=repr(1 / math.sqrt(4 * math.pi)), sim_BC="'periodic'")
    return kv


def sedov(n, radius, ell=6.0, tmax=0.05, cfl=0.6):
    """[-0.5,0.5]^2, outflow, gamma=1.4, hydro; E=1 in r <= 3.5 dx."""
    kv = dict(COMMON)
    kv.update(sim_gamma="1.4", sim_cfl=repr(cfl), sim_tmax=repr(tmax), sim_forceHydro=".true.",
              grid_Nx=str(n), grid_Ny=str(n), grid_xBeg="-0.5", grid_xEnd="0.5", grid_yBeg="-0.5", grid_yEnd="0.5",
              GP_maxRadius=str(radius), GP_ellOverDelta=repr(ell), IC_type="'sedov2d'",
              IC_shockCenter_x="0.0", IC_shockCenter_y="0.0", sim_BC="'outflow'")
    return kv


def blast(n, radius, p_ratio, theta, ell=6.0, tmax=0.02, cfl=0.8):
    """[-0.5,0.5]^2, periodic, gamma=5/3, rho=1, p_in = 0.1 p_ratio in r <= 0.1,
    p_out = 0.1, B = (10/sqrt(4 pi)) (cos theta, sin theta, 0)."""
    b = 10 / math.sqrt(4 * math.pi)
    kv = dict(COMMON)
    kv.update(sim_gamma=GAMMA_MHD, sim_cfl=repr(cfl), sim_tmax=repr(tmax), sim_forceHydro=".false.",
              grid_Nx=str(n), grid_Ny=str(n), grid_xBeg="-0.5", grid_xEnd="0.5", grid_yBeg="-0.5", grid_yEnd="0.5",
              GP_maxRadius=str(radius), GP_ellOverDelta=repr(ell), IC_type="'explosion2d'",
              IC_shockCenter_x="0.0", IC_shockCenter_y="0.0", IC_shockRad="0.1",
              IC_densIns="1.0", IC_densOut="1.0", IC_velxIns="0.0", IC_velyIns="0.0", IC_velzIns="0.0",
              IC_velxOut="0.0", IC_velyOut="0.0", IC_velzOut="0.0",
              IC_presIns=repr(0.1 * p_ratio), IC_presOut="0.1",
              IC_magx=repr(b * math.cos(theta)), IC_magy=repr(b * math.sin(theta)), IC_magz="0.0",
              sim_BC="'periodic'")
    return kv


def from_entry(e):
    """.par key/values of one workload manifest entry."""
    prob, n, R = e["problem"], int(e["n"]), int(e["radius"])
    ell = float(e.get("ell", 6.0))
    if prob == "OrszagTang2d":
        return orszag_tang(n, R, ell=ell, tmax=float(e["tmax"]))
    if prob == "sedov2d":
        return sedov(n, R, ell=ell, tmax=float(e["tmax"]))
    if prob == "explosion2d":
        return blast(n, R, float(e["p_ratio"]), float(e["theta"]), ell=ell, tmax=float(e["tmax"]),
                     cfl=float(e.get("cfl", 0.8)))
    raise ValueError(f"unknown problem {prob}")


def write_par(path, kv):
    with open(path, "w") as f:
        for k, v in kv.items():
            f.write(f"{k} = {v}\n")
    return path


def make(directory, name, kv):
    return write_par(os.path.join(str(directory), name + ".par"), kv)
