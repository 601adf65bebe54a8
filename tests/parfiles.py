"""Parameter-file builders for the tests (the reference's .par format)."""
import math
import os

COMMON = dict(
    sim_smallPressure="1.0e-12", sim_smallEnergy="1.0e-12", sim_smallDensity="1.0e-12", sim_smallB="1.0e-12",
    sim_riemannSolver="'hllc'", sim_nstepmax="1000000", sim_outputFreqTime="0.02", sim_outputFreqStep="0",
    sim_outputHdf5=".false.", sim_outputAscii=".false.", sim_dataFileBaseName="'data/run'")


def write_par(path, kv):
    with open(path, "w") as f:
        for k, v in kv.items():
            f.write(f"{k} = {v}\n")
    return path


def orszag_tang(n, radius, ell=6.0, tmax=0.5, cfl=0.8, standard=True):
    """Orszag-Tang vortex on [0,1]^2, periodic.  standard=True uses the
    textbook state (rho=25/(36 pi), p=5/(12 pi), B0=1/sqrt(4 pi)); False keeps
    the reference's own (IC_dens=1, p=B0=1/gamma)."""
    kv = dict(COMMON)
    kv.update(sim_gamma="1.66666666666666666", sim_cfl=repr(cfl), sim_tmax=repr(tmax), sim_forceHydro=".false.",
              grid_Nx=str(n), grid_Ny=str(n), grid_xBeg="0.0", grid_xEnd="1.0", grid_yBeg="0.0", grid_yEnd="1.0",
              GP_maxRadius=str(radius), GP_ellOverDelta=repr(ell), IC_type="'OrszagTang2d'", IC_U0="1.0",
              sim_BC="'periodic'")
    if standard:
        kv.update(IC_dens=repr(25 / (36 * math.pi)), IC_pres=repr(5 / (12 * math.pi)),
                  IC_B0=repr(1 / math.sqrt(4 * math.pi)))
    else:
        kv.update(IC_dens="1.0")
    return kv


def sedov(n, radius, ell=6.0, tmax=0.05, cfl=0.6):
    kv = dict(COMMON)
    kv.update(sim_gamma="1.4", sim_cfl=repr(cfl), sim_tmax=repr(tmax), sim_forceHydro=".true.",
              grid_Nx=str(n), grid_Ny=str(n), grid_xBeg="-0.5", grid_xEnd="0.5", grid_yBeg="-0.5", grid_yEnd="0.5",
              GP_maxRadius=str(radius), GP_ellOverDelta=repr(ell), IC_type="'sedov2d'",
              IC_shockCenter_x="0.0", IC_shockCenter_y="0.0", sim_BC="'outflow'")
    return kv


def blast(n, radius, p_ratio=100.0, theta=0.5, ell=6.0, tmax=0.02, cfl=0.8):
    """MHD blast (explosion2d form) on [-0.5,0.5]^2, periodic, gamma=5/3."""
    b = 10 / math.sqrt(4 * math.pi)
    kv = dict(COMMON)
    kv.update(sim_gamma="1.66666666666666666", sim_cfl=repr(cfl), sim_tmax=repr(tmax), sim_forceHydro=".false.",
              grid_Nx=str(n), grid_Ny=str(n), grid_xBeg="-0.5", grid_xEnd="0.5", grid_yBeg="-0.5", grid_yEnd="0.5",
              GP_maxRadius=str(radius), GP_ellOverDelta=repr(ell), IC_type="'explosion2d'",
              IC_shockCenter_x="0.0", IC_shockCenter_y="0.0", IC_shockRad="0.1",
              IC_densIns="1.0", IC_densOut="1.0", IC_velxIns="0.0", IC_velyIns="0.0", IC_velzIns="0.0",
              IC_velxOut="0.0", IC_velyOut="0.0", IC_velzOut="0.0",
              IC_presIns=repr(0.1 * p_ratio), IC_presOut="0.1",
              IC_magx=repr(b * math.cos(theta)), IC_magy=repr(b * math.sin(theta)), IC_magz="0.0",
              sim_BC="'periodic'")
    return kv


def make(tmpdir, name, kv):
    return write_par(os.path.join(str(tmpdir), name + ".par"), kv)
