// setup.cpp -- host-side set-up above the C ABI: the .par reader
// (src/readParamFile.f90), simulation_init (src/simulation.f90:35-78),
// grid_init (src/grid.f90:31-103), GP_init from a .par file and the initial
// conditions of src/initialCondition.f90:23-226.
//
// The .par file is parsed once into its lines (the reference rescans the
// file for every key); lookups keep the reference's rule: the first
// non-comment line whose text before '=' (trailing blanks trimmed) equals the
// key, with anything after '#' dropped, and a list-directed read of the first
// item after '='.

#include "hosono_gpu.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <utility>
#include <vector>

namespace {

const double kPi = 3.14159265358979323846;  // ACOS(-1.0), src/definitions.f90:39

struct ParFile {
    std::string path;
    std::vector<std::pair<std::string, std::string>> entries;
    bool ok = false;

    explicit ParFile(const char* p) : path(p ? p : "") {
        std::ifstream in(path);
        if (!in) return;
        ok = true;
        std::string line;
        while (std::getline(in, line)) {
            if (!line.empty() && line[0] == '#') continue;
            const size_t hash = line.find('#');
            if (hash != std::string::npos) line.resize(hash);
            const size_t eq = line.find('=');
            if (eq == std::string::npos) continue;
            std::string name = line.substr(0, eq);
            while (!name.empty() && (name.back() == ' ' || name.back() == '\t' || name.back() == '\r')) name.pop_back();
            entries.emplace_back(name, line.substr(eq + 1));
        }
    }

    const std::string* raw(const std::string& key) const {
        for (const auto& e : entries)
            if (e.first == key) return &e.second;
        return nullptr;
    }
};

struct Missing {
    std::string key;
};

std::string item(const std::string& v) {
    const size_t a = v.find_first_not_of(" \t\r");
    if (a == std::string::npos) return "";
    if (v[a] == '\'' || v[a] == '"') {
        const size_t b = v.find(v[a], a + 1);
        return v.substr(a + 1, b == std::string::npos ? std::string::npos : b - a - 1);
    }
    const size_t b = v.find_first_of(" \t\r,/", a);
    return v.substr(a, b == std::string::npos ? std::string::npos : b - a);
}

std::string get_str(const ParFile& f, const char* key) {
    const std::string* r = f.raw(key);
    if (!r) throw Missing{key};
    return item(*r);
}
double to_real(std::string t) {
    for (char& c : t)
        if (c == 'd' || c == 'D') c = 'e';
    return std::strtod(t.c_str(), nullptr);
}
double get_real(const ParFile& f, const char* key) { return to_real(get_str(f, key)); }
double get_real_or(const ParFile& f, const char* key, double dflt) {
    const std::string* r = f.raw(key);
    return r ? to_real(item(*r)) : dflt;
}
int get_int(const ParFile& f, const char* key) { return std::atoi(get_str(f, key).c_str()); }
bool get_logical(const ParFile& f, const char* key) {
    const std::string t = get_str(f, key);
    const size_t k = (!t.empty() && t[0] == '.') ? 1 : 0;
    return k < t.size() && (t[k] == 't' || t[k] == 'T');
}

void put_err(char* err, int len, const std::string& m) {
    if (err && len > 0) std::snprintf(err, (size_t)len, "%s", m.c_str());
}

// boundaryConditions_apply (src/boundaryConditions.f90:79-187) on a Fortran-order host array
void host_bc(const hosono_params* p, double* A, int nv) {
    const int g = p->ngc, nxt = p->nx + 2 * g, nyt = p->ny + 2 * g;
    auto src = [&](int i, int n) {
        if (i < g) return p->bc == HOSONO_BC_PERIODIC ? i + n : g;
        if (i >= g + n) return p->bc == HOSONO_BC_PERIODIC ? i - n : g + n - 1;
        return i;
    };
    for (int j = 0; j < nyt; j++)  // x direction on every row
        for (int i = 0; i < nxt; i++) {
            const int si = src(i, p->nx);
            if (si != i) std::memcpy(&A[(size_t)nv * ((size_t)j * nxt + i)], &A[(size_t)nv * ((size_t)j * nxt + si)], sizeof(double) * nv);
        }
    for (int j = 0; j < nyt; j++) {  // then y direction on every column
        const int sj = src(j, p->ny);
        if (sj != j) std::memcpy(&A[(size_t)nv * (size_t)j * nxt], &A[(size_t)nv * (size_t)sj * nxt], sizeof(double) * nv * nxt);
    }
}

}  // namespace

// keys simulation_init, GP_init and grid_init read, in the reference's read
// order (checked up front, so one call names every missing key): the sim_*
// keys, then GP_init's grid_xBeg .. grid_Ny, GP_ellOverDelta, GP_maxRadius
// (GP.f90:58-69); grid_init reads no key GP_init has not read before it
const char* const kRequiredKeys[] = {
    "sim_smallB",       "sim_smallPressure", "sim_smallDensity",   "sim_smallEnergy",    "sim_gamma",
    "sim_riemannSolver", "sim_cfl",          "sim_tmax",           "sim_nstepmax",       "sim_BC",
    "sim_dataFileBaseName", "sim_outputFreqTime", "sim_outputFreqStep", "sim_outputHdf5", "sim_outputAscii",
    "sim_forceHydro",   "grid_xBeg",         "grid_xEnd",          "grid_yBeg",          "grid_yEnd",
    "grid_Nx",          "grid_Ny",           "GP_ellOverDelta",    "GP_maxRadius"};

extern "C" int hosono_par_load(const char* parfile, hosono_params* p, hosono_run_info* run, char* err, int errlen) {
    if (!p) return HOSONO_EINVAL;
    ParFile f(parfile);
    if (!f.ok) {
        put_err(err, errlen, std::string("cannot open parameter file ") + (parfile ? parfile : "(null)"));
        return HOSONO_EPAR;
    }
    std::vector<std::string> missing;
    for (const char* k : kRequiredKeys)
        if (!f.raw(k)) missing.emplace_back(k);
    if (!missing.empty()) {  // the reference's message for the first, then the rest
        std::string m = "The parameter '" + missing[0] + "' was not found inside of '" + f.path + "'";
        for (size_t k = 1; k < missing.size(); k++) m += (k == 1 ? " (also missing: " : ", ") + missing[k];
        if (missing.size() > 1) m += ")";
        put_err(err, errlen, m);
        return HOSONO_EPAR;
    }
    try {
        hosono_params q{};
        hosono_run_info r{};
        // simulation_init, in the reference's read order
        q.small_b = get_real(f, "sim_smallB");
        q.small_pressure = get_real(f, "sim_smallPressure");
        q.small_density = get_real(f, "sim_smallDensity");
        q.small_energy = get_real(f, "sim_smallEnergy");
        q.gamma = get_real(f, "sim_gamma");
        const std::string rs = get_str(f, "sim_riemannSolver");
        q.cfl = get_real(f, "sim_cfl");
        r.tmax = get_real(f, "sim_tmax");
        r.nstepmax = get_int(f, "sim_nstepmax");
        const std::string bc = get_str(f, "sim_BC");
        std::snprintf(r.data_file_base, sizeof r.data_file_base, "%s", get_str(f, "sim_dataFileBaseName").c_str());
        r.output_freq_time = get_real(f, "sim_outputFreqTime");
        r.output_freq_step = get_int(f, "sim_outputFreqStep");
        (void)get_logical(f, "sim_outputHdf5");
        (void)get_logical(f, "sim_outputAscii");
        q.force_hydro = get_logical(f, "sim_forceHydro") ? 1 : 0;
        if (rs != "hllc" && rs != "hllcmhd") {
            put_err(err, errlen, "Unrecognized choice of riemann solver: " + rs);
            return HOSONO_EPAR;
        }
        q.riemann_solver = 1;
        if (bc == "outflow")
            q.bc = HOSONO_BC_OUTFLOW;
        else if (bc == "periodic")
            q.bc = HOSONO_BC_PERIODIC;
        else {
            put_err(err, errlen, "Unrecognized choice of boundary condition: " + bc);
            return HOSONO_EPAR;
        }
        // GP_init's radius and grid_init
        q.max_radius = get_int(f, "GP_maxRadius");
        r.ell_over_delta = get_real(f, "GP_ellOverDelta");
        q.nx = get_int(f, "grid_Nx");
        q.ny = get_int(f, "grid_Ny");
        r.x_beg = get_real(f, "grid_xBeg");
        r.x_end = get_real(f, "grid_xEnd");
        r.y_beg = get_real(f, "grid_yBeg");
        r.y_end = get_real(f, "grid_yEnd");
        if (q.max_radius < 1 || q.max_radius > 3 || q.nx < 1 || q.ny < 1) {
            put_err(err, errlen, "grid_Nx, grid_Ny must be positive and GP_maxRadius in 1..3");
            return HOSONO_EPAR;
        }
        q.ngc = q.max_radius + 2;
        q.dx = (r.x_end - r.x_beg) / q.nx;
        q.dy = (r.y_end - r.y_beg) / q.ny;
        q.mindxdy = std::fmin(q.dx, q.dy);
        q.maxdxdy = std::fmax(q.dx, q.dy);
        q.fp_mode = HOSONO_FP_STRICT;
        r.nx_tot = q.nx + 2 * q.ngc;
        r.ny_tot = q.ny + 2 * q.ngc;
        const std::string* ic = f.raw("IC_type");
        std::snprintf(r.ic_type, sizeof r.ic_type, "%s", ic ? item(*ic).c_str() : "");
        *p = q;
        if (run) *run = r;
    } catch (const Missing& m) {
        put_err(err, errlen, "The parameter '" + m.key + "' was not found inside of '" + f.path + "'");
        return HOSONO_EPAR;
    }
    return HOSONO_OK;
}

extern "C" int hosono_par_gp(const char* parfile, double* pv, double* qw, int* stenc, char* err, int errlen) {
    ParFile f(parfile);
    if (!f.ok) {
        put_err(err, errlen, "cannot open parameter file");
        return HOSONO_EPAR;
    }
    try {
        const int rc = hosono_gp_build(get_int(f, "GP_maxRadius"), get_str(f, "grid_xBeg").c_str(),
                                       get_str(f, "grid_xEnd").c_str(), get_int(f, "grid_Nx"),
                                       get_str(f, "grid_yBeg").c_str(), get_str(f, "grid_yEnd").c_str(),
                                       get_int(f, "grid_Ny"), get_str(f, "GP_ellOverDelta").c_str(), pv, qw, stenc);
        if (rc) put_err(err, errlen, "GP set-up failed (radius must be 1..3; covariance must be positive definite)");
        return rc;
    } catch (const Missing& m) {
        put_err(err, errlen, "The parameter '" + m.key + "' was not found inside of '" + f.path + "'");
        return HOSONO_EPAR;
    }
}

extern "C" int hosono_ic_set(const char* parfile, const hosono_params* p, double* U, double* V, char* err, int errlen) {
    if (!p || !U || !V) return HOSONO_EINVAL;
    ParFile f(parfile);
    if (!f.ok) {
        put_err(err, errlen, "cannot open parameter file");
        return HOSONO_EPAR;
    }
    const int g = p->ngc, nxt = p->nx + 2 * g, nyt = p->ny + 2 * g;
    const size_t cells = (size_t)nxt * nyt;
    const double gam = p->gamma;
    try {
        const double xb = get_real(f, "grid_xBeg"), yb = get_real(f, "grid_yBeg");
        // cell centres, src/grid.f90:92-97 (1-based index i -> 0-based i+1)
        auto xc = [&](int i) { return ((i + 1) - g - 0.5) * p->dx + xb; };
        auto yc = [&](int j) { return ((j + 1) - g - 0.5) * p->dy + yb; };
        for (size_t t = 0; t < cells * 10; t++) V[t] = 0.0;
        for (size_t t = 0; t < cells * 8; t++) U[t] = 0.0;
        const std::string type = get_str(f, "IC_type");
        auto Vc = [&](int i, int j) { return &V[10 * ((size_t)j * nxt + i)]; };
        if (type == "explosion2d") {  // :86-136
            const double cx = get_real(f, "IC_shockCenter_x"), cy = get_real(f, "IC_shockCenter_y");
            const double rad = get_real(f, "IC_shockRad");
            const double dIn = get_real(f, "IC_densIns"), dOut = get_real(f, "IC_densOut");
            const double uIn = get_real(f, "IC_velxIns"), vIn = get_real(f, "IC_velyIns"), wIn = get_real(f, "IC_velzIns");
            const double uOut = get_real(f, "IC_velxOut"), vOut = get_real(f, "IC_velyOut"), wOut = get_real(f, "IC_velzOut");
            const double pIn = get_real(f, "IC_presIns"), pOut = get_real(f, "IC_presOut");
            const double bx = get_real_or(f, "IC_magx", 0.0), by = get_real_or(f, "IC_magy", 0.0), bz = get_real_or(f, "IC_magz", 0.0);
            for (int j = g; j < g + p->ny; j++)
                for (int i = g; i < g + p->nx; i++) {
                    const double ddx = xc(i) - cx, ddy = yc(j) - cy;
                    const bool in = std::sqrt(ddx * ddx + ddy * ddy) <= rad;
                    double* v = Vc(i, j);
                    v[0] = in ? dIn : dOut;
                    v[1] = in ? uIn : uOut;
                    v[2] = in ? vIn : vOut;
                    v[3] = in ? wIn : wOut;
                    v[4] = in ? pIn : pOut;
                    v[5] = bx;
                    v[6] = by;
                    v[7] = bz;
                }
        } else if (type == "sedov2d") {  // :138-187
            const double cx = get_real(f, "IC_shockCenter_x"), cy = get_real(f, "IC_shockCenter_y");
            const double rad = 3.5 * std::fmin(p->dx, p->dy);
            const int nn = 2;
            const double pIn = 3 * (gam - 1) * 1.0 / ((nn + 1) * kPi * (rad * rad));
            for (int j = g; j < g + p->ny; j++)
                for (int i = g; i < g + p->nx; i++) {
                    const double ddx = xc(i) - cx, ddy = yc(j) - cy;
                    double* v = Vc(i, j);
                    v[0] = 1.0;
                    v[4] = std::sqrt(ddx * ddx + ddy * ddy) <= rad ? pIn : 1e-5;
                }
        } else if (type == "OrszagTang2d") {  // :189-226
            const double U0 = get_real(f, "IC_U0"), dens = get_real(f, "IC_dens");
            const double B0 = get_real_or(f, "IC_B0", 1 / gam), pres = get_real_or(f, "IC_pres", 1 / gam);
            for (int j = g; j < g + p->ny; j++)
                for (int i = g; i < g + p->nx; i++) {
                    const double xx = xc(i), yy = yc(j);
                    double* v = Vc(i, j);
                    v[0] = dens;
                    v[1] = -U0 * std::sin(kPi * yy * 2.0);
                    v[2] = U0 * std::sin(kPi * xx * 2.0);
                    v[3] = 0.0;
                    v[5] = -B0 * std::sin(kPi * yy * 2.0);
                    v[6] = B0 * std::sin(kPi * xx * 4.0);
                    v[7] = 0.0;
                    v[4] = pres;
                }
        } else {
            put_err(err, errlen, "Unrecognized choice of initial condition: " + type);
            return HOSONO_EPAR;
        }
        // :65-74 eint, gamma and convert_prim2cons (src/convert.f90:159-196)
        for (int j = g; j < g + p->ny; j++)
            for (int i = g; i < g + p->nx; i++) {
                double* v = Vc(i, j);
                double* u = &U[8 * ((size_t)j * nxt + i)];
                v[8] = v[4] / (gam - 1.0) / v[0];
                v[9] = gam;
                const double Bp = p->force_hydro ? 0.0 : 0.5 * (v[5] * v[5] + v[6] * v[6] + v[7] * v[7]);
                const double rhoEint = v[4] / (gam - 1.0);
                u[0] = v[0];
                u[1] = v[0] * v[1];
                u[2] = v[0] * v[2];
                u[3] = v[0] * v[3];
                u[4] = rhoEint + v[0] * (0.5 * (v[1] * v[1] + v[2] * v[2] + v[3] * v[3])) + Bp;
                u[5] = p->force_hydro ? 0.0 : v[5];
                u[6] = p->force_hydro ? 0.0 : v[6];
                u[7] = p->force_hydro ? 0.0 : v[7];
            }
        host_bc(p, U, 8);
        host_bc(p, V, 10);
    } catch (const Missing& m) {
        put_err(err, errlen, "The parameter '" + m.key + "' was not found inside of '" + f.path + "'");
        return HOSONO_EPAR;
    }
    return HOSONO_OK;
}

extern "C" int hosono_ic_describe(const char* parfile, const hosono_params* p, hosono_ic_desc* ic, double* xtab,
                                  double* ytab, char* err, int errlen) {
    if (!p || !ic || !xtab || !ytab) return HOSONO_EINVAL;
    ParFile f(parfile);
    if (!f.ok) {
        put_err(err, errlen, "cannot open parameter file");
        return HOSONO_EPAR;
    }
    const int g = p->ngc, nxt = p->nx + 2 * g, nyt = p->ny + 2 * g;
    const double gam = p->gamma;
    try {
        const double xb = get_real(f, "grid_xBeg"), yb = get_real(f, "grid_yBeg");
        // the expressions of hosono_ic_set, tabulated per column / row
        for (int i = 0; i < nxt; i++) {
            const double xx = ((i + 1) - g - 0.5) * p->dx + xb;
            xtab[i] = xx;
            xtab[nxt + i] = std::sin(kPi * xx * 2.0);
            xtab[2 * nxt + i] = std::sin(kPi * xx * 4.0);
        }
        for (int j = 0; j < nyt; j++) {
            const double yy = ((j + 1) - g - 0.5) * p->dy + yb;
            ytab[j] = yy;
            ytab[nyt + j] = std::sin(kPi * yy * 2.0);
        }
        hosono_ic_desc d{};
        const std::string type = get_str(f, "IC_type");
        if (type == "explosion2d") {
            d.type = HOSONO_IC_EXPLOSION;
            const char* keys[13] = {"IC_shockCenter_x", "IC_shockCenter_y", "IC_shockRad", "IC_densIns", "IC_densOut",
                                    "IC_velxIns", "IC_velyIns", "IC_velzIns", "IC_velxOut", "IC_velyOut",
                                    "IC_velzOut", "IC_presIns", "IC_presOut"};
            for (int k = 0; k < 13; k++) d.c[k] = get_real(f, keys[k]);
            d.c[13] = get_real_or(f, "IC_magx", 0.0);
            d.c[14] = get_real_or(f, "IC_magy", 0.0);
            d.c[15] = get_real_or(f, "IC_magz", 0.0);
        } else if (type == "sedov2d") {
            d.type = HOSONO_IC_SEDOV;
            d.c[0] = get_real(f, "IC_shockCenter_x");
            d.c[1] = get_real(f, "IC_shockCenter_y");
            const double rad = 3.5 * std::fmin(p->dx, p->dy);
            const int nn = 2;
            d.c[2] = rad;
            d.c[3] = 3 * (gam - 1) * 1.0 / ((nn + 1) * kPi * (rad * rad));
        } else if (type == "OrszagTang2d") {
            d.type = HOSONO_IC_ORSZAG_TANG;
            d.c[0] = get_real(f, "IC_U0");
            d.c[1] = get_real(f, "IC_dens");
            d.c[2] = get_real_or(f, "IC_B0", 1 / gam);
            d.c[3] = get_real_or(f, "IC_pres", 1 / gam);
        } else {
            put_err(err, errlen, "Unrecognized choice of initial condition: " + type);
            return HOSONO_EPAR;
        }
        *ic = d;
    } catch (const Missing& m) {
        put_err(err, errlen, "The parameter '" + m.key + "' was not found inside of '" + f.path + "'");
        return HOSONO_EPAR;
    }
    return HOSONO_OK;
}
