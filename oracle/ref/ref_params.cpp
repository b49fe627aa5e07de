// Run-time parameter definitions for the CPU oracle build of the reference.
//
// The reference keeps every simulation parameter as a compile-time global in
// src/constants.cpp (declared in include/constants.h:9-99) and expects users
// to edit that file per run.  The oracle instead defines the same globals
// here, initialised from a "name value" text file named by the environment
// variable PIC3D_REF_PARAMS, so one oracle binary can run every workload.
// All other reference translation units read these symbols through their
// extern declarations, so they see the values set here.  Test
// infrastructure only.
#include "constants.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>

namespace {

const std::map<std::string, double> &param_table() {
    static std::map<std::string, double> table = [] {
        std::map<std::string, double> t;
        const char *path = std::getenv("PIC3D_REF_PARAMS");
        if (!path) {
            std::fprintf(stderr, "oracle: PIC3D_REF_PARAMS is not set\n");
            std::exit(2);
        }
        FILE *f = std::fopen(path, "r");
        if (!f) {
            std::fprintf(stderr, "oracle: cannot open %s\n", path);
            std::exit(2);
        }
        char key[128];
        double v;
        while (std::fscanf(f, "%127s %lf", key, &v) == 2) t[key] = v;
        std::fclose(f);
        return t;
    }();
    return table;
}

double P(const char *name) {
    auto &t = param_table();
    auto it = t.find(name);
    if (it == t.end()) {
        std::fprintf(stderr, "oracle: parameter %s missing\n", name);
        std::exit(2);
    }
    return it->second;
}

int I(const char *name) { return (int)P(name); }

}  // namespace

const double Pi = P("Pi");
const double c1 = 1.0;
const double q_e = -1.0;
const double m_e = 1.0;
const double omega = P("omega");
const double epsilon_0 = 1.0;

const double l0 = P("l0");
const double t0 = P("t0");
const double Lx = P("Lx");
const double Ly = P("Ly");
const double Lz = P("Lz");
const int resx = I("resx");
const int resy = I("resy");
const int resz = I("resz");
const int rest = I("rest");
const int rank_len[3] = {1, 1, 1};
const int rank_period[3] = {I("period_x"), I("period_y"), I("period_z")};
int rank_reorder = 1;
int rank_coords[3] = {0, 0, 0};
int rank_xminus, rank_xplus, rank_yminus, rank_yplus, rank_zminus, rank_zplus;

const int local_xcells = I("local_xcells");
const int local_ycells = I("local_ycells");
const int local_zcells = I("local_zcells");
const int global_nx = local_xcells;
const int global_ny = local_ycells;
const int global_nz = local_zcells;
const int cell_per_particles = I("cell_per_particles");
const double density = P("density");
const double dx = P("dx");
const double dy = P("dy");
const double dz = P("dz");
const double dt = P("dt");
const double dt_half = P("dt_half");
const double simulation_time = P("simulation_time");
const int timesteps = I("timesteps");
const int output_interval = I("output_interval");
const int num_steps = 0;
bool is_periodic = false;
bool is_relativistic_poission = false;
const int num_kind = 2;

const int mem = I("mem");
MPI_Datatype type_field_Xdir, type_field_Ydir, type_field_Zdir, type_current_Xdir, type_current_Ydir,
    type_current_Zdir;

const double laser_amplitude = P("laser_amplitude");
const double laser_pulse_duration = P("laser_pulse_duration");
const double laser_start_time = P("laser_start_time");
const int laser_polarization = I("laser_polarization");
const double waist = P("waist");
const double xfocus = P("xfocus");
const double phase = P("phase");
const double yfocus = P("yfocus");
const double zfocus = P("zfocus");

int nc_xst, nc_xend;
int nc_xst_new, nc_xend_new;
int nc_xst_out, nc_xend_out;
double xst, xend;
int nc_yst, nc_yend;
int nc_yst_new, nc_yend_new;
int nc_yst_out, nc_yend_out;
double yst, yend;
int nc_zst, nc_zend;
int nc_zst_new, nc_zend_new;
int nc_zst_out, nc_zend_out;
double zst, zend;

double E_schwinger = P("E_schwinger");
// 4th-order shape-function coefficients (the quartic B-spline pieces).
const double alpha0 = 55.0 / 96.0, alpha1 = 5.0 / 24.0, alpha2 = 5.0 / 4.0, alpha3 = 5.0 / 6.0,
             beta0 = 115.0 / 192.0, beta2 = 5.0 / 8.0;

// The oracle harness loads particles from a file; the density profile of
// each workload is applied by the input generator, so these are unused.
double plasma_density(double, double, double) { return density; }
double plasma_density1(double, double, double) { return 0.0; }

const int g_data_size = 2849;
double g_data[g_data_size];

bool load_g_data() {
    const char *path = std::getenv("PIC3D_G_TXT");
    FILE *f = std::fopen(path ? path : "g.txt", "r");
    if (!f) return false;
    for (int i = 0; i < g_data_size; ++i) {
        if (std::fscanf(f, "%lf", &g_data[i]) != 1) {
            std::fclose(f);
            return false;
        }
    }
    std::fclose(f);
    return true;
}
