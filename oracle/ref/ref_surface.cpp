// Call-surface harness: exercises the functions of the reference PIC3D that
// its main sequence (main.cpp, src/simulation.cpp:154-205) does not reach
// or reaches only inside the loop, and dumps what they produce.  The same
// source is linked twice: against the reference's own src/*.cpp (CPU) and
// against the C++ drop-in shim over the GPU library, so the two dumps can be
// compared.  Test infrastructure only.
//
// Sequence (each line's results are appended to <out>):
//   initialize_domain; deterministic values in every host array
//   initialize_particles for both species (src/particle.cpp:50-111) with
//     the density profiles below                            -> both vectors
//   shape_function_2 / _4, g_factor, generate_laser_pulse, Gpulse at fixed
//     arguments                                             -> the values
//   update_electromagnetic_fields (full dt)                 -> all arrays
//   exchange_boundary_data on ex..bz                        -> all arrays
//   binomial_filter_currents; filter_field(rho_particle[0]) -> all arrays
//   exchange_boundary_current_fixed on jx..jz, rho_particle -> all arrays
//   currents_particle for a few moves of both species       -> all arrays
//   radiating_boundary at step 7; both field half-updates   -> all arrays
// Usage: pic3d_surface <out>  (parameters from PIC3D_REF_PARAMS, g table
// from PIC3D_G_TXT)
#include "boundary.h"
#include "constants.h"
#include "field.h"
#include "io_utils.h"
#include "mpi_utils.h"
#include "particle.h"
#include "simulation.h"

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

void filter_field(double ***data);   // src/particle.cpp:520 (no header declares it)

// the time loop is not run here; its writers only have to link
void output_data_hdf5(int, int, int, MPI_Comm, hid_t) {}
void output_particles_hdf5(int, int, int, MPI_Comm, const std::vector<std::vector<particle>> &, const int *) {}

namespace {

FILE *g_out = nullptr;

void put(const void *p, size_t bytes) {
    if (std::fwrite(p, 1, bytes, g_out) != bytes) std::exit(3);
}

long field_len() {
    return (long)(nc_zend_out - nc_zst_out + 1) * (nc_yend_out - nc_yst_out + 1) * (nc_xend_out - nc_xst_out + 1);
}
long ring_len() {
    return (long)(nc_zend_out - nc_zst_out + 3) * (nc_yend_out - nc_yst_out + 3) * (nc_xend_out - nc_xst_out + 3);
}
double *field_base(double ***a) { return &a[nc_zst_out][nc_yst_out][nc_xst_out]; }
double *ring_base(double ***a) { return &a[nc_zst_out - 1][nc_yst_out - 1][nc_xst_out - 1]; }

void dump_arrays() {
    double ***f[6] = {ex, ey, ez, bx, by, bz};
    for (auto a : f) put(field_base(a), sizeof(double) * field_len());
    double ***r[5] = {jx, jy, jz, rho_particle[0], rho_particle[1]};
    for (auto a : r) put(ring_base(a), sizeof(double) * ring_len());
}

void dump_particles(const std::vector<particle> &v, int n) {
    int64_t c = n;
    put(&c, sizeof c);
    put(v.data(), sizeof(particle) * (size_t)n);
}

// values in [-scale, scale) from a 64-bit LCG
uint64_t g_seed = 0x9E3779B97F4A7C15ull;
double next_value(double scale) {
    g_seed = g_seed * 6364136223846793005ull + 1442695040888963407ull;
    return scale * ((double)(g_seed >> 11) / 9007199254740992.0 * 2.0 - 1.0);
}

// electrons: linear ramp in x over the first half, zero in a slab
double density_e(double x, double y, double z) {
    if (x > 0.5 * global_nx) return density;
    if (y < 1.0) return 0.0;
    return density * x / (0.5 * global_nx) + 0.0 * z;
}
// protons: a box in the middle
double density_p(double x, double y, double z) {
    bool in = x > 0.25 * global_nx && x < 0.75 * global_nx && y > 0.25 * global_ny && z < 0.75 * global_nz;
    return in ? 0.5 * density : 0.0;
}

particle move(double x0, double y0, double z0, double x1, double y1, double z1, double q, double w) {
    particle p;
    std::memset(&p, 0, sizeof p);
    p.x_old = x0;
    p.y_old = y0;
    p.z_old = z0;
    p.x = x1;
    p.y = y1;
    p.z = z1;
    p.charge = q;
    p.weight = w;
    p.mass = 1.0;
    p.gamma = 1.0;
    return p;
}

}  // namespace

int main(int argc, char **argv) {
    static_assert(sizeof(particle) == 144, "reference particle struct layout");
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s <out>\n", argv[0]);
        return 2;
    }
    g_out = std::fopen(argv[1], "wb");
    if (!g_out) {
        std::perror(argv[1]);
        return 2;
    }
    MPI_Init(&argc, &argv);
    int my_rank, num_procs;
    MPI_Comm comm;
    MPI_Comm_size(MPI_COMM_WORLD, &num_procs);
    MPI_Cart_create(MPI_COMM_WORLD, 3, rank_len, rank_period, rank_reorder, &comm);
    MPI_Comm_rank(comm, &my_rank);
    MPI_Cart_coords(comm, my_rank, 3, rank_coords);
    MPI_Cart_shift(comm, 0, +1, &rank_xminus, &rank_xplus);
    MPI_Cart_shift(comm, 1, +1, &rank_yminus, &rank_yplus);
    MPI_Cart_shift(comm, 2, +1, &rank_zminus, &rank_zplus);

    initialize_domain(my_rank);
    // every host array gets deterministic values before the first device call
    double ***f[6] = {ex, ey, ez, bx, by, bz};
    for (auto a : f) {
        double *p = field_base(a);
        for (long i = 0; i < field_len(); ++i) p[i] = next_value(0.1);
    }
    double ***r[5] = {jx, jy, jz, rho_particle[0], rho_particle[1]};
    for (auto a : r) {
        double *p = ring_base(a);
        for (long i = 0; i < ring_len(); ++i) p[i] = next_value(0.01);
    }
    if (!load_g_data()) {
        std::fprintf(stderr, "surface: g.txt could not be read (set PIC3D_G_TXT)\n");
        return 2;
    }

    std::vector<std::vector<particle>> parts(num_kind);
    int num[2] = {0, 0};
    initialize_particles(parts[0], num[0], density_e, q_e, m_e, 0.01, -0.02, 0.03, 0.0, 0.0, 0.0, my_rank);
    initialize_particles(parts[1], num[1], density_p, -q_e, 1836.0 * m_e, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, my_rank);
    dump_particles(parts[0], num[0]);
    dump_particles(parts[1], num[1]);

    // scalar helpers
    const double xs[6] = {3.0, 3.2, 3.49999, 3.5, 4.75, 7.125};
    for (double x : xs) {
        double w2[3], w4[5];
        shape_function_2(x, w2);
        shape_function_4(x, w4);
        put(w2, sizeof w2);
        put(w4, sizeof w4);
    }
    const double chis[8] = {0.0, 0.004, 0.0071, 0.5, 3.3, 12.5, 55.0, 60.0};
    for (double c : chis) {
        double g = g_factor(c);
        put(&g, sizeof g);
    }
    const double tt[5] = {-1.0, 0.0, 0.3 * laser_pulse_duration, 0.77 * laser_pulse_duration, 2.0 * laser_pulse_duration};
    for (double t : tt) {
        double a = generate_laser_pulse(t, 0.0), b = generate_laser_pulse(t, 0.25 * laser_pulse_duration);
        double g1 = Gpulse(t, 0.0, 1.5 * dy, -2.0 * dz), g2 = Gpulse(t, 0.3, -0.7 * waist, 0.2 * waist);
        put(&a, sizeof a);
        put(&b, sizeof b);
        put(&g1, sizeof g1);
        put(&g2, sizeof g2);
    }

    update_electromagnetic_fields(my_rank, num_procs, comm);
    dump_arrays();
    for (auto a : f) exchange_boundary_data(a, comm);
    dump_arrays();
    binomial_filter_currents();
    filter_field(rho_particle[0]);
    dump_arrays();
    for (auto a : r) exchange_boundary_current_fixed(a, comm);
    dump_arrays();
    const double cx = 0.5 * global_nx, cy = 0.5 * global_ny, cz = 0.5 * global_nz;
    particle moves[4] = {
        move(cx + 0.1, cy + 0.2, cz + 0.3, cx + 0.4, cy + 0.1, cz + 0.35, q_e, 0.125),
        move(cx + 0.45, cy - 0.3, cz + 0.49, cx + 0.62, cy - 0.55, cz + 0.51, q_e, 0.25),   // crosses cell edges
        move(1.2, 2.7, cz, 0.9, 2.3, cz - 0.2, -q_e, 0.5),
        move(global_nx - 1.3, 1.6, 2.2, global_nx - 0.8, 1.4, 2.6, -q_e, 0.0625),
    };
    for (int i = 0; i < 4; ++i) currents_particle(moves[i], i < 2 ? 0 : 1);
    dump_arrays();
    radiating_boundary(my_rank, 1, 0, num_procs, 7);
    update_electromagnetic_fields_first(my_rank, num_procs, comm);
    update_electromagnetic_fields_second(my_rank, num_procs, comm);
    dump_arrays();

    std::fclose(g_out);
    free_memory();
    MPI_Finalize();
    return 0;
}
