// Harness main() for the CPU oracle build of the reference PIC3D sources.
//
// Replays the reference start-up sequence of main.cpp:19-87 on one rank:
// Cartesian topology, initialize_domain, the t=0 push + particle exchange
// (main.cpp:75-79), the step-0 output, then run_main_time_loop
// (src/simulation.cpp:154-205).  Differences from main.cpp, all required to
// run the reference deterministically on one CPU process:
//   * every array allocated by initialize_domain is zeroed first (the
//     reference allocates with new[] and never clears, simulation.cpp:337);
//   * particles are read from a binary file (two species, each as an array
//     of the reference's 144-byte `particle` struct) instead of
//     initialize_particles, so seeded random/Maxwellian inputs can be used;
//   * the HDF5 writers (src/io_utils.cpp) are replaced by raw dumps of the
//     full field buffers and particle vectors.
// Usage: pic3d_ref <particles.bin> <outdir|-> [time]
//   outdir "-" disables dumps.  With "time" the wall time of
//   run_main_time_loop is printed as one JSON line.
// Test infrastructure only.
#include "constants.h"
#include "field.h"
#include "io_utils.h"
#include "mpi_utils.h"
#include "particle.h"
#include "simulation.h"

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

static std::string g_outdir;

static long field_len() {
    return (long)(nc_zend_out - nc_zst_out + 1) * (nc_yend_out - nc_yst_out + 1) * (nc_xend_out - nc_xst_out + 1);
}
static long ring_len() {
    return (long)(nc_zend_out - nc_zst_out + 3) * (nc_yend_out - nc_yst_out + 3) * (nc_xend_out - nc_xst_out + 3);
}
static double *field_base(double ***a) { return &a[nc_zst_out][nc_yst_out][nc_xst_out]; }
static double *ring_base(double ***a) { return &a[nc_zst_out - 1][nc_yst_out - 1][nc_xst_out - 1]; }

void output_data_hdf5(int step, int, int, MPI_Comm, hid_t) {
    if (g_outdir.empty()) return;
    char name[512];
    std::snprintf(name, sizeof name, "%s/step_%05d.fields", g_outdir.c_str(), step);
    FILE *f = std::fopen(name, "wb");
    if (!f) { std::perror(name); std::exit(3); }
    double ***fields[6] = {ex, ey, ez, bx, by, bz};
    for (auto a : fields) std::fwrite(field_base(a), sizeof(double), field_len(), f);
    double ***rings[5] = {jx, jy, jz, rho_particle[0], rho_particle[1]};
    for (auto a : rings) std::fwrite(ring_base(a), sizeof(double), ring_len(), f);
    std::fclose(f);
}

void output_particles_hdf5(int step, int, int, MPI_Comm, const std::vector<std::vector<particle>> &particles,
                           const int *num_particles) {
    if (g_outdir.empty()) return;
    char name[512];
    std::snprintf(name, sizeof name, "%s/step_%05d.particles", g_outdir.c_str(), step);
    FILE *f = std::fopen(name, "wb");
    if (!f) { std::perror(name); std::exit(3); }
    for (int k = 0; k < num_kind; ++k) {
        int64_t n = num_particles[k];
        std::fwrite(&n, sizeof n, 1, f);
    }
    for (int k = 0; k < num_kind; ++k)
        std::fwrite(particles[k].data(), sizeof(particle), (size_t)num_particles[k], f);
    std::fclose(f);
}

int main(int argc, char **argv) {
    static_assert(sizeof(particle) == 144, "reference particle struct layout");
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s <particles.bin> <outdir|-> [time]\n", argv[0]);
        return 2;
    }
    if (std::strcmp(argv[2], "-") != 0) g_outdir = argv[2];
    bool timing = argc > 3 && std::strcmp(argv[3], "time") == 0;

    MPI_Init(&argc, &argv);
    int my_rank, num_procs;
    MPI_Comm my_comm;
    MPI_Comm_size(MPI_COMM_WORLD, &num_procs);
    MPI_Cart_create(MPI_COMM_WORLD, 3, rank_len, rank_period, rank_reorder, &my_comm);
    MPI_Comm_rank(my_comm, &my_rank);
    MPI_Cart_coords(my_comm, my_rank, 3, rank_coords);
    MPI_Cart_shift(my_comm, 0, +1, &rank_xminus, &rank_xplus);
    MPI_Cart_shift(my_comm, 1, +1, &rank_yminus, &rank_yplus);
    MPI_Cart_shift(my_comm, 2, +1, &rank_zminus, &rank_zplus);

    hid_t plist_id = H5P_DEFAULT;
    initialize_domain(my_rank);

    double ***fields[6] = {ex, ey, ez, bx, by, bz};
    for (auto a : fields) std::memset(field_base(a), 0, sizeof(double) * field_len());
    double ***rings[12] = {jx, jy, jz, rho_local, rho_particle[0], rho_particle[1], current_recv_xminus,
                           current_recv_xplus, current_recv_yminus, current_recv_yplus, current_recv_zminus,
                           current_recv_zplus};
    for (auto a : rings) std::memset(ring_base(a), 0, sizeof(double) * ring_len());

    if (!load_g_data()) {
        std::fprintf(stderr, "oracle: g.txt could not be read (set PIC3D_G_TXT)\n");
        return 2;
    }

    int num_particles[2];
    std::vector<std::vector<particle>> particles(num_kind);
    FILE *pf = std::fopen(argv[1], "rb");
    if (!pf) { std::perror(argv[1]); return 2; }
    int64_t counts[2];
    if (std::fread(counts, sizeof(int64_t), 2, pf) != 2) return 2;
    for (int k = 0; k < num_kind; ++k) {
        particles[k].resize((size_t)counts[k]);
        if (counts[k] && std::fread(particles[k].data(), sizeof(particle), (size_t)counts[k], pf) != (size_t)counts[k])
            return 2;
        num_particles[k] = (int)counts[k];
    }
    std::fclose(pf);

    auto t0c = std::chrono::steady_clock::now();
    update_particle_position_momentum(particles[0], num_particles[0], my_rank, 0);
    update_particle_position_momentum(particles[1], num_particles[1], my_rank, 1);
    exchange_particle_data(particles[0], num_particles[0], my_rank, my_comm);
    exchange_particle_data(particles[1], num_particles[1], my_rank, my_comm);
    output_data_hdf5(0, my_rank, num_procs, my_comm, plist_id);
    output_particles_hdf5(0, my_rank, num_procs, my_comm, particles, num_particles);

    auto t1c = std::chrono::steady_clock::now();
    int64_t n0 = (int64_t)num_particles[0] + num_particles[1];
    run_main_time_loop(particles, num_particles, my_rank, num_procs, plist_id, my_comm);
    auto t2c = std::chrono::steady_clock::now();
    int64_t n1 = (int64_t)num_particles[0] + num_particles[1];

    if (timing) {
        double loop_s = std::chrono::duration<double>(t2c - t1c).count();
        double init_s = std::chrono::duration<double>(t1c - t0c).count();
        std::printf("{\"steps\": %d, \"particles_start\": %lld, \"particles_end\": %lld, "
                    "\"loop_seconds\": %.6f, \"initial_push_seconds\": %.6f}\n",
                    timesteps, (long long)n0, (long long)n1, loop_s, init_s);
    }
    free_memory();
    MPI_Finalize();
    return 0;
}
