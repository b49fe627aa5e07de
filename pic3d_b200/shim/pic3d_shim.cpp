// C++ drop-in for the per-step translation units of PIC3D.
//
// Linked instead of the reference's src/field.cpp, src/particle.cpp,
// src/boundary.cpp, src/mpi_utils.cpp and src/simulation.cpp (its
// src/constants.cpp, src/io_utils.cpp and main.cpp stay as they are), this
// file defines every function and global those five files define, over the C
// ABI of libpic3d_b200.so (include/pic3d_gpu.h).  It is compiled against the
// reference's own headers (include/constants.h, field.h, particle.h,
// boundary.h, simulation.h, mpi_utils.h, io_utils.h).
//
// State.  initialize_domain creates one GPU context and the host arrays
// (ex..bz, jx..jz, rho_local, rho_particle, current_recv_*) with the
// reference's index ranges and contiguous z-major storage.  The device copy
// is authoritative:
//   host -> device  the host arrays at the first device call after
//                   initialize_domain (zero unless the caller set them); a
//                   species' particle vector at its first push;
//                   pic3d_shim_push_host() on request.
//   device -> host  every per-function call (update_electromagnetic_fields_*,
//                   update_particle_position_momentum, exchange_*,
//                   radiating_boundary, ...) returns with the host arrays and
//                   particle vector it changed brought up to date, so code
//                   written against the reference sees the reference's state
//                   between calls; run_main_time_loop keeps everything on the
//                   device and updates the host state only before each
//                   output_data_hdf5 / output_particles_hdf5 call and on
//                   return.  PIC3D_SHIM_LAZY=1 turns the per-function updates
//                   off (then call pic3d_shim_pull_host before reading).
// Particle vectors come back in the device's order (sorted by cell); ids
// identify particles.
//
// Environment: PIC3D_GPU_DEVICE (default 0), PIC3D_GPU_PRECISION (64, the
// default, or 32), PIC3D_SHIM_LAZY.
// Errors follow the reference's convention: a message on stderr and exit(1).
// One process, one GPU: rank_len must be {1, 1, 1}.
#include "boundary.h"
#include "constants.h"
#include "field.h"
#include "io_utils.h"
#include "mpi_utils.h"
#include "particle.h"
#include "simulation.h"

#include "pic3d_gpu.h"
#include "pic3d_shim.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

// ---------------------------------------------------------------------------
// globals of src/field.cpp:8-22
double max_error = 1.0;
double ***rho_local;
double ****rho_particle;
double ***ex;
double ***phi;
double ***phi_new;
double ***ey;
double ***ez;
double ***bx;
double ***by;
double ***bz;
double ***jx;
double ***jy;
double ***jz;
double ***current_recv_xminus, ***current_recv_xplus, ***current_recv_yminus, ***current_recv_yplus,
    ***current_recv_zminus, ***current_recv_zplus;

namespace {

pic_ctx *g_ctx = nullptr;
bool g_host_dirty = true;          // host arrays not yet copied to the device
bool g_uploaded[2] = {false, false};
const std::vector<particle> *g_owner[2] = {nullptr, nullptr};   // the vector each species came from
bool g_lazy = false;
std::vector<double> g_gtab_sent;   // g table as last copied to the device

[[noreturn]] void die(const char *where, const char *what) {
    std::fprintf(stderr, "pic3d_b200: %s: %s\n", where, what);
    std::fflush(stderr);
    std::exit(1);
}

void check(int status, const char *where) {
    if (status == PIC_OK) return;
    const char *msg = g_ctx ? pic_last_error(g_ctx) : "";
    std::fprintf(stderr, "pic3d_b200: %s failed (status %d): %s\n", where, status, msg ? msg : "");
    std::fflush(stderr);
    std::exit(1);
}

pic_ctx *ctx(const char *where) {
    if (!g_ctx) die(where, "called before initialize_domain");
    return g_ctx;
}

// first element of each device-mirrored host array, in PIC_EX..PIC_RHO1 order
double *host_base(int which) {
    double ***f[6] = {ex, ey, ez, bx, by, bz};
    if (which < 6) return &f[which][nc_zst_out][nc_yst_out][nc_xst_out];
    double ***r[5] = {jx, jy, jz, rho_particle[0], rho_particle[1]};
    return &r[which - 6][nc_zst_out - 1][nc_yst_out - 1][nc_xst_out - 1];
}

int64_t host_len(int which) {
    const int64_t nx = nc_xend_out - nc_xst_out + 1, ny = nc_yend_out - nc_yst_out + 1,
                  nz = nc_zend_out - nc_zst_out + 1;
    return which < 6 ? nx * ny * nz : (nx + 2) * (ny + 2) * (nz + 2);
}

int array_id(double ***a) {
    double ***all[11] = {ex, ey, ez, bx, by, bz, jx, jy, jz, rho_particle[0], rho_particle[1]};
    for (int i = 0; i < 11; ++i)
        if (a == all[i]) return i;
    return -1;
}

void push_arrays() {
    for (int i = 0; i < PIC_NARRAYS; ++i) check(pic_upload_array(g_ctx, i, host_base(i)), "upload array");
    g_host_dirty = false;
}

// the g table may be loaded after initialize_domain (main.cpp:49-58)
void push_g_table() {
    if (g_gtab_sent.size() == (size_t)g_data_size &&
        std::memcmp(g_gtab_sent.data(), g_data, sizeof(double) * g_data_size) == 0)
        return;
    check(pic_set_g_table(g_ctx, g_data, g_data_size), "set g table");
    g_gtab_sent.assign(g_data, g_data + g_data_size);
}

// every device call goes through here first
pic_ctx *ready(const char *where) {
    pic_ctx *c = ctx(where);
    if (g_host_dirty) push_arrays();
    push_g_table();
    return c;
}

void pull_arrays(unsigned mask) {
    if (g_lazy) return;
    for (int i = 0; i < PIC_NARRAYS; ++i)
        if (mask >> i & 1u) check(pic_download_array(g_ctx, i, host_base(i)), "download array");
}

constexpr unsigned kE = 0x7u, kB = 0x38u, kJ = 0x1C0u, kRho0 = 0x200u, kRho1 = 0x400u;

void pull_species(int kind, std::vector<particle> &v, int &num) {
    int64_t n = 0, got = 0;
    check(pic_num_particles(g_ctx, kind, &n), "num_particles");
    v.resize((size_t)n);
    check(pic_download_particles(g_ctx, kind, n ? v.data() : nullptr, n, &got), "download particles");
    v.resize((size_t)got);
    num = (int)got;
}

void upload_species(int kind, const std::vector<particle> &v, int num) {
    if (num < 0 || (size_t)num > v.size()) die("upload particles", "num_particles exceeds the vector's size");
    check(pic_upload_particles(g_ctx, kind, num ? v.data() : nullptr, num), "upload particles");
    g_uploaded[kind] = true;
    g_owner[kind] = &v;
}

template <typename T>
T *alloc_block(size_t n) {
    T *p = new (std::nothrow) T[n]();
    if (!p) die("host allocation", "out of memory");
    return p;
}

}  // namespace

// ---------------------------------------------------------------------------
// shim extras (pic3d_shim.h)

pic_ctx *pic3d_shim_context() { return g_ctx; }

void pic3d_shim_push_host(const std::vector<std::vector<particle>> *particles, const int *num_particles) {
    ctx("pic3d_shim_push_host");
    push_arrays();
    if (particles && num_particles)
        for (int k = 0; k < num_kind && k < 2; ++k) upload_species(k, (*particles)[k], num_particles[k]);
}

void pic3d_shim_pull_host(std::vector<std::vector<particle>> *particles, int *num_particles) {
    ctx("pic3d_shim_pull_host");
    const bool lazy = g_lazy;
    g_lazy = false;
    pull_arrays(kE | kB | kJ | kRho0 | kRho1);
    if (particles && num_particles)
        for (int k = 0; k < num_kind && k < 2; ++k)
            if (g_uploaded[k]) pull_species(k, (*particles)[k], num_particles[k]);
    g_lazy = lazy;
}

// ---------------------------------------------------------------------------
// index-range arrays (src/simulation.cpp:218-491): one contiguous block of
// values, z-major, addressed through row pointers offset by the lower bounds

double **dmatrix(long nrl, long nrh, long ncl, long nch) {
    const long nr = nrh - nrl + 1, nc = nch - ncl + 1;
    double *data = alloc_block<double>((size_t)(nr * nc));
    double **rows = alloc_block<double *>((size_t)nr);
    for (long r = 0; r < nr; ++r) rows[r] = data + r * nc - ncl;
    return rows - nrl;
}

void free_dmatrix(double **m, long nrl, long ncl) {
    if (!m) return;
    double **rows = m + nrl;
    delete[] (rows[0] + ncl);
    delete[] rows;
}

void free_dmatrix(double **m, long nrl) {
    // column lower bound unknown here: the reference's callers use 0
    free_dmatrix(m, nrl, 0);
}

double ***dtensor3(long nzl, long nzh, long nyl, long nyh, long nxl, long nxh) {
    const long nz = nzh - nzl + 1, ny = nyh - nyl + 1, nx = nxh - nxl + 1;
    double *data = alloc_block<double>((size_t)(nz * ny * nx));
    double **rows = alloc_block<double *>((size_t)(nz * ny));
    double ***planes = alloc_block<double **>((size_t)nz);
    for (long k = 0; k < nz; ++k) {
        planes[k] = rows + k * ny - nyl;
        for (long j = 0; j < ny; ++j) rows[k * ny + j] = data + (k * ny + j) * nx - nxl;
    }
    return planes - nzl;
}

void free_dtensor3(double ***m, long nzl, long nyl, long nxl) {
    if (!m) return;
    double ***planes = m + nzl;
    double **rows = planes[0] + nyl;
    delete[] (rows[0] + nxl);
    delete[] rows;
    delete[] planes;
}

double ****dtensor4(long n4l, long n4h, long n3l, long n3h, long n2l, long n2h, long n1l, long n1h) {
    const long n4 = n4h - n4l + 1, n3 = n3h - n3l + 1, n2 = n2h - n2l + 1, n1 = n1h - n1l + 1;
    double *data = alloc_block<double>((size_t)(n4 * n3 * n2 * n1));
    double **rows = alloc_block<double *>((size_t)(n4 * n3 * n2));
    double ***planes = alloc_block<double **>((size_t)(n4 * n3));
    double ****blocks = alloc_block<double ***>((size_t)n4);
    for (long b = 0; b < n4; ++b) {
        blocks[b] = planes + b * n3 - n3l;
        for (long k = 0; k < n3; ++k) {
            planes[b * n3 + k] = rows + (b * n3 + k) * n2 - n2l;
            for (long j = 0; j < n2; ++j)
                rows[(b * n3 + k) * n2 + j] = data + ((b * n3 + k) * n2 + j) * n1 - n1l;
        }
    }
    return blocks - n4l;
}

void free_dtensor4(double ****m, long n4l, long n3l, long n2l, long n1l) {
    if (!m) return;
    double ****blocks = m + n4l;
    double ***planes = blocks[0] + n3l;
    double **rows = planes[0] + n2l;
    delete[] (rows[0] + n1l);
    delete[] rows;
    delete[] planes;
    delete[] blocks;
}

// ---------------------------------------------------------------------------
// set-up (src/simulation.cpp:11-152)

void initialize_simulation(int my_rank, int num_procs) {
    if (my_rank != 0) return;
    std::printf("PIC simulation on the GPU (libpic3d_b200), %d process(es):\n", num_procs);
    std::printf("  timesteps %d, output every %d steps\n", timesteps, output_interval);
    std::printf("  domain Lx=%.2f, dx=%.6f, dt=%.6f, %d x %d x %d cells, mem %d\n", Lx, dx, dt, local_xcells,
                local_ycells, local_zcells, mem);
}

void initialize_domain(int my_rank) {
    if (rank_len[0] * rank_len[1] * rank_len[2] != 1 || my_rank != 0)
        die("initialize_domain", "the GPU path runs one process: rank_len must be {1, 1, 1}");
    if (g_ctx) die("initialize_domain", "called twice");
    // one rank at Cartesian coordinates (0, 0, 0): physical cells mem .. mem+n-1
    // of each buffer, global particle coordinate x in [0, n) at buffer x+mem-1
    const int n[3] = {local_xcells, local_ycells, local_zcells};
    int *st[3] = {&nc_xst, &nc_yst, &nc_zst}, *en[3] = {&nc_xend, &nc_yend, &nc_zend};
    int *nw[3] = {&nc_xst_new, &nc_yst_new, &nc_zst_new};
    int *so[3] = {&nc_xst_out, &nc_yst_out, &nc_zst_out}, *eo[3] = {&nc_xend_out, &nc_yend_out, &nc_zend_out};
    double *lo[3] = {&xst, &yst, &zst}, *hi[3] = {&xend, &yend, &zend};
    for (int d = 0; d < 3; ++d) {
        const int first = rank_coords[d] * n[d] + 1;
        *lo[d] = (double)(first - 1);
        *hi[d] = (double)(first + n[d] - 1);
        *nw[d] = first - mem;
        *st[d] = mem;
        *en[d] = mem + n[d] - 1;
        *so[d] = 0;
        *eo[d] = 2 * mem + n[d] - 1;
    }
    double ****fld[6] = {&ex, &ey, &ez, &bx, &by, &bz};
    for (auto f : fld) *f = dtensor3(nc_zst_out, nc_zend_out, nc_yst_out, nc_yend_out, nc_xst_out, nc_xend_out);
    double ****ring[10] = {&jx, &jy, &jz, &rho_local, &current_recv_xminus, &current_recv_xplus,
                           &current_recv_yminus, &current_recv_yplus, &current_recv_zminus, &current_recv_zplus};
    for (auto r : ring)
        *r = dtensor3(nc_zst_out - 1, nc_zend_out + 1, nc_yst_out - 1, nc_yend_out + 1, nc_xst_out - 1,
                      nc_xend_out + 1);
    rho_particle = dtensor4(0, num_kind - 1, nc_zst_out - 1, nc_zend_out + 1, nc_yst_out - 1, nc_yend_out + 1,
                            nc_xst_out - 1, nc_xend_out + 1);

    PicParams p;
    pic_default_params(&p);
    p.local_xcells = local_xcells;
    p.local_ycells = local_ycells;
    p.local_zcells = local_zcells;
    p.mem = mem;
    for (int d = 0; d < 3; ++d) p.rank_period[d] = rank_period[d];
    p.laser_polarization = laser_polarization;
    p.Pi = Pi;
    p.omega = omega;
    p.l0 = l0;
    p.Lx = Lx;
    p.dx = dx;
    p.dy = dy;
    p.dz = dz;
    p.dt = dt;
    p.dt_half = dt_half;
    p.laser_amplitude = laser_amplitude;
    p.laser_pulse_duration = laser_pulse_duration;
    p.laser_start_time = laser_start_time;
    p.waist = waist;
    p.xfocus = xfocus;
    p.yfocus = yfocus;
    p.zfocus = zfocus;
    p.phase = phase;
    p.E_schwinger = E_schwinger;
    // the two species of main.cpp:68-73
    p.charge[0] = q_e;
    p.mass[0] = m_e;
    p.charge[1] = -q_e;
    p.mass[1] = 1836.0 * m_e;
    p.spin = 1;
    if (const char *s = std::getenv("PIC3D_GPU_PRECISION")) p.precision = std::atoi(s);
    const char *dev = std::getenv("PIC3D_GPU_DEVICE");
    const char *lazy = std::getenv("PIC3D_SHIM_LAZY");
    g_lazy = lazy && std::atoi(lazy) != 0;
    int r = pic_create(&p, dev ? std::atoi(dev) : 0, &g_ctx);
    if (r != PIC_OK) {
        std::fprintf(stderr, "pic3d_b200: initialize_domain: pic_create failed (status %d)\n", r);
        std::exit(1);
    }
    g_host_dirty = true;
    g_uploaded[0] = g_uploaded[1] = false;
    g_owner[0] = g_owner[1] = nullptr;
    g_gtab_sent.clear();
}

void free_memory() {
    double ****fld[6] = {&ex, &ey, &ez, &bx, &by, &bz};
    for (auto f : fld) {
        free_dtensor3(*f, nc_zst_out, nc_yst_out, nc_xst_out);
        *f = nullptr;
    }
    double ****ring[10] = {&jx, &jy, &jz, &rho_local, &current_recv_xminus, &current_recv_xplus,
                           &current_recv_yminus, &current_recv_yplus, &current_recv_zminus, &current_recv_zplus};
    for (auto r : ring) {
        free_dtensor3(*r, nc_zst_out - 1, nc_yst_out - 1, nc_xst_out - 1);
        *r = nullptr;
    }
    free_dtensor4(rho_particle, 0, nc_zst_out - 1, nc_yst_out - 1, nc_xst_out - 1);
    rho_particle = nullptr;
    if (g_ctx) pic_destroy(g_ctx);
    g_ctx = nullptr;
}

// ---------------------------------------------------------------------------
// particle set-up (src/particle.cpp:50-111): a lattice of
// (n * cbrt(cell_per_particles)) points per axis at the centres of equal
// sub-intervals of [xst, xend), z outermost; weight density / ppc; points
// with weight <= 0 are skipped; id = rank * (cells * ppc) + index.  Host
// code: it runs once, before the per-step path, and the records go to the
// device at the first push.
void initialize_particles(std::vector<particle> &particles, int &num_particles,
                          double density_func(double, double, double), double charge, double mass,
                          double initial_px, double initial_py, double initial_pz, double initial_sx,
                          double initial_sy, double initial_sz, int my_rank) {
    const int capacity = local_xcells * local_ycells * local_zcells * cell_per_particles;
    const double per_axis = std::cbrt((double)cell_per_particles);
    const int nx = (int)(local_xcells * per_axis), ny = (int)(local_ycells * per_axis),
              nz = (int)(local_zcells * per_axis);
    const double hx = (xend - xst) / nx, hy = (yend - yst) / ny, hz = (zend - zst) / nz;
    const double gamma0 = std::sqrt(1 + (initial_px * initial_px + initial_py * initial_py +
                                         initial_pz * initial_pz));
    particles.resize((size_t)capacity);
    int count = 0;
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx && count < capacity; ++i) {
                const double x = xst + i * hx + hx / 2.0, y = yst + j * hy + hy / 2.0, z = zst + k * hz + hz / 2.0;
                const double w = density_func(x, y, z) / cell_per_particles;
                if (w <= 0.0) continue;
                particle &p = particles[(size_t)count];
                p.id = my_rank * capacity + count;
                p.x = x;
                p.y = y;
                p.z = z;
                p.px = initial_px;
                p.py = initial_py;
                p.pz = initial_pz;
                p.sx = initial_sx;
                p.sy = initial_sy;
                p.sz = initial_sz;
                p.gamma = gamma0;
                p.charge = charge;
                p.mass = mass;
                p.weight = w;
                p.rank = my_rank;
                ++count;
            }
    particles.resize((size_t)count);
    num_particles = count;
}

// ---------------------------------------------------------------------------
// per-step calls

void update_electromagnetic_fields(int, int, MPI_Comm) {
    check(pic_update_fields_full(ready("update_electromagnetic_fields")), "update_electromagnetic_fields");
    pull_arrays(kE | kB);
}

void update_electromagnetic_fields_first(int, int, MPI_Comm) {
    check(pic_update_fields_first(ready("update_electromagnetic_fields_first")),
          "update_electromagnetic_fields_first");
    pull_arrays(kE | kB);
}

void update_electromagnetic_fields_second(int, int, MPI_Comm) {
    check(pic_update_fields_second(ready("update_electromagnetic_fields_second")),
          "update_electromagnetic_fields_second");
    pull_arrays(kE | kB);
}

void radiating_boundary(int, int is_left, int is_right, int, int step) {
    check(pic_radiating_boundary(ready("radiating_boundary"), is_left, is_right, step), "radiating_boundary");
    pull_arrays(kB);
}

void clear_currents() {
    check(pic_clear_currents(ready("clear_currents")), "clear_currents");
    if (g_lazy) return;
    for (int i = PIC_JX; i <= PIC_RHO1; ++i) std::memset(host_base(i), 0, sizeof(double) * host_len(i));
}

void update_particle_position_momentum(std::vector<particle> &particles, int num_particles, int, int kind) {
    pic_ctx *c = ready("update_particle_position_momentum");
    if (kind < 0 || kind > 1) die("update_particle_position_momentum", "species index must be 0 or 1");
    if (!g_uploaded[kind]) upload_species(kind, particles, num_particles);
    check(pic_update_particles(c, kind), "update_particle_position_momentum");
    check(pic_synchronize(c), "update_particle_position_momentum");
    pull_arrays(kJ | (kind ? kRho1 : kRho0));
    if (!g_lazy) {
        int n = 0;
        pull_species(kind, particles, n);
    }
}

void exchange_particle_data(std::vector<particle> &particles, int &num_particles, int, MPI_Comm) {
    pic_ctx *c = ready("exchange_particle_data");
    // the call names no species: it is the one pushed from this vector
    int kind = -1;
    for (int k = 0; k < 2; ++k)
        if (g_uploaded[k] && g_owner[k] == &particles) kind = k;
    if (kind < 0) die("exchange_particle_data", "vector was not pushed by update_particle_position_momentum");
    check(pic_exchange_particles(c, kind), "exchange_particle_data");
    int64_t n = 0;
    check(pic_num_particles(c, kind, &n), "exchange_particle_data");
    num_particles = (int)n;
    if (!g_lazy) pull_species(kind, particles, num_particles);
}

void exchange_currents(MPI_Comm) {
    check(pic_exchange_currents(ready("exchange_currents")), "exchange_currents");
    pull_arrays(kJ | kRho0 | kRho1);
}

void exchange_boundary_data(double ***data, MPI_Comm) {
    pic_ctx *c = ready("exchange_boundary_data");
    const int id = array_id(data);
    if (id < PIC_EX || id > PIC_BZ) die("exchange_boundary_data", "array is not one of ex..bz");
    check(pic_exchange_boundary(c, id), "exchange_boundary_data");
    pull_arrays(1u << id);
}

void exchange_boundary_current_fixed(double ***data, MPI_Comm) {
    pic_ctx *c = ready("exchange_boundary_current_fixed");
    const int id = array_id(data);
    if (id < PIC_JX) die("exchange_boundary_current_fixed", "array is not one of jx, jy, jz, rho_particle[k]");
    check(pic_exchange_current(c, id), "exchange_boundary_current_fixed");
    pull_arrays(1u << id);
}

void filter_field(double ***data) {
    pic_ctx *c = ready("filter_field");
    const int id = array_id(data);
    if (id < PIC_JX) die("filter_field", "array is not one of jx, jy, jz, rho_particle[k]");
    check(pic_filter_current(c, id), "filter_field");
    pull_arrays(1u << id);
}

void binomial_filter_currents() {
    check(pic_binomial_filter_currents(ready("binomial_filter_currents")), "binomial_filter_currents");
    pull_arrays(kJ);
}

void currents_particle(const particle &p, int kind) {
    pic_ctx *c = ready("currents_particle");
    if (kind < 0 || kind > 1) die("currents_particle", "species index must be 0 or 1");
    check(pic_deposit_particle(c, kind, &p), "currents_particle");
    pull_arrays(kJ | (kind ? kRho1 : kRho0));
}

// the reference's scalar helpers, evaluated by the device code the kernels use

void shape_function_2(double x, double *Interpolation) {
    check(pic_eval(ctx("shape_function_2"), PIC_EVAL_SHAPE2, &x, 1, Interpolation, 3), "shape_function_2");
}

void shape_function_4(double x, double *Interpolation) {
    check(pic_eval(ctx("shape_function_4"), PIC_EVAL_SHAPE4, &x, 1, Interpolation, 5), "shape_function_4");
}

double g_factor(double x) {
    double g = 0.0;
    int r = pic_eval(ready("g_factor"), PIC_EVAL_G_FACTOR, &x, 1, &g, 1);
    if (r == PIC_ERANGE) {
        std::printf("Error: x value out of g_data range! x = %.2f\n", x);
        std::exit(1);
    }
    check(r, "g_factor");
    return g;
}

double generate_laser_pulse(double time, double position) {
    const double in[2] = {time, position};
    double out = 0.0;
    check(pic_eval(ctx("generate_laser_pulse"), PIC_EVAL_LASER_PULSE, in, 2, &out, 1), "generate_laser_pulse");
    return out;
}

double Gpulse(double time, double x, double y, double z) {
    const double in[4] = {time, x, y, z};
    double out = 0.0;
    check(pic_eval(ctx("Gpulse"), PIC_EVAL_GPULSE, in, 4, &out, 1), "Gpulse");
    return out;
}

// ---------------------------------------------------------------------------
// the time loop (src/simulation.cpp:154-205), fused on the device between
// outputs: BC, first field half, clear, both pushes, removal, fold, second
// field half per step, with the step counter restarting at 1

void run_main_time_loop(std::vector<std::vector<particle>> &particles, int *num_particles, int my_rank,
                        int num_procs, hid_t plist_id, MPI_Comm my_comm) {
    pic_ctx *c = ready("run_main_time_loop");
    for (int k = 0; k < num_kind && k < 2; ++k)
        if (!g_uploaded[k]) upload_species(k, particles[k], num_particles[k]);
    check(pic_set_step(c, 0), "run_main_time_loop");
    int step = 0;
    while (step < timesteps) {
        int next = timesteps;
        if (output_interval > 0) next = std::min(timesteps, (step / output_interval + 1) * output_interval);
        check(pic_run_steps(c, next - step), "run_main_time_loop");
        step = next;
        if (output_interval > 0 && step % output_interval == 0) {
            const bool lazy = g_lazy;
            g_lazy = false;
            pull_arrays(kE | kB | kJ | kRho0 | kRho1);
            for (int k = 0; k < num_kind && k < 2; ++k) pull_species(k, particles[k], num_particles[k]);
            g_lazy = lazy;
            output_data_hdf5(step, my_rank, num_procs, my_comm, plist_id);
            output_particles_hdf5(step, my_rank, num_procs, my_comm, particles, num_particles);
        }
    }
    check(pic_synchronize(c), "run_main_time_loop");
    if (!g_lazy) {
        pull_arrays(kE | kB | kJ | kRho0 | kRho1);
        for (int k = 0; k < num_kind && k < 2; ++k) pull_species(k, particles[k], num_particles[k]);
    } else {
        for (int k = 0; k < num_kind && k < 2; ++k) {
            int64_t n = 0;
            check(pic_num_particles(c, k, &n), "run_main_time_loop");
            num_particles[k] = (int)n;
        }
    }
    if (my_rank == 0) std::printf("PIC simulation completed on the GPU: %d timesteps.\n", timesteps);
}
