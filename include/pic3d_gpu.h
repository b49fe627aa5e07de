/*
 * pic3d_gpu.h — C ABI of the B200 implementation of the PIC3D per-timestep
 * loop (Yee FDTD E/B half-updates, field gather + relativistic Boris push
 * with 2nd/4th-order shapes, Esirkepov current deposition, laser /
 * absorbing / periodic boundaries) on one GPU.
 *
 * Every entry point takes plain pointers and sizes and returns an int status
 * (PIC_OK = 0).  The text of the last error is pic_last_error(ctx).  A
 * context owns one CUDA stream on one device; calls on one context must be
 * serialised by the caller.  Kernels never trap: a device-side problem
 * (a particle outside the buffers, a NaN momentum, a g-factor argument
 * outside the table, a bin overflow) sets a bit of a device status word,
 * the offending particle is left unchanged, and the next call that
 * synchronises (pic_synchronize, any download) returns the matching code.
 *
 * Layout shared with the reference (include/field.h:11-24,
 * src/simulation.cpp:132-144): fields ex..bz are (n+2*mem)^3 buffers and
 * jx, jy, jz, rho_electron, rho_proton are (n+2*mem+2)^3 ring buffers, each
 * z-major with x fastest, exactly as the reference dtensor3 blocks.  Host
 * arrays passed to upload/download are always FP64 in that layout; an FP32
 * context converts on the device.  Particles cross the ABI as the
 * reference's 144-byte `struct particle` (include/particle.h:9-29).
 */
#ifndef PIC3D_GPU_H
#define PIC3D_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------- */
#define PIC_OK 0
#define PIC_EINVAL 1    /* bad argument or parameter combination */
#define PIC_ENOMEM 2    /* device or host allocation failed */
#define PIC_EOOB 3      /* a particle's stencil left the field buffers */
#define PIC_ENAN 4      /* a non-finite momentum or position appeared */
#define PIC_ETIMEOUT 5  /* a bounded device-side wait gave up */
#define PIC_ECUDA 6     /* a CUDA runtime error */
#define PIC_EOVERFLOW 7 /* a particle bin or buffer overflowed */
#define PIC_ERANGE 8    /* g_factor argument outside the table (src/particle.cpp:632-636) */
#define PIC_ENOCONV 9   /* an iterative solve stopped at its iteration limit before its tolerance */

/* ---- array identifiers for upload / download ------------------------ */
enum {
    PIC_EX = 0, PIC_EY, PIC_EZ, PIC_BX, PIC_BY, PIC_BZ, /* field buffers */
    PIC_JX, PIC_JY, PIC_JZ, PIC_RHO0, PIC_RHO1,          /* ring buffers (rho_particle[0], [1]) */
    PIC_NARRAYS
};

/* ---- run parameters --------------------------------------------------
 * Names follow the reference globals of src/constants.cpp:5-85
 * (declared in include/constants.h:9-99).  One GPU holds the whole domain,
 * so local_*cells are also the global_n* sizes.                          */
typedef struct PicParams {
    int32_t local_xcells, local_ycells, local_zcells;
    int32_t mem;               /* ghost width; 2 selects 2nd-order, 4 selects 4th-order shapes (particle.cpp:184-203) */
    int32_t rank_period[3];    /* 1: periodic pair of faces (constants.cpp:25), 0: absorbing / laser */
    int32_t laser_polarization;/* 1 S, 2 P, 3 both (constants.cpp:60) */
    double Pi, omega, l0, Lx;
    double dx, dy, dz, dt, dt_half;
    double laser_amplitude, laser_pulse_duration, laser_start_time;
    double waist, xfocus, yfocus, zfocus, phase;
    double E_schwinger;        /* spin precession (constants.cpp:83) */
    double charge[2], mass[2]; /* species 0 (electrons) and 1 (protons): main.cpp:71,73 */
    int64_t capacity[2];       /* particle capacity per species (0: sized at first upload) */
    int32_t precision;         /* 64: FP64 everywhere; 32: FP32 fields/momenta/current, int32 cell + FP32 offsets */
    int32_t spin;              /* 1: electron spin precession (particle.cpp:318-368); 0: skipped */
    int32_t deposit_rho;       /* 1: per-species rho at the new positions every step (particle.cpp:503-514) */
    int32_t laser_envelope;    /* extension: 0 sine envelope (boundary.cpp:13), 1 Gaussian with intensity FWHM laser_pulse_duration */
    int32_t laser_profile;     /* extension: 0 Gaussian beam (boundary.cpp:38), 1 cubic-B-spline amplitude grid */
    int32_t tile;              /* edge of the shared-memory particle tile in cells (0: default 4, <0: no tiling) */
    int32_t sort_interval;     /* pushes between full counting sorts of the particles by tile (0: default 4,
                                  1 in adjoint contexts); between sorts each push re-bins only the particles
                                  that changed tile */
    int32_t adjoint;           /* 1: adjoint-capable context (stable particle order, removal marks particles dead;
                                  absorbing faces only); see pic_adjoint_* */
    int32_t absorbing;         /* extension: 1 = Silver-Mueller absorbing condition on every non-periodic face
                                  besides x-min (y and z faces, x-max), applied once per step with
                                  pic_radiating_boundary; the reference's x-max write (boundary.cpp:92-96) is
                                  then skipped.  0: reference faces (y / z ghosts stay zero, conductor-like) */
} PicParams;

typedef struct pic_ctx pic_ctx;

/* Fill *p with the defaults of a 4th-order FP64 run with no laser. */
void pic_default_params(PicParams *p);

/* Create a context on `device` (initialize_domain, src/simulation.cpp:23-152:
 * allocates and zeroes the field and ring buffers). */
int pic_create(const PicParams *p, int device, pic_ctx **out);
int pic_destroy(pic_ctx *ctx);
const char *pic_last_error(const pic_ctx *ctx);

/* Number of points of array `which` (field or ring buffer). */
int pic_array_len(const pic_ctx *ctx, int which, int64_t *n);

/* Host FP64 array in the reference layout <-> device. */
int pic_upload_array(pic_ctx *ctx, int which, const double *host);
int pic_download_array(pic_ctx *ctx, int which, double *host);

/* Particles of species `kind` as reference 144-byte records (particle.h:9-29).
 * Upload replaces the species' particles; every record must carry the
 * species' charge and mass and a finite weight (PIC_EINVAL otherwise), a
 * finite position and momentum (PIC_ENAN) and, in an FP32 context, a
 * position whose cell lies in -1 .. n along every absorbing axis (PIC_EOOB:
 * the packed cell index cannot hold it).  The checks run on the device while
 * converting; a bad record leaves the species empty.
 * Both directions stream through pinned host buffers owned by the context,
 * the host copy of one chunk overlapping the transfer of the next; the
 * caller's buffer may be ordinary (pageable) memory.  Download writes at most `cap` records and the
 * count to *n; order is the device order (records keep their id), gamma is
 * recomputed from the momentum as the push does (particle.cpp:309-311) and
 * x_old..z_old are the positions before the last push (particle.cpp:267-269). */
int pic_upload_particles(pic_ctx *ctx, int kind, const void *records, int64_t n);
int pic_download_particles(pic_ctx *ctx, int kind, void *records, int64_t cap, int64_t *n);
int pic_num_particles(pic_ctx *ctx, int kind, int64_t *n);

/* g-factor table (the reference's g.txt, loaded by load_g_data,
 * src/constants.cpp:114-136); needed only when spin precession meets
 * chi >= 0.005. */
int pic_set_g_table(pic_ctx *ctx, const double *g, int n);

/* Extension: profile_n x profile_n transverse amplitude coefficients
 * (row-major z, y) used when laser_profile = 1. */
int pic_set_laser_profile(pic_ctx *ctx, const double *coef, int profile_n);

/* ---- the reference call surface ------------------------------------- */
/* radiating_boundary(my_rank, is_left, is_right, num_procs, step): src/boundary.cpp:42-99 */
int pic_radiating_boundary(pic_ctx *ctx, int is_left, int is_right, int step);
/* update_electromagnetic_fields_first(...): src/field.cpp:56-86 (with exchange_boundary_data, src/mpi_utils.cpp:9-60) */
int pic_update_fields_first(pic_ctx *ctx);
/* update_electromagnetic_fields_second(...): src/field.cpp:88-117 */
int pic_update_fields_second(pic_ctx *ctx);
/* clear_currents(): src/particle.cpp:576-592 */
int pic_clear_currents(pic_ctx *ctx);
/* update_particle_position_momentum(particles, n, rank, kind): src/particle.cpp:113-370,
 * including currents_particle (src/particle.cpp:372-515) for every particle */
int pic_update_particles(pic_ctx *ctx, int kind);
/* exchange_particle_data(particles, n, rank, comm): src/mpi_utils.cpp:62-230 —
 * on one GPU: removal at non-periodic global faces */
int pic_exchange_particles(pic_ctx *ctx, int kind);
/* exchange_currents(comm): src/particle.cpp:594-601 (exchange_boundary_current_fixed,
 * src/mpi_utils.cpp:232-417) — periodic fold of J and rho */
int pic_exchange_currents(pic_ctx *ctx);
/* the t = 0 push + exchange of main.cpp:75-79 */
int pic_initial_push(pic_ctx *ctx);
/* `nsteps` iterations of run_main_time_loop (src/simulation.cpp:159-183);
 * the 1-based step counter continues from the last call */
int pic_run_steps(pic_ctx *ctx, int nsteps);
int pic_get_step(const pic_ctx *ctx, int *step);
int pic_set_step(pic_ctx *ctx, int step);

/* ---- the rest of the reference's per-step call surface ---------------- */
/* update_electromagnetic_fields (src/field.cpp:24-54): both curls with the
 * full dt, E then B, each followed by its halo (unused by the reference's
 * own loop) */
int pic_update_fields_full(pic_ctx *ctx);
/* exchange_boundary_data(data) (src/mpi_utils.cpp:9-60) on one field array
 * (PIC_EX..PIC_BZ): the periodic ghost fill */
int pic_exchange_boundary(pic_ctx *ctx, int array);
/* exchange_boundary_current_fixed(data) (src/mpi_utils.cpp:232-417) on one
 * ring array (PIC_JX..PIC_RHO1): the periodic fold */
int pic_exchange_current(pic_ctx *ctx, int array);
/* filter_field(data) (src/particle.cpp:520-567) on one ring array: one
 * binomial (1/4, 1/2, 1/4) pass along x, then y, then z over the physical
 * points */
int pic_filter_current(pic_ctx *ctx, int array);
/* binomial_filter_currents() (src/particle.cpp:569-574): jx, jy, jz */
int pic_binomial_filter_currents(pic_ctx *ctx);
/* currents_particle(p, kind) (src/particle.cpp:372-515) for one 144-byte
 * record: its move from (x_old, y_old, z_old) to (x, y, z) deposited into J
 * and rho_particle[kind]; a move of more than one cell is PIC_EOOB */
int pic_deposit_particle(pic_ctx *ctx, int kind, const void *record);
/* Device evaluation of the reference's scalar helpers with the kernels' own
 * code:
 *   PIC_EVAL_SHAPE2       shape_function_2(x)       in[1]  out[3]  (src/particle.cpp:8-19)
 *   PIC_EVAL_SHAPE4       shape_function_4(x)       in[1]  out[5]  (src/particle.cpp:21-48)
 *   PIC_EVAL_G_FACTOR     g_factor(x)               in[1]  out[1]  (src/particle.cpp:603-637;
 *                         outside the table: PIC_ERANGE)
 *   PIC_EVAL_LASER_PULSE  generate_laser_pulse(t,x) in[2]  out[1]  (src/boundary.cpp:8-27)
 *   PIC_EVAL_GPULSE       Gpulse(t,x,y,z)           in[4]  out[1]  (src/boundary.cpp:29-40) */
enum {
    PIC_EVAL_SHAPE2 = 0,
    PIC_EVAL_SHAPE4 = 1,
    PIC_EVAL_G_FACTOR = 2,
    PIC_EVAL_LASER_PULSE = 3,
    PIC_EVAL_GPULSE = 4
};
int pic_eval(pic_ctx *ctx, int what, const double *in, int nin, double *out, int nout);

/* Wait for the context's stream and report any device-side status. */
int pic_synchronize(pic_ctx *ctx);
/* The context's cudaStream_t (as void*), for callers that time or order work. */
int pic_get_stream(const pic_ctx *ctx, void **stream);

/* ---- diagnostics (FP64 device reductions, no reference counterpart) ---
 * out[0] field energy 1/2 sum(E^2+B^2) dV over physical cells
 * out[1] kinetic energy species 0, out[2] species 1: sum w m (gamma-1)
 * out[3] total charge species 0, out[4] species 1 (sum of rho over physical cells times dV)
 * out[5] max |div E - (rho0+rho1)| over physical nodes (Gauss residual) */
#define PIC_NDIAG 6
int pic_diagnostics(pic_ctx *ctx, double *out, int n);

/* ---- device-side particle loaders ------------------------------------
 * Both replace the species' particles like pic_upload_particles, without
 * host particle memory.
 *
 * pic_initialize_particles: initialize_particles (src/particle.cpp:50-111,
 * declared include/particle.h:32-37) on the device: cbrt(cell_per_particles)
 * lattice points per cell and axis at xst + i*norm + norm/2 (cell units),
 * weight density(x*dx, y*dy, z*dz) / cell_per_particles, points with weight
 * <= 0 skipped, ids 0.. in k, j, i order, momenta initial_p[3], spins
 * initial_s[3], x_old = 0, the species' charge and mass.  The density
 * function is data instead of a host callback: a uniform value, a box
 * (src/constants.cpp:87-101 is the box 5 l0 < x_phys <= 15 l0 on every axis
 * with value `density`), or a piecewise-linear profile in physical x.      */
enum { PIC_DENSITY_UNIFORM = 0, PIC_DENSITY_BOX = 1, PIC_DENSITY_XPROFILE = 2 };
typedef struct PicDensity {
    int32_t kind;            /* PIC_DENSITY_* */
    int32_t nknots;          /* XPROFILE: number of knots */
    double value;            /* UNIFORM / BOX: the density */
    double lo[3], hi[3];     /* BOX: `value` where lo[d] < coordinate_d * d_d <= hi[d] on every axis, else 0 */
    const double *knot_x;    /* XPROFILE: ascending physical x of the knots (host memory) */
    const double *knot_v;    /* XPROFILE: density at the knots; linear between, end values beyond */
} PicDensity;
int pic_initialize_particles(pic_ctx *ctx, int kind, const PicDensity *density, int cell_per_particles,
                             const double *initial_p, const double *initial_s);

/* pic_generate_thermal (no counterpart in the reference, whose loader is
 * the lattice above): a seeded thermal plasma, ppc particles per cell at
 * uniform random positions in the cell, momenta N(0, u_th^2) per component,
 * weight density / ppc, zero spins, ids 0.. in cell order (x fastest).
 * Counter-based (Philox4x32-10 keyed by seed and kind): the same seed gives
 * the same particles on any device and in any chunking.                   */
int pic_generate_thermal(pic_ctx *ctx, int kind, int ppc, double density, double u_th, uint64_t seed);

/* ---- initial electrostatic field (no counterpart in the reference) ----
 * The reference starts from E = 0 whatever the particles' charge.  This
 * solves, in FP64 whatever the context precision, A phi = rho - <rho> with
 * A the 7-point Laplacian of the Yee grid, and sets E = -grad phi on the
 * faces, Ex(i+1/2) = -(phi(i+1) - phi(i)) / dx (and Ey, Ez), so that the
 * discrete divergence pic_diagnostics uses equals rho - <rho>.  rho is the
 * charge density of both species deposited at the current particle
 * positions with the push's rho shape (src/particle.cpp:503-514) onto the
 * physical nodes; <rho> is its mean (a uniform neutralising background).
 * Periodic axes wrap; absorbing axes have E = 0 on the faces outside the
 * physical nodes (zero flux).  B, J, rho arrays and particles are not
 * touched.  Conjugate gradients run until ||b - A phi|| <= rel_tol ||b||
 * or max_iter iterations (PIC_ENOCONV, with E set from the last iterate).
 * out[0] iterations, out[1] final relative residual, out[2] <rho>,
 * out[3] max |div E - (rho - <rho>)| over the physical nodes, evaluated
 * from E as stored (FP32 contexts: after rounding E to FP32). */
#define PIC_NPOISSON 4
int pic_solve_initial_field(pic_ctx *ctx, double rel_tol, int max_iter, double *out, int nout);

/* ---- diagnostics without device allocation (no reference counterpart) --
 * For callers that cannot let a library call cudaMalloc (a host code that
 * reserves nearly all of HBM for its own arrays, or that allows device
 * memory only through its own pool; cudaMalloc / cudaFree would fail or
 * synchronise the device).  Needs no context: reads caller-owned FP64 device
 * arrays in the reference layout (rho0 / rho1 may be NULL) for the grid that
 * p->local_*cells, p->mem and p->dx.. describe, and writes 4 doubles to the
 * caller-owned device array `out`, stream-ordered on `stream`:
 * out[0] field energy, out[1] charge of species 0, out[2] charge of species 1,
 * out[3] max |div E - rho0 - rho1| — the same quantities as pic_diagnostics
 * out[0], out[3], out[4], out[5].  Its only scratch is a static device array
 * of one slot per z plane: grids with more than 2048 z planes are rejected
 * with PIC_EINVAL.  The first call on each device looks up that array's
 * address (no allocation); make it before capturing work on the device into
 * a stream.  All calls share the array: calls that overlap on the GPU race. */
int pic_field_diagnostics_noalloc(const PicParams *p, const double *ex, const double *ey, const double *ez,
                                  const double *bx, const double *by, const double *bz, const double *rho0,
                                  const double *rho1, double *out, void *stream);

/* ---- adjoint (no counterpart in the reference) ------------------------
 * Gradients of a final-state objective with respect to the particle weights
 * (hence a density profile) and the laser amplitude coefficients
 * (laser_profile = 1), by a hand-written adjoint of the per-step loop.
 * Needs a context created with PicParams.adjoint = 1 (absorbing faces,
 * stable particle order).  Usage, segment by segment from the last:
 *   pic_checkpoint_save/restore   device copies of the whole state
 *   pic_adjoint_tape(n) + pic_adjoint_record(1), then pic_initial_push /
 *   pic_run_steps re-run a segment recording each push's inputs
 *   pic_adjoint_seed_kinetic      objective = sum s(x) w m (gamma-1) over
 *                                 one species' particles at the current
 *                                 state, s = 1 inside [xlo, xhi), 0 outside,
 *                                 sin^2 ramps `ramp` cells wide at both
 *                                 ends (ramp 0: hard edges, not smooth in
 *                                 x); zeroes all adjoints
 *   pic_adjoint_backward(n)       n recorded steps in reverse
 *   pic_adjoint_weight_grad       d objective / d weight, per particle in
 *                                 upload order
 *   pic_adjoint_profile_grad      d objective / d laser coefficient */
int pic_checkpoint_save(pic_ctx *ctx, int slot);
int pic_checkpoint_restore(pic_ctx *ctx, int slot);
int pic_adjoint_tape(pic_ctx *ctx, int nsteps);
int pic_adjoint_record(pic_ctx *ctx, int on);
int pic_adjoint_seed_kinetic(pic_ctx *ctx, int kind, double xlo, double xhi, double ramp, double *objective);
int pic_adjoint_backward(pic_ctx *ctx, int nsteps);
int pic_adjoint_weight_grad(pic_ctx *ctx, int kind, double *grad, int64_t n);
int pic_adjoint_profile_grad(pic_ctx *ctx, double *grad, int n);
int pic_adjoint_release(pic_ctx *ctx);

/* ---- per-kernel timing with CUDA events (off by default) ------------- */
int pic_profile_enable(pic_ctx *ctx, int on);
/* names[i] (static strings), total_ms[i] and launches[i] for up to cap kernels */
int pic_profile_read(pic_ctx *ctx, const char **names, double *total_ms, int64_t *launches, int cap, int *count);
int pic_profile_reset(pic_ctx *ctx);

/* ---- particle order (tiled kernel) ------------------------------------
 * out[0]: particles in the visitor lists the next push reads (away from
 *         their tile's slice of the sorted arrays, pushed from the list of
 *         the tile they are in);
 * out[1]: 1 if the next push takes the particles away from home from those
 *         lists (they are complete and, in FP64, name at least 3 % of the
 *         species; else the global kernel pushes them after the tiles);
 * out[2]: pushes since the last full counting sort;
 * out[3]: particles the last push handed to the global-memory kernel.
 * Synchronises the context's stream.                                     */
int pic_particle_order_stats(pic_ctx *ctx, int kind, int64_t *out, int n);

/* ---- checkpoint of the whole state (fields, currents, particles, step) */
int pic_save(pic_ctx *ctx, const char *path);
int pic_load(pic_ctx *ctx, const char *path);

#ifdef __cplusplus
}
#endif

#endif /* PIC3D_GPU_H */
