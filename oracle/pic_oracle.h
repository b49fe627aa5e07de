/*
 * CPU oracle: a plain-C restatement of the reference PIC3D per-timestep loop
 * (one process, FP64).  TEST INFRASTRUCTURE ONLY — only tests/, the smoke
 * check and bench.py's CPU-baseline leg may load it; the GPU product never
 * calls it.
 *
 * Every function follows one reference function (file:line cited in
 * pic_oracle.c) with the same arithmetic in the same order, so that on the
 * same inputs it reproduces the reference build (oracle/_ref) bit for bit;
 * tests/test_oracle_pin.py checks this against the reference's own output.
 *
 * Array layout is the reference's: z-major, x fastest.
 *   field buffers ex..bz   : (n+2*mem)^3 points, buffer index 0..n+2mem-1
 *   ring buffers  jx..rho1 : (n+2*mem+2)^3 points, buffer index -1..n+2mem
 * Particles use the reference's 144-byte `particle` struct layout.
 */
#ifndef PIC3D_ORACLE_H
#define PIC3D_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_particle {
    int32_t id;
    int32_t pad0;
    double x, y, z;
    double x_old, y_old, z_old;
    double px, py, pz;
    double sx, sy, sz;
    double gamma, charge, mass, weight;
    int32_t rank;
    int32_t pad1;
} orc_particle;

typedef struct orc_state {
    /* parameters, named as in the reference src/constants.cpp */
    int32_t local_xcells, local_ycells, local_zcells, mem;
    int32_t rank_period[3];
    int32_t laser_polarization;
    double Pi, omega, l0, Lx;
    double dx, dy, dz, dt, dt_half;
    double laser_amplitude, laser_pulse_duration, laser_start_time;
    double waist, xfocus, yfocus, zfocus, phase;
    double E_schwinger;
    /* extensions beyond the reference (0 = reference behaviour) */
    int32_t laser_envelope;      /* 0: sine envelope (boundary.cpp:13), 1: Gaussian, FWHM = laser_pulse_duration */
    int32_t laser_profile;       /* 0: Gaussian beam (boundary.cpp:38), 1: bicubic amplitude grid */
    const double *profile_coef;  /* profile_n x profile_n coefficients over the physical y-z face */
    int32_t profile_n;
    int32_t absorbing;           /* 1: Silver-Mueller absorbing condition on the non-periodic y, z and x-max faces */
    int32_t g_data_size;
    const double *g_data;        /* g-factor table (reference g.txt), may be NULL when unused */
    /* arrays */
    double *ex, *ey, *ez, *bx, *by, *bz;
    double *jx, *jy, *jz, *rho0, *rho1;
    orc_particle *particles[2];
    int64_t num_particles[2];
    orc_particle *scratch;       /* capacity >= max(num_particles) */
    /* counters */
    int64_t out_of_bounds;       /* particles the reference reports as out of bounds (particle.cpp:123-130) */
    int64_t g_factor_errors;     /* g_factor arguments outside the table (particle.cpp:632-636) */
} orc_state;

void orc_shape_function_2(double x, double *w3);
void orc_shape_function_4(double x, double *w5);
double orc_g_factor(orc_state *s, double x);
double orc_gpulse(const orc_state *s, double time, double x, double y, double z);

void orc_radiating_boundary(orc_state *s, int is_left, int is_right, int step);
void orc_exchange_boundary_data(orc_state *s, double *a);
void orc_fields_first(orc_state *s);
void orc_fields_second(orc_state *s);
void orc_clear_currents(orc_state *s);
void orc_push(orc_state *s, int kind);
void orc_currents_particle(orc_state *s, const orc_particle *p, int kind);
void orc_exchange_particles(orc_state *s, int kind);
void orc_exchange_current(orc_state *s, double *a);
void orc_exchange_currents(orc_state *s);
void orc_initial(orc_state *s);
void orc_step(orc_state *s, int step);
void orc_run(orc_state *s, int first_step, int nsteps);

#ifdef __cplusplus
}
#endif

#endif
