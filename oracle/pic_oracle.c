/*
 * CPU oracle for the PIC3D per-timestep loop — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference algorithm (one process, FP64) used
 * by the tests and the CPU-baseline leg of bench.py to check the GPU path.
 * Each function names the reference function it follows (file:line in the
 * reference project).  Expressions keep the reference's operation order so
 * that results match the reference build bit for bit; the reference itself
 * loops over double*** views, this file uses flat index arithmetic.
 */
#include "pic_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ */
/* geometry (src/simulation.cpp:23-75 for one rank at Cartesian coords 0)
 *   physical cells      nc_st = mem .. nc_end = n + mem - 1
 *   field buffer        0 .. n + 2 mem - 1
 *   J / rho ring buffer -1 .. n + 2 mem
 *   particle coordinate x in [0, n) maps to buffer x - (1 - mem)          */

typedef struct {
    int n[3], fx, fy, fz, rx, ry, rz, nc_st[3], nc_end[3], nc_new[3];
    long fsz, rsz;
} geom;

static geom make_geom(const orc_state *s) {
    geom g;
    g.n[0] = s->local_xcells;
    g.n[1] = s->local_ycells;
    g.n[2] = s->local_zcells;
    for (int d = 0; d < 3; ++d) {
        g.nc_st[d] = s->mem;
        g.nc_end[d] = g.n[d] + s->mem - 1;
        g.nc_new[d] = 1 - s->mem;
    }
    g.fx = g.n[0] + 2 * s->mem;
    g.fy = g.n[1] + 2 * s->mem;
    g.fz = g.n[2] + 2 * s->mem;
    g.rx = g.fx + 2;
    g.ry = g.fy + 2;
    g.rz = g.fz + 2;
    g.fsz = (long)g.fx * g.fy * g.fz;
    g.rsz = (long)g.rx * g.ry * g.rz;
    return g;
}

/* field buffer index, k/j/i in 0..n+2mem-1 */
#define FI(g, k, j, i) (((long)(k) * (g).fy + (j)) * (g).fx + (i))
/* ring buffer index, k/j/i in -1..n+2mem */
#define RI(g, k, j, i) (((long)((k) + 1) * (g).ry + ((j) + 1)) * (g).rx + ((i) + 1))

static int neighbour(const orc_state *s, int d) { return s->rank_period[d] ? 0 : -2; }

/* ------------------------------------------------------------------ */
/* shape functions: src/particle.cpp:8-19 (3-point quadratic B-spline) and
 * :21-48 (5-point quartic), coefficients src/constants.cpp:84-85        */

static const double A0 = 55.0 / 96.0, A1 = 5.0 / 24.0, A2 = 5.0 / 4.0, A3 = 5.0 / 6.0;
static const double B0 = 115.0 / 192.0, B2 = 5.0 / 8.0;

void orc_shape_function_2(double x, double *w) {
    int ic = (int)(x + 0.5);
    double d = x - (double)ic;
    w[0] = 0.5 * (0.5 - d) * (0.5 - d);
    w[1] = 0.75 - d * d;
    w[2] = 0.5 * (0.5 + d) * (0.5 + d);
}

void orc_shape_function_4(double x, double *w) {
    int ii = (int)(x + 0.5);
    double d = x - (ii - 2);
    double u, u2;
    u = d - 2.5;
    u2 = u * u;
    w[0] = u2 * u2 / 24.0;
    u = d - 1.0;
    u2 = u * u;
    w[1] = -u2 * u2 / 6.0 + u2 * u * A3 - u2 * A2 + u * A1 + A0;
    u = d - 2.0;
    u2 = u * u;
    w[2] = u2 * u2 / 4.0 - u2 * B2 + B0;
    u = d - 3.0;
    u2 = u * u;
    w[3] = -u2 * u2 / 6.0 - u2 * u * A3 - u2 * A2 - u * A1 + A0;
    u = d - 1.5;
    u2 = u * u;
    w[4] = u2 * u2 / 24.0;
}

static void shape(const orc_state *s, double x, double *w) {
    if (s->mem == 2)
        orc_shape_function_2(x, w);
    else
        orc_shape_function_4(x, w);
}

/* g-factor lookup: src/particle.cpp:603-637 (piecewise-uniform table) */
double orc_g_factor(orc_state *s, double x) {
    int idx;
    if (x < 0.005 && x >= 0.0) return 2.003219;
    if (x >= 0.005 && x < 0.01)
        idx = (int)((x - 0.005) / 0.0001);
    else if (x >= 0.01 && x < 1)
        idx = (int)((x - 0.01) / 0.01) + 50;
    else if (x >= 1 && x < 10)
        idx = (int)((x - 1.0) / 0.01) + 150;
    else if (x >= 10 && x < 20)
        idx = (int)((x - 10.0) / 0.01) + 1050;
    else if (x >= 20 && x <= 100)
        idx = (int)((x - 20.0) / 0.1) + 2050;
    else {
        /* the reference prints and exit(1)s here */
        s->g_factor_errors++;
        return 2.003219;
    }
    if (!s->g_data || idx < 0 || idx >= s->g_data_size) {
        s->g_factor_errors++;
        return 2.003219;
    }
    return s->g_data[idx];
}

/* ------------------------------------------------------------------ */
/* laser source: src/boundary.cpp:8-27 (generate_laser_pulse) and :29-40
 * (Gpulse).  laser_envelope / laser_profile select extensions.          */

static double envelope(const orc_state *s, double time, double position) {
    double t = time - position - s->laser_start_time;
    if (s->laser_envelope == 1) {
        /* extension: Gaussian in amplitude whose intensity FWHM is
         * laser_pulse_duration, centred 1.5 durations after the start */
        double tau = s->laser_pulse_duration;
        if (t < 0.0 || t > 3.0 * tau) return 0.0;
        double r = (t - 1.5 * tau) / tau;
        return s->laser_amplitude * exp(-2.0 * log(2.0) * r * r);
    }
    double env = 0.0;
    if (t >= 0.0 && t <= 1.0 * s->laser_pulse_duration) env = sin(s->Pi * t / s->laser_pulse_duration);
    return s->laser_amplitude * env;
}

/* cubic B-spline basis, support |t| < 2 */
static double bspline3(double t) {
    double a = fabs(t);
    if (a < 1.0) return (4.0 - 6.0 * a * a + 3.0 * a * a * a) / 6.0;
    if (a < 2.0) {
        double b = 2.0 - a;
        return b * b * b / 6.0;
    }
    return 0.0;
}

/* extension: transverse amplitude from a profile_n x profile_n grid of
 * cubic-B-spline coefficients spanning the physical y-z face.  iy, iz are
 * buffer indices of the face row (the same indices the reference uses). */
static double profile_amplitude(const orc_state *s, int iy, int iz) {
    int nc = s->profile_n;
    double u = ((double)(iy - s->mem) + 0.5) / (double)s->local_ycells * (double)(nc - 1);
    double v = ((double)(iz - s->mem) + 0.5) / (double)s->local_zcells * (double)(nc - 1);
    double a = 0.0;
    for (int b = 0; b < nc; ++b) {
        double wv = bspline3(v - b);
        if (wv == 0.0) continue;
        for (int c = 0; c < nc; ++c) {
            double wu = bspline3(u - c);
            if (wu == 0.0) continue;
            a += s->profile_coef[b * nc + c] * wu * wv;
        }
    }
    return a;
}

double orc_gpulse(const orc_state *s, double time, double x, double y, double z) {
    double k = 2.0 * s->Pi / s->l0;
    double rl = 0.5 * k * s->waist * s->waist;
    double xe = x - s->xfocus;
    double ph = atan(xe / rl);
    double w = s->waist * sqrt(1 + pow(xe / rl, 2));
    double PHI = (xe / rl) * (y * y + z * z) / w / w - ph + k * xe - s->omega * time;
    return -1.0 * envelope(s, time, x) * s->waist / w * exp(-(y * y + z * z) / (w * w)) * cos(PHI + s->phase);
}

static double gpulse_profile(const orc_state *s, double time, double x, double y, double z, int iy, int iz) {
    if (s->laser_profile != 1) return orc_gpulse(s, time, x, y, z);
    double k = 2.0 * s->Pi / s->l0;
    double rl = 0.5 * k * s->waist * s->waist;
    double xe = x - s->xfocus;
    double ph = atan(xe / rl);
    double w = s->waist * sqrt(1 + pow(xe / rl, 2));
    double PHI = (xe / rl) * (y * y + z * z) / w / w - ph + k * xe - s->omega * time;
    return -1.0 * envelope(s, time, x) * profile_amplitude(s, iy, iz) * cos(PHI + s->phase);
}

/* radiating_boundary: src/boundary.cpp:42-99.  Silver-Mueller style update
 * of the B ghost column at x = mem-1 (laser source at x-min) and, when the
 * x-max face is not periodic, of column local_xcells+1 (boundary.cpp:92-96;
 * for mem > 1 that column lies inside the physical region). */
static void absorb_faces(orc_state *s);

void orc_radiating_boundary(orc_state *s, int is_left, int is_right, int step) {
    geom g = make_geom(s);
    double time = step * s->dt;
    double S_l = 0.0, P_l = 0.0, S_r = 0.0, P_r = 0.0;
    double alpha = 1 / (1 + s->dt / s->dx);
    double beta = 1 - s->dt / s->dx;
    const int m = s->mem, L = s->local_xcells;
    const double yst = 0.0, zst = 0.0;
    for (int j = g.nc_st[2]; j <= g.nc_end[2]; j++) {
        for (int i = g.nc_st[1]; i <= g.nc_end[1]; i++) {
            double y = (i + yst) * s->dy - s->yfocus;
            double z = (j + zst) * s->dz - s->zfocus;
            if (is_left) {
                if (s->laser_polarization == 1 || s->laser_polarization == 3) S_l = gpulse_profile(s, time, 0.0, y, z, i, j);
                if (s->laser_polarization == 2 || s->laser_polarization == 3) P_l = gpulse_profile(s, time, 0.0, y, z, i, j);
            }
            if (is_right) {
                if (s->laser_polarization == 1 || s->laser_polarization == 3) S_r = gpulse_profile(s, time, s->Lx, y, z, i, j);
                if (s->laser_polarization == 2 || s->laser_polarization == 3) P_r = gpulse_profile(s, time, s->Lx, y, z, i, j);
            }
            if (neighbour(s, 0) == -2) {
                s->bz[FI(g, j, i, m - 1)] =
                    alpha * (4 * S_l - 2 * s->ey[FI(g, j, i, m)] -
                             s->dt / s->dz * (s->bx[FI(g, j, i, m)] - s->bx[FI(g, j - 1, i, m)]) -
                             beta * s->bz[FI(g, j, i, m)] - s->dt * s->jy[RI(g, j, i, m)]);
                s->by[FI(g, j, i, m - 1)] =
                    alpha * (-4 * P_l + 2 * s->ez[FI(g, j, i, m)] +
                             s->dt / s->dy * (s->bx[FI(g, j, i, m)] - s->bx[FI(g, j, i - 1, m)]) -
                             beta * s->by[FI(g, j, i, m)] + s->dt * s->jz[RI(g, j, i, m)]);
            }
            if (neighbour(s, 0) == -2 && !s->absorbing) {
                s->bz[FI(g, j, i, L + 1)] =
                    alpha * (-4 * S_r + 2 * s->ey[FI(g, j, i, L)] -
                             s->dt / s->dz * (s->bx[FI(g, j, i, L)] - s->bx[FI(g, j - 1, i, L)]) -
                             beta * s->bz[FI(g, j, i, L)] + s->dt * s->jy[RI(g, j, i, L)]);
                s->by[FI(g, j, i, L + 1)] =
                    alpha * (4 * P_r - 2 * s->ez[FI(g, j, i, L)] +
                             s->dt / s->dy * (s->bx[FI(g, j, i, L)] - s->bx[FI(g, j, i - 1, L)]) -
                             beta * s->by[FI(g, j, i, L)] - s->dt * s->jz[RI(g, j, i, L)]);
            }
        }
    }
    absorb_faces(s);
}

/* ------------------------------------------------------------------ */
/* field halo: src/mpi_utils.cpp:9-60 on one rank.  A periodic dimension
 * copies its mem outermost physical planes into the opposite ghost planes
 * over the full extent of the other two dimensions; X, Y and Z complete in
 * that order.  Non-periodic faces are left untouched.                   */
void orc_exchange_boundary_data(orc_state *s, double *a) {
    geom g = make_geom(s);
    const int m = s->mem;
    if (neighbour(s, 0) != -2) {
        int n = g.n[0];
        for (int k = 0; k < g.fz; ++k)
            for (int j = 0; j < g.fy; ++j)
                for (int i = 0; i < m; ++i) {
                    a[FI(g, k, j, i)] = a[FI(g, k, j, n + i)];
                    a[FI(g, k, j, n + m + i)] = a[FI(g, k, j, m + i)];
                }
    }
    if (neighbour(s, 1) != -2) {
        int n = g.n[1];
        for (int k = 0; k < g.fz; ++k)
            for (int j = 0; j < m; ++j)
                for (int i = 0; i < g.fx; ++i) {
                    a[FI(g, k, n + m + j, i)] = a[FI(g, k, m + j, i)];
                    a[FI(g, k, j, i)] = a[FI(g, k, n + j, i)];
                }
    }
    if (neighbour(s, 2) != -2) {
        int n = g.n[2];
        for (int k = 0; k < m; ++k)
            for (int j = 0; j < g.fy; ++j)
                for (int i = 0; i < g.fx; ++i) {
                    a[FI(g, k, j, i)] = a[FI(g, n + k, j, i)];
                    a[FI(g, n + m + k, j, i)] = a[FI(g, m + k, j, i)];
                }
    }
}

/* E half-update over the physical cells: src/field.cpp:59-67 */
static void update_e(orc_state *s) {
    geom g = make_geom(s);
    const double h = s->dt_half;
    for (int k = g.nc_st[2]; k <= g.nc_end[2]; k++)
        for (int j = g.nc_st[1]; j <= g.nc_end[1]; j++)
            for (int i = g.nc_st[0]; i <= g.nc_end[0]; i++) {
                long c = FI(g, k, j, i);
                s->ex[c] += h * ((s->bz[c] - s->bz[FI(g, k, j - 1, i)]) / s->dy -
                                 (s->by[c] - s->by[FI(g, k - 1, j, i)]) / s->dz - s->jx[RI(g, k, j, i)]);
                s->ey[c] += h * ((s->bx[c] - s->bx[FI(g, k - 1, j, i)]) / s->dz -
                                 (s->bz[c] - s->bz[FI(g, k, j, i - 1)]) / s->dx - s->jy[RI(g, k, j, i)]);
                s->ez[c] += h * ((s->by[c] - s->by[FI(g, k, j, i - 1)]) / s->dx -
                                 (s->bx[c] - s->bx[FI(g, k, j - 1, i)]) / s->dy - s->jz[RI(g, k, j, i)]);
            }
    orc_exchange_boundary_data(s, s->ex);
    orc_exchange_boundary_data(s, s->ey);
    orc_exchange_boundary_data(s, s->ez);
}

/* B half-update over the physical cells: src/field.cpp:74-82 */
static void update_b(orc_state *s) {
    geom g = make_geom(s);
    const double h = s->dt_half;
    for (int k = g.nc_st[2]; k <= g.nc_end[2]; k++)
        for (int j = g.nc_st[1]; j <= g.nc_end[1]; j++)
            for (int i = g.nc_st[0]; i <= g.nc_end[0]; i++) {
                long c = FI(g, k, j, i);
                s->bx[c] -= h * ((s->ez[FI(g, k, j + 1, i)] - s->ez[c]) / s->dy -
                                 (s->ey[FI(g, k + 1, j, i)] - s->ey[c]) / s->dz);
                s->by[c] -= h * ((s->ex[FI(g, k + 1, j, i)] - s->ex[c]) / s->dz -
                                 (s->ez[FI(g, k, j, i + 1)] - s->ez[c]) / s->dx);
                s->bz[c] -= h * ((s->ey[FI(g, k, j, i + 1)] - s->ey[c]) / s->dx -
                                 (s->ex[FI(g, k, j + 1, i)] - s->ex[c]) / s->dy);
            }
    orc_exchange_boundary_data(s, s->bx);
    orc_exchange_boundary_data(s, s->by);
    orc_exchange_boundary_data(s, s->bz);
}

/* Extension (absorbing = 1; the reference has none): the first-order
 * Silver-Mueller condition of radiating_boundary's x-min update
 * (src/boundary.cpp:88-89) on the other non-periodic faces, once per step at
 * the same point (the end of orc_radiating_boundary).  Min faces (y, z) set
 * the ghost B row mem-1 with the x-min formula's axes relabelled cyclically;
 * max faces (y, z, x) set the last physical B row, reflected through the
 * face (tangential B flips sign; E and J do not), from the E and J of that
 * row and the B row below it.  alpha = 1/(1 + dt/h), beta = 1 - dt/h, h the
 * cell size across the face.  The x-min update's tangential-derivative term
 * is left out: with it, relabelled onto these faces, oblique waves grow
 * without bound (a random field in a box absorbing on every side gains 1e4
 * per 60 steps); without it the same field decays. */
static void absorb_faces(orc_state *s) {
    if (!s->absorbing) return;
    geom g = make_geom(s);
    const int m = s->mem;
    const double dt = s->dt, hx = s->dt / s->dx, hy = s->dt / s->dy, hz = s->dt / s->dz;
    for (int face = 0; face < 5; ++face) {
        const int ax = face < 2 ? 1 : (face < 4 ? 2 : 0);
        if (neighbour(s, ax) != -2) continue;
        const int lo = face == 0 || face == 2;
        const double h = ax == 0 ? hx : (ax == 1 ? hy : hz);
        const double alpha = 1.0 / (1.0 + h), beta = 1.0 - h, sg = lo ? 1.0 : -1.0;
        const int row = lo ? m : g.n[ax] + m - 1;
        for (int k = g.nc_st[2]; k <= g.nc_end[2]; k++)
            for (int j = g.nc_st[1]; j <= g.nc_end[1]; j++)
                for (int i = g.nc_st[0]; i <= g.nc_end[0]; i++) {
                    int q[3] = {i, j, k};
                    if (q[ax] != row) continue;
                    int t[3] = {i, j, k}, n[3] = {i, j, k};
                    if (lo) t[ax] -= 1; else n[ax] -= 1;   /* target row and the interior B row */
                    long c = FI(g, k, j, i), rc = RI(g, k, j, i);
                    long ct = FI(g, t[2], t[1], t[0]), cn = FI(g, n[2], n[1], n[0]);
                    if (ax == 1) {
                        s->bx[ct] = alpha * (sg * (-2.0 * s->ez[c] - dt * s->jz[rc]) - beta * s->bx[cn]);
                        s->bz[ct] = alpha * (sg * (2.0 * s->ex[c] + dt * s->jx[rc]) - beta * s->bz[cn]);
                    } else if (ax == 2) {
                        s->by[ct] = alpha * (sg * (-2.0 * s->ex[c] - dt * s->jx[rc]) - beta * s->by[cn]);
                        s->bx[ct] = alpha * (sg * (2.0 * s->ey[c] + dt * s->jy[rc]) - beta * s->bx[cn]);
                    } else {
                        s->bz[ct] = alpha * (sg * (-2.0 * s->ey[c] - dt * s->jy[rc]) - beta * s->bz[cn]);
                        s->by[ct] = alpha * (sg * (2.0 * s->ez[c] + dt * s->jz[rc]) - beta * s->by[cn]);
                    }
                }
    }
}

/* update_electromagnetic_fields_first: src/field.cpp:56-86 */
void orc_fields_first(orc_state *s) {
    update_e(s);
    update_b(s);
}

/* update_electromagnetic_fields_second: src/field.cpp:88-117 */
void orc_fields_second(orc_state *s) {
    update_b(s);
    update_e(s);
}

/* clear_currents: src/particle.cpp:576-592 (whole ring buffers) */
void orc_clear_currents(orc_state *s) {
    geom g = make_geom(s);
    size_t bytes = sizeof(double) * (size_t)g.rsz;
    memset(s->jx, 0, bytes);
    memset(s->jy, 0, bytes);
    memset(s->jz, 0, bytes);
    memset(s->rho0, 0, bytes);
    memset(s->rho1, 0, bytes);
}

/* ------------------------------------------------------------------ */
/* currents_particle: src/particle.cpp:372-515.  Esirkepov charge-
 * conserving Jx/Jy/Jz from the old and new shape factors, then the
 * species charge density at the new position.                           */

static inline double sfac(const double *S, int idx, int centre, int h) {
    return (idx >= centre - h && idx <= centre + h) ? S[idx - centre + h] : 0.0;
}

void orc_currents_particle(orc_state *s, const orc_particle *p, int kind) {
    geom g = make_geom(s);
    const int m = s->mem, h = m / 2;
    double x1 = p->x_old - g.nc_new[0], x2 = p->x - g.nc_new[0];
    double y1 = p->y_old - g.nc_new[1], y2 = p->y - g.nc_new[1];
    double z1 = p->z_old - g.nc_new[2], z2 = p->z - g.nc_new[2];
    double Sx0[5], Sx1[5], Sy0[5], Sy1[5], Sz0[5], Sz1[5];
    shape(s, x1, Sx0);
    shape(s, x2, Sx1);
    shape(s, y1, Sy0);
    shape(s, y2, Sy1);
    shape(s, z1, Sz0);
    shape(s, z2, Sz1);
    int i1 = (int)(x1 + 0.5), i2 = (int)(x2 + 0.5);
    int j1 = (int)(y1 + 0.5), j2 = (int)(y2 + 0.5);
    int k1 = (int)(z1 + 0.5), k2 = (int)(z2 + 0.5);
    int imin = (i1 < i2 ? i1 : i2) - h, imax = (i1 > i2 ? i1 : i2) + h;
    int jmin = (j1 < j2 ? j1 : j2) - h, jmax = (j1 > j2 ? j1 : j2) + h;
    int kmin = (k1 < k2 ? k1 : k2) - h, kmax = (k1 > k2 ? k1 : k2) + h;

    double q_w = p->charge * p->weight;
    double c_x = q_w * s->dx / s->dt;
    double c_y = q_w * s->dy / s->dt;
    double c_z = q_w * s->dz / s->dt;
    const double third = 1.0 / 3.0;

    for (int k = kmin; k <= kmax; k++) {
        double sz0 = sfac(Sz0, k, k1, h), sz1 = sfac(Sz1, k, k2, h), dsz = sz1 - sz0;
        for (int j = jmin; j <= jmax; j++) {
            double sy0 = sfac(Sy0, j, j1, h), sy1 = sfac(Sy1, j, j2, h), dsy = sy1 - sy0;
            double wyz = sy0 * sz0 + 0.5 * dsy * sz0 + 0.5 * sy0 * dsz + third * dsy * dsz;
            double acc = 0.0;
            for (int i = imin; i <= imax; i++) {
                acc += sfac(Sx1, i, i2, h) - sfac(Sx0, i, i1, h);
                s->jx[RI(g, k, j, i)] -= c_x * acc * wyz;
            }
        }
    }
    for (int k = kmin; k <= kmax; k++) {
        double sz0 = sfac(Sz0, k, k1, h), sz1 = sfac(Sz1, k, k2, h), dsz = sz1 - sz0;
        for (int i = imin; i <= imax; i++) {
            double sx0 = sfac(Sx0, i, i1, h), sx1 = sfac(Sx1, i, i2, h), dsx = sx1 - sx0;
            double wxz = sx0 * sz0 + 0.5 * dsx * sz0 + 0.5 * sx0 * dsz + third * dsx * dsz;
            double acc = 0.0;
            for (int j = jmin; j <= jmax; j++) {
                acc += sfac(Sy1, j, j2, h) - sfac(Sy0, j, j1, h);
                s->jy[RI(g, k, j, i)] -= c_y * acc * wxz;
            }
        }
    }
    for (int j = jmin; j <= jmax; j++) {
        double sy0 = sfac(Sy0, j, j1, h), sy1 = sfac(Sy1, j, j2, h), dsy = sy1 - sy0;
        for (int i = imin; i <= imax; i++) {
            double sx0 = sfac(Sx0, i, i1, h), sx1 = sfac(Sx1, i, i2, h), dsx = sx1 - sx0;
            double wxy = sx0 * sy0 + 0.5 * dsx * sy0 + 0.5 * sx0 * dsy + third * dsx * dsy;
            double acc = 0.0;
            for (int k = kmin; k <= kmax; k++) {
                acc += sfac(Sz1, k, k2, h) - sfac(Sz0, k, k1, h);
                s->jz[RI(g, k, j, i)] -= c_z * acc * wxy;
            }
        }
    }
    double *rho = kind == 0 ? s->rho0 : s->rho1;
    for (int k = kmin; k <= kmax; k++) {
        double sz = sfac(Sz1, k, k2, h);
        if (sz == 0.0) continue;
        for (int j = jmin; j <= jmax; j++) {
            double sy = sfac(Sy1, j, j2, h);
            if (sy == 0.0) continue;
            for (int i = imin; i <= imax; i++) rho[RI(g, k, j, i)] += q_w * sfac(Sx1, i, i2, h) * sy * sz;
        }
    }
}

/* ------------------------------------------------------------------ */
/* update_particle_position_momentum: src/particle.cpp:113-370.  Periodic
 * wrap, staggered gather, relativistic Boris push, move in cell units,
 * deposit, then electron spin precession.                               */

static double gather(const geom *g, const double *f, const double *wx, const double *wy, const double *wz,
                     int ic, int jc, int kc, int h) {
    double acc = 0.0;
    for (int k = -h; k <= h; k++)
        for (int j = -h; j <= h; j++)
            for (int i = -h; i <= h; i++)
                acc += wx[i + h] * wy[j + h] * wz[k + h] * f[FI(*g, kc + k, jc + j, ic + i)];
    return acc;
}

void orc_push(orc_state *s, int kind) {
    geom g = make_geom(s);
    const int h = s->mem / 2;
    const double xend = g.n[0], yend = g.n[1], zend = g.n[2];
    const int any_periodic = s->rank_period[0] || s->rank_period[1] || s->rank_period[2];
    orc_particle *P = s->particles[kind];
    for (int64_t n = 0; n < s->num_particles[kind]; ++n) {
        orc_particle *p = &P[n];
        p->rank = 0;
        if (p->x < 0.0 || p->x > xend || p->y < 0.0 || p->y > yend || p->z < 0.0 || p->z > zend) {
            if (!any_periodic) {
                s->out_of_bounds++;
            } else {
                if (s->rank_period[0] == 1) {
                    if (p->x < 0.0) p->x += g.n[0];
                    if (p->x > g.n[0]) p->x -= g.n[0];
                }
                if (s->rank_period[1] == 1) {
                    if (p->y < 0.0) p->y += g.n[1];
                    if (p->y > g.n[1]) p->y -= g.n[1];
                }
                if (s->rank_period[2] == 1) {
                    if (p->z < 0.0) p->z += g.n[2];
                    if (p->z > g.n[2]) p->z -= g.n[2];
                }
            }
        }
        double xc = p->x - g.nc_new[0], yc = p->y - g.nc_new[1], zc = p->z - g.nc_new[2];
        double wxp[5], wyp[5], wzp[5], wxd[5], wyd[5], wzd[5];
        shape(s, xc, wxp);
        shape(s, yc, wyp);
        shape(s, zc, wzp);
        shape(s, xc - 0.5, wxd);
        shape(s, yc - 0.5, wyd);
        shape(s, zc - 0.5, wzd);
        int ip = (int)(xc + 0.5), jp = (int)(yc + 0.5), kp = (int)(zc + 0.5);
        int id = (int)xc, jd = (int)yc, kd = (int)zc;

        double ex_p = gather(&g, s->ex, wxd, wyp, wzp, id, jp, kp, h);
        double ey_p = gather(&g, s->ey, wxp, wyd, wzp, ip, jd, kp, h);
        double ez_p = gather(&g, s->ez, wxp, wyp, wzd, ip, jp, kd, h);
        double bx_p = gather(&g, s->bx, wxp, wyd, wzd, ip, jd, kd, h);
        double by_p = gather(&g, s->by, wxd, wyp, wzd, id, jp, kd, h);
        double bz_p = gather(&g, s->bz, wxd, wyd, wzp, id, jd, kp, h);

        double px0 = p->px, py0 = p->py, pz0 = p->pz;
        p->x_old = p->x;
        p->y_old = p->y;
        p->z_old = p->z;
        double qm = p->charge / (p->mass) * s->dt_half;
        ex_p *= qm;
        ey_p *= qm;
        ez_p *= qm;
        bx_p *= qm;
        by_p *= qm;
        bz_p *= qm;
        double px1 = px0 + ex_p, py1 = py0 + ey_p, pz1 = pz0 + ez_p;
        double gm1 = sqrt(1.0 + (px1 * px1 + py1 * py1 + pz1 * pz1));
        double tx = bx_p / gm1, ty = by_p / gm1, tz = bz_p / gm1;
        double tt = 2.0 / (1.0 + tx * tx + ty * ty + tz * tz);
        double sx = tx * tt, sy = ty * tt, sz = tz * tt;
        double px2 = px1 + (py1 * tz - pz1 * ty);
        double py2 = py1 + (pz1 * tx - px1 * tz);
        double pz2 = pz1 + (px1 * ty - py1 * tx);
        double px3 = px1 + (py2 * sz - pz2 * sy);
        double py3 = py1 + (pz2 * sx - px2 * sz);
        double pz3 = pz1 + (px2 * sy - py2 * sx);
        p->px = px3 + ex_p;
        p->py = py3 + ey_p;
        p->pz = pz3 + ez_p;
        p->gamma = sqrt(1.0 + (p->px * p->px + p->py * p->py + p->pz * p->pz));
        p->x = p->x_old + p->px / p->gamma * s->dt / s->dx;
        p->y = p->y_old + p->py / p->gamma * s->dt / s->dy;
        p->z = p->z_old + p->pz / p->gamma * s->dt / s->dz;
        orc_currents_particle(s, p, kind);

        if (p->mass == 1.0) {
            /* electron spin precession, src/particle.cpp:318-368 */
            ex_p /= qm;
            ey_p /= qm;
            ez_p /= qm;
            bx_p /= qm;
            by_p /= qm;
            bz_p /= qm;
            double g0 = p->gamma;
            double vx = p->px / g0, vy = p->py / g0, vz = p->pz / g0;
            double pe_x = vx * ex_p, pe_y = vy * ey_p, pe_z = vz * ez_p;
            double fx = (ex_p + vy * bz_p - vz * by_p);
            double fy = (ey_p + vz * bx_p - vx * bz_p);
            double fz = (ez_p + vx * by_p - vy * bx_p);
            double chi = fx * fx + fy * fy + fz * fz - (pe_x + pe_y + pe_z) * (pe_x + pe_y + pe_z);
            if (chi < 0.0) chi = 0.0;
            chi = sqrt(chi) / s->E_schwinger * g0;
            double ga = orc_g_factor(s, chi);
            double al = -(ga / 2.0 - 1.0) * (g0) / (1.0 + g0);
            double be = (ga / 2.0 - 1.0) + 1.0 / g0;
            double gg = ga / 2.0 - g0 / (1.0 + g0);
            double vb = vx * bx_p + vy * by_p + vz * bz_p;
            double ox = al * vb * vx + be * bx_p + gg * (vy * ez_p - vz * ey_p);
            double oy = al * vb * vy + be * by_p + gg * (vz * ex_p - vx * ez_p);
            double oz = al * vb * vz + be * bz_p + gg * (vx * ey_p - vy * ex_p);
            double q2 = p->charge / p->mass * s->dt_half;
            tx = ox * q2;
            ty = oy * q2;
            tz = oz * q2;
            tt = 2.0 / (1.0 + tx * tx + ty * ty + tz * tz);
            double sxr = p->sx + (p->sy * tz - p->sz * ty);
            double syr = p->sy + (p->sz * tx - p->sx * tz);
            double szr = p->sz + (p->sx * ty - p->sy * tx);
            double nx = p->sx + (syr * tz - szr * ty) * tt;
            double ny = p->sy + (szr * tx - sxr * tz) * tt;
            double nz = p->sz + (sxr * ty - syr * tx) * tt;
            p->sx = nx;
            p->sy = ny;
            p->sz = nz;
        }
    }
}

/* ------------------------------------------------------------------ */
/* exchange_particle_data: src/mpi_utils.cpp:62-230 on one rank.  Per
 * dimension (X, then Y, then Z): particles below the lower edge (periodic)
 * go to the "minus" list, at or above the upper edge (periodic) to the
 * "plus" list, outside a non-periodic global edge are removed; stayers
 * keep their order and the vector becomes stayers, then the plus list (it
 * comes back as the message from the minus neighbour), then the minus list.
 * Positions are not wrapped here; the next push wraps them.             */
void orc_exchange_particles(orc_state *s, int kind) {
    geom g = make_geom(s);
    orc_particle *P = s->particles[kind];
    int64_t n = s->num_particles[kind];
    orc_particle *tmp = s->scratch;
    for (int d = 0; d < 3; ++d) {
        const double lo = 0.0, hi = g.n[d];
        int per = neighbour(s, d) != -2;
        int64_t nstay = 0, nplus = 0, nminus = 0;
        /* pass 1: stayers compacted in place, count plus / minus */
        for (int64_t i = 0; i < n; ++i) {
            double c = d == 0 ? P[i].x : d == 1 ? P[i].y : P[i].z;
            int cls; /* 0 stay, 1 minus, 2 plus, 3 removed */
            if (c < lo && per)
                cls = 1;
            else if (c >= hi && per)
                cls = 2;
            else if ((c < 0.0 && !per) || (c >= g.n[d] && !per))
                cls = 3;
            else
                cls = 0;
            if (cls == 1)
                nminus++;
            else if (cls == 2)
                tmp[nplus++] = P[i];
        }
        int64_t off = nplus;
        for (int64_t i = 0; i < n; ++i) {
            double c = d == 0 ? P[i].x : d == 1 ? P[i].y : P[i].z;
            if (c < lo && per) tmp[off++] = P[i];
        }
        for (int64_t i = 0; i < n; ++i) {
            double c = d == 0 ? P[i].x : d == 1 ? P[i].y : P[i].z;
            int keep;
            if (c < lo && per)
                keep = 0;
            else if (c >= hi && per)
                keep = 0;
            else if ((c < 0.0 && !per) || (c >= g.n[d] && !per))
                keep = 0;
            else
                keep = 1;
            if (keep) P[nstay++] = P[i];
        }
        memcpy(P + nstay, tmp, sizeof(orc_particle) * (size_t)(nplus + nminus));
        n = nstay + nplus + nminus;
    }
    s->num_particles[kind] = n;
}

/* exchange_boundary_current_fixed: src/mpi_utils.cpp:232-417 on one rank.
 * Periodic dimensions first add the (mem+1)-wide ghost slab on each side
 * into the opposite physical edge (X, Y, Z in turn, each over the whole
 * extent of the other two dimensions, using the slab values as they were
 * before that dimension's adds), then copy the physical edges back into
 * the ghost slabs (X, Y, Z).                                            */
void orc_exchange_current(orc_state *s, double *a) {
    geom g = make_geom(s);
    const int m = s->mem;
    int lo[3] = {-1, -1, -1}, hi[3] = {g.fx, g.fy, g.fz};
    double *sa = (double *)malloc(sizeof(double) * (size_t)g.rsz);
    double *sb = (double *)malloc(sizeof(double) * (size_t)g.rsz);
    for (int d = 0; d < 3; ++d) {
        if (neighbour(s, d) == -2) continue;
        int n = g.n[d];
        /* snapshot both ghost slabs, then add minus-side then plus-side */
        for (int t = 0; t <= m; ++t) {
            for (int u = lo[(d + 2) % 3]; u <= hi[(d + 2) % 3]; ++u)
                for (int v = lo[(d + 1) % 3]; v <= hi[(d + 1) % 3]; ++v) {
                    int idx_a[3], idx_b[3];
                    idx_a[d] = n + m + t; /* plus-side ghost slab   */
                    idx_b[d] = -1 + t;    /* minus-side ghost slab  */
                    idx_a[(d + 1) % 3] = idx_b[(d + 1) % 3] = v;
                    idx_a[(d + 2) % 3] = idx_b[(d + 2) % 3] = u;
                    long ra = RI(g, idx_a[2], idx_a[1], idx_a[0]);
                    long rb = RI(g, idx_b[2], idx_b[1], idx_b[0]);
                    sa[ra] = a[ra];
                    sb[rb] = a[rb];
                }
        }
        for (int t = 0; t <= m; ++t)
            for (int u = lo[(d + 2) % 3]; u <= hi[(d + 2) % 3]; ++u)
                for (int v = lo[(d + 1) % 3]; v <= hi[(d + 1) % 3]; ++v) {
                    int dst[3], src[3];
                    dst[d] = m + t;
                    src[d] = n + m + t;
                    dst[(d + 1) % 3] = src[(d + 1) % 3] = v;
                    dst[(d + 2) % 3] = src[(d + 2) % 3] = u;
                    a[RI(g, dst[2], dst[1], dst[0])] += sa[RI(g, src[2], src[1], src[0])];
                }
        for (int t = 0; t <= m; ++t)
            for (int u = lo[(d + 2) % 3]; u <= hi[(d + 2) % 3]; ++u)
                for (int v = lo[(d + 1) % 3]; v <= hi[(d + 1) % 3]; ++v) {
                    int dst[3], src[3];
                    dst[d] = n - 1 + t;
                    src[d] = -1 + t;
                    dst[(d + 1) % 3] = src[(d + 1) % 3] = v;
                    dst[(d + 2) % 3] = src[(d + 2) % 3] = u;
                    a[RI(g, dst[2], dst[1], dst[0])] += sb[RI(g, src[2], src[1], src[0])];
                }
    }
    for (int d = 0; d < 3; ++d) {
        if (neighbour(s, d) == -2) continue;
        int n = g.n[d];
        for (int t = 0; t <= m; ++t)
            for (int u = lo[(d + 2) % 3]; u <= hi[(d + 2) % 3]; ++u)
                for (int v = lo[(d + 1) % 3]; v <= hi[(d + 1) % 3]; ++v) {
                    int i0[3], i1[3], i2[3], i3[3];
                    i0[d] = -1 + t;    /* minus ghost  <- */
                    i1[d] = n - 1 + t; /* plus-side physical edge */
                    i2[d] = n + m + t; /* plus ghost   <- */
                    i3[d] = m + t;     /* minus-side physical edge */
                    for (int e = 1; e <= 2; ++e) {
                        int o = (d + e) % 3, val = e == 1 ? v : u;
                        i0[o] = i1[o] = i2[o] = i3[o] = val;
                    }
                    a[RI(g, i0[2], i0[1], i0[0])] = a[RI(g, i1[2], i1[1], i1[0])];
                    a[RI(g, i2[2], i2[1], i2[0])] = a[RI(g, i3[2], i3[1], i3[0])];
                }
    }
    free(sa);
    free(sb);
}

/* exchange_currents: src/particle.cpp:594-601 */
void orc_exchange_currents(orc_state *s) {
    orc_exchange_current(s, s->jx);
    orc_exchange_current(s, s->jy);
    orc_exchange_current(s, s->jz);
    orc_exchange_current(s, s->rho0);
    orc_exchange_current(s, s->rho1);
}

/* t = 0 sequence of main.cpp:75-79: one push + deposit of each species
 * with the fields as they are (zero at start), then the particle exchange;
 * the currents are neither cleared before nor folded after. */
void orc_initial(orc_state *s) {
    orc_push(s, 0);
    orc_push(s, 1);
    orc_exchange_particles(s, 0);
    orc_exchange_particles(s, 1);
}

/* one iteration of run_main_time_loop: src/simulation.cpp:159-183
 * (`step` is the 1-based step number the reference passes to
 * radiating_boundary) */
void orc_step(orc_state *s, int step) {
    orc_radiating_boundary(s, 1, 0, step);
    orc_fields_first(s);
    orc_clear_currents(s);
    orc_push(s, 0);
    orc_push(s, 1);
    orc_exchange_particles(s, 0);
    orc_exchange_particles(s, 1);
    orc_exchange_currents(s);
    orc_fields_second(s);
}

void orc_run(orc_state *s, int first_step, int nsteps) {
    for (int t = 0; t < nsteps; ++t) orc_step(s, first_step + t);
}
