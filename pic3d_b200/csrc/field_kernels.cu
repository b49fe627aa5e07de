// Field-side kernels: Yee E/B half-updates, periodic ghost fill, laser /
// Silver-Mueller x-boundary and the periodic J / rho fold.
//
// All are HBM-bound stencils or face/shell copies.  The Yee updates run one
// thread per physical cell with x fastest (coalesced); neighbour reads come
// through L1/L2.  The periodic halo exchange of the reference
// (src/mpi_utils.cpp:9-60) and the ghost accumulation of the currents
// (src/mpi_utils.cpp:232-417) become single-launch shell kernels: every
// ghost point pulls its periodic image, every boundary point sums and then
// broadcasts its images; each point has exactly one owning thread, so no
// atomics are needed.
#include "pic_kernels.cuh"
#include "push_core.cuh"

namespace pic {

Geom make_geom(const PicParams &p) {
    Geom g{};
    g.n[0] = p.local_xcells;
    g.n[1] = p.local_ycells;
    g.n[2] = p.local_zcells;
    g.mem = p.mem;
    for (int d = 0; d < 3; ++d) {
        g.f[d] = g.n[d] + 2 * p.mem;
        g.r[d] = g.f[d] + 2;
        g.per[d] = p.rank_period[d] ? 1 : 0;
    }
    // sizes in 64 bits from the extents, so that a caller's check of rsz
    // against the 32-bit index range is meaningful even where the plane
    // strides (int) would overflow; the strides are only used once that
    // check has passed
    g.fsz = (long long)g.f[0] * g.f[1] * g.f[2];
    g.rsz = (long long)g.r[0] * g.r[1] * g.r[2];
    g.fxy = (int)((long long)g.f[0] * g.f[1]);
    g.rxy = (int)((long long)g.r[0] * g.r[1]);
    return g;
}

// ---------------------------------------------------------------------------
// Yee half-updates over the physical cells (src/field.cpp:59-67 and :74-82)

template <typename real>
__global__ void __launch_bounds__(256) update_e_kernel(Geom g, real *__restrict__ ex, real *__restrict__ ey,
                                                       real *__restrict__ ez, const real *__restrict__ bx,
                                                       const real *__restrict__ by, const real *__restrict__ bz,
                                                       const real *__restrict__ jx, const real *__restrict__ jy,
                                                       const real *__restrict__ jz, real h, real idx, real idy,
                                                       real idz) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    int k = blockIdx.z;
    if (i >= g.n[0] || j >= g.n[1]) return;
    i += g.mem;
    j += g.mem;
    k += g.mem;
    const int c = g.fi(k, j, i), rc = g.ri(k, j, i);
    const int sy = g.f[0], sz = g.fxy;
    real bxc = bx[c], byc = by[c], bzc = bz[c];
    ex[c] += h * ((bzc - bz[c - sy]) * idy - (byc - by[c - sz]) * idz - jx[rc]);
    ey[c] += h * ((bxc - bx[c - sz]) * idz - (bzc - bz[c - 1]) * idx - jy[rc]);
    ez[c] += h * ((byc - by[c - 1]) * idx - (bxc - bx[c - sy]) * idy - jz[rc]);
}

template <typename real>
__global__ void __launch_bounds__(256) update_b_kernel(Geom g, const real *__restrict__ ex,
                                                       const real *__restrict__ ey, const real *__restrict__ ez,
                                                       real *__restrict__ bx, real *__restrict__ by,
                                                       real *__restrict__ bz, real h, real idx, real idy, real idz) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    int k = blockIdx.z;
    if (i >= g.n[0] || j >= g.n[1]) return;
    i += g.mem;
    j += g.mem;
    k += g.mem;
    const int c = g.fi(k, j, i);
    const int sy = g.f[0], sz = g.fxy;
    real exc = ex[c], eyc = ey[c], ezc = ez[c];
    bx[c] -= h * ((ez[c + sy] - ezc) * idy - (ey[c + sz] - eyc) * idz);
    by[c] -= h * ((ex[c + sz] - exc) * idz - (ez[c + 1] - ezc) * idx);
    bz[c] -= h * ((ey[c + 1] - eyc) * idx - (ex[c + sy] - exc) * idy);
}

// ---------------------------------------------------------------------------
// Periodic ghost fill (single-rank meaning of exchange_boundary_data,
// src/mpi_utils.cpp:9-60).  The reference copies X, then Y, then Z slabs over
// the full extent of the other dimensions; the result is that every point
// whose coordinate in a periodic dimension is a ghost holds the value of the
// point with each such coordinate replaced by its periodic image (other
// coordinates unchanged, ghosts of non-periodic faces included).  Each ghost
// point belongs to the slab of the first periodic dimension in which it is a
// ghost, so every point is written once.

struct ShellPlan {
    int ns;                 // number of slabs
    int dim[3];             // slab dimension
    int lo[3][3], ext[3][3];  // per slab, per axis: first coordinate and extent (slab axis: see kernel)
    long long start[4];
};

static ShellPlan ghost_plan(const Geom &g) {
    ShellPlan pl{};
    long long acc = 0;
    for (int d = 0; d < 3; ++d) {
        if (!g.per[d]) continue;
        int s = pl.ns++;
        pl.dim[s] = d;
        long long cnt = 1;
        for (int e = 0; e < 3; ++e) {
            if (e == d) {
                pl.lo[s][e] = 0;
                pl.ext[s][e] = 2 * g.mem;
            } else if (e < d && g.per[e]) {
                pl.lo[s][e] = g.mem;
                pl.ext[s][e] = g.n[e];
            } else {
                pl.lo[s][e] = 0;
                pl.ext[s][e] = g.f[e];
            }
            cnt *= pl.ext[s][e];
        }
        pl.start[s] = acc;
        acc += cnt;
    }
    pl.start[pl.ns] = acc;
    return pl;
}

template <typename real>
__global__ void ghost_fill_kernel(Geom g, ShellPlan pl, real *a0, real *a1, real *a2) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= pl.start[pl.ns]) return;
    int s = 0;
    while (s + 1 < pl.ns && t >= pl.start[s + 1]) ++s;
    long long l = t - pl.start[s];
    int c[3];
    for (int e = 0; e < 3; ++e) {
        int q = (int)(l % pl.ext[s][e]);
        l /= pl.ext[s][e];
        c[e] = pl.lo[s][e] + q;
    }
    const int d = pl.dim[s];
    // slab axis: 0..mem-1 low ghosts, mem..2mem-1 high ghosts
    c[d] = c[d] < g.mem ? c[d] : g.n[d] + c[d];
    int src[3];
    for (int e = 0; e < 3; ++e) {
        src[e] = c[e];
        if (g.per[e]) {
            if (c[e] < g.mem) src[e] = c[e] + g.n[e];
            else if (c[e] >= g.n[e] + g.mem) src[e] = c[e] - g.n[e];
        }
    }
    const int di = g.fi(c[2], c[1], c[0]), si = g.fi(src[2], src[1], src[0]);
    a0[di] = a0[si];
    if (a1) a1[di] = a1[si];
    if (a2) a2[di] = a2[si];
}

// ---------------------------------------------------------------------------
// Periodic current / charge fold (single-rank meaning of
// exchange_boundary_current_fixed, src/mpi_utils.cpp:232-417): the
// reference adds the (mem+1)-wide ghost slabs into the opposite physical
// edges X, Y, Z in turn and then copies the edges back to the ghosts.  The
// end state is: each point whose periodic coordinates are physical holds the
// sum over all its periodic images inside the ring, and every image holds
// that same sum; ring points of non-periodic faces are left as deposited.
// A physical coordinate c has an image c-n when c >= n-1 and c+n when
// c <= 2 mem.  Each owner point (first periodic axis with an image) sums its
// <= 8 images and writes the total to all of them.

static ShellPlan fold_plan(const Geom &g) {
    ShellPlan pl{};
    long long acc = 0;
    for (int d = 0; d < 3; ++d) {
        if (!g.per[d]) continue;
        int s = pl.ns++;
        pl.dim[s] = d;
        long long cnt = 1;
        for (int e = 0; e < 3; ++e) {
            if (e == d) {
                pl.lo[s][e] = 0;
                pl.ext[s][e] = 2 * (g.mem + 1);
            } else if (e < d && g.per[e]) {
                pl.lo[s][e] = 2 * g.mem + 1;              // physical coordinates without images
                pl.ext[s][e] = g.n[e] - 2 * g.mem - 2;
            } else if (g.per[e]) {
                pl.lo[s][e] = g.mem;
                pl.ext[s][e] = g.n[e];
            } else {
                pl.lo[s][e] = -1;
                pl.ext[s][e] = g.r[e];
            }
            cnt *= pl.ext[s][e];
        }
        pl.start[s] = acc;
        acc += cnt;
    }
    pl.start[pl.ns] = acc;
    return pl;
}

template <typename real>
__global__ void fold_kernel(Geom g, ShellPlan pl, real *a0, real *a1, real *a2, real *a3, real *a4) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= pl.start[pl.ns]) return;
    real *arr[5] = {a0, a1, a2, a3, a4};
    real *a = arr[blockIdx.y];
    if (!a) return;
    int s = 0;
    while (s + 1 < pl.ns && t >= pl.start[s + 1]) ++s;
    long long l = t - pl.start[s];
    int c[3];
    for (int e = 0; e < 3; ++e) {
        int q = (int)(l % pl.ext[s][e]);
        l /= pl.ext[s][e];
        c[e] = pl.lo[s][e] + q;
    }
    const int d = pl.dim[s];
    c[d] = c[d] <= g.mem ? g.mem + c[d] : g.n[d] - 1 + (c[d] - g.mem - 1);
    int img[3][2], nimg[3];
    for (int e = 0; e < 3; ++e) {
        img[e][0] = c[e];
        nimg[e] = 1;
        if (g.per[e]) {
            if (c[e] >= g.n[e] - 1) img[e][nimg[e]++] = c[e] - g.n[e];
            else if (c[e] <= 2 * g.mem) img[e][nimg[e]++] = c[e] + g.n[e];
        }
    }
    real tot = 0;
    for (int z = 0; z < nimg[2]; ++z)
        for (int y = 0; y < nimg[1]; ++y)
            for (int x = 0; x < nimg[0]; ++x) tot += a[g.ri(img[2][z], img[1][y], img[0][x])];
    for (int z = 0; z < nimg[2]; ++z)
        for (int y = 0; y < nimg[1]; ++y)
            for (int x = 0; x < nimg[0]; ++x) a[g.ri(img[2][z], img[1][y], img[0][x])] = tot;
}

// ---------------------------------------------------------------------------
// Laser source and x-boundary (src/boundary.cpp:8-99), one thread per
// physical (y, z) row.  The transverse coordinate is (buffer index)*dy -
// yfocus as in the reference (boundary.cpp:61-62).

struct LaserArgs {
    double Pi, omega, l0, Lx, dt, dx, dy, dz;
    double amp, dur, start, waist, xfocus, yfocus, zfocus, phase;
    int pol, envelope, profile, profile_n;
    const double *coef;
    double time;
    int is_left, is_right;
    int absorbing;   // extension: the x-max face takes the absorbing condition instead
};

__device__ double laser_envelope(const LaserArgs &L, double time, double position) {
    double t = time - position - L.start;
    if (L.envelope == 1) {
        if (t < 0.0 || t > 3.0 * L.dur) return 0.0;
        double r = (t - 1.5 * L.dur) / L.dur;
        return L.amp * exp(-2.0 * log(2.0) * r * r);
    }
    double env = (t >= 0.0 && t <= L.dur) ? sin(L.Pi * t / L.dur) : 0.0;
    return L.amp * env;
}

// Gpulse (boundary.cpp:29-40); with profile = 1 the Gaussian transverse
// factor waist/w*exp(-r^2/w^2) is replaced by the B-spline amplitude grid.
__device__ double gpulse(const LaserArgs &L, const Geom &g, double time, double x, double y, double z, int iy,
                         int iz) {
    double k = 2.0 * L.Pi / L.l0;
    double rl = 0.5 * k * L.waist * L.waist;
    double xe = x - L.xfocus;
    double ph = atan(xe / rl);
    double q = xe / rl;
    double w = L.waist * sqrt(1 + q * q);
    double PHI = (xe / rl) * (y * y + z * z) / w / w - ph + k * xe - L.omega * time;
    double amp;
    if (L.profile == 1) {
        int nc = L.profile_n;
        double u = ((double)(iy - g.mem) + 0.5) / (double)g.n[1] * (double)(nc - 1);
        double v = ((double)(iz - g.mem) + 0.5) / (double)g.n[2] * (double)(nc - 1);
        amp = 0.0;
        for (int b = 0; b < nc; ++b) {
            double wv = cubic_bspline(v - b);
            if (wv == 0.0) continue;
            for (int c = 0; c < nc; ++c) {
                double wu = cubic_bspline(u - c);
                if (wu == 0.0) continue;
                amp += L.coef[b * nc + c] * wu * wv;
            }
        }
    } else {
        amp = L.waist / w * exp(-(y * y + z * z) / (w * w));
    }
    return -1.0 * laser_envelope(L, time, x) * amp * cos(PHI + L.phase);
}

template <typename real>
__global__ void radiating_boundary_kernel(Geom g, LaserArgs L, const real *__restrict__ ey,
                                          const real *__restrict__ ez, const real *__restrict__ bx, real *by,
                                          real *bz, const real *__restrict__ jy, const real *__restrict__ jz) {
    int iy = blockIdx.x * blockDim.x + threadIdx.x;
    int iz = blockIdx.y * blockDim.y + threadIdx.y;
    if (iy >= g.n[1] || iz >= g.n[2]) return;
    iy += g.mem;
    iz += g.mem;
    const double alpha = 1 / (1 + L.dt / L.dx);
    const double beta = 1 - L.dt / L.dx;
    double y = iy * L.dy - L.yfocus;
    double z = iz * L.dz - L.zfocus;
    double S_l = 0.0, P_l = 0.0, S_r = 0.0, P_r = 0.0;
    if (L.is_left) {
        double s = gpulse(L, g, L.time, 0.0, y, z, iy, iz);
        if (L.pol == 1 || L.pol == 3) S_l = s;
        if (L.pol == 2 || L.pol == 3) P_l = s;
    }
    if (L.is_right) {
        double s = gpulse(L, g, L.time, L.Lx, y, z, iy, iz);
        if (L.pol == 1 || L.pol == 3) S_r = s;
        if (L.pol == 2 || L.pol == 3) P_r = s;
    }
    if (g.per[0]) return;  // rank_xminus / rank_xplus are not MPI_PROC_NULL
    const int m = g.mem, xr = g.n[0];
    {
        int c = g.fi(iz, iy, m), o = g.fi(iz, iy, m - 1), rc = g.ri(iz, iy, m);
        bz[o] = (real)(alpha * (4 * S_l - 2 * (double)ey[c] - L.dt / L.dz * ((double)bx[c] - (double)bx[c - g.fxy]) -
                                beta * (double)bz[c] - L.dt * (double)jy[rc]));
        by[o] = (real)(alpha * (-4 * P_l + 2 * (double)ez[c] + L.dt / L.dy * ((double)bx[c] - (double)bx[c - g.f[0]]) -
                                beta * (double)by[c] + L.dt * (double)jz[rc]));
    }
    if (!L.absorbing) {
        // the reference writes column local_xcells+1 (boundary.cpp:92-96)
        int c = g.fi(iz, iy, xr), o = g.fi(iz, iy, xr + 1), rc = g.ri(iz, iy, xr);
        bz[o] = (real)(alpha * (-4 * S_r + 2 * (double)ey[c] - L.dt / L.dz * ((double)bx[c] - (double)bx[c - g.fxy]) -
                                beta * (double)bz[c] + L.dt * (double)jy[rc]));
        by[o] = (real)(alpha * (4 * P_r - 2 * (double)ez[c] + L.dt / L.dy * ((double)bx[c] - (double)bx[c - g.f[0]]) -
                                beta * (double)by[c] - L.dt * (double)jz[rc]));
    }
}

// ---------------------------------------------------------------------------
// Absorbing faces (extension, PicParams.absorbing = 1).  The reference
// absorbs only at x-min, with the Silver-Mueller update of the ghost B
// column above; its y and z ghosts stay zero (a conductor).  The same
// first-order condition is applied on every other non-periodic face:
//   * y-min / z-min: the ghost B row mem-1 from the first physical row, the
//     reference's x-min update with the axes relabelled cyclically
//     (x -> y -> z -> x, then once more);
//   * y-max / z-max / x-max: the last physical B row (whose own update reads
//     the zero ghost E row above it) from the physical E and J of that row
//     and the B row below: the min-face update reflected through the face
//     (tangential B changes sign under the reflection, E, J and the normal
//     B do not).
// alpha = 1/(1 + dt/h), beta = 1 - dt/h with h the cell size across the
// face.  Two departures from the x-min formula, both for stability (the
// oracle's restatement, run on a random field in a box absorbing on every
// side, grows by 1e4 per 30-60 steps with either): the coefficients are
// those of one full step, so the update runs once per step, where the
// reference applies its x-min update (at the start of the step, with
// radiating_boundary), not after each half-step B update; and the x-min
// formula's tangential-derivative term is left out (relabelled onto these
// faces it amplifies oblique waves).  Energy reflection of a normal Gaussian
// pulse: 3e-4 at the min faces, 5e-3 at the max faces (whose row the next B
// half-update overwrites).  One thread per point
// of a face's physical rows; faces are separate launches (edge rows are
// written by one face each).

struct AbsorbArgs {
    double dt, idt[3];   // dt and dt/dx, dt/dy, dt/dz
    int face;            // 0 y-min, 1 y-max, 2 z-min, 3 z-max, 4 x-max
};

template <typename real>
__global__ void absorb_face_kernel(Geom g, AbsorbArgs A, const real *__restrict__ ex, const real *__restrict__ ey,
                                   const real *__restrict__ ez, real *bx, real *by, real *bz,
                                   const real *__restrict__ jx, const real *__restrict__ jy,
                                   const real *__restrict__ jz) {
    // the two in-face axes of this face
    const int ax = A.face < 2 ? 1 : (A.face < 4 ? 2 : 0);
    const int u_ax = ax == 0 ? 1 : 0, v_ax = ax == 2 ? 1 : 2;
    int u = blockIdx.x * blockDim.x + threadIdx.x, v = blockIdx.y * blockDim.y + threadIdx.y;
    if (u >= g.n[u_ax] || v >= g.n[v_ax]) return;
    int q[3];
    q[u_ax] = u + g.mem;
    q[v_ax] = v + g.mem;
    const bool lo = A.face == 0 || A.face == 2;
    q[ax] = lo ? g.mem : g.n[ax] + g.mem - 1;   // physical row next to the face
    const int st[3] = {1, g.f[0], g.fxy};
    const int c = g.fi(q[2], q[1], q[0]), rc = g.ri(q[2], q[1], q[0]);
    const double h = A.idt[ax];
    const double alpha = 1.0 / (1.0 + h), beta = 1.0 - h, dt = A.dt;
    const double sgn = lo ? 1.0 : -1.0;
    // target B index: ghost row below (min face) or this row (max face);
    // the interior B used by the update: this row (min) or the row below (max)
    const int tgt = lo ? c - st[ax] : c, inn = lo ? c : c - st[ax];
    if (ax == 1) {        // y faces: bx from ez, jz; bz from ex, jx
        bx[tgt] = (real)(alpha * (sgn * (-2.0 * (double)ez[c] - dt * (double)jz[rc]) - beta * (double)bx[inn]));
        bz[tgt] = (real)(alpha * (sgn * (2.0 * (double)ex[c] + dt * (double)jx[rc]) - beta * (double)bz[inn]));
    } else if (ax == 2) { // z faces: by from ex, jx; bx from ey, jy
        by[tgt] = (real)(alpha * (sgn * (-2.0 * (double)ex[c] - dt * (double)jx[rc]) - beta * (double)by[inn]));
        bx[tgt] = (real)(alpha * (sgn * (2.0 * (double)ey[c] + dt * (double)jy[rc]) - beta * (double)bx[inn]));
    } else {              // x-max: the reference's x-min update (boundary.cpp:88-89) reflected
        bz[tgt] = (real)(alpha * (sgn * (-2.0 * (double)ey[c] - dt * (double)jy[rc]) - beta * (double)bz[inn]));
        by[tgt] = (real)(alpha * (sgn * (2.0 * (double)ez[c] + dt * (double)jz[rc]) - beta * (double)by[inn]));
    }
}

template <typename real>
static void absorb_faces(pic_ctx *c) {
    const Geom &g = c->g;
    real **F = (real **)c->field;
    real **R = (real **)c->ring;
    AbsorbArgs A{};
    A.dt = c->p.dt;
    A.idt[0] = c->p.dt / c->p.dx;
    A.idt[1] = c->p.dt / c->p.dy;
    A.idt[2] = c->p.dt / c->p.dz;
    for (int face = 0; face < 5; ++face) {
        const int ax = face < 2 ? 1 : (face < 4 ? 2 : 0);
        if (g.per[ax]) continue;
        const int u_ax = ax == 0 ? 1 : 0, v_ax = ax == 2 ? 1 : 2;
        A.face = face;
        dim3 blk(32, 8), grd((g.n[u_ax] + 31) / 32, (g.n[v_ax] + 7) / 8);
        absorb_face_kernel<real><<<grd, blk, 0, c->stream>>>(g, A, F[0], F[1], F[2], F[3], F[4], F[5], R[0], R[1],
                                                             R[2]);
    }
}

void launch_absorbing_faces(pic_ctx *c) {
    if (c->p.absorbing != 1) return;
    prof_begin(c, "absorbing_faces");
    if (c->fp32) absorb_faces<float>(c); else absorb_faces<double>(c);
    prof_end(c);
}

// ---------------------------------------------------------------------------
// host launchers

template <typename real>
static void fields_e(pic_ctx *c, double coef) {
    const Geom &g = c->g;
    dim3 blk(32, 8), grd((g.n[0] + 31) / 32, (g.n[1] + 7) / 8, g.n[2]);
    real **F = (real **)c->field;
    real **R = (real **)c->ring;
    update_e_kernel<real><<<grd, blk, 0, c->stream>>>(g, F[0], F[1], F[2], F[3], F[4], F[5], R[0], R[1], R[2],
                                                      (real)coef, (real)(1.0 / c->p.dx),
                                                      (real)(1.0 / c->p.dy), (real)(1.0 / c->p.dz));
}

template <typename real>
static void fields_b(pic_ctx *c, double coef) {
    const Geom &g = c->g;
    dim3 blk(32, 8), grd((g.n[0] + 31) / 32, (g.n[1] + 7) / 8, g.n[2]);
    real **F = (real **)c->field;
    update_b_kernel<real><<<grd, blk, 0, c->stream>>>(g, F[0], F[1], F[2], F[3], F[4], F[5], (real)coef,
                                                      (real)(1.0 / c->p.dx), (real)(1.0 / c->p.dy),
                                                      (real)(1.0 / c->p.dz));
}

// ghost fill of up to three field arrays (null entries skipped)
template <typename real>
static void ghost_fill(pic_ctx *c, void *a0, void *a1, void *a2) {
    ShellPlan pl = ghost_plan(c->g);
    long long n = pl.start[pl.ns];
    if (n == 0) return;
    ghost_fill_kernel<real><<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->g, pl, (real *)a0, (real *)a1,
                                                                               (real *)a2);
}

static void ghost_fill_any(pic_ctx *c, void *a0, void *a1, void *a2) {
    if (c->fp32) ghost_fill<float>(c, a0, a1, a2); else ghost_fill<double>(c, a0, a1, a2);
}

void launch_update_e(pic_ctx *c, double coef) {
    prof_begin(c, "yee_update_e");
    if (c->fp32) fields_e<float>(c, coef); else fields_e<double>(c, coef);
    prof_end(c);
    prof_begin(c, "ghost_fill");
    ghost_fill_any(c, c->field[0], c->field[1], c->field[2]);
    prof_end(c);
}

void launch_update_b(pic_ctx *c, double coef) {
    prof_begin(c, "yee_update_b");
    if (c->fp32) fields_b<float>(c, coef); else fields_b<double>(c, coef);
    prof_end(c);
    prof_begin(c, "ghost_fill");
    ghost_fill_any(c, c->field[3], c->field[4], c->field[5]);
    prof_end(c);
}

void launch_ghost_fill_one(pic_ctx *c, int array) {
    prof_begin(c, "ghost_fill");
    ghost_fill_any(c, c->field[array], nullptr, nullptr);
    prof_end(c);
}

// fold of the ring arrays selected by `mask` (bit k: jx, jy, jz, rho0, rho1)
template <typename real>
static void fold(pic_ctx *c, unsigned mask) {
    ShellPlan pl = fold_plan(c->g);
    long long n = pl.start[pl.ns];
    if (n == 0) return;
    real *R[5];
    for (int k = 0; k < 5; ++k) R[k] = (mask >> k & 1u) ? (real *)c->ring[k] : nullptr;
    dim3 grd((unsigned)((n + 255) / 256), 5);
    fold_kernel<real><<<grd, 256, 0, c->stream>>>(c->g, pl, R[0], R[1], R[2], R[3], R[4]);
}

void launch_fold_currents(pic_ctx *c, unsigned mask) {
    prof_begin(c, "current_fold");
    if (c->fp32) fold<float>(c, mask); else fold<double>(c, mask);
    prof_end(c);
}

// ---------------------------------------------------------------------------
// One pass of the binomial current filter (filter_field,
// src/particle.cpp:520-567) along `axis`: every physical point becomes
// 0.25 a[i-1] + 0.5 a[i] + 0.25 a[i+1] of the values before the pass (`src`
// is a copy of the array taken before it); all other points are untouched.
// The products by 1/4 and 1/2 are exact, so the sum is the reference's
// (0.25 a + 0.5 b) + 0.25 c rounded twice, contracted or not.
template <typename real>
__global__ void binomial_pass_kernel(Geom g, int axis, const real *__restrict__ src, real *__restrict__ dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    const int k = blockIdx.z;
    if (i >= g.n[0]) return;
    const int fx = i + g.mem, fy = j + g.mem, fz = k + g.mem;
    const long long at = g.ri(fz, fy, fx);
    const long long step = axis == 0 ? 1 : (axis == 1 ? (long long)g.r[0] : (long long)g.rxy);
    const real a = src[at - step], b = src[at], cc = src[at + step];
    dst[at] = (real(0.25) * a + real(0.5) * b) + real(0.25) * cc;
}

void launch_binomial_pass(pic_ctx *c, int ring_index, int axis, void *scratch) {
    const Geom &g = c->g;
    const size_t bytes = (size_t)g.rsz * (c->fp32 ? 4 : 8);
    cudaMemcpyAsync(scratch, c->ring[ring_index], bytes, cudaMemcpyDeviceToDevice, c->stream);
    dim3 grd((unsigned)((g.n[0] + 127) / 128), (unsigned)g.n[1], (unsigned)g.n[2]);
    prof_begin(c, "binomial_filter");
    if (c->fp32)
        binomial_pass_kernel<float><<<grd, 128, 0, c->stream>>>(g, axis, (const float *)scratch,
                                                                 (float *)c->ring[ring_index]);
    else
        binomial_pass_kernel<double><<<grd, 128, 0, c->stream>>>(g, axis, (const double *)scratch,
                                                                  (double *)c->ring[ring_index]);
    prof_end(c);
}

template <typename real>
static void rb(pic_ctx *c, const LaserArgs &L) {
    const Geom &g = c->g;
    dim3 blk(32, 8), grd((g.n[1] + 31) / 32, (g.n[2] + 7) / 8);
    real **F = (real **)c->field;
    real **R = (real **)c->ring;
    radiating_boundary_kernel<real><<<grd, blk, 0, c->stream>>>(g, L, F[1], F[2], F[3], F[4], F[5], R[1], R[2]);
}

static LaserArgs laser_args(const pic_ctx *c, double time) {
    const PicParams &p = c->p;
    LaserArgs L{};
    L.Pi = p.Pi; L.omega = p.omega; L.l0 = p.l0; L.Lx = p.Lx; L.dt = p.dt; L.dx = p.dx; L.dy = p.dy; L.dz = p.dz;
    L.amp = p.laser_amplitude; L.dur = p.laser_pulse_duration; L.start = p.laser_start_time;
    L.waist = p.waist; L.xfocus = p.xfocus; L.yfocus = p.yfocus; L.zfocus = p.zfocus; L.phase = p.phase;
    L.pol = p.laser_polarization; L.envelope = p.laser_envelope;
    L.profile = (p.laser_profile == 1 && c->d_profile) ? 1 : 0;
    L.profile_n = c->profile_n; L.coef = c->d_profile;
    L.time = time;
    L.absorbing = p.absorbing == 1 ? 1 : 0;
    return L;
}

void launch_radiating_boundary(pic_ctx *c, int is_left, int is_right, int step) {
    if (!c->p.rank_period[0]) {   // periodic x: both x faces have a neighbour, nothing written
        LaserArgs L = laser_args(c, step * c->p.dt);
        L.is_left = is_left; L.is_right = is_right;
        prof_begin(c, "radiating_boundary");
        if (c->fp32) rb<float>(c, L); else rb<double>(c, L);
        prof_end(c);
    }
    launch_absorbing_faces(c);   // extension: the other non-periodic faces, same point of the step
}

// ---------------------------------------------------------------------------
// Device evaluation of the reference's scalar helpers with the same device
// code the kernels use: shape_function_2 / _4 (src/particle.cpp:8-48) at an
// absolute buffer coordinate, g_factor (:603-637), generate_laser_pulse and
// Gpulse (src/boundary.cpp:8-40, Gaussian transverse factor).
__global__ void eval_kernel(Geom g, LaserArgs L, const double *tab, int tab_n, int what, double a0, double a1,
                            double a2, double a3, double *out, unsigned *status) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    switch (what) {
        case 0: {   // quadratic shape at x: delta from the nearest node (int)(x + 0.5)
            double w[3];
            shape_weights(a0 - (double)(int)(a0 + 0.5), w);
            for (int q = 0; q < 3; ++q) out[q] = w[q];
            break;
        }
        case 1: {   // quartic shape
            double w[5];
            shape_weights(a0 - (double)(int)(a0 + 0.5), w);
            for (int q = 0; q < 5; ++q) out[q] = w[q];
            break;
        }
        case 2:     // g factor: out of the table's range is reported through status
            out[0] = g_factor_dev(tab, tab_n, a0, status);
            break;
        case 3:     // envelope (time, position)
            out[0] = laser_envelope(L, a0, a1);
            break;
        case 4:     // Gpulse(time, x, y, z)
            L.time = a0;
            L.profile = 0;
            out[0] = gpulse(L, g, a0, a1, a2, a3, 0, 0);
            break;
    }
}

int launch_eval(pic_ctx *c, int what, const double *in, double *d_out) {
    LaserArgs L = laser_args(c, 0.0);
    eval_kernel<<<1, 32, 0, c->stream>>>(c->g, L, c->d_gtab, c->gtab_n, what, in[0], in[1], in[2], in[3], d_out,
                                         c->d_status);
    return 0;
}

}  // namespace pic
