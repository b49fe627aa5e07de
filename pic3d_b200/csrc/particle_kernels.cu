// Particle kernels: fused field gather + relativistic Boris push + move +
// Esirkepov current deposition (+ per-species rho, + optional electron spin
// precession), removal at absorbing faces, and conversion between the
// reference's 144-byte particle records and the device structure of arrays.
//
// One thread per particle.  The gather reads the six staggered field
// components through the read-only path; the deposit adds J (and rho) with
// hardware atomics into the ring buffers, which the fold kernel then
// completes for periodic faces exactly as the reference's ghost exchange.
#include <cuda/std/type_traits>

#include "pic_kernels.cuh"

namespace pic {

template <typename real>
struct PushArgs {
    Geom g;
    const real *ex, *ey, *ez, *bx, *by, *bz;
    real *jx, *jy, *jz, *rho;
    const long long *count;
    // FP64 positions (cur -> nxt)
    double *x0, *y0, *z0;
    double *x1, *y1, *z1;
    // FP32 positions
    int *c0;
    const float *ox0, *oy0, *oz0;
    int *c1;
    float *ox1, *oy1, *oz1;
    CellPack cp;
    real *px, *py, *pz;
    const real *w;
    real *sx, *sy, *sz;
    const double *gtab;
    int gtab_n;
    real qm;                 // charge / mass * dt_half (particle.cpp:271)
    real charge;
    real dt_d[3];            // dt / dx, dt / dy, dt / dz
    double dt_s, dxs[3];     // dt and dx, dy, dz
    real d_dt[3];            // dx / dt, dy / dt, dz / dt (particle.cpp:423-425)
    double E_schwinger, dt_half_d, charge_d, mass_d;
    int electron;            // mass == m_e: spin precession applies (particle.cpp:319)
    unsigned *status;
};

__device__ __forceinline__ void set_status(unsigned *s, unsigned bit) { atomicOr(s, bit); }

// g_factor lookup (src/particle.cpp:603-637)
__device__ double g_factor_dev(const double *tab, int n, double x, unsigned *status) {
    int idx;
    if (x < 0.005 && x >= 0.0) return 2.003219;
    if (x >= 0.005 && x < 0.01) idx = (int)((x - 0.005) / 0.0001);
    else if (x >= 0.01 && x < 1) idx = (int)((x - 0.01) / 0.01) + 50;
    else if (x >= 1 && x < 10) idx = (int)((x - 1.0) / 0.01) + 150;
    else if (x >= 10 && x < 20) idx = (int)((x - 10.0) / 0.01) + 1050;
    else if (x >= 20 && x <= 100) idx = (int)((x - 20.0) / 0.1) + 2050;
    else { set_status(status, ST_RANGE); return 2.003219; }
    if (!tab || idx < 0 || idx >= n) { set_status(status, ST_RANGE); return 2.003219; }
    return tab[idx];
}

// factorised P^3 gather of one staggered component
template <typename real, int P>
__device__ __forceinline__ real gather(const real *__restrict__ f, const Geom &g, int i0, int j0, int k0,
                                       const real (&wx)[P], const real (&wy)[P], const real (&wz)[P]) {
    const real *base = f + g.fi(k0, j0, i0);
    real acc = 0;
#pragma unroll
    for (int k = 0; k < P; ++k) {
        real acck = 0;
#pragma unroll
        for (int j = 0; j < P; ++j) {
            const real *row = base + k * g.fxy + j * g.f[0];
            real s = 0;
#pragma unroll
            for (int i = 0; i < P; ++i) s += wx[i] * __ldg(row + i);
            acck += wy[j] * s;
        }
        acc += wz[k] * acck;
    }
    return acc;
}

// 1D pieces of the Esirkepov weights over the union span of the old and new
// supports (src/particle.cpp:403-419): s0 = old shape, ds = new - old,
// zero outside each support.  |i2 - i1| <= 1 (checked by the caller).
template <typename real, int P>
__device__ __forceinline__ void span1d(int i1, const real (&w0)[P], int i2, const real (&w1)[P], int &base,
                                       int &len, real (&s0)[P + 1], real (&ds)[P + 1]) {
    constexpr int H = P / 2;
    const int lo = min(i1, i2);
    base = lo - H;
    len = P + abs(i2 - i1);
    const bool o0 = i1 != lo, o1 = i2 != lo;
#pragma unroll
    for (int a = 0; a <= P; ++a) {
        real v0 = o0 ? (a >= 1 ? w0[a - 1] : real(0)) : (a < P ? w0[a] : real(0));
        real v1 = o1 ? (a >= 1 ? w1[a - 1] : real(0)) : (a < P ? w1[a] : real(0));
        s0[a] = v0;
        ds[a] = v1 - v0;
    }
}

__device__ __forceinline__ void atomic_add(double *p, double v) { atomicAdd(p, v); }
__device__ __forceinline__ void atomic_add(float *p, float v) { atomicAdd(p, v); }

// Esirkepov deposit (src/particle.cpp:427-500) and rho (:503-514)
template <typename real, int P>
__device__ __forceinline__ void deposit(const PushArgs<real> &a, const int (&i1)[3], const real (&w0)[3][P],
                                        const int (&i2)[3], const real (&w1)[3][P], real qw) {
    constexpr int H = P / 2;
    const Geom &g = a.g;
    int base[3], len[3];
    real s0[3][P + 1], ds[3][P + 1];
#pragma unroll
    for (int d = 0; d < 3; ++d) span1d<real, P>(i1[d], w0[d], i2[d], w1[d], base[d], len[d], s0[d], ds[d]);
    const real third = real(1.0 / 3.0), half = real(0.5);
    const real cx = qw * a.d_dt[0], cy = qw * a.d_dt[1], cz = qw * a.d_dt[2];
    const int rx = g.r[0], rxy = g.rxy;
    const int r0 = g.ri(base[2], base[1], base[0]);
    // Jx: running sum of ds along x times the yz weight
#pragma unroll
    for (int k = 0; k <= P; ++k) {
        if (k >= len[2]) break;
#pragma unroll
        for (int j = 0; j <= P; ++j) {
            if (j >= len[1]) break;
            real wyz = s0[1][j] * s0[2][k] + half * ds[1][j] * s0[2][k] + half * s0[1][j] * ds[2][k] +
                       third * ds[1][j] * ds[2][k];
            real acc = 0;
            real *row = a.jx + r0 + k * rxy + j * rx;
#pragma unroll
            for (int i = 0; i < P; ++i) {
                if (i >= len[0] - 1) break;
                acc += ds[0][i];
                atomic_add(row + i, -cx * acc * wyz);
            }
        }
    }
    // Jy
#pragma unroll
    for (int k = 0; k <= P; ++k) {
        if (k >= len[2]) break;
#pragma unroll
        for (int i = 0; i <= P; ++i) {
            if (i >= len[0]) break;
            real wxz = s0[0][i] * s0[2][k] + half * ds[0][i] * s0[2][k] + half * s0[0][i] * ds[2][k] +
                       third * ds[0][i] * ds[2][k];
            real acc = 0;
            real *col = a.jy + r0 + k * rxy + i;
#pragma unroll
            for (int j = 0; j < P; ++j) {
                if (j >= len[1] - 1) break;
                acc += ds[1][j];
                atomic_add(col + j * rx, -cy * acc * wxz);
            }
        }
    }
    // Jz
#pragma unroll
    for (int j = 0; j <= P; ++j) {
        if (j >= len[1]) break;
#pragma unroll
        for (int i = 0; i <= P; ++i) {
            if (i >= len[0]) break;
            real wxy = s0[0][i] * s0[1][j] + half * ds[0][i] * s0[1][j] + half * s0[0][i] * ds[1][j] +
                       third * ds[0][i] * ds[1][j];
            real acc = 0;
            real *col = a.jz + r0 + j * rx + i;
#pragma unroll
            for (int k = 0; k < P; ++k) {
                if (k >= len[2] - 1) break;
                acc += ds[2][k];
                atomic_add(col + k * rxy, -cz * acc * wxy);
            }
        }
    }
    if (a.rho) {
        real *rb = a.rho + g.ri(i2[2] - H, i2[1] - H, i2[0] - H);
#pragma unroll
        for (int k = 0; k < P; ++k)
#pragma unroll
            for (int j = 0; j < P; ++j) {
                real wjk = qw * w1[1][j] * w1[2][k];
#pragma unroll
                for (int i = 0; i < P; ++i) atomic_add(rb + k * rxy + j * rx + i, wjk * w1[0][i]);
            }
    }
}

template <typename real, int P, bool SPIN>
__global__ void __launch_bounds__(256) push_kernel(PushArgs<real> a) {
    constexpr bool F64 = cuda::std::is_same<real, double>::value;
    constexpr int H = P / 2;
    const Geom &g = a.g;
    const long long n = *a.count;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n;
         p += (long long)gridDim.x * blockDim.x) {
        // ---- position -> primal / dual index and offset per axis --------
        int ip[3], id[3];
        real dp[3], dd[3];
        double xd[3];   // FP64: wrapped absolute position
        int cc[3];      // FP32: cell
        real oo[3];     // FP32: offset
        if constexpr (F64) {
            xd[0] = a.x0[p];
            xd[1] = a.y0[p];
            xd[2] = a.z0[p];
            bool wrapped = false;
            // periodic wrap at push time (particle.cpp:123-167)
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                if (g.per[d]) {
                    if (xd[d] < 0.0) { xd[d] += g.n[d]; wrapped = true; }
                    if (xd[d] > (double)g.n[d]) { xd[d] -= g.n[d]; wrapped = true; }
                }
            }
            if (wrapped) {
                a.x0[p] = xd[0];
                a.y0[p] = xd[1];
                a.z0[p] = xd[2];
            }
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                double xc = xd[d] - (double)(1 - g.mem);
                ip[d] = (int)(xc + 0.5);
                dp[d] = xc - (double)ip[d];
                id[d] = (int)xc;
                dd[d] = (xc - 0.5) - (double)id[d];
            }
        } else {
            a.cp.unpack(a.c0[p], cc[0], cc[1], cc[2]);
            oo[0] = a.ox0[p];
            oo[1] = a.oy0[p];
            oo[2] = a.oz0[p];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                int b = cc[d] + g.mem - 1;
                bool up = oo[d] >= 0.5f;
                ip[d] = b + (up ? 1 : 0);
                dp[d] = up ? oo[d] - 1.0f : oo[d];
                id[d] = b;
                dd[d] = oo[d] - 0.5f;
            }
        }
        bool ok = true;
#pragma unroll
        for (int d = 0; d < 3; ++d) ok = ok && id[d] >= H && ip[d] <= g.f[d] - 1 - H;
        if (!ok) {
            set_status(a.status, ST_OOB);
            continue;
        }
        real wp[3][P], wd[3][P];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            shape_weights(dp[d], wp[d]);
            shape_weights(dd[d], wd[d]);
        }
        // ---- gather with Yee staggering (particle.cpp:207-259) ----------
        real e0 = gather<real, P>(a.ex, g, id[0] - H, ip[1] - H, ip[2] - H, wd[0], wp[1], wp[2]);
        real e1 = gather<real, P>(a.ey, g, ip[0] - H, id[1] - H, ip[2] - H, wp[0], wd[1], wp[2]);
        real e2 = gather<real, P>(a.ez, g, ip[0] - H, ip[1] - H, id[2] - H, wp[0], wp[1], wd[2]);
        real b0 = gather<real, P>(a.bx, g, ip[0] - H, id[1] - H, id[2] - H, wp[0], wd[1], wd[2]);
        real b1 = gather<real, P>(a.by, g, id[0] - H, ip[1] - H, id[2] - H, wd[0], wp[1], wd[2]);
        real b2 = gather<real, P>(a.bz, g, id[0] - H, id[1] - H, ip[2] - H, wd[0], wd[1], wp[2]);
        // ---- Boris (particle.cpp:271-306) --------------------------------
        const real qm = a.qm;
        real ex_p = e0 * qm, ey_p = e1 * qm, ez_p = e2 * qm;
        real bx_p = b0 * qm, by_p = b1 * qm, bz_p = b2 * qm;
        real px1 = a.px[p] + ex_p, py1 = a.py[p] + ey_p, pz1 = a.pz[p] + ez_p;
        real gm1 = sqrt(real(1) + (px1 * px1 + py1 * py1 + pz1 * pz1));
        real tx = bx_p / gm1, ty = by_p / gm1, tz = bz_p / gm1;
        real tt = real(2) / (real(1) + tx * tx + ty * ty + tz * tz);
        real sx = tx * tt, sy = ty * tt, sz = tz * tt;
        real px2 = px1 + (py1 * tz - pz1 * ty);
        real py2 = py1 + (pz1 * tx - px1 * tz);
        real pz2 = pz1 + (px1 * ty - py1 * tx);
        real pxn = px1 + (py2 * sz - pz2 * sy) + ex_p;
        real pyn = py1 + (pz2 * sx - px2 * sz) + ey_p;
        real pzn = pz1 + (px2 * sy - py2 * sx) + ez_p;
        real gam = sqrt(real(1) + (pxn * pxn + pyn * pyn + pzn * pzn));
        // ---- move in cell units (particle.cpp:313-315) -------------------
        const real disp[3] = {pxn / gam * a.dt_d[0], pyn / gam * a.dt_d[1], pzn / gam * a.dt_d[2]};
        int i2[3];
        real d2[3];
        double xn[3];
        int cn[3];
        real on[3];
        if constexpr (F64) {
            // x = x_old + px / gamma * dt / dx in the reference's order
            xn[0] = xd[0] + (double)pxn / (double)gam * a.dt_s / a.dxs[0];
            xn[1] = xd[1] + (double)pyn / (double)gam * a.dt_s / a.dxs[1];
            xn[2] = xd[2] + (double)pzn / (double)gam * a.dt_s / a.dxs[2];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                double xc = xn[d] - (double)(1 - g.mem);
                i2[d] = (int)(xc + 0.5);
                d2[d] = xc - (double)i2[d];
            }
        } else {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                real o = oo[d] + disp[d];
                int s = 0;
                if (o >= real(1)) { o -= real(1); s = 1; }
                else if (o < real(0)) {
                    o += real(1);
                    s = -1;
                    if (o >= real(1)) { o = real(0); s = 0; }
                }
                cn[d] = cc[d] + s;
                on[d] = o;
                int b = cn[d] + g.mem - 1;
                bool up = o >= real(0.5);
                i2[d] = b + (up ? 1 : 0);
                d2[d] = up ? o - real(1) : o;
            }
        }
        bool fin = isfinite(pxn) && isfinite(pyn) && isfinite(pzn);
        bool cfl = abs(i2[0] - ip[0]) <= 1 && abs(i2[1] - ip[1]) <= 1 && abs(i2[2] - ip[2]) <= 1;
        if (!fin || !cfl) {
            set_status(a.status, fin ? ST_CFL : ST_NAN);
            continue;
        }
        real w1[3][P];
#pragma unroll
        for (int d = 0; d < 3; ++d) shape_weights(d2[d], w1[d]);
        const real qw = a.charge * a.w[p];
        deposit<real, P>(a, ip, wp, i2, w1, qw);
        // ---- store --------------------------------------------------------
        a.px[p] = pxn;
        a.py[p] = pyn;
        a.pz[p] = pzn;
        if constexpr (F64) {
            a.x1[p] = xn[0];
            a.y1[p] = xn[1];
            a.z1[p] = xn[2];
        } else {
#pragma unroll
            for (int d = 0; d < 3; ++d)
                if (g.per[d]) cn[d] = cn[d] < 0 ? cn[d] + g.n[d] : (cn[d] >= g.n[d] ? cn[d] - g.n[d] : cn[d]);
            a.c1[p] = a.cp.pack(cn[0], cn[1], cn[2]);
            a.ox1[p] = on[0];
            a.oy1[p] = on[1];
            a.oz1[p] = on[2];
        }
        // ---- electron spin precession (particle.cpp:318-368) --------------
        if constexpr (SPIN) {
            if (a.electron) {
                double exq = e0, eyq = e1, ezq = e2, bxq = b0, byq = b1, bzq = b2;
                double g0 = gam;
                double vx = (double)pxn / g0, vy = (double)pyn / g0, vz = (double)pzn / g0;
                double pe = vx * exq + vy * eyq + vz * ezq;
                double fx = exq + vy * bzq - vz * byq;
                double fy = eyq + vz * bxq - vx * bzq;
                double fz = ezq + vx * byq - vy * bxq;
                double chi = fx * fx + fy * fy + fz * fz - pe * pe;
                chi = chi > 0.0 ? chi : 0.0;
                chi = sqrt(chi) / a.E_schwinger * g0;
                double gf = g_factor_dev(a.gtab, a.gtab_n, chi, a.status);
                double al = -(gf / 2.0 - 1.0) * g0 / (1.0 + g0);
                double be = (gf / 2.0 - 1.0) + 1.0 / g0;
                double gg = gf / 2.0 - g0 / (1.0 + g0);
                double vb = vx * bxq + vy * byq + vz * bzq;
                double ox = al * vb * vx + be * bxq + gg * (vy * ezq - vz * eyq);
                double oy = al * vb * vy + be * byq + gg * (vz * exq - vx * ezq);
                double oz = al * vb * vz + be * bzq + gg * (vx * eyq - vy * exq);
                double q2 = a.charge_d / a.mass_d * a.dt_half_d;
                double ux = ox * q2, uy = oy * q2, uz = oz * q2;
                double t2 = 2.0 / (1.0 + ux * ux + uy * uy + uz * uz);
                double s_x = a.sx[p], s_y = a.sy[p], s_z = a.sz[p];
                double rx = s_x + (s_y * uz - s_z * uy);
                double ry = s_y + (s_z * ux - s_x * uz);
                double rz = s_z + (s_x * uy - s_y * ux);
                a.sx[p] = (real)(s_x + (ry * uz - rz * uy) * t2);
                a.sy[p] = (real)(s_y + (rz * ux - rx * uz) * t2);
                a.sz[p] = (real)(s_z + (rx * uy - ry * ux) * t2);
            }
        }
    }
}

// ---------------------------------------------------------------------------

static int sm_count(pic_ctx *c) {
    static int n = 0;
    if (!n) cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, c->device);
    return n ? n : 148;
}

template <typename real, int P, bool SPIN>
static void push_t(pic_ctx *c, int kind) {
    Species &s = c->sp[kind];
    PushArgs<real> a{};
    a.g = c->g;
    real **F = (real **)c->field;
    real **R = (real **)c->ring;
    a.ex = F[0]; a.ey = F[1]; a.ez = F[2]; a.bx = F[3]; a.by = F[4]; a.bz = F[5];
    a.jx = R[0]; a.jy = R[1]; a.jz = R[2];
    a.rho = c->p.deposit_rho ? R[3 + kind] : nullptr;
    a.count = s.d_count;
    int cu = s.cur, nx = 1 - s.cur;
    a.x0 = s.x[cu]; a.y0 = s.y[cu]; a.z0 = s.z[cu];
    a.x1 = s.x[nx]; a.y1 = s.y[nx]; a.z1 = s.z[nx];
    a.c0 = s.cell[cu]; a.ox0 = s.ox[cu]; a.oy0 = s.oy[cu]; a.oz0 = s.oz[cu];
    a.c1 = s.cell[nx]; a.ox1 = s.ox[nx]; a.oy1 = s.oy[nx]; a.oz1 = s.oz[nx];
    a.cp = c->cp;
    a.px = (real *)s.px; a.py = (real *)s.py; a.pz = (real *)s.pz; a.w = (const real *)s.w;
    a.sx = (real *)s.sx; a.sy = (real *)s.sy; a.sz = (real *)s.sz;
    a.gtab = c->d_gtab; a.gtab_n = c->gtab_n;
    const PicParams &p = c->p;
    a.qm = (real)(p.charge[kind] / p.mass[kind] * p.dt_half);
    a.charge = (real)p.charge[kind];
    a.dt_d[0] = (real)(p.dt / p.dx); a.dt_d[1] = (real)(p.dt / p.dy); a.dt_d[2] = (real)(p.dt / p.dz);
    a.dt_s = p.dt; a.dxs[0] = p.dx; a.dxs[1] = p.dy; a.dxs[2] = p.dz;
    a.d_dt[0] = (real)(p.dx / p.dt); a.d_dt[1] = (real)(p.dy / p.dt); a.d_dt[2] = (real)(p.dz / p.dt);
    a.E_schwinger = p.E_schwinger; a.dt_half_d = p.dt_half; a.charge_d = p.charge[kind]; a.mass_d = p.mass[kind];
    a.electron = p.mass[kind] == 1.0;
    a.status = c->d_status;
    long long n = s.n_host;
    if (n > 0) {
        long long blocks = (n + 255) / 256;
        long long maxb = (long long)sm_count(c) * 8;
        push_kernel<real, P, SPIN><<<(unsigned)(blocks < maxb ? blocks : maxb), 256, 0, c->stream>>>(a);
    }
    s.cur = nx;
}

void launch_push(pic_ctx *c, int kind) {
    Species &s = c->sp[kind];
    bool spin = c->p.spin && s.sx && s.spin_nonzero && c->p.mass[kind] == 1.0;
    prof_begin(c, "push_gather_deposit");
    if (c->fp32) {
        if (c->order == 2) spin ? push_t<float, 3, true>(c, kind) : push_t<float, 3, false>(c, kind);
        else spin ? push_t<float, 5, true>(c, kind) : push_t<float, 5, false>(c, kind);
    } else {
        if (c->order == 2) spin ? push_t<double, 3, true>(c, kind) : push_t<double, 3, false>(c, kind);
        else spin ? push_t<double, 5, true>(c, kind) : push_t<double, 5, false>(c, kind);
    }
    prof_end(c);
}

// ---------------------------------------------------------------------------
// Removal at non-periodic global faces (the only effect of
// exchange_particle_data, src/mpi_utils.cpp:62-230, on one rank): a particle
// with x < 0 or x >= n along a non-periodic axis is dropped.  Holes below the
// new count are filled from survivors above it (order is not preserved).

struct RemoveArgs {
    Geom g;
    CellPack cp;
    int fp32;
    long long *count;         // in/out
    long long *ctr;           // [0] removed, [1] holes, [2] movers
    int *holes, *movers;
    const double *x, *y, *z;
    const int *cell;
};

__device__ __forceinline__ bool is_dead(const RemoveArgs &a, long long i) {
    if (a.fp32) {
        int cx, cy, cz;
        a.cp.unpack(a.cell[i], cx, cy, cz);
        int c[3] = {cx, cy, cz};
        bool dead = false;
#pragma unroll
        for (int d = 0; d < 3; ++d)
            if (!a.g.per[d]) dead = dead || c[d] < 0 || c[d] >= a.g.n[d];
        return dead;
    }
    double c[3] = {a.x[i], a.y[i], a.z[i]};
    bool dead = false;
#pragma unroll
    for (int d = 0; d < 3; ++d)
        if (!a.g.per[d]) dead = dead || c[d] < 0.0 || c[d] >= (double)a.g.n[d];
    return dead;
}

__global__ void count_dead_kernel(RemoveArgs a) {
    long long n = *a.count;
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    bool dead = i < n && is_dead(a, i);
    unsigned m = __ballot_sync(0xffffffffu, dead);
    if ((threadIdx.x & 31) == 0 && m) atomicAdd((unsigned long long *)&a.ctr[0], (unsigned long long)__popc(m));
}

__global__ void list_moves_kernel(RemoveArgs a) {
    long long n = *a.count;
    long long nn = n - a.ctr[0];
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    bool dead = is_dead(a, i);
    if (i < nn && dead) a.holes[atomicAdd((unsigned long long *)&a.ctr[1], 1ull)] = (int)i;
    if (i >= nn && !dead) a.movers[atomicAdd((unsigned long long *)&a.ctr[2], 1ull)] = (int)i;
}

template <typename T>
__device__ __forceinline__ void mv(T *p, int dst, int src) {
    if (p) p[dst] = p[src];
}

struct MoveArgs {
    long long *ctr;
    long long *count;
    const int *holes, *movers;
    double *d[16];
    float *f[16];
    int *i[3];
};

__global__ void apply_moves_kernel(MoveArgs a) {
    long long m = a.ctr[2];
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    int dst = a.holes[t], src = a.movers[t];
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        mv(a.d[k], dst, src);
        mv(a.f[k], dst, src);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) mv(a.i[k], dst, src);
}

__global__ void finish_remove_kernel(long long *count, long long *ctr) {
    *count = *count - ctr[0];
}

void launch_remove(pic_ctx *c, int kind) {
    const Geom &g = c->g;
    if (g.per[0] && g.per[1] && g.per[2]) return;
    Species &s = c->sp[kind];
    long long n = s.n_host;
    if (n == 0) return;
    prof_begin(c, "remove_particles");
    RemoveArgs a{};
    a.g = g;
    a.cp = c->cp;
    a.fp32 = c->fp32;
    a.count = s.d_count;
    a.ctr = c->d_scratch_ll;
    a.holes = c->d_list;
    a.movers = c->d_list + c->list_cap / 2;
    int cu = s.cur;
    a.x = s.x[cu]; a.y = s.y[cu]; a.z = s.z[cu];
    a.cell = s.cell[cu];
    cudaMemsetAsync(c->d_scratch_ll, 0, 3 * sizeof(long long), c->stream);
    unsigned blocks = (unsigned)((n + 255) / 256);
    count_dead_kernel<<<blocks, 256, 0, c->stream>>>(a);
    list_moves_kernel<<<blocks, 256, 0, c->stream>>>(a);
    MoveArgs m{};
    m.ctr = a.ctr;
    m.count = s.d_count;
    m.holes = a.holes;
    m.movers = a.movers;
    int k = 0, kf = 0;
    for (int b = 0; b < 2; ++b) {
        if (c->fp32) {
            m.f[kf++] = s.ox[b]; m.f[kf++] = s.oy[b]; m.f[kf++] = s.oz[b];
        } else {
            m.d[k++] = s.x[b]; m.d[k++] = s.y[b]; m.d[k++] = s.z[b];
        }
    }
    void *mom[7] = {s.px, s.py, s.pz, s.w, s.sx, s.sy, s.sz};
    for (void *v : mom) {
        if (!v) continue;
        if (c->fp32) m.f[kf++] = (float *)v; else m.d[k++] = (double *)v;
    }
    m.i[0] = s.id;
    m.i[1] = s.cell[0];
    m.i[2] = s.cell[1];
    (void)k;
    apply_moves_kernel<<<blocks, 256, 0, c->stream>>>(m);
    finish_remove_kernel<<<1, 1, 0, c->stream>>>(s.d_count, c->d_scratch_ll);
    prof_end(c);
}

// ---------------------------------------------------------------------------
// reference record <-> structure of arrays

struct Rec {
    int id, pad0;
    double x, y, z, x_old, y_old, z_old, px, py, pz, sx, sy, sz, gamma, charge, mass, weight;
    int rank, pad1;
};
static_assert(sizeof(Rec) == 144, "reference particle record");

struct ConvArgs {
    Geom g;
    CellPack cp;
    int fp32;
    long long n, off;
    Rec *rec;
    int cur;
    double *x[2], *y[2], *z[2];
    int *cell[2];
    float *ox[2], *oy[2], *oz[2];
    void *px, *py, *pz, *w, *sx, *sy, *sz;
    int *id;
    double charge, mass;
};

__device__ void to_cell(const Geom &g, const CellPack &cp, int per_wrap, double x, double y, double z, int &cell,
                        float &ox, float &oy, float &oz) {
    double v[3] = {x, y, z};
    int c[3];
    float o[3];
    for (int d = 0; d < 3; ++d) {
        double f = floor(v[d]);
        float r = (float)(v[d] - f);
        int ci = (int)f;
        if (r >= 1.0f) { r = 0.0f; ci += 1; }
        if (per_wrap && g.per[d]) { ci %= g.n[d]; if (ci < 0) ci += g.n[d]; }
        c[d] = ci;
        o[d] = r;
    }
    cell = cp.pack(c[0], c[1], c[2]);
    ox = o[0];
    oy = o[1];
    oz = o[2];
}

__global__ void records_to_soa_kernel(ConvArgs a) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.n) return;
    const Rec r = a.rec[t];
    long long i = a.off + t;
    int cu = a.cur, pv = 1 - a.cur;
    if (a.fp32) {
        to_cell(a.g, a.cp, 1, r.x, r.y, r.z, a.cell[cu][i], a.ox[cu][i], a.oy[cu][i], a.oz[cu][i]);
        to_cell(a.g, a.cp, 1, r.x_old, r.y_old, r.z_old, a.cell[pv][i], a.ox[pv][i], a.oy[pv][i], a.oz[pv][i]);
        ((float *)a.px)[i] = (float)r.px;
        ((float *)a.py)[i] = (float)r.py;
        ((float *)a.pz)[i] = (float)r.pz;
        ((float *)a.w)[i] = (float)r.weight;
        if (a.sx) {
            ((float *)a.sx)[i] = (float)r.sx;
            ((float *)a.sy)[i] = (float)r.sy;
            ((float *)a.sz)[i] = (float)r.sz;
        }
    } else {
        a.x[cu][i] = r.x; a.y[cu][i] = r.y; a.z[cu][i] = r.z;
        a.x[pv][i] = r.x_old; a.y[pv][i] = r.y_old; a.z[pv][i] = r.z_old;
        ((double *)a.px)[i] = r.px;
        ((double *)a.py)[i] = r.py;
        ((double *)a.pz)[i] = r.pz;
        ((double *)a.w)[i] = r.weight;
        if (a.sx) {
            ((double *)a.sx)[i] = r.sx;
            ((double *)a.sy)[i] = r.sy;
            ((double *)a.sz)[i] = r.sz;
        }
    }
    a.id[i] = r.id;
}

__global__ void soa_to_records_kernel(ConvArgs a) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.n) return;
    long long i = a.off + t;
    int cu = a.cur, pv = 1 - a.cur;
    Rec r;
    r.id = a.id[i];
    r.pad0 = 0;
    double px, py, pz;
    if (a.fp32) {
        int cx, cy, cz;
        a.cp.unpack(a.cell[cu][i], cx, cy, cz);
        r.x = (double)cx + (double)a.ox[cu][i];
        r.y = (double)cy + (double)a.oy[cu][i];
        r.z = (double)cz + (double)a.oz[cu][i];
        a.cp.unpack(a.cell[pv][i], cx, cy, cz);
        r.x_old = (double)cx + (double)a.ox[pv][i];
        r.y_old = (double)cy + (double)a.oy[pv][i];
        r.z_old = (double)cz + (double)a.oz[pv][i];
        px = ((float *)a.px)[i];
        py = ((float *)a.py)[i];
        pz = ((float *)a.pz)[i];
        r.weight = ((float *)a.w)[i];
        r.sx = a.sx ? ((float *)a.sx)[i] : 0.0;
        r.sy = a.sy ? ((float *)a.sy)[i] : 0.0;
        r.sz = a.sz ? ((float *)a.sz)[i] : 0.0;
    } else {
        r.x = a.x[cu][i]; r.y = a.y[cu][i]; r.z = a.z[cu][i];
        r.x_old = a.x[pv][i]; r.y_old = a.y[pv][i]; r.z_old = a.z[pv][i];
        px = ((double *)a.px)[i];
        py = ((double *)a.py)[i];
        pz = ((double *)a.pz)[i];
        r.weight = ((double *)a.w)[i];
        r.sx = a.sx ? ((double *)a.sx)[i] : 0.0;
        r.sy = a.sy ? ((double *)a.sy)[i] : 0.0;
        r.sz = a.sz ? ((double *)a.sz)[i] : 0.0;
    }
    r.px = px;
    r.py = py;
    r.pz = pz;
    // gamma as the push computes it (particle.cpp:309-311), without contraction
    r.gamma = __dsqrt_rn(__dadd_rn(1.0, __dadd_rn(__dadd_rn(__dmul_rn(px, px), __dmul_rn(py, py)), __dmul_rn(pz, pz))));
    r.charge = a.charge;
    r.mass = a.mass;
    r.rank = 0;
    r.pad1 = 0;
    a.rec[t] = r;
}

static ConvArgs conv_args(pic_ctx *c, int kind, void *rec, int64_t n, int64_t off) {
    Species &s = c->sp[kind];
    ConvArgs a{};
    a.g = c->g;
    a.cp = c->cp;
    a.fp32 = c->fp32;
    a.n = n;
    a.off = off;
    a.rec = (Rec *)rec;
    a.cur = s.cur;
    for (int b = 0; b < 2; ++b) {
        a.x[b] = s.x[b]; a.y[b] = s.y[b]; a.z[b] = s.z[b];
        a.cell[b] = s.cell[b]; a.ox[b] = s.ox[b]; a.oy[b] = s.oy[b]; a.oz[b] = s.oz[b];
    }
    a.px = s.px; a.py = s.py; a.pz = s.pz; a.w = s.w;
    a.sx = s.sx; a.sy = s.sy; a.sz = s.sz;
    a.id = s.id;
    a.charge = c->p.charge[kind];
    a.mass = c->p.mass[kind];
    return a;
}

void launch_upload_particles(pic_ctx *c, int kind, const void *d_records, int64_t n, int64_t offset) {
    if (n <= 0) return;
    ConvArgs a = conv_args(c, kind, (void *)d_records, n, offset);
    records_to_soa_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(a);
}

void launch_download_particles(pic_ctx *c, int kind, void *d_records, int64_t n, int64_t offset) {
    if (n <= 0) return;
    ConvArgs a = conv_args(c, kind, d_records, n, offset);
    soa_to_records_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(a);
}

__global__ void convert_kernel(float *f, double *d, long long n, int to_float) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (to_float) f[i] = (float)d[i];
    else d[i] = (double)f[i];
}

// FP32 contexts: dst/src between a device float array and FP64 staging
void launch_convert_array(pic_ctx *c, void *dst, const void *src, long long n, int to_device) {
    unsigned b = (unsigned)((n + 255) / 256);
    if (to_device) convert_kernel<<<b, 256, 0, c->stream>>>((float *)dst, (double *)src, n, 1);
    else convert_kernel<<<b, 256, 0, c->stream>>>((float *)src, (double *)dst, n, 0);
}

}  // namespace pic
