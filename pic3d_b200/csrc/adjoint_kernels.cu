// Hand-written adjoint of the per-timestep loop (no counterpart in the
// reference), for gradients of a final-state objective with respect to the
// particle weights (hence a density profile) and the laser's transverse
// amplitude coefficients.
//
// Forward step n (absorbing faces):  BC(t_n) -> E half -> B half -> clear J ->
// push+deposit -> removal -> B half -> E half.  The adjoint runs the
// transposes in reverse order.  The field updates are linear, so their
// transposes need no stored values; the push needs the particles before the
// push and the fields it gathered (after the first half-update), which a
// tape records while a checkpointed segment is recomputed.
//
//   * Yee transposes: one thread per buffer point in gather form (each
//     thread writes only its own point, no atomics).
//   * BC transpose: one thread per face row; adds into neighbours with
//     atomics and accumulates d objective / d(profile coefficient).
//   * push adjoint: one thread per particle; recomputes the gather with
//     shape-derivative weights, takes the Boris Jacobian by forward-mode
//     dual numbers (three passes of three tangents), contracts the current
//     adjoint with the Esirkepov factors to get the derivatives of the
//     deposit with respect to the old and new positions and the weight,
//     and scatters the gathered-field adjoints back to the grid.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "pic_kernels.cuh"
#include "push_core.cuh"

namespace pic {

// ---------------------------------------------------------------------------
// forward-mode dual numbers with N tangents

template <typename T, int N>
struct Dual {
    T v;
    T d[N];
};

template <typename T, int N>
__device__ __forceinline__ Dual<T, N> dconst(T v) {
    Dual<T, N> r;
    r.v = v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = T(0);
    return r;
}
template <typename T, int N>
__device__ __forceinline__ Dual<T, N> operator+(const Dual<T, N> &a, const Dual<T, N> &b) {
    Dual<T, N> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <typename T, int N>
__device__ __forceinline__ Dual<T, N> operator-(const Dual<T, N> &a, const Dual<T, N> &b) {
    Dual<T, N> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <typename T, int N>
__device__ __forceinline__ Dual<T, N> operator*(const Dual<T, N> &a, const Dual<T, N> &b) {
    Dual<T, N> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <typename T, int N>
__device__ __forceinline__ Dual<T, N> operator*(const Dual<T, N> &a, T s) {
    Dual<T, N> r;
    r.v = a.v * s;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * s;
    return r;
}
template <typename T, int N>
__device__ __forceinline__ Dual<T, N> operator/(const Dual<T, N> &a, const Dual<T, N> &b) {
    Dual<T, N> r;
    T inv = T(1) / b.v;
    r.v = a.v * inv;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * inv;
    return r;
}
template <typename T, int N>
__device__ __forceinline__ Dual<T, N> dsqrt(const Dual<T, N> &a) {
    Dual<T, N> r;
    r.v = sqrt(a.v);
    T h = T(0.5) / r.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * h;
    return r;
}

// Boris rotation and move (particle.cpp:271-315) on duals; inputs p, e, b
// (fields unscaled), outputs p' and the displacement in cells
template <typename T, int N>
__device__ __forceinline__ void boris_dual(const Dual<T, N> (&p)[3], const Dual<T, N> (&e)[3],
                                           const Dual<T, N> (&b)[3], T qm, const T (&dtd)[3], Dual<T, N> (&pn)[3],
                                           Dual<T, N> (&disp)[3]) {
    Dual<T, N> ep[3], bp[3], p1[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        ep[d] = e[d] * qm;
        bp[d] = b[d] * qm;
        p1[d] = p[d] + ep[d];
    }
    Dual<T, N> one = dconst<T, N>(T(1));
    Dual<T, N> gm1 = dsqrt(one + (p1[0] * p1[0] + p1[1] * p1[1] + p1[2] * p1[2]));
    Dual<T, N> t[3] = {bp[0] / gm1, bp[1] / gm1, bp[2] / gm1};
    Dual<T, N> tt = dconst<T, N>(T(2)) / (one + t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
    Dual<T, N> s[3] = {t[0] * tt, t[1] * tt, t[2] * tt};
    Dual<T, N> p2[3] = {p1[0] + (p1[1] * t[2] - p1[2] * t[1]), p1[1] + (p1[2] * t[0] - p1[0] * t[2]),
                        p1[2] + (p1[0] * t[1] - p1[1] * t[0])};
    pn[0] = p1[0] + (p2[1] * s[2] - p2[2] * s[1]) + ep[0];
    pn[1] = p1[1] + (p2[2] * s[0] - p2[0] * s[2]) + ep[1];
    pn[2] = p1[2] + (p2[0] * s[1] - p2[1] * s[0]) + ep[2];
    Dual<T, N> gam = dsqrt(one + (pn[0] * pn[0] + pn[1] * pn[1] + pn[2] * pn[2]));
#pragma unroll
    for (int d = 0; d < 3; ++d) disp[d] = (pn[d] / gam) * dtd[d];
}

// derivatives of the shape weights with respect to the position
template <typename real>
__device__ __forceinline__ void shape_derivs(real d, real (&w)[3]) {
    const real h = real(0.5);
    w[0] = -(h - d);
    w[1] = real(-2) * d;
    w[2] = h + d;
}
template <typename real>
__device__ __forceinline__ void shape_derivs(real d, real (&w)[5]) {
    real u, u2;
    u = d - real(0.5);
    u2 = u * u;
    w[0] = u2 * u * real(1.0 / 6.0);
    u = d + real(1.0);
    u2 = u * u;
    w[1] = -u2 * u * real(4.0 / 6.0) + u2 * real(15.0 / 6.0) - u * real(10.0 / 4.0) + real(5.0 / 24.0);
    u = d;
    u2 = u * u;
    w[2] = u2 * u - u * real(5.0 / 4.0);
    u = d - real(1.0);
    u2 = u * u;
    w[3] = -u2 * u * real(4.0 / 6.0) - u2 * real(15.0 / 6.0) - u * real(10.0 / 4.0) - real(5.0 / 24.0);
    u = d + real(0.5);
    u2 = u * u;
    w[4] = u2 * u * real(1.0 / 6.0);
}

// gather of one component with its gradient with respect to the position
template <typename real, int P, bool LDG>
__device__ __forceinline__ void gather_grad(const View<const real> &f, int i0, int j0, int k0,
                                            const real (&wx)[P], const real (&wy)[P], const real (&wz)[P],
                                            const real (&dx)[P], const real (&dy)[P], const real (&dz)[P], real &e,
                                            real (&gr)[3]) {
    e = 0;
    gr[0] = gr[1] = gr[2] = 0;
    for (int k = 0; k < P; ++k) {
        real a = 0, ax = 0, ay = 0;
#pragma unroll
        for (int j = 0; j < P; ++j) {
            const real *row = f.at(k0 + k, j0 + j, i0);
            real s = 0, sd = 0;
#pragma unroll
            for (int i = 0; i < P; ++i) {
                real v = LDG ? __ldg(row + i) : row[i];
                s += wx[i] * v;
                sd += dx[i] * v;
            }
            a += wy[j] * s;
            ax += wy[j] * sd;
            ay += dy[j] * s;
        }
        const real wzk = pick(wz, k), dzk = pick(dz, k);
        e += wzk * a;
        gr[0] += wzk * ax;
        gr[1] += wzk * ay;
        gr[2] += dzk * a;
    }
}

template <typename real, int P>
__device__ __forceinline__ void scatter_adj(real *f, const Geom &g, int i0, int j0, int k0, const real (&wx)[P],
                                            const real (&wy)[P], const real (&wz)[P], real lam) {
    if (lam == real(0)) return;
    for (int k = 0; k < P; ++k) {
        const real lk = lam * pick(wz, k);
#pragma unroll
        for (int j = 0; j < P; ++j) {
            real *row = f + g.fi(k0 + k, j0 + j, i0);
            const real lj = lk * wy[j];
#pragma unroll
            for (int i = 0; i < P; ++i) atomic_add(row + i, lj * wx[i]);
        }
    }
}

// union-span arrays of a quantity of the old (a0 at centre i1) and new (a1
// at centre i2) positions, as span1d does for the weights
template <typename T, int P>
__device__ __forceinline__ void span_pair(int i1, const T (&a0)[P], int i2, const T (&a1)[P], T (&u0)[P + 1],
                                          T (&u1)[P + 1]) {
    const int lo = min(i1, i2);
    const bool o0 = i1 != lo, o1 = i2 != lo;
#pragma unroll
    for (int a = 0; a <= P; ++a) {
        u0[a] = o0 ? (a >= 1 ? a0[a - 1] : T(0)) : (a < P ? a0[a] : T(0));
        u1[a] = o1 ? (a >= 1 ? a1[a - 1] : T(0)) : (a < P ? a1[a] : T(0));
    }
}

// Adjoint of one Esirkepov component.  Axis `c` carries the running sum of
// ds = s1 - s0, axes `u` and `v` the weight
// W = 1/3 s0u s0v + 1/6 s1u s0v + 1/6 s0u s1v + 1/3 s1u s1v.
// Returns G1 = sum(lam * J) / w and adds dG1/ds0, dG1/ds1 into g0, g1.
template <int P, bool LDG, typename LT>
__device__ __forceinline__ double esirkepov_adj(const LT *lam, int sc, int su, int sv, int lc, int lu, int lv,
                                                double coef, const double (&s0c)[P + 1], const double (&s1c)[P + 1],
                                                const double (&s0u)[P + 1], const double (&s1u)[P + 1],
                                                const double (&s0v)[P + 1], const double (&s1v)[P + 1],
                                                double (&g0c)[P + 1], double (&g1c)[P + 1], double (&g0u)[P + 1],
                                                double (&g1u)[P + 1], double (&g0v)[P + 1], double (&g1v)[P + 1]) {
    constexpr double third = 1.0 / 3.0, sixth = 1.0 / 6.0;
    double C[P + 1];
    double acc = 0.0;
#pragma unroll
    for (int a = 0; a <= P; ++a) {
        acc += s1c[a] - s0c[a];
        C[a] = (a < lc - 1) ? acc : 0.0;   // the last running-sum point is not deposited
    }
    double M[P + 1];
#pragma unroll
    for (int a = 0; a <= P; ++a) M[a] = 0.0;
    double G = 0.0;
    for (int b = 0; b < lv; ++b) {
        const double s0b = pick(s0v, b), s1b = pick(s1v, b);
        double dv0 = 0.0, dv1 = 0.0;
#pragma unroll
        for (int a = 0; a <= P; ++a) {
            if (a >= lu) break;
            const double W = third * s0u[a] * s0b + sixth * s1u[a] * s0b + sixth * s0u[a] * s1b + third * s1u[a] * s1b;
            double T = 0.0;
            const LT *row = lam + b * sv + a * su;
#pragma unroll
            for (int q = 0; q < P; ++q) {
                if (q >= lc - 1) break;
                const double l = (double)(LDG ? __ldg(row + q * sc) : row[q * sc]);
                T += C[q] * l;
                M[q] += l * W;
            }
            G += T * W;
            g0u[a] += coef * T * (third * s0b + sixth * s1b);
            g1u[a] += coef * T * (sixth * s0b + third * s1b);
            dv0 += T * (third * s0u[a] + sixth * s1u[a]);
            dv1 += T * (sixth * s0u[a] + third * s1u[a]);
        }
        // add into g0v[b], g1v[b] for a run-time b
#pragma unroll
        for (int q = 0; q <= P; ++q)
            if (q == b) {
                g0v[q] += coef * dv0;
                g1v[q] += coef * dv1;
            }
    }
    // dG/dds(q') = coef * sum_{q >= q'} M(q); ds = s1 - s0
    double suf = 0.0;
#pragma unroll
    for (int q = P; q >= 0; --q) {
        suf += M[q];
        g1c[q] += coef * suf;
        g0c[q] -= coef * suf;
    }
    return coef * G;
}

template <typename real>
struct AdjPushArgs {
    Geom g;
    CellPack cp;
    long long n;
    // tape: particles before the push, fields after the first half-update
    const double *x, *y, *z;
    const int *cell;
    const float *ox, *oy, *oz;
    const real *px, *py, *pz;
    const unsigned char *dead;
    const real *f[6];
    const real *w;
    // adjoints
    const real *lj[3];         // d objective / dJ (ring buffers)
    real *lf[6];               // d objective / d(E, B) after the first half-update (field buffers)
    real *lx, *ly, *lz, *lpx, *lpy, *lpz;   // per particle, in: after the push, out: before it
    double *lw;                // per particle, accumulated
    real qm, charge;
    real dt_d[3];
    double d_dt[3];
    int scatter_fields;        // 0 for the t = 0 push (fields identically zero there)
    unsigned *status;
    const int *idx;            // optional particle list (count *nidx); null: all n particles
    const unsigned long long *nidx;
};

// One particle's push adjoint (everything but the scatter of the gathered
// field adjoints): per-particle adjoints updated in place, the weight
// adjoint accumulated, and lin[3..8] = d objective / d(gathered E, B) left
// for the caller to scatter with the gather weights.  fv: the tape's six
// field components; lj: the three J adjoints (ring layout or a shared box),
// both addressed in buffer coordinates.  Returns false if the particle is
// skipped (its stencil leaves the buffers).
template <typename real, int P, bool LDG>
__device__ __forceinline__ bool adj_particle(const AdjPushArgs<real> &a, long long p, const View<const real> (&fv)[6],
                                             const View<const real> (&lj)[3], real (&lin)[9]) {
    constexpr bool F64 = sizeof(real) == 8;
    constexpr int H = P / 2;
    const Geom &g = a.g;
    {
        // ---- old position --------------------------------------------------
        int ip[3], id[3], cc[3] = {0, 0, 0};
        real dp[3], dd[3];
        double xd[3] = {0, 0, 0};
        real oo[3] = {0, 0, 0};
        if constexpr (F64) {
            xd[0] = a.x[p];
            xd[1] = a.y[p];
            xd[2] = a.z[p];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                double xc = xd[d] - (double)(1 - g.mem);
                ip[d] = (int)(xc + 0.5);
                dp[d] = xc - (double)ip[d];
                id[d] = (int)xc;
                dd[d] = (xc - 0.5) - (double)id[d];
            }
        } else {
            a.cp.unpack(a.cell[p], cc[0], cc[1], cc[2]);
            oo[0] = a.ox[p];
            oo[1] = a.oy[p];
            oo[2] = a.oz[p];
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
            return false;
        }
        // ---- gather with gradients (Yee staggering, particle.cpp:207-259) -
        real ev[6], eg[6][3];
        {
        real wp[3][P], wd[3][P], gp[3][P], gd[3][P];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            shape_weights(dp[d], wp[d]);
            shape_weights(dd[d], wd[d]);
            shape_derivs(dp[d], gp[d]);
            shape_derivs(dd[d], gd[d]);
        }
        gather_grad<real, P, LDG>(fv[0], id[0] - H, ip[1] - H, ip[2] - H, wd[0], wp[1], wp[2], gd[0], gp[1], gp[2], ev[0], eg[0]);
        gather_grad<real, P, LDG>(fv[1], ip[0] - H, id[1] - H, ip[2] - H, wp[0], wd[1], wp[2], gp[0], gd[1], gp[2], ev[1], eg[1]);
        gather_grad<real, P, LDG>(fv[2], ip[0] - H, ip[1] - H, id[2] - H, wp[0], wp[1], wd[2], gp[0], gp[1], gd[2], ev[2], eg[2]);
        gather_grad<real, P, LDG>(fv[3], ip[0] - H, id[1] - H, id[2] - H, wp[0], wd[1], wd[2], gp[0], gd[1], gd[2], ev[3], eg[3]);
        gather_grad<real, P, LDG>(fv[4], id[0] - H, ip[1] - H, id[2] - H, wd[0], wp[1], wd[2], gd[0], gp[1], gd[2], ev[4], eg[4]);
        gather_grad<real, P, LDG>(fv[5], id[0] - H, id[1] - H, ip[2] - H, wd[0], wd[1], wp[2], gd[0], gd[1], gp[2], ev[5], eg[5]);
        }
        // ---- Boris Jacobian: three passes of three tangents (p, e, b) -----
        const real pin[3] = {a.px[p], a.py[p], a.pz[p]};
        // values only here (the displacement fixes the new position); the
        // tangents are formed after the deposit adjoint, contracted at once
        real disp_v[3];
        {
            Dual<real, 1> P_[3], E_[3], B_[3], pn[3], ds[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                P_[d] = dconst<real, 1>(pin[d]);
                E_[d] = dconst<real, 1>(ev[d]);
                B_[d] = dconst<real, 1>(ev[3 + d]);
            }
            boris_dual<real, 1>(P_, E_, B_, a.qm, a.dt_d, pn, ds);
#pragma unroll
            for (int o = 0; o < 3; ++o) disp_v[o] = ds[o].v;
        }
        // ---- new position, as the forward deposit forms it ----------------
        int i2[3];
        double d2[3], d0[3];
        if constexpr (F64) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                double xc = (xd[d] + (double)disp_v[d]) - (double)(1 - g.mem);
                i2[d] = (int)(xc + 0.5);
                d2[d] = xc - (double)i2[d];
                d0[d] = dp[d];
            }
        } else {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                double u = (double)oo[d] + (double)disp_v[d];
                double f = floor(u + 0.5);
                i2[d] = cc[d] + g.mem - 1 + (int)f;
                d2[d] = u - f;
                d0[d] = (double)dp[d];
            }
        }
        bool cfl = abs(i2[0] - ip[0]) <= 1 && abs(i2[1] - ip[1]) <= 1 && abs(i2[2] - ip[2]) <= 1;
        if (!cfl) {
            set_status(a.status, ST_CFL);
            return false;
        }
        // ---- deposit adjoint ----------------------------------------------
        double s0[3][P + 1], s1[3][P + 1];   // weights on the common span
        double g0[3][P + 1], g1[3][P + 1];   // dG1 / d(weights)
        int base[3], len[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            double w0[P], w1[P];
            shape_weights(d0[d], w0);
            shape_weights(d2[d], w1);
            span_pair<double, P>(ip[d], w0, i2[d], w1, s0[d], s1[d]);
            base[d] = min(ip[d], i2[d]) - H;
            len[d] = P + abs(i2[d] - ip[d]);
#pragma unroll
            for (int q = 0; q <= P; ++q) g0[d][q] = g1[d][q] = 0.0;
        }
        const double qd = (double)a.charge;
        double G1 = 0.0;
        // Jx: running sum along x, weight from y and z (particle.cpp:427-450);
        // the J adjoints are read in place from the ring buffers
#pragma unroll 1
        for (int comp = 0; comp < 3; ++comp) {
            const real *lbuf = lj[comp].at(base[2], base[1], base[0]);
            const int sX = 1, sY = lj[comp].sy, sZ = lj[comp].sz;
            if (comp == 0)
                G1 += esirkepov_adj<P, LDG>(lbuf, sX, sY, sZ, len[0], len[1], len[2], -qd * a.d_dt[0], s0[0], s1[0],
                                       s0[1], s1[1], s0[2], s1[2], g0[0], g1[0], g0[1], g1[1], g0[2], g1[2]);
            else if (comp == 1)
                G1 += esirkepov_adj<P, LDG>(lbuf, sY, sX, sZ, len[1], len[0], len[2], -qd * a.d_dt[1], s0[1], s1[1],
                                       s0[0], s1[0], s0[2], s1[2], g0[1], g1[1], g0[0], g1[0], g0[2], g1[2]);
            else
                G1 += esirkepov_adj<P, LDG>(lbuf, sZ, sX, sY, len[2], len[0], len[1], -qd * a.d_dt[2], s0[2], s1[2],
                                       s0[0], s1[0], s0[1], s1[1], g0[2], g1[2], g0[0], g1[0], g0[1], g1[1]);
        }
        const double wgt = (double)a.w[p];
        a.lw[p] += G1;
        double dGx0[3], dGx1[3];   // d G / d x_old, d G / d x_new
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            double v0[P], v1[P], t0[P + 1], t1[P + 1];   // weight derivatives on the span
            shape_derivs(d0[d], v0);
            shape_derivs(d2[d], v1);
            span_pair<double, P>(ip[d], v0, i2[d], v1, t0, t1);
            double s_0 = 0.0, s_1 = 0.0;
#pragma unroll
            for (int q = 0; q <= P; ++q) {
                s_0 += g0[d][q] * t0[q];
                s_1 += g1[d][q] * t1[q];
            }
            dGx0[d] = wgt * s_0;
            dGx1[d] = wgt * s_1;
        }
        // ---- chain rule: lin = J^T (lp', lx') with J = d(p', disp) / d(p, e,
        // b), one forward-mode pass of three tangents per input group ------
        const real lxn[3] = {a.lx[p] + (real)dGx1[0], a.ly[p] + (real)dGx1[1], a.lz[p] + (real)dGx1[2]};
        const real lpn[3] = {a.lpx[p], a.lpy[p], a.lpz[p]};
#pragma unroll
        for (int pass = 0; pass < 3; ++pass) {
            Dual<real, 3> P_[3], E_[3], B_[3], pn[3], ds[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                P_[d] = dconst<real, 3>(pin[d]);
                E_[d] = dconst<real, 3>(ev[d]);
                B_[d] = dconst<real, 3>(ev[3 + d]);
            }
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                if (pass == 0) P_[d].d[d] = real(1);
                if (pass == 1) E_[d].d[d] = real(1);
                if (pass == 2) B_[d].d[d] = real(1);
            }
            boris_dual<real, 3>(P_, E_, B_, a.qm, a.dt_d, pn, ds);
#pragma unroll
            for (int t = 0; t < 3; ++t) {
                real s = 0;
#pragma unroll
                for (int o = 0; o < 3; ++o) s += lpn[o] * pn[o].d[t] + lxn[o] * ds[o].d[t];
                lin[3 * pass + t] = s;
            }
        }
        real lxo[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            real s = lxn[d] + (real)dGx0[d];
#pragma unroll
            for (int c = 0; c < 6; ++c) s += lin[3 + c] * eg[c][d];
            lxo[d] = s;
        }
        a.lx[p] = lxo[0];
        a.ly[p] = lxo[1];
        a.lz[p] = lxo[2];
        a.lpx[p] = lin[0];
        a.lpy[p] = lin[1];
        a.lpz[p] = lin[2];
        return true;
    }
}

// The gather weights of the six staggered components of a particle at its
// tape position (primal/dual index and offset per axis), for the scatter.
template <typename real, int P>
__device__ __forceinline__ void gather_stencils(const AdjPushArgs<real> &a, long long p, int (&ip)[3], int (&id)[3],
                                                real (&wp)[3][P], real (&wd)[3][P]) {
    const Geom &g = a.g;
    if constexpr (sizeof(real) == 8) {
        const double xd[3] = {a.x[p], a.y[p], a.z[p]};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            double xc = xd[d] - (double)(1 - g.mem);
            ip[d] = (int)(xc + 0.5);
            id[d] = (int)xc;
            shape_weights((real)(xc - (double)ip[d]), wp[d]);
            shape_weights((real)((xc - 0.5) - (double)id[d]), wd[d]);
        }
    } else {
        int cc[3];
        a.cp.unpack(a.cell[p], cc[0], cc[1], cc[2]);
        const real oo[3] = {a.ox[p], a.oy[p], a.oz[p]};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const int b = cc[d] + g.mem - 1;
            const bool up = oo[d] >= 0.5f;
            ip[d] = b + (up ? 1 : 0);
            id[d] = b;
            shape_weights(up ? oo[d] - 1.0f : oo[d], wp[d]);
            shape_weights(oo[d] - 0.5f, wd[d]);
        }
    }
}

template <typename real, int P>
__global__ void __launch_bounds__(128) adj_push_kernel(AdjPushArgs<real> a) {
    constexpr int H = P / 2;
    const Geom &g = a.g;
    View<const real> fv[6], lj[3];
#pragma unroll
    for (int c = 0; c < 6; ++c) fv[c] = View<const real>{a.f[c], g.f[0], g.fxy, 0};
#pragma unroll
    for (int c = 0; c < 3; ++c) lj[c] = View<const real>{a.lj[c], g.r[0], g.rxy, g.rxy + g.r[0] + 1};
    const long long n = a.idx ? (long long)*a.nidx : a.n;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const long long p = a.idx ? (long long)a.idx[t] : t;
        if (a.dead && a.dead[p]) continue;
        real lin[9];
        if (!adj_particle<real, P, true>(a, p, fv, lj, lin)) continue;
        if (a.scatter_fields) {
            int ip[3], id[3];
            real wp[3][P], wd[3][P];   // the gather weights again (cheaper than keeping them live)
            gather_stencils<real, P>(a, p, ip, id, wp, wd);
            scatter_adj<real, P>(a.lf[0], g, id[0] - H, ip[1] - H, ip[2] - H, wd[0], wp[1], wp[2], lin[3]);
            scatter_adj<real, P>(a.lf[1], g, ip[0] - H, id[1] - H, ip[2] - H, wp[0], wd[1], wp[2], lin[4]);
            scatter_adj<real, P>(a.lf[2], g, ip[0] - H, ip[1] - H, id[2] - H, wp[0], wp[1], wd[2], lin[5]);
            scatter_adj<real, P>(a.lf[3], g, ip[0] - H, id[1] - H, id[2] - H, wp[0], wd[1], wd[2], lin[6]);
            scatter_adj<real, P>(a.lf[4], g, id[0] - H, ip[1] - H, id[2] - H, wd[0], wp[1], wd[2], lin[7]);
            scatter_adj<real, P>(a.lf[5], g, id[0] - H, id[1] - H, ip[2] - H, wd[0], wd[1], wp[2], lin[8]);
        }
    }
}

// ---------------------------------------------------------------------------
// Tiled push adjoint.  The tape holds the particles in the order of the
// forward push, i.e. sorted by tile at the last sort; with each sort the tape
// also keeps the tile boundaries of that order.  One CTA per tile:
//   1. stages the tape's six field components over the tile's gather box
//      and the three J adjoints over its deposit box in shared memory;
//   2. runs each particle's push adjoint from shared memory, keeping the
//      adjoints of its gathered E and B (six values) and their largest
//      magnitude per component;
//   3. adds every particle's field adjoint times its gather weights into
//      fixed-point shared accumulators (20-bit limbs as the forward deposit,
//      scaled so that the largest value fits), then flushes them with one
//      pass of global atomics.
// Particles that left their tile since the sort, and tiles with more
// particles than the scratch holds, go to the global kernel afterwards.

struct AdjTileGeom {
    int T, nt[3];
    int GE, DE;
    int gsy, gsz, gsize, dsy, dsz, dsize;
    int cap;                 // particles per tile the shared scratch holds
};

template <typename real>
constexpr int adj_limbs() { return sizeof(real) == 8 ? 3 : 2; }

// Zeros are added like any value: a per-point zero test measured 9 % slower
// on the whole reverse sweep (as on the forward deposit).
template <typename real, int NL>
__device__ __forceinline__ void fixed_add(unsigned *a, int lstride, real q) {
    if constexpr (NL == 3) {
        const long long qi = __double_as_longlong((double)q + 6755399441055744.0) - 0x4338000000000000LL;
        atomicAdd(a, (unsigned)(qi & 0xFFFFF));
        atomicAdd(a + lstride, (unsigned)((qi >> 20) & 0xFFFFF));
        atomicAdd(a + 2 * lstride, (unsigned)(int)(qi >> 40));
    } else {
        const int qi = __float2int_rn((float)q);
        atomicAdd(a, (unsigned)qi & 0xFFFFFu);
        atomicAdd(a + lstride, (unsigned)(qi >> 20));
    }
}

// TT: the tile edge as a compile-time constant (0: from tg), which makes
// every shared-box stride a constant.
template <typename real, int P, int TT>
__global__ void __launch_bounds__(256, 1) adj_tile_kernel(AdjPushArgs<real> a, AdjTileGeom tg, const unsigned *toffs,
                                                          int *strag, unsigned long long *nstrag) {
    AdjTileGeom t = tg;
    if constexpr (TT > 0) {
        constexpr int ge = TT + 2 * (P / 2) + 1, de = TT + 2 * (P / 2) + 3;
        constexpr int gy = padded_row(ge, TT), gz = padded_plane(ge, TT);
        constexpr int dy = padded_row(de, TT), dz = padded_plane(de, TT);
        t.T = TT; t.GE = ge; t.DE = de;
        t.gsy = gy; t.gsz = gz; t.gsize = ge * gz;
        t.dsy = dy; t.dsz = dz; t.dsize = de * dz;
    }
    constexpr int H = P / 2, NL = adj_limbs<real>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Geom &g = a.g;
    const int T = t.T, GE = t.GE, DE = t.DE, GS = t.gsize, DS = t.dsize;
    real *sf = reinterpret_cast<real *>(smem_raw);              // 6 x GS
    real *sl = sf + 6 * GS;                                       // 3 x DS
    real *slin = sl + 3 * DS;                                     // cap x 6
    unsigned *acc = reinterpret_cast<unsigned *>(slin + 6 * t.cap);   // 6 x NL x GS
    unsigned *smax = acc + 6 * NL * GS;                           // 6 (bits of non-negative values)
    unsigned char *flag = reinterpret_cast<unsigned char *>(smax + 8);   // cap
    const int tile = blockIdx.x;
    const int tx = tile % t.nt[0], ty = (tile / t.nt[0]) % t.nt[1], tz = tile / (t.nt[0] * t.nt[1]);
    const int t0[3] = {tx * T, ty * T, tz * T};
    int gO[3], dO[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        gO[d] = t0[d] + g.mem - 1 - H;
        dO[d] = t0[d] + g.mem - 2 - H;
    }
    long long pa = toffs[tile], pb = toffs[tile + 1];
    pb = pb < a.n ? pb : a.n;
    if (pa > pb) pa = pb;
    const long long m = pb - pa;
    if (m == 0) return;
    const bool use_smem = m <= t.cap;
    if (!use_smem) {
        for (long long i = threadIdx.x; i < m; i += blockDim.x) {
            const long long p = pa + i;
            if (!(a.dead && a.dead[p])) strag[atomicAdd(nstrag, 1ull)] = (int)p;
        }
        return;
    }
    const int G2 = GE * GE, G3 = G2 * GE, D2 = DE * DE, D3 = D2 * DE;
    for (int e = threadIdx.x; e < 6 * G3; e += blockDim.x) {
        int c = e / G3, l = e - c * G3;
        int lz = l / G2, r = l - lz * G2, ly = r / GE, lx = r - ly * GE;
        int x = gO[0] + lx, y = gO[1] + ly, z = gO[2] + lz;
        real v = 0;
        if (x >= 0 && x < g.f[0] && y >= 0 && y < g.f[1] && z >= 0 && z < g.f[2]) v = __ldg(a.f[c] + g.fi(z, y, x));
        sf[c * GS + lz * t.gsz + ly * t.gsy + lx] = v;
    }
    for (int e = threadIdx.x; e < 3 * D3; e += blockDim.x) {
        int c = e / D3, l = e - c * D3;
        int lz = l / D2, r = l - lz * D2, ly = r / DE, lx = r - ly * DE;
        int x = dO[0] + lx, y = dO[1] + ly, z = dO[2] + lz;
        real v = 0;
        if (x >= -1 && x <= g.f[0] && y >= -1 && y <= g.f[1] && z >= -1 && z <= g.f[2]) v = __ldg(a.lj[c] + g.ri(z, y, x));
        sl[c * DS + lz * t.dsz + ly * t.dsy + lx] = v;
    }
    for (int e = threadIdx.x; e < 6 * NL * GS; e += blockDim.x) acc[e] = 0u;
    if (threadIdx.x < 6) smax[threadIdx.x] = 0u;
    __syncthreads();
    View<const real> fv[6], lj[3];
#pragma unroll
    for (int c = 0; c < 6; ++c) fv[c] = View<const real>{sf + c * GS, t.gsy, t.gsz, -(gO[2] * t.gsz + gO[1] * t.gsy + gO[0])};
#pragma unroll
    for (int c = 0; c < 3; ++c) lj[c] = View<const real>{sl + c * DS, t.dsy, t.dsz, -(dO[2] * t.dsz + dO[1] * t.dsy + dO[0])};
    // 2. the particles' push adjoints
    for (long long i = threadIdx.x; i < m; i += blockDim.x) {
        const long long p = pa + i;
        flag[i] = 0;
        if (a.dead && a.dead[p]) continue;
        int idl[3];   // dual index per axis (the cell's lower primal point)
        if constexpr (sizeof(real) == 8) {
            idl[0] = (int)(a.x[p] - (double)(1 - g.mem));
            idl[1] = (int)(a.y[p] - (double)(1 - g.mem));
            idl[2] = (int)(a.z[p] - (double)(1 - g.mem));
        } else {
            int cc[3];
            a.cp.unpack(a.cell[p], cc[0], cc[1], cc[2]);
#pragma unroll
            for (int d = 0; d < 3; ++d) idl[d] = cc[d] + g.mem - 1;
        }
        bool inside = true;
#pragma unroll
        for (int d = 0; d < 3; ++d) inside = inside && idl[d] >= t0[d] + g.mem - 1 && idl[d] < t0[d] + g.mem - 1 + T;
        if (!inside) {
            strag[atomicAdd(nstrag, 1ull)] = (int)p;
            continue;
        }
        real lin[9];
        if (!adj_particle<real, P, false>(a, p, fv, lj, lin)) continue;
        if (!a.scatter_fields) continue;
        flag[i] = 1;
        // per component the largest magnitude of the tile: reduced over the
        // warp's active lanes first, one shared atomic per warp
        const unsigned am = __activemask();
        const bool leader = (threadIdx.x & 31) == __ffs(am) - 1;
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            slin[c * t.cap + i] = lin[3 + c];
            const unsigned mag = __reduce_max_sync(am, __float_as_uint((float)fabs(lin[3 + c])));
            if (leader) atomicMax(smax + c, mag);
        }
    }
    if (!a.scatter_fields) return;
    __syncthreads();
    // 3. field adjoints into fixed point, then one flush
    const double lim = sizeof(real) == 8 ? 2251799813685248.0 /* 2^51 */ : 2147483648.0 /* 2^31 */;
    real scale[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        const double mx = (double)__uint_as_float(smax[c]);
        scale[c] = mx > 0.0 ? (real)(lim / (1.01 * mx)) : real(0);
    }
    for (long long i = threadIdx.x; i < m; i += blockDim.x) {
        if (!flag[i]) continue;
        int ip[3], id[3];
        real wp[3][P], wd[3][P];
        gather_stencils<real, P>(a, pa + i, ip, id, wp, wd);
        // stencil origin per component (Yee staggering as in the gather)
        const int o[6][3] = {{id[0], ip[1], ip[2]}, {ip[0], id[1], ip[2]}, {ip[0], ip[1], id[2]},
                             {ip[0], id[1], id[2]}, {id[0], ip[1], id[2]}, {id[0], id[1], ip[2]}};
#pragma unroll 1
        for (int c = 0; c < 6; ++c) {
            const real q = slin[c * t.cap + i] * scale[c];
            if (q == real(0)) continue;
            // dual axes: Ex x; Ey y; Ez z; Bx y, z; By x, z; Bz x, y
            const bool dx_ = c == 0 || c == 4 || c == 5, dy_ = c == 1 || c == 3 || c == 5,
                       dz_ = c == 2 || c == 3 || c == 4;
            real wx[P], wy[P], wz[P];
#pragma unroll
            for (int q2 = 0; q2 < P; ++q2) {
                wx[q2] = dx_ ? wd[0][q2] : wp[0][q2];
                wy[q2] = dy_ ? wd[1][q2] : wp[1][q2];
                wz[q2] = dz_ ? wd[2][q2] : wp[2][q2];
            }
            unsigned *ac = acc + c * NL * GS;
            const int b0 = (o[c][2] - H - gO[2]) * t.gsz + (o[c][1] - H - gO[1]) * t.gsy + (o[c][0] - H - gO[0]);
#pragma unroll 1
            for (int k = 0; k < P; ++k) {
                const real qk = q * pick(wz, k);
#pragma unroll
                for (int j = 0; j < P; ++j) {
                    const real qj = qk * wy[j];
#pragma unroll
                    for (int ii = 0; ii < P; ++ii) fixed_add<real, NL>(ac + b0 + k * t.gsz + j * t.gsy + ii, GS, qj * wx[ii]);
                }
            }
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < 6 * G3; e += blockDim.x) {
        int c = e / G3, l = e - c * G3;
        if (scale[c] == real(0)) continue;
        int lz = l / G2, r = l - lz * G2, ly = r / GE, lx = r - ly * GE;
        const unsigned *q = acc + c * NL * GS + lz * t.gsz + ly * t.gsy + lx;
        long long tot;
        if constexpr (NL == 2) tot = ((long long)(int)q[GS] << 20) + (long long)q[0];
        else tot = ((long long)(int)q[2 * GS] << 40) + ((long long)q[GS] << 20) + (long long)q[0];
        if (tot == 0) continue;
        int x = gO[0] + lx, y = gO[1] + ly, z = gO[2] + lz;
        if (x >= 0 && x < g.f[0] && y >= 0 && y < g.f[1] && z >= 0 && z < g.f[2])
            atomic_add(a.lf[c] + g.fi(z, y, x), (real)((double)tot / (double)scale[c]));
    }
}

__global__ void tile_bounds_kernel(const unsigned *offs, long long keys_per_tile, int ntiles, unsigned *out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t <= ntiles) out[t] = offs[(long long)t * keys_per_tile];
}

// ---------------------------------------------------------------------------
// transposes of the Yee half-updates (physical cells only, absorbing faces)

__device__ __forceinline__ bool physical(const Geom &g, int k, int j, int i) {
    return i >= g.mem && i < g.n[0] + g.mem && j >= g.mem && j < g.n[1] + g.mem && k >= g.mem && k < g.n[2] + g.mem;
}

// transpose of E += h (curl B - J): lamB += h curl^T lamE, lamJ -= h lamE
template <typename real>
__global__ void adj_update_e_kernel(Geom g, const real *lex, const real *ley, const real *lez, real *lbx, real *lby,
                                    real *lbz, real *ljx, real *ljy, real *ljz, real h, real idx, real idy, real idz) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.fsz) return;
    int i = (int)(t % g.f[0]), j = (int)((t / g.f[0]) % g.f[1]), k = (int)(t / g.fxy);
    const int q = (int)t;
    auto L = [&](const real *a, int kk, int jj, int ii) -> real {
        return (ii < g.f[0] && jj < g.f[1] && kk < g.f[2] && physical(g, kk, jj, ii)) ? a[g.fi(kk, jj, ii)] : real(0);
    };
    real ex0 = L(lex, k, j, i), ey0 = L(ley, k, j, i), ez0 = L(lez, k, j, i);
    lbz[q] += h * idy * (ex0 - L(lex, k, j + 1, i)) - h * idx * (ey0 - L(ley, k, j, i + 1));
    lby[q] += -h * idz * (ex0 - L(lex, k + 1, j, i)) + h * idx * (ez0 - L(lez, k, j, i + 1));
    lbx[q] += h * idz * (ey0 - L(ley, k + 1, j, i)) - h * idy * (ez0 - L(lez, k, j + 1, i));
    if (physical(g, k, j, i)) {
        const int r = g.ri(k, j, i);
        ljx[r] -= h * ex0;
        ljy[r] -= h * ey0;
        ljz[r] -= h * ez0;
    }
}

// transpose of B -= h curl E: lamE -= h curl^T lamB
template <typename real>
__global__ void adj_update_b_kernel(Geom g, real *lex, real *ley, real *lez, const real *lbx, const real *lby,
                                    const real *lbz, real h, real idx, real idy, real idz) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.fsz) return;
    int i = (int)(t % g.f[0]), j = (int)((t / g.f[0]) % g.f[1]), k = (int)(t / g.fxy);
    const int q = (int)t;
    auto L = [&](const real *a, int kk, int jj, int ii) -> real {
        return (ii >= 0 && jj >= 0 && kk >= 0 && physical(g, kk, jj, ii)) ? a[g.fi(kk, jj, ii)] : real(0);
    };
    real bx0 = L(lbx, k, j, i), by0 = L(lby, k, j, i), bz0 = L(lbz, k, j, i);
    lez[q] += -h * idy * L(lbx, k, j - 1, i) + h * idy * bx0 + h * idx * L(lby, k, j, i - 1) - h * idx * by0;
    ley[q] += h * idz * L(lbx, k - 1, j, i) - h * idz * bx0 - h * idx * L(lbz, k, j, i - 1) + h * idx * bz0;
    lex[q] += -h * idz * L(lby, k - 1, j, i) + h * idz * by0 + h * idy * L(lbz, k, j - 1, i) - h * idy * bz0;
}

// transpose of radiating_boundary (boundary.cpp:42-99) at time t: the two
// B columns it overwrites hand their adjoint to the inputs of the formula
// and to the laser source; d source / d coefficient accumulates in lprof.
struct AdjBcArgs {
    Geom g;
    double dt, dx, dy, dz;
    double Pi, omega, l0, amp, dur, start, waist, xfocus, yfocus, zfocus, phase, time;
    int pol, envelope, profile_n;
    double *lprof;
};

__device__ double adj_envelope(const AdjBcArgs &L, double t) {
    t = t - L.start;
    if (L.envelope == 1) {
        if (t < 0.0 || t > 3.0 * L.dur) return 0.0;
        double r = (t - 1.5 * L.dur) / L.dur;
        return L.amp * exp(-2.0 * log(2.0) * r * r);
    }
    return (t >= 0.0 && t <= L.dur) ? L.amp * sin(L.Pi * t / L.dur) : 0.0;
}

template <typename real>
__global__ void adj_bc_kernel(AdjBcArgs A, real *lex, real *ley, real *lez, real *lbx, real *lby, real *lbz,
                              real *ljy, real *ljz) {
    (void)lex;
    const Geom &g = A.g;
    int iy = blockIdx.x * blockDim.x + threadIdx.x;
    int iz = blockIdx.y * blockDim.y + threadIdx.y;
    if (iy >= g.n[1] || iz >= g.n[2]) return;
    iy += g.mem;
    iz += g.mem;
    const double alpha = 1 / (1 + A.dt / A.dx), beta = 1 - A.dt / A.dx;
    const int m = g.mem, L = g.n[0];
    double lsrc = 0.0;
    for (int side = 0; side < 2; ++side) {
        const int col = side == 0 ? m : L, out = side == 0 ? m - 1 : L + 1;
        const int c = g.fi(iz, iy, col), o = g.fi(iz, iy, out), rc = g.ri(iz, iy, col);
        const double Lz = lbz[o], Ly = lby[o];
        lbz[o] = 0;
        lby[o] = 0;
        const double sg = side == 0 ? 1.0 : -1.0;   // right column: signs of the E and J terms flip
        atomic_add(ley + c, (real)(-2 * alpha * sg * Lz));
        atomic_add(lbx + c, (real)(-alpha * A.dt / A.dz * Lz + alpha * A.dt / A.dy * Ly));
        atomic_add(lbx + c - g.fxy, (real)(alpha * A.dt / A.dz * Lz));
        atomic_add(lbx + c - g.f[0], (real)(-alpha * A.dt / A.dy * Ly));
        atomic_add(lbz + c, (real)(-alpha * beta * Lz));
        atomic_add(ljy + rc, (real)(-alpha * A.dt * sg * Lz));
        atomic_add(lez + c, (real)(2 * alpha * sg * Ly));
        atomic_add(lby + c, (real)(-alpha * beta * Ly));
        atomic_add(ljz + rc, (real)(alpha * A.dt * sg * Ly));
        if (side == 0) {
            if (A.pol == 1 || A.pol == 3) lsrc += 4 * alpha * Lz;
            if (A.pol == 2 || A.pol == 3) lsrc += -4 * alpha * Ly;
        }
    }
    if (!A.lprof || lsrc == 0.0) return;
    // d source / d coefficient (laser_profile = 1): -env * B_c(u) B_b(v) * cos(PHI + phase)
    const double k = 2.0 * A.Pi / A.l0, rl = 0.5 * k * A.waist * A.waist, xe = 0.0 - A.xfocus;
    const double y = iy * A.dy - A.yfocus, z = iz * A.dz - A.zfocus;
    const double q = xe / rl, w = A.waist * sqrt(1 + q * q);
    const double PHI = (xe / rl) * (y * y + z * z) / w / w - atan(xe / rl) + k * xe - A.omega * A.time;
    const double f = -1.0 * adj_envelope(A, A.time) * cos(PHI + A.phase);
    if (f == 0.0) return;
    const int nc = A.profile_n;
    const double u = ((double)(iy - g.mem) + 0.5) / (double)g.n[1] * (double)(nc - 1);
    const double v = ((double)(iz - g.mem) + 0.5) / (double)g.n[2] * (double)(nc - 1);
    for (int b = 0; b < nc; ++b) {
        double wv = cubic_bspline(v - b);
        if (wv == 0.0) continue;
        for (int cidx = 0; cidx < nc; ++cidx) {
            double wu = cubic_bspline(u - cidx);
            if (wu == 0.0) continue;
            atomicAdd(A.lprof + b * nc + cidx, lsrc * f * wu * wv);
        }
    }
}

// smooth window over [xlo, xhi): 0 outside, 1 inside, sin^2 ramps of width
// `ramp` cells at both ends (ramp = 0: a hard window); returns s(x), ds/dx
__device__ inline void window_weight(double x, double xlo, double xhi, double ramp, double &s, double &ds) {
    s = 0.0;
    ds = 0.0;
    if (!(x >= xlo && x < xhi)) return;
    const double half_pi = 1.5707963267948966;
    s = 1.0;
    if (ramp > 0.0) {
        const double up = (x - xlo) / ramp, down = (xhi - x) / ramp;
        if (up < 1.0) {
            double sn = sin(half_pi * up), cs = cos(half_pi * up);
            s = sn * sn;
            ds = 2.0 * sn * cs * half_pi / ramp;
        }
        if (down < 1.0) {
            double sn = sin(half_pi * down), cs = cos(half_pi * down);
            double s2 = sn * sn, d2 = -2.0 * sn * cs * half_pi / ramp;
            ds = ds * s2 + s * d2;
            s *= s2;
        }
    }
}

// objective: kinetic energy sum s(x) w m (gamma - 1) of the alive particles
// of a species, s the window weight above; seeds d objective / d (x, p, w)
template <typename real>
__global__ void adj_seed_kinetic_kernel(Geom g, CellPack cp, int fp32, long long n, const double *x, const int *cell,
                                        const float *ox, const real *px, const real *py, const real *pz,
                                        const real *w, const unsigned char *dead, double mass, double xlo,
                                        double xhi, double ramp, real *lx, real *lpx, real *lpy, real *lpz,
                                        double *lw, double *loss) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double contrib = 0.0;
    if (p < n && !(dead && dead[p])) {
        double xp;
        if (fp32) {
            int cx, cy, cz;
            cp.unpack(cell[p], cx, cy, cz);
            xp = (double)cx + (double)ox[p];
        } else {
            xp = x[p];
        }
        double sw, dsw;
        window_weight(xp, xlo, xhi, ramp, sw, dsw);
        if (sw != 0.0) {
            double a = px[p], b = py[p], c = pz[p];
            double u2 = a * a + b * b + c * c, gam = sqrt(1.0 + u2);
            double gm1 = u2 / (gam + 1.0);
            double wt = w[p];
            contrib = sw * wt * mass * gm1;
            lx[p] += (real)(dsw * wt * mass * gm1);
            lpx[p] += (real)(sw * wt * mass * a / gam);
            lpy[p] += (real)(sw * wt * mass * b / gam);
            lpz[p] += (real)(sw * wt * mass * c / gam);
            lw[p] += sw * mass * gm1;
        }
    }
    // warp reduction of the loss
    for (int o = 16; o > 0; o >>= 1) contrib += __shfl_down_sync(0xffffffffu, contrib, o);
    if ((threadIdx.x & 31) == 0 && contrib != 0.0) atomicAdd(loss, contrib);
}

}  // namespace pic

// moves of per-particle arrays between orders (bit copies)
template <typename T>
__global__ void scatter_to_kernel(const T *in, const int *to, T *out, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[to[i]] = in[i];
}
template <typename T>
__global__ void gather_from_kernel(const T *in, const int *from, T *out, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = in[from[i]];
}

// ===========================================================================
// host side: checkpoints, tape and the C ABI
// ===========================================================================

using namespace pic;

struct Blob {
    std::vector<std::pair<void *, size_t>> parts;   // (device pointer, bytes) at save time
    void *buf = nullptr;
    size_t bytes = 0;
    int step = 0;
    int cur[2] = {0, 0};
    long long count[2] = {0, 0};
    int field_part = 0;          // tape: index of the first of the six field parts
    int perm_part[2] = {-1, -1}; // tape: the sort permutation run right before this push, per species
    int toff_part[2] = {-1, -1}; // tape: tile boundaries of the particle order of this push, per species
};

struct AdjState {
    std::vector<Blob> ckpt;
    std::vector<Blob> tape;
    int tape_len = 0;
    bool recording = false;
    // adjoint arrays
    void *lf[6] = {};        // field-buffer adjoints (E, B)
    void *lj[3] = {};        // ring-buffer adjoints (J)
    void *lpart[2][6] = {};  // per species: lx, ly, lz, lpx, lpy, lpz
    double *lw[2] = {};
    double *lprof = nullptr;
    double *loss = nullptr;
    int nprof = 0;
    // tiled contexts: upload index of each particle in the order the
    // per-particle adjoints are held in (valid once seeded), and scratch
    int *lam_orig[2] = {};
    bool lam_valid = false;
    unsigned *toffs[2] = {};   // tiled contexts: tile boundaries extracted for the tape
    void *tmp = nullptr;
    size_t tmp_bytes = 0;
};

static std::vector<std::pair<pic_ctx *, AdjState *>> g_adj;

static AdjState *adj_of(pic_ctx *c, bool create) {
    for (auto &e : g_adj)
        if (e.first == c) return e.second;
    if (!create) return nullptr;
    g_adj.push_back({c, new AdjState()});
    return g_adj.back().second;
}

static size_t rsize(const pic_ctx *c) { return c->fp32 ? 4 : 8; }

// pieces of the particle state (current positions, momenta, dead flags)
static void particle_parts(pic_ctx *c, std::vector<std::pair<void *, size_t>> &v) {
    for (int k = 0; k < 2; ++k) {
        Species &s = c->sp[k];
        size_t n = (size_t)s.n_host;
        if (n == 0) continue;
        if (c->fp32) {
            v.push_back({s.a.cell[s.cur], n * 4});
            v.push_back({s.a.ox[s.cur], n * 4});
            v.push_back({s.a.oy[s.cur], n * 4});
            v.push_back({s.a.oz[s.cur], n * 4});
        } else {
            v.push_back({s.a.x[s.cur], n * 8});
            v.push_back({s.a.y[s.cur], n * 8});
            v.push_back({s.a.z[s.cur], n * 8});
        }
        v.push_back({s.a.px, n * rsize(c)});
        v.push_back({s.a.py, n * rsize(c)});
        v.push_back({s.a.pz, n * rsize(c)});
        if (s.dead) v.push_back({s.dead, n});
    }
}

// a checkpoint additionally holds what a sort moves but the tape need not:
// weights, ids and upload indices (tiled contexts)
static void checkpoint_parts(pic_ctx *c, std::vector<std::pair<void *, size_t>> &v) {
    particle_parts(c, v);
    for (int k = 0; k < 2; ++k) {
        Species &s = c->sp[k];
        size_t n = (size_t)s.n_host;
        if (n == 0 || !s.orig) continue;
        v.push_back({s.a.w, n * rsize(c)});
        v.push_back({s.a.id, n * sizeof(int)});
        v.push_back({s.orig, n * sizeof(int)});
    }
    for (int f = 0; f < 6; ++f) v.push_back({c->field[f], (size_t)c->g.fsz * rsize(c)});
    for (int f = 0; f < 5; ++f) v.push_back({c->ring[f], (size_t)c->g.rsz * rsize(c)});
}

static int blob_save(pic_ctx *c, Blob &b, const std::vector<std::pair<void *, size_t>> &parts) {
    size_t total = 0;
    for (auto &p : parts) total += (p.second + 255) & ~(size_t)255;
    if (b.bytes < total) {
        if (b.buf) cudaFree(b.buf);
        b.buf = nullptr;
        b.bytes = 0;
        if (cudaMalloc(&b.buf, total) != cudaSuccess) {
            c->err = "adjoint: out of device memory for a checkpoint / tape slot";
            return PIC_ENOMEM;
        }
        b.bytes = total;
    }
    b.parts = parts;
    size_t off = 0;
    for (auto &p : parts) {
        cudaMemcpyAsync((char *)b.buf + off, p.first, p.second, cudaMemcpyDeviceToDevice, c->stream);
        off += (p.second + 255) & ~(size_t)255;
    }
    b.step = c->step;
    for (int k = 0; k < 2; ++k) {
        b.cur[k] = c->sp[k].cur;
        b.count[k] = c->sp[k].n_host;
    }
    return PIC_OK;
}

// the tape slot's device pointer of part `idx`
static void *blob_part(const Blob &b, int idx) {
    size_t off = 0;
    for (int i = 0; i < idx; ++i) off += (b.parts[i].second + 255) & ~(size_t)255;
    return (char *)b.buf + off;
}

namespace pic {
// called by the step orchestration right before each push while recording
void adjoint_record_hook(pic_ctx *c) {
    AdjState *A = adj_of(c, false);
    if (!A || !A->recording) return;
    if (A->tape_len >= (int)A->tape.size()) {
        c->err = "adjoint tape full";
        return;
    }
    std::vector<std::pair<void *, size_t>> parts;
    particle_parts(c, parts);
    const int field_part = (int)parts.size();
    for (int f = 0; f < 6; ++f) parts.push_back({c->field[f], (size_t)c->g.fsz * rsize(c)});
    int perm_part[2] = {-1, -1}, toff_part[2] = {-1, -1};
    for (int k = 0; k < 2; ++k) {
        Species &s = c->sp[k];
        if (!s.perm_fresh || s.n_host == 0) continue;
        perm_part[k] = (int)parts.size();
        parts.push_back({s.perm, (size_t)s.n_host * sizeof(int)});
        s.perm_fresh = false;
    }
    const int ntiles = c->ntile[0] * c->ntile[1] * c->ntile[2];
    for (int k = 0; k < 2; ++k) {
        Species &s = c->sp[k];
        if (c->tile <= 0 || s.n_host == 0 || !s.sorted || !A->toffs[k]) continue;
        const long long kpt = (long long)c->tile * c->tile * c->tile * kOctants;
        tile_bounds_kernel<<<(ntiles + 256) / 256, 256, 0, c->stream>>>(s.offs, kpt, ntiles, A->toffs[k]);
        toff_part[k] = (int)parts.size();
        parts.push_back({A->toffs[k], (size_t)(ntiles + 1) * sizeof(unsigned)});
    }
    prof_begin(c, "adjoint_tape_record");
    Blob &b = A->tape[A->tape_len];
    if (blob_save(c, b, parts) == PIC_OK) {
        b.field_part = field_part;
        b.perm_part[0] = perm_part[0];
        b.perm_part[1] = perm_part[1];
        b.toff_part[0] = toff_part[0];
        b.toff_part[1] = toff_part[1];
        A->tape_len++;
    }
    prof_end(c);
}
}  // namespace pic

static int ensure_adj_arrays(pic_ctx *c, AdjState *A) {
    const size_t rs = rsize(c);
    auto alloc = [&](void **p, size_t bytes) -> bool {
        if (*p) return true;
        if (cudaMalloc(p, bytes) != cudaSuccess) return false;
        return true;
    };
    bool ok = true;
    for (int f = 0; f < 6; ++f) ok = ok && alloc(&A->lf[f], (size_t)c->g.fsz * rs);
    for (int f = 0; f < 3; ++f) ok = ok && alloc(&A->lj[f], (size_t)c->g.rsz * rs);
    for (int k = 0; k < 2; ++k) {
        size_t n = (size_t)std::max<int64_t>(c->sp[k].cap, 1);
        for (int q = 0; q < 6; ++q) ok = ok && alloc(&A->lpart[k][q], n * rs);
        ok = ok && alloc((void **)&A->lw[k], n * sizeof(double));
    }
    ok = ok && alloc((void **)&A->loss, sizeof(double));
    if (c->sp[0].orig || c->sp[1].orig) {
        size_t n = (size_t)std::max<int64_t>(std::max(c->sp[0].cap, c->sp[1].cap), 1);
        for (int k = 0; k < 2; ++k) ok = ok && alloc((void **)&A->lam_orig[k], n * sizeof(int));
        if (A->tmp_bytes < n * sizeof(double)) {
            if (A->tmp) cudaFree(A->tmp);
            A->tmp = nullptr;
            A->tmp_bytes = 0;
        }
        ok = ok && alloc(&A->tmp, n * sizeof(double));
        if (ok) A->tmp_bytes = n * sizeof(double);
    }
    int np = std::max(c->profile_n * c->profile_n, 1);
    if (A->nprof != np && A->lprof) {
        cudaFree(A->lprof);
        A->lprof = nullptr;
    }
    ok = ok && alloc((void **)&A->lprof, (size_t)np * sizeof(double));
    A->nprof = np;
    if (!ok) {
        c->err = "adjoint: out of device memory";
        return PIC_ENOMEM;
    }
    return PIC_OK;
}

// the per-particle arrays a sort moves that the reverse sweep reads:
// position and momentum adjoints, weight adjoint, weights, upload index
static int moved_arrays(pic_ctx *c, AdjState *A, int k, void **arr, size_t *es) {
    int m = 0;
    for (int q = 0; q < 6; ++q) { arr[m] = A->lpart[k][q]; es[m++] = rsize(c); }
    arr[m] = A->lw[k]; es[m++] = sizeof(double);
    arr[m] = c->sp[k].a.w; es[m++] = rsize(c);
    arr[m] = c->sp[k].orig; es[m++] = sizeof(int);
    return m;
}

static void scatter_to(pic_ctx *c, const void *in, const int *to, void *out, size_t es, long long n) {
    const unsigned blocks = (unsigned)((n + 255) / 256);
    if (es == 8) scatter_to_kernel<unsigned long long><<<blocks, 256, 0, c->stream>>>(
        (const unsigned long long *)in, to, (unsigned long long *)out, n);
    else scatter_to_kernel<unsigned><<<blocks, 256, 0, c->stream>>>((const unsigned *)in, to, (unsigned *)out, n);
}

static void gather_from(pic_ctx *c, const void *in, const int *from, void *out, size_t es, long long n) {
    const unsigned blocks = (unsigned)((n + 255) / 256);
    if (es == 8) gather_from_kernel<unsigned long long><<<blocks, 256, 0, c->stream>>>(
        (const unsigned long long *)in, from, (unsigned long long *)out, n);
    else gather_from_kernel<unsigned><<<blocks, 256, 0, c->stream>>>((const unsigned *)in, from, (unsigned *)out, n);
}

// undo one recorded sort of species k (perm[new] = old): every moved array
// goes back to the order before that sort
static void unsort_species(pic_ctx *c, AdjState *A, int k, const int *perm, long long n) {
    void *arr[9];
    size_t es[9];
    const int m = moved_arrays(c, A, k, arr, es);
    for (int q = 0; q < m; ++q) {
        cudaMemcpyAsync(A->tmp, arr[q], (size_t)n * es[q], cudaMemcpyDeviceToDevice, c->stream);
        scatter_to(c, A->tmp, perm, arr[q], es[q], n);
    }
}

// the adjoints are held in the order given by lam_orig (upload indices);
// bring them into the context's current order (its orig array): a segment
// recomputed from a checkpoint sorts again and need not end in the order
// the later segment's reverse sweep started from
static void remap_adjoints(pic_ctx *c, AdjState *A) {
    if (!A->lam_valid) return;
    for (int k = 0; k < 2; ++k) {
        Species &s = c->sp[k];
        const long long n = s.n_host;
        if (!s.orig || n == 0) continue;
        void *arr[9];
        size_t es[9];
        const int m = moved_arrays(c, A, k, arr, es) - 2;   // the adjoints only (weights, orig are current)
        for (int q = 0; q < m; ++q) {
            scatter_to(c, arr[q], A->lam_orig[k], A->tmp, es[q], n);
            gather_from(c, A->tmp, s.orig, arr[q], es[q], n);
        }
    }
}

static void note_adjoint_order(pic_ctx *c, AdjState *A) {
    for (int k = 0; k < 2; ++k) {
        Species &s = c->sp[k];
        if (s.orig && s.n_host > 0)
            cudaMemcpyAsync(A->lam_orig[k], s.orig, (size_t)s.n_host * sizeof(int), cudaMemcpyDeviceToDevice,
                            c->stream);
    }
    A->lam_valid = c->sp[0].orig || c->sp[1].orig;
}

template <typename real, int P>
static void adj_push_launch(pic_ctx *c, AdjState *A, const Blob &b, int kind, int part_base, int scatter) {
    Species &s = c->sp[kind];
    AdjPushArgs<real> a{};
    a.g = c->g;
    a.cp = c->cp;
    a.n = b.count[kind];
    int idx = part_base;
    if (c->fp32) {
        a.cell = (const int *)blob_part(b, idx++);
        a.ox = (const float *)blob_part(b, idx++);
        a.oy = (const float *)blob_part(b, idx++);
        a.oz = (const float *)blob_part(b, idx++);
    } else {
        a.x = (const double *)blob_part(b, idx++);
        a.y = (const double *)blob_part(b, idx++);
        a.z = (const double *)blob_part(b, idx++);
    }
    a.px = (const real *)blob_part(b, idx++);
    a.py = (const real *)blob_part(b, idx++);
    a.pz = (const real *)blob_part(b, idx++);
    a.dead = s.dead ? (const unsigned char *)blob_part(b, idx++) : nullptr;
    for (int f = 0; f < 6; ++f) a.f[f] = (const real *)blob_part(b, b.field_part + f);
    a.w = (const real *)s.a.w;
    for (int f = 0; f < 3; ++f) a.lj[f] = (const real *)A->lj[f];
    for (int f = 0; f < 6; ++f) a.lf[f] = (real *)A->lf[f];
    real **lp = (real **)A->lpart[kind];
    a.lx = lp[0]; a.ly = lp[1]; a.lz = lp[2]; a.lpx = lp[3]; a.lpy = lp[4]; a.lpz = lp[5];
    a.lw = A->lw[kind];
    const PicParams &p = c->p;
    a.qm = (real)(p.charge[kind] / p.mass[kind] * p.dt_half);
    a.charge = (real)p.charge[kind];
    a.dt_d[0] = (real)(p.dt / p.dx); a.dt_d[1] = (real)(p.dt / p.dy); a.dt_d[2] = (real)(p.dt / p.dz);
    a.d_dt[0] = p.dx / p.dt; a.d_dt[1] = p.dy / p.dt; a.d_dt[2] = p.dz / p.dt;
    a.scatter_fields = scatter;
    a.status = c->d_status;
    long long blocks = (a.n + 127) / 128;
    if (c->tile > 0 && b.toff_part[kind] >= 0) {
        // one CTA per tile, then the particles it handed back
        const TileBoxes bx = tile_boxes(c);
        AdjTileGeom tg{};
        tg.T = c->tile;
        for (int d = 0; d < 3; ++d) tg.nt[d] = c->ntile[d];
        tg.GE = bx.GE; tg.DE = bx.DE;
        tg.gsy = bx.gsy; tg.gsz = bx.gsz; tg.gsize = bx.gsize;
        tg.dsy = bx.dsy; tg.dsz = bx.dsz; tg.dsize = bx.dsize;
        const size_t rs = sizeof(real), nl = adj_limbs<real>();
        const size_t fixed = (6 * (size_t)bx.gsize + 3 * (size_t)bx.dsize) * rs + (6 * nl * bx.gsize + 8) * 4;
        const size_t budget = 227 * 1024;
        tg.cap = fixed + 64 < budget ? (int)std::min<size_t>(4095, (budget - fixed - 64) / (6 * rs + 1)) : 0;
        const size_t smem = fixed + (size_t)tg.cap * (6 * rs + 1);
        const int ntiles = c->ntile[0] * c->ntile[1] * c->ntile[2];
        cudaMemsetAsync(c->d_nstrag + kind, 0, sizeof(unsigned long long), c->stream);
        prof_begin(c, "adjoint_tile_push_deposit");
        if (tg.cap > 0) {
            const unsigned *toffs = (const unsigned *)blob_part(b, b.toff_part[kind]);
            if (c->tile == 4) {   // the default edge: strides as constants
                cudaFuncSetAttribute(adj_tile_kernel<real, P, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
                adj_tile_kernel<real, P, 4><<<ntiles, 256, smem, c->stream>>>(a, tg, toffs, s.strag, c->d_nstrag + kind);
            } else {
                cudaFuncSetAttribute(adj_tile_kernel<real, P, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
                adj_tile_kernel<real, P, 0><<<ntiles, 256, smem, c->stream>>>(a, tg, toffs, s.strag, c->d_nstrag + kind);
            }
            a.idx = s.strag;
            a.nidx = c->d_nstrag + kind;
        }
        prof_end(c);
    }
    prof_begin(c, "adjoint_push_deposit");
    adj_push_kernel<real, P><<<(unsigned)std::min<long long>(blocks, 148 * 16), 128, 0, c->stream>>>(a);
    prof_end(c);
}

template <typename real>
static void adj_fields_e(pic_ctx *c, AdjState *A) {
    const Geom &g = c->g;
    real **F = (real **)A->lf;
    real **J = (real **)A->lj;
    prof_begin(c, "adjoint_yee_e");
    adj_update_e_kernel<real><<<(unsigned)((g.fsz + 255) / 256), 256, 0, c->stream>>>(
        g, F[0], F[1], F[2], F[3], F[4], F[5], J[0], J[1], J[2], (real)c->p.dt_half, (real)(1.0 / c->p.dx),
        (real)(1.0 / c->p.dy), (real)(1.0 / c->p.dz));
    prof_end(c);
}

template <typename real>
static void adj_fields_b(pic_ctx *c, AdjState *A) {
    const Geom &g = c->g;
    real **F = (real **)A->lf;
    prof_begin(c, "adjoint_yee_b");
    adj_update_b_kernel<real><<<(unsigned)((g.fsz + 255) / 256), 256, 0, c->stream>>>(
        g, F[0], F[1], F[2], F[3], F[4], F[5], (real)c->p.dt_half, (real)(1.0 / c->p.dx), (real)(1.0 / c->p.dy),
        (real)(1.0 / c->p.dz));
    prof_end(c);
}

template <typename real>
static void adj_bc(pic_ctx *c, AdjState *A, int step) {
    const Geom &g = c->g;
    const PicParams &p = c->p;
    AdjBcArgs B{};
    B.g = g;
    B.dt = p.dt; B.dx = p.dx; B.dy = p.dy; B.dz = p.dz;
    B.Pi = p.Pi; B.omega = p.omega; B.l0 = p.l0; B.amp = p.laser_amplitude; B.dur = p.laser_pulse_duration;
    B.start = p.laser_start_time; B.waist = p.waist; B.xfocus = p.xfocus; B.yfocus = p.yfocus; B.zfocus = p.zfocus;
    B.phase = p.phase; B.time = step * p.dt; B.pol = p.laser_polarization; B.envelope = p.laser_envelope;
    B.profile_n = c->profile_n;
    B.lprof = (p.laser_profile == 1 && c->d_profile) ? A->lprof : nullptr;
    real **F = (real **)A->lf;
    real **J = (real **)A->lj;
    dim3 blk(32, 8), grd((g.n[1] + 31) / 32, (g.n[2] + 7) / 8);
    prof_begin(c, "adjoint_boundary");
    adj_bc_kernel<real><<<grd, blk, 0, c->stream>>>(B, F[0], F[1], F[2], F[3], F[4], F[5], J[1], J[2]);
    prof_end(c);
}

template <typename real>
static int adj_backward_t(pic_ctx *c, AdjState *A, int nsteps) {
    for (int t = 0; t < nsteps; ++t) {
        if (A->tape_len == 0) {
            c->err = "adjoint: tape exhausted";
            return PIC_EINVAL;
        }
        const Blob &b = A->tape[--A->tape_len];
        const int step = b.step;   // 0: the t = 0 push; n >= 1: loop iteration n
        const bool loop = step >= 1;
        if (loop) {
            // second half (field.cpp:88-117): B then E forward, so E then B here
            adj_fields_e<real>(c, A);
            adj_fields_b<real>(c, A);
        }
        // push + deposit of both species, in reverse species order
        int base[2] = {0, 0};
        {
            int idx = 0;
            for (int k = 0; k < 2; ++k) {
                base[k] = idx;
                if (b.count[k] == 0) continue;
                idx += (c->fp32 ? 4 : 3) + 3 + (c->sp[k].dead ? 1 : 0);
            }
        }
        for (int k = 1; k >= 0; --k) {
            if (b.count[k] == 0) continue;
            if (c->order == 2) adj_push_launch<real, 3>(c, A, b, k, base[k], loop);
            else adj_push_launch<real, 5>(c, A, b, k, base[k], loop);
        }
        // the push ran right after a sort: back to the order before it
        for (int k = 0; k < 2; ++k)
            if (b.perm_part[k] >= 0) unsort_species(c, A, k, (const int *)blob_part(b, b.perm_part[k]), b.count[k]);
        // clear_currents: J before the clear does not reach the deposit
        prof_begin(c, "adjoint_clear");
        for (int f = 0; f < 3; ++f) cudaMemsetAsync(A->lj[f], 0, (size_t)c->g.rsz * rsize(c), c->stream);
        prof_end(c);
        if (loop) {
            // first half (field.cpp:56-86): E then B forward
            adj_fields_b<real>(c, A);
            adj_fields_e<real>(c, A);
            adj_bc<real>(c, A, step);
        }
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        c->err = std::string("adjoint: ") + cudaGetErrorString(e);
        return PIC_ECUDA;
    }
    return PIC_OK;
}

extern "C" {

int pic_checkpoint_save(pic_ctx *c, int slot) {
    if (!c || slot < 0) return PIC_EINVAL;
    AdjState *A = adj_of(c, true);
    if ((int)A->ckpt.size() <= slot) A->ckpt.resize(slot + 1);
    std::vector<std::pair<void *, size_t>> parts;
    checkpoint_parts(c, parts);
    return blob_save(c, A->ckpt[slot], parts);
}

int pic_checkpoint_restore(pic_ctx *c, int slot) {
    if (!c || slot < 0) return PIC_EINVAL;
    AdjState *A = adj_of(c, false);
    if (!A || slot >= (int)A->ckpt.size() || !A->ckpt[slot].buf) {
        c->err = "no such checkpoint";
        return PIC_EINVAL;
    }
    Blob &b = A->ckpt[slot];
    for (int k = 0; k < 2; ++k) {
        if (c->sp[k].n_host != b.count[k]) {
            c->err = "checkpoint particle count differs from the context's";
            return PIC_EINVAL;
        }
        c->sp[k].cur = b.cur[k];
    }
    // the arrays' current buffers (a sort since the save may have swapped them)
    std::vector<std::pair<void *, size_t>> parts;
    checkpoint_parts(c, parts);
    if (parts.size() != b.parts.size()) {
        c->err = "checkpoint layout differs from the context's";
        return PIC_EINVAL;
    }
    size_t off = 0;
    for (size_t i = 0; i < parts.size(); ++i) {
        cudaMemcpyAsync(parts[i].first, (char *)b.buf + off, parts[i].second, cudaMemcpyDeviceToDevice, c->stream);
        off += (parts[i].second + 255) & ~(size_t)255;
    }
    for (int k = 0; k < 2; ++k) {
        c->sp[k].sorted = false;   // the next push sorts (and the tape records that permutation)
        c->sp[k].perm_fresh = false;
    }
    c->step = b.step;
    return PIC_OK;
}

int pic_adjoint_tape(pic_ctx *c, int nsteps) {
    if (!c || nsteps < 0) return PIC_EINVAL;
    if (!c->p.adjoint) {
        c->err = "the context was not created with adjoint = 1";
        return PIC_EINVAL;
    }
    AdjState *A = adj_of(c, true);
    if ((int)A->tape.size() < nsteps) A->tape.resize(nsteps);
    A->tape_len = 0;
    if (c->tile > 0) {
        const size_t nt = (size_t)c->ntile[0] * c->ntile[1] * c->ntile[2] + 1;
        for (int k = 0; k < 2; ++k)
            if (!A->toffs[k] && cudaMalloc((void **)&A->toffs[k], nt * sizeof(unsigned)) != cudaSuccess) {
                A->toffs[k] = nullptr;
                c->err = "adjoint: out of device memory for the tile boundaries";
                return PIC_ENOMEM;
            }
    }
    return PIC_OK;
}

int pic_adjoint_record(pic_ctx *c, int on) {
    if (!c) return PIC_EINVAL;
    AdjState *A = adj_of(c, true);
    A->recording = on != 0;
    return PIC_OK;
}

int pic_adjoint_seed_kinetic(pic_ctx *c, int kind, double xlo, double xhi, double ramp, double *loss) {
    if (!c || kind < 0 || kind > 1 || !(ramp >= 0.0) || !(xhi >= xlo) || 2.0 * ramp > xhi - xlo) {
        if (c) c->err = "adjoint: window needs xlo <= xhi and 0 <= 2 ramp <= xhi - xlo";
        return PIC_EINVAL;
    }
    if (!c->p.adjoint) {
        c->err = "the context was not created with adjoint = 1";
        return PIC_EINVAL;
    }
    AdjState *A = adj_of(c, true);
    int r = ensure_adj_arrays(c, A);
    if (r) return r;
    const size_t rs = rsize(c);
    for (int f = 0; f < 6; ++f) cudaMemsetAsync(A->lf[f], 0, (size_t)c->g.fsz * rs, c->stream);
    for (int f = 0; f < 3; ++f) cudaMemsetAsync(A->lj[f], 0, (size_t)c->g.rsz * rs, c->stream);
    for (int k = 0; k < 2; ++k) {
        size_t n = (size_t)std::max<int64_t>(c->sp[k].cap, 1);
        for (int q = 0; q < 6; ++q) cudaMemsetAsync(A->lpart[k][q], 0, n * rs, c->stream);
        cudaMemsetAsync(A->lw[k], 0, n * sizeof(double), c->stream);
    }
    cudaMemsetAsync(A->lprof, 0, (size_t)A->nprof * sizeof(double), c->stream);
    cudaMemsetAsync(A->loss, 0, sizeof(double), c->stream);
    Species &s = c->sp[kind];
    long long n = s.n_host;
    if (n > 0) {
        unsigned blocks = (unsigned)((n + 255) / 256);
        if (c->fp32)
            adj_seed_kinetic_kernel<float><<<blocks, 256, 0, c->stream>>>(
                c->g, c->cp, 1, n, nullptr, s.a.cell[s.cur], s.a.ox[s.cur], (float *)s.a.px, (float *)s.a.py,
                (float *)s.a.pz, (float *)s.a.w, s.dead, c->p.mass[kind], xlo, xhi, ramp, (float *)A->lpart[kind][0], (float *)A->lpart[kind][3],
                (float *)A->lpart[kind][4], (float *)A->lpart[kind][5], A->lw[kind], A->loss);
        else
            adj_seed_kinetic_kernel<double><<<blocks, 256, 0, c->stream>>>(
                c->g, c->cp, 0, n, s.a.x[s.cur], nullptr, nullptr, (double *)s.a.px, (double *)s.a.py,
                (double *)s.a.pz, (double *)s.a.w, s.dead, c->p.mass[kind], xlo, xhi, ramp, (double *)A->lpart[kind][0], (double *)A->lpart[kind][3],
                (double *)A->lpart[kind][4], (double *)A->lpart[kind][5], A->lw[kind], A->loss);
    }
    note_adjoint_order(c, A);
    double l = 0.0;
    cudaMemcpyAsync(&l, A->loss, sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return PIC_ECUDA;
    if (loss) *loss = l;
    return PIC_OK;
}

int pic_adjoint_backward(pic_ctx *c, int nsteps) {
    if (!c || nsteps < 0) return PIC_EINVAL;
    AdjState *A = adj_of(c, false);
    if (!A || !A->lf[0]) {
        c->err = "adjoint: seed the objective first";
        return PIC_EINVAL;
    }
    remap_adjoints(c, A);
    int r = c->fp32 ? adj_backward_t<float>(c, A, nsteps) : adj_backward_t<double>(c, A, nsteps);
    note_adjoint_order(c, A);
    return r;
}

int pic_adjoint_weight_grad(pic_ctx *c, int kind, double *out, int64_t n) {
    if (!c || kind < 0 || kind > 1 || !out) return PIC_EINVAL;
    AdjState *A = adj_of(c, false);
    if (!A || !A->lw[kind]) return PIC_EINVAL;
    if (n > c->sp[kind].n_host) n = c->sp[kind].n_host;
    const double *src = A->lw[kind];
    Species &s = c->sp[kind];
    if (s.orig && n > 0 && s.n_host > 0) {   // sorted context: back to upload order
        scatter_to(c, A->lw[kind], s.orig, A->tmp, sizeof(double), s.n_host);
        src = (const double *)A->tmp;
    }
    cudaMemcpyAsync(out, src, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    return cudaStreamSynchronize(c->stream) == cudaSuccess ? PIC_OK : PIC_ECUDA;
}

int pic_adjoint_profile_grad(pic_ctx *c, double *out, int n) {
    if (!c || !out) return PIC_EINVAL;
    AdjState *A = adj_of(c, false);
    if (!A || !A->lprof) return PIC_EINVAL;
    n = std::min(n, A->nprof);
    cudaMemcpyAsync(out, A->lprof, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    return cudaStreamSynchronize(c->stream) == cudaSuccess ? PIC_OK : PIC_ECUDA;
}

int pic_adjoint_release(pic_ctx *c) {
    if (!c) return PIC_EINVAL;
    for (size_t i = 0; i < g_adj.size(); ++i) {
        if (g_adj[i].first != c) continue;
        AdjState *A = g_adj[i].second;
        for (auto &b : A->ckpt)
            if (b.buf) cudaFree(b.buf);
        for (auto &b : A->tape)
            if (b.buf) cudaFree(b.buf);
        for (void *p : A->lf) if (p) cudaFree(p);
        for (void *p : A->lj) if (p) cudaFree(p);
        for (auto &sp : A->lpart) for (void *p : sp) if (p) cudaFree(p);
        for (double *p : A->lw) if (p) cudaFree(p);
        if (A->lprof) cudaFree(A->lprof);
        if (A->loss) cudaFree(A->loss);
        for (int *p : A->lam_orig) if (p) cudaFree(p);
        for (unsigned *p : A->toffs) if (p) cudaFree(p);
        if (A->tmp) cudaFree(A->tmp);
        delete A;
        g_adj.erase(g_adj.begin() + (long)i);
        return PIC_OK;
    }
    return PIC_OK;
}

}  // extern "C"
