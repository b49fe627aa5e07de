// Per-particle body of update_particle_position_momentum
// (src/particle.cpp:113-370) with currents_particle (:372-515), shared by
// the global-memory kernel and the tiled shared-memory kernel.  Field reads
// and current adds go through `View`s, so the same code addresses either
// the global buffers or a CTA's shared-memory tile.
#pragma once

#include <cuda/std/type_traits>

#include "pic_internal.cuh"

namespace pic {

// Record particle p (home tile `home`) if its new cell lies in another tile.
// A cell outside the grid on a periodic axis (an FP64 position exactly at
// x = n, wrapped only at the next push) cannot be binned: the next push
// falls back to the global kernel for particles away from home.  Outside on
// a non-periodic axis the particle is removed before the next push.
// `here`, `lo`: a tile the cell is likely in (the pushing CTA's) and its
// first cell per axis (here < 0: none), which spares the divisions.
__device__ __forceinline__ void vis_note(const VisSink &v, const Geom &g, int p, int home, const int (&cell)[3],
                                         int here = -1, const int *lo = nullptr) {
    if (!v.raw) return;
    int t = -1;
    if (here >= 0) {
        bool in_here = true;
#pragma unroll
        for (int d = 0; d < 3; ++d) in_here = in_here && cell[d] >= lo[d] && cell[d] < lo[d] + v.T;
        if (in_here) t = here;
    }
    if (t == home) return;
    if (t < 0) {
        bool in = true, per_out = false;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const bool o = cell[d] < 0 || cell[d] >= g.n[d];
            in = in && !o;
            per_out = per_out || (o && g.per[d]);
        }
        if (!in) {
            if (per_out) v.vs->valid_next = 0u;
            return;
        }
        t = ((cell[2] / v.T) * v.nt[1] + cell[1] / v.T) * v.nt[0] + cell[0] / v.T;
        if (t == home) return;
    }
    const unsigned long long s = atomicAdd(&v.vs->nraw, 1ull);
    if ((long long)s >= v.cap) {
        v.vs->valid_next = 0u;
        return;
    }
    v.raw[3 * s] = p;
    v.raw[3 * s + 1] = home;
    v.raw[3 * s + 2] = t;
}

template <typename real>
struct PushArgs {
    Geom g;
    const real *ex, *ey, *ez, *bx, *by, *bz;
    real *jx, *jy, *jz, *rho;
    const long long *count;
    const int *idx;          // optional list of particle indices (count entries); null: all particles
    int idx_pairs;           // idx holds (index, home tile) pairs
    VisSink vsink;           // visitor recording (raw null: off)
    const unsigned char *dead;   // adjoint mode: particles already removed are skipped (null otherwise)
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
    int electron;            // spin precession applies to this species (particle.cpp:318-319)
    unsigned *status;
};

// A 3D array seen through buffer coordinates: element (k, j, i) is at
// p[k*sz + j*sy + i + o].
template <typename T>
struct View {
    T *p;
    int sy, sz, o;
    __device__ __forceinline__ T *at(int k, int j, int i) const { return p + (k * sz + j * sy + i + o); }
};

__device__ __forceinline__ void set_status(unsigned *s, unsigned bit) { atomicOr(s, bit); }

// a[i] for a register array and a run-time index, as a chain of selects
// (keeps `a` in registers; used where an outer stencil loop stays rolled to
// keep the kernel's code small enough for the instruction cache)
template <typename T, int N>
__device__ __forceinline__ T pick(const T (&a)[N], int i) {
    T v = a[0];
#pragma unroll
    for (int q = 1; q < N; ++q) v = (i == q) ? a[q] : v;
    return v;
}

// g_factor lookup (src/particle.cpp:603-637)
__device__ __forceinline__ double g_factor_dev(const double *tab, int n, double x, unsigned *status) {
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

// factorised P^3 gather of one staggered component, starting at (k0,j0,i0)
// The outer loop is unrolled too except for FP32 at 4th order, whose fully
// unrolled kernel overflows the instruction cache (unrolled: FP32 2nd order
// 6 % faster, FP64 1-3 %; FP32 4th order 8 % slower).
template <typename real, int P>
__device__ __forceinline__ constexpr bool gather_rolled() { return sizeof(real) == 4 && P == 5; }

template <typename real, int P, bool LDG>
__device__ __forceinline__ real gather_plane(const real *plane, int sy, const real (&wx)[P], const real (&wy)[P]) {
    real acck = 0;
#pragma unroll
    for (int j = 0; j < P; ++j) {
        const real *row = plane + j * sy;
        real s = 0;
#pragma unroll
        for (int i = 0; i < P; ++i) s += wx[i] * (LDG ? __ldg(row + i) : row[i]);
        acck += wy[j] * s;
    }
    return acck;
}

template <typename real, int P, bool LDG>
__device__ __forceinline__ real gather(const View<const real> &v, int i0, int j0, int k0, const real (&wx)[P],
                                       const real (&wy)[P], const real (&wz)[P]) {
    const real *base = v.at(k0, j0, i0);
    real acc = 0;
    if constexpr (gather_rolled<real, P>()) {
#pragma unroll 1
        for (int k = 0; k < P; ++k) acc += pick(wz, k) * gather_plane<real, P, LDG>(base + k * v.sz, v.sy, wx, wy);
    } else {
#pragma unroll
        for (int k = 0; k < P; ++k) acc += wz[k] * gather_plane<real, P, LDG>(base + k * v.sz, v.sy, wx, wy);
    }
    return acc;
}

// One axis of a particle's Esirkepov move (src/particle.cpp:403-419): the
// union span of the old and new supports starts at buffer index `base` and
// has `len` points (P, or P + 1 when the primal index changed; |i2 - i1| <= 1
// is checked by the caller); s0 = old shape, ds = new - old, both zero
// outside their supports; w1 = new shape on i2 - H .. i2 + H (rho).
template <typename real, int P>
struct Axis1D {
    int base, len, i2;
    real s0[P + 1], ds[P + 1], w1[P];
};

// From the old and new primal offsets in FP64 (FP64 positions, and the
// single-record deposit of either precision): both weight sets in FP64 and
// ds as their difference, as the reference forms it.
template <typename real, int P>
__device__ __forceinline__ void axis_from_offsets(int i1, double d0, int i2, double d1, Axis1D<real, P> &ax) {
    constexpr int H = P / 2;
    double w0[P], w1[P];
    shape_weights(d0, w0);
    shape_weights(d1, w1);
    const int lo = min(i1, i2);
    ax.base = lo - H;
    ax.len = P + abs(i2 - i1);
    ax.i2 = i2;
    const bool o0 = i1 != lo, o1 = i2 != lo;
#pragma unroll
    for (int a = 0; a <= P; ++a) {
        double v0 = o0 ? (a >= 1 ? w0[a - 1] : 0.0) : (a < P ? w0[a] : 0.0);
        double v1 = o1 ? (a >= 1 ? w1[a - 1] : 0.0) : (a < P ? w1[a] : 0.0);
        ax.s0[a] = (real)v0;
        ax.ds[a] = (real)(v1 - v0);
    }
#pragma unroll
    for (int q = 0; q < P; ++q) ax.w1[q] = (real)w1[q];
}

// Change of the shape weights over a move by e that stays on one polynomial
// piece: dw[k] = w_k(d + e) - w_k(d), formed without subtracting weights.
// Every term carries a factor e, so a slow particle's differences keep full
// FP32 relative accuracy.  The outer weights are binomial expansions of
// their single powers; the inner ones follow from the two identities every
// B-spline shape satisfies, sum_k w_k = 1 and sum_k k w_k = d (centred k),
// which give sum_k dw_k = 0 and sum_k k dw_k = e.
__device__ __forceinline__ void shape_diff(float d, float e, float (&dw)[3]) {
    const float a = 0.5f - d, b = 0.5f + d;
    dw[0] = 0.5f * e * (e - 2.0f * a);
    dw[2] = 0.5f * e * (2.0f * b + e);
    dw[1] = -(dw[0] + dw[2]);
}

__device__ __forceinline__ float quartic_step(float x, float e) {   // (x + e)^4 - x^4
    return e * (4.0f * x * x * x + e * (6.0f * x * x + e * (4.0f * x + e)));
}

__device__ __forceinline__ void shape_diff(float d, float e, float (&dw)[5]) {
    dw[0] = quartic_step(d - 0.5f, e) * (1.0f / 24.0f);
    dw[4] = quartic_step(d + 0.5f, e) * (1.0f / 24.0f);
    dw[2] = 0.25f * quartic_step(d, e) - 0.625f * e * (2.0f * d + e);
    const float sum = dw[0] + dw[2] + dw[4];             // = -(dw1 + dw3)
    const float mom = e + 2.0f * dw[0] - 2.0f * dw[4];   // =   dw3 - dw1
    dw[1] = -0.5f * (sum + mom);
    dw[3] = 0.5f * (mom - sum);
}

// FP32: old primal index i1 and offset d0 in [-1/2, 1/2), move e (cells),
// new primal index i2 (from the stored new position).  A move that crosses
// the knot between two primal indices (offset 1/2) is split there: the old
// support's change up to the knot plus the new support's change from it.
template <int P>
__device__ __forceinline__ void axis_from_move(int i1, float d0, float e, int i2, Axis1D<float, P> &ax) {
    constexpr int H = P / 2;
    float w0[P];
    shape_weights(d0, w0);
    ax.i2 = i2;
    if (i2 == i1) {
        float dw[P];
        shape_diff(d0, e, dw);
        ax.base = i1 - H;
        ax.len = P;
#pragma unroll
        for (int a = 0; a < P; ++a) {
            ax.s0[a] = w0[a];
            ax.ds[a] = dw[a];
        }
        ax.s0[P] = 0.0f;
        ax.ds[P] = 0.0f;
        shape_weights(d0 + e, ax.w1);
        return;
    }
    const bool up = i2 > i1;
    const float t0 = (up ? 0.5f : -0.5f) - d0;   // old offset to the knot
    const float t1 = e - t0;                        // knot to the new position
    float dold[P], dnew[P];
    shape_diff(d0, t0, dold);
    shape_diff(up ? -0.5f : 0.5f, t1, dnew);
    ax.base = min(i1, i2) - H;
    ax.len = P + 1;
#pragma unroll
    for (int a = 0; a <= P; ++a) {
        // lower support at a = 0 .. P-1, upper at a = 1 .. P
        const float lo_o = a < P ? (up ? dold[a] : dnew[a]) : 0.0f;
        const float hi_o = a >= 1 ? (up ? dnew[a - 1] : dold[a - 1]) : 0.0f;
        ax.ds[a] = lo_o + hi_o;
        ax.s0[a] = up ? (a < P ? w0[a] : 0.0f) : (a >= 1 ? w0[a - 1] : 0.0f);
    }
    shape_weights((up ? -0.5f : 0.5f) + t1, ax.w1);
}

__device__ __forceinline__ void atomic_add(double *p, double v) { atomicAdd(p, v); }
__device__ __forceinline__ void atomic_add(float *p, float v) { atomicAdd(p, v); }

// Where deposited current goes.  Both accumulators address a 3D array
// through buffer coordinates with strides (sy, sz) and offset o, like View.
// The deposit multiplies every value by coef(c) before add(c, ...).
//   GlobalAcc: hardware atomics into the global ring buffers (coef 1).
//   FixedAcc:  a CTA's shared-memory tile; values come scaled by
//              coef(c) = scale[c], are rounded to a 64-bit integer and split
//              into 18-bit limbs added with native 32-bit integer atomics
//              (NL = 2 limbs for FP32, 3 for FP64).  Integer sums do not
//              depend on the order of the additions.  (Shared-memory 64-bit
//              integer atomics measured 2.6x slower on the whole kernel.)
// One contribution stays below 2^kFixedBits (31 FP32, 49 FP64), so that
// 16383 additions per point fit: the unsigned 18-bit limb sums in 32 bits,
// the signed top limb sums (below 2^13 resp. 2^15 each) in 32 bits, and
// the reassembled total in 64 bits.
constexpr int kLimbBits = 18;
constexpr unsigned kLimbMask = (1u << kLimbBits) - 1u;
template <typename real>
constexpr int fixed_bits() { return sizeof(real) == 8 ? 49 : 31; }
template <typename real>
struct GlobalAcc {
    real *p[4];  // jx, jy, jz, rho (rho may be null)
    int sy, sz, o;
    __device__ __forceinline__ bool has_rho() const { return p[3] != nullptr; }
    __device__ __forceinline__ real coef(int) const { return real(1); }
    __device__ __forceinline__ void add(int c, int idx, real v) const { atomic_add(p[c] + idx, v); }
};

template <typename real, int NL>
struct FixedAcc {
    unsigned *p[4];   // limb 0 of jx, jy, jz, rho; limb l at + l * lstride
    int lstride;
    int sy, sz, o;
    real scale[4];    // per component: |value * scale| < 2^fixed_bits
    __device__ __forceinline__ bool has_rho() const { return p[3] != nullptr; }
    __device__ __forceinline__ real coef(int c) const { return scale[c]; }
    // q is already scaled.  Rounded to the nearest integer and split into
    // limbs q = l2*2^36 + l1*2^18 + l0 (FP64) or q = h*2^18 + l0 (FP32),
    // with l0, l1 in [0, 2^18) and the top limb signed.  FP64 rounds by the
    // add-a-magic-constant method (the sum's low mantissa bits are the
    // integer), FP32 by a float-to-int conversion.  Zeros are added like
    // any value: a per-point zero test measured 10-20 % slower than the
    // shared atomics it saves.
    __device__ __forceinline__ void add(int c, int idx, real q) const {
        unsigned *a = p[c] + idx;
        if constexpr (NL == 3) {                                           // |q| < 2^51
            const long long qi = __double_as_longlong(q + 6755399441055744.0) - 0x4338000000000000LL;
            atomicAdd(a, (unsigned)qi & kLimbMask);
            atomicAdd(a + lstride, (unsigned)(qi >> kLimbBits) & kLimbMask);
            atomicAdd(a + 2 * lstride, (unsigned)(int)(qi >> (2 * kLimbBits)));
        } else {                                                           // |q| < 2^31
            const int qi = __float2int_rn(q);
            atomicAdd(a, (unsigned)qi & kLimbMask);
            atomicAdd(a + lstride, (unsigned)(qi >> kLimbBits));
        }
    }
};

// The middle loop of a current component over m = 0 .. len-1 (len <= P+1),
// calling body(m, s0[m], ds[m]): fully unrolled, or rolled with the two
// weights picked from registers.
template <bool ROLL, int P, typename real, class F>
__device__ __forceinline__ void mid_loop(int len, const real (&s0)[P + 1], const real (&ds)[P + 1], F &&body) {
    if constexpr (ROLL) {
#pragma unroll 1
        for (int m = 0; m <= P; ++m) {
            if (m >= len) break;
            body(m, pick(s0, m), pick(ds, m));
        }
    } else {
#pragma unroll
        for (int m = 0; m <= P; ++m) {
            if (m >= len) break;
            body(m, s0[m], ds[m]);
        }
    }
}

// Esirkepov deposit (src/particle.cpp:427-500) and rho (:503-514) from the
// three axes' factors.  The last point of each running sum (the sum of all
// ds, zero up to rounding) is not added.  `moved`: the particle changed
// position (one at rest adds no current, only rho).
template <typename real, int P, class Acc>
__device__ __forceinline__ void deposit(const Acc &acc, const real (&dxdt)[3], const Axis1D<real, P> (&ax)[3],
                                        bool moved, real qw) {
    constexpr int H = P / 2;
    const int base[3] = {ax[0].base, ax[1].base, ax[2].base};
    const int len[3] = {ax[0].len, ax[1].len, ax[2].len};
    const real(&s0x)[P + 1] = ax[0].s0;
    const real(&s0y)[P + 1] = ax[1].s0;
    const real(&s0z)[P + 1] = ax[2].s0;
    const real(&dsx)[P + 1] = ax[0].ds;
    const real(&dsy)[P + 1] = ax[1].ds;
    const real(&dsz)[P + 1] = ax[2].ds;
    const real third = real(1.0 / 3.0), half = real(0.5);
    const real cx = qw * dxdt[0] * acc.coef(0), cy = qw * dxdt[1] * acc.coef(1), cz = qw * dxdt[2] * acc.coef(2);
    const int rx = acc.sy, rxy = acc.sz;
    const int r0 = base[2] * rxy + base[1] * rx + base[0] + acc.o;
    // The middle loops stay rolled for FP32 at 4th order: its fully unrolled
    // code overflows the instruction cache (measured 10 % faster rolled),
    // while FP64 and 2nd order run faster unrolled.
    constexpr bool kRollMid = sizeof(real) == 4 && P == 5;
    if (moved) {
        // Jx: running sum of ds along x times the yz weight
#pragma unroll 1
        for (int k = 0; k < len[2]; ++k) {
            const real sz0 = pick(s0z, k), szd = pick(dsz, k);
            mid_loop<kRollMid, P>(len[1], s0y, dsy, [&](int j, real sy0, real syd) {
                const real wyz = sy0 * sz0 + half * syd * sz0 + half * sy0 * szd + third * syd * szd;
                const real cw = -cx * wyz;
                real a = 0;
                const int row = r0 + k * rxy + j * rx;
#pragma unroll
                for (int i = 0; i < P; ++i) {
                    if (i >= len[0] - 1) break;
                    a += dsx[i];
                    acc.add(0, row + i, cw * a);
                }
            });
        }
        // Jy
#pragma unroll 1
        for (int k = 0; k < len[2]; ++k) {
            const real sz0 = pick(s0z, k), szd = pick(dsz, k);
            mid_loop<kRollMid, P>(len[0], s0x, dsx, [&](int i, real sx0, real sxd) {
                const real wxz = sx0 * sz0 + half * sxd * sz0 + half * sx0 * szd + third * sxd * szd;
                const real cw = -cy * wxz;
                real a = 0;
                const int col = r0 + k * rxy + i;
#pragma unroll
                for (int j = 0; j < P; ++j) {
                    if (j >= len[1] - 1) break;
                    a += dsy[j];
                    acc.add(1, col + j * rx, cw * a);
                }
            });
        }
        // Jz
#pragma unroll 1
        for (int j = 0; j < len[1]; ++j) {
            const real sy0 = pick(s0y, j), syd = pick(dsy, j);
            mid_loop<kRollMid, P>(len[0], s0x, dsx, [&](int i, real sx0, real sxd) {
                const real wxy = sx0 * sy0 + half * sxd * sy0 + half * sx0 * syd + third * sxd * syd;
                const real cw = -cz * wxy;
                real a = 0;
                const int col = r0 + j * rx + i;
#pragma unroll
                for (int k = 0; k < P; ++k) {
                    if (k >= len[2] - 1) break;
                    a += dsz[k];
                    acc.add(2, col + k * rxy, cw * a);
                }
            });
        }
    }
    if (acc.has_rho()) {
        const real qwr = qw * acc.coef(3);
        const int rb = (ax[2].i2 - H) * rxy + (ax[1].i2 - H) * rx + (ax[0].i2 - H) + acc.o;
#pragma unroll 1
        for (int k = 0; k < P; ++k) {
            const real wk = qwr * pick(ax[2].w1, k);
#pragma unroll
            for (int j = 0; j < P; ++j) {
                real wjk = wk * ax[1].w1[j];
#pragma unroll
                for (int i = 0; i < P; ++i) acc.add(3, rb + k * rxy + j * rx + i, wjk * ax[0].w1[i]);
            }
        }
    }
}

// Decoded old position of particle p: primal / dual buffer index and
// offset per axis.  FP64 applies the push-time periodic wrap
// (particle.cpp:123-167) and writes the wrapped position back.
template <typename real>
struct OldPos {
    int ip[3], id[3];
    real dp[3], dd[3];
    double xd[3];
    int cc[3];
    real oo[3];
};

// What one push reads of particle p: FP64 position (x, y, z) or FP32 packed
// cell + offsets, then momenta and weight, as words of the precision's size
// (so that the tile kernel can stage them with asynchronous copies).
template <typename real>
struct PartIn {
    using word = typename cuda::std::conditional<sizeof(real) == 8, unsigned long long, unsigned>::type;
    static constexpr int kWords = sizeof(real) == 8 ? 7 : 8;   // all inputs
    static constexpr int kPos = sizeof(real) == 8 ? 3 : 4;     // the position words
    word v[kWords];
};

// where push_body reads momenta and weight: the particle arrays (i = the
// particle) or rows of the tile kernel's staging buffer (i = the lane)
template <typename real>
struct PmSrc {
    const real *px, *py, *pz, *w;
    long long i;
};

template <typename real>
__device__ __forceinline__ const typename PartIn<real>::word *particle_word_src(const PushArgs<real> &a, long long p,
                                                                                 int k) {
    using word = typename PartIn<real>::word;
    if constexpr (sizeof(real) == 8) {
        const double *src[7] = {a.x0, a.y0, a.z0, a.px, a.py, a.pz, a.w};
        return reinterpret_cast<const word *>(src[k] + p);
    } else {
        const void *src[8] = {a.c0, a.ox0, a.oy0, a.oz0, a.px, a.py, a.pz, a.w};
        return reinterpret_cast<const word *>(src[k]) + p;
    }
}

template <typename real>
__device__ __forceinline__ void load_position(const PushArgs<real> &a, long long p, PartIn<real> &in) {
#pragma unroll
    for (int k = 0; k < PartIn<real>::kPos; ++k) in.v[k] = *particle_word_src(a, p, k);
}

template <typename real>
__device__ __forceinline__ real part_real(const PartIn<real> &in, int k) {
    if constexpr (sizeof(real) == 8) return __longlong_as_double((long long)in.v[k]);
    else return __uint_as_float(in.v[k]);
}

template <typename real>
__device__ __forceinline__ void decode_old(const PushArgs<real> &a, long long p, const PartIn<real> &in,
                                           OldPos<real> &o) {
    constexpr bool F64 = cuda::std::is_same<real, double>::value;
    const Geom &g = a.g;
    if constexpr (F64) {
        o.xd[0] = part_real(in, 0);
        o.xd[1] = part_real(in, 1);
        o.xd[2] = part_real(in, 2);
        bool wrapped = false;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (g.per[d]) {
                if (o.xd[d] < 0.0) { o.xd[d] += g.n[d]; wrapped = true; }
                if (o.xd[d] > (double)g.n[d]) { o.xd[d] -= g.n[d]; wrapped = true; }
            }
        }
        if (wrapped) {
            a.x0[p] = o.xd[0];
            a.y0[p] = o.xd[1];
            a.z0[p] = o.xd[2];
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            double xc = o.xd[d] - (double)(1 - g.mem);
            o.ip[d] = (int)(xc + 0.5);
            o.dp[d] = xc - (double)o.ip[d];
            o.id[d] = (int)xc;
            o.dd[d] = (xc - 0.5) - (double)o.id[d];
        }
    } else {
        a.cp.unpack((int)in.v[0], o.cc[0], o.cc[1], o.cc[2]);
        o.oo[0] = __uint_as_float(in.v[1]);
        o.oo[1] = __uint_as_float(in.v[2]);
        o.oo[2] = __uint_as_float(in.v[3]);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            int b = o.cc[d] + g.mem - 1;
            bool up = o.oo[d] >= 0.5f;
            o.ip[d] = b + (up ? 1 : 0);
            o.dp[d] = up ? o.oo[d] - 1.0f : o.oo[d];
            o.id[d] = b;
            o.dd[d] = o.oo[d] - 0.5f;
        }
    }
}

// Everything after the position decode: gather, Boris, move, deposit,
// store, spin.  fv: the six field views; jv: view for the current arrays
// (jx..rho share its strides).
// Returns false when the particle was skipped (non-finite momentum or a move
// over a cell: status set, nothing stored).  The new state is stored before
// the deposit (fewer values live through its loops); note(cnew) is called
// then with the new cell as the next push's decode will see it.
template <typename real, int P, bool SPIN, bool LDG, class Acc, class Note>
__device__ __forceinline__ bool push_body(const PushArgs<real> &a, long long p, const OldPos<real> &o,
                                          const PmSrc<real> &pm, const View<const real> (&fv)[6], const Acc &acc,
                                          Note &&note) {
    int cnew[3];
    constexpr bool F64 = cuda::std::is_same<real, double>::value;
    constexpr int H = P / 2;
    const Geom &g = a.g;
    real wp[3][P], wd[3][P];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        shape_weights(o.dp[d], wp[d]);
        shape_weights(o.dd[d], wd[d]);
    }
    // gather with Yee staggering (particle.cpp:207-259)
    const int *ip = o.ip, *id = o.id;
    real e0 = gather<real, P, LDG>(fv[0], id[0] - H, ip[1] - H, ip[2] - H, wd[0], wp[1], wp[2]);
    real e1 = gather<real, P, LDG>(fv[1], ip[0] - H, id[1] - H, ip[2] - H, wp[0], wd[1], wp[2]);
    real e2 = gather<real, P, LDG>(fv[2], ip[0] - H, ip[1] - H, id[2] - H, wp[0], wp[1], wd[2]);
    real b0 = gather<real, P, LDG>(fv[3], ip[0] - H, id[1] - H, id[2] - H, wp[0], wd[1], wd[2]);
    real b1 = gather<real, P, LDG>(fv[4], id[0] - H, ip[1] - H, id[2] - H, wd[0], wp[1], wd[2]);
    real b2 = gather<real, P, LDG>(fv[5], id[0] - H, id[1] - H, ip[2] - H, wd[0], wd[1], wp[2]);
    // Boris (particle.cpp:271-306)
    const real qm = a.qm;
    real ex_p = e0 * qm, ey_p = e1 * qm, ez_p = e2 * qm;
    real bx_p = b0 * qm, by_p = b1 * qm, bz_p = b2 * qm;
    real px1 = pm.px[pm.i] + ex_p, py1 = pm.py[pm.i] + ey_p, pz1 = pm.pz[pm.i] + ez_p;
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
    // move in cell units (particle.cpp:313-315)
    int i2[3];
    double d2[3];   // FP64: new primal offsets
    double xn[3];
    int cn[3];
    real on[3];
    real disp[3];   // FP32: the move in cells
    if constexpr (F64) {
        xn[0] = o.xd[0] + (double)pxn / (double)gam * a.dt_s / a.dxs[0];
        xn[1] = o.xd[1] + (double)pyn / (double)gam * a.dt_s / a.dxs[1];
        xn[2] = o.xd[2] + (double)pzn / (double)gam * a.dt_s / a.dxs[2];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            double xc = xn[d] - (double)(1 - g.mem);
            i2[d] = (int)(xc + 0.5);
            d2[d] = xc - (double)i2[d];
        }
    } else {
        disp[0] = pxn / gam * a.dt_d[0];
        disp[1] = pyn / gam * a.dt_d[1];
        disp[2] = pzn / gam * a.dt_d[2];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            // stored position: cell + FP32 offset in [0, 1)
            real q = o.oo[d] + disp[d];
            int s = 0;
            if (q >= real(1)) { q -= real(1); s = 1; }
            else if (q < real(0)) {
                q += real(1);
                s = -1;
                if (q >= real(1)) { q = real(0); s = 0; }
            }
            cn[d] = o.cc[d] + s;
            on[d] = q;
            // new primal index of the stored position
            i2[d] = cn[d] + g.mem - 1 + (q >= real(0.5) ? 1 : 0);
        }
    }
    bool fin = isfinite(pxn) && isfinite(pyn) && isfinite(pzn);
    bool cfl = abs(i2[0] - ip[0]) <= 1 && abs(i2[1] - ip[1]) <= 1 && abs(i2[2] - ip[2]) <= 1;
    if (!fin || !cfl) {
        set_status(a.status, fin ? ST_CFL : ST_NAN);
        return false;
    }
    // store
    a.px[p] = pxn;
    a.py[p] = pyn;
    a.pz[p] = pzn;
    if constexpr (F64) {
        a.x1[p] = xn[0];
        a.y1[p] = xn[1];
        a.z1[p] = xn[2];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            // the wrap and truncation of decode_old
            double v = xn[d];
            if (g.per[d]) {
                if (v < 0.0) v += g.n[d];
                if (v > (double)g.n[d]) v -= g.n[d];
            }
            const double xc = v - (double)(1 - g.mem);
            cnew[d] = xc >= 0.0 ? (int)xc - (g.mem - 1) : -1;
        }
    } else {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (g.per[d]) cn[d] = cn[d] < 0 ? cn[d] + g.n[d] : (cn[d] >= g.n[d] ? cn[d] - g.n[d] : cn[d]);
            cnew[d] = cn[d];
        }
        a.c1[p] = a.cp.pack(cn[0], cn[1], cn[2]);
        a.ox1[p] = on[0];
        a.oy1[p] = on[1];
        a.oz1[p] = on[2];
    }
    note(cnew);
    const real qw = a.charge * pm.w[pm.i];
    Axis1D<real, P> ax[3];
    bool moved = false;
    if constexpr (F64) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            axis_from_offsets<real, P>(o.ip[d], o.dp[d], i2[d], d2[d], ax[d]);
            moved = moved || i2[d] != o.ip[d] || d2[d] != o.dp[d];
        }
    } else {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            axis_from_move<P>(o.ip[d], o.dp[d], disp[d], i2[d], ax[d]);
            moved = moved || disp[d] != real(0);
        }
    }
    deposit<real, P>(acc, a.d_dt, ax, moved, qw);
    // electron spin precession (particle.cpp:318-368)
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
    return true;
}

// bounds check of the old position against the global buffers: the whole
// gather and deposit stencil must stay inside (see the ring / field extents)
template <typename real>
__device__ __forceinline__ bool in_buffers(const Geom &g, const OldPos<real> &o, int H) {
    bool ok = true;
#pragma unroll
    for (int d = 0; d < 3; ++d) ok = ok && o.id[d] >= H && o.ip[d] <= g.f[d] - 1 - H;
    return ok;
}

template <typename real>
__device__ __forceinline__ void global_views(const PushArgs<real> &a, View<const real> (&fv)[6],
                                             GlobalAcc<real> &acc) {
    const Geom &g = a.g;
    const real *f[6] = {a.ex, a.ey, a.ez, a.bx, a.by, a.bz};
#pragma unroll
    for (int c = 0; c < 6; ++c) fv[c] = View<const real>{f[c], g.f[0], g.fxy, 0};
    acc = GlobalAcc<real>{{a.jx, a.jy, a.jz, a.rho}, g.r[0], g.rxy, g.rxy + g.r[0] + 1};
}

// spin precession runs for electrons (mass == m_e, particle.cpp:319) when
// enabled and some spin is non-zero (with all spins zero it is an exact no-op)
inline bool spin_active(const pic_ctx *c, int kind) {
    const Species &s = c->sp[kind];
    return c->p.spin && s.a.sx && s.spin_nonzero && c->p.mass[kind] == 1.0;
}

// kernel arguments for species `kind` of context c (host side)
template <typename real>
inline PushArgs<real> make_push_args(pic_ctx *c, int kind) {
    Species &s = c->sp[kind];
    PushArgs<real> a{};
    a.g = c->g;
    real **F = (real **)c->field;
    real **R = (real **)c->ring;
    a.ex = F[0]; a.ey = F[1]; a.ez = F[2]; a.bx = F[3]; a.by = F[4]; a.bz = F[5];
    a.jx = R[0]; a.jy = R[1]; a.jz = R[2];
    a.rho = (c->p.deposit_rho && !c->rho_skip) ? R[3 + kind] : nullptr;
    a.count = s.d_count;
    const int cu = s.cur, nx = 1 - s.cur;
    a.x0 = s.a.x[cu]; a.y0 = s.a.y[cu]; a.z0 = s.a.z[cu];
    a.x1 = s.a.x[nx]; a.y1 = s.a.y[nx]; a.z1 = s.a.z[nx];
    a.c0 = s.a.cell[cu]; a.ox0 = s.a.ox[cu]; a.oy0 = s.a.oy[cu]; a.oz0 = s.a.oz[cu];
    a.c1 = s.a.cell[nx]; a.ox1 = s.a.ox[nx]; a.oy1 = s.a.oy[nx]; a.oz1 = s.a.oz[nx];
    a.cp = c->cp;
    a.px = (real *)s.a.px; a.py = (real *)s.a.py; a.pz = (real *)s.a.pz; a.w = (const real *)s.a.w;
    a.sx = (real *)s.a.sx; a.sy = (real *)s.a.sy; a.sz = (real *)s.a.sz;
    a.gtab = c->d_gtab; a.gtab_n = c->gtab_n;
    const PicParams &p = c->p;
    a.qm = (real)(p.charge[kind] / p.mass[kind] * p.dt_half);
    a.charge = (real)p.charge[kind];
    a.dt_d[0] = (real)(p.dt / p.dx); a.dt_d[1] = (real)(p.dt / p.dy); a.dt_d[2] = (real)(p.dt / p.dz);
    a.dt_s = p.dt; a.dxs[0] = p.dx; a.dxs[1] = p.dy; a.dxs[2] = p.dz;
    a.d_dt[0] = (real)(p.dx / p.dt); a.d_dt[1] = (real)(p.dy / p.dt); a.d_dt[2] = (real)(p.dz / p.dt);
    a.E_schwinger = p.E_schwinger; a.dt_half_d = p.dt_half; a.charge_d = p.charge[kind]; a.mass_d = p.mass[kind];
    a.electron = spin_active(c, kind) ? 1 : 0;
    a.status = c->d_status;
    a.dead = s.dead;
    return a;
}

}  // namespace pic
