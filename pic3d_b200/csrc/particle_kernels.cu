// Particle kernels: fused field gather + relativistic Boris push + move +
// Esirkepov current deposition (+ per-species rho, + optional electron spin
// precession), removal at absorbing faces, and conversion between the
// reference's 144-byte particle records and the device structure of arrays.
//
// One thread per particle.  The gather reads the six staggered field
// components through the read-only path; the deposit adds J (and rho) with
// hardware atomics into the ring buffers, which the fold kernel then
// completes for periodic faces exactly as the reference's ghost exchange.
#include "pic_kernels.cuh"
#include "push_core.cuh"

namespace pic {

template <typename real, int P, bool SPIN>
__global__ void __launch_bounds__(256) push_kernel(PushArgs<real> a) {
    constexpr int H = P / 2;
    const long long n = *a.count;
    View<const real> fv[6];
    GlobalAcc<real> acc;
    global_views(a, fv, acc);
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const long long p = a.idx ? (long long)a.idx[a.idx_pairs ? 2 * t : t] : t;
        if (a.dead && a.dead[p]) continue;
        PartIn<real> in;
        load_position(a, p, in);
        OldPos<real> o;
        decode_old(a, p, in, o);
        if (!in_buffers(a.g, o, H)) {
            set_status(a.status, ST_OOB);
            continue;
        }
        const PmSrc<real> pm{a.px, a.py, a.pz, a.w, p};
        push_body<real, P, SPIN, true>(a, p, o, pm, fv, acc, [&](const int (&cn)[3]) {
            if (a.idx_pairs) vis_note(a.vsink, a.g, (int)p, a.idx[2 * t + 1], cn);
        });
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
    PushArgs<real> a = make_push_args<real>(c, kind);
    long long n = s.n_host;
    if (n > 0) {
        long long blocks = (n + 255) / 256;
        long long maxb = (long long)sm_count(c) * 8;
        push_kernel<real, P, SPIN><<<(unsigned)(blocks < maxb ? blocks : maxb), 256, 0, c->stream>>>(a);
    }
    s.cur = 1 - s.cur;
}

// the particles listed in idx as (index, home tile) pairs (count on the
// device): those the tiled kernel left to the global kernel; each one that
// ends away from its home tile is recorded as a visitor (when vsink is on)
template <typename real, int P, bool SPIN>
static void push_list_t(pic_ctx *c, int kind, const int *idx, const unsigned long long *count, const VisSink &vsink) {
    Species &s = c->sp[kind];
    PushArgs<real> a = make_push_args<real>(c, kind);
    a.idx = idx;
    a.idx_pairs = 1;
    a.vsink = vsink;
    a.count = reinterpret_cast<const long long *>(count);
    long long n = s.n_host;
    if (n > 0) {
        long long blocks = (n + 255) / 256;
        long long maxb = (long long)sm_count(c) * 4;
        push_kernel<real, P, SPIN><<<(unsigned)(blocks < maxb ? blocks : maxb), 256, 0, c->stream>>>(a);
    }
}

void launch_push_list(pic_ctx *c, int kind, const int *idx, const unsigned long long *count, const VisSink &v) {
    bool spin = spin_active(c, kind);
    if (c->fp32) {
        if (c->order == 2) spin ? push_list_t<float, 3, true>(c, kind, idx, count, v) : push_list_t<float, 3, false>(c, kind, idx, count, v);
        else spin ? push_list_t<float, 5, true>(c, kind, idx, count, v) : push_list_t<float, 5, false>(c, kind, idx, count, v);
    } else {
        if (c->order == 2) spin ? push_list_t<double, 3, true>(c, kind, idx, count, v) : push_list_t<double, 3, false>(c, kind, idx, count, v);
        else spin ? push_list_t<double, 5, true>(c, kind, idx, count, v) : push_list_t<double, 5, false>(c, kind, idx, count, v);
    }
}

void launch_push(pic_ctx *c, int kind) {
    bool spin = spin_active(c, kind);
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
    // visitor lists (vsink.raw null: none): a moved particle now belongs to
    // the sorted slice of the tile whose range holds its hole
    VisSink vsink;
    RemoveArgs at;          // the moved particle's position (current buffer)
    const unsigned *offs;   // per-key start offsets of the last sort
    long long keys_per_tile;
};

// the cell the next push's decode will see (as push_body reports it)
__device__ __forceinline__ void current_cell(const RemoveArgs &a, long long i, int (&c)[3]) {
    if (a.fp32) {
        a.cp.unpack(a.cell[i], c[0], c[1], c[2]);
        return;
    }
    const double v0[3] = {a.x[i], a.y[i], a.z[i]};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double v = v0[d];
        if (a.g.per[d]) {
            if (v < 0.0) v += a.g.n[d];
            if (v > (double)a.g.n[d]) v -= a.g.n[d];
        }
        const double xc = v - (double)(1 - a.g.mem);
        c[d] = xc >= 0.0 ? (int)xc - (a.g.mem - 1) : -1;
    }
}

// the tile whose slice of the sorted arrays holds index i
__device__ __forceinline__ int home_tile(const unsigned *offs, long long keys_per_tile, int ntiles, long long i) {
    int lo = 0, hi = ntiles - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if ((long long)offs[(long long)mid * keys_per_tile] <= i) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

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
    if (a.vsink.raw) {
        int c[3];
        current_cell(a.at, src, c);
        const int nt = a.vsink.nt[0] * a.vsink.nt[1] * a.vsink.nt[2];
        vis_note(a.vsink, a.at.g, dst, home_tile(a.offs, a.keys_per_tile, nt, dst), c);
    }
}

// Entries the push recorded for particles that the compaction removes or
// moves are dropped (tile -1); apply_moves records the moved ones anew.
__global__ void vis_drop_kernel(RemoveArgs a, int *raw, const VisState *vs, long long cap) {
    const long long n = *a.count, nn = n - a.ctr[0];
    const long long ne = min((long long)vs->nraw, cap);
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += (long long)gridDim.x * blockDim.x) {
        const long long i = raw[3 * e];
        if (i >= nn || is_dead(a, i)) raw[3 * e + 2] = -1;
    }
}

__global__ void finish_remove_kernel(long long *count, long long *ctr) { *count = *count - ctr[0]; }

__global__ void mark_dead_kernel(RemoveArgs a, unsigned char *dead) {
    long long n = *a.count;
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && !dead[i] && is_dead(a, i)) dead[i] = 1;
}

void launch_remove(pic_ctx *c, int kind) {
    const Geom &g = c->g;
    if (g.per[0] && g.per[1] && g.per[2]) return;
    Species &s = c->sp[kind];
    long long n = s.n_host;
    if (n == 0) return;
    if (s.dead) {
        // adjoint mode: particle indices must stay stable across steps
        RemoveArgs a{};
        a.g = g;
        a.cp = c->cp;
        a.fp32 = c->fp32;
        a.count = s.d_count;
        a.x = s.a.x[s.cur]; a.y = s.a.y[s.cur]; a.z = s.a.z[s.cur];
        a.cell = s.a.cell[s.cur];
        prof_begin(c, "mark_dead");
        mark_dead_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(a, s.dead);
        prof_end(c);
        return;
    }
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
    a.x = s.a.x[cu]; a.y = s.a.y[cu]; a.z = s.a.z[cu];
    a.cell = s.a.cell[cu];
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
            m.f[kf++] = s.a.ox[b]; m.f[kf++] = s.a.oy[b]; m.f[kf++] = s.a.oz[b];
        } else {
            m.d[k++] = s.a.x[b]; m.d[k++] = s.a.y[b]; m.d[k++] = s.a.z[b];
        }
    }
    void *mom[7] = {s.a.px, s.a.py, s.a.pz, s.a.w, s.a.sx, s.a.sy, s.a.sz};
    for (void *v : mom) {
        if (!v) continue;
        if (c->fp32) m.f[kf++] = (float *)v; else m.d[k++] = (double *)v;
    }
    m.i[0] = s.a.id;
    m.i[1] = s.a.cell[0];
    m.i[2] = s.a.cell[1];
    (void)k;
    if (s.vs && s.sorted) {
        m.vsink = vis_sink_of(c, s);
        m.at = a;
        m.offs = s.offs;
        m.keys_per_tile = (long long)c->tile * c->tile * c->tile * kOctants;
        vis_drop_kernel<<<148 * 4, 256, 0, c->stream>>>(a, s.vraw, s.vs, s.vcap);
    }
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
    // upload checks (null: none): check[0] |= 1 charge/mass differ from the
    // species', 2 non-finite weight, 4 non-zero spin, 8 non-finite position
    // or momentum, 16 (FP32) a position whose cell the packed index cannot
    // hold; check[1] = max |weight| as the bits of a non-negative double
    unsigned long long *check;
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
    if (a.check) {
        // warp-reduced record checks (every lane takes part, in range or not)
        unsigned long long f = 0, wb = 0;
        if (t < a.n) {
            const Rec &q = a.rec[t];
            if (q.charge != a.charge || q.mass != a.mass) f |= 1ull;
            if (!isfinite(q.weight)) f |= 2ull;
            else wb = (unsigned long long)__double_as_longlong(fabs(q.weight));
            if (q.sx != 0.0 || q.sy != 0.0 || q.sz != 0.0) f |= 4ull;
            const double v[6] = {q.x, q.y, q.z, q.px, q.py, q.pz};
            bool fin = true;
#pragma unroll
            for (int d = 0; d < 6; ++d) fin = fin && isfinite(v[d]);
            if (!fin) f |= 8ull;
            if (fin && a.fp32) {
                // the packed FP32 cell holds -1 .. n per axis (after the
                // periodic wrap): a position beyond cannot be stored
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const double fl = floor(v[d]);
                    if (!a.g.per[d] && (fl < -1.0 || fl > (double)a.g.n[d])) f |= 16ull;
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            f |= __shfl_xor_sync(0xffffffffu, f, o);
            const unsigned long long v = __shfl_xor_sync(0xffffffffu, wb, o);
            wb = v > wb ? v : wb;
        }
        if ((threadIdx.x & 31) == 0) {
            if (f) atomicOr(a.check, f);
            if (wb) atomicMax(a.check + 1, wb);
        }
    }
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
        a.x[b] = s.a.x[b]; a.y[b] = s.a.y[b]; a.z[b] = s.a.z[b];
        a.cell[b] = s.a.cell[b]; a.ox[b] = s.a.ox[b]; a.oy[b] = s.a.oy[b]; a.oz[b] = s.a.oz[b];
    }
    a.px = s.a.px; a.py = s.a.py; a.pz = s.a.pz; a.w = s.a.w;
    a.sx = s.a.sx; a.sy = s.a.sy; a.sz = s.a.sz;
    a.id = s.a.id;
    a.charge = c->p.charge[kind];
    a.mass = c->p.mass[kind];
    return a;
}

void launch_upload_particles(pic_ctx *c, int kind, const void *d_records, int64_t n, int64_t offset,
                             unsigned long long *check) {
    if (n <= 0) return;
    ConvArgs a = conv_args(c, kind, (void *)d_records, n, offset);
    a.check = check;
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

// ---------------------------------------------------------------------------
// Device-side particle generators: they write reference records [off,
// off + n) into a staging buffer, which records_to_soa_kernel then converts
// (the same path as an upload from host memory).

// initialize_particles (src/particle.cpp:50-111): the lattice points with a
// positive density, in the reference's k, j, i order.  The density of the
// supported profiles is positive on a product of per-axis index sets, so
// the q-th created particle is the q-th point of that product; the host
// passes the coordinates of the kept indices per axis (ax, ay, az) and the
// weight per kept x index (wx) or one weight for all (wconst).
__global__ void lattice_records_kernel(LatticeArgs a) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.n) return;
    const long long q = a.off + t;
    const long long i = q % a.nvx, j = (q / a.nvx) % a.nvy, k = q / (a.nvx * a.nvy);
    Rec r{};
    r.id = (int)q;   // my_rank * num_particles + particle_index with rank 0
    r.x = a.ax[i];
    r.y = a.ay[j];
    r.z = a.az[k];
    r.px = a.p[0];
    r.py = a.p[1];
    r.pz = a.p[2];
    r.sx = a.s[0];
    r.sy = a.s[1];
    r.sz = a.s[2];
    r.gamma = a.gamma;
    r.charge = a.charge;
    r.mass = a.mass;
    r.weight = a.wx ? a.wx[i] : a.wconst;
    ((Rec *)a.rec)[t] = r;
}

// Philox4x32-10 (Salmon, Moraes, Dror and Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC 2011): a counter-based generator, 10 rounds of two
// 32x32->64 multiplies with a Weyl-sequence key schedule.
__device__ __forceinline__ void philox4x32_10(unsigned (&c)[4], unsigned k0, unsigned k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const unsigned lo0 = 0xD2511F53u * c[0], hi0 = __umulhi(0xD2511F53u, c[0]);
        const unsigned lo1 = 0xCD9E8D57u * c[2], hi1 = __umulhi(0xCD9E8D57u, c[2]);
        const unsigned n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

// seeded thermal plasma: ppc particles per cell at uniform random offsets in
// the cell, momenta N(0, u_th^2) per component (Box-Muller), weight
// density / ppc, id = index.  Particle q draws two Philox blocks with
// counters (q, 0) and (q, 1) under key (seed, kind).
__global__ void thermal_records_kernel(ThermalArgs a) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.n) return;
    const long long q = a.off + t;
    const long long cell = q / a.ppc;
    const long long cx = cell % a.nx, cy = (cell / a.nx) % a.ny, cz = cell / ((long long)a.nx * a.ny);
    unsigned u[8];
    for (int h = 0; h < 2; ++h) {
        unsigned c[4] = {(unsigned)q, (unsigned)(q >> 32), (unsigned)h, 0u};
        philox4x32_10(c, a.key0, a.key1);
        for (int e = 0; e < 4; ++e) u[4 * h + e] = c[e];
    }
    const double inv32 = 2.3283064365386963e-10;   // 2^-32
    Rec r{};
    r.id = (int)q;
    r.x = (double)cx + (double)u[0] * inv32;
    r.y = (double)cy + (double)u[1] * inv32;
    r.z = (double)cz + (double)u[2] * inv32;
    // Box-Muller: radius from a uniform in (0, 1], angle from one in [0, 1)
    const double two_pi = 6.283185307179586;
    const double r0 = sqrt(-2.0 * log(((double)u[3] + 1.0) * inv32));
    const double r1 = sqrt(-2.0 * log(((double)u[5] + 1.0) * inv32));
    const double t0 = two_pi * (double)u[4] * inv32, t1 = two_pi * (double)u[6] * inv32;
    r.px = a.u_th * r0 * cos(t0);
    r.py = a.u_th * r0 * sin(t0);
    r.pz = a.u_th * r1 * cos(t1);
    r.gamma = sqrt(1.0 + (r.px * r.px + r.py * r.py + r.pz * r.pz));
    r.charge = a.charge;
    r.mass = a.mass;
    r.weight = a.weight;
    ((Rec *)a.rec)[t] = r;
}

void launch_lattice_records(pic_ctx *c, const LatticeArgs &a) {
    if (a.n > 0) lattice_records_kernel<<<(unsigned)((a.n + 255) / 256), 256, 0, c->stream>>>(a);
}

void launch_thermal_records(pic_ctx *c, const ThermalArgs &a) {
    if (a.n > 0) thermal_records_kernel<<<(unsigned)((a.n + 255) / 256), 256, 0, c->stream>>>(a);
}

// ---------------------------------------------------------------------------
// Deposit of one particle's move from (xo, yo, zo) to (xn, yn, zn), absolute
// cell coordinates, with charge x weight qw: the reference's
// currents_particle (src/particle.cpp:372-515) for a single record, through
// the same deposit code as the push kernels (J always, rho when enabled).
template <typename real, int P>
__global__ void deposit_one_kernel(PushArgs<real> a, double xo, double yo, double zo, double xn, double yn,
                                   double zn, double qw) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    constexpr int H = P / 2;
    const Geom &g = a.g;
    const double po[3] = {xo, yo, zo}, pn[3] = {xn, yn, zn};
    int i1[3], i2[3];
    double d0[3], d1[3];
    for (int d = 0; d < 3; ++d) {
        const double x1 = po[d] - (double)(1 - g.mem), x2 = pn[d] - (double)(1 - g.mem);
        if (!(x1 >= 0.0 && x2 >= 0.0 && x1 < (double)g.f[d] && x2 < (double)g.f[d])) {
            set_status(a.status, ST_OOB);
            return;
        }
        i1[d] = (int)(x1 + 0.5);
        i2[d] = (int)(x2 + 0.5);
        d0[d] = x1 - (double)i1[d];
        d1[d] = x2 - (double)i2[d];
        // the deposit span [min - H, max + H + 1) must lie in the ring (-1 .. f)
        if (abs(i2[d] - i1[d]) > 1 || min(i1[d], i2[d]) - H < -1 || max(i1[d], i2[d]) + H + 1 > g.f[d]) {
            set_status(a.status, abs(i2[d] - i1[d]) > 1 ? ST_CFL : ST_OOB);
            return;
        }
    }
    View<const real> fv[6];
    GlobalAcc<real> acc;
    global_views(a, fv, acc);
    Axis1D<real, P> ax[3];
    bool moved = false;
    for (int d = 0; d < 3; ++d) {
        axis_from_offsets<real, P>(i1[d], d0[d], i2[d], d1[d], ax[d]);
        moved = moved || i1[d] != i2[d] || d0[d] != d1[d];
    }
    deposit<real, P>(acc, a.d_dt, ax, moved, (real)qw);
}

__global__ void iota_kernel(int *a, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = (int)i;
}

void launch_iota(pic_ctx *c, int *a, long long n) {
    iota_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(a, n);
}

void launch_deposit_one(pic_ctx *c, int kind, const double (&xo)[3], const double (&xn)[3], double qw) {
    if (c->fp32) {
        PushArgs<float> a = make_push_args<float>(c, kind);
        if (c->order == 2) deposit_one_kernel<float, 3><<<1, 32, 0, c->stream>>>(a, xo[0], xo[1], xo[2], xn[0], xn[1], xn[2], qw);
        else deposit_one_kernel<float, 5><<<1, 32, 0, c->stream>>>(a, xo[0], xo[1], xo[2], xn[0], xn[1], xn[2], qw);
    } else {
        PushArgs<double> a = make_push_args<double>(c, kind);
        if (c->order == 2) deposit_one_kernel<double, 3><<<1, 32, 0, c->stream>>>(a, xo[0], xo[1], xo[2], xn[0], xn[1], xn[2], qw);
        else deposit_one_kernel<double, 5><<<1, 32, 0, c->stream>>>(a, xo[0], xo[1], xo[2], xn[0], xn[1], xn[2], qw);
    }
}

}  // namespace pic
