// Tiled gather + push + deposit with shared-memory staging.
//
// Particles of each species are kept in counting-sort order by tile (T^3
// cells), then by half-cell octant of the position (which side of the cell
// centre on each axis: it fixes the primal stencil index relative to the
// cell), then by cell.  One CTA owns one tile:
//   1. it stages the six field components of the tile plus the gather halo
//      (T + 2H + 1 points per axis) in shared memory,
//   2. clears shared-memory accumulators for jx, jy, jz, rho0, rho1 over the
//      deposit footprint (T + 2H + 3 points per axis),
//   3. pushes the particles whose sort key falls in the tile, both species,
//      gathering from and depositing into shared memory; a particle that has
//      left the tile since the last sort takes the global-memory path in the
//      same loop (read-only loads, global atomics),
//   4. flushes the accumulators with one coalesced pass of global atomics
//      (zero entries skipped); halos of neighbouring tiles overlap, hence the
//      atomics.
// A warp takes 32 consecutive particles of the sorted list: mostly one
// octant and consecutive cells, so at a common stencil point their
// shared-memory addresses fall in different banks.
//
// The counting sort (key histogram, exclusive scan, scatter into the second
// set of arrays) runs every `sort_interval` pushes and after an upload.
#include <algorithm>
#include <cmath>

#include "pic_kernels.cuh"
#include "push_core.cuh"

namespace pic {

struct TileGeom {
    int T, nt[3];
    long long nkeys;
    int GE, DE, nacc;
    // padded shared-memory strides: row gsy/dsy, plane gsz/dsz, array gsize/dsize
    int gsy, gsz, gsize, dsy, dsz, dsize;
};

// Row and plane strides of a shared-memory box of extent e for tile edge T.
// Lanes of a warp take 32 consecutive cells of the tile (cell index
// x + T*y + T*T*z); with row stride = T (mod 2T) and plane stride = T*T
// (mod 2T*T) those 32 cells start in 32 different banks, so a warp's loads
// and atomics at a common stencil offset are conflict-free (2 wavefronts
// per 8-byte access, the minimum).
static inline void padded_strides(int e, int T, int &sy, int &sz) {
    sy = padded_row(e, T);
    sz = padded_plane(e, T);
}

template <int P>
__host__ __device__ constexpr int gather_extent(int T) { return T + 2 * (P / 2) + 1; }
template <int P>
__host__ __device__ constexpr int deposit_extent(int T) { return T + 2 * (P / 2) + 3; }

// Sort key of a particle in cell (cx, cy, cz) whose position in the cell
// lies in half-cell octant `oct` (bit d set: offset >= 1/2 along axis d, so
// its primal stencil index is the cell's plus one along d): tile, then
// octant, then cell within the tile.
__device__ __forceinline__ int cell_key(const TileGeom &t, int cx, int cy, int cz, int oct) {
    const int T = t.T;
    int tx = cx / T, ty = cy / T, tz = cz / T;
    int lx = cx - tx * T, ly = cy - ty * T, lz = cz - tz * T;
    return ((((tz * t.nt[1] + ty) * t.nt[0] + tx) * kOctants + oct) * T + lz) * T * T + ly * T + lx;
}

// cell of a particle for sorting (FP64: periodic wrap as the next push
// will apply it; clamped into the domain)
__device__ __forceinline__ int particle_key(const Geom &g, const TileGeom &t, const CellPack &cp, int fp32,
                                            const double *x, const double *y, const double *z, const int *cell,
                                            const float *ox, const float *oy, const float *oz, long long i) {
    int c[3], oct = 0;
    if (fp32) {
        cp.unpack(cell[i], c[0], c[1], c[2]);
        oct = (ox[i] >= 0.5f ? 1 : 0) | (oy[i] >= 0.5f ? 2 : 0) | (oz[i] >= 0.5f ? 4 : 0);
    } else {
        double v[3] = {x[i], y[i], z[i]};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (g.per[d]) {
                if (v[d] < 0.0) v[d] += g.n[d];
                if (v[d] > (double)g.n[d]) v[d] -= g.n[d];
            }
            const double f = floor(v[d]);
            c[d] = (int)f;
            oct |= (v[d] - f >= 0.5 ? 1 : 0) << d;
        }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) c[d] = min(max(c[d], 0), g.n[d] - 1);
    return cell_key(t, c[0], c[1], c[2], oct);
}

// ---------------------------------------------------------------------------
// counting sort

struct SortArgs {
    Geom g;
    TileGeom t;
    CellPack cp;
    int fp32;
    const long long *count;
    const double *x, *y, *z;
    const int *cell;
    const float *ox, *oy, *oz;
    int *keys;
    unsigned *hist;
};

__global__ void sort_keys_kernel(SortArgs a) {
    long long n = *a.count;
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned act = __ballot_sync(0xffffffffu, i < n);
    if (i >= n) return;
    int key = particle_key(a.g, a.t, a.cp, a.fp32, a.x, a.y, a.z, a.cell, a.ox, a.oy, a.oz, i);
    a.keys[i] = key;
    unsigned peers = __match_any_sync(act, key);
    int lane = threadIdx.x & 31;
    if (lane == __ffs(peers) - 1) atomicAdd(&a.hist[key], (unsigned)__popc(peers));
}

// exclusive scan of n unsigned values in place; block sums in `sums`
__global__ void scan_blocks_kernel(unsigned *v, long long n, unsigned *sums) {
    __shared__ unsigned warp_tot[32];
    const int per = 4;
    long long base = (long long)blockIdx.x * blockDim.x * per + (long long)threadIdx.x * per;
    unsigned loc[per];
    unsigned s = 0;
#pragma unroll
    for (int k = 0; k < per; ++k) {
        loc[k] = base + k < n ? v[base + k] : 0u;
        s += loc[k];
    }
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned incl = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_tot[w] = incl;
    __syncthreads();
    if (w == 0) {
        int nw = blockDim.x >> 5;
        unsigned t = lane < nw ? warp_tot[lane] : 0u;
        unsigned ti = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            unsigned u = __shfl_up_sync(0xffffffffu, ti, o);
            if (lane >= o) ti += u;
        }
        if (lane < nw) warp_tot[lane] = ti - t;
        if (lane == nw - 1) sums[blockIdx.x] = ti;
    }
    __syncthreads();
    unsigned run = warp_tot[w] + incl - s;
#pragma unroll
    for (int k = 0; k < per; ++k) {
        if (base + k < n) v[base + k] = run;
        run += loc[k];
    }
}

// exclusive scan of the block sums (single block, any count), total in sums[nb]
__global__ void scan_sums_kernel(unsigned *sums, int nb) {
    __shared__ unsigned carry;
    __shared__ unsigned warp_tot[32];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int off = 0; off < nb; off += blockDim.x) {
        int i = off + threadIdx.x;
        unsigned s = i < nb ? sums[i] : 0u;
        int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        unsigned incl = s;
        for (int o = 1; o < 32; o <<= 1) {
            unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) warp_tot[w] = incl;
        __syncthreads();
        if (w == 0) {
            int nw = blockDim.x >> 5;
            unsigned t = lane < nw ? warp_tot[lane] : 0u;
            unsigned ti = t;
            for (int o = 1; o < 32; o <<= 1) {
                unsigned u = __shfl_up_sync(0xffffffffu, ti, o);
                if (lane >= o) ti += u;
            }
            if (lane < nw) warp_tot[lane] = ti - t;
        }
        __syncthreads();
        unsigned excl = carry + warp_tot[w] + incl - s;
        if (i < nb) sums[i] = excl;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = excl + s;
        __syncthreads();
    }
    if (threadIdx.x == 0) sums[nb] = carry;
}

__global__ void scan_add_kernel(unsigned *v, long long n, const unsigned *sums, int per_block, unsigned *offs_out,
                                unsigned *cursor_out) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        unsigned o = v[i] + sums[i / per_block];
        offs_out[i] = o;
        cursor_out[i] = o;
    }
    if (i == n) {
        int nb = (int)((n + per_block - 1) / per_block);
        offs_out[n] = sums[nb];
    }
}

struct ScatterArgs {
    const long long *count;
    long long cap;
    unsigned *status;
    const int *keys;
    unsigned *cursor;
    // up to 16 8-byte and 16 4-byte arrays moved src -> dst
    const double *ds[16];
    double *dd[16];
    int nd;
    const float *fs[16];
    float *fd[16];
    int nf;
    const int *is[4];
    int *id_[4];
    int ni;
    const unsigned char *bs;   // one byte array (adjoint mode: dead flags), or null
    unsigned char *bd;
    int *perm;                 // adjoint mode: perm[dst] = src, the gather form of this sort
};

__global__ void scatter_kernel(ScatterArgs a) {
    long long n = *a.count;
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned act = __ballot_sync(0xffffffffu, i < n);
    if (i >= n) return;
    int key = a.keys[i];
    unsigned peers = __match_any_sync(act, key);
    int lane = threadIdx.x & 31;
    int leader = __ffs(peers) - 1;
    unsigned base = 0;
    if (lane == leader) base = atomicAdd(&a.cursor[key], (unsigned)__popc(peers));
    base = __shfl_sync(peers, base, leader);
    unsigned dst = base + __popc(peers & ((1u << lane) - 1u));
    if ((long long)dst >= a.cap) {  // cannot happen with a consistent histogram; never write past the arrays
        atomicOr(a.status, ST_OVERFLOW);
        return;
    }
    for (int k = 0; k < a.nd; ++k) a.dd[k][dst] = a.ds[k][i];
    for (int k = 0; k < a.nf; ++k) a.fd[k][dst] = a.fs[k][i];
    for (int k = 0; k < a.ni; ++k) a.id_[k][dst] = a.is[k][i];
    if (a.bs) a.bd[dst] = a.bs[i];
    if (a.perm) a.perm[dst] = (int)i;
}

// ---------------------------------------------------------------------------
// visitor lists: a counting sort by tile of the (index, home, tile) entries
// the last push recorded

__global__ void vis_reset_kernel(VisState *vs) {
    vs->nraw = 0;
    vs->nvis = 0;
    vs->valid_cur = 1u;
    vs->valid_next = 1u;
}

// entries with tile -1 were dropped by the removal compaction
__global__ void vis_hist_kernel(const int *raw, const VisState *vs, long long cap, unsigned *cnt) {
    const long long n = min((long long)vs->nraw, cap);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        if (raw[3 * i + 2] >= 0) atomicAdd(&cnt[raw[3 * i + 2]], 1u);
}

__global__ void vis_scatter_kernel(const int *raw, const VisState *vs, long long cap, unsigned *cursor, int *vis) {
    const long long n = min((long long)vs->nraw, cap);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        if (raw[3 * i + 2] < 0) continue;
        const unsigned slot = atomicAdd(&cursor[raw[3 * i + 2]], 1u);
        vis[2 * slot] = raw[3 * i];
        vis[2 * slot + 1] = raw[3 * i + 1];
    }
}

// FP64: below this fraction of a species away from home, the particles away
// from home are pushed by the global-memory kernel instead.  On the
// 256x128x128 thermal plasma (1.4 % away two pushes after a sort) the
// visitor lists measured even at 2nd order and 4 % slower at 4th (a tile's
// few visitors add a partial round of batches, and the FP64 kernel has the
// longer rounds); on the laser run (6 % away, relativistic electrons) they
// win.  FP32 uses them at any fraction (1.6 % faster at 2nd order, 2.6 % at
// 4th on the thermal plasma).
inline double visitor_min_fraction(const pic_ctx *c) { return c->fp32 ? 0.0 : 0.03; }

__host__ __device__ inline bool visitor_lists_pay(unsigned long long entries, long long particles, double min_frac) {
    return (double)entries >= min_frac * (double)particles;
}

// the lists just built are the ones the coming push reads; it records into
// an empty raw list
__global__ void vis_rotate_kernel(VisState *vs, long long cap, const long long *count, double min_frac) {
    vs->nvis = min((long long)vs->nraw, cap);
    vs->valid_cur = vs->valid_next && visitor_lists_pay(vs->nvis, *count, min_frac);
    vs->nraw = 0;
    vs->valid_next = 1u;
}

static void launch_vis_build(pic_ctx *c, Species &s) {
    const long long nt = (long long)c->ntile[0] * c->ntile[1] * c->ntile[2];
    const int per_block = 1024 * 4;
    const int sb = (int)((nt + per_block - 1) / per_block);
    const unsigned grid = 148 * 4;
    cudaMemsetAsync(s.vis_cnt, 0, (size_t)(nt + 1) * sizeof(unsigned), c->stream);
    vis_hist_kernel<<<grid, 256, 0, c->stream>>>(s.vraw, s.vs, s.vcap, s.vis_cnt);
    scan_blocks_kernel<<<sb, 1024, 0, c->stream>>>(s.vis_cnt, nt, c->d_blocksums);
    scan_sums_kernel<<<1, 1024, 0, c->stream>>>(c->d_blocksums, sb);
    scan_add_kernel<<<(unsigned)((nt + 1 + 255) / 256), 256, 0, c->stream>>>(s.vis_cnt, nt, c->d_blocksums, per_block,
                                                                             s.vis_off, s.vis_cnt);
    vis_scatter_kernel<<<grid, 256, 0, c->stream>>>(s.vraw, s.vs, s.vcap, s.vis_cnt, s.vis);
    vis_rotate_kernel<<<1, 1, 0, c->stream>>>(s.vs, s.vcap, s.d_count, visitor_min_fraction(c));
}

static TileGeom tile_geom(const pic_ctx *c) {
    TileGeom t{};
    t.T = c->tile;
    for (int d = 0; d < 3; ++d) t.nt[d] = c->ntile[d];
    t.nkeys = c->nkeys;
    return t;
}

void launch_sort(pic_ctx *c, int kind) {
    Species &s = c->sp[kind];
    const long long n = s.n_host;
    if (n <= 0 || c->tile <= 0) return;
    prof_begin(c, "sort_particles");
    const long long K = c->nkeys;
    cudaMemsetAsync(c->d_hist, 0, (size_t)(K + 1) * sizeof(unsigned), c->stream);
    SortArgs a{};
    a.g = c->g;
    a.t = tile_geom(c);
    a.cp = c->cp;
    a.fp32 = c->fp32;
    a.count = s.d_count;
    a.x = s.a.x[s.cur]; a.y = s.a.y[s.cur]; a.z = s.a.z[s.cur];
    a.cell = s.a.cell[s.cur];
    a.ox = s.a.ox[s.cur]; a.oy = s.a.oy[s.cur]; a.oz = s.a.oz[s.cur];
    a.keys = s.keys;
    a.hist = c->d_hist;
    unsigned nb = (unsigned)((n + 255) / 256);
    sort_keys_kernel<<<nb, 256, 0, c->stream>>>(a);
    const int per_block = 1024 * 4;
    int sb = (int)((K + per_block - 1) / per_block);
    scan_blocks_kernel<<<sb, 1024, 0, c->stream>>>(c->d_hist, K, c->d_blocksums);
    scan_sums_kernel<<<1, 1024, 0, c->stream>>>(c->d_blocksums, sb);
    // offsets into s.offs; the cursor reuses d_hist
    scan_add_kernel<<<(unsigned)((K + 1 + 255) / 256), 256, 0, c->stream>>>(c->d_hist, K, c->d_blocksums,
                                                                            per_block, s.offs, c->d_hist);
    ScatterArgs sa{};
    sa.count = s.d_count;
    sa.cap = s.cap;
    sa.status = c->d_status;
    sa.keys = s.keys;
    sa.cursor = c->d_hist;
    // The sort runs right before a push, which overwrites the previous-position
    // buffer: only the current one moves (the adjoint's tape keeps both).
    for (int b = 0; b < 2; ++b) {
        if (b != s.cur && !c->p.adjoint) continue;
        if (c->fp32) {
            sa.fs[sa.nf] = s.a.ox[b]; sa.fd[sa.nf++] = s.b.ox[b];
            sa.fs[sa.nf] = s.a.oy[b]; sa.fd[sa.nf++] = s.b.oy[b];
            sa.fs[sa.nf] = s.a.oz[b]; sa.fd[sa.nf++] = s.b.oz[b];
            sa.is[sa.ni] = s.a.cell[b]; sa.id_[sa.ni++] = s.b.cell[b];
        } else {
            sa.ds[sa.nd] = s.a.x[b]; sa.dd[sa.nd++] = s.b.x[b];
            sa.ds[sa.nd] = s.a.y[b]; sa.dd[sa.nd++] = s.b.y[b];
            sa.ds[sa.nd] = s.a.z[b]; sa.dd[sa.nd++] = s.b.z[b];
        }
    }
    void *src[7] = {s.a.px, s.a.py, s.a.pz, s.a.w, s.a.sx, s.a.sy, s.a.sz};
    void *dst[7] = {s.b.px, s.b.py, s.b.pz, s.b.w, s.b.sx, s.b.sy, s.b.sz};
    for (int k = 0; k < 7; ++k) {
        if (!src[k]) continue;
        if (c->fp32) { sa.fs[sa.nf] = (float *)src[k]; sa.fd[sa.nf++] = (float *)dst[k]; }
        else { sa.ds[sa.nd] = (double *)src[k]; sa.dd[sa.nd++] = (double *)dst[k]; }
    }
    sa.is[sa.ni] = s.a.id; sa.id_[sa.ni++] = s.b.id;
    if (s.orig) {   // adjoint mode: upload index, dead flags, and the permutation for the tape
        sa.is[sa.ni] = s.orig; sa.id_[sa.ni++] = s.orig_b;
        sa.bs = s.dead;
        sa.bd = s.dead_b;
        sa.perm = s.perm;
    }
    scatter_kernel<<<nb, 256, 0, c->stream>>>(sa);
    std::swap(s.a, s.b);
    if (s.orig) {
        std::swap(s.orig, s.orig_b);
        std::swap(s.dead, s.dead_b);
        s.perm_fresh = true;
    }
    s.sorted = true;
    s.pushes_since_sort = 0;
    if (s.vs) {   // every particle is at home: empty visitor lists
        cudaMemsetAsync(s.vis_off, 0, (size_t)(c->ntile[0] * c->ntile[1] * c->ntile[2] + 1) * sizeof(unsigned),
                        c->stream);
        vis_reset_kernel<<<1, 1, 0, c->stream>>>(s.vs);
    }
    s.vis_built_for = 0;
    prof_end(c);
}

void launch_sort_due(pic_ctx *c, int mask) {
    if (c->tile <= 0) return;
    for (int k = 0; k < 2; ++k) {
        Species &s = c->sp[k];
        if (!((mask >> k) & 1) || s.n_host <= 0) continue;
        if (!s.sorted || s.pushes_since_sort >= c->sort_interval) launch_sort(c, k);
    }
}

// Before a push: a full sort when due, else this push's visitor lists from
// what the last push recorded (once per push: pushes_since_sort counts them).
static void prepare_push(pic_ctx *c, int mask) {
    if (c->tile <= 0) return;
    for (int k = 0; k < 2; ++k) {
        Species &s = c->sp[k];
        if (!((mask >> k) & 1) || s.n_host <= 0) continue;
        if (!s.sorted || s.pushes_since_sort >= c->sort_interval) {
            launch_sort(c, k);
        } else if (s.vs && s.vis_built_for != s.pushes_since_sort) {
            prof_begin(c, "visitor_lists");
            launch_vis_build(c, s);
            prof_end(c);
        }
        s.vis_built_for = s.pushes_since_sort;
    }
}

// ---------------------------------------------------------------------------
// the tile kernel

// limbs of the shared-memory fixed-point accumulators
template <typename real>
constexpr int limbs() { return sizeof(real) == 8 ? 3 : 2; }
// |value * scale| stays below 2^fixed_bits: with at most kMaxTileParticles
// additions per point the limb sums fit in 32 bits and the reassembled
// total in 64 bits (FixedAcc)
constexpr int kMaxTileParticles = 16383;

// Asynchronous global -> shared copies (cp.async): a CTA issues every copy
// of a batch without waiting on any, then waits once.  src_bytes 0 fills the
// destination with zeros and reads nothing.
template <int BYTES>
__device__ __forceinline__ void cp_async(void *dst, const void *src, int src_bytes = BYTES) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(d), "l"(src), "n"(BYTES), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// word offset (from the accumulators) of the particle input buffers: after
// the five accumulators, rounded up to 16 bytes
__host__ __device__ constexpr int particle_buffer_offset(int acc_words) { return (acc_words + 3) & ~3; }

template <typename real>
struct TileArgs {
    PushArgs<real> sp[2];
    const unsigned *offs[2];
    int active[2];
    TileGeom t;
    real *ring[5];
    const real *field[6];
    real scale[4];          // jx, jy, jz, rho
    double inv_scale[4];
    int *strag[2];          // (index, home tile) of particles left for the global kernel
    unsigned long long *nstrag;
    // visitor lists of this push (vis_off null: none) and the recording of
    // the next push's (vsink.raw null: off)
    const int *vis[2];
    const unsigned *vis_off[2];
    const VisState *vs[2];
    VisSink vsink[2];
};

// Threads per CTA of an ordinary step (the kernel's launch bounds ask for
// two CTAs per SM at 256 threads, one at 512: 128 registers either way).
// Two CTAs of 256 threads (128 registers) where the shared memory of two
// fits: FP32 (measured 1.46x faster at 4th order than one CTA with more
// registers) and FP64 at 2nd order (107 KB per CTA on a step without rho;
// 15.6 vs 19.4 ms per launch on the 256x128x128 thermal plasma against one
// CTA of 512), while one CTA of the other overlaps its staging and flush.
// FP64 at 4th order (160 KB) allows one CTA per SM: 512 threads at 128
// registers (a few spills) measured 12 % faster on the laser workload than
// 256 at 237 registers, while 384 lost (a tile's 512 particles per species
// then leave a third of the second round idle).  Three FP32 CTAs per SM at
// 2nd order measured slower than two.
template <typename real, int P>
constexpr int tile_threads() { return sizeof(real) == 4 || P == 3 ? 256 : 512; }

// TT: the tile edge as a compile-time constant (0: from the arguments).
// With the edge known, every stride of the shared boxes is a constant and
// the stencil addresses fold into instruction offsets.
// NT: threads per CTA of this instantiation (512: one CTA per SM)
template <typename real, int P, bool SPIN, int TT, int NT>
__global__ void __launch_bounds__(NT, (NT >= 512 ? 1 : 2)) tile_push_kernel(TileArgs<real> ta) {
    constexpr int H = P / 2;
    constexpr int NL = limbs<real>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    real *sf = reinterpret_cast<real *>(smem_raw);
    const Geom &g = ta.sp[0].g;
    const int T = TT > 0 ? TT : ta.t.T;
    const int GE = gather_extent<P>(T), DE = deposit_extent<P>(T);
    int gsy, gsz, GS, dsy, dsz, DS;
    if constexpr (TT > 0) {
        constexpr int ge = gather_extent<P>(TT), de = deposit_extent<P>(TT);
        constexpr int gy = padded_row(ge, TT), gz = padded_plane(ge, TT);
        constexpr int dy = padded_row(de, TT), dz = padded_plane(de, TT);
        gsy = gy; gsz = gz; GS = ge * gz;
        dsy = dy; dsz = dz; DS = de * dz;
    } else {
        gsy = ta.t.gsy; gsz = ta.t.gsz; GS = ta.t.gsize;
        dsy = ta.t.dsy; dsz = ta.t.dsz; DS = ta.t.dsize;
    }
    const int G2 = GE * GE, G3 = G2 * GE, D2 = DE * DE, D3 = D2 * DE;
    unsigned *sa = reinterpret_cast<unsigned *>(sf + 6 * GS);   // [component][limb][DS]
    // per warp, two slots of one batch of particle inputs, [word][lane],
    // and the (index, home tile) of each lane's particle per slot
    using PWord = typename PartIn<real>::word;
    constexpr int KW = PartIn<real>::kWords;
    PWord *sp_in = reinterpret_cast<PWord *>(sa + particle_buffer_offset(ta.t.nacc * NL * DS)) + (threadIdx.x >> 5) * 2 * KW * 32;
    int2 *sp_loc = reinterpret_cast<int2 *>(reinterpret_cast<PWord *>(sa + particle_buffer_offset(ta.t.nacc * NL * DS)) +
                                            (blockDim.x >> 5) * 2 * KW * 32) + (threadIdx.x >> 5) * 2 * 32;
    const int nacc = ta.t.nacc;
    const int tile = blockIdx.x;
    const int tx = tile % ta.t.nt[0], ty = (tile / ta.t.nt[0]) % ta.t.nt[1], tz = tile / (ta.t.nt[0] * ta.t.nt[1]);
    const int t0[3] = {tx * T, ty * T, tz * T};
    int gO[3], dO[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        gO[d] = t0[d] + g.mem - 1 - H;   // field buffer coordinate of the first staged point
        dO[d] = t0[d] + g.mem - 2 - H;   // buffer coordinate of the first accumulator point
    }
    // particle ranges of this tile: its slice of the sorted arrays (home
    // particles) and its visitor list
    const long long T3 = (long long)T * T * T * kOctants;   // keys per tile
    long long pa[2] = {0, 0}, pb[2] = {0, 0}, va[2] = {0, 0}, vb[2] = {0, 0};
    bool vvalid[2] = {false, false};
    long long mtot = 0;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        if (!ta.active[k]) continue;
        const long long n = *ta.sp[k].count;
        pa[k] = ta.offs[k][tile * T3];
        pb[k] = ta.offs[k][(tile + 1) * T3];
        pb[k] = pb[k] < n ? pb[k] : n;
        if (pa[k] > pb[k]) pa[k] = pb[k];
        vvalid[k] = ta.vs[k] && ta.vs[k]->valid_cur;
        if (vvalid[k] && ta.vis_off[k]) {
            va[k] = ta.vis_off[k][tile];
            vb[k] = ta.vis_off[k][tile + 1];
        }
        mtot += pb[k] - pa[k] + vb[k] - va[k];
    }
    if (mtot == 0) return;
    const bool use_smem = mtot <= kMaxTileParticles;
    // 1. stage fields (asynchronous copies; points outside the buffers read
    // as zero), 2. clear accumulators
    if (use_smem) {
        for (int e = threadIdx.x; e < 6 * G3; e += blockDim.x) {
            int c = e / G3, l = e - c * G3;
            int lz = l / G2, r = l - lz * G2, ly = r / GE, lx = r - ly * GE;
            int x = gO[0] + lx, y = gO[1] + ly, z = gO[2] + lz;
            const bool in = x >= 0 && x < g.f[0] && y >= 0 && y < g.f[1] && z >= 0 && z < g.f[2];
            cp_async<sizeof(real)>(sf + c * GS + lz * gsz + ly * gsy + lx,
                                   ta.field[c] + (in ? g.fi(z, y, x) : 0), in ? (int)sizeof(real) : 0);
        }
        cp_async_commit();
        for (int e = threadIdx.x; e < nacc * NL * DS; e += blockDim.x) sa[e] = 0u;
    }
    cp_async_wait_all();
    __syncthreads();

    View<const real> fs[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) fs[c] = View<const real>{sf + c * GS, gsy, gsz, -(gO[2] * gsz + gO[1] * gsy + gO[0])};
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    // a warp takes 32 consecutive particles of the tile's list: mostly one
    // octant, so the lanes' primal stencils sit at the same offset from
    // their cells and their shared-memory accesses at a common stencil point
    // fall in different banks (the padded strides)
    const int lo_id[3] = {t0[0] + g.mem - 1, t0[1] + g.mem - 1, t0[2] + g.mem - 1};

    // 3. particles of both species
#pragma unroll 1
    for (int k = 0; k < 2; ++k) {
        const long long mh = pb[k] - pa[k];         // home particles, then visitors
        const long long m = mh + vb[k] - va[k];
        if (m <= 0) continue;
        const PushArgs<real> &a = ta.sp[k];
        FixedAcc<real, NL> af;
#pragma unroll
        for (int c = 0; c < 3; ++c) af.p[c] = sa + c * NL * DS;
        af.p[3] = (a.rho && nacc == 5) ? sa + (3 + k) * NL * DS : nullptr;
        af.lstride = DS;
        af.sy = dsy;
        af.sz = dsz;
        af.o = -(dO[2] * dsz + dO[1] * dsy + dO[0]);
#pragma unroll
        for (int c = 0; c < 4; ++c) af.scale[c] = ta.scale[c];
        // The particle of list position i: a home particle, or an entry of
        // the visitor list.  Its inputs are copied asynchronously into slot
        // `slot` of this warp's buffer one batch ahead of its push.
        const long long pak = pa[k];
        const int2 *visk = reinterpret_cast<const int2 *>(ta.vis[k]) + va[k];
        auto prefetch = [&](long long i, int slot) {
            if (i >= m) return;
            int2 e = make_int2((int)(pak + i), tile);
            if (i >= mh) e = visk[i - mh];
            sp_loc[slot * 32 + lane] = e;
            PWord *dst = sp_in + slot * KW * 32 + lane;
#pragma unroll
            for (int w = 0; w < KW; ++w) cp_async<sizeof(PWord)>(dst + w * 32, particle_word_src(a, (long long)e.x, w));
        };
        long long idx = (long long)warp * 32 + lane;
        int slot = 0;
        prefetch(idx, 0);
        cp_async_commit();
#pragma unroll 1
        for (long long base = (long long)warp * 32; base < m; base += (long long)nwarp * 32) {
            cp_async_wait_all();
            const int2 loc = sp_loc[slot * 32 + lane];
            const long long p = loc.x;
            const int home = loc.y;
            const bool dead = idx < m && a.dead && a.dead[p];   // adjoint mode: removed particles stay, dead
            // the next batch into the other slot
            prefetch(idx + (long long)nwarp * 32, slot ^ 1);
            cp_async_commit();
            const PWord *row = sp_in + slot * KW * 32 + lane;
            if (idx < m && !dead) {
                PartIn<real> in;
#pragma unroll
                for (int w = 0; w < PartIn<real>::kPos; ++w) in.v[w] = row[w * 32];
                OldPos<real> o;
                decode_old(a, p, in, o);
                bool inside = true;
#pragma unroll
                for (int d = 0; d < 3; ++d) inside = inside && o.id[d] >= lo_id[d] && o.id[d] < lo_id[d] + T;
                if (!in_buffers(g, o, H)) {
                    set_status(a.status, ST_OOB);
                } else if (inside && use_smem) {
                    constexpr int mo = PartIn<real>::kPos;   // momenta, then weight
                    const real *pr = reinterpret_cast<const real *>(sp_in + slot * KW * 32);
                    const PmSrc<real> pm{pr + mo * 32, pr + (mo + 1) * 32, pr + (mo + 2) * 32, pr + (mo + 3) * 32, lane};
                    push_body<real, P, SPIN, false>(a, p, o, pm, fs, af, [&](const int (&cn)[3]) {
                        vis_note(ta.vsink[k], g, (int)p, home, cn, tile, t0);
                    });
                } else if (!inside && idx < mh && vvalid[k]) {
                    // away from home: pushed from the visitor list of the tile it is in
                } else {
                    // a crowded tile, or away from home without valid visitor
                    // lists: pushed by the global kernel after this one
                    const unsigned long long q = atomicAdd(ta.nstrag + k, 1ull);
                    ta.strag[k][2 * q] = (int)p;
                    ta.strag[k][2 * q + 1] = home;
                }
            }
            idx += (long long)nwarp * 32;
            slot ^= 1;
        }
        cp_async_wait_all();
    }
    if (!use_smem) return;
    __syncthreads();
    // 4. reassemble the limbs and flush with one pass of global atomics
    for (int e = threadIdx.x; e < nacc * D3; e += blockDim.x) {
        int c = e / D3, l = e - c * D3;
        int lz = l / D2, r = l - lz * D2, ly = r / DE, lx = r - ly * DE;
        const unsigned *q = sa + c * NL * DS + lz * dsz + ly * dsy + lx;
        long long tot;
        if constexpr (NL == 2) tot = ((long long)(int)q[DS] << kLimbBits) + (long long)q[0];
        else
            tot = ((long long)(int)q[2 * DS] << (2 * kLimbBits)) + ((long long)q[DS] << kLimbBits) + (long long)q[0];
        if (tot == 0) continue;
        int x = dO[0] + lx, y = dO[1] + ly, z = dO[2] + lz;
        // FP32: single-precision arithmetic (the sum rounded to 24 bits)
        const real v = (real)tot * (real)ta.inv_scale[c < 3 ? c : 3];
        if (x >= -1 && x <= g.f[0] && y >= -1 && y <= g.f[1] && z >= -1 && z <= g.f[2])
            atomic_add(ta.ring[c] + g.ri(z, y, x), v);
        else
            set_status(ta.sp[0].status, ST_OOB);
    }
}

static TileGeom tile_layout(const pic_ctx *c) {
    TileGeom t = tile_geom(c);
    const int P = c->order == 2 ? 3 : 5;
    t.GE = t.T + 2 * (P / 2) + 1;
    t.DE = t.T + 2 * (P / 2) + 3;
    padded_strides(t.GE, t.T, t.gsy, t.gsz);
    padded_strides(t.DE, t.T, t.dsy, t.dsz);
    t.gsize = t.GE * t.gsz;
    t.dsize = t.DE * t.dsz;
    t.nacc = (c->p.deposit_rho && !c->rho_skip) ? 5 : 3;
    return t;
}

TileBoxes tile_boxes(const pic_ctx *c) {
    const TileGeom t = tile_layout(c);
    return TileBoxes{t.GE, t.DE, t.gsy, t.gsz, t.gsize, t.dsy, t.dsz, t.dsize};
}

// Threads per CTA of a launch.  FP64 at 2nd order on a step whose rho is
// observed: its five accumulators (131 KB per CTA) leave room for one CTA
// per SM, so that CTA takes 512 threads instead of 256.
static int tile_launch_threads(const pic_ctx *c) {
    const bool o2 = c->order == 2;
    if (!c->fp32 && o2 && tile_layout(c).nacc == 5) return 512;
    return c->fp32 ? (o2 ? tile_threads<float, 3>() : tile_threads<float, 5>())
                   : (o2 ? tile_threads<double, 3>() : tile_threads<double, 5>());
}

size_t tile_smem_bytes(const pic_ctx *c) {
    const TileGeom t = tile_layout(c);
    const size_t rs = c->fp32 ? 4 : 8, nl = c->fp32 ? 2 : 3;
    const size_t warps = (size_t)tile_launch_threads(c) / 32;
    const size_t words = c->fp32 ? PartIn<float>::kWords : PartIn<double>::kWords;
    // the accumulators of this launch: jx, jy, jz, and rho0, rho1 on a step whose rho is observed
    return 6 * (size_t)t.gsize * rs + 4 * (size_t)particle_buffer_offset((int)(t.nacc * nl * t.dsize)) +
           warps * 2 * 32 * (words * rs + sizeof(int2));
}

VisSink vis_sink_of(const pic_ctx *c, const Species &s) {
    VisSink v{};
    if (!s.vs) return v;
    v.raw = s.vraw;
    v.vs = s.vs;
    v.cap = s.vcap;
    v.T = c->tile;
    for (int d = 0; d < 3; ++d) v.nt[d] = c->ntile[d];
    return v;
}

template <typename real, int P, bool SPIN>
static void tile_push_t(pic_ctx *c, int mask) {
    TileArgs<real> ta{};
    double qw_max = 0.0;
    for (int k = 0; k < 2; ++k) {
        ta.sp[k] = make_push_args<real>(c, k);
        ta.offs[k] = c->sp[k].offs;
        ta.active[k] = ((mask >> k) & 1) && c->sp[k].n_host > 0;
        if (ta.active[k]) qw_max = std::max(qw_max, std::fabs(c->p.charge[k]) * c->sp[k].max_abs_w);
    }
    ta.t = tile_layout(c);
    for (int k = 0; k < 5; ++k) ta.ring[k] = (real *)c->ring[k];
    for (int k = 0; k < 6; ++k) ta.field[k] = (const real *)c->field[k];
    // one contribution is at most |q w| d/dt (J: the running sum of ds and the
    // Esirkepov weight are both within [-1, 1]) or |q w| smax^3 (rho, smax the
    // largest shape weight: 3/4 at 2nd order, 115/192 at 4th)
    const double dmax = std::max(c->p.dx, std::max(c->p.dy, c->p.dz));
    const double lim = std::ldexp(1.0, fixed_bits<real>());
    const double smax = P == 3 ? 0.75 : 115.0 / 192.0;
    const double bj = 1.01 * qw_max * dmax / c->p.dt, br = 1.01 * qw_max * smax * smax * smax;
    for (int k = 0; k < 4; ++k) {
        double b = k < 3 ? bj : br;
        double s = b > 0.0 ? lim / b : 1.0;
        ta.scale[k] = (real)s;
        ta.inv_scale[k] = 1.0 / (double)ta.scale[k];
    }
    for (int k = 0; k < 2; ++k) {
        Species &s = c->sp[k];
        ta.strag[k] = s.strag;
        ta.vis[k] = s.vis;
        ta.vis_off[k] = s.vis_off;
        ta.vs[k] = s.vs;
        ta.vsink[k] = vis_sink_of(c, s);
    }
    ta.nstrag = c->d_nstrag;
    cudaMemsetAsync(c->d_nstrag, 0, 2 * sizeof(unsigned long long), c->stream);
    size_t smem = tile_smem_bytes(c);
    const int ntiles = c->ntile[0] * c->ntile[1] * c->ntile[2];
    constexpr int NT = tile_threads<real, P>();
    auto launch = [&](auto kernel, int threads) {
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kernel<<<ntiles, threads, smem, c->stream>>>(ta);
    };
    const bool wide = tile_launch_threads(c) != NT;
    if constexpr (sizeof(real) == 8 && NT != 512) {
        if (wide) {
            if (c->tile == 4) launch(tile_push_kernel<real, P, SPIN, 4, 512>, 512);
            else launch(tile_push_kernel<real, P, SPIN, 0, 512>, 512);
            return;
        }
    }
    if (c->tile == 4) launch(tile_push_kernel<real, P, SPIN, 4, NT>, NT);   // the default edge: strides as constants
    else launch(tile_push_kernel<real, P, SPIN, 0, NT>, NT);
}

// the counts pic_particle_order_stats reports (host side, synchronising)
int tile_order_stats(pic_ctx *c, int kind, long long (&out)[4]) {
    Species &s = c->sp[kind];
    out[0] = out[1] = out[3] = 0;
    out[2] = s.pushes_since_sort;
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return PIC_ECUDA;
    if (s.vs && s.sorted) {
        // the lists the next push will read: built from what the last push
        // recorded unless a full sort comes first
        VisState v{};
        long long n = 0;
        if (cudaMemcpy(&v, s.vs, sizeof v, cudaMemcpyDeviceToHost) != cudaSuccess) return PIC_ECUDA;
        if (cudaMemcpy(&n, s.d_count, sizeof n, cudaMemcpyDeviceToHost) != cudaSuccess) return PIC_ECUDA;
        const bool built = s.vis_built_for == s.pushes_since_sort;
        out[0] = built ? (long long)v.nvis : std::min<long long>((long long)v.nraw, s.vcap);
        out[1] = built ? v.valid_cur
                       : (v.valid_next && visitor_lists_pay((unsigned long long)out[0], n, visitor_min_fraction(c)));
    }
    if (c->d_nstrag) {
        unsigned long long ns[2] = {0, 0};
        if (cudaMemcpy(ns, c->d_nstrag, sizeof ns, cudaMemcpyDeviceToHost) != cudaSuccess) return PIC_ECUDA;
        out[3] = (long long)ns[kind];
    }
    return PIC_OK;
}

void launch_tile_push(pic_ctx *c, int mask) {
    prepare_push(c, mask);
    bool spin = ((mask & 1) && spin_active(c, 0)) || ((mask & 2) && spin_active(c, 1));
    prof_begin(c, "tile_push_gather_deposit");
    if (c->fp32) {
        if (c->order == 2) spin ? tile_push_t<float, 3, true>(c, mask) : tile_push_t<float, 3, false>(c, mask);
        else spin ? tile_push_t<float, 5, true>(c, mask) : tile_push_t<float, 5, false>(c, mask);
    } else {
        if (c->order == 2) spin ? tile_push_t<double, 3, true>(c, mask) : tile_push_t<double, 3, false>(c, mask);
        else spin ? tile_push_t<double, 5, true>(c, mask) : tile_push_t<double, 5, false>(c, mask);
    }
    prof_end(c);
    prof_begin(c, "straggler_push");
    for (int k = 0; k < 2; ++k)
        if (((mask >> k) & 1) && c->sp[k].n_host > 0)
            launch_push_list(c, k, c->sp[k].strag, c->d_nstrag + k, vis_sink_of(c, c->sp[k]));
    prof_end(c);
    for (int k = 0; k < 2; ++k) {
        Species &s = c->sp[k];
        if (!((mask >> k) & 1) || s.n_host <= 0) continue;
        s.cur = 1 - s.cur;
        s.pushes_since_sort += 1;
    }
}

}  // namespace pic
