// Internal declarations shared by the CUDA translation units of
// libpic3d_b200.so.  Not part of the public ABI (see include/pic3d_gpu.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/pic3d_gpu.h"

namespace pic {

// ---------------------------------------------------------------------------
// device status bits (OR-ed by kernels, read back by pic_synchronize)
enum : unsigned {
    ST_OOB = 1u << 0,       // stencil would leave the buffers: particle skipped
    ST_NAN = 1u << 1,       // non-finite momentum / position
    ST_RANGE = 1u << 2,     // g_factor argument outside the table
    ST_OVERFLOW = 1u << 3,  // a bin or list overflowed
    ST_TIMEOUT = 1u << 4,   // bounded wait gave up
    ST_CFL = 1u << 5,       // a particle moved a cell or more in one step
};

// ---------------------------------------------------------------------------
// geometry of one rank's buffers (src/simulation.cpp:23-75, 132-144):
// physical cells mem..n+mem-1, field buffer 0..n+2mem-1, ring -1..n+2mem.
// Particle coordinate x (cells, domain [0,n)) sits at buffer x + mem - 1.
struct Geom {
    int n[3];      // physical cells
    int mem;       // ghost width
    int f[3];      // field buffer extent n + 2 mem
    int r[3];      // ring extent n + 2 mem + 2
    int per[3];    // periodic faces
    int fxy, rxy;  // plane strides
    long long fsz, rsz;

    __host__ __device__ __forceinline__ int fi(int k, int j, int i) const { return (k * f[1] + j) * f[0] + i; }
    __host__ __device__ __forceinline__ int ri(int k, int j, int i) const {
        return ((k + 1) * r[1] + (j + 1)) * r[0] + (i + 1);
    }
};

Geom make_geom(const PicParams &p);

// ---------------------------------------------------------------------------
// shape functions as functions of delta = x - round(x) in [-0.5, 0.5):
// quadratic B-spline (src/particle.cpp:8-19) and quartic B-spline
// (src/particle.cpp:21-48 with the coefficients of src/constants.cpp:84-85).
template <typename real>
__device__ __forceinline__ void shape_weights(real d, real (&w)[3]) {
    const real h = real(0.5);
    w[0] = h * (h - d) * (h - d);
    w[1] = real(0.75) - d * d;
    w[2] = h * (h + d) * (h + d);
}

template <typename real>
__device__ __forceinline__ void shape_weights(real d, real (&w)[5]) {
    const real a0 = real(55.0 / 96.0), a1 = real(5.0 / 24.0), a2 = real(5.0 / 4.0), a3 = real(5.0 / 6.0);
    const real b0 = real(115.0 / 192.0), b2 = real(5.0 / 8.0);
    real u, u2;
    u = d - real(0.5);
    u2 = u * u;
    w[0] = u2 * u2 * real(1.0 / 24.0);
    u = d + real(1.0);
    u2 = u * u;
    w[1] = -u2 * u2 * real(1.0 / 6.0) + u2 * u * a3 - u2 * a2 + u * a1 + a0;
    u = d;
    u2 = u * u;
    w[2] = u2 * u2 * real(0.25) - u2 * b2 + b0;
    u = d - real(1.0);
    u2 = u * u;
    w[3] = -u2 * u2 * real(1.0 / 6.0) - u2 * u * a3 - u2 * a2 - u * a1 + a0;
    u = d + real(0.5);
    u2 = u * u;
    w[4] = u2 * u2 * real(1.0 / 24.0);
}

// cubic B-spline basis of the laser amplitude grid (extension), support |t| < 2
__device__ __forceinline__ double cubic_bspline(double t) {
    double a = fabs(t);
    if (a < 1.0) return (4.0 - 6.0 * a * a + 3.0 * a * a * a) / 6.0;
    if (a < 2.0) {
        double b = 2.0 - a;
        return b * b * b / 6.0;
    }
    return 0.0;
}

// ---------------------------------------------------------------------------
// particle storage (structure of arrays, one set per species)
//   FP64: x,y,z absolute cell coordinates as in the reference, two buffers
//         (current and previous positions) that swap every push.
//   FP32: packed int32 cell index + three FP32 in-cell offsets in [0,1).
struct PartArrays {
    double *x[2] = {nullptr, nullptr}, *y[2] = {nullptr, nullptr}, *z[2] = {nullptr, nullptr};
    int *cell[2] = {nullptr, nullptr};
    float *ox[2] = {nullptr, nullptr}, *oy[2] = {nullptr, nullptr}, *oz[2] = {nullptr, nullptr};
    void *px = nullptr, *py = nullptr, *pz = nullptr, *w = nullptr;   // double* or float* by precision
    void *sx = nullptr, *sy = nullptr, *sz = nullptr;                 // spins (only when spin is on)
    int *id = nullptr;
};

// half-cell octants per cell in the particle sort key (tile, octant, cell)
constexpr int kOctants = 8;

// Visitor-list state of one species on the device.  valid_cur: the lists
// the running push reads name every particle that is away from its home
// tile (else the push falls back to handing such particles to the global
// kernel).  valid_next: the same for the entries the running push appends;
// cleared when vraw overflows, when removal compacts the arrays, or when a
// particle lands outside the tile grid on a periodic axis.
struct VisState {
    unsigned long long nraw;   // entries appended to vraw by the running push
    unsigned valid_cur, valid_next;
    unsigned long long nvis;   // entries of the current lists
};

// Where a push records the particles that end away from their home tile
// (raw null: not recorded).  See Species::vraw.
struct VisSink {
    int *raw;                    // (index, home tile, new tile) triples
    VisState *vs;
    long long cap;               // triples
    int T, nt[3];
};

struct Species {
    int64_t cap = 0;
    int64_t n_host = 0;      // host copy of the count (upper bound between syncs)
    long long *d_count = nullptr;
    int cur = 0;             // which position buffer is current
    PartArrays a;            // the particles
    PartArrays b;            // destination of the counting sort (same shapes)
    int *keys = nullptr;     // per-particle sort key
    int *strag = nullptr;    // particles the tiled kernel hands to the global kernel: (index, home tile) pairs
    // Incremental re-binning between full sorts.  A particle's home tile is
    // the tile whose slice of the sorted arrays holds it; a particle whose
    // cell lies in another tile is a visitor there.  Each push appends
    // (index, home, new tile) for every particle that ends away from home
    // (vraw); before the next push a counting sort of those entries by tile
    // gives each tile its visitor list (vis, (index, home) pairs, vis_off).
    int *vraw = nullptr;
    int *vis = nullptr;
    unsigned *vis_off = nullptr;   // ntiles + 1
    unsigned *vis_cnt = nullptr;   // ntiles + 1 (histogram, then cursor)
    int64_t vcap = 0;              // entries of vraw / vis
    VisState *vs = nullptr;        // device counters and flags
    int vis_built_for = -1;        // pushes_since_sort when the lists were last built
    unsigned char *dead = nullptr;  // adjoint mode: 1 once a particle left through an absorbing face
    // adjoint mode with tiles: the sort moves every per-particle array, so
    // the upload index travels with the particle (orig) and each sort's
    // gather permutation (perm[new] = old) is kept for the tape
    int *orig = nullptr, *orig_b = nullptr;
    unsigned char *dead_b = nullptr;
    int *perm = nullptr;
    bool perm_fresh = false;   // perm holds a sort the tape has not recorded yet
    unsigned *offs = nullptr;  // per-key start offsets after the last sort (nkeys + 1)
    bool sorted = false;     // offs describes the current order
    int pushes_since_sort = 0;
    double max_abs_w = 0.0;  // largest |weight| uploaded (weights never change afterwards)
    bool spin_nonzero = false;
};

// bit layout of the FP32 packed cell: (cx+1) | (cy+1) << bx | (cz+1) << (bx+by)
struct CellPack {
    int bx, by, bz;
    unsigned mx, my;
    __host__ __device__ __forceinline__ int pack(int cx, int cy, int cz) const {
        return (int)((unsigned)(cx + 1) | ((unsigned)(cy + 1) << bx) | ((unsigned)(cz + 1) << (bx + by)));
    }
    __host__ __device__ __forceinline__ void unpack(int c, int &cx, int &cy, int &cz) const {
        unsigned u = (unsigned)c;
        cx = (int)(u & mx) - 1;
        cy = (int)((u >> bx) & my) - 1;
        cz = (int)(u >> (bx + by)) - 1;
    }
};

struct ProfEntry {
    const char *name;
    cudaEvent_t a, b;
};

}  // namespace pic

// the opaque context of the C ABI
struct pic_ctx {
    PicParams p{};
    pic::Geom g{};
    pic::CellPack cp{};
    int device = 0;
    int fp32 = 0;
    int order = 4;
    cudaStream_t stream = nullptr;
    void *field[6] = {};   // ex ey ez bx by bz (double* or float*)
    void *ring[5] = {};    // jx jy jz rho0 rho1
    pic::Species sp[2];
    unsigned *d_status = nullptr;
    double *d_gtab = nullptr;
    int gtab_n = 0;
    double *d_profile = nullptr;
    int profile_n = 0;
    // scratch (conversion staging and compaction lists)
    void *d_stage = nullptr;
    size_t stage_bytes = 0;
    long long *d_scratch_ll = nullptr;   // small counters
    int *d_list = nullptr;               // compaction index lists
    int64_t list_cap = 0;
    double *d_diag = nullptr;
    // pinned host staging for particle uploads / downloads: two buffers of
    // kPinRecords records each, used alternately so that the host copy of
    // one chunk overlaps the DMA of the other
    void *h_pin[2] = {nullptr, nullptr};
    int64_t pin_records = 0;
    cudaEvent_t pin_ev[2] = {nullptr, nullptr};
    // tiling / sorting
    int tile = 0;                        // tile edge in cells (0: global-memory kernel only)
    int ntile[3] = {0, 0, 0};
    long long nkeys = 0;                 // ntiles * kOctants * tile^3
    unsigned *d_hist = nullptr;          // nkeys + 1
    unsigned *d_blocksums = nullptr;
    unsigned long long *d_nstrag = nullptr;   // straggler counts, one per species
    int sort_interval = 4;
    // rho is observable only between ABI calls: the intermediate steps of
    // one pic_run_steps call neither clear, deposit nor fold it (set while
    // such a step runs; never in adjoint mode, whose checkpoints copy rho)
    bool rho_skip = false;
    int steps_since_sort = 0;
    int step = 0;
    std::string err;
    // profiling
    bool prof = false;
    std::vector<pic::ProfEntry> prof_events;
    std::vector<std::pair<const char *, std::pair<double, int64_t>>> prof_acc;
};
