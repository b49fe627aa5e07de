// Field diagnostics that allocate no device memory.
//
// pic_diagnostics (diag_kernels.cu) needs a context, whose creation
// allocates, and it accumulates into context-owned scratch.  Some callers
// cannot let a library call cudaMalloc: a host code that reserves nearly all
// of HBM for its own particle and field arrays up front (allocation would
// fail), or one that allows device memory only through its own pool
// (cudaMalloc / cudaFree also synchronise the device and stall work queued
// on other streams).  pic_field_diagnostics_noalloc serves them: it reads
// caller-owned FP64 arrays and writes caller-owned output, and its only
// scratch is the file-scope array below.
//
// The scratch holds one partial sum per physical z plane (field energy,
// charge of each species, largest Gauss residual), so the grid may have at
// most PIC_NOALLOC_MAX_PLANES planes along z; larger grids are rejected with
// PIC_EINVAL.  Every device that loads the library holds this 64 KiB until
// the process exits.  Each call writes the slots of planes [0, nz) before
// reading them, so nothing has to start at zero, and the final sum runs in
// plane order: the result does not depend on the launch.  All calls share
// the array, so calls that overlap on the GPU (different streams, or several
// host threads) race: serialise them.
#include <cmath>
#include <cstdio>
#include <mutex>

#include "pic_kernels.cuh"

#define PIC_NOALLOC_MAX_PLANES 2048
#define PIC_NOALLOC_MAX_DEVICES 64

namespace pic {

static __device__ __align__(256) double g_noalloc_plane_partials[4 * PIC_NOALLOC_MAX_PLANES];

namespace {

// Host code only sees a host-side stand-in for the array's name; the device
// address comes from cudaGetSymbolAddress, looked up once per device with
// that device current (the first call on each device does this; it queries
// an address and allocates nothing).
double *g_scratch_addr[PIC_NOALLOC_MAX_DEVICES] = {};
std::mutex g_scratch_mu;

int scratch_for_current_device(double **out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return PIC_ECUDA;
    if (dev < 0 || dev >= PIC_NOALLOC_MAX_DEVICES) return PIC_EINVAL;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_plane_partials);
        if (e != cudaSuccess || !p) {
            std::fprintf(stderr, "pic_field_diagnostics_noalloc: cudaGetSymbolAddress: %s\n",
                         cudaGetErrorString(e));
            return PIC_ECUDA;
        }
        g_scratch_addr[dev] = static_cast<double *>(p);
    }
    *out = g_scratch_addr[dev];
    return PIC_OK;
}

}  // namespace

// largest of two residuals with NaN winning (fmax and a plain compare would
// drop a NaN residual and report a finite Gauss error for a NaN field)
__device__ __forceinline__ double nan_max(double a, double b) { return (a != a || a > b) ? a : b; }

// one CTA per physical z plane: partial sums in a fixed tree order
__global__ void __launch_bounds__(256) noalloc_plane_kernel(Geom g, const double *__restrict__ ex,
                                                            const double *__restrict__ ey,
                                                            const double *__restrict__ ez,
                                                            const double *__restrict__ bx,
                                                            const double *__restrict__ by,
                                                            const double *__restrict__ bz,
                                                            const double *__restrict__ r0,
                                                            const double *__restrict__ r1, double idx,
                                                            double idy, double idz, double *partials) {
    __shared__ double red[4][256];
    const int k = blockIdx.x + g.mem;
    const int ncell = g.n[0] * g.n[1];
    double e = 0.0, q0 = 0.0, q1 = 0.0, gmax = 0.0;
    for (int t = threadIdx.x; t < ncell; t += blockDim.x) {
        int i = t % g.n[0] + g.mem, j = t / g.n[0] + g.mem;
        int c = g.fi(k, j, i), rc = g.ri(k, j, i);
        double a = ex[c], b = ey[c], d = ez[c], u = bx[c], v = by[c], w = bz[c];
        e += a * a + b * b + d * d + u * u + v * v + w * w;
        double s0 = r0 ? r0[rc] : 0.0, s1 = r1 ? r1[rc] : 0.0;
        q0 += s0;
        q1 += s1;
        double div = (ex[c] - ex[c - 1]) * idx + (ey[c] - ey[c - g.f[0]]) * idy + (ez[c] - ez[c - g.fxy]) * idz;
        double res = fabs(div - s0 - s1);
        gmax = nan_max(res, gmax);
    }
    red[0][threadIdx.x] = e;
    red[1][threadIdx.x] = q0;
    red[2][threadIdx.x] = q1;
    red[3][threadIdx.x] = gmax;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            red[0][threadIdx.x] += red[0][threadIdx.x + s];
            red[1][threadIdx.x] += red[1][threadIdx.x + s];
            red[2][threadIdx.x] += red[2][threadIdx.x + s];
            red[3][threadIdx.x] = nan_max(red[3][threadIdx.x], red[3][threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double *o = partials + 4 * blockIdx.x;
        o[0] = red[0][0];
        o[1] = red[1][0];
        o[2] = red[2][0];
        o[3] = red[3][0];
    }
}

// planes summed in order by one thread: out = {field energy, charge of
// species 0, charge of species 1, max Gauss residual}
__global__ void noalloc_planes_sum_kernel(const double *partials, int nz, double dV, double *out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double e = 0.0, q0 = 0.0, q1 = 0.0, gmax = 0.0;
    for (int k = 0; k < nz; ++k) {
        e += partials[4 * k + 0];
        q0 += partials[4 * k + 1];
        q1 += partials[4 * k + 2];
        gmax = nan_max(partials[4 * k + 3], gmax);
    }
    out[0] = 0.5 * e * dV;
    out[1] = q0 * dV;
    out[2] = q1 * dV;
    out[3] = gmax;
}

}  // namespace pic

extern "C" int pic_field_diagnostics_noalloc(const PicParams *p, const double *ex, const double *ey,
                                             const double *ez, const double *bx, const double *by,
                                             const double *bz, const double *rho0, const double *rho1,
                                             double *out, void *stream) {
    using namespace pic;
    if (!p || !ex || !ey || !ez || !bx || !by || !bz || !out) return PIC_EINVAL;
    if (p->mem != 2 && p->mem != 4) return PIC_EINVAL;
    if (p->local_xcells < 1 || p->local_ycells < 1 || p->local_zcells < 1) return PIC_EINVAL;
    if (p->local_zcells > PIC_NOALLOC_MAX_PLANES) {
        std::fprintf(stderr,
                     "pic_field_diagnostics_noalloc: %d z planes exceed the static scratch of %d planes\n",
                     p->local_zcells, PIC_NOALLOC_MAX_PLANES);
        return PIC_EINVAL;
    }
    if (p->local_xcells > (1 << 20) || p->local_ycells > (1 << 20)) return PIC_EINVAL;
    const Geom g = make_geom(*p);
    if (g.rsz >= (1ll << 31)) return PIC_EINVAL;
    double *partials = nullptr;
    int r = scratch_for_current_device(&partials);
    if (r != PIC_OK) return r;
    // An error already pending on this thread belongs to earlier work, not to
    // these launches: report it without consuming it and launch nothing.
    cudaError_t before = cudaPeekAtLastError();
    if (before != cudaSuccess) {
        std::fprintf(stderr, "pic_field_diagnostics_noalloc: CUDA error pending from earlier work: %s\n",
                     cudaGetErrorString(before));
        return PIC_ECUDA;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    noalloc_plane_kernel<<<g.n[2], 256, 0, s>>>(g, ex, ey, ez, bx, by, bz, rho0, rho1, 1.0 / p->dx, 1.0 / p->dy,
                                                 1.0 / p->dz, partials);
    cudaError_t e = cudaPeekAtLastError();
    if (e == cudaSuccess) {
        noalloc_planes_sum_kernel<<<1, 32, 0, s>>>(partials, g.n[2], p->dx * p->dy * p->dz, out);
        e = cudaPeekAtLastError();
    }
    if (e != cudaSuccess) {
        cudaGetLastError();   // this launch's own error: consumed here, reported by the status
        std::fprintf(stderr, "pic_field_diagnostics_noalloc: launch failed: %s\n", cudaGetErrorString(e));
        return PIC_ECUDA;
    }
    return PIC_OK;
}
