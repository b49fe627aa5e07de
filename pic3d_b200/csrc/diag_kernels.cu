// FP64 diagnostics: field energy, kinetic energy and charge per species,
// and the largest Gauss-law residual |div E - rho| over physical nodes.
// The reference has no diagnostics; these run in FP64 in both precisions.
#include "pic_kernels.cuh"

namespace pic {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ void block_add(double v, double *out) {
    __shared__ double part[32];
    v = warp_sum(v);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) part[wid] = v;
    __syncthreads();
    if (wid == 0) {
        int nw = (blockDim.x + 31) >> 5;
        v = lane < nw ? part[lane] : 0.0;
        v = warp_sum(v);
        if (lane == 0) atomicAdd(out, v);
    }
    __syncthreads();
}

template <typename real>
__global__ void field_diag_kernel(Geom g, const real *ex, const real *ey, const real *ez, const real *bx,
                                  const real *by, const real *bz, const real *r0, const real *r1, double dV,
                                  double idx, double idy, double idz, double *out) {
    long long ncell = (long long)g.n[0] * g.n[1] * g.n[2];
    double e = 0.0, q0 = 0.0, q1 = 0.0, gmax = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < ncell;
         t += (long long)gridDim.x * blockDim.x) {
        int i = (int)(t % g.n[0]) + g.mem;
        int j = (int)((t / g.n[0]) % g.n[1]) + g.mem;
        int k = (int)(t / ((long long)g.n[0] * g.n[1])) + g.mem;
        int c = g.fi(k, j, i), rc = g.ri(k, j, i);
        double a = ex[c], b = ey[c], d = ez[c], u = bx[c], v = by[c], w = bz[c];
        e += a * a + b * b + d * d + u * u + v * v + w * w;
        double rho0 = r0 ? (double)r0[rc] : 0.0, rho1 = r1 ? (double)r1[rc] : 0.0;
        q0 += rho0;
        q1 += rho1;
        double div = ((double)ex[c] - (double)ex[c - 1]) * idx + ((double)ey[c] - (double)ey[c - g.f[0]]) * idy +
                     ((double)ez[c] - (double)ez[c - g.fxy]) * idz;
        double res = fabs(div - rho0 - rho1);
        gmax = (res != res || res > gmax) ? res : gmax;   // a NaN residual wins and stays
    }
    block_add(0.5 * e * dV, out + 0);
    block_add(q0 * dV, out + 3);
    block_add(q1 * dV, out + 4);
    // max of non-negative doubles through their ordered bit patterns (a
    // positive NaN orders above every finite value and +inf)
    atomicMax((unsigned long long *)(out + 5), (unsigned long long)__double_as_longlong(gmax));
}

template <typename real>
__global__ void kinetic_kernel(const real *px, const real *py, const real *pz, const real *w,
                               const long long *count, double mass, double *out) {
    long long n = *count;
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        double a = px[i], b = py[i], c = pz[i];
        double u2 = a * a + b * b + c * c;
        // gamma - 1 without cancellation
        double gm1 = u2 / (sqrt(1.0 + u2) + 1.0);
        s += (double)w[i] * mass * gm1;
    }
    block_add(s, out);
}

template <typename real>
static void diag_t(pic_ctx *c, double *d_out) {
    const Geom &g = c->g;
    real **F = (real **)c->field;
    real **R = (real **)c->ring;
    const PicParams &p = c->p;
    double dV = p.dx * p.dy * p.dz;
    field_diag_kernel<real><<<148 * 4, 256, 0, c->stream>>>(g, F[0], F[1], F[2], F[3], F[4], F[5], R[3], R[4],
                                                            dV, 1.0 / p.dx, 1.0 / p.dy, 1.0 / p.dz, d_out);
    for (int k = 0; k < 2; ++k) {
        Species &s = c->sp[k];
        if (!s.a.px || s.n_host == 0) continue;
        kinetic_kernel<real><<<148 * 4, 256, 0, c->stream>>>((real *)s.a.px, (real *)s.a.py, (real *)s.a.pz,
                                                             (real *)s.a.w, s.d_count, p.mass[k], d_out + 1 + k);
    }
}

void launch_diagnostics(pic_ctx *c, double *d_out) {
    cudaMemsetAsync(d_out, 0, PIC_NDIAG * sizeof(double), c->stream);
    if (c->fp32) diag_t<float>(c, d_out); else diag_t<double>(c, d_out);
}

}  // namespace pic
