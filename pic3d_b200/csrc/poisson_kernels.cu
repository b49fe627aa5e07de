// Initial electrostatic field by an FP64 Poisson solve (no counterpart in
// the reference, which starts from E = 0 with a non-neutral random rho).
//
// The charge density of both species is deposited at the current particle
// positions with the shape the push uses for rho (src/particle.cpp:503-514:
// primal index (int)(x + 0.5), 2nd / 4th-order weights) onto the physical
// nodes, the mean is removed (the neutralising background of a single-
// species plasma; an exact solution needs a mean-free right-hand side
// because the operator below is singular), and
//
//     A phi = rho - <rho>,   A phi = sum_d (2 phi_p - phi_{p+e_d} - phi_{p-e_d}) / h_d^2
//
// is solved by conjugate gradients with E = -grad phi on the Yee faces:
// Ex(i+1/2) = -(phi(i+1) - phi(i)) / dx, and likewise Ey, Ez.  The discrete
// divergence the field diagnostics use, (Ex(i+1/2) - Ex(i-1/2)) / dx + ...,
// of that E is exactly A phi, so after the solve div E = rho - <rho> to the
// solver tolerance.  Periodic axes wrap; on absorbing axes the faces outside
// the physical nodes carry E = 0 (the reference's ghost values stay 0 there),
// a zero-flux (Neumann) condition on phi.  B is not touched.
//
// Conjugate gradients: the direction update p = r + beta p is folded into
// the operator kernel (it recomputes r + beta p at the six neighbours), so
// an iteration is four launches: operator + partial dot, scalar step,
// vector update + partial dots, scalar step.  Dot products are summed per
// block and then by one block in a fixed order (run-to-run reproducible);
// the scalars stay on the device and the host reads the residual every
// kCheckEvery iterations.  The constants are the operator's null space:
// the residual is used with its mean removed (the mean comes with r.r from
// the same pass), so rounding cannot feed a growing constant into phi once
// the iteration reaches the rounding floor.
#include <cmath>
#include <cstring>
#include <string>

#include "pic_kernels.cuh"

namespace pic {
namespace {

constexpr int kThreads = 256;
constexpr int kCheckEvery = 32;

struct NodeGrid {
    int n[3];
    int per[3];
    double ih2[3];   // 1 / h_d^2
    long long N;
};

__device__ __forceinline__ void node_coords(const NodeGrid &g, long long p, int &i, int &j, int &k) {
    i = (int)(p % g.n[0]);
    long long q = p / g.n[0];
    j = (int)(q % g.n[1]);
    k = (int)(q / g.n[1]);
}

// neighbour index along axis d in direction s (+1 / -1); -1 when outside a
// non-periodic axis
__device__ __forceinline__ long long neighbour(const NodeGrid &g, int i, int j, int k, int d, int s) {
    int c[3] = {i, j, k};
    c[d] += s;
    if (c[d] < 0 || c[d] >= g.n[d]) {
        if (!g.per[d]) return -1;
        c[d] = c[d] < 0 ? c[d] + g.n[d] : c[d] - g.n[d];
    }
    return ((long long)c[2] * g.n[1] + c[1]) * g.n[0] + c[0];
}

__device__ __forceinline__ double block_sum(double v, double *sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double t = 0.0;
    if (w == 0) {
        t = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    }
    return t;   // valid in thread 0
}

// rho of one species at the current positions onto the physical nodes
template <typename real, int P>
__global__ void deposit_rho_nodes_kernel(NodeGrid ng, Geom g, CellPack cp, int fp32, const double *x,
                                         const double *y, const double *z, const int *cell, const float *ox,
                                         const float *oy, const float *oz, const real *w, const long long *count,
                                         double charge, double *rho) {
    constexpr int H = P / 2;
    const long long n = *count;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        double v[3];
        if (fp32) {
            int c[3];
            cp.unpack(cell[t], c[0], c[1], c[2]);
            v[0] = (double)c[0] + (double)ox[t];
            v[1] = (double)c[1] + (double)oy[t];
            v[2] = (double)c[2] + (double)oz[t];
        } else {
            v[0] = x[t];
            v[1] = y[t];
            v[2] = z[t];
        }
        int base[3];
        double wt[3][P];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            // the push's periodic wrap (src/particle.cpp:123-167), then the
            // primal index in buffer coordinates (:173-181)
            if (g.per[d]) {
                if (v[d] < 0.0) v[d] += g.n[d];
                if (v[d] > (double)g.n[d]) v[d] -= g.n[d];
            }
            const double xc = v[d] - (double)(1 - g.mem);
            const int ip = (int)(xc + 0.5);
            shape_weights(xc - (double)ip, wt[d]);
            base[d] = ip - H - g.mem;   // physical node index of the first stencil point
        }
        const double qw = charge * (double)w[t];
        for (int a = 0; a < P; ++a) {
            int k = base[2] + a;
            if (k < 0 || k >= ng.n[2]) {
                if (!ng.per[2]) continue;
                k = k < 0 ? k + ng.n[2] : k - ng.n[2];
            }
            for (int b = 0; b < P; ++b) {
                int j = base[1] + b;
                if (j < 0 || j >= ng.n[1]) {
                    if (!ng.per[1]) continue;
                    j = j < 0 ? j + ng.n[1] : j - ng.n[1];
                }
                const double wjk = qw * wt[2][a] * wt[1][b];
#pragma unroll
                for (int e = 0; e < P; ++e) {
                    int i = base[0] + e;
                    if (i < 0 || i >= ng.n[0]) {
                        if (!ng.per[0]) continue;
                        i = i < 0 ? i + ng.n[0] : i - ng.n[0];
                    }
                    atomicAdd(rho + ((long long)k * ng.n[1] + j) * ng.n[0] + i, wjk * wt[0][e]);
                }
            }
        }
    }
}

// partial sums of v over blocks
__global__ void partial_sum_kernel(const double *v, long long N, double *part) {
    __shared__ double sh[32];
    double s = 0.0;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (long long)gridDim.x * blockDim.x)
        s += v[p];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// scalar slots
enum { S_RR = 0, S_PAP, S_ALPHA, S_BETA, S_BB, S_MEAN, S_RMEAN, S_NS };

// one block: sums of the partials in a fixed order (second set optional),
// then the CG scalar step `mode`: 0 s[slot] = sum; 1 alpha = rr / pAp;
// 2 with the mean-removed residual norm rr_new = sum(r^2) - N mean(r)^2:
// beta = rr_new / rr, rr = rr_new, rmean = mean(r); 3 mean = sum / N
__global__ void finish_kernel(const double *part, const double *part2, int nb, double *s, int slot, int mode,
                              double N) {
    __shared__ double sh[32];
    double v = 0.0, u = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) v += part[b];
    v = block_sum(v, sh);
    if (part2) {
        for (int b = threadIdx.x; b < nb; b += blockDim.x) u += part2[b];
        u = block_sum(u, sh);
    }
    if (threadIdx.x != 0) return;
    if (mode == 0) {
        s[slot] = v;
    } else if (mode == 1) {
        s[S_PAP] = v;
        s[S_ALPHA] = v != 0.0 ? s[S_RR] / v : 0.0;
    } else if (mode == 2) {
        const double m = u / N;
        const double rr = fmax(v - N * m * m, 0.0);
        s[S_BETA] = s[S_RR] != 0.0 ? rr / s[S_RR] : 0.0;
        s[S_RR] = rr;
        s[S_RMEAN] = m;
    } else {
        s[S_MEAN] = v / N;
    }
}

// b = rho - mean, r = b, p = 0 (beta = 0 makes the first direction r), x = 0;
// partial sums of b.b
__global__ void init_kernel(long long N, double *rho, double *r, double *pv, double *x, const double *s,
                            double *part) {
    __shared__ double sh[32];
    const double mean = s[S_MEAN];
    double acc = 0.0;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < N; q += (long long)gridDim.x * blockDim.x) {
        const double b = rho[q] - mean;
        rho[q] = b;
        r[q] = b;
        pv[q] = 0.0;
        x[q] = 0.0;
        acc += b * b;
    }
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

// new direction pn = (r - rmean) + beta p (recomputed at the six
// neighbours from r and the old p, so it needs no launch of its own),
// Ap = A pn, and partial sums of pn.Ap.  The caller swaps p and pn after the
// vector update.
__global__ void apply_kernel(NodeGrid g, const double *r, const double *p, double *pn, double *Ap, const double *s,
                             double *part) {
    __shared__ double sh[32];
    const double beta = s[S_BETA], rm = s[S_RMEAN];
    double acc = 0.0;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < g.N; q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        node_coords(g, q, i, j, k);
        const double pc = (r[q] - rm) + beta * p[q];
        double a = 0.0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
#pragma unroll
            for (int sgn = -1; sgn <= 1; sgn += 2) {
                const long long nb = neighbour(g, i, j, k, d, sgn);
                if (nb >= 0) a += (pc - ((r[nb] - rm) + beta * p[nb])) * g.ih2[d];
            }
        }
        pn[q] = pc;
        Ap[q] = a;
        acc += pc * a;
    }
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

// x += alpha p, r -= alpha Ap, partial sums of r.r and of r
__global__ void update_kernel(long long N, double *x, double *r, const double *p, const double *Ap, const double *s,
                              double *part, double *part2) {
    __shared__ double sh[32];
    const double alpha = s[S_ALPHA];
    double acc = 0.0, sum = 0.0;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < N; q += (long long)gridDim.x * blockDim.x) {
        x[q] += alpha * p[q];
        const double rn = r[q] - alpha * Ap[q];
        r[q] = rn;
        acc += rn * rn;
        sum += rn;
    }
    acc = block_sum(acc, sh);
    sum = block_sum(sum, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = acc;
        part2[blockIdx.x] = sum;
    }
}

// E = -grad phi on the faces of the physical nodes (buffer index of node
// (i, j, k) is (i + mem, j + mem, k + mem)); faces beyond the last node of
// an absorbing axis get 0
template <typename real>
__global__ void field_from_phi_kernel(NodeGrid ng, Geom g, const double *phi, double idx, double idy, double idz,
                                      real *ex, real *ey, real *ez) {
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < ng.N;
         q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        node_coords(ng, q, i, j, k);
        const double pc = phi[q];
        const double ih[3] = {idx, idy, idz};
        double e[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const long long nb = neighbour(ng, i, j, k, d, +1);
            e[d] = nb >= 0 ? -(phi[nb] - pc) * ih[d] : 0.0;
        }
        const int b = g.fi(k + g.mem, j + g.mem, i + g.mem);
        ex[b] = (real)e[0];
        ey[b] = (real)e[1];
        ez[b] = (real)e[2];
    }
}

// max |div E - b| over the physical nodes from the stored E (E's own
// precision), with b = rho - <rho>; max of non-negative doubles through
// their ordered bit patterns
template <typename real>
__global__ void residual_kernel(NodeGrid ng, Geom g, const real *ex, const real *ey, const real *ez, double idx,
                                double idy, double idz, const double *b, unsigned long long *out) {
    double m = 0.0;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < ng.N;
         q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        node_coords(ng, q, i, j, k);
        const int c = g.fi(k + g.mem, j + g.mem, i + g.mem);
        const double div = ((double)ex[c] - (double)ex[c - 1]) * idx + ((double)ey[c] - (double)ey[c - g.f[0]]) * idy +
                           ((double)ez[c] - (double)ez[c - g.fxy]) * idz;
        m = fmax(m, fabs(div - b[q]));
    }
    atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

template <typename real>
int solve(pic_ctx *c, double rel_tol, int max_iter, double *res) {
    const Geom &g = c->g;
    NodeGrid ng{};
    const double h[3] = {c->p.dx, c->p.dy, c->p.dz};
    for (int d = 0; d < 3; ++d) {
        ng.n[d] = g.n[d];
        ng.per[d] = g.per[d];
        ng.ih2[d] = 1.0 / (h[d] * h[d]);
    }
    ng.N = (long long)g.n[0] * g.n[1] * g.n[2];
    const long long N = ng.N;
    const int nb = (int)std::min<long long>((N + kThreads - 1) / kThreads, 148LL * 8);
    cudaStream_t st = c->stream;
    // scratch: rho / b, phi, r, p, pn, Ap, partials, scalars, residual word
    double *buf = nullptr;
    const size_t bytes = (size_t)(6 * N + 2 * nb + S_NS + 1) * sizeof(double);
    cudaError_t e = cudaMallocAsync((void **)&buf, bytes, st);
    if (e != cudaSuccess) {
        c->err = std::string("pic_solve_initial_field: cudaMallocAsync: ") + cudaGetErrorString(e);
        return e == cudaErrorMemoryAllocation ? PIC_ENOMEM : PIC_ECUDA;
    }
    double *b = buf, *x = b + N, *r = x + N, *p = r + N, *pn = p + N, *Ap = pn + N;
    double *part = Ap + N, *part2 = part + nb, *s = part2 + nb;
    unsigned long long *maxw = (unsigned long long *)(s + S_NS);
    cudaMemsetAsync(b, 0, (size_t)N * sizeof(double), st);
    cudaMemsetAsync(s, 0, (S_NS + 1) * sizeof(double), st);
    for (int k = 0; k < 2; ++k) {
        Species &sp = c->sp[k];
        if (sp.n_host <= 0) continue;
        const int cu = sp.cur;
        const unsigned grid = (unsigned)std::min<long long>((sp.n_host + kThreads - 1) / kThreads, 148LL * 16);
        if (c->order == 2)
            deposit_rho_nodes_kernel<real, 3><<<grid, kThreads, 0, st>>>(
                ng, g, c->cp, c->fp32, sp.a.x[cu], sp.a.y[cu], sp.a.z[cu], sp.a.cell[cu], sp.a.ox[cu], sp.a.oy[cu],
                sp.a.oz[cu], (const real *)sp.a.w, sp.d_count, c->p.charge[k], b);
        else
            deposit_rho_nodes_kernel<real, 5><<<grid, kThreads, 0, st>>>(
                ng, g, c->cp, c->fp32, sp.a.x[cu], sp.a.y[cu], sp.a.z[cu], sp.a.cell[cu], sp.a.ox[cu], sp.a.oy[cu],
                sp.a.oz[cu], (const real *)sp.a.w, sp.d_count, c->p.charge[k], b);
    }
    partial_sum_kernel<<<nb, kThreads, 0, st>>>(b, N, part);
    finish_kernel<<<1, kThreads, 0, st>>>(part, nullptr, nb, s, 0, 3, (double)N);
    init_kernel<<<nb, kThreads, 0, st>>>(N, b, r, p, x, s, part);
    finish_kernel<<<1, kThreads, 0, st>>>(part, nullptr, nb, s, S_BB, 0, 0.0);
    // rr = bb, beta = 0
    cudaMemcpyAsync(s + S_RR, s + S_BB, sizeof(double), cudaMemcpyDeviceToDevice, st);
    double hs[S_NS] = {};
    cudaMemcpyAsync(hs, s, sizeof(hs), cudaMemcpyDeviceToHost, st);
    e = cudaStreamSynchronize(st);
    int it = 0;
    double rel = 0.0;
    const double bb = hs[S_BB];
    if (e == cudaSuccess && bb > 0.0) {
        while (it < max_iter) {
            apply_kernel<<<nb, kThreads, 0, st>>>(ng, r, p, pn, Ap, s, part);
            finish_kernel<<<1, kThreads, 0, st>>>(part, nullptr, nb, s, 0, 1, 0.0);
            update_kernel<<<nb, kThreads, 0, st>>>(N, x, r, pn, Ap, s, part, part2);
            finish_kernel<<<1, kThreads, 0, st>>>(part, part2, nb, s, 0, 2, (double)N);
            std::swap(p, pn);
            ++it;
            if (it % kCheckEvery == 0 || it == max_iter) {
                cudaMemcpyAsync(hs, s, sizeof(hs), cudaMemcpyDeviceToHost, st);
                e = cudaStreamSynchronize(st);
                if (e != cudaSuccess) break;
                rel = std::sqrt(hs[S_RR] / bb);
                if (rel <= rel_tol) break;
            }
        }
    }
    if (e == cudaSuccess) {
        real **F = (real **)c->field;
        for (int a = 0; a < 3; ++a) cudaMemsetAsync(F[a], 0, (size_t)g.fsz * sizeof(real), st);
        field_from_phi_kernel<real><<<nb, kThreads, 0, st>>>(ng, g, x, 1.0 / h[0], 1.0 / h[1], 1.0 / h[2], F[0], F[1],
                                                             F[2]);
        for (int a = 0; a < 3; ++a) launch_ghost_fill_one(c, a);
        residual_kernel<real><<<nb, kThreads, 0, st>>>(ng, g, F[0], F[1], F[2], 1.0 / h[0], 1.0 / h[1], 1.0 / h[2],
                                                       b, maxw);
        cudaMemcpyAsync(hs, s, sizeof(hs), cudaMemcpyDeviceToHost, st);
        unsigned long long mw = 0;
        cudaMemcpyAsync(&mw, maxw, sizeof(mw), cudaMemcpyDeviceToHost, st);
        e = cudaStreamSynchronize(st);
        double gmax;
        std::memcpy(&gmax, &mw, sizeof(gmax));
        res[0] = it;
        res[1] = bb > 0.0 ? std::sqrt(hs[S_RR] / bb) : 0.0;
        res[2] = hs[S_MEAN];
        res[3] = gmax;
    }
    cudaFreeAsync(buf, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        c->err = std::string("pic_solve_initial_field: ") + cudaGetErrorString(e);
        return PIC_ECUDA;
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        c->err = std::string("pic_solve_initial_field: ") + cudaGetErrorString(e);
        return PIC_ECUDA;
    }
    return PIC_OK;
}

}  // namespace
}  // namespace pic

extern "C" int pic_solve_initial_field(pic_ctx *c, double rel_tol, int max_iter, double *out, int nout) {
    if (!c || !out || nout < PIC_NPOISSON || !(rel_tol > 0.0) || max_iter < 1) {
        if (c) c->err = "pic_solve_initial_field: needs rel_tol > 0, max_iter >= 1 and out[4]";
        return PIC_EINVAL;
    }
    cudaSetDevice(c->device);
    double res[PIC_NPOISSON] = {};
    const int r = c->fp32 ? pic::solve<float>(c, rel_tol, max_iter, res) : pic::solve<double>(c, rel_tol, max_iter, res);
    for (int k = 0; k < PIC_NPOISSON; ++k) out[k] = res[k];
    if (r == PIC_OK && !(res[1] <= rel_tol)) {
        c->err = "pic_solve_initial_field: conjugate gradients reached max_iter before rel_tol (relative residual " +
                 std::to_string(res[1]) + "); E holds the last iterate";
        return PIC_ENOCONV;
    }
    return r;
}
