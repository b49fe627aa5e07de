// C ABI of libpic3d_b200.so (include/pic3d_gpu.h): context lifetime, device
// memory, host <-> device conversion and the per-step orchestration of the
// reference's run_main_time_loop (src/simulation.cpp:159-183).
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "pic_kernels.cuh"

using namespace pic;

namespace {

int fail(pic_ctx *c, int code, const std::string &msg) {
    if (c) c->err = msg;
    return code;
}

#define CK(call)                                                                                       \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess)                                                                         \
            return fail(c, e_ == cudaErrorMemoryAllocation ? PIC_ENOMEM : PIC_ECUDA,                   \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                           \
    } while (0)

int launch_check(pic_ctx *c, const char *what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(c, PIC_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return PIC_OK;
}

size_t real_size(const pic_ctx *c) { return c->fp32 ? sizeof(float) : sizeof(double); }

int bits_for(int n) {
    int b = 1;
    while ((1 << b) < n + 2) ++b;
    return b;
}

template <typename T>
int dalloc(pic_ctx *c, T **p, size_t bytes) {
    *p = nullptr;
    if (bytes == 0) return PIC_OK;
    cudaError_t e = cudaMalloc((void **)p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        return fail(c, PIC_ENOMEM, std::string("cudaMalloc(") + std::to_string(bytes) + "): " + cudaGetErrorString(e));
    }
    return PIC_OK;
}

void free_arrays(PartArrays &a) {
    void *ptrs[] = {a.x[0], a.x[1], a.y[0], a.y[1], a.z[0], a.z[1], a.cell[0], a.cell[1], a.ox[0], a.ox[1],
                    a.oy[0], a.oy[1], a.oz[0], a.oz[1], a.px, a.py, a.pz, a.w, a.sx, a.sy, a.sz, a.id};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    a = PartArrays{};
}

void free_species(Species &s) {
    free_arrays(s.a);
    free_arrays(s.b);
    if (s.d_count) cudaFree(s.d_count);
    if (s.keys) cudaFree(s.keys);
    if (s.strag) cudaFree(s.strag);
    if (s.dead) cudaFree(s.dead);
    void *adj[4] = {s.orig, s.orig_b, s.dead_b, s.perm};
    for (void *p : adj)
        if (p) cudaFree(p);
    void *vis[5] = {s.vraw, s.vis, s.vis_off, s.vis_cnt, s.vs};
    for (void *p : vis)
        if (p) cudaFree(p);
    if (s.offs) cudaFree(s.offs);
    s = Species{};
}

int alloc_arrays(pic_ctx *c, PartArrays &a, size_t n, bool spin) {
    const size_t rs = real_size(c);
    int r = PIC_OK;
    for (int b = 0; b < 2 && r == PIC_OK; ++b) {
        if (c->fp32) {
            r = r ? r : dalloc(c, &a.cell[b], n * sizeof(int));
            r = r ? r : dalloc(c, &a.ox[b], n * sizeof(float));
            r = r ? r : dalloc(c, &a.oy[b], n * sizeof(float));
            r = r ? r : dalloc(c, &a.oz[b], n * sizeof(float));
        } else {
            r = r ? r : dalloc(c, &a.x[b], n * sizeof(double));
            r = r ? r : dalloc(c, &a.y[b], n * sizeof(double));
            r = r ? r : dalloc(c, &a.z[b], n * sizeof(double));
        }
    }
    void **mom[4] = {&a.px, &a.py, &a.pz, &a.w};
    for (void **m : mom) r = r ? r : dalloc(c, (char **)m, n * rs);
    if (spin) {
        void **sp[3] = {&a.sx, &a.sy, &a.sz};
        for (void **m : sp) r = r ? r : dalloc(c, (char **)m, n * rs);
    }
    r = r ? r : dalloc(c, &a.id, n * sizeof(int));
    return r;
}

int alloc_species(pic_ctx *c, int kind, int64_t cap, bool spin) {
    Species &s = c->sp[kind];
    free_species(s);
    s.cap = cap;
    const size_t n = (size_t)(cap > 0 ? cap : 1);
    int r = alloc_arrays(c, s.a, n, spin);
    if (c->tile > 0 && cap > 0) {
        r = r ? r : alloc_arrays(c, s.b, n, spin);
        r = r ? r : dalloc(c, &s.keys, n * sizeof(int));
        r = r ? r : dalloc(c, &s.strag, 2 * n * sizeof(int));
        r = r ? r : dalloc(c, &s.offs, (size_t)(c->nkeys + 1) * sizeof(unsigned));
        if (!c->p.adjoint) {
            // visitor lists for half of the capacity (a full list only makes
            // the next push fall back to the global kernel)
            const size_t nt = (size_t)c->ntile[0] * c->ntile[1] * c->ntile[2];
            s.vcap = (int64_t)(n / 2 + 1024);
            r = r ? r : dalloc(c, &s.vraw, 3 * (size_t)s.vcap * sizeof(int));
            r = r ? r : dalloc(c, &s.vis, 2 * (size_t)s.vcap * sizeof(int));
            r = r ? r : dalloc(c, &s.vis_off, (nt + 1) * sizeof(unsigned));
            r = r ? r : dalloc(c, &s.vis_cnt, (nt + 1) * sizeof(unsigned));
            r = r ? r : dalloc(c, &s.vs, sizeof(VisState));
        }
    }
    r = r ? r : dalloc(c, &s.d_count, sizeof(long long));
    if (c->p.adjoint && cap > 0) r = r ? r : dalloc(c, &s.dead, n);
    if (c->p.adjoint && c->tile > 0 && cap > 0) {
        r = r ? r : dalloc(c, &s.orig, n * sizeof(int));
        r = r ? r : dalloc(c, &s.orig_b, n * sizeof(int));
        r = r ? r : dalloc(c, &s.dead_b, n);
        r = r ? r : dalloc(c, &s.perm, n * sizeof(int));
    }
    if (r != PIC_OK) {
        free_species(s);
        return r;
    }
    cudaMemsetAsync(s.d_count, 0, sizeof(long long), c->stream);
    if (s.dead) cudaMemsetAsync(s.dead, 0, n, c->stream);
    if (s.vs) cudaMemsetAsync(s.vs, 0, sizeof(VisState), c->stream);
    return PIC_OK;
}

int ensure_stage(pic_ctx *c, size_t bytes) {
    if (c->stage_bytes >= bytes) return PIC_OK;
    if (c->d_stage) cudaFree(c->d_stage);
    c->d_stage = nullptr;
    c->stage_bytes = 0;
    int r = dalloc(c, (char **)&c->d_stage, bytes);
    if (r == PIC_OK) c->stage_bytes = bytes;
    return r;
}

int ensure_lists(pic_ctx *c, int64_t n) {
    if (c->list_cap >= 2 * n) return PIC_OK;
    if (c->d_list) cudaFree(c->d_list);
    c->d_list = nullptr;
    c->list_cap = 0;
    int r = dalloc(c, &c->d_list, (size_t)(2 * n) * sizeof(int));
    if (r == PIC_OK) c->list_cap = 2 * n;
    return r;
}

const int64_t kChunk = 1 << 20;  // particle records staged per copy
const int64_t kPinRecords = 1 << 18;   // records per pinned host staging buffer (37.7 MB)

// the two pinned staging buffers, at least min(n, kPinRecords) records
// each, and their events (allocated on first use, grown when needed)
int ensure_pinned(pic_ctx *c, int64_t n) {
    const int64_t want = n < kPinRecords ? (n > 0 ? n : 1) : kPinRecords;
    if (c->pin_records < want) {
        for (int b = 0; b < 2; ++b) {
            if (c->h_pin[b]) {
                if (c->pin_ev[b]) cudaEventSynchronize(c->pin_ev[b]);
                cudaFreeHost(c->h_pin[b]);
                c->h_pin[b] = nullptr;
            }
        }
        c->pin_records = 0;
        for (int b = 0; b < 2; ++b) {
            cudaError_t e = cudaHostAlloc(&c->h_pin[b], (size_t)want * 144, cudaHostAllocDefault);
            if (e != cudaSuccess) {
                c->h_pin[b] = nullptr;
                return fail(c, PIC_ENOMEM, std::string("cudaHostAlloc: ") + cudaGetErrorString(e));
            }
        }
        c->pin_records = want;
    }
    for (int b = 0; b < 2; ++b) {
        if (!c->pin_ev[b]) {
            cudaError_t e = cudaEventCreateWithFlags(&c->pin_ev[b], cudaEventDisableTiming);
            if (e != cudaSuccess) {
                c->pin_ev[b] = nullptr;
                return fail(c, PIC_ECUDA, std::string("cudaEventCreate: ") + cudaGetErrorString(e));
            }
        }
    }
    return PIC_OK;
}

// memcpy of a large block split over the host's cores.  Host copies into
// and out of the pinned staging buffers run at several times one core's
// rate; the worker threads live for the whole process (a copy of one 38 MB
// chunk is too short to start threads for it).
namespace {
class CopyPool {
  public:
    static CopyPool &get() {
        static CopyPool pool;
        return pool;
    }
    void copy(void *dst, const void *src, size_t bytes) {
        const int np = bytes >= (4u << 20) ? nparts_ : 1;
        if (np <= 1 || workers_.empty()) {
            std::memcpy(dst, src, bytes);
            return;
        }
        std::lock_guard<std::mutex> one_job(job_);   // callers on several host threads take turns
        std::unique_lock<std::mutex> lk(m_);
        dst_ = (char *)dst;
        src_ = (const char *)src;
        bytes_ = bytes;
        part_ = ((bytes + np - 1) / np + 63) & ~(size_t)63;
        nparts_job_ = np;
        next_.store(0);
        left_ = np;
        ++gen_;
        lk.unlock();
        cv_.notify_all();
        work();
        lk.lock();
        done_.wait(lk, [&] { return left_ == 0; });
    }
    ~CopyPool() {
        {
            std::lock_guard<std::mutex> lk(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto &t : workers_) t.join();
    }

  private:
    CopyPool() {
        const unsigned hw = std::thread::hardware_concurrency();
        nparts_ = (int)std::min(16u, hw > 0 ? hw : 1u);
        for (int t = 1; t < nparts_; ++t) workers_.emplace_back([this] { loop(); });
    }
    // take parts of the current job until none is left
    void work() {
        int k;
        while ((k = next_.fetch_add(1)) < nparts_job_) {
            const size_t lo = std::min(bytes_, part_ * k), hi = std::min(bytes_, part_ * (k + 1));
            if (hi > lo) std::memcpy(dst_ + lo, src_ + lo, hi - lo);
            std::lock_guard<std::mutex> lk(m_);
            if (--left_ == 0) done_.notify_one();
        }
    }
    void loop() {
        unsigned long long seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(m_);
                cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
            }
            work();
        }
    }
    std::vector<std::thread> workers_;
    std::mutex job_, m_;
    std::condition_variable cv_, done_;
    char *dst_ = nullptr;
    const char *src_ = nullptr;
    size_t bytes_ = 0, part_ = 0;
    int nparts_ = 1, nparts_job_ = 0, left_ = 0;
    std::atomic<int> next_{0};
    unsigned long long gen_ = 0;
    bool stop_ = false;
};
}  // namespace

void par_memcpy(void *dst, const void *src, size_t bytes) { CopyPool::get().copy(dst, src, bytes); }

// A host <-> device copy of `bytes` through the two pinned staging buffers:
// the host copy of one chunk overlaps the DMA of the other (a copy from or
// to pageable memory runs at a few GB/s).
static int staged_h2d(pic_ctx *c, void *dev, const void *host, size_t bytes) {
    int r = ensure_pinned(c, kPinRecords);
    if (r) return r;
    const size_t chunk = (size_t)kPinRecords * 144;
    for (size_t off = 0, i = 0; off < bytes; off += chunk, ++i) {
        const size_t m = std::min(chunk, bytes - off);
        const int b = (int)(i & 1);
        CK(cudaEventSynchronize(c->pin_ev[b]));
        par_memcpy(c->h_pin[b], (const char *)host + off, m);
        CK(cudaMemcpyAsync((char *)dev + off, c->h_pin[b], m, cudaMemcpyHostToDevice, c->stream));
        CK(cudaEventRecord(c->pin_ev[b], c->stream));
    }
    return PIC_OK;
}

static int staged_d2h(pic_ctx *c, void *host, const void *dev, size_t bytes) {
    int r = ensure_pinned(c, kPinRecords);
    if (r) return r;
    const size_t chunk = (size_t)kPinRecords * 144;
    const size_t nch = (bytes + chunk - 1) / chunk;
    auto enqueue = [&](size_t i) -> cudaError_t {
        const size_t off = i * chunk, m = std::min(chunk, bytes - off);
        cudaError_t e = cudaMemcpyAsync(c->h_pin[i & 1], (const char *)dev + off, m, cudaMemcpyDeviceToHost, c->stream);
        return e != cudaSuccess ? e : cudaEventRecord(c->pin_ev[i & 1], c->stream);
    };
    if (nch) CK(enqueue(0));
    for (size_t i = 0; i < nch; ++i) {
        if (i + 1 < nch) CK(enqueue(i + 1));
        CK(cudaEventSynchronize(c->pin_ev[i & 1]));
        const size_t off = i * chunk;
        par_memcpy((char *)host + off, c->h_pin[i & 1], std::min(chunk, bytes - off));
    }
    return PIC_OK;
}

int array_info(const pic_ctx *c, int which, void **dptr, long long *n) {
    if (which < 0 || which >= PIC_NARRAYS) return PIC_EINVAL;
    if (which < 6) {
        *dptr = c->field[which];
        *n = c->g.fsz;
    } else {
        *dptr = c->ring[which - 6];
        *n = c->g.rsz;
    }
    return PIC_OK;
}

int sync_status(pic_ctx *c) {
    CK(cudaStreamSynchronize(c->stream));
    unsigned st = 0;
    CK(cudaMemcpy(&st, c->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost));
    for (int k = 0; k < 2; ++k)
        if (c->sp[k].d_count) {
            long long n = 0;
            CK(cudaMemcpy(&n, c->sp[k].d_count, sizeof(long long), cudaMemcpyDeviceToHost));
            c->sp[k].n_host = n;
        }
    if (st) {
        CK(cudaMemset(c->d_status, 0, sizeof(unsigned)));
        if (st & ST_NAN) return fail(c, PIC_ENAN, "non-finite particle momentum or position (particle skipped)");
        if (st & ST_OOB) return fail(c, PIC_EOOB, "particle stencil outside the field buffers (particle skipped)");
        if (st & ST_CFL) return fail(c, PIC_EOOB, "particle moved a cell or more in one step (particle skipped)");
        if (st & ST_RANGE) return fail(c, PIC_ERANGE, "g_factor argument outside the g table");
        if (st & ST_OVERFLOW) return fail(c, PIC_EOVERFLOW, "particle bin overflow");
        if (st & ST_TIMEOUT) return fail(c, PIC_ETIMEOUT, "device wait gave up");
    }
    return PIC_OK;
}

// Species set-up shared by pic_upload_particles and the device generators:
// capacity for n particles, cleared sort / removal state, and the staging
// buffer for one chunk of records.
int begin_fill(pic_ctx *c, int kind, int64_t n, bool spin_nonzero, double wmax) {
    Species &s = c->sp[kind];
    bool want_spin = c->p.spin && c->p.mass[kind] == 1.0;
    if (n > s.cap || (want_spin && !s.a.sx)) {
        int r = alloc_species(c, kind, n > c->p.capacity[kind] ? n : c->p.capacity[kind], want_spin);
        if (r) return r;
    }
    s.cur = 0;
    s.sorted = false;
    s.perm_fresh = false;
    if (s.dead) cudaMemsetAsync(s.dead, 0, (size_t)s.cap, c->stream);
    s.spin_nonzero = spin_nonzero;
    s.max_abs_w = wmax;
    return ensure_stage(c, (size_t)(n < kChunk ? n : kChunk) * 144);
}

// the count of a filled species, and the compaction lists sized for it
int end_fill(pic_ctx *c, int kind, int64_t n, const char *what) {
    Species &s = c->sp[kind];
    long long cnt = n;
    CK(cudaMemcpyAsync(s.d_count, &cnt, sizeof(long long), cudaMemcpyHostToDevice, c->stream));
    if (s.orig && n > 0) launch_iota(c, s.orig, n);   // upload index of every particle
    CK(cudaStreamSynchronize(c->stream));
    s.n_host = n;
    int r = ensure_lists(c, n > c->sp[1 - kind].cap ? n : c->sp[1 - kind].cap);
    if (r) return r;
    return launch_check(c, what);
}

// piecewise-linear density in physical x through the knots, the end values
// beyond them
double xprofile(const PicDensity &d, double x) {
    const int m = d.nknots;
    if (x <= d.knot_x[0]) return d.knot_v[0];
    if (x >= d.knot_x[m - 1]) return d.knot_v[m - 1];
    int k = 1;
    while (d.knot_x[k] < x) ++k;
    const double x0 = d.knot_x[k - 1], x1 = d.knot_x[k];
    return d.knot_v[k - 1] + (d.knot_v[k] - d.knot_v[k - 1]) * ((x - x0) / (x1 - x0));
}

}  // namespace

// ---------------------------------------------------------------------------
namespace pic {

void prof_begin(pic_ctx *c, const char *name) {
    if (!c->prof) return;
    ProfEntry e{name, nullptr, nullptr};
    cudaEventCreate(&e.a);
    cudaEventCreate(&e.b);
    cudaEventRecord(e.a, c->stream);
    c->prof_events.push_back(e);
}

void prof_end(pic_ctx *c) {
    if (!c->prof || c->prof_events.empty()) return;
    cudaEventRecord(c->prof_events.back().b, c->stream);
}

}  // namespace pic

static void prof_collect(pic_ctx *c) {
    if (c->prof_events.empty()) return;
    cudaStreamSynchronize(c->stream);
    for (auto &e : c->prof_events) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e.a, e.b);
        bool found = false;
        for (auto &acc : c->prof_acc)
            if (std::strcmp(acc.first, e.name) == 0) {
                acc.second.first += ms;
                acc.second.second += 1;
                found = true;
            }
        if (!found) c->prof_acc.push_back({e.name, {ms, 1}});
        cudaEventDestroy(e.a);
        cudaEventDestroy(e.b);
    }
    c->prof_events.clear();
}

// ---------------------------------------------------------------------------
extern "C" {

void pic_default_params(PicParams *p) {
    std::memset(p, 0, sizeof(*p));
    p->local_xcells = p->local_ycells = p->local_zcells = 32;
    p->mem = 4;
    p->rank_period[0] = p->rank_period[1] = p->rank_period[2] = 1;
    p->laser_polarization = 1;
    p->Pi = 3.1415926536;
    p->omega = 1.0;
    p->l0 = 2.0 * p->Pi;
    p->Lx = 32.0;
    p->dx = p->dy = p->dz = 1.0;
    p->dt = 0.95 / std::sqrt(3.0);
    p->dt_half = p->dt / 2.0;
    p->laser_pulse_duration = 10.0 * 2.0 * p->Pi;
    p->waist = 3.0 * 2.0 * p->Pi;
    p->E_schwinger = 4.1215e5;
    p->charge[0] = -1.0;
    p->mass[0] = 1.0;
    p->charge[1] = 1.0;
    p->mass[1] = 1836.0;
    p->precision = 64;
    p->spin = 1;
    p->deposit_rho = 1;
}

int pic_create(const PicParams *pp, int device, pic_ctx **out) {
    if (!pp || !out) return PIC_EINVAL;
    *out = nullptr;
    pic_ctx *c = new pic_ctx();
    c->p = *pp;
    const PicParams &p = c->p;
    auto bad = [&](const std::string &m) {
        std::string msg = "pic_create: " + m;
        std::fprintf(stderr, "%s\n", msg.c_str());
        delete c;
        return PIC_EINVAL;
    };
    if (p.mem != 2 && p.mem != 4) return bad("mem must be 2 (2nd-order shape) or 4 (4th-order shape)");
    if (p.precision != 32 && p.precision != 64) return bad("precision must be 32 or 64");
    const int n[3] = {p.local_xcells, p.local_ycells, p.local_zcells};
    const double d[3] = {p.dx, p.dy, p.dz};
    for (int k = 0; k < 3; ++k) {
        // periodic axes: the ghost slabs of both sides must not overlap
        // (the reference halo exchange needs the same); absorbing axes: the
        // x-max boundary column local_xcells+1 must not meet the x-min one
        if (p.rank_period[k] && n[k] < 2 * p.mem + 2) return bad("a periodic axis needs at least 2*mem+2 cells");
        if (!p.rank_period[k] && n[k] < p.mem) return bad("an absorbing axis needs at least mem cells");
        if (!(d[k] > 0.0)) return bad("cell sizes must be positive");
        if (!(p.dt > 0.0) || !(p.dt < d[k])) return bad("dt must satisfy 0 < dt < min(dx,dy,dz) (a particle moves less than a cell per step)");
    }
    if (!(p.mass[0] > 0.0) || !(p.mass[1] > 0.0)) return bad("species masses must be positive");
    if (p.absorbing != 0 && p.absorbing != 1) return bad("absorbing must be 0 or 1");
    for (int k = 0; k < 3; ++k)
        if (n[k] < 1 || n[k] > (1 << 20)) return bad("cell counts must lie in [1, 2^20]");
    c->g = make_geom(p);
    if (c->g.rsz >= (1ll << 31)) return bad("grid too large for 32-bit buffer indexing");
    c->fp32 = p.precision == 32;
    c->order = p.mem == 2 ? 2 : 4;
    c->cp.bx = bits_for(n[0]);
    c->cp.by = bits_for(n[1]);
    c->cp.bz = bits_for(n[2]);
    c->cp.mx = (1u << c->cp.bx) - 1;
    c->cp.my = (1u << c->cp.by) - 1;
    if (c->fp32 && c->cp.bx + c->cp.by + c->cp.bz > 31) return bad("grid too large for the packed int32 cell index");
    // tiling: 0 -> default edge of 4 cells, < 0 -> global-memory kernel only
    c->tile = p.tile == 0 ? 4 : (p.tile < 0 ? 0 : p.tile);
    if (p.adjoint) {
        // removal only marks particles dead (no compaction); the counting
        // sort still runs, recording each permutation for the reverse sweep
        if (p.rank_period[0] || p.rank_period[1] || p.rank_period[2])
            return bad("the adjoint supports absorbing faces only");
        if (p.absorbing) return bad("the adjoint has no transpose of the absorbing-faces extension");
    }
    // Between full sorts the visitor lists keep every particle on the
    // shared-memory path, but the kernel slows as the order decays (the
    // thermal plasma: 10.8 ms per launch 4 pushes after a sort, 12.4 ms 64
    // pushes after); a sort every 4 pushes measured fastest overall.
    // Adjoint contexts have no visitor lists: they sort before every push,
    // so that no particle leaves the shared-memory path of the forward or
    // of the reverse sweep (each sort's permutation goes on the tape).
    c->sort_interval = p.sort_interval > 0 ? p.sort_interval : (p.adjoint ? 1 : 4);
    if (c->tile > 0) {
        for (int d = 0; d < 3; ++d) c->ntile[d] = (n[d] + c->tile - 1) / c->tile;
        c->nkeys = (long long)c->ntile[0] * c->ntile[1] * c->ntile[2] * kOctants * c->tile * c->tile * c->tile;
        if (c->nkeys >= (1ll << 31)) return bad("too many sort keys");
        if (tile_smem_bytes(c) > 227 * 1024) return bad("tile too large for shared memory");
    }
    c->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        std::fprintf(stderr, "pic_create: cudaSetDevice(%d): %s\n", device, cudaGetErrorString(e));
        delete c;
        return PIC_ECUDA;
    }
    e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete c;
        return PIC_ECUDA;
    }
    const size_t rs = real_size(c);
    int r = PIC_OK;
    for (int k = 0; k < 6 && r == PIC_OK; ++k) r = dalloc(c, (char **)&c->field[k], (size_t)c->g.fsz * rs);
    for (int k = 0; k < 5 && r == PIC_OK; ++k) r = dalloc(c, (char **)&c->ring[k], (size_t)c->g.rsz * rs);
    r = r ? r : dalloc(c, &c->d_status, sizeof(unsigned));
    r = r ? r : dalloc(c, &c->d_scratch_ll, 8 * sizeof(long long));
    r = r ? r : dalloc(c, &c->d_diag, PIC_NDIAG * sizeof(double));
    if (c->tile > 0) {
        r = r ? r : dalloc(c, &c->d_hist, (size_t)(c->nkeys + 1) * sizeof(unsigned));
        r = r ? r : dalloc(c, &c->d_blocksums, (size_t)(c->nkeys / 4096 + 2) * sizeof(unsigned));
        r = r ? r : dalloc(c, &c->d_nstrag, 2 * sizeof(unsigned long long));
    }
    if (r != PIC_OK) {
        std::fprintf(stderr, "pic_create: %s\n", c->err.c_str());
        pic_destroy(c);
        return r;
    }
    for (int k = 0; k < 6; ++k) cudaMemsetAsync(c->field[k], 0, (size_t)c->g.fsz * rs, c->stream);
    for (int k = 0; k < 5; ++k) cudaMemsetAsync(c->ring[k], 0, (size_t)c->g.rsz * rs, c->stream);
    cudaMemsetAsync(c->d_status, 0, sizeof(unsigned), c->stream);
    for (int k = 0; k < 2; ++k) {
        r = alloc_species(c, k, pp->capacity[k] > 0 ? pp->capacity[k] : 0, p.spin && p.mass[k] == 1.0);
        if (r != PIC_OK) {
            pic_destroy(c);
            return r;
        }
    }
    e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        pic_destroy(c);
        return PIC_ECUDA;
    }
    *out = c;
    return PIC_OK;
}

int pic_destroy(pic_ctx *c) {
    if (!c) return PIC_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    pic_adjoint_release(c);
    for (auto &e : c->prof_events) {
        cudaEventDestroy(e.a);
        cudaEventDestroy(e.b);
    }
    for (void *p : c->field)
        if (p) cudaFree(p);
    for (void *p : c->ring)
        if (p) cudaFree(p);
    for (auto &s : c->sp) free_species(s);
    for (int b = 0; b < 2; ++b) {
        if (c->h_pin[b]) cudaFreeHost(c->h_pin[b]);
        if (c->pin_ev[b]) cudaEventDestroy(c->pin_ev[b]);
    }
    void *ptrs[] = {c->d_status, c->d_gtab, c->d_profile, c->d_stage, c->d_scratch_ll, c->d_list, c->d_diag,
                    c->d_hist, c->d_blocksums, c->d_nstrag};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return PIC_OK;
}

const char *pic_last_error(const pic_ctx *c) { return c ? c->err.c_str() : "no context"; }

int pic_array_len(const pic_ctx *c, int which, int64_t *n) {
    if (!c || !n) return PIC_EINVAL;
    void *d;
    long long len;
    if (array_info(c, which, &d, &len) != PIC_OK) return PIC_EINVAL;
    *n = len;
    return PIC_OK;
}

int pic_upload_array(pic_ctx *c, int which, const double *host) {
    if (!c || !host) return PIC_EINVAL;
    cudaSetDevice(c->device);
    void *d;
    long long n;
    if (array_info(c, which, &d, &n) != PIC_OK) return fail(c, PIC_EINVAL, "bad array id");
    if (!c->fp32) {
        int r = staged_h2d(c, d, host, (size_t)n * sizeof(double));
        if (r) return r;
    } else {
        int r = ensure_stage(c, (size_t)n * sizeof(double));
        r = r ? r : staged_h2d(c, c->d_stage, host, (size_t)n * sizeof(double));
        if (r) return r;
        launch_convert_array(c, d, c->d_stage, n, 1);
    }
    CK(cudaStreamSynchronize(c->stream));
    return launch_check(c, "pic_upload_array");
}

int pic_download_array(pic_ctx *c, int which, double *host) {
    if (!c || !host) return PIC_EINVAL;
    cudaSetDevice(c->device);
    void *d;
    long long n;
    if (array_info(c, which, &d, &n) != PIC_OK) return fail(c, PIC_EINVAL, "bad array id");
    int st = sync_status(c);
    if (!c->fp32) {
        int r = staged_d2h(c, host, d, (size_t)n * sizeof(double));
        if (r) return r;
    } else {
        int r = ensure_stage(c, (size_t)n * sizeof(double));
        if (r) return r;
        launch_convert_array(c, c->d_stage, d, n, 0);
        r = staged_d2h(c, host, c->d_stage, (size_t)n * sizeof(double));
        if (r) return r;
    }
    CK(cudaStreamSynchronize(c->stream));
    return st;
}

int pic_upload_particles(pic_ctx *c, int kind, const void *records, int64_t n) {
    if (!c || kind < 0 || kind > 1 || n < 0 || (n > 0 && !records)) return PIC_EINVAL;
    cudaSetDevice(c->device);
    const char *rec = (const char *)records;
    int r = begin_fill(c, kind, n, false, 0.0);
    if (r) return r;
    r = ensure_pinned(c, n);
    if (r) return r;
    // the records' checks (charge and mass equal to the species', finite
    // weights, any non-zero spin, largest |weight|) run in the conversion
    // kernel: two words of device scratch
    unsigned long long *chk = (unsigned long long *)(c->d_scratch_ll + 4);
    CK(cudaMemsetAsync(chk, 0, 2 * sizeof(unsigned long long), c->stream));
    // pipeline: the host copy of chunk i into pinned buffer i % 2 overlaps
    // the DMA and conversion of chunk i - 1
    int64_t i = 0;
    for (int64_t off = 0; off < n; off += kPinRecords, ++i) {
        const int64_t m = n - off < kPinRecords ? n - off : kPinRecords;
        const int b = (int)(i & 1);
        CK(cudaEventSynchronize(c->pin_ev[b]));
        par_memcpy(c->h_pin[b], rec + 144 * off, (size_t)m * 144);
        CK(cudaMemcpyAsync(c->d_stage, c->h_pin[b], (size_t)m * 144, cudaMemcpyHostToDevice, c->stream));
        launch_upload_particles(c, kind, c->d_stage, m, off, chk);
        CK(cudaEventRecord(c->pin_ev[b], c->stream));
    }
    unsigned long long hc[2] = {0, 0};
    CK(cudaMemcpyAsync(hc, chk, sizeof(hc), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (hc[0] & 27ull) {
        // a bad record leaves the species empty
        r = end_fill(c, kind, 0, "pic_upload_particles");
        if (r) return r;
        if (hc[0] & 1ull) return fail(c, PIC_EINVAL, "particle record charge/mass differs from the species parameters");
        if (hc[0] & 2ull) return fail(c, PIC_EINVAL, "non-finite particle weight");
        if (hc[0] & 8ull) return fail(c, PIC_ENAN, "non-finite particle position or momentum");
        return fail(c, PIC_EOOB, "particle position beyond the cells an FP32 context can store (-1 .. n on an "
                                 "absorbing axis)");
    }
    Species &s = c->sp[kind];
    s.spin_nonzero = (hc[0] & 4ull) != 0;
    std::memcpy(&s.max_abs_w, &hc[1], sizeof(double));
    return end_fill(c, kind, n, "pic_upload_particles");
}

int pic_initialize_particles(pic_ctx *c, int kind, const PicDensity *dens, int cell_per_particles,
                             const double *initial_p, const double *initial_s) {
    if (!c || kind < 0 || kind > 1 || !dens || cell_per_particles < 1 || !initial_p || !initial_s) return PIC_EINVAL;
    cudaSetDevice(c->device);
    const PicParams &p = c->p;
    const int n[3] = {p.local_xcells, p.local_ycells, p.local_zcells};
    const double h[3] = {p.dx, p.dy, p.dz};
    if (dens->kind == PIC_DENSITY_XPROFILE) {
        if (dens->nknots < 1 || !dens->knot_x || !dens->knot_v) return fail(c, PIC_EINVAL, "x profile needs knots");
        for (int k = 1; k < dens->nknots; ++k)
            if (!(dens->knot_x[k] > dens->knot_x[k - 1])) return fail(c, PIC_EINVAL, "x profile knots must ascend");
    } else if (dens->kind != PIC_DENSITY_UNIFORM && dens->kind != PIC_DENSITY_BOX) {
        return fail(c, PIC_EINVAL, "unknown density profile kind");
    }
    // lattice of src/particle.cpp:58-63 (one rank: xst = 0, xend = n)
    std::vector<double> coord[3], wx;
    for (int d = 0; d < 3; ++d) {
        const int num = (int)(n[d] * std::cbrt(cell_per_particles));
        const double xst = 0.0, xend = (double)n[d];
        const double norm = (xend - xst) / num;
        for (int i = 0; i < num; ++i) {
            const double pos = xst + (i) * norm + norm / 2.0;   // particle.cpp:73-75
            const double phys = pos * h[d];
            bool keep = true;
            if (dens->kind == PIC_DENSITY_BOX) keep = phys > dens->lo[d] && phys <= dens->hi[d];
            if (dens->kind == PIC_DENSITY_XPROFILE && d == 0) {
                const double v = xprofile(*dens, phys) / cell_per_particles;
                keep = v > 0.0;
                if (keep) wx.push_back(v);
            }
            if (keep) coord[d].push_back(pos);
        }
    }
    double wconst = 0.0;
    if (dens->kind != PIC_DENSITY_XPROFILE) {
        wconst = dens->value / cell_per_particles;
        if (!(wconst > 0.0))
            for (auto &v : coord) v.clear();
    }
    if (!std::isfinite(wconst)) return fail(c, PIC_EINVAL, "non-finite density");
    for (double v : wx)
        if (!std::isfinite(v)) return fail(c, PIC_EINVAL, "non-finite density");
    const int64_t total = (int64_t)coord[0].size() * (int64_t)coord[1].size() * (int64_t)coord[2].size();
    const int64_t capacity = (int64_t)n[0] * n[1] * n[2] * cell_per_particles;
    if (total > capacity || total >= (1ll << 31)) return fail(c, PIC_EINVAL, "too many particles for int ids");
    double wmax = std::fabs(wconst);
    for (double v : wx) wmax = std::max(wmax, std::fabs(v));
    const bool spin_nonzero = initial_s[0] != 0.0 || initial_s[1] != 0.0 || initial_s[2] != 0.0;
    int r = begin_fill(c, kind, total, spin_nonzero, wmax);
    if (r) return r;
    // per-axis tables next to the records in one device buffer
    const size_t tab = coord[0].size() + coord[1].size() + coord[2].size() + wx.size();
    double *d_tab = nullptr;
    r = dalloc(c, &d_tab, std::max<size_t>(tab, 1) * sizeof(double));
    if (r) return r;
    size_t o = 0;
    const double *dptr[4];
    std::vector<double> *src[4] = {&coord[0], &coord[1], &coord[2], &wx};
    for (int k = 0; k < 4; ++k) {
        dptr[k] = d_tab + o;
        if (!src[k]->empty())
            cudaMemcpyAsync(d_tab + o, src[k]->data(), src[k]->size() * sizeof(double), cudaMemcpyHostToDevice,
                            c->stream);
        o += src[k]->size();
    }
    LatticeArgs a{};
    a.ax = dptr[0]; a.ay = dptr[1]; a.az = dptr[2];
    a.wx = wx.empty() ? nullptr : dptr[3];
    a.wconst = wconst;
    a.nvx = (long long)coord[0].size();
    a.nvy = (long long)coord[1].size();
    for (int d = 0; d < 3; ++d) { a.p[d] = initial_p[d]; a.s[d] = initial_s[d]; }
    a.gamma = std::sqrt(1 + (initial_p[0] * initial_p[0] + initial_p[1] * initial_p[1] + initial_p[2] * initial_p[2]));
    a.charge = p.charge[kind];
    a.mass = p.mass[kind];
    a.rec = c->d_stage;
    cudaError_t e = cudaSuccess;
    for (int64_t off = 0; off < total && e == cudaSuccess; off += kChunk) {
        a.off = off;
        a.n = total - off < kChunk ? total - off : kChunk;
        launch_lattice_records(c, a);
        launch_upload_particles(c, kind, c->d_stage, a.n, off);
        e = cudaStreamSynchronize(c->stream);
    }
    cudaFree(d_tab);
    CK(e);
    return end_fill(c, kind, total, "pic_initialize_particles");
}

int pic_generate_thermal(pic_ctx *c, int kind, int ppc, double density, double u_th, uint64_t seed) {
    if (!c || kind < 0 || kind > 1 || ppc < 1 || !(density > 0.0) || !(u_th >= 0.0) || !std::isfinite(u_th))
        return PIC_EINVAL;
    cudaSetDevice(c->device);
    const PicParams &p = c->p;
    const int64_t total = (int64_t)p.local_xcells * p.local_ycells * p.local_zcells * ppc;
    if (total >= (1ll << 31)) return fail(c, PIC_EINVAL, "too many particles for int ids");
    const double w = density / ppc;
    int r = begin_fill(c, kind, total, false, w);
    if (r) return r;
    ThermalArgs a{};
    a.nx = p.local_xcells;
    a.ny = p.local_ycells;
    a.ppc = ppc;
    a.key0 = (unsigned)seed;
    a.key1 = (unsigned)(seed >> 32) ^ (0x9E3779B9u * (unsigned)(kind + 1));
    a.u_th = u_th;
    a.weight = w;
    a.charge = p.charge[kind];
    a.mass = p.mass[kind];
    a.rec = c->d_stage;
    for (int64_t off = 0; off < total; off += kChunk) {
        a.off = off;
        a.n = total - off < kChunk ? total - off : kChunk;
        launch_thermal_records(c, a);
        launch_upload_particles(c, kind, c->d_stage, a.n, off);
    }
    CK(cudaStreamSynchronize(c->stream));
    return end_fill(c, kind, total, "pic_generate_thermal");
}

int pic_download_particles(pic_ctx *c, int kind, void *records, int64_t cap, int64_t *n) {
    if (!c || kind < 0 || kind > 1 || !n) return PIC_EINVAL;
    cudaSetDevice(c->device);
    int st = sync_status(c);
    if (st == PIC_ECUDA) return st;
    Species &s = c->sp[kind];
    int64_t cnt = s.n_host;
    *n = cnt;
    if (cnt > cap) return fail(c, PIC_EINVAL, "download buffer too small");
    if (cnt == 0) return st;
    int r = ensure_stage(c, (size_t)(cnt < kPinRecords ? cnt : kPinRecords) * 144);
    r = r ? r : ensure_pinned(c, cnt);
    if (r) return r;
    char *rec = (char *)records;
    // conversion + DMA of chunk i + 1 into pinned buffer (i + 1) % 2 overlap
    // the host copy of chunk i out of the other buffer
    const int64_t nch = (cnt + kPinRecords - 1) / kPinRecords;
    auto enqueue = [&](int64_t i) -> cudaError_t {
        const int64_t off = i * kPinRecords, m = cnt - off < kPinRecords ? cnt - off : kPinRecords;
        launch_download_particles(c, kind, c->d_stage, m, off);
        cudaError_t e = cudaMemcpyAsync(c->h_pin[i & 1], c->d_stage, (size_t)m * 144, cudaMemcpyDeviceToHost,
                                        c->stream);
        return e != cudaSuccess ? e : cudaEventRecord(c->pin_ev[i & 1], c->stream);
    };
    CK(enqueue(0));
    for (int64_t i = 0; i < nch; ++i) {
        if (i + 1 < nch) CK(enqueue(i + 1));
        CK(cudaEventSynchronize(c->pin_ev[i & 1]));
        const int64_t off = i * kPinRecords, m = cnt - off < kPinRecords ? cnt - off : kPinRecords;
        par_memcpy(rec + 144 * off, c->h_pin[i & 1], (size_t)m * 144);
    }
    r = launch_check(c, "pic_download_particles");
    return r ? r : st;
}

int pic_num_particles(pic_ctx *c, int kind, int64_t *n) {
    if (!c || kind < 0 || kind > 1 || !n) return PIC_EINVAL;
    int st = sync_status(c);
    *n = c->sp[kind].n_host;
    return st;
}

int pic_set_g_table(pic_ctx *c, const double *g, int n) {
    if (!c || !g || n <= 0) return PIC_EINVAL;
    cudaSetDevice(c->device);
    if (c->d_gtab) cudaFree(c->d_gtab);
    c->d_gtab = nullptr;
    int r = dalloc(c, &c->d_gtab, (size_t)n * sizeof(double));
    if (r) return r;
    CK(cudaMemcpy(c->d_gtab, g, (size_t)n * sizeof(double), cudaMemcpyHostToDevice));
    c->gtab_n = n;
    return PIC_OK;
}

int pic_set_laser_profile(pic_ctx *c, const double *coef, int pn) {
    if (!c || !coef || pn < 2) return PIC_EINVAL;
    cudaSetDevice(c->device);
    if (c->d_profile && c->profile_n != pn) {
        cudaFree(c->d_profile);
        c->d_profile = nullptr;
    }
    if (!c->d_profile) {
        int r = dalloc(c, &c->d_profile, (size_t)pn * pn * sizeof(double));
        if (r) return r;
    }
    CK(cudaMemcpyAsync(c->d_profile, coef, (size_t)pn * pn * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->profile_n = pn;
    return PIC_OK;
}

// ---- reference call surface ---------------------------------------------

int pic_radiating_boundary(pic_ctx *c, int is_left, int is_right, int step) {
    if (!c) return PIC_EINVAL;
    launch_radiating_boundary(c, is_left, is_right, step);
    return launch_check(c, "radiating_boundary");
}

int pic_update_fields_first(pic_ctx *c) {
    if (!c) return PIC_EINVAL;
    launch_update_e(c, c->p.dt_half);
    launch_update_b(c, c->p.dt_half);
    return launch_check(c, "update_fields_first");
}

int pic_update_fields_second(pic_ctx *c) {
    if (!c) return PIC_EINVAL;
    launch_update_b(c, c->p.dt_half);
    launch_update_e(c, c->p.dt_half);
    return launch_check(c, "update_fields_second");
}

int pic_clear_currents(pic_ctx *c) {
    if (!c) return PIC_EINVAL;
    prof_begin(c, "clear_currents");
    const int n = c->rho_skip ? 3 : 5;
    for (int k = 0; k < n; ++k) CK(cudaMemsetAsync(c->ring[k], 0, (size_t)c->g.rsz * real_size(c), c->stream));
    prof_end(c);
    return PIC_OK;
}

int pic_update_particles(pic_ctx *c, int kind) {
    if (!c || kind < 0 || kind > 1) return PIC_EINVAL;
    if (c->sp[kind].n_host > 0) {
        if (c->tile > 0) launch_tile_push(c, 1 << kind);
        else launch_push(c, kind);
    }
    return launch_check(c, "update_particles");
}

// both species in one launch when tiled (the two pushes only read the
// fields and add into J, so fusing them changes nothing but the order of
// the additions)
static int push_both(pic_ctx *c) {
    if (c->tile > 0) {
        if (c->sp[0].n_host > 0 || c->sp[1].n_host > 0) launch_tile_push(c, 3);
        return launch_check(c, "update_particles");
    }
    int r = pic_update_particles(c, 0);
    return r ? r : pic_update_particles(c, 1);
}

int pic_exchange_particles(pic_ctx *c, int kind) {
    if (!c || kind < 0 || kind > 1) return PIC_EINVAL;
    if (c->sp[kind].n_host > 0) launch_remove(c, kind);
    return launch_check(c, "exchange_particles");
}

int pic_exchange_currents(pic_ctx *c) {
    if (!c) return PIC_EINVAL;
    launch_fold_currents(c, c->rho_skip ? 7u : 31u);
    return launch_check(c, "exchange_currents");
}

int pic_update_fields_full(pic_ctx *c) {
    if (!c) return PIC_EINVAL;
    launch_update_e(c, c->p.dt);
    launch_update_b(c, c->p.dt);
    return launch_check(c, "update_fields_full");
}

int pic_exchange_boundary(pic_ctx *c, int array) {
    if (!c) return PIC_EINVAL;
    if (array < PIC_EX || array > PIC_BZ) return fail(c, PIC_EINVAL, "exchange_boundary: not a field array");
    launch_ghost_fill_one(c, array);
    return launch_check(c, "exchange_boundary");
}

int pic_exchange_current(pic_ctx *c, int array) {
    if (!c) return PIC_EINVAL;
    if (array < PIC_JX || array > PIC_RHO1) return fail(c, PIC_EINVAL, "exchange_current: not a ring array");
    launch_fold_currents(c, 1u << (array - PIC_JX));
    return launch_check(c, "exchange_current");
}

int pic_filter_current(pic_ctx *c, int array) {
    if (!c) return PIC_EINVAL;
    if (array < PIC_JX || array > PIC_RHO1) return fail(c, PIC_EINVAL, "filter_current: not a ring array");
    int r = ensure_stage(c, (size_t)c->g.rsz * real_size(c));
    if (r) return r;
    for (int axis = 0; axis < 3; ++axis) launch_binomial_pass(c, array - PIC_JX, axis, c->d_stage);
    return launch_check(c, "filter_current");
}

int pic_binomial_filter_currents(pic_ctx *c) {
    int r = PIC_OK;
    for (int a = PIC_JX; a <= PIC_JZ && r == PIC_OK; ++a) r = pic_filter_current(c, a);
    return r;
}

int pic_deposit_particle(pic_ctx *c, int kind, const void *record) {
    if (!c || kind < 0 || kind > 1 || !record) return PIC_EINVAL;
    // 144-byte reference record: x, y, z at bytes 8..31, x_old.. at 32..55,
    // charge at 112, weight at 128
    const unsigned char *b = (const unsigned char *)record;
    double xn[3], xo[3], q, w;
    std::memcpy(xn, b + 8, sizeof xn);
    std::memcpy(xo, b + 32, sizeof xo);
    std::memcpy(&q, b + 112, sizeof q);
    std::memcpy(&w, b + 128, sizeof w);
    launch_deposit_one(c, kind, xo, xn, q * w);
    int r = launch_check(c, "deposit_particle");
    return r ? r : sync_status(c);
}

int pic_eval(pic_ctx *c, int what, const double *in, int nin, double *out, int nout) {
    static const int need_in[] = {1, 1, 1, 2, 4}, need_out[] = {3, 5, 1, 1, 1};
    if (!c || what < 0 || what > 4 || !in || !out) return PIC_EINVAL;
    if (nin < need_in[what] || nout < need_out[what]) return fail(c, PIC_EINVAL, "pic_eval: argument count");
    if (what == PIC_EVAL_G_FACTOR && !c->d_gtab) return fail(c, PIC_EINVAL, "pic_eval: no g table loaded");
    double a[4] = {0, 0, 0, 0};
    for (int i = 0; i < need_in[what]; ++i) a[i] = in[i];
    launch_eval(c, what, a, c->d_diag);
    int r = launch_check(c, "eval");
    if (r) return r;
    CK(cudaMemcpyAsync(out, c->d_diag, (size_t)need_out[what] * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    return sync_status(c);
}

int pic_initial_push(pic_ctx *c) {
    if (!c) return PIC_EINVAL;
    int r;
    launch_sort_due(c, 3);   // before the tape records the particles: the push runs in sorted order
    adjoint_record_hook(c);
    if ((r = push_both(c))) return r;
    if ((r = pic_exchange_particles(c, 0))) return r;
    return pic_exchange_particles(c, 1);
}

// One iteration of run_main_time_loop.  rho (a diagnostic: it never feeds
// the fields) is cleared, deposited and folded only when the step's rho can
// be observed, i.e. on the last step of a pic_run_steps call.
static int run_one_step(pic_ctx *c, bool rho_observed) {
    c->step += 1;
    c->rho_skip = !rho_observed && !c->p.adjoint;
    int r;
    if ((r = pic_radiating_boundary(c, 1, 0, c->step))) return r;
    if ((r = pic_update_fields_first(c))) return r;
    if ((r = pic_clear_currents(c))) return r;
    launch_sort_due(c, 3);
    adjoint_record_hook(c);
    if ((r = push_both(c))) return r;
    if ((r = pic_exchange_particles(c, 0))) return r;
    if ((r = pic_exchange_particles(c, 1))) return r;
    if ((r = pic_exchange_currents(c))) return r;
    return pic_update_fields_second(c);
}

int pic_run_steps(pic_ctx *c, int nsteps) {
    if (!c || nsteps < 0) return PIC_EINVAL;
    cudaSetDevice(c->device);
    for (int t = 0; t < nsteps; ++t) {
        int r = run_one_step(c, t + 1 == nsteps);
        c->rho_skip = false;
        if (r) return r;
    }
    return PIC_OK;
}

int pic_get_step(const pic_ctx *c, int *step) {
    if (!c || !step) return PIC_EINVAL;
    *step = c->step;
    return PIC_OK;
}

int pic_set_step(pic_ctx *c, int step) {
    if (!c) return PIC_EINVAL;
    c->step = step;
    return PIC_OK;
}

int pic_synchronize(pic_ctx *c) {
    if (!c) return PIC_EINVAL;
    cudaSetDevice(c->device);
    return sync_status(c);
}

int pic_particle_order_stats(pic_ctx *c, int kind, int64_t *out, int n) {
    if (!c || kind < 0 || kind > 1 || !out || n < 1) return PIC_EINVAL;
    cudaSetDevice(c->device);
    long long v[4] = {0, 0, 0, 0};
    if (c->tile > 0) {
        int r = tile_order_stats(c, kind, v);
        if (r) return r;
    }
    for (int i = 0; i < n && i < 4; ++i) out[i] = v[i];
    return PIC_OK;
}

int pic_get_stream(const pic_ctx *c, void **stream) {
    if (!c || !stream) return PIC_EINVAL;
    *stream = (void *)c->stream;
    return PIC_OK;
}

int pic_diagnostics(pic_ctx *c, double *out, int n) {
    if (!c || !out || n < 1) return PIC_EINVAL;
    cudaSetDevice(c->device);
    launch_diagnostics(c, c->d_diag);
    double tmp[PIC_NDIAG];
    CK(cudaMemcpyAsync(tmp, c->d_diag, sizeof tmp, cudaMemcpyDeviceToHost, c->stream));
    int st = sync_status(c);
    for (int i = 0; i < n && i < PIC_NDIAG; ++i) out[i] = tmp[i];
    return st;
}

int pic_profile_enable(pic_ctx *c, int on) {
    if (!c) return PIC_EINVAL;
    c->prof = on != 0;
    return PIC_OK;
}

int pic_profile_reset(pic_ctx *c) {
    if (!c) return PIC_EINVAL;
    prof_collect(c);
    c->prof_acc.clear();
    return PIC_OK;
}

int pic_profile_read(pic_ctx *c, const char **names, double *total_ms, int64_t *launches, int cap, int *count) {
    if (!c || !count) return PIC_EINVAL;
    prof_collect(c);
    int k = 0;
    for (auto &a : c->prof_acc) {
        if (k < cap) {
            if (names) names[k] = a.first;
            if (total_ms) total_ms[k] = a.second.first;
            if (launches) launches[k] = a.second.second;
        }
        ++k;
    }
    *count = k;
    return PIC_OK;
}

// ---- checkpoint ---------------------------------------------------------

int pic_save(pic_ctx *c, const char *path) {
    if (!c || !path) return PIC_EINVAL;
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(c, PIC_EINVAL, std::string("cannot open ") + path);
    const char magic[8] = {'P', 'I', 'C', '3', 'D', 'B', '2', '2'};
    std::fwrite(magic, 1, 8, f);
    std::fwrite(&c->p, sizeof(PicParams), 1, f);
    std::fwrite(&c->step, sizeof(int), 1, f);
    int r = PIC_OK;
    for (int a = 0; a < PIC_NARRAYS && r == PIC_OK; ++a) {
        int64_t n = 0;
        pic_array_len(c, a, &n);
        std::vector<double> buf((size_t)n);
        r = pic_download_array(c, a, buf.data());
        std::fwrite(buf.data(), sizeof(double), (size_t)n, f);
    }
    for (int k = 0; k < 2 && r == PIC_OK; ++k) {
        int64_t n = 0;
        r = pic_num_particles(c, k, &n);
        std::vector<char> rec((size_t)n * 144);
        if (r == PIC_OK) r = pic_download_particles(c, k, rec.data(), n, &n);
        std::fwrite(&n, sizeof(int64_t), 1, f);
        std::fwrite(rec.data(), 1, rec.size(), f);
    }
    std::fclose(f);
    return r;
}

int pic_load(pic_ctx *c, const char *path) {
    if (!c || !path) return PIC_EINVAL;
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(c, PIC_EINVAL, std::string("cannot open ") + path);
    char magic[8];
    PicParams p;
    int step = 0;
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "PIC3DB22", 8) == 0 &&
              std::fread(&p, sizeof p, 1, f) == 1 && std::fread(&step, sizeof(int), 1, f) == 1;
    if (!ok || p.local_xcells != c->p.local_xcells || p.local_ycells != c->p.local_ycells ||
        p.local_zcells != c->p.local_zcells || p.mem != c->p.mem) {
        std::fclose(f);
        return fail(c, PIC_EINVAL, "checkpoint does not match this context's grid");
    }
    int r = PIC_OK;
    for (int a = 0; a < PIC_NARRAYS && r == PIC_OK; ++a) {
        int64_t n = 0;
        pic_array_len(c, a, &n);
        std::vector<double> buf((size_t)n);
        if (std::fread(buf.data(), sizeof(double), (size_t)n, f) != (size_t)n) r = fail(c, PIC_EINVAL, "short file");
        if (r == PIC_OK) r = pic_upload_array(c, a, buf.data());
    }
    for (int k = 0; k < 2 && r == PIC_OK; ++k) {
        int64_t n = 0;
        if (std::fread(&n, sizeof n, 1, f) != 1) { r = fail(c, PIC_EINVAL, "short file"); break; }
        std::vector<char> rec((size_t)n * 144);
        if (std::fread(rec.data(), 1, rec.size(), f) != rec.size()) { r = fail(c, PIC_EINVAL, "short file"); break; }
        r = pic_upload_particles(c, k, rec.data(), n);
    }
    std::fclose(f);
    if (r == PIC_OK) c->step = step;
    return r;
}

}  // extern "C"
