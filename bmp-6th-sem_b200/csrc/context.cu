// context.cu -- pic_* C ABI: context lifetime, particle I/O, step operators,
// grid access.  Operators enqueue on the context stream; host-copy getters
// synchronise.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "pic_internal.h"

#if defined(__x86_64__)
#include <emmintrin.h>
#endif

namespace picb200 {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int status, const std::string& msg) {
    g_last_error = msg;
    return status;
}

static int check_species(pic_ctx* c, int s) {
    if (!c) return fail(PIC_ERR_ARG, "null context");
    if (s < 0 || s >= c->cfg.num_species) return fail(PIC_ERR_ARG, "species index out of range");
    return PIC_OK;
}

// ---------------------------------------------------------------------------
// Host <-> device streaming of large arrays (particles, grids).  Caller memory
// is ordinary pageable memory, so every copy passes through pinned staging:
// two kPipeChunk buffers alternate, the host-side work on one chunk (a copy,
// or the Point <-> record conversion, split over a pool of threads)
// overlapping the DMA of the other.
// ---------------------------------------------------------------------------
namespace {

class HostPool {
  public:
    static HostPool& get() {
        static HostPool pool;
        return pool;
    }

    // fn(begin, end) over [0, n) in one part per thread, part boundaries
    // multiples of `align`; on the calling thread alone below `serial_below`.
    void run(size_t n, size_t align, size_t serial_below, const std::function<void(size_t, size_t)>& fn) {
        if (n < serial_below || workers_.empty()) {
            if (n) fn(0, n);
            return;
        }
        std::lock_guard<std::mutex> one_at_a_time(call_mu_);
        const int parts = (int)workers_.size() + 1;
        {
            std::lock_guard<std::mutex> lk(mu_);
            job_ = &fn;
            n_ = n;
            align_ = align;
            parts_ = parts;
            pending_ = parts - 1;
            ++gen_;
        }
        cv_.notify_all();
        part(0);
        std::unique_lock<std::mutex> lk(mu_);
        done_.wait(lk, [&] { return pending_ == 0; });
        job_ = nullptr;
    }

    void copy(void* dst, const void* src, size_t bytes) {
        char* d = static_cast<char*>(dst);
        const char* s = static_cast<const char*>(src);
        run(bytes, 64, 4u << 20, [&](size_t a, size_t b) { std::memcpy(d + a, s + a, b - a); });
    }

    ~HostPool() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : workers_) t.join();
    }

  private:
    HostPool() {
        const unsigned hw = std::thread::hardware_concurrency();
        const int n = (int)std::min<unsigned>(hw ? hw : 1u, 16u) - 1;
        for (int i = 0; i < n; ++i) workers_.emplace_back([this, i] { loop(i + 1); });
    }

    void part(int i) {
        // ceil(n / parts) rounded up to the alignment: the parts cover [0, n)
        const size_t per = ((n_ + parts_ - 1) / parts_ + align_ - 1) / align_ * align_;
        const size_t a = std::min(n_, per * (size_t)i), b = std::min(n_, per * (size_t)(i + 1));
        if (b > a) (*job_)(a, b);
    }

    void loop(int i) {
        uint64_t seen = 0;
        for (;;) {
            std::unique_lock<std::mutex> lk(mu_);
            cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
            if (stop_) return;
            seen = gen_;
            lk.unlock();
            part(i);
            lk.lock();
            if (--pending_ == 0) done_.notify_one();
        }
    }

    std::vector<std::thread> workers_;
    std::mutex call_mu_, mu_;
    std::condition_variable cv_, done_;
    uint64_t gen_ = 0;
    int pending_ = 0, parts_ = 1;
    bool stop_ = false;
    const std::function<void(size_t, size_t)>* job_ = nullptr;
    size_t n_ = 0, align_ = 1;
};

constexpr size_t kPipeChunk = 32u << 20;

}  // namespace

static int ensure_pipe(pic_ctx* c) {
    for (int b = 0; b < 2; ++b) {
        if (!c->pipe_buf[b]) PIC_CUDA(cudaMallocHost(&c->pipe_buf[b], kPipeChunk));
        if (!c->pipe_ev[b]) PIC_CUDA(cudaEventCreateWithFlags(&c->pipe_ev[b], cudaEventDisableTiming));
    }
    return PIC_OK;
}

// host (pageable) -> device, enqueued on the context stream; returns when
// the last chunk has been handed to the DMA engine.
static int stream_to_device(pic_ctx* c, void* dev, const void* host, size_t bytes) {
    PIC_TRY(ensure_pipe(c));
    PIC_CUDA(cudaStreamSynchronize(c->stream));  // staging may still feed an earlier copy
    for (size_t off = 0, k = 0; off < bytes; off += kPipeChunk, ++k) {
        const size_t m = std::min(kPipeChunk, bytes - off);
        const int b = (int)(k & 1);
        if (k >= 2) PIC_CUDA(cudaEventSynchronize(c->pipe_ev[b]));  // its previous DMA is done
        HostPool::get().copy(c->pipe_buf[b], static_cast<const char*>(host) + off, m);
        PIC_CUDA(cudaMemcpyAsync(static_cast<char*>(dev) + off, c->pipe_buf[b], m,
                                 cudaMemcpyHostToDevice, c->stream));
        PIC_CUDA(cudaEventRecord(c->pipe_ev[b], c->stream));
    }
    return PIC_OK;
}

// device -> host (pageable), after the work queued on the stream; synchronous.
static int stream_to_host(pic_ctx* c, void* host, const void* dev, size_t bytes) {
    PIC_TRY(ensure_pipe(c));
    const size_t nchunks = (bytes + kPipeChunk - 1) / kPipeChunk;
    auto issue = [&](size_t k) -> int {
        const size_t off = k * kPipeChunk, m = std::min(kPipeChunk, bytes - off);
        const int b = (int)(k & 1);
        PIC_CUDA(cudaMemcpyAsync(c->pipe_buf[b], static_cast<const char*>(dev) + off, m,
                                 cudaMemcpyDeviceToHost, c->stream));
        PIC_CUDA(cudaEventRecord(c->pipe_ev[b], c->stream));
        return PIC_OK;
    };
    if (nchunks == 0) return PIC_OK;
    PIC_TRY(issue(0));
    for (size_t k = 0; k < nchunks; ++k) {
        // the other buffer was emptied in the previous iteration
        if (k + 1 < nchunks) PIC_TRY(issue(k + 1));
        const int b = (int)(k & 1);
        PIC_CUDA(cudaEventSynchronize(c->pipe_ev[b]));
        const size_t off = k * kPipeChunk, m = std::min(kPipeChunk, bytes - off);
        HostPool::get().copy(static_cast<char*>(host) + off, c->pipe_buf[b], m);
    }
    return PIC_OK;
}

// Device -> host copy (pageable destination), synchronous.
static int copy_to_host(pic_ctx* c, void* host, const void* dev, size_t bytes) {
    return stream_to_host(c, host, dev, bytes);
}

static int copy_to_device(pic_ctx* c, void* dev, const void* host, size_t bytes) {
    return stream_to_device(c, dev, host, bytes);
}

// Reference Point -> record, as InsertKernel bins it (src/particles.cpp:
// 230-235): cell ((int)(y*(1/dy)), (int)(x*(1/dx))), the FP32 offset being
// the FP64 remainder clamped below 1.  Dead (pointer == -1) and out-of-domain
// points get kNoCell.  Plain IEEE double arithmetic (the host build does not
// contract products into FMAs).
static inline PointRec point_to_rec(const pic_point& p, int nx, int ny, double inv_dx,
                                    double inv_dy) {
    PointRec r{kNoCell, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (p.pointer == -1) return r;
    const double sx = p.x * inv_dx, sy = p.y * inv_dy;
    if (!(sx >= 0.0 && sy >= 0.0 && sx < (double)nx && sy < (double)ny)) return r;
    const int gx = (int)sx, gy = (int)sy;
    constexpr float kOneBelow = 0x1.fffffep-1f;
    r.cell = (uint32_t)gy * (uint32_t)nx + (uint32_t)gx;
    r.fx = std::min((float)(sx - gx), kOneBelow);
    r.fy = std::min((float)(sy - gy), kOneBelow);
    r.vx = (float)p.vx;
    r.vy = (float)p.vy;
    r.vz = (float)p.vz;
    return r;
}

// Record -> reference Point: x = (gx + fx)*dx in FP64; pointer = the
// particle's index in the output.
static inline void rec_to_point(const PointRec& r, int nx, double dx, double dy, int64_t index,
                                pic_point& p) {
    const int gx = (int)(r.cell % (uint32_t)nx), gy = (int)(r.cell / (uint32_t)nx);
    p.x = ((double)gx + (double)r.fx) * dx;
    p.y = ((double)gy + (double)r.fy) * dy;
    p.z = 0.0;
    p.vx = r.vx;
    p.vy = r.vy;
    p.vz = r.vz;
    p.pointer = (int32_t)index;
    p.pad_ = 0;
}

// Stores of 8-byte words that bypass the cache (no read-for-ownership of
// the destination line): the conversions below are bound by host memory
// traffic, and their outputs are not read again by this thread.
static inline void put8(void* dst, const void* src) {
#if defined(__x86_64__)
    long long v;
    std::memcpy(&v, src, 8);
    _mm_stream_si64(static_cast<long long*>(dst), v);
#else
    std::memcpy(dst, src, 8);
#endif
}

static inline void store_fence() {
#if defined(__x86_64__)
    _mm_sfence();
#endif
}

static inline void stream_rec(PointRec* dst, const PointRec& r) {
    const char* s = reinterpret_cast<const char*>(&r);
    char* d = reinterpret_cast<char*>(dst);
    put8(d, s);
    put8(d + 8, s + 8);
    put8(d + 16, s + 16);
}

static inline void stream_point(pic_point* dst, const pic_point& p) {
    const char* s = reinterpret_cast<const char*>(&p);
    char* d = reinterpret_cast<char*>(dst);
    for (int w = 0; w < 7; ++w) put8(d + 8 * w, s + 8 * w);
}

constexpr size_t kRecsPerChunk = kPipeChunk / sizeof(PointRec);

// Host Points -> device records: the pool converts a chunk into a pinned
// buffer while the DMA engine moves the previous one.
static int points_to_device(pic_ctx* c, PointRec* dev, const pic_point* host, int64_t n) {
    PIC_TRY(ensure_pipe(c));
    PIC_CUDA(cudaStreamSynchronize(c->stream));
    const int nx = c->nx, ny = c->ny;
    const double inv_dx = 1.0 / c->dx, inv_dy = 1.0 / c->dy;
    for (int64_t off = 0, k = 0; off < n; off += (int64_t)kRecsPerChunk, ++k) {
        const size_t m = (size_t)std::min<int64_t>((int64_t)kRecsPerChunk, n - off);
        const int b = (int)(k & 1);
        if (k >= 2) PIC_CUDA(cudaEventSynchronize(c->pipe_ev[b]));
        PointRec* buf = static_cast<PointRec*>(c->pipe_buf[b]);
        const pic_point* src = host + off;
        HostPool::get().run(m, 64, 1u << 16, [&](size_t a, size_t e) {
            for (size_t i = a; i < e; ++i) stream_rec(buf + i, point_to_rec(src[i], nx, ny, inv_dx, inv_dy));
            store_fence();
        });
        PIC_CUDA(cudaMemcpyAsync(dev + off, buf, m * sizeof(PointRec), cudaMemcpyHostToDevice,
                                 c->stream));
        PIC_CUDA(cudaEventRecord(c->pipe_ev[b], c->stream));
    }
    return PIC_OK;
}

// Device records -> host Points, after the work queued on the stream;
// synchronous.  The DMA of chunk k+1 overlaps the pool's expansion of chunk k.
static int points_to_host(pic_ctx* c, pic_point* host, const PointRec* dev, int64_t n) {
    PIC_TRY(ensure_pipe(c));
    const int64_t nchunks = (n + (int64_t)kRecsPerChunk - 1) / (int64_t)kRecsPerChunk;
    auto span = [&](int64_t k) {
        return (size_t)std::min<int64_t>((int64_t)kRecsPerChunk, n - k * (int64_t)kRecsPerChunk);
    };
    auto issue = [&](int64_t k) -> int {
        const int b = (int)(k & 1);
        PIC_CUDA(cudaMemcpyAsync(c->pipe_buf[b], dev + k * (int64_t)kRecsPerChunk,
                                 span(k) * sizeof(PointRec), cudaMemcpyDeviceToHost, c->stream));
        PIC_CUDA(cudaEventRecord(c->pipe_ev[b], c->stream));
        return PIC_OK;
    };
    if (nchunks == 0) return PIC_OK;
    const int nx = c->nx;
    const double dx = c->dx, dy = c->dy;
    PIC_TRY(issue(0));
    for (int64_t k = 0; k < nchunks; ++k) {
        if (k + 1 < nchunks) PIC_TRY(issue(k + 1));
        const int b = (int)(k & 1);
        PIC_CUDA(cudaEventSynchronize(c->pipe_ev[b]));
        const PointRec* buf = static_cast<const PointRec*>(c->pipe_buf[b]);
        const int64_t off = k * (int64_t)kRecsPerChunk;
        pic_point* dst = host + off;
        HostPool::get().run(span(k), 64, 1u << 16, [&](size_t a, size_t e) {
            for (size_t i = a; i < e; ++i) {
                pic_point p;
                rec_to_point(buf[i], nx, dx, dy, off + (int64_t)i, p);
                stream_point(dst + i, p);
            }
            store_fence();
        });
    }
    return PIC_OK;
}

static cudaEvent_t pool_event(pic_ctx* c) {
    if (!c->ev_pool.empty()) {
        cudaEvent_t e = c->ev_pool.back();
        c->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

void prof_begin(pic_ctx* c, int phase) {
    (void)phase;
    if (!c->profiling) return;
    c->prof_open = pool_event(c);
    cudaEventRecord(c->prof_open, c->stream);
}

void prof_end(pic_ctx* c, int phase) {
    if (!c->profiling || !c->prof_open) return;
    cudaEvent_t b = pool_event(c);
    cudaEventRecord(b, c->stream);
    c->prof_pending.push_back({phase, c->prof_open, b});
    c->prof_open = nullptr;
}

static void free_ctx(pic_ctx* c) {
    ws_free(c);
    for (auto& p : c->prof_pending) {
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    for (auto e : c->ev_pool) cudaEventDestroy(e);
    for (int s = 0; s < PIC_MAX_SPECIES; ++s) species_free(c->sp[s]);
    poisson_free(c);
    cudaFree(c->rho);
    cudaFree(c->phi);
    cudaFree(c->bz);
    cudaFree(c->fld);
    cudaFree(c->mask);
    cudaFree(c->dir_val);
    cudaFree(c->efield64);
    cudaFree(c->scan_partials);
    cudaFree(c->staging);
    if (c->host_staging) cudaFreeHost(c->host_staging);
    for (int b = 0; b < 2; ++b) {
        if (c->pipe_buf[b]) cudaFreeHost(c->pipe_buf[b]);
        if (c->pipe_ev[b]) cudaEventDestroy(c->pipe_ev[b]);
    }
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

}  // namespace picb200

using namespace picb200;

extern "C" {

const char* pic_last_error(void) { return g_last_error.c_str(); }

const char* pic_status_string(int status) {
    switch (status) {
        case PIC_OK: return "ok";
        case PIC_ERR_ARG: return "bad argument";
        case PIC_ERR_CONFIG: return "invalid configuration";
        case PIC_ERR_CAPACITY: return "capacity exceeded";
        case PIC_ERR_NOT_CONVERGED: return "Poisson solve did not converge";
        case PIC_ERR_CUDA: return "CUDA error";
        case PIC_ERR_STATE: return "operator called in the wrong state";
        case PIC_ERR_IO: return "I/O error";
        case PIC_ERR_NO_DEVICE: return "no usable sm_100 device";
        case PIC_ERR_TIMEOUT: return "bounded device wait gave up";
        default: return "unknown status";
    }
}

int pic_config_default(pic_config* cfg) {
    if (!cfg) return fail(PIC_ERR_ARG, "null config");
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->nx = cfg->ny = 128;
    cfg->xmax = cfg->ymax = 128 * 2.5e-4;
    cfg->dt = 5e-11;
    cfg->epsilon = 8.854e-12;
    cfg->poisson_solver = PIC_SOLVER_MG_PCG;
    cfg->warm_start = PIC_WARM_PREVIOUS;
    cfg->poisson_tol = 1e-8;
    cfg->poisson_maxit = 500;
    cfg->deposit_energy = 1;
    cfg->timesteps = 100;
    cfg->print_interval = 1;
    return PIC_OK;
}

int pic_create(const pic_config* cfg_in, pic_ctx** out) {
    if (!cfg_in || !out) return fail(PIC_ERR_ARG, "null argument");
    *out = nullptr;
    const pic_config& cfg = *cfg_in;
    if (cfg.nx < 4 || cfg.ny < 4) return fail(PIC_ERR_CONFIG, "nx and ny must be >= 4");
    if ((int64_t)cfg.nx * cfg.ny > (1ll << 30)) return fail(PIC_ERR_CONFIG, "grid too large");
    if (!(cfg.xmax > 0) || !(cfg.ymax > 0) || !(cfg.dt > 0) || !(cfg.epsilon > 0))
        return fail(PIC_ERR_CONFIG, "xmax, ymax, dt and epsilon must be positive");
    if (cfg.num_species < 1 || cfg.num_species > PIC_MAX_SPECIES)
        return fail(PIC_ERR_CONFIG, "num_species must be 1..4");
    if (cfg.num_rects < 0 || cfg.num_rects > PIC_MAX_RECTS)
        return fail(PIC_ERR_CONFIG, "num_rects must be 0..32");
    const int GX = cfg.nx + 1, GY = cfg.ny + 1;
    std::vector<uint8_t> mask((size_t)GX * GY, 0);
    std::vector<double> dval((size_t)GX * GY, 0.0);
    for (int r = 0; r < cfg.num_rects; ++r) {
        const pic_rect& R = cfg.rects[r];
        if (R.x1 < 0 || R.y1 < 0 || R.x2 >= GX || R.y2 >= GY || R.x1 > R.x2 || R.y1 > R.y2)
            return fail(PIC_ERR_CONFIG, "electrode rectangle outside the node grid");
        // setPotentialBoundary / overwritePhi order: later rectangles win
        for (int j = R.y1; j <= R.y2; ++j)
            for (int i = R.x1; i <= R.x2; ++i) {
                mask[(size_t)j * GX + i] = 1;
                dval[(size_t)j * GX + i] = R.potential;
            }
    }
    const bool periodic = cfg.periodic_y != 0;
    if (!periodic) {
        for (int i = 0; i < GX; ++i)
            if (!mask[i] || !mask[(size_t)(GY - 1) * GX + i])
                return fail(PIC_ERR_CONFIG, "every wall node must be an electrode (generateCoeffs)");
        for (int j = 0; j < GY; ++j)
            if (!mask[(size_t)j * GX] || !mask[(size_t)j * GX + GX - 1])
                return fail(PIC_ERR_CONFIG, "every wall node must be an electrode (generateCoeffs)");
    } else {
        // generateCoeffsPeriodic (src/poissonSolver.cpp:82-180) couples i-1
        // and i+1 across row ends: the x walls of the solved rows must be
        // electrodes
        for (int j = 0; j < GY - 1; ++j)
            if (!mask[(size_t)j * GX] || !mask[(size_t)j * GX + GX - 1])
                return fail(PIC_ERR_CONFIG,
                            "periodic in y: the x = 0 and x = nx node columns must be electrodes");
        if (cfg.warm_start == PIC_WARM_LEARNED)
            return fail(PIC_ERR_CONFIG, "periodic in y: the learned warm start is not available");
    }

    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(PIC_ERR_NO_DEVICE, "no CUDA device visible");
    if (cfg.device < 0 || cfg.device >= ndev) return fail(PIC_ERR_ARG, "device ordinal out of range");
    cudaDeviceProp prop{};
    PIC_CUDA(cudaGetDeviceProperties(&prop, cfg.device));
    if (prop.major != 10)
        return fail(PIC_ERR_NO_DEVICE, std::string("library is built for sm_100a; device is ") +
                                           prop.name);
    PIC_CUDA(cudaSetDevice(cfg.device));

    pic_ctx* c = new pic_ctx();
    c->cfg = cfg;
    if (c->cfg.poisson_tol <= 0) c->cfg.poisson_tol = 1e-8;
    if (c->cfg.poisson_maxit <= 0) c->cfg.poisson_maxit = 500;
    c->nx = cfg.nx;
    c->ny = cfg.ny;
    c->GX = GX;
    c->GY = GY;
    c->nodes = (int64_t)GX * GY;
    c->ncells = (int64_t)cfg.nx * cfg.ny;
    c->periodic = periodic;
    c->solve_rows = periodic ? GY - 1 : GY;
    c->solve_nodes = (int64_t)GX * c->solve_rows;
    c->dx = cfg.xmax / cfg.nx;  // readPICDAT, src/particles.cpp:360-361
    c->dy = cfg.ymax / cfg.ny;
    c->device = cfg.device;
    auto bail = [&](int st) {
        free_ctx(c);
        return st;
    };
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(PIC_ERR_CUDA, "stream creation failed"));
    c->own_stream = true;
    const size_t n = (size_t)c->nodes;
    if (cudaMalloc(&c->rho, n * 8) || cudaMalloc(&c->phi, n * 8) || cudaMalloc(&c->bz, n * 8) ||
        cudaMalloc(&c->fld, n * sizeof(float4)) || cudaMalloc(&c->mask, n) ||
        cudaMalloc(&c->dir_val, n * 8) || cudaMalloc(&c->efield64, n * 16) ||
        cudaMalloc(&c->scan_partials, ((size_t)c->ncells / 2048 + 2) * 4))
        return bail(fail(PIC_ERR_CUDA, "device allocation failed for the grids"));
    std::vector<double> bz(n, cfg.b0);  // initMagneticField, src/particles.cpp:709-720
    std::vector<double> phi0(n, 0.0);
    for (size_t i = 0; i < n; ++i)
        if (mask[i]) phi0[i] = dval[i];  // initPoissonSolver -> overwritePhi
    if (cudaMemcpy(c->mask, mask.data(), n, cudaMemcpyHostToDevice) ||
        cudaMemcpy(c->dir_val, dval.data(), n * 8, cudaMemcpyHostToDevice) ||
        cudaMemcpy(c->bz, bz.data(), n * 8, cudaMemcpyHostToDevice) ||
        cudaMemcpy(c->phi, phi0.data(), n * 8, cudaMemcpyHostToDevice) ||
        cudaMemset(c->rho, 0, n * 8) || cudaMemset(c->fld, 0, n * sizeof(float4)))
        return bail(fail(PIC_ERR_CUDA, "grid initialisation copy failed"));
    c->bz_uniform = true;
    c->bz_value = cfg.b0;
    int st = fields_set_bz(c);
    if (st) return bail(st);
    for (int s = 0; s < cfg.num_species; ++s)
        if ((st = species_setup(c, s))) return bail(st);
    if ((st = poisson_setup(c))) return bail(st);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess)
        return bail(fail(PIC_ERR_CUDA, "context initialisation failed"));
    *out = c;
    return PIC_OK;
}

void pic_destroy(pic_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    free_ctx(c);
}

int pic_set_stream(pic_ctx* c, void* stream) {
    if (!c) return fail(PIC_ERR_ARG, "null context");
    PIC_CUDA(cudaStreamSynchronize(c->stream));
    if (c->own_stream) cudaStreamDestroy(c->stream);
    if (stream) {
        c->stream = static_cast<cudaStream_t>(stream);
        c->own_stream = false;
    } else {
        PIC_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        c->own_stream = true;
    }
    return PIC_OK;
}

void* pic_get_stream(pic_ctx* c) { return c ? (void*)c->stream : nullptr; }

int pic_synchronize(pic_ctx* c) {
    if (!c) return fail(PIC_ERR_ARG, "null context");
    PIC_CUDA(cudaStreamSynchronize(c->stream));
    return PIC_OK;
}

int pic_reserve(pic_ctx* c, int s, int64_t capacity) {
    PIC_TRY(check_species(c, s));
    if (capacity < 0) return fail(PIC_ERR_ARG, "negative capacity");
    return species_reserve(c, s, capacity);
}

int pic_import_points(pic_ctx* c, int s, const pic_point* host, int64_t n) {
    PIC_TRY(check_species(c, s));
    if (n < 0 || (n > 0 && !host)) return fail(PIC_ERR_ARG, "bad point array");
    if (n > (int64_t)0xF0000000ll) return fail(PIC_ERR_CAPACITY, "too many points");
    PointRec* dev = nullptr;
    PIC_TRY(particles_import_staging(c, n, &dev));
    PIC_TRY(points_to_device(c, dev, host, n));
    return particles_import(c, s, n);
}

int pic_export_points(pic_ctx* c, int s, pic_point* host, int64_t capacity, int64_t* n_out) {
    PIC_TRY(check_species(c, s));
    int64_t n = 0;
    PIC_TRY(particles_count(c, s, &n));
    if (n_out) *n_out = n;
    if (!host) return PIC_OK;  // size query
    if (capacity < n) return fail(PIC_ERR_CAPACITY, "export buffer smaller than the particle count");
    if (n == 0) return PIC_OK;
    PIC_TRY(ensure_staging(c, (size_t)n * sizeof(PointRec)));
    PointRec* dev = static_cast<PointRec*>(c->staging);
    int64_t n2 = 0;
    PIC_TRY(particles_export(c, s, dev, &n2));
    return points_to_host(c, host, dev, n);
}

int pic_export_state(pic_ctx* c, int s, int32_t* cell, float* fx, float* fy, float* vx,
                     float* vy, float* vz, int64_t capacity, int64_t* n_out) {
    PIC_TRY(check_species(c, s));
    int64_t n = 0;
    PIC_TRY(particles_count(c, s, &n));
    if (n_out) *n_out = n;
    if (!cell && !fx && !fy && !vx && !vy && !vz) return PIC_OK;
    if (!cell || !fx || !fy || !vx || !vy || !vz) return fail(PIC_ERR_ARG, "null output array");
    if (capacity < n) return fail(PIC_ERR_CAPACITY, "output arrays smaller than the particle count");
    if (n == 0) return PIC_OK;
    PIC_TRY(ensure_staging(c, (size_t)n * 24));
    PIC_TRY(particles_export_state(c, s, c->staging, n));
    std::vector<char> h((size_t)n * 24);
    PIC_TRY(copy_to_host(c, h.data(), c->staging, h.size()));
    const size_t b = (size_t)n * 4;
    std::memcpy(cell, h.data(), b);
    std::memcpy(fx, h.data() + b, b);
    std::memcpy(fy, h.data() + 2 * b, b);
    std::memcpy(vx, h.data() + 3 * b, b);
    std::memcpy(vy, h.data() + 4 * b, b);
    std::memcpy(vz, h.data() + 5 * b, b);
    return PIC_OK;
}

int pic_load_plasma(pic_ctx* c, int s, const pic_plasma_desc* d) {
    PIC_TRY(check_species(c, s));
    if (!d) return fail(PIC_ERR_ARG, "null plasma description");
    return particles_load_plasma(c, s, d);
}

int pic_particle_count(pic_ctx* c, int s, int64_t* n) {
    PIC_TRY(check_species(c, s));
    if (!n) return fail(PIC_ERR_ARG, "null output");
    return particles_count(c, s, n);
}

int pic_bin_counts(pic_ctx* c, int s, int32_t* host) {
    PIC_TRY(check_species(c, s));
    if (!host) return fail(PIC_ERR_ARG, "null output");
    PIC_TRY(ensure_staging(c, (size_t)c->nodes * 4));
    PIC_TRY(particles_bin_counts(c, s, static_cast<int32_t*>(c->staging)));
    return copy_to_host(c, host, c->staging, (size_t)c->nodes * 4);
}

int pic_left_exits(pic_ctx* c, int s, int64_t* n) {
    PIC_TRY(check_species(c, s));
    unsigned long long v = 0;
    PIC_CUDA(cudaMemcpyAsync(&v, c->sp[s].counters, 8, cudaMemcpyDeviceToHost, c->stream));
    PIC_CUDA(cudaStreamSynchronize(c->stream));
    PIC_CUDA(cudaMemsetAsync(c->sp[s].counters, 0, 8, c->stream));
    if (n) *n = (int64_t)v;
    return PIC_OK;
}

int pic_source_default(pic_source_desc* d) {
    if (!d) return fail(PIC_ERR_ARG, "null argument");
    *d = pic_source_desc{};
    d->reinject_x = 0.024;  // src/utils.cpp:398
    d->te_ev = 2.0;
    d->ti_ev = 0.026;
    d->x11 = 0.0025;  // src/types.cpp:103-105
    d->x22 = 0.01;
    d->xm = 0.00625;
    d->ionimax = 5.23e23;  // src/utils.cpp:500
    d->rate_div = 1.67e6;  // src/utils.cpp:502
    d->reinject = 1;
    d->pairs = 1;
    d->seed = 0x5A1CE5ull;
    return PIC_OK;
}

int pic_generate_new_particles(pic_ctx* c, const pic_source_desc* d, int64_t* n_e, int64_t* n_p) {
    if (!c || !d) return fail(PIC_ERR_ARG, "null argument");
    return particles_generate(c, d, n_e, n_p);
}

int pic_zero_rho(pic_ctx* c) {
    if (!c) return fail(PIC_ERR_ARG, "null context");
    PIC_CUDA(cudaMemsetAsync(c->rho, 0, (size_t)c->nodes * 8, c->stream));
    return PIC_OK;
}

int pic_charge_deposition(pic_ctx* c, int s) {
    PIC_TRY(check_species(c, s));
    if (!c->sp[s].acc_fresh) PIC_TRY(particles_deposit(c, s));
    return particles_flush_rho(c, s);
}

int pic_poisson_solve(pic_ctx* c, int iteration) {
    if (!c) return fail(PIC_ERR_ARG, "null context");
    (void)iteration;
    return poisson_solve(c);
}

int pic_move_particles(pic_ctx* c, int s, int iteration) {
    PIC_TRY(check_species(c, s));
    (void)iteration;
    if (!c->fields_valid) PIC_TRY(fields_from_phi(c));
    return particles_push(c, s);
}

int pic_compact_particles(pic_ctx* c, int s) { return check_species(c, s); }
int pic_cleanup_map(pic_ctx* c, int s) { return check_species(c, s); }

int pic_particle_phase(pic_ctx* c, int iteration) {
    if (!c) return fail(PIC_ERR_ARG, "null context");
    if (!c->fields_valid) PIC_TRY(fields_from_phi(c));
    for (int s = 0; s < c->cfg.num_species; ++s) {
        if (!c->sp[s].acc_fresh) PIC_TRY(particles_deposit(c, s));
        PIC_TRY(particles_push(c, s));
    }
    (void)iteration;
    return PIC_OK;
}

int pic_step(pic_ctx* c, int iteration) {
    if (!c) return fail(PIC_ERR_ARG, "null context");
    PIC_TRY(pic_zero_rho(c));
    for (int s = 0; s < c->cfg.num_species; ++s) PIC_TRY(pic_charge_deposition(c, s));
    PIC_TRY(pic_poisson_solve(c, iteration));
    for (int s = 0; s < c->cfg.num_species; ++s) PIC_TRY(pic_move_particles(c, s, iteration));
    return PIC_OK;
}

int pic_get_rho(pic_ctx* c, double* host) {
    if (!c || !host) return fail(PIC_ERR_ARG, "null argument");
    return copy_to_host(c, host, c->rho, (size_t)c->nodes * 8);
}

int pic_get_phi(pic_ctx* c, double* host) {
    if (!c || !host) return fail(PIC_ERR_ARG, "null argument");
    return copy_to_host(c, host, c->phi, (size_t)c->nodes * 8);
}

int pic_get_efield(pic_ctx* c, pic_field* host) {
    if (!c || !host) return fail(PIC_ERR_ARG, "null argument");
    PIC_TRY(efield_export(c));
    return copy_to_host(c, host, c->efield64, (size_t)c->nodes * 16);
}

int pic_get_final_mesh(pic_ctx* c, int s, double* host) {
    PIC_TRY(check_species(c, s));
    if (!host) return fail(PIC_ERR_ARG, "null output");
    return copy_to_host(c, host, c->sp[s].final_mesh, (size_t)c->nodes * 8);
}

int pic_get_energy_mesh(pic_ctx* c, int s, double* host) {
    PIC_TRY(check_species(c, s));
    if (!host) return fail(PIC_ERR_ARG, "null output");
    return copy_to_host(c, host, c->sp[s].energy_mesh, (size_t)c->nodes * 8);
}

int pic_set_rho(pic_ctx* c, const double* host) {
    if (!c || !host) return fail(PIC_ERR_ARG, "null argument");
    return copy_to_device(c, c->rho, host, (size_t)c->nodes * 8);
}

int pic_set_phi(pic_ctx* c, const double* host) {
    if (!c || !host) return fail(PIC_ERR_ARG, "null argument");
    PIC_TRY(copy_to_device(c, c->phi, host, (size_t)c->nodes * 8));
    c->ps.have_prev = true;
    c->fields_valid = false;
    return PIC_OK;
}

int pic_update_fields_from_phi(pic_ctx* c) {
    if (!c) return fail(PIC_ERR_ARG, "null context");
    PIC_TRY(overwrite_phi(c));
    return fields_from_phi(c);
}

int pic_set_bz(pic_ctx* c, const double* host) {
    if (!c || !host) return fail(PIC_ERR_ARG, "null argument");
    PIC_TRY(copy_to_device(c, c->bz, host, (size_t)c->nodes * 8));
    c->bz_uniform = true;
    c->bz_value = host[0];
    for (int64_t i = 1; i < c->nodes; ++i)
        if (host[i] != host[0]) {
            c->bz_uniform = false;
            break;
        }
    return fields_set_bz(c);
}

int pic_set_profiling(pic_ctx* c, int on) {
    if (!c) return fail(PIC_ERR_ARG, "null context");
    c->profiling = on != 0;
    return PIC_OK;
}

int pic_profile_read(pic_ctx* c, double* ms, int64_t* calls, int reset) {
    if (!c) return fail(PIC_ERR_ARG, "null context");
    PIC_CUDA(cudaStreamSynchronize(c->stream));
    for (auto& p : c->prof_pending) {
        float t = 0;
        PIC_CUDA(cudaEventElapsedTime(&t, p.a, p.b));
        c->prof_ms[p.phase] += t;
        c->prof_calls[p.phase] += 1;
        c->ev_pool.push_back(p.a);
        c->ev_pool.push_back(p.b);
    }
    c->prof_pending.clear();
    for (int i = 0; i < PIC_NUM_PHASES; ++i) {
        if (ms) ms[i] = c->prof_ms[i];
        if (calls) calls[i] = c->prof_calls[i];
        if (reset) {
            c->prof_ms[i] = 0;
            c->prof_calls[i] = 0;
        }
    }
    return PIC_OK;
}

int pic_set_tile_shape(pic_ctx* c, int shape) {
    if (!c) return fail(PIC_ERR_ARG, "null context");
    if (shape < 0 || shape >= particles_num_tile_shapes()) return fail(PIC_ERR_ARG, "unknown tile shape");
    c->tile_shape = shape;
    return PIC_OK;
}

int pic_autotune(pic_ctx* c, int* shape_out, double* ms_per_shape) {
    if (!c) return fail(PIC_ERR_ARG, "null context");
    // cache key: device, grid, particles (two significant digits), species
    int64_t n = 0;
    for (int s = 0; s < c->cfg.num_species; ++s) {
        int64_t m = 0;
        PIC_TRY(particles_count(c, s, &m));
        n += m;
    }
    cudaDeviceProp prop{};
    PIC_CUDA(cudaGetDeviceProperties(&prop, c->device));
    int64_t rounded = n;
    int64_t scale = 1;
    while (rounded >= 100) {
        rounded /= 10;
        scale *= 10;
    }
    std::string dev(prop.name);
    for (char& ch : dev)
        if (ch == ' ') ch = '_';
    char key[256];
    std::snprintf(key, sizeof(key), "%s %d %d %lld %d", dev.c_str(), c->nx, c->ny,
                  (long long)(rounded * scale), c->cfg.num_species);
    const char* path = std::getenv("PIC_TUNE_CACHE");
    const int nshapes = particles_num_tile_shapes();
    if (path && !ms_per_shape) {
        if (FILE* f = std::fopen(path, "r")) {
            char line[512];
            int found = -1;
            while (std::fgets(line, sizeof(line), f)) {
                const size_t kl = std::strlen(key);
                if (std::strncmp(line, key, kl) == 0 && line[kl] == ' ') found = std::atoi(line + kl + 1);
            }
            std::fclose(f);
            if (found >= 0 && found < nshapes) {
                c->tile_shape = found;
                if (shape_out) *shape_out = found;
                return PIC_OK;
            }
        }
    }
    std::vector<double> ms((size_t)nshapes, 0.0);
    PIC_TRY(particles_time_shapes(c, 3, ms.data()));
    int best = 0;
    for (int k = 1; k < nshapes; ++k)
        if (ms[k] < ms[best]) best = k;
    c->tile_shape = best;
    if (shape_out) *shape_out = best;
    if (ms_per_shape)
        for (int k = 0; k < nshapes; ++k) ms_per_shape[k] = ms[k];
    if (path) {
        if (FILE* f = std::fopen(path, "a")) {
            std::fprintf(f, "%s %d\n", key, best);
            std::fclose(f);
        }
    }
    return PIC_OK;
}

int pic_debug_set_wait_limits(pic_ctx* c, int64_t barrier_polls, int64_t tensor_wait_cycles) {
    if (!c) return fail(PIC_ERR_ARG, "null context");
    PIC_CUDA(cudaSetDevice(c->cfg.device));
    PIC_CUDA(cudaStreamSynchronize(c->stream));
    PIC_TRY(poisson_set_spin_limit(barrier_polls));
    PIC_TRY(ws_set_wait_limit(tensor_wait_cycles));
    return PIC_OK;
}

int pic_debug_vcycle(pic_ctx* c, const float* rhs, float* out, int per_sweep) {
    if (!c || !rhs || !out) return fail(PIC_ERR_ARG, "null argument");
    PIC_CUDA(cudaSetDevice(c->cfg.device));
    PIC_CUDA(cudaStreamSynchronize(c->stream));
    return poisson_debug_vcycle(c, rhs, out, per_sweep);
}

int pic_launch_count(pic_ctx* c, int64_t* n) {
    if (!c || !n) return fail(PIC_ERR_ARG, "null argument");
    *n = c->launches;
    return PIC_OK;
}

int pic_set_poisson(pic_ctx* c, int solver, int warm, double tol, int maxit) {
    if (!c) return fail(PIC_ERR_ARG, "null context");
    if (solver != PIC_SOLVER_MG_PCG && solver != PIC_SOLVER_JACOBI_PCG)
        return fail(PIC_ERR_ARG, "unknown solver");
    if (warm < PIC_WARM_ZERO || warm > PIC_WARM_LEARNED) return fail(PIC_ERR_ARG, "unknown warm start");
    if (!(tol > 0) || maxit <= 0) return fail(PIC_ERR_ARG, "tol and maxit must be positive");
    if (c->periodic && warm == PIC_WARM_LEARNED)
        return fail(PIC_ERR_CONFIG, "periodic in y: the learned warm start is not available");
    c->ps.solver = solver;
    c->ps.warm = warm;
    c->ps.tol = tol;
    c->ps.maxit = maxit;
    return PIC_OK;
}

int pic_set_poisson_graph(pic_ctx* c, int enable) {
    if (!c) return fail(PIC_ERR_ARG, "null context");
    c->ps.graph_off = enable == 0;
    return PIC_OK;
}

int pic_poisson_start_relres(pic_ctx* c, double* relres0) {
    if (!c || !relres0) return fail(PIC_ERR_ARG, "null argument");
    *relres0 = c->ps.last_relres0;
    return PIC_OK;
}

int pic_poisson_stats(pic_ctx* c, int* iters, double* relres, double* ms) {
    if (!c) return fail(PIC_ERR_ARG, "null context");
    if (iters) *iters = c->ps.last_iters;
    if (relres) *relres = c->ps.last_relres;
    if (ms) *ms = c->ps.last_ms;
    return PIC_OK;
}

}  // extern "C"
