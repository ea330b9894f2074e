// ensemble.cu -- many independent PIC instances advanced together.
//
// An ensemble holds N contexts on one device and one stream (instances of
// uneven grid size, electrode voltage, Bz and density, as a parameter scan
// runs them).  One step of all of them is one launch per phase: the charge
// deposit conversion of every species of every instance, ONE persistent
// cooperative launch for all the Poisson solves (poisson.cu), and per species
// one push launch and one side-list launch over all instances
// (particles.cu).  Per-instance arguments live in device tables the host
// rewrites before each step, so the phase launches can be captured once in a
// CUDA graph and replayed.  The particle-kernel tile shape is picked by
// timing (pic_ensemble_autotune).  No reference counterpart: the reference
// runs one simulation per process.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "pic_internal.h"

using namespace picb200;

struct pic_ensemble {
    int n = 0;
    std::vector<pic_ctx*> cs;
    cudaStream_t stream = nullptr;
    ParticleBatchImpl* pb = nullptr;
    // batched Poisson
    char* h_insts = nullptr;  // pinned
    void* d_insts = nullptr;
    size_t desc = 0;
    void* d_fused = nullptr;
    double* d_partials = nullptr;
    int* d_active = nullptr;
    int* d_inst_of = nullptr;              // block -> instance of the solve launch
    std::vector<int> blk0, nblk;           // each instance's block range
    size_t smem = 0;
    int blocks = 0;
    const double** d_scal_ptrs = nullptr;
    double* d_scal_all = nullptr;
    double* h_scal_all = nullptr;  // pinned
    cudaEvent_t ev[4] = {};
    int shape = 0;
    bool energy = true;
    bool use_graph = true;
    cudaGraphExec_t graph = nullptr;
    bool graph_failed = false;
    double last_ms[3] = {0, 0, 0};  // deposit, Poisson (+E), push
};

namespace {

__global__ void k_gather_scal(const double* const* src, int n, double* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * 16) return;
    out[i] = src[i / 16][i % 16];
}

void free_ensemble(pic_ensemble* e) {
    if (e->graph) cudaGraphExecDestroy(e->graph);
    batch_destroy(e->pb);
    for (auto* c : e->cs) pic_destroy(c);
    if (e->h_insts) cudaFreeHost(e->h_insts);
    if (e->h_scal_all) cudaFreeHost(e->h_scal_all);
    cudaFree(e->d_insts);
    cudaFree(e->d_fused);
    cudaFree(e->d_partials);
    cudaFree(e->d_inst_of);
    cudaFree(e->d_active);
    cudaFree(e->d_scal_ptrs);
    cudaFree(e->d_scal_all);
    for (auto& v : e->ev)
        if (v) cudaEventDestroy(v);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
}

// The phases of one step, enqueued on e->stream (tables already uploaded).
// While capturing, the timing events become event-record nodes.
int enqueue_step(pic_ensemble* e, bool capturing) {
    cudaStream_t st = e->stream;
    const unsigned evflags = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
    PIC_CUDA(cudaEventRecordWithFlags(e->ev[0], st, evflags));
    PIC_TRY(batch_deposit(e->pb, st));
    PIC_CUDA(cudaEventRecordWithFlags(e->ev[1], st, evflags));
    PIC_TRY(poisson_batch_launch(e->d_insts, e->n, e->d_inst_of, e->d_partials,
                                 reinterpret_cast<unsigned*>(e->d_active), e->d_active + e->n, e->smem,
                                 e->blocks, st));
    PIC_CUDA(cudaEventRecordWithFlags(e->ev[2], st, evflags));
    PIC_TRY(batch_push(e->pb, e->shape, e->energy, st));
    PIC_CUDA(cudaEventRecordWithFlags(e->ev[3], st, evflags));
    k_gather_scal<<<(e->n * 16 + 127) / 128, 128, 0, st>>>(e->d_scal_ptrs, e->n, e->d_scal_all);
    PIC_CUDA(cudaMemcpyAsync(e->h_scal_all, e->d_scal_all, (size_t)e->n * 16 * sizeof(double),
                             cudaMemcpyDeviceToHost, st));
    PIC_CUDA(cudaGetLastError());
    return PIC_OK;
}

int upload_poisson(pic_ensemble* e) {
    for (int i = 0; i < e->n; ++i)
        PIC_TRY(poisson_batch_describe(e->cs[i], e->h_insts + (size_t)i * e->desc,
                                       static_cast<char*>(e->d_fused) + (size_t)i * 1024, e->blk0[i],
                                       e->nblk[i]));
    PIC_CUDA(cudaMemcpyAsync(e->d_insts, e->h_insts, (size_t)e->n * e->desc, cudaMemcpyHostToDevice,
                             e->stream));
    return PIC_OK;
}

}  // namespace

extern "C" {

int pic_ensemble_create(const pic_config* cfgs, int n, pic_ensemble** out) {
    if (!cfgs || n <= 0 || !out) return fail(PIC_ERR_ARG, "ensemble: bad arguments");
    *out = nullptr;
    for (int i = 1; i < n; ++i)
        if (cfgs[i].device != cfgs[0].device || cfgs[i].num_species != cfgs[0].num_species ||
            (cfgs[i].deposit_energy != 0) != (cfgs[0].deposit_energy != 0))
            return fail(PIC_ERR_CONFIG, "ensemble: instances must share device, species count and energy mesh mode");
    PIC_CUDA(cudaSetDevice(cfgs[0].device));
    auto* e = new pic_ensemble();
    auto bail = [&](int st) {
        free_ensemble(e);
        return st;
    };
    e->n = n;
    e->energy = cfgs[0].deposit_energy != 0;
    if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(PIC_ERR_CUDA, "ensemble: stream creation failed"));
    for (int i = 0; i < n; ++i) {
        pic_ctx* c = nullptr;
        int st = pic_create(&cfgs[i], &c);
        if (st != PIC_OK) return bail(st);
        e->cs.push_back(c);
        if ((st = pic_set_stream(c, e->stream)) != PIC_OK) return bail(st);
    }
    int st = batch_create(e->cs.data(), n, &e->pb);
    if (st != PIC_OK) return bail(st);
    // batched Poisson: descriptors, fused-level tables, scratch
    e->desc = poisson_batch_desc_bytes();
    size_t smem = 0;
    std::vector<char> fused((size_t)n * 1024, 0);
    for (int i = 0; i < n; ++i) {
        size_t fb = 0;
        const void* f = poisson_fused_table(e->cs[i], &fb);
        if (fb > 1024) return bail(fail(PIC_ERR_CONFIG, "ensemble: fused-level table too large"));
        std::memcpy(fused.data() + (size_t)i * 1024, f, fb);
        smem = std::max(smem, poisson_fused_smem(e->cs[i]));
    }
    e->smem = smem;
    if ((st = poisson_batch_blocks(smem, &e->blocks)) != PIC_OK) return bail(st);
    if (e->blocks < n) return bail(fail(PIC_ERR_CONFIG, "ensemble: more instances than co-resident solver blocks"));
    std::vector<const double*> scal_ptrs;
    for (auto* c : e->cs) scal_ptrs.push_back(c->ps.scal);
    // the solve's blocks: at least one per instance, the rest in proportion
    // to the instances' node counts (largest remainders)
    {
        double total = 0;
        for (auto* c : e->cs) total += (double)c->nodes;
        e->nblk.assign(n, 1);
        const int spare = e->blocks - n;
        std::vector<std::pair<double, int>> rem;
        int given = 0;
        for (int i = 0; i < n; ++i) {
            const double share = spare * (double)e->cs[i]->nodes / total;
            const int whole = (int)share;
            e->nblk[i] += whole;
            given += whole;
            rem.push_back({share - whole, i});
        }
        std::sort(rem.begin(), rem.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
        for (int k = 0; k < spare - given && k < n; ++k) e->nblk[rem[k].second] += 1;
        std::vector<int> inst_of((size_t)e->blocks, -1);
        e->blk0.assign(n, 0);
        int b = 0;
        for (int i = 0; i < n; ++i) {
            e->blk0[i] = b;
            for (int k = 0; k < e->nblk[i]; ++k) inst_of[(size_t)b++] = i;
        }
        if (cudaMalloc(&e->d_inst_of, inst_of.size() * sizeof(int)) ||
            cudaMemcpy(e->d_inst_of, inst_of.data(), inst_of.size() * sizeof(int), cudaMemcpyHostToDevice))
            return bail(fail(PIC_ERR_CUDA, "ensemble: allocation failed"));
    }
    if (cudaMallocHost(&e->h_insts, (size_t)n * e->desc) || cudaMalloc(&e->d_insts, (size_t)n * e->desc) ||
        cudaMalloc(&e->d_fused, fused.size()) ||
        cudaMalloc(&e->d_partials, (size_t)e->blocks * 2 * sizeof(double)) ||
        cudaMalloc(&e->d_active, (size_t)(n + 1) * sizeof(int)) ||  // barrier counters + error flag
        cudaMalloc(&e->d_scal_ptrs, (size_t)n * sizeof(double*)) ||
        cudaMalloc(&e->d_scal_all, (size_t)n * 16 * sizeof(double)) ||
        cudaMallocHost(&e->h_scal_all, (size_t)n * 16 * sizeof(double)))
        return bail(fail(PIC_ERR_CUDA, "ensemble: allocation failed"));
    if (cudaMemset(e->d_active, 0, (size_t)(n + 1) * sizeof(int)) ||
        cudaMemcpy(e->d_fused, fused.data(), fused.size(), cudaMemcpyHostToDevice) ||
        cudaMemcpy(e->d_scal_ptrs, scal_ptrs.data(), (size_t)n * sizeof(double*), cudaMemcpyHostToDevice))
        return bail(fail(PIC_ERR_CUDA, "ensemble: table upload failed"));
    for (auto& v : e->ev)
        if (cudaEventCreate(&v) != cudaSuccess) return bail(fail(PIC_ERR_CUDA, "ensemble: event creation failed"));
    *out = e;
    return PIC_OK;
}

void pic_ensemble_destroy(pic_ensemble* e) {
    if (e) free_ensemble(e);
}

int pic_ensemble_size(pic_ensemble* e) { return e ? e->n : 0; }

pic_ctx* pic_ensemble_instance(pic_ensemble* e, int i) {
    if (!e || i < 0 || i >= e->n) {
        fail(PIC_ERR_ARG, "ensemble: instance index out of range");
        return nullptr;
    }
    return e->cs[i];
}

int pic_ensemble_use_graph(pic_ensemble* e, int on) {
    if (!e) return fail(PIC_ERR_ARG, "null ensemble");
    e->use_graph = on != 0;
    return PIC_OK;
}

int pic_ensemble_step(pic_ensemble* e, int iteration) {
    if (!e) return fail(PIC_ERR_ARG, "null ensemble");
    (void)iteration;
    // first step after loading: deposit the current positions (per instance)
    for (auto* c : e->cs)
        for (int s = 0; s < c->cfg.num_species; ++s)
            if (!c->sp[s].acc_fresh) PIC_TRY(particles_deposit(c, s));
    PIC_TRY(batch_prepare(e->pb, e->cs.data(), e->stream));
    PIC_TRY(upload_poisson(e));
    if (e->use_graph && !e->graph && !e->graph_failed) {
        cudaGraph_t g = nullptr;
        bool ok = cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
        const int st = ok ? enqueue_step(e, true) : PIC_ERR_CUDA;
        ok = (cudaStreamEndCapture(e->stream, &g) == cudaSuccess) && ok && st == PIC_OK;
        if (ok) ok = cudaGraphInstantiate(&e->graph, g, 0) == cudaSuccess;
        if (g) cudaGraphDestroy(g);
        if (!ok) {
            e->graph = nullptr;
            e->graph_failed = true;  // direct launches from now on
            cudaGetLastError();
        }
    }
    if (e->graph) {
        PIC_CUDA(cudaGraphLaunch(e->graph, e->stream));
    } else {
        PIC_TRY(enqueue_step(e, false));
    }
    PIC_CUDA(cudaStreamSynchronize(e->stream));
    batch_commit(e->cs.data(), e->n);
    // the events are recorded by the graph's event-record nodes (or directly)
    float t[3] = {0, 0, 0};
    for (int k = 0; k < 3; ++k) PIC_CUDA(cudaEventElapsedTime(&t[k], e->ev[k], e->ev[k + 1]));
    for (int k = 0; k < 3; ++k) e->last_ms[k] = t[k];
    int status = PIC_OK;
    for (int i = 0; i < e->n; ++i) {
        const int st = poisson_batch_finish(e->cs[i], e->h_scal_all + (size_t)i * 16, t[1]);
        if (st != PIC_OK && status == PIC_OK) status = st;
    }
    return status;
}

int pic_ensemble_timing(pic_ensemble* e, double* deposit_ms, double* poisson_ms, double* push_ms) {
    if (!e) return fail(PIC_ERR_ARG, "null ensemble");
    if (deposit_ms) *deposit_ms = e->last_ms[0];
    if (poisson_ms) *poisson_ms = e->last_ms[1];
    if (push_ms) *push_ms = e->last_ms[2];
    return PIC_OK;
}

int pic_ensemble_info(pic_ensemble* e, int* graph_active, int* tile_shape, int* solver_blocks) {
    if (!e) return fail(PIC_ERR_ARG, "null ensemble");
    if (graph_active) *graph_active = e->graph ? 1 : 0;
    if (tile_shape) *tile_shape = e->shape;
    if (solver_blocks) *solver_blocks = e->blocks;
    return PIC_OK;
}

int pic_ensemble_autotune(pic_ensemble* e, int* shape, double* ms_per_shape) {
    if (!e) return fail(PIC_ERR_ARG, "null ensemble");
    for (auto* c : e->cs) {
        if (!c->fields_valid) PIC_TRY(fields_from_phi(c));
    }
    PIC_TRY(batch_prepare(e->pb, e->cs.data(), e->stream));
    const int nsh = particles_num_tile_shapes();
    std::vector<double> ms((size_t)nsh, 0.0);
    PIC_TRY(batch_time_shapes(e->pb, e->cs.data(), e->stream, 3, e->energy, ms.data()));
    int best = 0;
    for (int k = 1; k < nsh; ++k)
        if (ms[k] < ms[best]) best = k;
    if (best != e->shape && e->graph) {
        cudaGraphExecDestroy(e->graph);  // captured with the old shape
        e->graph = nullptr;
    }
    e->shape = best;
    if (shape) *shape = best;
    if (ms_per_shape)
        for (int k = 0; k < nsh; ++k) ms_per_shape[k] = ms[k];
    return PIC_OK;
}

}  // extern "C"
