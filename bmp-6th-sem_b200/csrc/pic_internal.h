// pic_internal.h -- shared declarations of the B200 PIC library (not part of
// the public ABI).  Host C++17 + CUDA for sm_100a.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "pic_capi.h"

namespace picb200 {

// ---------------------------------------------------------------------------
// Error plumbing
// ---------------------------------------------------------------------------
void set_error(const std::string& msg);
int fail(int status, const std::string& msg);

#define PIC_CUDA(call)                                                              \
    do {                                                                            \
        cudaError_t e_ = (call);                                                    \
        if (e_ != cudaSuccess)                                                      \
            return ::picb200::fail(PIC_ERR_CUDA, std::string(#call) + ": " +        \
                                                     cudaGetErrorString(e_));       \
    } while (0)

#define PIC_TRY(call)                \
    do {                             \
        int s_ = (call);             \
        if (s_ != PIC_OK) return s_; \
    } while (0)

// ---------------------------------------------------------------------------
// Fixed-point deposit scales
// ---------------------------------------------------------------------------
// Each particle's bilinear weights are built from per-axis offsets rounded to
// 20 bits: qx = round(fx*2^20), so the four corner weights are exact 40-bit
// products that sum to exactly 2^40.  Node sums stay below 2^63 for up to
// 2^23 particles touching one node.
constexpr int kAxisBits = 20;
constexpr double kChargeUnit = 1.0 / 1099511627776.0;  // 2^-40
// The energy mesh (a diagnostic: printEnergy) uses each particle's kinetic
// energy, clamped below 1024 eV, times its FP32 corner weights, rounded to an
// integer number of 2^-22 eV: one contribution stays below 2^32.
constexpr double kEnergyUnit = 1.0 / 4194304.0;  // 2^-22
constexpr float kEnergyClampEv = 1023.9375f;      // (2^32 - 2^18) * 2^-22
// Particle slots a cell may hold (the per-lane moment sums of the deposit
// need at most 2^11 particles per lane).  A re-layout flags cells whose
// capacity would exceed it.
constexpr uint32_t kMaxPerCell = 1u << 16;

// ---------------------------------------------------------------------------
// Particle kernel tiling
// ---------------------------------------------------------------------------
constexpr int kWarps = 8;   // 256 threads per block (a tile of 256 cells)

struct SpeciesConsts {
    float h;          // 0.5*(q/m)*dt
    float dtdx, dtdy; // dt/dx, dt/dy
    float half_inv_abs_qm;  // 0.5/|q/m| -> kinetic energy in eV
    // uniform Bz (bzu != 0): the Boris rotation factors t = h*Bz and
    // s = 2t/(1+t^2), the same for every particle
    int bzu;
    float bt, bs;
    int pery;  // periodic in y: the cell row wraps modulo ny
};

// A particle as it crosses the host link: cell index (gy*nx + gx;
// kNoCell: dropped) and the FP32 state, 24 bytes where the reference Point
// has 56.  The host's thread pool converts between the two.
struct PointRec {
    uint32_t cell;
    float fx, fy, vx, vy, vz;
};
static_assert(sizeof(PointRec) == 24, "PointRec layout");
constexpr uint32_t kNoCell = 0xffffffffu;

// Cell-sorted state of one species (one buffer of a double buffer):
// a[i] = {fx, fy, vx, vy}, vz[i].
struct ParticleSoA {
    float4* a;
    float* vz;
};

// Particles held outside the cell layout (a mover that found its target
// cell full, or one that jumped more than one cell): state plus target cell.
struct LooseList {
    float4* a = nullptr;
    float* vz = nullptr;
    uint32_t* cell = nullptr;
    uint32_t* count = nullptr;  // device counter (entries may exceed cap: then lost)
    uint32_t cap = 0;
};

// Slot layout.  Cell c owns slots base[c] .. base[c+1] of each buffer; its
// particles are the front run base[c] .. base[c]+front[c] (those that stayed
// in the cell at the last push, or all of them after a re-layout) and the
// back run base[c+1]-back[c] .. base[c+1] (those that moved in).  The free
// gap between the runs absorbs the next push's incoming movers.
struct Species {
    pic_species_desc desc{};
    double ctom = 0, weighing = 0;
    SpeciesConsts k{};
    int64_t capacity = 0;           // slots per buffer
    float* store = nullptr;         // 2 buffers x 5 arrays x capacity floats
    ParticleSoA buf[2]{};
    int cur = 0;
    uint32_t* base = nullptr;       // [ncells+1] slot layout (both buffers)
    uint32_t* base_next = nullptr;  // [ncells+1] layout being built
    uint32_t* front[2] = {nullptr, nullptr};  // [ncells] per buffer
    uint32_t* back[2] = {nullptr, nullptr};   // [ncells] per buffer
    uint32_t* cnt = nullptr;        // [ncells] scratch: particles per cell
    uint32_t* dense = nullptr;      // [ncells+1] scratch: exclusive scan of cnt
    uint32_t* list_counts = nullptr;  // [4] device counters of the lists below
    LooseList ovf;                  // push output: not yet placed
    LooseList loose[2];             // [lcur]: part of the state, not yet placed
    int lcur = 0;
    uint32_t* host_flags = nullptr; // pinned: loose count + counters after the last push
    cudaEvent_t flags_ev = nullptr;
    bool flags_pending = false;
    unsigned long long* acc_q = nullptr;  // [nodes] fixed-point charge weights
    unsigned long long* acc_e = nullptr;  // [nodes] fixed-point energy weights
    double* final_mesh = nullptr;   // [nodes]
    double* energy_mesh = nullptr;  // [nodes]
    unsigned long long* counters = nullptr;  // [0] left exits, [1] cell limit, [2] lost particles
    bool acc_fresh = false;         // acc_* hold the deposit of the current positions
};

// Multigrid level (FP32).
// A multigrid level: GX x GY nodes.  Periodic in y, GY counts the distinct
// rows (the row above the last is row 0).
struct MGLevel {
    int nx, ny, GX, GY;
    int64_t nodes;
    float cx, cy, cd;  // 1/dx^2, 1/dy^2, 2(cx+cy)
    uint8_t* mask;     // 1 = Dirichlet
    float* x;
    float* b;
    float* xo;         // the up sweep's output (its tiles read x around them)
};

struct PoissonState {
    int solver = PIC_SOLVER_MG_PCG;
    int warm = PIC_WARM_PREVIOUS;
    double tol = 1e-8;
    int maxit = 500;
    std::vector<MGLevel> levels;
    double* r = nullptr;
    double* z = nullptr;
    double* p[2] = {nullptr, nullptr};
    double* q = nullptr;
    double* partials = nullptr;  // per-block partial dot products
    double* scal = nullptr;      // device scalars (see poisson.cu)
    double* host_scal = nullptr; // pinned mirror of scal
    int pcur = 0;
    int nblocks = 0;
    bool have_prev = false;
    int last_iters = 0;
    double last_relres = 0, last_ms = 0;
    double last_relres0 = 0;  // relative residual of the last solve's starting guess
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float* net_guess = nullptr;  // learned warm start output (nodes), optional
    // false: no multigrid hierarchy (periodic in y with an odd row count, or
    // a coarsest level too large for one block); the solve is
    // Jacobi-preconditioned
    bool mg_ok = true;
    // levels >= fused_first run in one thread block (k_mg_fused)
    int fused_first = 0;
    size_t fused_smem = 0;
    alignas(16) unsigned char fused_desc[1024] = {};
    // the PCG loop as a graph with a device-side while node, per solver
    cudaStream_t cap_stream = nullptr;
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    int body_nodes[2] = {0, 0};
    bool graph_failed = false;
    bool graph_off = false;  // pic_set_poisson_graph(ctx, 0): direct launches
    // exact coarse solve of levels[fused_first] (single contexts; poisson.cu)
    bool direct = false;
    int direct_nf = 0;
    float* direct_inv = nullptr;  // [nf][nf] FP32 inverse over the level's free nodes
    int* direct_free = nullptr;   // level node index of each free node
};

}  // namespace picb200

struct pic_ws;  // learned warm start (warmstart.cu)

struct pic_ctx {
    pic_config cfg{};
    int nx = 0, ny = 0, GX = 0, GY = 0;
    int64_t nodes = 0, ncells = 0;
    double dx = 0, dy = 0;
    // periodic in y: the potential is solved on node rows 0..GY-2 (row GY-1
    // repeats row 0); otherwise on all GY rows.  solve_nodes = GX*solve_rows.
    bool periodic = false;
    int solve_rows = 0;
    int64_t solve_nodes = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    // grids (device)
    double* rho = nullptr;
    double* phi = nullptr;
    double* bz = nullptr;          // FP64 node Bz
    float4* fld = nullptr;         // {Ex, Ey, Bz, 0} FP32 per node for the push
    uint8_t* mask = nullptr;       // electrode nodes
    double* dir_val = nullptr;     // electrode potential per node
    double* efield64 = nullptr;    // interleaved FP64 E for export
    // scratch shared by operators
    uint32_t* scan_partials = nullptr;
    void* staging = nullptr;       // device staging for host<->device copies
    size_t staging_bytes = 0;
    void* host_staging = nullptr;  // pinned host staging
    size_t host_staging_bytes = 0;
    void* pipe_buf[2] = {nullptr, nullptr};  // pinned chunks of the host<->device pipeline
    cudaEvent_t pipe_ev[2] = {nullptr, nullptr};
    picb200::Species sp[PIC_MAX_SPECIES];
    picb200::PoissonState ps;
    bool fields_valid = false;
    int tile_shape = 0;            // particle-kernel tile shape (see particles.cu)
    uint64_t source_calls = 0;     // particle-source calls (RNG counter)
    bool bz_uniform = true;        // every node has the same Bz (bz_value)
    double bz_value = 0.0;
    // instrumentation
    bool profiling = false;
    struct ProfEvent {
        int phase;
        cudaEvent_t a, b;
    };
    std::vector<ProfEvent> prof_pending;
    std::vector<cudaEvent_t> ev_pool;
    cudaEvent_t prof_open = nullptr;
    double prof_ms[PIC_NUM_PHASES] = {};
    int64_t prof_calls[PIC_NUM_PHASES] = {};
    int64_t launches = 0;
    // learned warm start
    pic_ws* ws = nullptr;
    bool ws_record = false;
};

namespace picb200 {

// context.cu: phase timing (no-ops unless profiling is on)
void prof_begin(pic_ctx* c, int phase);
void prof_end(pic_ctx* c, int phase);

// particles.cu
int species_setup(pic_ctx* c, int s);
int species_reserve(pic_ctx* c, int s, int64_t capacity);
void species_free(Species& sp);
// Stages n records for import; returns the device address to copy them to.
int particles_import_staging(pic_ctx* c, int64_t n, PointRec** dev_recs);
int particles_import(pic_ctx* c, int s, int64_t n);  // records already staged
int ensure_staging(pic_ctx* c, size_t bytes);
// The species as records in cell order (dev_out: n records).
int particles_export(pic_ctx* c, int s, PointRec* dev_out, int64_t* n_out);
int particles_load_plasma(pic_ctx* c, int s, const pic_plasma_desc* d);
// raw state into 6 consecutive arrays of n entries (int32 cell, 5 floats)
int particles_export_state(pic_ctx* c, int s, void* dev, int64_t n);
int particles_deposit(pic_ctx* c, int s);       // fresh deposit of current positions
int particles_flush_rho(pic_ctx* c, int s);     // acc -> final/energy mesh, rho +=
int particles_push(pic_ctx* c, int s);          // pass1 + scan + pass2 (+deposit)
int particles_count(pic_ctx* c, int s, int64_t* n);
int particles_bin_counts(pic_ctx* c, int s, int32_t* dev_counts);
// batched particle phases over an ensemble's contexts (particles.cu)
struct ParticleBatchImpl;
int batch_create(pic_ctx** cs, int n, ParticleBatchImpl** out);
void batch_destroy(ParticleBatchImpl* B);
int batch_prepare(ParticleBatchImpl* B, pic_ctx** cs, cudaStream_t st);
int batch_deposit(ParticleBatchImpl* B, cudaStream_t st);
int batch_push(ParticleBatchImpl* B, int shape, bool energy, cudaStream_t st);
void batch_commit(pic_ctx** cs, int n);
int batch_time_shapes(ParticleBatchImpl* B, pic_ctx** cs, cudaStream_t st, int reps, bool energy,
                      double* ms);
int particles_generate(pic_ctx* c, const pic_source_desc* d, int64_t* n_e, int64_t* n_p);
int particles_num_tile_shapes();
int particles_time_shapes(pic_ctx* c, int reps, double* ms);  // ms[particles_num_tile_shapes()]

// warmstart.cu
void ws_free(pic_ctx* c);
bool ws_tracking(const pic_ctx* c);  // hooks must run at every solve
int ws_before_solve(pic_ctx* c, bool want_guess);  // 1 when a guess is in ps.net_guess
int ws_check_fault();  // after a synchronisation: PIC_ERR_TIMEOUT if a warm-start kernel gave up
int ws_set_wait_limit(int64_t cycles);     // tensor-core pipeline wait bound (<= 0: default)
int poisson_set_spin_limit(int64_t polls); // batched-solve barrier poll bound (<= 0: default)
int ws_after_solve(pic_ctx* c, bool record);

// poisson.cu
int poisson_setup(pic_ctx* c);
void poisson_free(pic_ctx* c);
int poisson_debug_vcycle(pic_ctx* c, const float* rhs, float* out, int per_sweep);
int poisson_solve(pic_ctx* c);
int fields_from_phi(pic_ctx* c);
int overwrite_phi(pic_ctx* c);  // electrode nodes take their potential
int efield_export(pic_ctx* c);
int fields_set_bz(pic_ctx* c);
// batched solve of many contexts (poisson.cu)
size_t poisson_batch_desc_bytes();
size_t poisson_batch_max_fused_smem();
int poisson_batch_describe(pic_ctx* c, void* host_desc, const void* dev_fused, int blk0, int nblk);
const void* poisson_fused_table(pic_ctx* c, size_t* bytes);
size_t poisson_fused_smem(pic_ctx* c);
int poisson_batch_blocks(size_t smem, int* blocks);
int poisson_batch_launch(const void* dev_insts, int n, const int* inst_of, double* partials,
                         unsigned* barriers, int* err, size_t smem, int blocks, cudaStream_t st);
int poisson_batch_finish(pic_ctx* c, const double* scal, float ms);

}  // namespace picb200
