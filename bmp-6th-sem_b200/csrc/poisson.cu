// poisson.cu -- Poisson solve on the electrode mesh and the E field, sm_100a.
//
// Replaces (SYCL-PIC-poissonsolver/src/poissonSolver.cpp):
//   setPotentialBoundary + generateCoeffs (:64-79, :183-241): the 5-point
//     operator over all nodes, electrode rows fixed -- here matrix-free;
//   overwriteRho (:384-402): b = -rho, b = -V at electrode nodes -- done in
//     place on the device rho, as the reference does on the host;
//   PARDISO phases 11/22/33 (:505-535) -- here preconditioned CG:
//     * PIC_SOLVER_MG_PCG: FP64 CG (vectors, dot products, residual) with an
//       FP32 geometric-multigrid V-cycle as preconditioner;
//     * PIC_SOLVER_JACOBI_PCG: the plain path, FP64 CG with the diagonal;
//   overwritePhi (:364-382) and calculateElectricField (:433-456).
//
// The solve works on the reduced SPD system left after eliminating the
// electrode rows: for a non-electrode node i
//   (2/dx^2 + 2/dy^2) phi_i - (phi_w + phi_e)/dx^2 - (phi_s + phi_n)/dy^2 = b_i
// with electrode neighbours held at their potentials.  Convergence is
// ||b_red - A_red phi|| <= tol * ||b_red|| in the 2-norm over non-electrode
// nodes, b_red carrying the known electrode neighbours across.  Every wall
// node must be an electrode, as generateCoeffs requires.
//
// Dot products are reduced deterministically: per-block partials, then the
// last block to finish sums them in block order.
//
// Multigrid: vertex-centred coarsening nx_{l+1} = ceil(nx_l/2); coarse node I
// sits on fine node 2I; a coarse node is Dirichlet when its fine node is, or
// when it falls outside the fine grid.  Operators are rediscretised with
// spacing 2^l*dx; restriction is full weighting, prolongation bilinear, the
// smoother red-black Gauss-Seidel with the colour order reversed after the
// coarse correction, so the V-cycle is a symmetric preconditioner.  A level
// above the small ones is two kernels, all of its sweeps on shared-memory
// tiles with recomputed halos (k_mg_down, k_mg_up).  The small levels (from
// the first whose hierarchy fits a 16 KB budget) are either solved exactly
// -- the first of them inverted once at set-up, applied as one dense product
// (k_mg_direct) -- or, in the batched ensemble solve and when that level is
// too large, run inside one thread block (k_mg_fused: RB-GS on each, the
// coarsest with symmetric sweeps).
//
// The PCG loop is one CUDA graph: a while-conditional node whose body is one
// iteration (V-cycle with r.z, p update with A p, x/r update with the
// convergence test); the last kernel sets the condition on the device, so a
// solve costs one graph launch and one host synchronisation.  Without
// conditional-node support the same kernels run from a host loop.
#include <cooperative_groups.h>
#include <utility>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "pic_internal.h"

namespace picb200 {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kRedThreads = 256;
constexpr int kNu = 2;            // RB-GS sweeps before and after the coarse correction
constexpr int kCoarseSweeps = 8;  // symmetric sweep pairs on the coarsest level (<= 2 cells)

// device scalar slots
enum {
    S_BB = 0,   // ||b_red||^2
    S_RR = 1,   // ||r||^2
    S_RZ = 2,   // r.z (current)
    S_PQ = 3,   // p.Ap
    S_RZ_OLD = 4,
    S_TRUE_RR = 5,
    S_COUNT = 6,  // [6] is the arrival counter (as double bits)
    S_IT = 7,     // iterations done
    S_TOL2 = 8,   // tol^2
    S_MAXIT = 9,  // iteration limit
    S_STATUS = 10, // 0 running/converged, 1 iteration limit, 2 not finite
    S_RR0 = 11     // r.r of the solve's starting guess
};

struct Grid64 {
    int GX, GY;
    int64_t n;  // solved nodes: GX * (GY, or GY-1 when periodic in y)
    double cx, cy, cd;
};

// ---- deterministic block reduction with last-block finalisation ---------

// Returns true in the last block (after `out` is written).
template <int ND>
__device__ __forceinline__ bool reduce_finalize(double (&v)[ND], double* partials, int nblocks,
                                                unsigned int* arrive, double* out, int slot0) {
    __shared__ double sh[ND][kRedThreads / 32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        double x = v[d];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
        if (lane == 0) sh[d][warp] = x;
    }
    __syncthreads();
    const int bid = blockIdx.x + blockIdx.y * gridDim.x;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            double t = 0;
            for (int w = 0; w < kRedThreads / 32; ++w) t += sh[d][w];
            partials[(size_t)d * nblocks + bid] = t;
        }
        __threadfence();
        const unsigned prev = atomicAdd(arrive, 1u);
        last = (prev == (unsigned)nblocks - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    // the last block sums the partials in block order: fixed order, fixed result
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        double x = 0;
        // each thread owns a contiguous chunk, then a fixed-shape tree
        const int chunk = (nblocks + kRedThreads - 1) / kRedThreads;
        const int b0 = threadIdx.x * chunk;
        for (int b = b0; b < min(nblocks, b0 + chunk); ++b)
            x += ((volatile double*)partials)[(size_t)d * nblocks + b];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
        __syncthreads();
        if (lane == 0) sh[d][warp] = x;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0;
            for (int w = 0; w < kRedThreads / 32; ++w) t += sh[d][w];
            out[slot0 + d] = t;
        }
    }
    if (threadIdx.x == 0) *arrive = 0u;
    return true;
}

__device__ __forceinline__ double dirv(const uint8_t* mask, const double* dv, int64_t k) {
    return mask[k] ? dv[k] : 0.0;
}

// The nodes one row up / down, rows wrapping at n = GX * rows.  Periodic in
// y the system wraps (generateCoeffsPeriodic, src/poissonSolver.cpp:82-180);
// with walls the first and last rows are electrodes, whose stencils are
// never evaluated, so there the wrap is never taken.
template <typename I>
__device__ __forceinline__ I row_up(I k, I n, int GX) {
    const I u = k + GX;
    return u >= n ? u - n : u;
}
template <typename I>
__device__ __forceinline__ I row_dn(I k, I n, int GX) {
    const I d = k - GX;
    return d < 0 ? d + n : d;
}

// Programmatic dependent launch (the PCG iteration's kernels are launched
// with it): wait until the grid before this one in the stream has finished
// and its writes are visible, then let the next grid start launching its
// blocks, which wait here in turn.  The launch of each small kernel then
// overlaps the end of the one before.  Called first thing, by every thread.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;\n" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}

// overwriteRho (src/poissonSolver.cpp:384-402) in place: b = -rho, electrode
// nodes b = -V.  Also imposes the electrode potentials on phi and, for a
// zero warm start, clears phi.
__global__ void k_overwrite_rho(int64_t nodes, const uint8_t* mask, const double* dir_val,
                                double* rho, double* phi, int zero_start) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nodes) return;
    if (mask[i]) {
        rho[i] = -dir_val[i];
        phi[i] = dir_val[i];
    } else {
        rho[i] = -rho[i];
        if (zero_start) phi[i] = 0.0;
    }
}

__global__ void k_apply_guess(int64_t nodes, const uint8_t* mask, const float* guess, double* phi) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nodes || mask[i]) return;
    phi[i] = (double)guess[i];
}

// r = b - A x (0 at electrode nodes); r32 = (float)r; partials of r.r and
// b_red.b_red.
__global__ void __launch_bounds__(kRedThreads) k_pcg_setup(Grid64 g, const uint8_t* mask,
                                                           const double* dv, const double* b,
                                                           const double* x, double* r,
                                                           float* r32, double* partials,
                                                           int nblocks, unsigned* arrive,
                                                           double* scal) {
    const int64_t nodes = g.n;
    double acc[2] = {0.0, 0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nodes;
         i += (int64_t)gridDim.x * blockDim.x) {
        double ri = 0.0;
        if (!mask[i]) {
            const int64_t up = row_up(i, nodes, g.GX), dn = row_dn(i, nodes, g.GX);
            const double ax = g.cd * x[i] - g.cx * (x[i - 1] + x[i + 1]) - g.cy * (x[dn] + x[up]);
            ri = b[i] - ax;
            const double br = b[i] + g.cx * (dirv(mask, dv, i - 1) + dirv(mask, dv, i + 1)) +
                              g.cy * (dirv(mask, dv, dn) + dirv(mask, dv, up));
            acc[1] += br * br;
        }
        r[i] = ri;
        r32[i] = (float)ri;
        acc[0] += ri * ri;
    }
    reduce_finalize<2>(acc, partials, nblocks, arrive, scal, S_RR);
    // slots: S_RR = r.r, S_RR+1 = S_RZ holds bb temporarily; moved by k_fix_bb
}

__global__ void k_fix_bb(double* scal, double tol2, int maxit, int restart) {
    scal[S_BB] = scal[S_RZ];
    scal[S_RZ] = 0.0;
    scal[S_RZ_OLD] = 0.0;
    scal[S_TOL2] = tol2;
    scal[S_MAXIT] = (double)maxit;
    scal[S_STATUS] = 0.0;
    if (!restart) {
        scal[S_IT] = 0.0;
        scal[S_RR0] = scal[S_RR];
    }
}

// z = M^-1 r (from the MG output or the diagonal); partial r.z
__global__ void __launch_bounds__(kRedThreads) k_pcg_rz(int64_t nodes, const uint8_t* mask,
                                                        const double* r, const float* z32,
                                                        double inv_diag, int jacobi, double* z,
                                                        double* partials, int nblocks,
                                                        unsigned* arrive, double* scal) {
    pdl_enter();
    double acc[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nodes;
         i += (int64_t)gridDim.x * blockDim.x) {
        double zi = 0.0;
        if (!mask[i]) zi = jacobi ? r[i] * inv_diag : (double)z32[i];
        z[i] = zi;
        acc[0] += r[i] * zi;
    }
    reduce_finalize<1>(acc, partials, nblocks, arrive, scal, S_RZ);
}

// p = z + beta p and q = A p, the latter as A z + beta q (q holds A p of the
// previous direction), so one pass reads z's neighbours and no kernel
// boundary is needed between the two; partial p.q.  beta = rz/rz_old, 0 on
// the first iteration after a (re)start (marked by rz_old == 0).
// z is FP64 (k_pcg_rz's) or the V-cycle's FP32 output (0 at electrodes)
template <typename Z>
__global__ void __launch_bounds__(kRedThreads) k_pcg_pq(Grid64 g, const uint8_t* mask,
                                                        const Z* zs, double* p, double* q,
                                                        double* partials, int nblocks,
                                                        unsigned* arrive, double* scal) {
    pdl_enter();
    const double ro = scal[S_RZ_OLD];
    const double beta = ro == 0.0 ? 0.0 : scal[S_RZ] / ro;
    const int64_t nodes = g.n;
    auto z = [&](int64_t k) { return (double)zs[k]; };
    double acc[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nodes;
         i += (int64_t)gridDim.x * blockDim.x) {
        double pi = 0.0, qi = 0.0;
        if (!mask[i]) {
            const double az = g.cd * z(i) - g.cx * (z(i - 1) + z(i + 1)) -
                              g.cy * (z(row_dn(i, nodes, g.GX)) + z(row_up(i, nodes, g.GX)));
            // (after a restart p and q are not read: beta == 0)
            pi = beta == 0.0 ? z(i) : z(i) + beta * p[i];
            qi = beta == 0.0 ? az : az + beta * q[i];
        }
        p[i] = pi;
        q[i] = qi;
        acc[0] += pi * qi;
    }
    reduce_finalize<1>(acc, partials, nblocks, arrive, scal, S_PQ);
}

// x += alpha p; r -= alpha q; r32 = r; partial r.r.  Also shifts rz -> rz_old.
// The last block then ends the iteration: counts it, keeps rz for the next
// beta, decides whether to go on (and tells the graph's while node when
// there is one).
__global__ void __launch_bounds__(kRedThreads) k_pcg_update(int64_t nodes, const uint8_t* mask,
                                                            const double* p, const double* q,
                                                            double* x, double* r, float* r32,
                                                            double* partials, int nblocks,
                                                            unsigned* arrive, double* scal,
                                                            cudaGraphConditionalHandle handle,
                                                            int use_handle) {
    pdl_enter();
    const double alpha = scal[S_RZ] / scal[S_PQ];
    double acc[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nodes;
         i += (int64_t)gridDim.x * blockDim.x) {
        double ri = 0.0;
        if (!mask[i]) {
            x[i] += alpha * p[i];
            ri = r[i] - alpha * q[i];
        }
        r[i] = ri;
        r32[i] = (float)ri;
        acc[0] += ri * ri;
    }
    if (!reduce_finalize<1>(acc, partials, nblocks, arrive, scal, S_RR) || threadIdx.x != 0) return;
    const double it = scal[S_IT] + 1.0;
    scal[S_IT] = it;
    scal[S_RZ_OLD] = scal[S_RZ];
    const double rr = scal[S_RR];
    const bool finite = isfinite(rr);
    bool go = finite && rr > scal[S_TOL2] * scal[S_BB];
    if (go && it >= scal[S_MAXIT]) {
        go = false;
        scal[S_STATUS] = 1.0;
    }
    if (!finite) scal[S_STATUS] = 2.0;
    if (use_handle) cudaGraphSetConditional(handle, go ? 1u : 0u);
}

// true residual of the final iterate (reported relres)
__global__ void __launch_bounds__(kRedThreads) k_true_residual(Grid64 g, const uint8_t* mask,
                                                               const double* b, const double* x,
                                                               double* partials, int nblocks,
                                                               unsigned* arrive, double* scal) {
    const int64_t nodes = g.n;
    double acc[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nodes;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (!mask[i]) {
            const double ax = g.cd * x[i] - g.cx * (x[i - 1] + x[i + 1]) -
                              g.cy * (x[row_dn(i, nodes, g.GX)] + x[row_up(i, nodes, g.GX)]);
            const double ri = b[i] - ax;
            acc[0] += ri * ri;
        }
    }
    reduce_finalize<1>(acc, partials, nblocks, arrive, scal, S_TRUE_RR);
}

// ---- multigrid (FP32) ------------------------------------------------------

// icd = 1 / cd (rounded once): the Gauss-Seidel updates multiply by it
struct LevelDev {
    int nx, ny, GX, GY;
    float cx, cy, cd, icd;
    const uint8_t* mask;
    float* x;
    float* b;
};

__host__ __device__ __forceinline__ LevelDev as_dev(const MGLevel& L) {
    return LevelDev{L.nx, L.ny, L.GX, L.GY, L.cx, L.cy, L.cd, 1.0f / L.cd, L.mask, L.x, L.b};
}

// one Gauss-Seidel half sweep over the nodes of one colour
__global__ void k_mg_rbgs(LevelDev L, int color) {
    pdl_enter();
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = 2 * h + ((j + color) & 1);
    if (i >= L.GX || j >= L.GY) return;
    const int k = j * L.GX + i, n = L.GX * L.GY;
    if (L.mask[k]) return;
    const float s = __fmaf_rn(L.cx, L.x[k - 1] + L.x[k + 1],
                              __fmaf_rn(L.cy, L.x[row_dn(k, n, L.GX)] + L.x[row_up(k, n, L.GX)], L.b[k]));
    L.x[k] = s * L.icd;
}

// b - A x at one node from its value c and its neighbours west, east, down,
// up; every operation rounded as written (no contraction), so each kernel
// that computes a residual gets the same bits
__device__ __forceinline__ float mg_residual(float b, float c, float w, float e, float d, float u,
                                             float cx, float cy, float cd) {
    const float ax = __fsub_rn(__fsub_rn(__fmul_rn(cd, c), __fmul_rn(cx, __fadd_rn(w, e))),
                               __fmul_rn(cy, __fadd_rn(d, u)));
    return __fsub_rn(b, ax);
}

// Residual at fine node (i, j); 0 outside the x range and at electrodes.
// Rows wrap (only reached periodic in y: with walls the restriction of an
// interior coarse node stays inside the fine rows).
__device__ __forceinline__ float fine_residual(const LevelDev& F, int i, int j) {
    if (i < 0 || i >= F.GX) return 0.0f;
    j = j < 0 ? j + F.GY : (j >= F.GY ? j - F.GY : j);
    const int k = j * F.GX + i, n = F.GX * F.GY;
    if (F.mask[k]) return 0.0f;
    return mg_residual(F.b[k], F.x[k], F.x[k - 1], F.x[k + 1], F.x[row_dn(k, n, F.GX)],
                       F.x[row_up(k, n, F.GX)], F.cx, F.cy, F.cd);
}

// b_coarse = full weighting of the fine residual
__global__ void k_mg_restrict(LevelDev F, LevelDev C) {
    pdl_enter();
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    const int J = blockIdx.y * blockDim.y + threadIdx.y;
    if (I >= C.GX || J >= C.GY) return;
    const int64_t kc = (int64_t)J * C.GX + I;
    if (C.mask[kc]) {
        C.b[kc] = 0.0f;
        return;
    }
    const int i = 2 * I, j = 2 * J;
    float s = 4.0f * fine_residual(F, i, j);
    s += 2.0f * (fine_residual(F, i - 1, j) + fine_residual(F, i + 1, j) +
                 fine_residual(F, i, j - 1) + fine_residual(F, i, j + 1));
    s += fine_residual(F, i - 1, j - 1) + fine_residual(F, i + 1, j - 1) +
         fine_residual(F, i - 1, j + 1) + fine_residual(F, i + 1, j + 1);
    C.b[kc] = s * 0.0625f;
}

// The first black half sweep after a zero start or after the coarse
// correction, fused with what precedes it.  A Gauss-Seidel update of a node
// reads only its neighbours, and the red sweep that follows overwrites every
// red node without reading it, so the red values these steps would write
// are only needed here: each black node computes its four red neighbours'
// values itself (the same arithmetic as the separate kernels, so the same
// bits) and nothing else is written.  Both need kNu >= 2 (a red sweep
// before anything reads red nodes again).
static_assert(kNu >= 2, "the fused first sweeps need a later red sweep");

// zero start: red x = b/cd (Dirichlet 0), then the black sweep
__global__ void k_mg_init_black(LevelDev L) {
    pdl_enter();
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = 2 * h + ((j + 1) & 1);
    if (i >= L.GX || j >= L.GY) return;
    const int k = j * L.GX + i, n = L.GX * L.GY;
    if (L.mask[k]) return;
    auto xr = [&](int m) { return L.mask[m] ? 0.0f : L.b[m] * L.icd; };
    const float s = __fmaf_rn(L.cx, xr(k - 1) + xr(k + 1),
                              __fmaf_rn(L.cy, xr(row_dn(k, n, L.GX)) + xr(row_up(k, n, L.GX)), L.b[k]));
    L.x[k] = s * L.icd;
}

// x at fine node (i, j) plus the bilinear interpolation of the coarse
// correction (Dirichlet nodes unchanged)
__device__ __forceinline__ float prolonged(const LevelDev& F, const LevelDev& C, int i, int j) {
    const int k = j * F.GX + i;
    if (F.mask[k]) return F.x[k];
    const int I = i >> 1, J = j >> 1;
    const int J1 = J + 1 == C.GY ? 0 : J + 1;  // wraps only periodic in y
    const bool ox = i & 1, oy = j & 1;
    auto X = [&](int a, int b) { return C.x[(int64_t)b * C.GX + a]; };
    float v;
    if (!ox && !oy) v = X(I, J);
    else if (ox && !oy) v = 0.5f * (X(I, J) + X(I + 1, J));
    else if (!ox && oy) v = 0.5f * (X(I, J) + X(I, J1));
    else v = 0.25f * (X(I, J) + X(I + 1, J) + X(I, J1) + X(I + 1, J1));
    return F.x[k] + v;
}

// coarse correction, then the black sweep
__global__ void k_mg_prolong_black(LevelDev F, LevelDev C) {
    pdl_enter();
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = 2 * h + ((j + 1) & 1);
    if (i >= F.GX || j >= F.GY) return;
    const int k = j * F.GX + i;
    if (F.mask[k]) return;
    const int jd = j == 0 ? F.GY - 1 : j - 1, ju = j + 1 == F.GY ? 0 : j + 1;
    const float s = __fmaf_rn(F.cx, prolonged(F, C, i - 1, j) + prolonged(F, C, i + 1, j),
                              __fmaf_rn(F.cy, prolonged(F, C, i, jd) + prolonged(F, C, i, ju), F.b[k]));
    F.x[k] = s * F.icd;
}


// ---- a whole level a kernel (temporal blocking) ----------------------------
//
// The per-sweep kernels above take 4 kNu launches a level, each a full pass
// over the level's nodes.  Here a block copies a tile of the level, with a
// halo, into shared memory and runs all of the level's sweeps there, the
// region it has right shrinking by one node a sweep; only the tile's core is
// written back.  Every node goes through the operations of the per-sweep
// kernels in the same order, so the iterates are the same bits; the halo
// nodes are recomputed by each neighbouring tile.
//   k_mg_down: zero start, black, (red, black) x (kNu - 1), residual and its
//     full weighting into the coarse right-hand side.  Core 32 x 32 fine
//     nodes (16 x 16 coarse), halo 2 kNu + 1 (sweeps, residual, weighting).
//   k_mg_up: coarse correction, black, red, (black, red) x (kNu - 1).  Core
//     32 x 32, halo 2 kNu.  Its halo reads the level's x where neighbouring
//     tiles write their cores, so it writes a second array (MGLevel::xo).
// Region rows wrap at the level's row count like row_up / row_dn (only
// periodic in y matters: with walls the first and last rows are electrodes,
// never updated, so nothing crosses them); a level smaller than the region
// just appears more than once in it, each copy updated alike.  Columns left
// and right of the level are electrodes of value 0 (the x walls are
// electrodes, so their values are never used).
constexpr int kTileCore = 32;
constexpr int kDownHalo = 2 * kNu + 1;
constexpr int kUpHalo = 2 * kNu;
constexpr int kDownSide = kTileCore + 2 * kDownHalo;
constexpr int kUpSide = kTileCore + 2 * kUpHalo;
constexpr int kUpCoarse = kUpSide / 2 + 1;  // coarse nodes under an up tile, a side
static_assert(kUpHalo % 2 == 0, "up tiles start on an even node");
constexpr int kTileThreads = 256;      // the finest level's kernels (and r.z)
constexpr int kTileThreadsSmall = 1024; // levels of fewer tiles than two per SM: shorter chains
static_assert(kDownSide % 2 == 0 && kUpSide % 2 == 0, "tile rows hold as many nodes of each colour");

// level row of region row j (rows wrap at the level's row count)
__device__ __forceinline__ int tile_row(int j, int GY) {
    j %= GY;
    return j < 0 ? j + GY : j;
}

// Region nodes a thread loads: all its loads are issued before the first
// result is used (the load phase is one round trip to memory, not one per
// node).
template <int S, int NT>
constexpr int tile_loads() { return (S * S + NT - 1) / NT; }

// one colour over the region's inner nodes (k_mg_rbgs's arithmetic); region
// node (li, lj) is level node (i0 + li, j0 + lj), colour (i + j) & 1 (rows
// wrap only at an even row count, so wrapping keeps the colour)
template <int S, int NT>
__device__ __forceinline__ void tile_half_sweep(float* x, const float* b, const uint8_t* m, float cx,
                                                float cy, float icd, int color, int i0, int j0) {
    constexpr int HS = S / 2;
    for (int h = threadIdx.x; h < HS * S; h += NT) {
        const int lj = h / HS;
        const int li = 2 * (h - lj * HS) + ((i0 + j0 + lj + color) & 1);
        const int t = lj * S + li;
        if (li == 0 || lj == 0 || li == S - 1 || lj == S - 1 || m[t]) continue;
        const float s = __fmaf_rn(cx, x[t - 1] + x[t + 1], __fmaf_rn(cy, x[t - S] + x[t + S], b[t]));
        x[t] = s * icd;
    }
    __syncthreads();
}

// level F's smoothing from a zero start, then C.b = restriction of F's residual
template <int NT>
__global__ void __launch_bounds__(NT) k_mg_down(LevelDev F, LevelDev C) {
    constexpr int S = kDownSide, H = kDownHalo, CC = kTileCore / 2;
    __shared__ float sx[S * S], sb[S * S], sr[S * S];
    __shared__ uint8_t sm[S * S];
    pdl_enter();
    const int I0 = blockIdx.x * CC, J0 = blockIdx.y * CC;  // first coarse node of the tile
    const int i0 = 2 * I0 - H, j0 = 2 * J0 - H;            // level node of region node (0, 0)
    {
        constexpr int NL = tile_loads<S, NT>();
        int kk[NL];
        uint8_t mv[NL];
        float bv[NL];
#pragma unroll
        for (int u = 0; u < NL; ++u) {
            const int t = threadIdx.x + u * NT, li = t % S, lj = t / S, i = i0 + li;
            kk[u] = (t < S * S && i >= 0 && i < F.GX) ? tile_row(j0 + lj, F.GY) * F.GX + i : -1;
        }
#pragma unroll
        for (int u = 0; u < NL; ++u) {
            mv[u] = kk[u] < 0 ? 1 : F.mask[kk[u]];
            bv[u] = kk[u] < 0 ? 0.0f : F.b[kk[u]];
        }
#pragma unroll
        for (int u = 0; u < NL; ++u) {
            const int t = threadIdx.x + u * NT, li = t % S, lj = t / S;
            if (t >= S * S) break;
            sm[t] = mv[u];
            sb[t] = bv[u];
            // zero start: the black sweep reads red x = b / cd (electrodes 0;
            // as a product with icd, like every update);
            // black values are written before anything reads them
            sx[t] = (!mv[u] && ((i0 + li + j0 + lj) & 1) == 0) ? bv[u] * F.icd : 0.0f;
        }
    }
    __syncthreads();
    tile_half_sweep<S, NT>(sx, sb, sm, F.cx, F.cy, F.icd, 1, i0, j0);
    for (int s = 1; s < kNu; ++s) {
        tile_half_sweep<S, NT>(sx, sb, sm, F.cx, F.cy, F.icd, 0, i0, j0);
        tile_half_sweep<S, NT>(sx, sb, sm, F.cx, F.cy, F.icd, 1, i0, j0);
    }
    for (int t = threadIdx.x; t < S * S; t += NT) {
        const int li = t % S, lj = t / S;
        float rv = 0.0f;
        if (li > 0 && lj > 0 && li < S - 1 && lj < S - 1 && !sm[t])
            rv = mg_residual(sb[t], sx[t], sx[t - 1], sx[t + 1], sx[t - S], sx[t + S], F.cx, F.cy, F.cd);
        sr[t] = rv;
        const int i = i0 + li, j = j0 + lj;
        if (li >= H && lj >= H && li < H + kTileCore && lj < H + kTileCore && !sm[t] && j < F.GY)
            F.x[j * F.GX + i] = sx[t];
    }
    __syncthreads();
    // full weighting, in k_mg_restrict's order
    for (int t = threadIdx.x; t < CC * CC; t += NT) {
        const int I = I0 + t % CC, J = J0 + t / CC;
        if (I >= C.GX || J >= C.GY) continue;
        const int64_t kc = (int64_t)J * C.GX + I;
        if (C.mask[kc]) {
            C.b[kc] = 0.0f;
            continue;
        }
        const int c = (2 * J - j0) * S + (2 * I - i0);
        float s = 4.0f * sr[c];
        s += 2.0f * (sr[c - 1] + sr[c + 1] + sr[c - S] + sr[c + S]);
        s += sr[c - S - 1] + sr[c - S + 1] + sr[c + S - 1] + sr[c + S + 1];
        C.b[kc] = s * 0.0625f;
    }
}

// Where the finest level's k_mg_up also starts the PCG iteration: z is its
// output (FP32, electrodes 0), and it reduces r.z into scal[S_RZ] like
// k_pcg_rz (per-block partials over the tile cores, summed in block order).
struct RzArgs {
    const double* r;
    double* partials;
    unsigned* arrive;
    double* scal;
};


// xo = level F's x corrected by C.x and smoothed; with kRz also r.z
template <bool kRz, int NT>
__global__ void __launch_bounds__(NT) k_mg_up(LevelDev F, LevelDev C, float* xo, RzArgs R) {
    static_assert(!kRz || NT == kRedThreads, "the r.z reduction is the PCG block reduction");
    constexpr int S = kUpSide, H = kUpHalo;
    __shared__ float sx[S * S], sb[S * S], sc[kUpCoarse * kUpCoarse];
    __shared__ uint8_t sm[S * S];
    pdl_enter();
    const int i0 = blockIdx.x * kTileCore - H, j0 = blockIdx.y * kTileCore - H;
    {
        // the coarse correction's tile first: coarse nodes (i0 / 2 + a,
        // j0 / 2 + b), rows wrapped like the fine ones (periodic in y the row
        // counts are even, so (j mod GY) / 2 = (j / 2) mod (GY / 2)); columns
        // outside the level read 0 (only electrode or outside nodes use them)
        const int I0 = i0 >> 1, J0 = j0 >> 1;
        for (int t = threadIdx.x; t < kUpCoarse * kUpCoarse; t += NT) {
            const int I = I0 + t % kUpCoarse, J = tile_row(J0 + t / kUpCoarse, C.GY);
            sc[t] = (I >= 0 && I < C.GX) ? C.x[J * C.GX + I] : 0.0f;
        }
        // the node's mask, b and x, all loaded before any is used
        constexpr int NL = tile_loads<S, NT>();
        int kk[NL];
        uint8_t mv[NL];
        float bv[NL], xv[NL];
#pragma unroll
        for (int u = 0; u < NL; ++u) {
            const int t = threadIdx.x + u * NT, i = i0 + t % S;
            const int j = tile_row(j0 + t / S, F.GY);
            kk[u] = (t < S * S && i >= 0 && i < F.GX) ? j * F.GX + i : -1;
        }
#pragma unroll
        for (int u = 0; u < NL; ++u) {
            const bool in = kk[u] >= 0;
            mv[u] = in ? F.mask[kk[u]] : 1;
            bv[u] = in ? F.b[kk[u]] : 0.0f;
            xv[u] = in ? F.x[kk[u]] : 0.0f;
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < NL; ++u) {
            const int t = threadIdx.x + u * NT, li = t % S, lj = t / S, i = i0 + li;
            if (t >= S * S) break;
            sm[t] = mv[u];
            sb[t] = bv[u];
            float v = xv[u];
            if (!mv[u]) {
                // prolonged(): x + the bilinear interpolation of the coarse correction
                const int j = j0 + lj;
                const bool ox = i & 1, oy = j & 1;
                const float* c = sc + ((j >> 1) - J0) * kUpCoarse + ((i >> 1) - I0);
                float cv;
                if (!ox && !oy) cv = c[0];
                else if (ox && !oy) cv = 0.5f * (c[0] + c[1]);
                else if (!ox && oy) cv = 0.5f * (c[0] + c[kUpCoarse]);
                else cv = 0.25f * (c[0] + c[1] + c[kUpCoarse] + c[kUpCoarse + 1]);
                v = xv[u] + cv;
            }
            sx[t] = v;
        }
    }
    __syncthreads();
    tile_half_sweep<S, NT>(sx, sb, sm, F.cx, F.cy, F.icd, 1, i0, j0);
    tile_half_sweep<S, NT>(sx, sb, sm, F.cx, F.cy, F.icd, 0, i0, j0);
    for (int s = 1; s < kNu; ++s) {
        tile_half_sweep<S, NT>(sx, sb, sm, F.cx, F.cy, F.icd, 1, i0, j0);
        tile_half_sweep<S, NT>(sx, sb, sm, F.cx, F.cy, F.icd, 0, i0, j0);
    }
    double acc[1] = {0.0};
    for (int t = threadIdx.x; t < kTileCore * kTileCore; t += NT) {
        const int li = H + t % kTileCore, lj = H + t / kTileCore;
        const int i = i0 + li, j = j0 + lj;
        if (i >= F.GX || j >= F.GY || sm[lj * S + li]) continue;
        const float z = sx[lj * S + li];
        xo[j * F.GX + i] = z;
        if (kRz) acc[0] += R.r[j * F.GX + i] * (double)z;
    }
    if (kRz) reduce_finalize<1>(acc, R.partials, gridDim.x * gridDim.y, R.arrive, R.scal, S_RZ);
}


// All levels from `first` down to the coarsest in one thread block, in
// shared memory: the same operations as the per-level kernels (zero-start red
// sweep, black, (red, black) x (kNu-1), restrict; coarsest: symmetric sweeps;
// then prolong + (black, red) x kNu), with block barriers between them.
constexpr int kMaxFused = 12;
constexpr int kFusedThreads = 1024;

struct FusedLevels {
    int n;  // fused levels
    int GX[kMaxFused], GY[kMaxFused];
    float cx[kMaxFused], cy[kMaxFused], cd[kMaxFused];
    int ox[kMaxFused], ob[kMaxFused], om[kMaxFused];  // byte offsets in shared memory
    uint32_t rcp_hw[kMaxFused];  // ceil(2^32 / ceil(GX/2))
    const uint8_t* gmask[kMaxFused];
    const float* gb;  // right-hand side of the first fused level
    float* gx;        // its solution (output)
    int sweeps;
    int small;  // first level worked by warp 0 alone (n: none)
    int mpre[kMaxFused + 1];  // prefix sums of the levels' node counts
};
// every thread's share of the masks and of the first level's b, loaded in
// one round trip (the setup keeps the fused levels within this)
constexpr int kFusedLoads = 8;

__device__ __forceinline__ void fused_body(const FusedLevels& F, unsigned char* smem) {
    auto X = [&](int l) { return reinterpret_cast<float*>(smem + F.ox[l]); };
    auto B = [&](int l) { return reinterpret_cast<float*>(smem + F.ob[l]); };
    auto M = [&](int l) { return reinterpret_cast<uint8_t*>(smem + F.om[l]); };
    const int tid = threadIdx.x;
    {
        const int n0 = F.GX[0] * F.GY[0], total = F.mpre[F.n];
        uint8_t mv[kFusedLoads];
        float bv[kFusedLoads];
        int lv[kFusedLoads];
#pragma unroll
        for (int u = 0; u < kFusedLoads; ++u) {
            const int k = tid + u * kFusedThreads;
            int l = 0;
            while (l + 1 < F.n && k >= F.mpre[l + 1]) ++l;
            lv[u] = l;
            mv[u] = k < total ? F.gmask[l][k - F.mpre[l]] : 0;
            bv[u] = k < n0 ? F.gb[k] : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < kFusedLoads; ++u) {
            const int k = tid + u * kFusedThreads;
            if (k < total) M(lv[u])[k - F.mpre[lv[u]]] = mv[u];
            if (k < n0) B(0)[k] = bv[u];
        }
    }
    __syncthreads();
    // Levels from F.small on are worked by warp 0 alone, with warp barriers
    // between the phases (a block barrier of 1024 threads costs more than
    // the few hundred nodes of such a level); the others by the whole block.
    const int ls = F.small;
    auto stride = [&](int l) { return l >= ls ? 32 : kFusedThreads; };
    auto sync = [&](int l) {
        if (l >= ls) __syncwarp();
        else __syncthreads();
    };
    // one colour: h enumerates (row, half-column); hw = ceil(GX/2), and
    // h / hw comes from a 32-bit reciprocal (exact for these sizes)
    auto sweep = [&](int l, int color) {
        const int GX = F.GX[l], GY = F.GY[l], hw = (GX + 1) >> 1;
        const uint32_t rcp = F.rcp_hw[l];
        float* x = X(l);
        const float* b = B(l);
        const uint8_t* m = M(l);
        const float cx = F.cx[l], cy = F.cy[l], icd = 1.0f / F.cd[l];
        for (int h = tid; h < hw * GY; h += stride(l)) {
            const int j = (int)__umulhi((uint32_t)h, rcp);
            const int i = 2 * (h - j * hw) + ((j + color) & 1);
            if (i >= GX) continue;
            const int k = j * GX + i, n = GX * GY;
            if (m[k]) continue;
            x[k] = __fmaf_rn(cx, x[k - 1] + x[k + 1],
                             __fmaf_rn(cy, x[row_dn(k, n, GX)] + x[row_up(k, n, GX)], b[k])) * icd;
        }
        sync(l);
    };
    auto residual = [&](int l, int i, int j) -> float {
        const int GX = F.GX[l], GY = F.GY[l];
        if (i < 0 || i >= GX) return 0.0f;
        j = j < 0 ? j + GY : (j >= GY ? j - GY : j);  // wraps only periodic in y
        const int k = j * GX + i, n = GX * GY;
        if (M(l)[k]) return 0.0f;
        const float* x = X(l);
        const float ax = F.cd[l] * x[k] - F.cx[l] * (x[k - 1] + x[k + 1]) -
                         F.cy[l] * (x[row_dn(k, n, GX)] + x[row_up(k, n, GX)]);
        return B(l)[k] - ax;
    };
    // zero start, smoothing, restriction into level l + 1
    auto down = [&](int l) {
        const int GX = F.GX[l], n = GX * F.GY[l];
        for (int k = tid; k < n; k += stride(l)) {
            const int i = k % GX, j = k / GX;
            X(l)[k] = (((i + j) & 1) == 0 && !M(l)[k]) ? B(l)[k] / F.cd[l] : 0.0f;
        }
        sync(l);
        sweep(l, 1);
        for (int s = 1; s < kNu; ++s) {
            sweep(l, 0);
            sweep(l, 1);
        }
        const int CGX = F.GX[l + 1], cn = CGX * F.GY[l + 1];
        for (int kc = tid; kc < cn; kc += stride(l)) {
            if (M(l + 1)[kc]) {
                B(l + 1)[kc] = 0.0f;
                continue;
            }
            const int i = 2 * (kc % CGX), j = 2 * (kc / CGX);
            float s = 4.0f * residual(l, i, j);
            s += 2.0f * (residual(l, i - 1, j) + residual(l, i + 1, j) + residual(l, i, j - 1) +
                         residual(l, i, j + 1));
            s += residual(l, i - 1, j - 1) + residual(l, i + 1, j - 1) + residual(l, i - 1, j + 1) +
                 residual(l, i + 1, j + 1);
            B(l + 1)[kc] = s * 0.0625f;
        }
        sync(l);
    };
    // coarsest level: symmetric sweeps from zero
    auto coarsest = [&]() {
        const int l = F.n - 1, n = F.GX[l] * F.GY[l];
        for (int k = tid; k < n; k += stride(l)) X(l)[k] = 0.0f;
        sync(l);
        for (int s = 0; s < F.sweeps; ++s) {
            sweep(l, 0);
            sweep(l, 1);
        }
        for (int s = 0; s < F.sweeps; ++s) {
            sweep(l, 1);
            sweep(l, 0);
        }
    };
    // coarse correction from level l + 1, then smoothing
    auto up = [&](int l) {
        const int GX = F.GX[l], n = GX * F.GY[l], CGX = F.GX[l + 1];
        const float* xc = X(l + 1);
        for (int k = tid; k < n; k += stride(l)) {
            if (M(l)[k]) continue;
            const int i = k % GX, j = k / GX, I = i >> 1, J = j >> 1;
            const int J1 = J + 1 == F.GY[l + 1] ? 0 : J + 1;  // wraps only periodic in y
            const bool ox = i & 1, oy = j & 1;
            float v;
            if (!ox && !oy) v = xc[J * CGX + I];
            else if (ox && !oy) v = 0.5f * (xc[J * CGX + I] + xc[J * CGX + I + 1]);
            else if (!ox && oy) v = 0.5f * (xc[J * CGX + I] + xc[J1 * CGX + I]);
            else v = 0.25f * (xc[J * CGX + I] + xc[J * CGX + I + 1] + xc[J1 * CGX + I] + xc[J1 * CGX + I + 1]);
            X(l)[k] += v;
        }
        sync(l);
        for (int s = 0; s < kNu; ++s) {
            sweep(l, 1);
            sweep(l, 0);
        }
    };
    const int last = F.n - 1;
    for (int l = 0; l < last && l < ls; ++l) down(l);
    if (tid < 32) {  // the small levels (a no-op when there are none)
        for (int l = ls; l < last; ++l) down(l);
        if (last >= ls) coarsest();
        for (int l = last - 1; l >= ls; --l) up(l);
    }
    if (last < ls) coarsest();
    __syncthreads();
    for (int l = min(ls, last) - 1; l >= 0; --l) up(l);
    {
        const int n = F.GX[0] * F.GY[0];
        for (int k = tid; k < n; k += kFusedThreads) F.gx[k] = X(0)[k];
    }
}

__global__ void __launch_bounds__(kFusedThreads) k_mg_fused(FusedLevels F) {
    pdl_enter();
    extern __shared__ __align__(16) unsigned char smem[];
    fused_body(F, smem);
}

// ---- exact solve of the first fused level (single contexts) -------------------
//
// Below the tiled levels the V-cycle needs the coarse-grid correction, the
// solution of that level's own system A x = b (Dirichlet 0 at its
// electrodes).  When the level has at most kDirectMax free nodes the
// library inverts A once at set-up (FP64 Cholesky on the host, the inverse
// kept in FP32 on the device) and the correction is one dense product in a
// multi-block kernel (k_mg_direct), in place of the one-block chain of
// smaller levels (k_mg_fused, still used by the batched ensemble solve).
// The exact coarse solve is symmetric positive definite, so the
// preconditioner stays a valid one for CG.
constexpr int kDirectMax = 1200;

// inverse of the level's operator over its free nodes (row-major, nf x nf),
// or false when Cholesky breaks down (not positive definite)
static bool invert_level(int GX, int GY, double cx, double cy, double cd, const std::vector<uint8_t>& mask,
                         std::vector<int>& freen, std::vector<float>& inv) {
    const int n = GX * GY;
    std::vector<int> fidx(n, -1);
    freen.clear();
    for (int k = 0; k < n; ++k)
        if (!mask[k]) {
            fidx[k] = (int)freen.size();
            freen.push_back(k);
        }
    const int nf = (int)freen.size();
    std::vector<double> A((size_t)nf * nf, 0.0);
    for (int f = 0; f < nf; ++f) {
        const int k = freen[f];
        A[(size_t)f * nf + f] += cd;
        const int up = k + GX >= n ? k + GX - n : k + GX, dn = k - GX < 0 ? k - GX + n : k - GX;
        const int nb[4] = {k - 1, k + 1, dn, up};
        const double cf[4] = {cx, cx, cy, cy};
        for (int e = 0; e < 4; ++e) {
            const int g = (nb[e] >= 0 && nb[e] < n) ? fidx[nb[e]] : -1;
            if (g >= 0) A[(size_t)f * nf + g] -= cf[e];
        }
    }
    // envelope: first nonzero column of each row (fill-in stays inside it)
    std::vector<int> first(nf);
    for (int i = 0; i < nf; ++i) {
        int j = 0;
        while (j < i && A[(size_t)i * nf + j] == 0.0) ++j;
        first[i] = j;
    }
    // in-place Cholesky, lower triangle: A = L L^T
    for (int j = 0; j < nf; ++j) {
        double* Lj = &A[(size_t)j * nf];
        double s = Lj[j];
        for (int k = first[j]; k < j; ++k) s -= Lj[k] * Lj[k];
        if (!(s > 0.0)) return false;
        Lj[j] = std::sqrt(s);
        for (int i = j + 1; i < nf; ++i) {
            if (first[i] > j) continue;
            double* Li = &A[(size_t)i * nf];
            double t = Li[j];
            for (int k = std::max(first[i], first[j]); k < j; ++k) t -= Li[k] * Lj[k];
            Li[j] = t / Lj[j];
        }
    }
    // columns of the inverse: L y = e_c, then L^T x = y
    std::vector<std::vector<int>> below(nf);  // rows k > i with L[k][i] in the envelope
    for (int k = 0; k < nf; ++k)
        for (int i = first[k]; i < k; ++i) below[i].push_back(k);
    inv.assign((size_t)nf * nf, 0.f);
    std::vector<double> y(nf), x(nf);
    for (int c = 0; c < nf; ++c) {
        for (int i = 0; i < c; ++i) y[i] = 0.0;
        for (int i = c; i < nf; ++i) {
            const double* Li = &A[(size_t)i * nf];
            double t = i == c ? 1.0 : 0.0;
            for (int k = std::max(first[i], c); k < i; ++k) t -= Li[k] * y[k];
            y[i] = t / Li[i];
        }
        for (int i = nf - 1; i >= 0; --i) {
            double t = y[i];
            for (int k : below[i]) t -= A[(size_t)k * nf + i] * x[k];
            x[i] = t / A[(size_t)i * nf + i];
        }
        for (int i = 0; i < nf; ++i) inv[(size_t)i * nf + c] = (float)x[i];
    }
    return true;
}

// x[free_idx[i]] = sum_j inv[i][j] b[free_idx[j]]: a warp a row (lanes over
// j, then a fixed shuffle tree), b's free values staged in shared memory
__global__ void __launch_bounds__(256) k_mg_direct(const float* __restrict__ inv, const int* __restrict__ freen,
                                                   int nf, const float* __restrict__ b, float* __restrict__ x) {
    extern __shared__ float bs[];
    pdl_enter();
    for (int j = threadIdx.x; j < nf; j += 256) bs[j] = b[freen[j]];
    __syncthreads();
    const int lane = threadIdx.x & 31, i = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (i >= nf) return;
    const float* row = inv + (int64_t)i * nf;
    float s = 0.f;
#pragma unroll 4
    for (int j = lane; j < nf; j += 32) s = fmaf(row[j], bs[j], s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
    if (lane == 0) x[freen[i]] = s;
}

// injected Dirichlet mask of a coarse level: the x walls (and, unless
// periodic in y, the y walls) are Dirichlet, inner nodes take the fine
// node's flag
__global__ void k_mg_coarse_mask(const uint8_t* fmask, int fGX, int fGY, uint8_t* cmask, int cGX,
                                 int cGY, int periodic) {
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    const int J = blockIdx.y * blockDim.y + threadIdx.y;
    if (I >= cGX || J >= cGY) return;
    const int i = 2 * I, j = 2 * J;
    uint8_t m = 1;
    if (I > 0 && I < cGX - 1 && (periodic || (J > 0 && J < cGY - 1)) && i < fGX && j < fGY)
        m = fmask[(int64_t)j * fGX + i];
    cmask[(int64_t)J * cGX + I] = m;
}

// ---- E field ----------------------------------------------------------------
// With walls (calculateElectricField, src/poissonSolver.cpp:433-456): central
// differences inside; boundary nodes take the value of the nearest interior
// node (columns first, then rows, as the reference copies).
// Periodic in y (calculateElectricFieldPeriodic, :411-430): E_x one-sided at
// the first and last column, central elsewhere; E_y central with rows taken
// modulo GY-1; both on every row.

__device__ __forceinline__ void efield_at(const double* phi, int GX, int GY, double dx, double dy,
                                          int i, int j, int periodic, double& ex, double& ey) {
    if (periodic) {
        const int64_t k = (int64_t)j * GX + i;
        if (i == 0) ex = -((phi[k + 1] - phi[k]) / dx);
        else if (i == GX - 1) ex = -((phi[k] - phi[k - 1]) / dx);
        else ex = -((phi[k + 1] - phi[k - 1]) / (2 * dx));
        const int P = GY - 1;
        const int ju = j + 1 >= P ? j + 1 - P : j + 1, jd = j == 0 ? P - 1 : j - 1;
        ey = -((phi[(int64_t)ju * GX + i] - phi[(int64_t)jd * GX + i]) / (2 * dy));
        return;
    }
    const int ci = min(max(i, 1), GX - 2), cj = min(max(j, 1), GY - 2);
    const int64_t k = (int64_t)cj * GX + ci;
    ex = -((phi[k + 1] - phi[k - 1]) / (2 * dx));
    ey = -((phi[k + GX] - phi[k - GX]) / (2 * dy));
}

__global__ void k_efield(const double* phi, const double* bz, int GX, int GY, double dx, double dy,
                         int periodic, float4* fld) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= GX || j >= GY) return;
    double ex, ey;
    efield_at(phi, GX, GY, dx, dy, i, j, periodic, ex, ey);
    const int64_t k = (int64_t)j * GX + i;
    fld[k] = make_float4((float)ex, (float)ey, (float)bz[k], 0.0f);
}

__global__ void k_efield64(const double* phi, int GX, int GY, double dx, double dy, int periodic,
                           double* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= GX || j >= GY) return;
    double ex, ey;
    efield_at(phi, GX, GY, dx, dy, i, j, periodic, ex, ey);
    const int64_t k = (int64_t)j * GX + i;
    out[2 * k] = ex;
    out[2 * k + 1] = ey;
}

__global__ void k_set_bz_field(const double* bz, int64_t nodes, float4* fld) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nodes) return;
    float4 f = fld[k];
    f.z = (float)bz[k];
    fld[k] = f;
}

inline dim3 grid2d(int nx, int ny, dim3 b) {
    return dim3((unsigned)((nx + b.x - 1) / b.x), (unsigned)((ny + b.y - 1) / b.y));
}

Grid64 fine_grid(pic_ctx* c) {
    Grid64 g;
    g.GX = c->GX;
    g.GY = c->GY;
    g.n = c->solve_nodes;
    g.cx = 1.0 / (c->dx * c->dx);
    g.cy = 1.0 / (c->dy * c->dy);
    g.cd = 2.0 * (g.cx + g.cy);
    return g;
}

unsigned* arrive_ptr(PoissonState& ps) { return reinterpret_cast<unsigned*>(ps.scal + S_COUNT); }

// V-cycle on level 0 (b = r32 -> x = z32) enqueued on stream st; returns
// the number of kernels launched.
// Launch with programmatic stream serialisation (see pdl_enter).
template <typename... P, typename... A>
void launch_pdl(void (*k)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, A&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k, std::forward<A>(args)...);
}

// One V-cycle on st from levels[0].b; the result is in vcycle_out().
// Returns the number of kernels.  Levels above the fused ones take two
// kernels each (k_mg_down, k_mg_up); with with_rz the finest k_mg_up also
// reduces r.z for the PCG iteration.
// The V-cycle's coarsest step, from levels[fused_first].b into its x: the
// exact solve when set up, else the one-block chain of the small levels.
static void enqueue_coarse(pic_ctx* c, cudaStream_t st) {
    PoissonState& ps = c->ps;
    if (ps.direct) {
        const MGLevel& L = ps.levels[ps.fused_first];
        launch_pdl(k_mg_direct, dim3((unsigned)((ps.direct_nf + 7) / 8)), dim3(256), (size_t)ps.direct_nf * 4, st,
                   (const float*)ps.direct_inv, (const int*)ps.direct_free, ps.direct_nf, (const float*)L.b, L.x);
    } else {
        launch_pdl(k_mg_fused, dim3(1), dim3(kFusedThreads), ps.fused_smem, st,
                   *reinterpret_cast<const FusedLevels*>(ps.fused_desc));
    }
}

// fewer tiles than two per SM: blocks of kTileThreadsSmall (the level's time
// is one block's latency, which more threads a tile shorten)
static bool small_grid(dim3 g) { return (int64_t)g.x * g.y < 2 * 148; }

int enqueue_vcycle(pic_ctx* c, cudaStream_t st, bool with_rz) {
    PoissonState& ps = c->ps;
    const int kf = ps.fused_first;
    const dim3 tb(kTileThreads);
    int launches = 0;
    for (int l = 0; l < kf; ++l) {
        const LevelDev F = as_dev(ps.levels[l]);
        const LevelDev C = as_dev(ps.levels[l + 1]);
        const int cc = kTileCore / 2;
        const dim3 grid((C.GX + cc - 1) / cc, (C.GY + cc - 1) / cc);
        if (small_grid(grid))
            launch_pdl(k_mg_down<kTileThreadsSmall>, grid, dim3(kTileThreadsSmall), 0, st, F, C);
        else
            launch_pdl(k_mg_down<kTileThreads>, grid, tb, 0, st, F, C);
        launches += 1;
    }
    enqueue_coarse(c, st);
    launches += 1;
    for (int l = kf - 1; l >= 0; --l) {
        const LevelDev F = as_dev(ps.levels[l]);
        LevelDev C = as_dev(ps.levels[l + 1]);
        if (l + 1 < kf) C.x = ps.levels[l + 1].xo;  // what the coarser k_mg_up wrote
        const dim3 grid((F.GX + kTileCore - 1) / kTileCore, (F.GY + kTileCore - 1) / kTileCore);
        if (l == 0 && with_rz)
            launch_pdl(k_mg_up<true, kTileThreads>, grid, tb, 0, st, F, C, ps.levels[l].xo,
                       RzArgs{ps.r, ps.partials, arrive_ptr(ps), ps.scal});
        else if (small_grid(grid))
            launch_pdl(k_mg_up<false, kTileThreadsSmall>, grid, dim3(kTileThreadsSmall), 0, st, F, C,
                       ps.levels[l].xo, RzArgs{});
        else
            launch_pdl(k_mg_up<false, kTileThreads>, grid, tb, 0, st, F, C, ps.levels[l].xo, RzArgs{});
        launches += 1;
    }
    return launches;
}

const float* vcycle_out(const PoissonState& ps) {
    return ps.fused_first > 0 ? ps.levels[0].xo : ps.levels[0].x;
}

// The same V-cycle with one kernel a half sweep, updating each level's x in
// place (the result in levels[0].x): the check of the tiled one.
void enqueue_vcycle_per_sweep(pic_ctx* c, cudaStream_t st) {
    PoissonState& ps = c->ps;
    const int kf = ps.fused_first;
    const dim3 b2(32, 8);
    for (int l = 0; l < kf; ++l) {
        const LevelDev F = as_dev(ps.levels[l]);
        const LevelDev C = as_dev(ps.levels[l + 1]);
        const dim3 gh = grid2d((F.GX + 1) / 2, F.GY, b2);
        launch_pdl(k_mg_init_black, gh, b2, 0, st, F);
        for (int s = 1; s < kNu; ++s) {
            launch_pdl(k_mg_rbgs, gh, b2, 0, st, F, 0);
            launch_pdl(k_mg_rbgs, gh, b2, 0, st, F, 1);
        }
        launch_pdl(k_mg_restrict, grid2d(C.GX, C.GY, b2), b2, 0, st, F, C);
    }
    enqueue_coarse(c, st);
    for (int l = kf - 1; l >= 0; --l) {
        const LevelDev F = as_dev(ps.levels[l]);
        const LevelDev C = as_dev(ps.levels[l + 1]);
        const dim3 gh = grid2d((F.GX + 1) / 2, F.GY, b2);
        launch_pdl(k_mg_prolong_black, gh, b2, 0, st, F, C);
        launch_pdl(k_mg_rbgs, gh, b2, 0, st, F, 0);
        for (int s = 1; s < kNu; ++s) {
            launch_pdl(k_mg_rbgs, gh, b2, 0, st, F, 1);
            launch_pdl(k_mg_rbgs, gh, b2, 0, st, F, 0);
        }
    }
}

// One V-cycle applied to a host right-hand side (FP32, one value a node),
// tiled (per_sweep 0) or one kernel a half sweep (1); the result into out.
int debug_vcycle(pic_ctx* c, const float* rhs, float* out, int per_sweep) {
    PoissonState& ps = c->ps;
    if (!ps.mg_ok) return fail(PIC_ERR_CONFIG, "no multigrid hierarchy on this grid");
    const size_t bytes = (size_t)ps.levels[0].nodes * sizeof(float);
    PIC_CUDA(cudaMemcpyAsync(ps.levels[0].b, rhs, bytes, cudaMemcpyHostToDevice, c->stream));
    if (per_sweep) enqueue_vcycle_per_sweep(c, c->stream);
    else enqueue_vcycle(c, c->stream, false);
    PIC_CUDA(cudaGetLastError());
    PIC_CUDA(cudaMemcpyAsync(out, per_sweep ? ps.levels[0].x : vcycle_out(ps), bytes, cudaMemcpyDeviceToHost,
                             c->stream));
    PIC_CUDA(cudaStreamSynchronize(c->stream));
    return PIC_OK;
}

// One PCG iteration enqueued on st; returns the number of kernels.
int enqueue_iteration(pic_ctx* c, cudaStream_t st, bool jacobi,
                      cudaGraphConditionalHandle handle, int use_handle) {
    PoissonState& ps = c->ps;
    const Grid64 g = fine_grid(c);
    const int nb = ps.nblocks;
    unsigned* arrive = arrive_ptr(ps);
    int launches = 0;
    const dim3 gb(nb), tb(kRedThreads);
    // with tiled levels the finest k_mg_up computes r.z and pq reads its
    // FP32 output; otherwise k_pcg_rz makes z
    const bool rz_in_vcycle = !jacobi && ps.fused_first > 0;
    if (!jacobi) launches += enqueue_vcycle(c, st, rz_in_vcycle);
    if (rz_in_vcycle) {
        launch_pdl(k_pcg_pq<float>, gb, tb, 0, st, g, c->mask, vcycle_out(ps), ps.p[0], ps.q, ps.partials,
                   nb, arrive, ps.scal);
    } else {
        launch_pdl(k_pcg_rz, gb, tb, 0, st, g.n, c->mask, ps.r, vcycle_out(ps), 1.0 / g.cd,
                   jacobi ? 1 : 0, ps.z, ps.partials, nb, arrive, ps.scal);
        launch_pdl(k_pcg_pq<double>, gb, tb, 0, st, g, c->mask, (const double*)ps.z, ps.p[0], ps.q,
                   ps.partials, nb, arrive, ps.scal);
        launches += 1;
    }
    launch_pdl(k_pcg_update, gb, tb, 0, st, g.n, c->mask, ps.p[0], ps.q, c->phi, ps.r,
               ps.levels[0].b, ps.partials, nb, arrive, ps.scal, handle, use_handle);
    return launches + 2;
}

__global__ void k_cond_init(const double* scal, cudaGraphConditionalHandle handle) {
    const double rr = scal[S_RR], bb = scal[S_BB];
    cudaGraphSetConditional(handle, (bb > 0.0 && rr > scal[S_TOL2] * bb) ? 1u : 0u);
}

// Graph: k_cond_init -> while (condition) { one PCG iteration }.
int build_graph(pic_ctx* c, bool jacobi) {
    PoissonState& ps = c->ps;
    const int slot = jacobi ? 1 : 0;
    cudaGraph_t graph = nullptr;
    cudaGraphConditionalHandle handle;
    PIC_CUDA(cudaGraphCreate(&graph, 0));
    auto fail_graph = [&](cudaError_t e) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        return fail(PIC_ERR_CUDA, std::string("PCG graph: ") + cudaGetErrorString(e));
    };
    cudaError_t e = cudaGraphConditionalHandleCreate(&handle, graph, 0, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) return fail_graph(e);
    cudaGraphNode_t n0;
    double* scal = ps.scal;
    void* args[] = {&scal, &handle};
    cudaKernelNodeParams kp{};
    kp.func = (void*)k_cond_init;
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(1);
    kp.kernelParams = args;
    if ((e = cudaGraphAddKernelNode(&n0, graph, nullptr, 0, &kp)) != cudaSuccess) return fail_graph(e);
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t wnode;
    if ((e = cudaGraphAddNode(&wnode, graph, &n0, 1, &cp)) != cudaSuccess) return fail_graph(e);
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    if ((e = cudaStreamBeginCaptureToGraph(ps.cap_stream, body, nullptr, nullptr, 0,
                                           cudaStreamCaptureModeRelaxed)) != cudaSuccess)
        return fail_graph(e);
    ps.body_nodes[slot] = enqueue_iteration(c, ps.cap_stream, jacobi, handle, 1);
    if ((e = cudaStreamEndCapture(ps.cap_stream, &body)) != cudaSuccess) return fail_graph(e);
    if ((e = cudaGraphInstantiate(&ps.gexec[slot], graph, 0)) != cudaSuccess) return fail_graph(e);
    cudaGraphDestroy(graph);
    return PIC_OK;
}

}  // namespace

int poisson_debug_vcycle(pic_ctx* c, const float* rhs, float* out, int per_sweep) {
    return debug_vcycle(c, rhs, out, per_sweep);
}

// ---------------------------------------------------------------------------

int poisson_setup(pic_ctx* c) {
    PoissonState& ps = c->ps;
    ps.solver = c->cfg.poisson_solver;
    ps.warm = c->cfg.warm_start;
    ps.tol = c->cfg.poisson_tol > 0 ? c->cfg.poisson_tol : 1e-8;
    ps.maxit = c->cfg.poisson_maxit > 0 ? c->cfg.poisson_maxit : 500;
    const size_t n = (size_t)c->nodes;
    PIC_CUDA(cudaMalloc(&ps.r, n * 8));
    PIC_CUDA(cudaMalloc(&ps.z, n * 8));
    PIC_CUDA(cudaMalloc(&ps.p[0], n * 8));
    PIC_CUDA(cudaMalloc(&ps.p[1], n * 8));
    PIC_CUDA(cudaMalloc(&ps.q, n * 8));
    PIC_CUDA(cudaMemsetAsync(ps.p[0], 0, n * 8, c->stream));
    PIC_CUDA(cudaMemsetAsync(ps.p[1], 0, n * 8, c->stream));
    PIC_CUDA(cudaMemsetAsync(ps.q, 0, n * 8, c->stream));
    ps.nblocks = (int)std::min<int64_t>((c->nodes + kRedThreads - 1) / kRedThreads, 148 * 8);
    // room for the PCG kernels' partials and for the finest k_mg_up's (one per tile)
    const size_t up_tiles = (size_t)((c->GX + kTileCore - 1) / kTileCore) *
                            (size_t)((c->solve_rows + kTileCore - 1) / kTileCore);
    PIC_CUDA(cudaMalloc(&ps.partials, std::max((size_t)ps.nblocks * 4, up_tiles) * sizeof(double)));
    PIC_CUDA(cudaMalloc(&ps.scal, 16 * sizeof(double)));
    PIC_CUDA(cudaMemsetAsync(ps.scal, 0, 16 * sizeof(double), c->stream));
    PIC_CUDA(cudaMallocHost(&ps.host_scal, 16 * sizeof(double)));
    PIC_CUDA(cudaEventCreate(&ps.ev0));
    PIC_CUDA(cudaEventCreate(&ps.ev1));
    // multigrid hierarchy.  Periodic in y a level has `ny` distinct rows,
    // which must be even for the red-black sweeps; coarsening halves them
    // while the result stays even.
    int nx = c->nx, ny = c->ny;
    const bool per = c->periodic;
    ps.mg_ok = !per || ny % 2 == 0;
    double hx = c->dx, hy = c->dy;
    const uint8_t* prev_mask = c->mask;
    int pGX = c->GX, pGY = c->solve_rows;
    for (int l = 0; l < 16; ++l) {
        MGLevel L{};
        L.nx = nx;
        L.ny = ny;
        L.GX = nx + 1;
        L.GY = per ? ny : ny + 1;
        L.nodes = (int64_t)L.GX * L.GY;
        L.cx = (float)(1.0 / (hx * hx));
        L.cy = (float)(1.0 / (hy * hy));
        L.cd = 2.0f * (L.cx + L.cy);
        PIC_CUDA(cudaMalloc(&L.x, (size_t)L.nodes * 4));
        PIC_CUDA(cudaMalloc(&L.b, (size_t)L.nodes * 4));
        PIC_CUDA(cudaMalloc(&L.xo, (size_t)L.nodes * 4));
        PIC_CUDA(cudaMemsetAsync(L.x, 0, (size_t)L.nodes * 4, c->stream));
        PIC_CUDA(cudaMemsetAsync(L.xo, 0, (size_t)L.nodes * 4, c->stream));
        PIC_CUDA(cudaMemsetAsync(L.b, 0, (size_t)L.nodes * 4, c->stream));
        if (l == 0) {
            L.mask = c->mask;
        } else {
            PIC_CUDA(cudaMalloc(&L.mask, (size_t)L.nodes));
            const dim3 b2(32, 8);
            k_mg_coarse_mask<<<grid2d(L.GX, L.GY, b2), b2, 0, c->stream>>>(prev_mask, pGX, pGY,
                                                                           L.mask, L.GX, L.GY,
                                                                           per ? 1 : 0);
            PIC_CUDA(cudaGetLastError());
        }
        ps.levels.push_back(L);
        if (!ps.mg_ok) break;  // level 0 only: the PCG's single-precision residual
        if (per ? (nx <= 2 || ny % 4 != 0) : std::min(nx, ny) <= 2) break;
        prev_mask = L.mask;
        pGX = L.GX;
        pGY = L.GY;
        nx = (nx + 1) / 2;
        ny = per ? ny / 2 : (ny + 1) / 2;
        hx *= 2;
        hy *= 2;
    }
    // fuse every level from the first whose hierarchy fits in shared memory
    const int L = (int)ps.levels.size();
    auto level_bytes = [&](int l) {
        const size_t n = (size_t)ps.levels[l].nodes;
        return ((n * 4 + 15) & ~(size_t)15) * 2 + ((n + 15) & ~(size_t)15);
    };
    // small levels only (33^2 and below): one SM does them, and a level of
    // 65^2 runs faster as tiled kernels over many SMs; a coarsest level too
    // large for that budget (periodic in y, coarsening stopped early) may
    // take up to 64 KB
    int kf = L;
    for (size_t budget : {(size_t)16 * 1024, (size_t)64 * 1024}) {
        size_t total = 0;
        for (int l = L - 1; l >= 0; --l) {
            if (total + level_bytes(l) > budget || L - l > kMaxFused) break;
            total += level_bytes(l);
            kf = l;
        }
        if (kf < L) break;
    }
    if (kf == L && ps.mg_ok) {
        // only periodic in y can stop coarsening early (rows no longer even)
        if (!per) return fail(PIC_ERR_CONFIG, "coarsest multigrid level does not fit in shared memory");
        ps.mg_ok = false;
    }
    if (!ps.mg_ok) {
        PIC_CUDA(cudaStreamCreateWithFlags(&ps.cap_stream, cudaStreamNonBlocking));
        return PIC_OK;
    }
    ps.fused_first = kf;
    FusedLevels F{};
    F.n = L - kf;
    size_t off = 0;
    for (int l = kf; l < L; ++l) {
        const MGLevel& M = ps.levels[l];
        const int i = l - kf;
        const size_t n = (size_t)M.nodes;
        F.GX[i] = M.GX;
        F.GY[i] = M.GY;
        F.cx[i] = M.cx;
        F.cy[i] = M.cy;
        F.cd[i] = M.cd;
        F.ox[i] = (int)off;
        off += (n * 4 + 15) & ~(size_t)15;
        F.ob[i] = (int)off;
        off += (n * 4 + 15) & ~(size_t)15;
        F.om[i] = (int)off;
        off += (n + 15) & ~(size_t)15;
        F.gmask[i] = M.mask;
        const uint32_t hw = (uint32_t)((M.GX + 1) / 2);
        F.rcp_hw[i] = (uint32_t)((0x100000000ull + hw - 1) / hw);
    }
    F.gb = ps.levels[kf].b;
    F.gx = ps.levels[kf].x;
    // levels of at most 64 nodes: warp 0 alone
    F.small = F.n;
    for (int i = 0; i < F.n; ++i)
        if ((int64_t)F.GX[i] * F.GY[i] <= 64) {
            F.small = i;
            break;
        }
    F.mpre[0] = 0;
    for (int i = 0; i < F.n; ++i) F.mpre[i + 1] = F.mpre[i] + F.GX[i] * F.GY[i];
    if (F.mpre[F.n] > kFusedLoads * kFusedThreads)
        return fail(PIC_ERR_CONFIG, "coarse multigrid levels too large for the one-block kernel");
    // The coarsest level's sweeps: a single free node is exact after one
    // sweep pair (later ones recompute the same value), so one pair does
    {
        const MGLevel& Lc = ps.levels[L - 1];
        std::vector<uint8_t> m((size_t)Lc.nodes);
        PIC_CUDA(cudaMemcpyAsync(m.data(), Lc.mask, m.size(), cudaMemcpyDeviceToHost, c->stream));
        PIC_CUDA(cudaStreamSynchronize(c->stream));
        int64_t free_nodes = 0;
        for (uint8_t v : m) free_nodes += v ? 0 : 1;
        F.sweeps = free_nodes <= 1 ? 1 : kCoarseSweeps;
    }
    static_assert(sizeof(FusedLevels) <= sizeof(ps.fused_desc), "fused level table");
    std::memcpy(ps.fused_desc, &F, sizeof(F));
    ps.fused_smem = off;
    // the attribute belongs to the kernel, shared by every context of the
    // process: it only ever grows, so contexts created earlier keep working
    cudaFuncAttributes fa{};
    PIC_CUDA(cudaFuncGetAttributes(&fa, k_mg_fused));
    if ((int)off > fa.maxDynamicSharedSizeBytes)
        PIC_CUDA(cudaFuncSetAttribute(k_mg_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)off));
    // the exact coarse solve of the first fused level, when it is small
    if (ps.levels[kf].nodes <= kDirectMax) {
        const MGLevel& Lk = ps.levels[kf];
        std::vector<uint8_t> m((size_t)Lk.nodes);
        PIC_CUDA(cudaMemcpyAsync(m.data(), Lk.mask, m.size(), cudaMemcpyDeviceToHost, c->stream));
        PIC_CUDA(cudaStreamSynchronize(c->stream));
        std::vector<int> freen;
        std::vector<float> inv;
        if (invert_level(Lk.GX, Lk.GY, Lk.cx, Lk.cy, Lk.cd, m, freen, inv) && !freen.empty()) {
            ps.direct_nf = (int)freen.size();
            PIC_CUDA(cudaMalloc(&ps.direct_inv, inv.size() * sizeof(float)));
            PIC_CUDA(cudaMalloc(&ps.direct_free, freen.size() * sizeof(int)));
            PIC_CUDA(cudaMemcpy(ps.direct_inv, inv.data(), inv.size() * sizeof(float), cudaMemcpyHostToDevice));
            PIC_CUDA(cudaMemcpy(ps.direct_free, freen.data(), freen.size() * sizeof(int), cudaMemcpyHostToDevice));
            ps.direct = true;
        }
    }
    PIC_CUDA(cudaStreamCreateWithFlags(&ps.cap_stream, cudaStreamNonBlocking));
    return PIC_OK;
}

void poisson_free(pic_ctx* c) {
    PoissonState& ps = c->ps;
    for (size_t l = 0; l < ps.levels.size(); ++l) {
        cudaFree(ps.levels[l].x);
        cudaFree(ps.levels[l].xo);
        cudaFree(ps.levels[l].b);
        if (l > 0) cudaFree(ps.levels[l].mask);
    }
    ps.levels.clear();
    cudaFree(ps.direct_inv);
    cudaFree(ps.direct_free);
    ps.direct_inv = nullptr;
    ps.direct_free = nullptr;
    ps.direct = false;
    cudaFree(ps.r);
    cudaFree(ps.z);
    cudaFree(ps.p[0]);
    cudaFree(ps.p[1]);
    cudaFree(ps.q);
    cudaFree(ps.partials);
    cudaFree(ps.scal);
    cudaFree(ps.net_guess);
    if (ps.host_scal) cudaFreeHost(ps.host_scal);
    if (ps.ev0) cudaEventDestroy(ps.ev0);
    if (ps.ev1) cudaEventDestroy(ps.ev1);
    for (int i = 0; i < 2; ++i)
        if (ps.gexec[i]) cudaGraphExecDestroy(ps.gexec[i]);
    if (ps.cap_stream) cudaStreamDestroy(ps.cap_stream);
    ps = PoissonState{};
}

int poisson_solve(pic_ctx* c) {
    PoissonState& ps = c->ps;
    const int64_t nodes = c->nodes;
    const Grid64 g = fine_grid(c);
    const int nb = ps.nblocks;
    unsigned* arrive = arrive_ptr(ps);
    const bool jacobi = ps.solver == PIC_SOLVER_JACOBI_PCG || !ps.mg_ok;
    const int slot = jacobi ? 1 : 0;
    PIC_CUDA(cudaEventRecord(ps.ev0, c->stream));
    prof_begin(c, PIC_PHASE_POISSON);
    const bool zero_start = (ps.warm == PIC_WARM_ZERO) || !ps.have_prev;
    k_overwrite_rho<<<(unsigned)((nodes + 255) / 256), 256, 0, c->stream>>>(
        nodes, c->mask, c->dir_val, c->rho, c->phi, zero_start ? 1 : 0);
    c->launches += 1;
    const bool learned = ps.warm == PIC_WARM_LEARNED;
    const bool ws_active = learned || ws_tracking(c);
    if (ws_active) {
        const int guess = ws_before_solve(c, learned && ps.have_prev);
        if (guess < 0) return guess;
        if (guess == 1) {
            // the network's guess replaces phi on non-electrode nodes
            k_apply_guess<<<(unsigned)((nodes + 255) / 256), 256, 0, c->stream>>>(
                nodes, c->mask, ps.net_guess, c->phi);
            c->launches += 1;
        }
    }
    if (!ps.gexec[slot] && !ps.graph_failed) {
        if (build_graph(c, jacobi) != PIC_OK) ps.graph_failed = true;  // host loop below
    }
    const double tol2 = ps.tol * ps.tol;
    int restarts = 0;
    double bb = 0, true_rr = 0;
    int status = PIC_OK;
    for (;;) {
        k_pcg_setup<<<nb, kRedThreads, 0, c->stream>>>(g, c->mask, c->dir_val, c->rho, c->phi,
                                                       ps.r, ps.levels[0].b, ps.partials, nb,
                                                       arrive, ps.scal);
        k_fix_bb<<<1, 1, 0, c->stream>>>(ps.scal, tol2, ps.maxit, restarts > 0 ? 1 : 0);
        c->launches += 2;
        PIC_CUDA(cudaGetLastError());
        if (ps.gexec[slot] && !ps.graph_off) {
            PIC_CUDA(cudaGraphLaunch(ps.gexec[slot], c->stream));
        } else {
            // host-driven loop: one synchronisation per iteration
            PIC_CUDA(cudaMemcpyAsync(ps.host_scal, ps.scal, 16 * sizeof(double),
                                     cudaMemcpyDeviceToHost, c->stream));
            PIC_CUDA(cudaStreamSynchronize(c->stream));
            double rr = ps.host_scal[S_RR];
            const double b0 = ps.host_scal[S_BB];
            double it = ps.host_scal[S_IT];
            while (b0 > 0 && rr > tol2 * b0 && std::isfinite(rr) && it < ps.maxit) {
                c->launches += enqueue_iteration(c, c->stream, jacobi, 0, 0);
                PIC_CUDA(cudaGetLastError());
                PIC_CUDA(cudaMemcpyAsync(ps.host_scal, ps.scal, 16 * sizeof(double),
                                         cudaMemcpyDeviceToHost, c->stream));
                PIC_CUDA(cudaStreamSynchronize(c->stream));
                rr = ps.host_scal[S_RR];
                it = ps.host_scal[S_IT];
            }
        }
        // the recursively updated residual can drift from b - A x: check the
        // true residual and restart from the current iterate if needed
        k_true_residual<<<nb, kRedThreads, 0, c->stream>>>(g, c->mask, c->rho, c->phi, ps.partials,
                                                           nb, arrive, ps.scal);
        c->launches += 1;
        PIC_CUDA(cudaMemcpyAsync(ps.host_scal, ps.scal, 16 * sizeof(double), cudaMemcpyDeviceToHost,
                                 c->stream));
        PIC_CUDA(cudaStreamSynchronize(c->stream));
        bb = ps.host_scal[S_BB];
        true_rr = ps.host_scal[S_TRUE_RR];
        const double st = ps.host_scal[S_STATUS];
        if (st != 0.0) {
            status = PIC_ERR_NOT_CONVERGED;
            break;
        }
        if (bb <= 0 || true_rr <= tol2 * bb || restarts >= 3) break;
        ++restarts;
    }
    const int it = (int)ps.host_scal[S_IT];
    if (ps.gexec[slot] && !ps.graph_off) c->launches += (int64_t)it * ps.body_nodes[slot] + 1;
    if (ws_active && status == PIC_OK) PIC_TRY(ws_after_solve(c, c->ws_record));
    if (c->periodic) PIC_TRY(overwrite_phi(c));  // the last row repeats row 0
    PIC_TRY(fields_from_phi(c));
    prof_end(c, PIC_PHASE_POISSON);
    PIC_CUDA(cudaEventRecord(ps.ev1, c->stream));
    PIC_CUDA(cudaStreamSynchronize(c->stream));
    float ms = 0;
    PIC_CUDA(cudaEventElapsedTime(&ms, ps.ev0, ps.ev1));
    ps.last_ms = ms;
    ps.last_iters = it;
    ps.last_relres = bb > 0 ? std::sqrt(true_rr / bb) : 0.0;
    ps.last_relres0 = bb > 0 ? std::sqrt(ps.host_scal[S_RR0] / bb) : 0.0;
    ps.have_prev = true;
    if (learned) PIC_TRY(ws_check_fault());  // the guess's kernels gave up a bounded wait
    if (status != PIC_OK)
        return fail(status, "Poisson PCG did not reach the tolerance within poisson_maxit");
    return PIC_OK;
}

// overwritePhi (src/poissonSolver.cpp:364-382): periodic in y, row 0 is
// first copied into the last row; then electrode nodes take their potential.
// The thread of a first-row node also writes the last-row node of its
// column, from the first row's value before the electrodes.
__global__ void k_overwrite_phi(int64_t nodes, int GX, int periodic, const uint8_t* mask,
                                const double* dv, double* phi) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nodes) return;
    const int64_t last = nodes - GX;
    if (periodic) {
        if (i >= last) return;
        if (i < GX) {
            const double v0 = phi[i];
            phi[last + i] = mask[last + i] ? dv[last + i] : v0;
            phi[i] = mask[i] ? dv[i] : v0;
            return;
        }
    }
    if (mask[i]) phi[i] = dv[i];
}

int overwrite_phi(pic_ctx* c) {
    k_overwrite_phi<<<(unsigned)((c->nodes + 255) / 256), 256, 0, c->stream>>>(
        c->nodes, c->GX, c->periodic ? 1 : 0, c->mask, c->dir_val, c->phi);
    c->launches += 1;
    PIC_CUDA(cudaGetLastError());
    return PIC_OK;
}

int fields_from_phi(pic_ctx* c) {
    const dim3 b2(32, 8);
    k_efield<<<grid2d(c->GX, c->GY, b2), b2, 0, c->stream>>>(c->phi, c->bz, c->GX, c->GY, c->dx,
                                                             c->dy, c->periodic ? 1 : 0, c->fld);
    c->launches += 1;
    PIC_CUDA(cudaGetLastError());
    c->fields_valid = true;
    return PIC_OK;
}

int efield_export(pic_ctx* c) {
    const dim3 b2(32, 8);
    k_efield64<<<grid2d(c->GX, c->GY, b2), b2, 0, c->stream>>>(c->phi, c->GX, c->GY, c->dx, c->dy,
                                                               c->periodic ? 1 : 0, c->efield64);
    PIC_CUDA(cudaGetLastError());
    return PIC_OK;
}

int fields_set_bz(pic_ctx* c) {
    k_set_bz_field<<<(unsigned)((c->nodes + 255) / 256), 256, 0, c->stream>>>(c->bz, c->nodes,
                                                                              c->fld);
    PIC_CUDA(cudaGetLastError());
    return PIC_OK;
}

}  // namespace picb200

// ---------------------------------------------------------------------------
// Batched solve: the Poisson solves of many instances (an ensemble) in ONE
// persistent cooperative launch.  Every phase of the PCG iteration and of the
// V-cycle loops over the instances that are still iterating, each instance's
// nodes spread over the whole grid, with grid-wide barriers between phases;
// an instance's fused coarse levels run in one block (block i for instance
// i).  Dot products are reduced per warp into a per-instance table and
// summed by one block per instance in fixed order: deterministic.  The solve
// ends with the true residual and the E field of every instance.
// ---------------------------------------------------------------------------
namespace picb200 {
namespace {

constexpr int kMaxBatchLevels = 10;

struct BatchInst {
    int GX, GY;
    double cx, cy, cd;
    double dx, dy;
    int64_t nodes;  // all GX*GY nodes
    int64_t sn;     // solved nodes (GX*(GY-1) when periodic in y)
    int periodic;
    const uint8_t* mask;
    const double* dv;
    double* rho;  // becomes the right-hand side b
    double* phi;
    double* r;
    double* z;
    double* p;
    double* q;
    const double* bz;
    float4* fld;
    int kf;  // multigrid levels before the fused ones
    LevelDev lev[kMaxBatchLevels];  // levels 0 .. kf
    const FusedLevels* fused;
    double* scal;
    double tol2;
    int maxit;
    int zero_start;
    int blk0, nblk;  // the blocks of the launch that work on this instance
};

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Barrier of the nblk blocks working on one instance: a monotonic arrival
// counter (zeroed before the launch); the blocks are co-resident (cooperative
// launch).  The wait is bounded: past kSpinLimit polls the barrier sets
// *err and lets the block go on, so a fault can never hang the GPU (the
// host then reports PIC_ERR_TIMEOUT).
constexpr unsigned kSpinLimit = 1u << 26;
__device__ unsigned g_spin_limit = kSpinLimit;  // a test lowers it to make the barriers give up

struct GroupBarrier {
    unsigned* ctr;
    unsigned target;
    int nblk;
    int* err;
    __device__ __forceinline__ void sync() {
        __syncthreads();
        if (threadIdx.x == 0) {
            target += (unsigned)nblk;
            __threadfence();
            atomicAdd(ctr, 1u);
            unsigned polls = 0;
            const unsigned limit = g_spin_limit;
            while (ld_acquire(ctr) < target) {
                if (++polls > limit) {
                    atomicExch(err, 1);
                    break;
                }
                __nanosleep(64);
            }
            __threadfence();
        }
        __syncthreads();
    }
};

// Blocks blk0 .. blk0+nblk of the launch work on instance inst_of[block] and
// meet at the instance's own barriers between phases; each instance iterates
// until its own convergence.
__global__ void __launch_bounds__(kFusedThreads) k_poisson_batch(const BatchInst* __restrict__ insts,
                                                                  int n, const int* __restrict__ inst_of,
                                                                  double* partials, unsigned* barriers,
                                                                  int* err) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double s_red[2][kFusedThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int me = inst_of[blockIdx.x];  // -1: a spare block
    if (me < 0) return;
    const BatchInst* I = insts + me;
    GroupBarrier grid{barriers + me, 0u, I->nblk, err};
    const int64_t ltid = (int64_t)(blockIdx.x - I->blk0) * blockDim.x + threadIdx.x;
    const int64_t lsize = (int64_t)I->nblk * blockDim.x;
    const bool first = blockIdx.x == I->blk0;

    // block sums of two values -> partials[block][0..1]
    auto put2 = [&](double a, double b) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(kFull, a, o);
            b += __shfl_xor_sync(kFull, b, o);
        }
        if (lane == 0) {
            s_red[0][warp] = a;
            s_red[1][warp] = b;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double ta = 0.0, tb = 0.0;
            for (int w = 0; w < (int)(blockDim.x / 32); ++w) {
                ta += s_red[0][w];
                tb += s_red[1][w];
            }
            partials[2 * blockIdx.x] = ta;
            partials[2 * blockIdx.x + 1] = tb;
        }
    };
    // the instance's first block: sum of its blocks' partials, fixed order
    auto total = [&](int v) {
        double t = 0.0;
        for (int b = I->blk0; b < I->blk0 + I->nblk; ++b) t += partials[2 * b + v];
        return t;
    };
    auto stencil64 = [&](const double* x, int64_t k) {
        return I->cd * x[k] - I->cx * (x[k - 1] + x[k + 1]) -
               I->cy * (x[row_dn(k, I->sn, I->GX)] + x[row_up(k, I->sn, I->GX)]);
    };

    // overwriteRho and the electrode potentials (zero start: phi = 0 elsewhere)
    if (I) {
        for (int64_t k = ltid; k < I->nodes; k += lsize) {
            if (I->mask[k]) {
                I->rho[k] = -I->dv[k];
                I->phi[k] = I->dv[k];
            } else {
                I->rho[k] = -I->rho[k];
                if (I->zero_start) I->phi[k] = 0.0;
            }
        }
    }
    grid.sync();
    // r = b - A x, MG input r32; |r|^2 and |b_red|^2
    if (I) {
        double rr = 0.0, bb = 0.0;
        for (int64_t k = ltid; k < I->sn; k += lsize) {
            double ri = 0.0;
            if (!I->mask[k]) {
                ri = I->rho[k] - stencil64(I->phi, k);
                const double br = I->rho[k] + I->cx * (dirv(I->mask, I->dv, k - 1) + dirv(I->mask, I->dv, k + 1)) +
                                  I->cy * (dirv(I->mask, I->dv, row_dn(k, I->sn, I->GX)) +
                                           dirv(I->mask, I->dv, row_up(k, I->sn, I->GX)));
                bb += br * br;
            }
            I->r[k] = ri;
            I->lev[0].b[k] = (float)ri;
            rr += ri * ri;
        }
        put2(rr, bb);
    }
    grid.sync();
    if (first && threadIdx.x == 0) {
        const double rr = total(0), bb = total(1);
        I->scal[S_RR] = rr;
        I->scal[S_BB] = bb;
        I->scal[S_RZ_OLD] = 0.0;
        I->scal[S_IT] = 0.0;
        I->scal[S_STATUS] = 0.0;
        I->scal[S_COUNT] = (bb > 0.0 && rr > I->tol2 * bb) ? 1.0 : 0.0;  // go on
    }
    grid.sync();
    const int maxkf = I->kf;
    for (int it = 0; it < I->maxit; ++it) {
        if (I->scal[S_COUNT] == 0.0) break;  // the same value for all the instance's blocks
        const bool on = true;
        // ---- V-cycle: levels above the fused ones ----
        // one colour of a Gauss-Seidel sweep; four nodes per thread and
        // round, their loads issued before their stores (memory-level
        // parallelism: one block per SM)
        auto half_sweep = [&](int l, int color) {
            if (on && l < I->kf) {
                const LevelDev& L = I->lev[l];
                const int hw = (L.GX + 1) >> 1, n = hw * L.GY, ls = (int)lsize, nl = L.GX * L.GY;
                for (int h0 = (int)ltid; h0 < n; h0 += 4 * ls) {
                    int k[4];
                    bool ok[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int h = h0 + u * ls;
                        const int j = h / hw;
                        const int x = 2 * (h - j * hw) + ((j + color) & 1);
                        k[u] = j * L.GX + x;
                        ok[u] = h < n && x < L.GX;
                        ok[u] = ok[u] && !L.mask[k[u]];
                    }
                    float v[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                        v[u] = ok[u] ? __fmaf_rn(L.cx, L.x[k[u] - 1] + L.x[k[u] + 1],
                                                 __fmaf_rn(L.cy, L.x[row_dn(k[u], nl, L.GX)] + L.x[row_up(k[u], nl, L.GX)],
                                                           L.b[k[u]]))
                                     : 0.0f;
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                        if (ok[u]) L.x[k[u]] = v[u] * L.icd;
                }
            }
            grid.sync();
        };
        // the first black sweep fused with the zero start (mode 0) or with
        // the coarse correction (mode 1): each black node computes its red
        // neighbours' values itself (as k_mg_init_black / k_mg_prolong_black)
        auto first_black = [&](int l, int mode) {
            if (on && l < I->kf) {
                const LevelDev& L = I->lev[l];
                const LevelDev& C = I->lev[l + 1];
                const int hw = (L.GX + 1) >> 1, n = hw * L.GY, ls = (int)lsize, nl = L.GX * L.GY;
                for (int h = (int)ltid; h < n; h += ls) {
                    const int j = h / hw;
                    const int x = 2 * (h - j * hw) + ((j + 1) & 1);
                    if (x >= L.GX) continue;
                    const int k = j * L.GX + x;
                    if (L.mask[k]) continue;
                    float w, e, d, u;
                    if (mode == 0) {
                        auto xr = [&](int m) { return L.mask[m] ? 0.0f : L.b[m] * L.icd; };
                        w = xr(k - 1);
                        e = xr(k + 1);
                        d = xr(row_dn(k, nl, L.GX));
                        u = xr(row_up(k, nl, L.GX));
                    } else {
                        const int jd = j == 0 ? L.GY - 1 : j - 1, ju = j + 1 == L.GY ? 0 : j + 1;
                        w = prolonged(L, C, x - 1, j);
                        e = prolonged(L, C, x + 1, j);
                        d = prolonged(L, C, x, jd);
                        u = prolonged(L, C, x, ju);
                    }
                    L.x[k] = __fmaf_rn(L.cx, w + e, __fmaf_rn(L.cy, d + u, L.b[k])) * L.icd;
                }
            }
            grid.sync();
        };
        for (int l = 0; l < maxkf; ++l) {
            first_black(l, 0);
            for (int s = 1; s < kNu; ++s) {
                half_sweep(l, 0);
                half_sweep(l, 1);
            }
            if (on && l < I->kf) {
                const LevelDev& F = I->lev[l];
                const LevelDev& C = I->lev[l + 1];
                const int nc = C.GX * C.GY;
#pragma unroll 4
                for (int kc = (int)ltid; kc < nc; kc += (int)lsize) {
                    if (C.mask[kc]) {
                        C.b[kc] = 0.0f;
                        continue;
                    }
                    const int jc = kc / C.GX;
                    const int x = 2 * (kc - jc * C.GX), j = 2 * jc;
                    float s = 4.0f * fine_residual(F, x, j);
                    s += 2.0f * (fine_residual(F, x - 1, j) + fine_residual(F, x + 1, j) +
                                 fine_residual(F, x, j - 1) + fine_residual(F, x, j + 1));
                    s += fine_residual(F, x - 1, j - 1) + fine_residual(F, x + 1, j - 1) +
                         fine_residual(F, x - 1, j + 1) + fine_residual(F, x + 1, j + 1);
                    C.b[kc] = s * 0.0625f;
                }
            }
            grid.sync();
        }
        if (on && first) fused_body(*I->fused, smem);
        grid.sync();
        for (int l = maxkf - 1; l >= 0; --l) {
            first_black(l, 1);
            half_sweep(l, 0);
            for (int s = 1; s < kNu; ++s) {
                half_sweep(l, 1);
                half_sweep(l, 0);
            }
        }
        // ---- PCG update ----
        if (on) {
            double rz = 0.0;
            const float* __restrict__ x0 = I->lev[0].x;
            const double* __restrict__ rv = I->r;
            double* __restrict__ zv = I->z;
            const uint8_t* __restrict__ mk = I->mask;
            const int nn = (int)I->sn;
#pragma unroll 4
            for (int k = (int)ltid; k < nn; k += (int)lsize) {
                const double zi = mk[k] ? 0.0 : (double)x0[k];
                zv[k] = zi;
                rz += rv[k] * zi;
            }
            put2(rz, 0.0);
        }
        grid.sync();
        if (on && first && threadIdx.x == 0) I->scal[S_RZ] = total(0);
        grid.sync();
        if (on) {
            const double ro = I->scal[S_RZ_OLD];
            const double beta = ro == 0.0 ? 0.0 : I->scal[S_RZ] / ro;
            const double* __restrict__ zv = I->z;
            double* __restrict__ pv = I->p;
            const uint8_t* __restrict__ mk = I->mask;
            const int nn = (int)I->sn;
#pragma unroll 4
            // (the first iteration does not read p: what a solve that gave up
            // left there, NaN included, never reaches the next one)
            for (int k = (int)ltid; k < nn; k += (int)lsize)
                pv[k] = mk[k] ? 0.0 : (beta == 0.0 ? zv[k] : zv[k] + beta * pv[k]);
        }
        grid.sync();
        if (on) {
            double pq = 0.0;
            const double* __restrict__ pv = I->p;
            double* __restrict__ qv = I->q;
            const uint8_t* __restrict__ mk = I->mask;
            const int nn = (int)I->sn, GX = I->GX;
            const double cd = I->cd, cx = I->cx, cy = I->cy;
#pragma unroll 4
            for (int k = (int)ltid; k < nn; k += (int)lsize) {
                const double qi = mk[k] ? 0.0
                                        : cd * pv[k] - cx * (pv[k - 1] + pv[k + 1]) -
                                              cy * (pv[row_dn(k, nn, GX)] + pv[row_up(k, nn, GX)]);
                qv[k] = qi;
                pq += pv[k] * qi;
            }
            put2(pq, 0.0);
        }
        grid.sync();
        if (on && first && threadIdx.x == 0) I->scal[S_PQ] = total(0);
        grid.sync();
        if (on) {
            const double alpha = I->scal[S_RZ] / I->scal[S_PQ];
            double rr = 0.0;
            const double* __restrict__ pv = I->p;
            const double* __restrict__ qv = I->q;
            double* __restrict__ xv = I->phi;
            double* __restrict__ rv = I->r;
            float* __restrict__ b0 = I->lev[0].b;
            const uint8_t* __restrict__ mk = I->mask;
            const int nn = (int)I->sn;
#pragma unroll 4
            for (int k = (int)ltid; k < nn; k += (int)lsize) {
                double ri = 0.0;
                if (!mk[k]) {
                    xv[k] += alpha * pv[k];
                    ri = rv[k] - alpha * qv[k];
                }
                rv[k] = ri;
                b0[k] = (float)ri;
                rr += ri * ri;
            }
            put2(rr, 0.0);
        }
        grid.sync();
        if (on && first && threadIdx.x == 0) {
            const double rr = total(0);
            const double its = I->scal[S_IT] + 1.0;
            I->scal[S_IT] = its;
            I->scal[S_RZ_OLD] = I->scal[S_RZ];
            I->scal[S_RR] = rr;
            const bool finite = isfinite(rr);
            bool go = finite && rr > I->tol2 * I->scal[S_BB];
            if (go && its >= (double)I->maxit) {
                go = false;
                I->scal[S_STATUS] = 1.0;
            }
            if (!finite) I->scal[S_STATUS] = 2.0;
            I->scal[S_COUNT] = go ? 1.0 : 0.0;
        }
        grid.sync();
    }
    // true residual of every instance, then its E field
    if (I) {
        double rr = 0.0;
        for (int64_t k = ltid; k < I->sn; k += lsize) {
            if (I->mask[k]) continue;
            const double ri = I->rho[k] - stencil64(I->phi, k);
            rr += ri * ri;
        }
        put2(rr, 0.0);
    }
    grid.sync();
    if (first && threadIdx.x == 0) {
        I->scal[S_TRUE_RR] = total(0);
        if (*err) I->scal[S_STATUS] = 3.0;
    }
    if (I->periodic) {
        // overwritePhi: the last row repeats row 0 (final, electrodes
        // included), then takes its own electrodes
        const int64_t last = I->nodes - I->GX;
        for (int64_t i = ltid; i < I->GX; i += lsize)
            I->phi[last + i] = I->mask[last + i] ? I->dv[last + i] : I->phi[i];
        grid.sync();
    }
    if (I) {
        for (int64_t k = ltid; k < I->nodes; k += lsize) {
            const int x = (int)(k % I->GX), j = (int)(k / I->GX);
            double ex, ey;
            efield_at(I->phi, I->GX, I->GY, I->dx, I->dy, x, j, I->periodic, ex, ey);
            I->fld[k] = make_float4((float)ex, (float)ey, (float)I->bz[k], 0.0f);
        }
    }
}

}  // namespace

// Host side of the batched solve: descriptors live in device memory owned by
// the caller (`dev_insts`, `partials`, `active`); built once per ensemble.
size_t poisson_batch_desc_bytes() { return sizeof(BatchInst); }
size_t poisson_batch_max_fused_smem() { return 64 * 1024 + 1024; }

int poisson_batch_describe(pic_ctx* c, void* host_desc, const void* dev_fused, int blk0, int nblk) {
    PoissonState& ps = c->ps;
    if (ps.fused_first + 1 > kMaxBatchLevels) return fail(PIC_ERR_CONFIG, "too many multigrid levels for the batched solve");
    if (ps.warm == PIC_WARM_LEARNED) return fail(PIC_ERR_CONFIG, "the batched solve has no learned warm start");
    if (ps.solver != PIC_SOLVER_MG_PCG || !ps.mg_ok)
        return fail(PIC_ERR_CONFIG, "the batched solve is MG-PCG only (periodic in y: ny must be even)");
    BatchInst I{};
    const Grid64 g = fine_grid(c);
    I.GX = g.GX;
    I.GY = g.GY;
    I.cx = g.cx;
    I.cy = g.cy;
    I.cd = g.cd;
    I.dx = c->dx;
    I.dy = c->dy;
    I.nodes = c->nodes;
    I.sn = c->solve_nodes;
    I.periodic = c->periodic ? 1 : 0;
    I.mask = c->mask;
    I.dv = c->dir_val;
    I.rho = c->rho;
    I.phi = c->phi;
    I.r = ps.r;
    I.z = ps.z;
    I.p = ps.p[0];
    I.q = ps.q;
    I.bz = c->bz;
    I.fld = c->fld;
    I.kf = ps.fused_first;
    for (int l = 0; l <= ps.fused_first; ++l) I.lev[l] = as_dev(ps.levels[l]);
    I.fused = static_cast<const FusedLevels*>(dev_fused);
    I.scal = ps.scal;
    I.tol2 = ps.tol * ps.tol;
    I.maxit = ps.maxit;
    I.zero_start = (ps.warm == PIC_WARM_ZERO || !ps.have_prev) ? 1 : 0;
    I.blk0 = blk0;
    I.nblk = nblk;
    std::memcpy(host_desc, &I, sizeof(I));
    return PIC_OK;
}

// The instance's fused-level table, for a device copy.
const void* poisson_fused_table(pic_ctx* c, size_t* bytes) {
    *bytes = sizeof(FusedLevels);
    return c->ps.fused_desc;
}

size_t poisson_fused_smem(pic_ctx* c) { return c->ps.fused_smem; }

int poisson_batch_launch(const void* dev_insts, int n, const int* inst_of, double* partials,
                         unsigned* barriers, int* err, size_t smem, int blocks, cudaStream_t st) {
    // the barriers' arrival counters start at zero
    PIC_CUDA(cudaMemsetAsync(barriers, 0, (size_t)n * sizeof(unsigned), st));
    PIC_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
    void* args[] = {(void*)&dev_insts, (void*)&n, (void*)&inst_of, (void*)&partials, (void*)&barriers,
                    (void*)&err};
    PIC_CUDA(cudaLaunchCooperativeKernel((const void*)k_poisson_batch, dim3(blocks), dim3(kFusedThreads),
                                         args, smem, st));
    return PIC_OK;
}

// Poll bound of the batched solve's barriers on the current device; polls <=
// 0 restores the default.
int poisson_set_spin_limit(int64_t polls) {
    const unsigned v = polls > 0 ? (unsigned)std::min<int64_t>(polls, kSpinLimit) : kSpinLimit;
    PIC_CUDA(cudaMemcpyToSymbol(g_spin_limit, &v, sizeof(v)));
    return PIC_OK;
}

int poisson_batch_blocks(size_t smem, int* blocks) {
    cudaFuncAttributes fa{};  // (grows only: other ensembles may be alive)
    PIC_CUDA(cudaFuncGetAttributes(&fa, k_poisson_batch));
    if ((int)smem > fa.maxDynamicSharedSizeBytes)
        PIC_CUDA(cudaFuncSetAttribute(k_poisson_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0, dev = 0, sms = 0;
    PIC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_poisson_batch, kFusedThreads, smem));
    PIC_CUDA(cudaGetDevice(&dev));
    PIC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    *blocks = per_sm * sms;
    if (*blocks <= 0) return fail(PIC_ERR_CONFIG, "the batched solve does not fit on the device");
    return PIC_OK;
}

// After a batched solve: the instance's statistics as poisson_solve leaves
// them, from a host copy of its 16 scalars.
int poisson_batch_finish(pic_ctx* c, const double* scal, float ms) {
    PoissonState& ps = c->ps;
    std::memcpy(ps.host_scal, scal, 16 * sizeof(double));
    const double bb = scal[S_BB], trr = scal[S_TRUE_RR];
    ps.last_iters = (int)scal[S_IT];
    ps.last_relres = bb > 0 ? std::sqrt(trr / bb) : 0.0;
    ps.last_ms = ms;
    ps.have_prev = true;
    c->fields_valid = true;
    if (scal[S_STATUS] == 3.0) return fail(PIC_ERR_TIMEOUT, "batched Poisson solve: a block barrier timed out");
    if (scal[S_STATUS] != 0.0)
        return fail(PIC_ERR_NOT_CONVERGED, "Poisson PCG did not reach the tolerance within poisson_maxit");
    return PIC_OK;
}

}  // namespace picb200
