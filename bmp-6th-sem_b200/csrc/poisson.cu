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
// coarse correction, so the V-cycle is a symmetric preconditioner.  The
// coarsest level (min(nx,ny) <= 4) gets symmetric RB-GS sweeps in one block.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "pic_internal.h"

namespace picb200 {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kRedThreads = 256;
constexpr int kNu = 2;            // RB-GS sweeps before and after the coarse correction
constexpr int kCoarseSweeps = 40; // symmetric sweep pairs on the coarsest level

// device scalar slots
enum {
    S_BB = 0,   // ||b_red||^2
    S_RR = 1,   // ||r||^2
    S_RZ = 2,   // r.z (current)
    S_PQ = 3,   // p.Ap
    S_RZ_OLD = 4,
    S_TRUE_RR = 5,
    S_COUNT = 6  // [6] is the arrival counter (as double bits)
};

struct Grid64 {
    int GX, GY;
    double cx, cy, cd;
};

// ---- deterministic block reduction with last-block finalisation ---------

template <int ND>
__device__ __forceinline__ void reduce_finalize(double (&v)[ND], double* partials, int nblocks,
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
    if (!last) return;
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
}

__device__ __forceinline__ double dirv(const uint8_t* mask, const double* dv, int64_t k) {
    return mask[k] ? dv[k] : 0.0;
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
    const int64_t nodes = (int64_t)g.GX * g.GY;
    double acc[2] = {0.0, 0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nodes;
         i += (int64_t)gridDim.x * blockDim.x) {
        double ri = 0.0;
        if (!mask[i]) {
            const double ax = g.cd * x[i] - g.cx * (x[i - 1] + x[i + 1]) - g.cy * (x[i - g.GX] + x[i + g.GX]);
            ri = b[i] - ax;
            const double br = b[i] + g.cx * (dirv(mask, dv, i - 1) + dirv(mask, dv, i + 1)) +
                              g.cy * (dirv(mask, dv, i - g.GX) + dirv(mask, dv, i + g.GX));
            acc[1] += br * br;
        }
        r[i] = ri;
        r32[i] = (float)ri;
        acc[0] += ri * ri;
    }
    reduce_finalize<2>(acc, partials, nblocks, arrive, scal, S_RR);
    // slots: S_RR = r.r, S_RR+1 = S_RZ holds bb temporarily; moved by k_fix_bb
}

__global__ void k_fix_bb(double* scal) {
    scal[S_BB] = scal[S_RZ];
    scal[S_RZ] = 0.0;
    scal[S_RZ_OLD] = 0.0;
}

// z = M^-1 r (from the MG output or the diagonal); partial r.z
__global__ void __launch_bounds__(kRedThreads) k_pcg_rz(int64_t nodes, const uint8_t* mask,
                                                        const double* r, const float* z32,
                                                        double inv_diag, int jacobi, double* z,
                                                        double* partials, int nblocks,
                                                        unsigned* arrive, double* scal) {
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

// p = z + beta p_old (beta = rz/rz_old, 0 on the first iteration);
// q = A p; partial p.q
__global__ void __launch_bounds__(kRedThreads) k_pcg_p_ap(Grid64 g, const uint8_t* mask,
                                                          const double* z, const double* p_old,
                                                          double* p_new, double* q, int first,
                                                          double* partials, int nblocks,
                                                          unsigned* arrive, double* scal) {
    const int64_t nodes = (int64_t)g.GX * g.GY;
    const double beta = first ? 0.0 : scal[S_RZ] / scal[S_RZ_OLD];
    double acc[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nodes;
         i += (int64_t)gridDim.x * blockDim.x) {
        double pi = 0.0, qi = 0.0;
        if (!mask[i]) {
            auto P = [&](int64_t k) { return mask[k] ? 0.0 : z[k] + beta * p_old[k]; };
            pi = z[i] + beta * p_old[i];
            qi = g.cd * pi - g.cx * (P(i - 1) + P(i + 1)) - g.cy * (P(i - g.GX) + P(i + g.GX));
        }
        p_new[i] = pi;
        q[i] = qi;
        acc[0] += pi * qi;
    }
    reduce_finalize<1>(acc, partials, nblocks, arrive, scal, S_PQ);
}

// x += alpha p; r -= alpha q; r32 = r; partial r.r.  Also shifts rz -> rz_old.
__global__ void __launch_bounds__(kRedThreads) k_pcg_update(int64_t nodes, const uint8_t* mask,
                                                            const double* p, const double* q,
                                                            double* x, double* r, float* r32,
                                                            double* partials, int nblocks,
                                                            unsigned* arrive, double* scal) {
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
    reduce_finalize<1>(acc, partials, nblocks, arrive, scal, S_RR);
}

__global__ void k_shift_rz(double* scal) { scal[S_RZ_OLD] = scal[S_RZ]; }

// true residual of the final iterate (reported relres)
__global__ void __launch_bounds__(kRedThreads) k_true_residual(Grid64 g, const uint8_t* mask,
                                                               const double* b, const double* x,
                                                               double* partials, int nblocks,
                                                               unsigned* arrive, double* scal) {
    const int64_t nodes = (int64_t)g.GX * g.GY;
    double acc[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nodes;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (!mask[i]) {
            const double ax = g.cd * x[i] - g.cx * (x[i - 1] + x[i + 1]) - g.cy * (x[i - g.GX] + x[i + g.GX]);
            const double ri = b[i] - ax;
            acc[0] += ri * ri;
        }
    }
    reduce_finalize<1>(acc, partials, nblocks, arrive, scal, S_TRUE_RR);
}

// ---- multigrid (FP32) ------------------------------------------------------

struct LevelDev {
    int nx, ny, GX, GY;
    float cx, cy, cd;
    const uint8_t* mask;
    float* x;
    float* b;
};

__host__ __device__ __forceinline__ LevelDev as_dev(const MGLevel& L) {
    return LevelDev{L.nx, L.ny, L.GX, L.GY, L.cx, L.cy, L.cd, L.mask, L.x, L.b};
}

// x = b/cd on red non-Dirichlet nodes, 0 elsewhere: the first red sweep from
// a zero guess.
__global__ void k_mg_init(LevelDev L) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= L.GX || j >= L.GY) return;
    const int64_t k = (int64_t)j * L.GX + i;
    L.x[k] = (((i + j) & 1) == 0 && !L.mask[k]) ? L.b[k] / L.cd : 0.0f;
}

// one Gauss-Seidel half sweep over the nodes of one colour
__global__ void k_mg_rbgs(LevelDev L, int color) {
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = 2 * h + ((j + color) & 1);
    if (i >= L.GX || j >= L.GY) return;
    const int64_t k = (int64_t)j * L.GX + i;
    if (L.mask[k]) return;
    const float s = __fmaf_rn(L.cx, L.x[k - 1] + L.x[k + 1], __fmaf_rn(L.cy, L.x[k - L.GX] + L.x[k + L.GX], L.b[k]));
    L.x[k] = s / L.cd;
}

__device__ __forceinline__ float fine_residual(const LevelDev& F, int i, int j) {
    if (i < 0 || j < 0 || i >= F.GX || j >= F.GY) return 0.0f;
    const int64_t k = (int64_t)j * F.GX + i;
    if (F.mask[k]) return 0.0f;
    const float ax = F.cd * F.x[k] - F.cx * (F.x[k - 1] + F.x[k + 1]) - F.cy * (F.x[k - F.GX] + F.x[k + F.GX]);
    return F.b[k] - ax;
}

// b_coarse = full weighting of the fine residual
__global__ void k_mg_restrict(LevelDev F, LevelDev C) {
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

// x_fine += bilinear interpolation of x_coarse (non-Dirichlet fine nodes)
__global__ void k_mg_prolong(LevelDev F, LevelDev C) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= F.GX || j >= F.GY) return;
    const int64_t k = (int64_t)j * F.GX + i;
    if (F.mask[k]) return;
    const int I = i >> 1, J = j >> 1;
    const bool ox = i & 1, oy = j & 1;
    auto X = [&](int a, int b) { return C.x[(int64_t)b * C.GX + a]; };
    float v;
    if (!ox && !oy) v = X(I, J);
    else if (ox && !oy) v = 0.5f * (X(I, J) + X(I + 1, J));
    else if (!ox && oy) v = 0.5f * (X(I, J) + X(I, J + 1));
    else v = 0.25f * (X(I, J) + X(I + 1, J) + X(I, J + 1) + X(I + 1, J + 1));
    F.x[k] += v;
}

// coarsest level: zero start, then symmetric RB-GS sweeps in one block
__global__ void k_mg_coarse(LevelDev L, int sweeps) {
    const int n = L.GX * L.GY;
    for (int k = threadIdx.x; k < n; k += blockDim.x) L.x[k] = 0.0f;
    __syncthreads();
    for (int s = 0; s < 2 * sweeps; ++s) {
        for (int half = 0; half < 2; ++half) {
            // forward sweeps: red then black; backward sweeps: black then red
            const int color = (s < sweeps) ? half : 1 - half;
            for (int k = threadIdx.x; k < n; k += blockDim.x) {
                const int i = k % L.GX, j = k / L.GX;
                if (((i + j) & 1) != color || L.mask[k]) continue;
                const float t = L.b[k] + L.cx * (L.x[k - 1] + L.x[k + 1]) + L.cy * (L.x[k - L.GX] + L.x[k + L.GX]);
                L.x[k] = t / L.cd;
            }
            __syncthreads();
        }
    }
}

// injected Dirichlet mask of a coarse level
__global__ void k_mg_coarse_mask(const uint8_t* fmask, int fGX, int fGY, uint8_t* cmask, int cGX,
                                 int cGY) {
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    const int J = blockIdx.y * blockDim.y + threadIdx.y;
    if (I >= cGX || J >= cGY) return;
    const int i = 2 * I, j = 2 * J;
    uint8_t m = 1;
    if (I > 0 && J > 0 && I < cGX - 1 && J < cGY - 1 && i < fGX && j < fGY)
        m = fmask[(int64_t)j * fGX + i];
    cmask[(int64_t)J * cGX + I] = m;
}

// ---- E field (calculateElectricField, src/poissonSolver.cpp:433-456) -----
// Interior: central differences.  Boundary nodes take the value of the
// nearest interior node (columns first, then rows, as the reference copies).

__device__ __forceinline__ void efield_at(const double* phi, int GX, int GY, double dx, double dy,
                                          int i, int j, double& ex, double& ey) {
    const int ci = min(max(i, 1), GX - 2), cj = min(max(j, 1), GY - 2);
    const int64_t k = (int64_t)cj * GX + ci;
    ex = -((phi[k + 1] - phi[k - 1]) / (2 * dx));
    ey = -((phi[k + GX] - phi[k - GX]) / (2 * dy));
}

__global__ void k_efield(const double* phi, const double* bz, int GX, int GY, double dx, double dy,
                         float4* fld) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= GX || j >= GY) return;
    double ex, ey;
    efield_at(phi, GX, GY, dx, dy, i, j, ex, ey);
    const int64_t k = (int64_t)j * GX + i;
    fld[k] = make_float4((float)ex, (float)ey, (float)bz[k], 0.0f);
}

__global__ void k_efield64(const double* phi, int GX, int GY, double dx, double dy, double* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= GX || j >= GY) return;
    double ex, ey;
    efield_at(phi, GX, GY, dx, dy, i, j, ex, ey);
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
    g.cx = 1.0 / (c->dx * c->dx);
    g.cy = 1.0 / (c->dy * c->dy);
    g.cd = 2.0 * (g.cx + g.cy);
    return g;
}

unsigned* arrive_ptr(PoissonState& ps) { return reinterpret_cast<unsigned*>(ps.scal + S_COUNT); }

int vcycle(pic_ctx* c) {
    PoissonState& ps = c->ps;
    const int L = (int)ps.levels.size();
    const dim3 b2(32, 8);
    for (int l = 0; l < L - 1; ++l) {
        const LevelDev F = as_dev(ps.levels[l]);
        const LevelDev C = as_dev(ps.levels[l + 1]);
        const dim3 gn = grid2d(F.GX, F.GY, b2);
        const dim3 gh = grid2d((F.GX + 1) / 2, F.GY, b2);
        k_mg_init<<<gn, b2, 0, c->stream>>>(F);
        k_mg_rbgs<<<gh, b2, 0, c->stream>>>(F, 1);
        for (int s = 1; s < kNu; ++s) {
            k_mg_rbgs<<<gh, b2, 0, c->stream>>>(F, 0);
            k_mg_rbgs<<<gh, b2, 0, c->stream>>>(F, 1);
        }
        k_mg_restrict<<<grid2d(C.GX, C.GY, b2), b2, 0, c->stream>>>(F, C);
    }
    k_mg_coarse<<<1, 256, 0, c->stream>>>(as_dev(ps.levels[L - 1]), kCoarseSweeps);
    c->launches += 1 + (int64_t)(L - 1) * (2 + 2 * kNu + 2 * kNu);
    for (int l = L - 2; l >= 0; --l) {
        const LevelDev F = as_dev(ps.levels[l]);
        const LevelDev C = as_dev(ps.levels[l + 1]);
        const dim3 gh = grid2d((F.GX + 1) / 2, F.GY, b2);
        k_mg_prolong<<<grid2d(F.GX, F.GY, b2), b2, 0, c->stream>>>(F, C);
        for (int s = 0; s < kNu; ++s) {
            k_mg_rbgs<<<gh, b2, 0, c->stream>>>(F, 1);
            k_mg_rbgs<<<gh, b2, 0, c->stream>>>(F, 0);
        }
    }
    PIC_CUDA(cudaGetLastError());
    return PIC_OK;
}

}  // namespace

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
    ps.nblocks = (int)std::min<int64_t>((c->nodes + kRedThreads - 1) / kRedThreads, 148 * 8);
    PIC_CUDA(cudaMalloc(&ps.partials, (size_t)ps.nblocks * 4 * sizeof(double)));
    PIC_CUDA(cudaMalloc(&ps.scal, 16 * sizeof(double)));
    PIC_CUDA(cudaMemsetAsync(ps.scal, 0, 16 * sizeof(double), c->stream));
    PIC_CUDA(cudaMallocHost(&ps.host_scal, 16 * sizeof(double)));
    PIC_CUDA(cudaEventCreate(&ps.ev0));
    PIC_CUDA(cudaEventCreate(&ps.ev1));
    // multigrid hierarchy
    int nx = c->nx, ny = c->ny;
    double hx = c->dx, hy = c->dy;
    const uint8_t* prev_mask = c->mask;
    int pGX = c->GX, pGY = c->GY;
    for (int l = 0; l < 16; ++l) {
        MGLevel L{};
        L.nx = nx;
        L.ny = ny;
        L.GX = nx + 1;
        L.GY = ny + 1;
        L.nodes = (int64_t)L.GX * L.GY;
        L.cx = (float)(1.0 / (hx * hx));
        L.cy = (float)(1.0 / (hy * hy));
        L.cd = 2.0f * (L.cx + L.cy);
        PIC_CUDA(cudaMalloc(&L.x, (size_t)L.nodes * 4));
        PIC_CUDA(cudaMalloc(&L.b, (size_t)L.nodes * 4));
        PIC_CUDA(cudaMemsetAsync(L.x, 0, (size_t)L.nodes * 4, c->stream));
        PIC_CUDA(cudaMemsetAsync(L.b, 0, (size_t)L.nodes * 4, c->stream));
        if (l == 0) {
            L.mask = c->mask;
        } else {
            PIC_CUDA(cudaMalloc(&L.mask, (size_t)L.nodes));
            const dim3 b2(32, 8);
            k_mg_coarse_mask<<<grid2d(L.GX, L.GY, b2), b2, 0, c->stream>>>(prev_mask, pGX, pGY,
                                                                           L.mask, L.GX, L.GY);
            PIC_CUDA(cudaGetLastError());
        }
        ps.levels.push_back(L);
        if (std::min(nx, ny) <= 4) break;
        prev_mask = L.mask;
        pGX = L.GX;
        pGY = L.GY;
        nx = (nx + 1) / 2;
        ny = (ny + 1) / 2;
        hx *= 2;
        hy *= 2;
    }
    return PIC_OK;
}

void poisson_free(pic_ctx* c) {
    PoissonState& ps = c->ps;
    for (size_t l = 0; l < ps.levels.size(); ++l) {
        cudaFree(ps.levels[l].x);
        cudaFree(ps.levels[l].b);
        if (l > 0) cudaFree(ps.levels[l].mask);
    }
    ps.levels.clear();
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
    ps = PoissonState{};
}

int poisson_solve(pic_ctx* c) {
    PoissonState& ps = c->ps;
    const int64_t nodes = c->nodes;
    const Grid64 g = fine_grid(c);
    const int nb = ps.nblocks;
    unsigned* arrive = arrive_ptr(ps);
    PIC_CUDA(cudaEventRecord(ps.ev0, c->stream));
    prof_begin(c, PIC_PHASE_POISSON);
    const bool zero_start = (ps.warm == PIC_WARM_ZERO) || !ps.have_prev;
    k_overwrite_rho<<<(unsigned)((nodes + 255) / 256), 256, 0, c->stream>>>(
        nodes, c->mask, c->dir_val, c->rho, c->phi, zero_start ? 1 : 0);
    if (ps.warm == PIC_WARM_LEARNED && ps.have_prev && ps.net_guess) {
        // the network's guess replaces phi on non-electrode nodes
        k_apply_guess<<<(unsigned)((nodes + 255) / 256), 256, 0, c->stream>>>(nodes, c->mask,
                                                                              ps.net_guess, c->phi);
    }
    float* r32 = ps.levels[0].b;
    float* z32 = ps.levels[0].x;
    // r = b - A x, ||r||^2 and ||b_red||^2 into the device scalars
    auto setup = [&]() -> int {
        k_pcg_setup<<<nb, kRedThreads, 0, c->stream>>>(g, c->mask, c->dir_val, c->rho, c->phi,
                                                       ps.r, r32, ps.partials, nb, arrive, ps.scal);
        k_fix_bb<<<1, 1, 0, c->stream>>>(ps.scal);
        c->launches += 2;
        PIC_CUDA(cudaGetLastError());
        PIC_CUDA(cudaMemcpyAsync(ps.host_scal, ps.scal, 8 * sizeof(double), cudaMemcpyDeviceToHost,
                                 c->stream));
        PIC_CUDA(cudaStreamSynchronize(c->stream));
        return PIC_OK;
    };
    PIC_TRY(setup());
    c->launches += 1;  // overwrite
    const double bb = ps.host_scal[S_BB];
    double rr = ps.host_scal[S_RR];
    const double target = ps.tol * ps.tol * bb;
    int it = 0, restarts = 0;
    int status = PIC_OK;
    const bool jacobi = ps.solver == PIC_SOLVER_JACOBI_PCG;
    double true_rr = rr;
    for (;;) {
        bool first = true;
        while (rr > target && bb > 0) {
            if (it >= ps.maxit) {
                status = PIC_ERR_NOT_CONVERGED;
                break;
            }
            if (!jacobi) PIC_TRY(vcycle(c));
            k_pcg_rz<<<nb, kRedThreads, 0, c->stream>>>(nodes, c->mask, ps.r, z32, 1.0 / g.cd,
                                                        jacobi ? 1 : 0, ps.z, ps.partials, nb,
                                                        arrive, ps.scal);
            double* p_old = ps.p[ps.pcur];
            double* p_new = ps.p[ps.pcur ^ 1];
            k_pcg_p_ap<<<nb, kRedThreads, 0, c->stream>>>(g, c->mask, ps.z, p_old, p_new, ps.q,
                                                          first ? 1 : 0, ps.partials, nb, arrive,
                                                          ps.scal);
            ps.pcur ^= 1;
            k_pcg_update<<<nb, kRedThreads, 0, c->stream>>>(nodes, c->mask, p_new, ps.q, c->phi,
                                                            ps.r, r32, ps.partials, nb, arrive,
                                                            ps.scal);
            k_shift_rz<<<1, 1, 0, c->stream>>>(ps.scal);
            c->launches += 4;
            PIC_CUDA(cudaGetLastError());
            PIC_CUDA(cudaMemcpyAsync(ps.host_scal + S_RR, ps.scal + S_RR, sizeof(double),
                                     cudaMemcpyDeviceToHost, c->stream));
            PIC_CUDA(cudaStreamSynchronize(c->stream));
            rr = ps.host_scal[S_RR];
            first = false;
            ++it;
            if (!std::isfinite(rr)) {
                status = PIC_ERR_NOT_CONVERGED;
                break;
            }
        }
        // the recursively updated residual can drift from b - A x: check the
        // true residual and restart from the current iterate if it is above
        // the target
        k_true_residual<<<nb, kRedThreads, 0, c->stream>>>(g, c->mask, c->rho, c->phi, ps.partials,
                                                           nb, arrive, ps.scal);
        c->launches += 1;
        PIC_CUDA(cudaMemcpyAsync(ps.host_scal + S_TRUE_RR, ps.scal + S_TRUE_RR, sizeof(double),
                                 cudaMemcpyDeviceToHost, c->stream));
        PIC_CUDA(cudaStreamSynchronize(c->stream));
        true_rr = ps.host_scal[S_TRUE_RR];
        if (status != PIC_OK || bb <= 0 || true_rr <= target || restarts >= 3) break;
        ++restarts;
        PIC_TRY(setup());
        rr = ps.host_scal[S_RR];
    }
    PIC_TRY(fields_from_phi(c));
    prof_end(c, PIC_PHASE_POISSON);
    PIC_CUDA(cudaEventRecord(ps.ev1, c->stream));
    PIC_CUDA(cudaStreamSynchronize(c->stream));
    float ms = 0;
    PIC_CUDA(cudaEventElapsedTime(&ms, ps.ev0, ps.ev1));
    ps.last_ms = ms;
    ps.last_iters = it;
    ps.last_relres = bb > 0 ? std::sqrt(true_rr / bb) : 0.0;
    ps.have_prev = true;
    if (status != PIC_OK)
        return fail(status, "Poisson PCG did not reach the tolerance within poisson_maxit");
    return PIC_OK;
}

int fields_from_phi(pic_ctx* c) {
    const dim3 b2(32, 8);
    k_efield<<<grid2d(c->GX, c->GY, b2), b2, 0, c->stream>>>(c->phi, c->bz, c->GX, c->GY, c->dx,
                                                             c->dy, c->fld);
    c->launches += 1;
    PIC_CUDA(cudaGetLastError());
    c->fields_valid = true;
    return PIC_OK;
}

int efield_export(pic_ctx* c) {
    const dim3 b2(32, 8);
    k_efield64<<<grid2d(c->GX, c->GY, b2), b2, 0, c->stream>>>(c->phi, c->GX, c->GY, c->dx, c->dy,
                                                               c->efield64);
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
