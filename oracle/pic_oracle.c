/*
 * pic_oracle.c -- FP64 CPU restatement of the 2D electrostatic PIC step of
 * SYCL-PIC-poissonsolver (vansh268p/BMP-6th-sem).
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: tests/, the smoke check
 * in __graft_entry__.py and the CPU-baseline leg of bench.py load it.  It is
 * never linked into, called by, or used as a fallback for the CUDA library.
 *
 * Two layers live here:
 *   1. Semantic restatement (orc_*): the reference's arithmetic, step by step,
 *      in FP64 -- bucket keys, the per-bucket CIC deposit, the bilinear gather
 *      plus Boris push with absorbing walls, the electrode mask, the CSR Poisson
 *      operator, overwriteRho / overwritePhi and the E field.
 *   2. Reference-structure port (orc_hm_* / orc_ref_*): the reference's
 *      per-node hashmap (insert with free-list reuse and linear probing,
 *      deletion, per-bucket cleanup, tail compaction) driving the same
 *      deposit and mover, threaded with OpenMP.  bench.py times this layer as
 *      the reference's CPU path, which cannot be built here (no SYCL compiler,
 *      no oneMKL/oneDPL/TBB).
 *
 * Parity status: the Poisson layer is pinned against the reference's own
 * PARDISO dumps (SYCL-PIC-poissonsolver/validation_dumps, 257x257 nodes).
 * Binning, deposit and push are pinned against the reference's own code run
 * here: oracle/ref_build.py compiles the bodies of deterministic_mover,
 * MoverKernel and interpolate's kernels from a reference checkout into a
 * host harness, and tests/test_oracle_ref_pin.py finds the push (walled and
 * periodic in y), the wall deletions, left exits, re-binned buckets and the
 * deposit equal to this file's bit for bit.  The periodic Poisson variants
 * (orc_build_csr_periodic, orc_overwrite_phi_periodic, orc_efield_periodic)
 * have no reference fixtures; the tests pin them by properties of the
 * periodic system instead.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Point: SYCL-PIC-poissonsolver/include/point.hpp:11-14 (6 doubles + int, 56 B). */
typedef struct {
    double x, y, z, vx, vy, vz;
    int32_t pointer;
    int32_t pad_;
} orc_point;

/* GridParams subset: include/species_ds.hpp:6-10.  nodes = (nx+1) x (ny+1).
 * width/height are GRID_WIDTH/GRID_HEIGHT (the XMAX/YMAX read from
 * M_PICDAT.DAT, src/particles.cpp:352-368), the bounds of the mover's wall
 * test; 0 means nx*dx / ny*dy. */
typedef struct {
    int32_t nx, ny;
    double dx, dy;
    double width, height;
} orc_grid;

static inline double grid_width(const orc_grid* g) { return g->width > 0 ? g->width : g->nx * g->dx; }
static inline double grid_height(const orc_grid* g) { return g->height > 0 ? g->height : g->ny * g->dy; }

/* Geometry: include/point.hpp:21-24 (inclusive node-index rectangle + volts). */
typedef struct {
    int32_t x1, y1, x2, y2;
    double potential;
} orc_geom;

int orc_sizeof_point(void) { return (int)sizeof(orc_point); }

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ------------------------------------------------------------------------- */
/* Binning key                                                                */
/* ------------------------------------------------------------------------- */

/* src/particles.cpp:230-235 (InsertKernel) and src/mover.cpp:309-324:
 * bucket = gy*GRID_X + gx with gx = (int)(x * (1/dx)).  Dead particles
 * (pointer == -1) get key -1. */
void orc_bucket_keys(const orc_grid* g, const orc_point* p, int64_t n, int32_t* keys) {
    const double inv_dx = 1.0 / g->dx, inv_dy = 1.0 / g->dy;
    const int64_t GX = g->nx + 1;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        if (p[i].pointer == -1) { keys[i] = -1; continue; }
        const int gx = (int)(p[i].x * inv_dx);
        const int gy = (int)(p[i].y * inv_dy);
        keys[i] = (int32_t)((int64_t)gy * GX + gx);
    }
}

/* Stable counting sort of particle indices by bucket key (live particles only).
 * counts[nodes], start[nodes+1], order[n_live]. Returns n_live. */
int64_t orc_bucket_sort(const int32_t* keys, int64_t n, int32_t nodes,
                        int32_t* counts, int64_t* start, int64_t* order) {
    memset(counts, 0, sizeof(int32_t) * (size_t)nodes);
    for (int64_t i = 0; i < n; ++i)
        if (keys[i] >= 0) counts[keys[i]]++;
    start[0] = 0;
    for (int32_t k = 0; k < nodes; ++k) start[k + 1] = start[k] + counts[k];
    int64_t* cur = (int64_t*)malloc(sizeof(int64_t) * (size_t)nodes);
    memcpy(cur, start, sizeof(int64_t) * (size_t)nodes);
    for (int64_t i = 0; i < n; ++i)
        if (keys[i] >= 0) order[cur[keys[i]]++] = i;
    free(cur);
    return start[nodes];
}

/* ------------------------------------------------------------------------- */
/* Deposit                                                                    */
/* ------------------------------------------------------------------------- */

/* One bucket's sums, src/interpolation.cpp:78-99: unnormalised bilinear
 * weights (dx-lx)(dy-ly), lx(dy-ly), (dx-lx)ly, lx*ly and the same weighted by
 * the particle's kinetic energy 0.5*v^2/|q/m| (eV). */
static inline void bucket_sums(const orc_grid* g, const orc_point* p, const int64_t* idx,
                               int64_t cnt, int gx, int gy, double denom, double s[8]) {
    for (int k = 0; k < 8; ++k) s[k] = 0.0;
    for (int64_t j = 0; j < cnt; ++j) {
        const orc_point* q = &p[idx[j]];
        const double lx = q->x - gx * g->dx;
        const double ly = q->y - gy * g->dy;
        const double v2 = q->vx * q->vx + q->vy * q->vy + q->vz * q->vz;
        const double en = 0.5 * v2 * denom;
        const double w1 = (g->dx - lx) * (g->dy - ly);
        const double w2 = lx * (g->dy - ly);
        const double w3 = (g->dx - lx) * ly;
        const double w4 = lx * ly;
        s[0] += w1; s[1] += w2; s[2] += w3; s[3] += w4;
        s[4] += w1 * en; s[5] += w2 * en; s[6] += w3 * en; s[7] += w4 * en;
    }
}

/* interpolate(), src/interpolation.cpp:13-171, semantic form.
 *   final_mesh[node]  = weighing * sum of the node's corner weights
 *   energy_mesh[node] = weighing * sum of energy-weighted corner weights
 *   rho[node]        += final_mesh[node] * (-charge/eps)      (RhoKernel :164-171)
 * weighing = actual*surfArea/(sim*dx*dy*dx*dy) (src/particles.cpp:303-305).
 * Buckets are visited in key order, particles within a bucket in array order.
 * rho may be NULL. */
void orc_deposit(const orc_grid* g, const orc_point* p, int64_t n, double weighing,
                 double ctom, double charge, double eps,
                 double* final_mesh, double* energy_mesh, double* rho) {
    const int32_t GX = g->nx + 1, GY = g->ny + 1;
    const int32_t nodes = GX * GY;
    int32_t* keys = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    int32_t* counts = (int32_t*)malloc(sizeof(int32_t) * (size_t)nodes);
    int64_t* start = (int64_t*)malloc(sizeof(int64_t) * (size_t)(nodes + 1));
    int64_t* order = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    double* corner = (double*)calloc((size_t)nodes * 8, sizeof(double));
    orc_bucket_keys(g, p, n, keys);
    orc_bucket_sort(keys, n, nodes, counts, start, order);
    const double denom = 1.0 / fabs(ctom);
#pragma omp parallel for schedule(dynamic, 64)
    for (int32_t b = 0; b < nodes; ++b) {
        const int gx = b % GX, gy = b / GX;
        /* InterReductionKernel :119 -- the last node row/column owns no cell. */
        if (gx + 1 >= GX || gy + 1 >= GY) continue;
        double s[8];
        bucket_sums(g, p, order + start[b], counts[b], gx, gy, denom, s);
        const int32_t p1 = gy * GX + gx, p2 = p1 + 1, p3 = p1 + GX, p4 = p3 + 1;
        corner[0 * (size_t)nodes + p1] = s[0] * weighing;
        corner[1 * (size_t)nodes + p2] = s[1] * weighing;
        corner[2 * (size_t)nodes + p3] = s[2] * weighing;
        corner[3 * (size_t)nodes + p4] = s[3] * weighing;
        corner[4 * (size_t)nodes + p1] = s[4] * weighing;
        corner[5 * (size_t)nodes + p2] = s[5] * weighing;
        corner[6 * (size_t)nodes + p3] = s[6] * weighing;
        corner[7 * (size_t)nodes + p4] = s[7] * weighing;
    }
    const double chrg = -charge / eps;
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < nodes; ++i) {
        /* ReducePartialMeshesKernel :150-163 sums the four corner meshes in order. */
        double f = 0.0, e = 0.0;
        for (int k = 0; k < 4; ++k) {
            f += corner[(size_t)k * nodes + i];
            e += corner[(size_t)(k + 4) * nodes + i];
        }
        final_mesh[i] = f;
        energy_mesh[i] = e;
        if (rho) rho[i] += f * chrg;
    }
    free(keys); free(counts); free(start); free(order); free(corner);
}

/* ------------------------------------------------------------------------- */
/* Gather + Boris push + absorbing walls                                      */
/* ------------------------------------------------------------------------- */

/* deterministic_mover(), src/mover.cpp:103-176.  efield is the interleaved
 * Field array (fx, fy per node), bz the node magnetic field.  The cell used
 * for the gather is (int)(x/dx) -- a division, as at :115-116.  Every
 * expression keeps the reference's operand order and association (products
 * left to right, e.g. (E*(dx-lx))*(dy-ly)), so that with the same compiler
 * flags (no FMA contraction) the result is the reference's bit for bit. */
static inline void mover_one(orc_point* q, const orc_grid* g, double pctm, double dt,
                             const double* efield, const double* bz) {
    const int GX = g->nx + 1;
    const double dx = g->dx, dy = g->dy;
    double px = q->x, py = q->y, pz = q->z, pvx = q->vx, pvy = q->vy, pvz = q->vz;
    const int gx = (int)(px / dx);
    const int gy = (int)(py / dy);
    const double lx = px - gx * dx;
    const double ly = py - gy * dy;
    const int n1 = gy * GX + gx, n2 = gy * GX + (gx + 1), n3 = (gy + 1) * GX + gx,
              n4 = (gy + 1) * GX + (gx + 1);
    const double Epx = (efield[2 * n1] * (dx - lx) * (dy - ly) + efield[2 * n2] * lx * (dy - ly) +
                        efield[2 * n3] * (dx - lx) * ly + efield[2 * n4] * lx * ly) / (dx * dy);
    const double Epy = (efield[2 * n1 + 1] * (dx - lx) * (dy - ly) +
                        efield[2 * n2 + 1] * lx * (dy - ly) + efield[2 * n3 + 1] * (dx - lx) * ly +
                        efield[2 * n4 + 1] * lx * ly) / (dx * dy);
    const double Bpz = (bz[n1] * (dx - lx) * (dy - ly) + bz[n2] * lx * (dy - ly) +
                        bz[n3] * (dx - lx) * ly + bz[n4] * lx * ly) / (dx * dy);
    /* Boris with Bz only, :151-166. */
    const double Vxminus = pvx + 0.5 * pctm * Epx * dt;
    const double Vyminus = pvy + 0.5 * pctm * Epy * dt;
    const double t = 0.5 * pctm * Bpz * dt;
    const double Vxprime = Vxminus + Vyminus * t;
    const double Vyprime = Vyminus - Vxminus * t;
    const double s = 2 * t / (1 + t * t);
    pvx = Vxminus + Vyprime * s + 0.5 * pctm * Epx * dt;
    pvy = Vyminus - Vxprime * s + 0.5 * pctm * Epy * dt;
    px = px + dt * pvx;
    py = py + dt * pvy;
    pz = pz + dt * pvz;
    q->x = px; q->y = py; q->z = pz; q->vx = pvx; q->vy = pvy; q->vz = pvz;
}

/* modulo(), src/mover.cpp:13-22: x wrapped into [0, y); a negative exact
 * multiple of y gives 0. */
static inline double ref_modulo(double x, double y) {
    if (x < 0) {
        if ((int)(x / y) == x / y) return 0;
        return y - fmod(-x, y);
    }
    return fmod(x, y);
}

/* MoverKernel, src/mover.cpp:304-366, semantic form: push every live
 * particle; with periodic_y the new y is first wrapped by modulo(y, H)
 * (:317-320).  A particle with x outside [0,W) or y outside [0,H) is deleted
 * (pointer = -1) and counted as a left exit when x < 0.  Returns the number
 * deleted; *left_exits receives the x<0 count. */
int64_t orc_push_mode(const orc_grid* g, orc_point* p, int64_t n, double ctom, double dt,
                      const double* efield, const double* bz, int32_t periodic_y,
                      int64_t* left_exits) {
    const double W = grid_width(g), H = grid_height(g);
    int64_t deleted = 0, left = 0;
#pragma omp parallel for schedule(static) reduction(+ : deleted, left)
    for (int64_t i = 0; i < n; ++i) {
        orc_point* q = &p[i];
        if (q->pointer == -1) continue;
        mover_one(q, g, ctom, dt, efield, bz);
        if (periodic_y) q->y = ref_modulo(q->y, H);
        const double px = q->x, py = q->y;
        if (px >= W || px < 0.0 || py >= H || py < 0) {
            q->pointer = -1;
            deleted++;
            if (px < 0.0) left++;
        }
    }
    if (left_exits) *left_exits = left;
    return deleted;
}

int64_t orc_push(const orc_grid* g, orc_point* p, int64_t n, double ctom, double dt,
                 const double* efield, const double* bz, int64_t* left_exits) {
    return orc_push_mode(g, p, n, ctom, dt, efield, bz, 0, left_exits);
}

/* calculate_energy(), src/utils.cpp:77-118: sum of 0.5*v^2/|q/m| (eV). */
double orc_kinetic_energy(const orc_point* p, int64_t n, double ctom) {
    const double denom = fabs(ctom);
    double tot = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : tot)
    for (int64_t i = 0; i < n; ++i) {
        if (p[i].pointer == -1) continue;
        const double v2 = p[i].vx * p[i].vx + p[i].vy * p[i].vy + p[i].vz * p[i].vz;
        tot += 0.5 * v2 / denom;
    }
    return tot;
}

/* ------------------------------------------------------------------------- */
/* Poisson pieces                                                             */
/* ------------------------------------------------------------------------- */

/* readGeometry(), src/particles.cpp:677-681: fractions -> node indices,
 * (int)((GRID-1)*fraction). */
void orc_geom_from_fractions(int32_t GX, int32_t GY, const double* frac5, int32_t count,
                             orc_geom* out) {
    for (int32_t i = 0; i < count; ++i) {
        const double* f = frac5 + 5 * i;
        out[i].x1 = (int32_t)((double)(GX - 1) * f[0]);
        out[i].y1 = (int32_t)((double)(GY - 1) * f[1]);
        out[i].x2 = (int32_t)((double)(GX - 1) * f[2]);
        out[i].y2 = (int32_t)((double)(GY - 1) * f[3]);
        out[i].potential = f[4];
    }
}

/* setPotentialBoundary(), src/poissonSolver.cpp:64-79 (inclusive ranges). */
void orc_electrode_mask(int32_t GX, int32_t GY, const orc_geom* geo, int32_t count,
                        uint8_t* mask) {
    memset(mask, 0, (size_t)GX * GY);
    for (int32_t i = 0; i < count; ++i)
        for (int32_t k = geo[i].y1; k <= geo[i].y2; ++k)
            for (int32_t j = geo[i].x1; j <= geo[i].x2; ++j) mask[(size_t)k * GX + j] = 1;
}

/* generateCoeffs(), src/poissonSolver.cpp:183-241, 0-based CSR over all nodes:
 * electrode row = [-1]; interior row = [-1/dy^2, -1/dx^2, 2(1/dx^2+1/dy^2),
 * -1/dx^2, -1/dy^2] at columns i-GX, i-1, i, i+1, i+GX.  Returns nnz. */
int64_t orc_build_csr(int32_t GX, int32_t GY, double dx, double dy, const uint8_t* mask,
                      int64_t* row_ptr, int64_t* col, double* val) {
    const double inv_dx2 = 1.0 / (dx * dx), inv_dy2 = 1.0 / (dy * dy);
    int64_t idx = 0;
    row_ptr[0] = 0;
    for (int64_t i = 0; i < (int64_t)GX * GY; ++i) {
        if (mask[i] == 1) {
            val[idx] = -1; col[idx] = i; idx++;
        } else {
            val[idx + 0] = -inv_dy2; col[idx + 0] = i - GX;
            val[idx + 1] = -inv_dx2; col[idx + 1] = i - 1;
            val[idx + 2] = 2 * (inv_dx2 + inv_dy2); col[idx + 2] = i;
            val[idx + 3] = -inv_dx2; col[idx + 3] = i + 1;
            val[idx + 4] = -inv_dy2; col[idx + 4] = i + GX;
            idx += 5;
        }
        row_ptr[i + 1] = idx;
    }
    return idx;
}

/* generateCoeffsPeriodic(), src/poissonSolver.cpp:82-180, 0-based CSR over
 * the N = GX*(GY-1) nodes of rows 0..GY-2 (row GY-1 is row 0): electrode row
 * = [-1]; other rows the 5-point stencil with the row above the last row
 * being row 0 and the row below row 0 the last row (columns i+-GX modulo N).
 * Returns nnz, or -1 when a non-electrode node lies in the first or last
 * column (the reference's i-1 / i+1 would then reach into another row, or
 * outside the matrix at node 0). */
int64_t orc_build_csr_periodic(int32_t GX, int32_t GY, double dx, double dy, const uint8_t* mask,
                               int64_t* row_ptr, int64_t* col, double* val) {
    const double inv_dx2 = 1.0 / (dx * dx), inv_dy2 = 1.0 / (dy * dy);
    const int64_t N = (int64_t)GX * (GY - 1);
    int64_t idx = 0;
    row_ptr[0] = 0;
    for (int64_t i = 0; i < N; ++i) {
        if (mask[i] == 1) {
            val[idx] = -1; col[idx] = i; idx++;
        } else {
            const int64_t c = i % GX;
            if (c == 0 || c == GX - 1) return -1;
            val[idx + 0] = -inv_dy2; col[idx + 0] = (i - GX + N) % N;
            val[idx + 1] = -inv_dx2; col[idx + 1] = i - 1;
            val[idx + 2] = 2 * (inv_dx2 + inv_dy2); col[idx + 2] = i;
            val[idx + 3] = -inv_dx2; col[idx + 3] = i + 1;
            val[idx + 4] = -inv_dy2; col[idx + 4] = (i + GX) % N;
            idx += 5;
        }
        row_ptr[i + 1] = idx;
    }
    return idx;
}

/* overwriteRho(), src/poissonSolver.cpp:384-402: electrode nodes <- V, then
 * the whole array is negated (it becomes PARDISO's right-hand side). */
void orc_overwrite_rho(int32_t GX, int32_t GY, const orc_geom* geo, int32_t count, double* rho) {
    for (int32_t i = 0; i < count; ++i)
        for (int32_t j = geo[i].y1; j <= geo[i].y2; ++j)
            for (int32_t k = geo[i].x1; k <= geo[i].x2; ++k) rho[(size_t)j * GX + k] = geo[i].potential;
    for (int64_t i = 0; i < (int64_t)GX * GY; ++i) rho[i] = -rho[i];
}

/* overwritePhi(), src/poissonSolver.cpp:364-382 (non-periodic). */
void orc_overwrite_phi(int32_t GX, int32_t GY, const orc_geom* geo, int32_t count, double* phi) {
    (void)GY;
    for (int32_t i = 0; i < count; ++i)
        for (int32_t j = geo[i].y1; j <= geo[i].y2; ++j)
            for (int32_t k = geo[i].x1; k <= geo[i].x2; ++k) phi[(size_t)j * GX + k] = geo[i].potential;
}

/* overwritePhi() with periodicBoundary, src/poissonSolver.cpp:364-382: row 0
 * is copied into row GY-1, then the electrode potentials are imposed. */
void orc_overwrite_phi_periodic(int32_t GX, int32_t GY, const orc_geom* geo, int32_t count,
                                double* phi) {
    memcpy(phi + (size_t)(GY - 1) * GX, phi, sizeof(double) * (size_t)GX);
    orc_overwrite_phi(GX, GY, geo, count, phi);
}

/* calculateElectricFieldPeriodic(), src/poissonSolver.cpp:411-430: fx is
 * one-sided at the first and last column and central elsewhere, on every
 * row; fy is central with rows taken modulo GY-1, on every row. */
void orc_efield_periodic(int32_t GX, int32_t GY, double dx, double dy, const double* phi,
                         double* efield) {
    for (int32_t i = 0; i < GY; ++i) {
        const size_t a = (size_t)i * GX;
        efield[2 * a] = -((phi[a + 1] - phi[a]) / dx);
        for (int32_t j = 1; j < GX - 1; ++j)
            efield[2 * (a + j)] = -((phi[a + j + 1] - phi[a + j - 1]) / (2 * dx));
        const size_t b = a + GX - 1;
        efield[2 * b] = -((phi[b] - phi[b - 1]) / dx);
    }
    const int32_t P = GY - 1;
    for (int32_t j = 0; j < GX; ++j)
        for (int32_t i = 0; i < GY; ++i) {
            const size_t up = (size_t)((i + 1) % P) * GX + j, dn = (size_t)((i - 1 + P) % P) * GX + j;
            efield[2 * ((size_t)i * GX + j) + 1] = -((phi[up] - phi[dn]) / (2 * dy));
        }
}

/* calculateElectricField(), src/poissonSolver.cpp:433-456: central
 * differences inside, then first/last column copy their neighbour, then
 * first/last row copy theirs.  efield is interleaved (fx, fy). */
void orc_efield(int32_t GX, int32_t GY, double dx, double dy, const double* phi, double* efield) {
    for (int32_t i = 1; i < GY - 1; ++i)
        for (int32_t j = 1; j < GX - 1; ++j) {
            const size_t n = (size_t)i * GX + j;
            efield[2 * n] = -((phi[n + 1] - phi[n - 1]) / (2 * dx));
            efield[2 * n + 1] = -((phi[n + GX] - phi[n - GX]) / (2 * dy));
        }
    for (int32_t i = 0; i < GY; ++i) {
        const size_t a = (size_t)i * GX, b = (size_t)(i + 1) * GX - 1;
        efield[2 * a] = efield[2 * (a + 1)]; efield[2 * a + 1] = efield[2 * (a + 1) + 1];
        efield[2 * b] = efield[2 * (b - 1)]; efield[2 * b + 1] = efield[2 * (b - 1) + 1];
    }
    for (int32_t j = 0; j < GX; ++j) {
        const size_t a = (size_t)j, a1 = (size_t)GX + j;
        const size_t b = (size_t)GX * (GY - 1) + j, b1 = (size_t)GX * (GY - 2) + j;
        efield[2 * a] = efield[2 * a1]; efield[2 * a + 1] = efield[2 * a1 + 1];
        efield[2 * b] = efield[2 * b1]; efield[2 * b + 1] = efield[2 * b1 + 1];
    }
}

/* y = A x for the generateCoeffs operator (matrix free).  Electrode rows give
 * -x[i]; interior rows the 5-point stencil. */
void orc_apply_a(int32_t GX, int32_t GY, double dx, double dy, const uint8_t* mask,
                 const double* x, double* y) {
    const double cx = 1.0 / (dx * dx), cy = 1.0 / (dy * dy), cd = 2 * (cx + cy);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)GX * GY; ++i) {
        if (mask[i]) { y[i] = -x[i]; continue; }
        y[i] = -cy * x[i - GX] - cx * x[i - 1] + cd * x[i] - cx * x[i + 1] - cy * x[i + GX];
    }
}

/* FP64 conjugate gradients on the SPD system left once the electrode rows of
 * A phi = b are eliminated (b = the overwritten rho).  phi holds the start
 * guess on entry (electrode values are imposed first) and the solution on
 * exit.  Stops when ||b_int - A_int phi|| <= tol*||b_int|| over the
 * non-electrode rows.  Returns the iteration count; *relres the final ratio. */
int orc_cg_solve(int32_t GX, int32_t GY, double dx, double dy, const uint8_t* mask,
                 const double* b, double* phi, double tol, int maxit, double* relres) {
    const int64_t n = (int64_t)GX * GY;
    double* r = (double*)malloc(sizeof(double) * (size_t)n);
    double* pv = (double*)calloc((size_t)n, sizeof(double));
    double* q = (double*)malloc(sizeof(double) * (size_t)n);
    for (int64_t i = 0; i < n; ++i)
        if (mask[i]) phi[i] = -b[i];
    orc_apply_a(GX, GY, dx, dy, mask, phi, q);
    double rr = 0.0, bb = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        r[i] = mask[i] ? 0.0 : b[i] - q[i];
        pv[i] = r[i];
        rr += r[i] * r[i];
        /* right-hand side of the reduced system: b_i plus the known electrode
         * neighbours moved across */
        if (!mask[i]) {
            const double cx = 1.0 / (dx * dx), cy = 1.0 / (dy * dy);
            double bi = b[i];
            if (mask[i - 1]) bi += cx * phi[i - 1];
            if (mask[i + 1]) bi += cx * phi[i + 1];
            if (mask[i - GX]) bi += cy * phi[i - GX];
            if (mask[i + GX]) bi += cy * phi[i + GX];
            bb += bi * bi;
        }
    }
    const double bn = sqrt(bb) > 0 ? sqrt(bb) : 1.0;
    int it = 0;
    while (sqrt(rr) > tol * bn && it < maxit) {
        orc_apply_a(GX, GY, dx, dy, mask, pv, q);
        double pq = 0.0;
        for (int64_t i = 0; i < n; ++i)
            if (!mask[i]) pq += pv[i] * q[i];
        const double alpha = rr / pq;
        double rr_new = 0.0;
        for (int64_t i = 0; i < n; ++i) {
            if (mask[i]) continue;
            phi[i] += alpha * pv[i];
            r[i] -= alpha * q[i];
            rr_new += r[i] * r[i];
        }
        const double beta = rr_new / rr;
        rr = rr_new;
        for (int64_t i = 0; i < n; ++i) pv[i] = mask[i] ? 0.0 : r[i] + beta * pv[i];
        it++;
    }
    if (relres) *relres = sqrt(rr) / bn;
    free(r); free(pv); free(q);
    return it;
}

/* ------------------------------------------------------------------------- */
/* Reference-structure port: the per-node hashmap (sycl_hashmap.hpp)          */
/* ------------------------------------------------------------------------- */

/* DeviceView, include/sycl_hashmap.hpp:18-240.  keys: -1 empty, 0 deleted,
 * 1 occupied; values: particle index (or free-list link); key_idx[b]: bucket
 * high-water mark; delete_idx[b]: free-list head. */
typedef struct {
    int32_t* keys;
    int32_t* values;
    int32_t* key_idx;
    int32_t* delete_idx;
    int64_t capacity;
    int32_t probing_length;
    int32_t nbuckets;
} orc_hmap;

static inline int32_t ld(int32_t* a) { return __atomic_load_n(a, __ATOMIC_ACQUIRE); }
static inline void st(int32_t* a, int32_t v) { __atomic_store_n(a, v, __ATOMIC_RELEASE); }
static inline int cas(int32_t* a, int32_t* expected, int32_t v) {
    return __atomic_compare_exchange_n(a, expected, v, 0, __ATOMIC_ACQ_REL, __ATOMIC_ACQUIRE);
}

/* SyclHashMap ctor + initKernel/initKeyKernel (src/particles.cpp:181, 202-221):
 * capacity = nbuckets*probing_length*slack. */
orc_hmap* orc_hm_create(int32_t nbuckets, int32_t probing_length, double slack) {
    orc_hmap* m = (orc_hmap*)calloc(1, sizeof(orc_hmap));
    m->nbuckets = nbuckets;
    m->probing_length = probing_length;
    m->capacity = (int64_t)((double)nbuckets * probing_length * slack);
    m->keys = (int32_t*)malloc(sizeof(int32_t) * (size_t)m->capacity);
    m->values = (int32_t*)malloc(sizeof(int32_t) * (size_t)m->capacity);
    m->key_idx = (int32_t*)malloc(sizeof(int32_t) * (size_t)nbuckets);
    m->delete_idx = (int32_t*)malloc(sizeof(int32_t) * (size_t)nbuckets);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m->capacity; ++i) { m->keys[i] = -1; m->values[i] = -1; }
    for (int32_t b = 0; b < nbuckets; ++b) { m->key_idx[b] = 0; m->delete_idx[b] = -1; }
    return m;
}

void orc_hm_destroy(orc_hmap* m) {
    if (!m) return;
    free(m->keys); free(m->values); free(m->key_idx); free(m->delete_idx); free(m);
}

/* pop_from_free_list, sycl_hashmap.hpp:36-58. */
static int32_t hm_pop_free(orc_hmap* m, int32_t b) {
    int32_t head, next;
    do {
        head = ld(&m->delete_idx[b]);
        if (head == -1) return -1;
        next = ld(&m->values[head]);
    } while (!cas(&m->delete_idx[b], &head, next));
    return head;
}

/* insert, sycl_hashmap.hpp:131-197: reuse a deleted slot, else probe from the
 * bucket's high-water mark.  The reference writes key_idx non-atomically after
 * the CAS (a race that can hide a slot from the deposit); this port raises it
 * with an atomic max, the intended semantics. */
static int32_t hm_insert(orc_hmap* m, int32_t key, int32_t value) {
    int32_t idx = hm_pop_free(m, key);
    while (idx != -1) {
        int32_t expected = 0;
        if (cas(&m->keys[idx], &expected, 1)) {
            st(&m->values[idx], value);
            return idx;
        }
        idx = hm_pop_free(m, key);
    }
    const int64_t hash = (int64_t)key * m->probing_length;
    for (int32_t i = ld(&m->key_idx[key]); i < m->probing_length; ++i) {
        const int64_t pi = hash + i;
        if (pi >= m->capacity) return -1;
        int32_t expected = -1;
        if (cas(&m->keys[pi], &expected, key)) {
            st(&m->keys[pi], 1);
            st(&m->values[pi], value);
            int32_t cur = ld(&m->key_idx[key]);
            while (cur < i + 1 && !cas(&m->key_idx[key], &cur, i + 1)) {}
            return (int32_t)pi;
        }
    }
    return -1;
}

/* deletion, sycl_hashmap.hpp:199-231: mark deleted, push on the free list. */
static void hm_delete(orc_hmap* m, int32_t slot) {
    const int32_t b = slot / m->probing_length;
    st(&m->keys[slot], 0);
    int32_t old_head;
    do {
        old_head = ld(&m->delete_idx[b]);
        st(&m->values[slot], old_head);
    } while (!cas(&m->delete_idx[b], &old_head, slot));
}

/* registerParticle's InsertKernel, src/particles.cpp:227-237.  Returns the
 * number of failed inserts (map overflow). */
int64_t orc_ref_register(orc_hmap* m, const orc_grid* g, orc_point* p, int64_t n) {
    const double inv_dx = 1.0 / g->dx, inv_dy = 1.0 / g->dy;
    const int32_t GX = g->nx + 1;
    int64_t failed = 0;
#pragma omp parallel for schedule(static) reduction(+ : failed)
    for (int64_t i = 0; i < n; ++i) {
        const int gx = (int)(p[i].x * inv_dx), gy = (int)(p[i].y * inv_dy);
        p[i].pointer = hm_insert(m, gy * GX + gx, (int32_t)i);
        if (p[i].pointer == -1) failed++;
    }
    return failed;
}

/* Bucket fill counts (live slots below the high-water mark). */
void orc_hm_counts(const orc_hmap* m, int32_t* counts) {
#pragma omp parallel for schedule(static)
    for (int32_t b = 0; b < m->nbuckets; ++b) {
        int32_t c = 0;
        const int64_t base = (int64_t)b * m->probing_length;
        for (int32_t i = 0; i < m->key_idx[b]; ++i)
            if (m->keys[base + i] == 1 && m->values[base + i] != -1) c++;
        counts[b] = c;
    }
}

/* Member particle indices of bucket b, in slot order; returns the count. */
int32_t orc_hm_members(const orc_hmap* m, int32_t b, int32_t* out, int32_t cap) {
    int32_t c = 0;
    const int64_t base = (int64_t)b * m->probing_length;
    for (int32_t i = 0; i < m->key_idx[b]; ++i)
        if (m->keys[base + i] == 1 && m->values[base + i] != -1) {
            if (c < cap) out[c] = m->values[base + i];
            c++;
        }
    return c;
}

/* interpolate() over the hashmap, src/interpolation.cpp:56-171: each bucket
 * sums over its slots below key_idx that are occupied. */
void orc_ref_deposit(const orc_hmap* m, const orc_grid* g, const orc_point* p, double weighing,
                     double ctom, double charge, double eps, double* final_mesh,
                     double* energy_mesh, double* rho) {
    const int32_t GX = g->nx + 1, GY = g->ny + 1, nodes = GX * GY;
    double* corner = (double*)calloc((size_t)nodes * 8, sizeof(double));
    const double denom = 1.0 / fabs(ctom);
#pragma omp parallel for schedule(dynamic, 64)
    for (int32_t b = 0; b < nodes; ++b) {
        const int gx = b % GX, gy = b / GX;
        if (gx + 1 >= GX || gy + 1 >= GY) continue;
        const int64_t base = (int64_t)b * m->probing_length;
        double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int32_t i = 0; i < m->key_idx[b]; ++i) {
            if (m->keys[base + i] == 0 || m->values[base + i] == -1) continue;
            const orc_point* q = &p[m->values[base + i]];
            const double lx = q->x - gx * g->dx, ly = q->y - gy * g->dy;
            const double v2 = q->vx * q->vx + q->vy * q->vy + q->vz * q->vz;
            const double en = 0.5 * v2 * denom;
            const double w1 = (g->dx - lx) * (g->dy - ly), w2 = lx * (g->dy - ly),
                         w3 = (g->dx - lx) * ly, w4 = lx * ly;
            s[0] += w1; s[1] += w2; s[2] += w3; s[3] += w4;
            s[4] += w1 * en; s[5] += w2 * en; s[6] += w3 * en; s[7] += w4 * en;
        }
        const int32_t p1 = gy * GX + gx, p2 = p1 + 1, p3 = p1 + GX, p4 = p3 + 1;
        corner[0 * (size_t)nodes + p1] = s[0] * weighing;
        corner[1 * (size_t)nodes + p2] = s[1] * weighing;
        corner[2 * (size_t)nodes + p3] = s[2] * weighing;
        corner[3 * (size_t)nodes + p4] = s[3] * weighing;
        corner[4 * (size_t)nodes + p1] = s[4] * weighing;
        corner[5 * (size_t)nodes + p2] = s[5] * weighing;
        corner[6 * (size_t)nodes + p3] = s[6] * weighing;
        corner[7 * (size_t)nodes + p4] = s[7] * weighing;
    }
    const double chrg = -charge / eps;
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < nodes; ++i) {
        double f = 0.0, e = 0.0;
        for (int k = 0; k < 4; ++k) {
            f += corner[(size_t)k * nodes + i];
            e += corner[(size_t)(k + 4) * nodes + i];
        }
        final_mesh[i] = f;
        energy_mesh[i] = e;
        if (rho) rho[i] += f * chrg;
    }
    free(corner);
}

/* mover() / MoverKernel over the hashmap, src/mover.cpp:304-420: push, then
 * delete out-of-bounds particles (recording the hole in empty_space) or
 * rehash on a cell change.  Failed inserts are retried once (MoverInsertions);
 * returns the number still failing (the reference exits on that). */
int64_t orc_ref_mover(orc_hmap* m, const orc_grid* g, orc_point* p, int64_t n, double ctom,
                      double dt, const double* efield, const double* bz, int32_t* empty_space,
                      int64_t* n_empty, int64_t* new_additions) {
    const double W = grid_width(g), H = grid_height(g);
    const double inv_dx = 1.0 / g->dx, inv_dy = 1.0 / g->dy;
    const int32_t GX = g->nx + 1;
    int64_t holes = *n_empty, left = 0;
    int32_t* retry = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    int64_t nretry = 0;
#pragma omp parallel for schedule(static) reduction(+ : left)
    for (int64_t i = 0; i < n; ++i) {
        orc_point q = p[i];
        if (q.pointer == -1) continue;
        const int gxb = (int)(q.x * inv_dx), gyb = (int)(q.y * inv_dy);
        mover_one(&q, g, ctom, dt, efield, bz);
        const double px = q.x, py = q.y;
        const int gya = (int)(py * inv_dy), gxa = (int)(px * inv_dx);
        if (px >= W || px < 0.0 || py >= H || py < 0) {
            hm_delete(m, q.pointer);
            q.pointer = -1;
            const int64_t k = __atomic_fetch_add(&holes, 1, __ATOMIC_RELAXED);
            if (k < n) empty_space[k] = (int32_t)i;
            if (px < 0.0) left++;
        } else if (gxb != gxa || gyb != gya) {
            hm_delete(m, q.pointer);
            q.pointer = hm_insert(m, gya * GX + gxa, (int32_t)i);
            if (q.pointer == -1) {
                const int64_t k = __atomic_fetch_add(&nretry, 1, __ATOMIC_RELAXED);
                retry[k] = (int32_t)i;
            }
        }
        p[i] = q;
    }
    int64_t failed = 0;
    for (int64_t k = 0; k < nretry; ++k) {
        orc_point* q = &p[retry[k]];
        const int gx = (int)(q->x * inv_dx), gy = (int)(q->y * inv_dy);
        q->pointer = hm_insert(m, gy * GX + gx, retry[k]);
        if (q->pointer == -1) failed++;
    }
    free(retry);
    *n_empty = holes < n ? holes : n;
    if (new_additions) *new_additions += left;
    return failed;
}

/* cleanup + cleanup_clear_freelist per bucket, sycl_hashmap.hpp:60-129,
 * driven by cleanup_map (src/utils.cpp:30-44). */
void orc_ref_cleanup(orc_hmap* m, orc_point* p) {
#pragma omp parallel for schedule(dynamic, 256)
    for (int32_t b = 0; b < m->nbuckets; ++b) {
        const int64_t base = (int64_t)b * m->probing_length;
        int32_t k = m->key_idx[b] - 1;
        if (k >= 0) {
            /* pop_from_deleted (non-atomic, single owner) */
            int32_t fs = m->delete_idx[b];
            if (fs != -1) m->delete_idx[b] = m->values[fs];
            while (fs != -1 && k != -1) {
                while (k >= 0 && m->keys[k + base] == 0) k--;
                if (k < 0) {
                    m->values[fs] = m->delete_idx[b];
                    m->delete_idx[b] = fs;
                    break;
                }
                if (fs >= k + base) {
                    m->keys[fs] = -1;
                    m->values[fs] = -1;
                } else {
                    m->keys[k + base] = -1;
                    m->keys[fs] = 1;
                    m->values[fs] = m->values[k + base];
                    m->values[k + base] = -1;
                    k--;
                    p[m->values[fs]].pointer = fs;
                }
                fs = m->delete_idx[b];
                if (fs != -1) m->delete_idx[b] = m->values[fs];
            }
            m->key_idx[b] = k + 1;
        }
        if (m->key_idx[b] - 1 < 0) {
            int32_t head = m->delete_idx[b];
            while (head != -1) {
                const int32_t next = m->values[head];
                m->keys[head] = -1;
                m->values[head] = -1;
                head = next;
            }
            m->delete_idx[b] = -1;
            m->key_idx[b] = 0;
        }
    }
}

/* compact_particles(), src/utils.cpp:249-372: fill holes below the new end
 * from live particles at the tail and patch the map's values.  Returns the
 * new particle count. */
int64_t orc_ref_compact(orc_hmap* m, orc_point* p, int64_t end, const int32_t* empty_space,
                        int64_t n_empty) {
    if (n_empty == 0) return end;
    const int64_t keep = end - n_empty;
    int64_t* dst = (int64_t*)malloc(sizeof(int64_t) * (size_t)n_empty);
    int64_t* src = (int64_t*)malloc(sizeof(int64_t) * (size_t)n_empty);
    int64_t nd = 0, ns = 0;
    for (int64_t i = 0; i < n_empty; ++i)
        if (empty_space[i] < keep) dst[nd++] = empty_space[i];
    for (int64_t i = 0; i < n_empty; ++i)
        if (p[end - i - 1].pointer != -1) src[ns++] = end - i - 1;
    const int64_t moves = nd < ns ? nd : ns;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < moves; ++i) {
        p[dst[i]] = p[src[i]];
        if (p[dst[i]].pointer != -1) m->values[p[dst[i]].pointer] = (int32_t)dst[i];
        p[src[i]].pointer = -1;
    }
    free(dst); free(src);
    return keep;
}

/* ------------------------------------------------------------------------- */
/* Synthetic plasma for the CPU baseline (bench.py's reference arm)           */
/* ------------------------------------------------------------------------- */

/* splitmix64 (Steele, Lea, Flood, "Fast splittable pseudorandom number
 * generators", OOPSLA 2014) as a counter-based generator: the value of
 * counter c under key k. */
static inline uint64_t sm64(uint64_t k, uint64_t c) {
    uint64_t z = k + (c + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static inline double u01(uint64_t k, uint64_t c) { return (double)(sm64(k, c) >> 11) * 0x1.0p-53; }

/* Particles per cell of the workload description: ppc background plus
 * floor(blob_peak * exp(-r^2/(2 sigma^2)) + u), r from the blob centre in
 * cells (cell centres).  Writes counts[nx*ny]; returns the total. */
int64_t orc_plasma_counts(int32_t nx, int32_t ny, int32_t ppc, double blob_peak, double cx,
                          double cy, double sigma, uint64_t seed, int64_t* counts) {
    int64_t total = 0;
#pragma omp parallel for schedule(static) reduction(+ : total)
    for (int64_t c = 0; c < (int64_t)nx * ny; ++c) {
        int64_t k = ppc;
        if (blob_peak > 0) {
            const double rx = (double)(c % nx) + 0.5 - cx, ry = (double)(c / nx) + 0.5 - cy;
            k += (int64_t)floor(blob_peak * exp(-(rx * rx + ry * ry) / (2 * sigma * sigma)) +
                                u01(seed ^ 0xB10Bull, (uint64_t)c));
        }
        counts[c] = k;
        total += k;
    }
    return total;
}

/* Fills the Points of the cells' counts (start = exclusive prefix of the
 * counts): positions uniform in the cell, velocities Maxwellian with sigma
 * v_th per component (Box-Muller), blob particles (index in cell >= ppc)
 * adding (drift_vx, drift_vy).  Point i goes to out[perm(i)], perm a
 * bijection of [0, n) (a 4-round Feistel network on the next power of two,
 * cycle-walked), so that the array order is random with respect to the
 * cells, as the reference's initParticlesRandomly leaves it. */
void orc_plasma_fill(int32_t nx, int32_t ny, double dx, double dy, int32_t ppc, double v_th,
                     double drift_vx, double drift_vy, uint64_t seed, const int64_t* counts,
                     const int64_t* start, int64_t n, orc_point* out) {
    int bits = 1;
    while ((1ll << bits) < n) ++bits;
    const int lo = bits / 2, hi = bits - lo;
    const uint64_t lmask = (1ull << lo) - 1, hmask = (1ull << hi) - 1;
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t c = 0; c < (int64_t)nx * ny; ++c) {
        const int gx = (int)(c % nx), gy = (int)(c / nx);
        for (int64_t j = 0; j < counts[c]; ++j) {
            const uint64_t i = (uint64_t)(start[c] + j);
            /* Feistel permutation of i within [0, 2^bits), walked until < n */
            uint64_t x = i;
            do {
                uint64_t L = x >> lo, R = x & lmask;
                for (int r = 0; r < 4; ++r) {
                    /* alternate halves of width hi and lo */
                    const uint64_t F = sm64(seed + (uint64_t)r, R);
                    const uint64_t nL = R, nR = (L ^ F) & ((r & 1) ? lmask : hmask);
                    L = nL;
                    R = nR;
                }
                x = ((L & hmask) << lo) | (R & lmask);
            } while (x >= (uint64_t)n);
            orc_point* p = &out[x];
            const uint64_t k = seed ^ 0x5EEDull;
            p->x = (gx + u01(k, 8 * i)) * dx;
            p->y = (gy + u01(k, 8 * i + 1)) * dy;
            p->z = 0.0;
            double g[4];
            for (int h = 0; h < 2; ++h) {
                const double u1 = 1.0 - u01(k, 8 * i + 2 + 2 * h), u2 = u01(k, 8 * i + 3 + 2 * h);
                const double rr = sqrt(-2.0 * log(u1));
                g[2 * h] = rr * cos(6.283185307179586 * u2);
                g[2 * h + 1] = rr * sin(6.283185307179586 * u2);
            }
            const int blob = j >= ppc;
            p->vx = v_th * g[0] + (blob ? drift_vx : 0.0);
            p->vy = v_th * g[1] + (blob ? drift_vy : 0.0);
            p->vz = v_th * g[2];
            p->pointer = 0;
            p->pad_ = 0;
        }
    }
}
