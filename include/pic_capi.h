/*
 * pic_capi.h -- C ABI of the B200-native 2D electrostatic PIC step.
 *
 * Drop-in for the operator surface of SYCL-PIC-poissonsolver
 * (vansh268p/BMP-6th-sem), SYCL-PIC-poissonsolver/src/sycl_pic_ctypes.cpp:46-272:
 * cell binning, CIC charge deposition, field gather + Boris push and the
 * Poisson solve on the geometry.conf electrode mesh.  Plain C types only:
 * pointers, sizes, status codes.  All device memory is owned by the library.
 *
 * Two surfaces:
 *   1. pic_* -- context-handle API.  One pic_ctx per simulation instance;
 *      operators enqueue work on the context's CUDA stream and return a
 *      status code (0 ok, negative = PIC_ERR_*).  pic_last_error() gives the
 *      message of the most recent failure on the calling thread.
 *   2. sycl_pic_* -- the reference's own names and signatures, backed by one
 *      process-global context, synchronous, returning elapsed wall seconds
 *      exactly as the reference does.  They return -1.0 (or -1 / NULL) where
 *      the reference would have called exit(); the reason is in
 *      pic_last_error().
 *
 * Array layouts at the boundary are the reference's:
 *   - particles: pic_point AoS, 56 B (include/point.hpp:11-14);
 *   - grids: row-major [GRID_Y][GRID_X] double, GRID_X = NX+1, GRID_Y = NY+1
 *     (src/particles.cpp:357-368, 728-734);
 *   - electric field: interleaved pic_field {fx, fy} per node
 *     (include/point.hpp:16-19).
 * Inside the library particles are cell-sorted SoA (int cell implied by the
 * sort, FP32 in-cell offsets, FP32 velocities); see pic_import_points.
 */
#ifndef PIC_CAPI_H
#define PIC_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PIC_CAPI_VERSION 1
#define PIC_MAX_SPECIES 4
#define PIC_MAX_RECTS 32

/* ---- status codes ------------------------------------------------------ */
#define PIC_OK 0
#define PIC_ERR_ARG (-1)           /* bad argument (null pointer, bad species, size) */
#define PIC_ERR_CONFIG (-2)        /* invalid configuration or input file          */
#define PIC_ERR_CAPACITY (-3)      /* particle buffer or fixed-point range exceeded */
#define PIC_ERR_NOT_CONVERGED (-4) /* Poisson solve hit its iteration limit         */
#define PIC_ERR_CUDA (-5)          /* CUDA runtime error                            */
#define PIC_ERR_STATE (-6)         /* operator called in the wrong state            */
#define PIC_ERR_IO (-7)            /* file could not be read or written             */
#define PIC_ERR_NO_DEVICE (-8)     /* no usable sm_100 device                       */
#define PIC_ERR_TIMEOUT (-9)       /* a bounded device wait gave up                 */

/* ---- boundary record types (reference layouts) ------------------------- */

/* Point, SYCL-PIC-poissonsolver/include/point.hpp:11-14.  z is not tracked
 * by the library (no reference computation reads it); export writes z=0.
 * pointer: -1 marks a dead particle on import; export writes the particle's
 * position in the cell-sorted order. */
typedef struct pic_point {
    double x, y, z, vx, vy, vz;
    int32_t pointer;
    int32_t pad_;
} pic_point;

/* Field, include/point.hpp:16-19. */
typedef struct pic_field {
    double fx, fy;
} pic_field;

/* Geometry, include/point.hpp:21-24: inclusive node-index rectangle held at
 * `potential` volts (readGeometry converts geometry.conf fractions with
 * (int)((GRID-1)*fraction), src/particles.cpp:677-681). */
typedef struct pic_rect {
    int32_t x1, y1, x2, y2;
    double potential;
} pic_rect;

/* One row of M_PICDAT.DAT's species table (src/particles.cpp:590-608). */
typedef struct pic_species_desc {
    double charge;       /* C, with sign                            */
    double mass;         /* kg                                      */
    double sim_count;    /* "SimulationParticles" (weight formula)  */
    double actual_count; /* "ActualParticles"                       */
} pic_species_desc;

#define PIC_SOLVER_MG_PCG 0     /* geometric-multigrid-preconditioned CG */
#define PIC_SOLVER_JACOBI_PCG 1 /* plain path: diagonal-preconditioned CG */

#define PIC_WARM_ZERO 0     /* start every solve from phi = 0             */
#define PIC_WARM_PREVIOUS 1 /* start from the previous step's phi          */
#define PIC_WARM_LEARNED 2  /* start from the conv network's prediction    */

typedef struct pic_config {
    int32_t nx, ny;       /* cells; nodes are (nx+1) x (ny+1)             */
    double xmax, ymax;    /* domain size (m); dx = xmax/nx, dy = ymax/ny  */
    double dt;            /* s                                            */
    double epsilon;       /* F/m                                          */
    double b0;            /* uniform Bz (T) (initMagneticField)           */
    double surf_area;     /* m^2 for the weight formula; 0 -> xmax*ymax   */
    int32_t num_species;
    pic_species_desc species[PIC_MAX_SPECIES];
    int32_t num_rects;    /* electrode rectangles, applied in order       */
    pic_rect rects[PIC_MAX_RECTS];
    int32_t poisson_solver;   /* PIC_SOLVER_*                              */
    int32_t warm_start;       /* PIC_WARM_*                                */
    double poisson_tol;       /* relative residual target, default 1e-8   */
    int32_t poisson_maxit;    /* default 500                               */
    int32_t deposit_energy;   /* 1: also build the energy mesh (default)   */
    int32_t device;           /* CUDA device ordinal                       */
    int32_t timesteps;        /* informational (M_PICDAT TIMESTEPS)        */
    int32_t print_interval;   /* informational (M_PICDAT printInterval)    */
    /* 1: periodic in y (M_PICDAT periodicBoundary; src/poissonSolver.cpp:
     * 82-180, 411-430, src/mover.cpp:317-320).  The potential is solved on
     * node rows 0..ny-1, row ny is a copy of row 0 (then the electrodes),
     * E_y wraps, E_x is one-sided at the x walls, and the push wraps y into
     * [0, ymax).  The node columns x = 0 and x = nx must be electrodes on
     * rows 0..ny-1.  Multigrid needs ny even (a Jacobi-preconditioned solve
     * is used otherwise); the learned warm start is not available. */
    int32_t periodic_y;
} pic_config;

/* Uniform Maxwellian plasma plus an optional Gaussian blob, generated on the
 * device with Philox-4x32-10 (counter = particle id, key = seed).  Cell c gets
 * ppc background particles and floor(blob_peak_ppc*exp(-r^2/(2 sigma^2)) + u)
 * blob particles (u uniform per cell), r measured in cells from the blob
 * centre.  Velocities: per-component sigma = sqrt(e*T/m); blob particles add
 * (drift_vx, drift_vy). */
typedef struct pic_plasma_desc {
    int32_t ppc;              /* background particles per cell             */
    double temperature_ev;
    double blob_peak_ppc;     /* 0 -> no blob                              */
    double blob_cx, blob_cy;  /* blob centre in cell units                 */
    double blob_sigma;        /* cells                                     */
    double drift_vx, drift_vy;/* m/s, blob particles only                  */
    uint64_t seed;
} pic_plasma_desc;

typedef struct pic_ctx pic_ctx;

/* ---- lifetime ---------------------------------------------------------- */
const char* pic_last_error(void);
const char* pic_status_string(int status);
int pic_config_default(pic_config* cfg);
/* Reads M_PICDAT.DAT + geometry.conf (readPICDAT src/particles.cpp:308-633,
 * readGeometry :636-686) into a config.  Species counts come from the file. */
int pic_config_from_files(const char* picdat_path, const char* geometry_path, pic_config* cfg);
int pic_create(const pic_config* cfg, pic_ctx** out);
void pic_destroy(pic_ctx* ctx);
/* Run the context on a caller-owned cudaStream_t (NULL -> library stream). */
int pic_set_stream(pic_ctx* ctx, void* cuda_stream);
void* pic_get_stream(pic_ctx* ctx);
int pic_synchronize(pic_ctx* ctx);

/* ---- particles --------------------------------------------------------- */
int pic_reserve(pic_ctx* ctx, int species, int64_t capacity);
/* Replace a species' particles with n host Points (reference AoS).  The cell
 * is (int)(x*(1/dx)), (int)(y*(1/dy)) as in InsertKernel
 * (src/particles.cpp:230-235); the FP32 offset is the FP64 remainder.
 * Dead (pointer == -1) or out-of-domain points are dropped.  A cell holds at
 * most 43,680 particles (its slots, n + n/2 + 16, stay within 2^16):
 * PIC_ERR_CAPACITY beyond that. */
int pic_import_points(pic_ctx* ctx, int species, const pic_point* host, int64_t n);
int pic_export_points(pic_ctx* ctx, int species, pic_point* host, int64_t capacity,
                      int64_t* n_out);
/* The internal cell-sorted state, unconverted: cell index (gy*nx + gx),
 * FP32 offsets and velocities, in storage order.  Each output array holds
 * `capacity` entries; *n_out receives the particle count (all pointers NULL:
 * size query).  No reference counterpart: it exposes the library's own
 * layout for exact checks. */
int pic_export_state(pic_ctx* ctx, int species, int32_t* cell, float* fx, float* fy, float* vx,
                     float* vy, float* vz, int64_t capacity, int64_t* n_out);
int pic_load_plasma(pic_ctx* ctx, int species, const pic_plasma_desc* desc);
int pic_particle_count(pic_ctx* ctx, int species, int64_t* n_out);
/* Live particles per bucket, indexed like the reference's key_idx
 * (gy*GRID_X + gx, GRID_X*GRID_Y entries). */
int pic_bin_counts(pic_ctx* ctx, int species, int32_t* host_counts);
/* Particles that left through x < 0 since the last call (new_additions,
 * src/mover.cpp:344-351); the counter is reset by the read. */
int pic_left_exits(pic_ctx* ctx, int species, int64_t* n_out);

/* Particle sources of the reference's generate_new_particles
 * (src/sycl_pic_ctypes.cpp:212-236): generate_new_electrons re-injects, as
 * electrons (species 0), the electrons lost through x < 0 beyond the ions
 * (species 1) lost there since the last call, at x = reinject_x with y
 * uniform (src/utils.cpp:374-489); generate_pairs creates ceil(fn) electron-
 * ion pairs, fn = YMAX dt (2/pi) (x22 - x11) ionimax / rate_div, each at
 * x = xm + asin(2u-1)(x22-x11)/pi, y uniform, kept inside (0, XMAX)
 * (src/utils.cpp:495-566).  Velocities are the reference's Maxwellian draw
 * v sqrt(-ln u) (cos, sin)(2 pi u'), v = sqrt(2|q/m|T).  The reference's
 * constants are the defaults (pic_source_default); draws are Philox with
 * the call number and particle index as counter (the reference uses rand()). */
typedef struct pic_source_desc {
    double reinject_x;    /* m (reference: 0.024)                         */
    double te_ev, ti_ev;  /* temperatures of new electrons / ions (eV)    */
    double x11, x22, xm;  /* ionisation band (m): 0.0025, 0.01, 0.00625   */
    double ionimax;       /* 5.23e23                                      */
    double rate_div;      /* 1.67e6                                       */
    int32_t reinject;     /* 1: re-inject electrons                       */
    int32_t pairs;        /* 1: create ionisation pairs                   */
    uint64_t seed;
} pic_source_desc;
int pic_source_default(pic_source_desc* d);
/* New particles join the state at once (placed in their cells by the next
 * push); n_electrons / n_pairs receive what was created. */
int pic_generate_new_particles(pic_ctx* ctx, const pic_source_desc* d, int64_t* n_electrons,
                               int64_t* n_pairs);

/* ---- step operators (reference order, src/main.cpp:130-257) ------------ */
int pic_zero_rho(pic_ctx* ctx);
int pic_charge_deposition(pic_ctx* ctx, int species);
int pic_poisson_solve(pic_ctx* ctx, int iteration);
int pic_move_particles(pic_ctx* ctx, int species, int iteration);
int pic_compact_particles(pic_ctx* ctx, int species); /* no-op: the sort compacts */
int pic_cleanup_map(pic_ctx* ctx, int species);       /* no-op: no hashmap       */
/* zero_rho, deposit every species, Poisson, E, push every species. */
int pic_step(pic_ctx* ctx, int iteration);
/* bin + deposit + push for every species, with the E field held fixed. */
int pic_particle_phase(pic_ctx* ctx, int iteration);

/* ---- grids (host copies in the reference layout) ------------------------ */
int pic_get_rho(pic_ctx* ctx, double* host);
int pic_get_phi(pic_ctx* ctx, double* host);
int pic_get_efield(pic_ctx* ctx, pic_field* host);
int pic_get_final_mesh(pic_ctx* ctx, int species, double* host);
int pic_get_energy_mesh(pic_ctx* ctx, int species, double* host);
int pic_set_rho(pic_ctx* ctx, const double* host);
int pic_set_phi(pic_ctx* ctx, const double* host);
/* The reference Python extension's update_fields_from_phi
 * (src/sycl_pic_module.cpp:216-223): electrode nodes of phi take their
 * potential (overwritePhi, src/poissonSolver.cpp:364-382), then E from phi
 * (calculateElectricField, src/poissonSolver.cpp:433-456). */
int pic_update_fields_from_phi(pic_ctx* ctx);
int pic_set_bz(pic_ctx* ctx, const double* host);
/* The reference's text snapshots (printNumberDensity, printEnergy,
 * printElectricField, printPhi: src/utils.cpp:829-991): one file per
 * quantity, dir/<quantity>/<iteration>, GRID_Y lines of GRID_X "%lf" values
 * separated by single spaces, for electronDensity and ionDensity (final_mesh
 * times scale_factor), electronenergy and ionenergy (0.66667 energy/(n+1)),
 * Ex, Ey and potential.  Folders are created as needed.  PIC_ERR_IO when a
 * folder or file cannot be created or written (the reference exits). */
int pic_write_diagnostics(pic_ctx* ctx, const char* dir, int iteration, double scale_factor);

/* ---- instrumentation (no reference counterpart; the reference returns
 * host wall seconds per operator, src/sycl_pic_ctypes.cpp:127-236) ------- */
#define PIC_PHASE_PUSH 0         /* the push pass: gather, Boris, binning, fused deposit */
#define PIC_PHASE_FIXUP 1        /* side list: movers whose target cell was full      */
#define PIC_PHASE_RELAYOUT 2     /* slot-layout rebuilds (rare)                        */
#define PIC_PHASE_DEPOSIT 3      /* stand-alone deposit of current positions          */
#define PIC_PHASE_FLUSH 4        /* accumulators -> final/energy mesh, rho             */
#define PIC_PHASE_POISSON 5      /* whole Poisson solve incl. E field                  */
#define PIC_NUM_PHASES 6
/* When on, CUDA events bracket every phase on the context stream. */
int pic_set_profiling(pic_ctx* ctx, int on);
/* Synchronises, returns accumulated device milliseconds and calls per phase. */
int pic_profile_read(pic_ctx* ctx, double* ms, int64_t* calls, int reset);
/* Kernel launches issued by this context since creation. */
int pic_launch_count(pic_ctx* ctx, int64_t* n);
/* Test hook (no reference counterpart).  The library's only device-side
 * waits are bounded: the batched ensemble solve's block barriers give up
 * after a number of polls (default 2^26), the learned warm start's
 * tensor-core pipeline waits after a number of SM clock cycles (default
 * 2^31, about a second); either then records a flag and lets its kernel
 * finish, and the operator returns PIC_ERR_TIMEOUT.  This lowers the two
 * bounds on the context's device so that a test can make the waits run out
 * without any fault; values <= 0 restore the defaults.  Device-wide: it
 * affects every context on that device. */
int pic_debug_set_wait_limits(pic_ctx* ctx, int64_t barrier_polls, int64_t tensor_wait_cycles);
/* Test hook (no reference counterpart).  Applies one multigrid V-cycle (the
 * PCG's preconditioner) to rhs, one FP32 value per node in the context's
 * node order, and writes the result to out (host buffers).  per_sweep = 0
 * runs the solver's own V-cycle (a level's sweeps in one kernel, on tiles in
 * shared memory), 1 the same V-cycle with one kernel per half sweep; the
 * two give the same bits.  PIC_ERR_CONFIG when the grid has no multigrid
 * hierarchy.  Overwrites the solver's multigrid work arrays: not during a
 * solve in flight on another stream. */
int pic_debug_vcycle(pic_ctx* ctx, const float* rhs, float* out, int per_sweep);

/* ---- tuning (no reference counterpart) -----------------------------------
 * The particle kernels are built for PIC_NUM_TILE_SHAPES tile shapes of 256
 * cells: 0 = 64x4 (default), 1 = 256x1, 2 = 128x2, 3 = 16x16. */
#define PIC_NUM_TILE_SHAPES 4
int pic_set_tile_shape(pic_ctx* ctx, int tile_shape);
/* Times the push of the current particles with every tile shape (the
 * simulation state is left as it was; the accumulators are redeposited at the
 * next charge_deposition) and keeps the fastest.  When the environment
 * variable PIC_TUNE_CACHE names a file and ms_per_shape is NULL, a choice
 * recorded there for the same device, grid and particle count is used
 * without timing; new choices are appended to it.  ms_per_shape, when not
 * NULL, receives PIC_NUM_TILE_SHAPES timings (ms per push of all species). */
int pic_autotune(pic_ctx* ctx, int* tile_shape, double* ms_per_shape);

/* ---- allocation-free deposit ---------------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory when they deposit -- a host framework that owns a fixed device
 * memory budget and only hands out buffers it has already sized, or a
 * time-critical loop where cudaMalloc/cudaFree (which may synchronise the
 * device) are not allowed.  Deposits n reference Points (device memory,
 * 56-byte records; pointer == -1 and out-of-domain points are skipped) of
 * one species on an nx x ny cell grid: dev_final_mesh[(nx+1)*(ny+1)] is
 * overwritten with the species' final_mesh and, when dev_rho is not NULL,
 * final_mesh * (-charge/epsilon) is added to dev_rho.  Same arithmetic as
 * pic_import_points + pic_charge_deposition (bit-identical final_mesh); no
 * energy mesh.  Enqueued on cuda_stream (NULL: the default stream); calls no
 * cudaMalloc, cudaFree or allocating library routine.
 *   - Scratch: one file-scope device array of 2^19 64-bit accumulators
 *     (4 MiB; grids up to 524,288 nodes, larger ones are rejected with
 *     PIC_ERR_CAPACITY), held by every GPU that loads the library until the
 *     process exits, cleared at the start of every call.
 *   - The first call on a device looks up the array's device address
 *     (cudaGetSymbolAddress) with that device current; make that first call
 *     before any stream capture.  The address is kept per device and CUDA
 *     context: after a cudaDeviceReset the next call sees a new context and
 *     looks the address up again (so, after a reset too, make one call
 *     before capturing).
 *   - All calls share the one array: calls that overlap on the GPU (other
 *     streams, other host threads) race and must be serialised by the caller. */
int pic_deposit_points_noalloc(const pic_point* dev_points, int64_t n, int32_t nx, int32_t ny,
                               double xmax, double ymax, const pic_species_desc* species,
                               double surf_area, double epsilon, double* dev_final_mesh,
                               double* dev_rho, void* cuda_stream);

/* ---- learned warm start ------------------------------------------------
 * Replaces the reference's ML surrogate slot (src/poisson_ml_bridge.py:55-106)
 * with a PCG initial guess: a 3-level conv encoder-decoder (32 channels, 3x3,
 * BF16 tensor-core kernels with FP32 accumulation) predicting phi_n from
 * phi_{n-1}, the change of the right-hand side and the electrode mask.  PCG
 * then runs to the same tolerance, so the answer never depends on it. */
/* max_pairs > 0: (re)start recording (input, target) pairs at each Poisson
 * solve into a new dataset that keeps the newest max_pairs; the scales
 * normalise phi (V), the RHS change times dx^2 (V) and the target
 * phi_n - phi_{n-1} (V).  All three 0: each is set to its root-mean-square
 * over the non-electrode nodes of the first recorded pair (read back with
 * pic_ws_scales).  max_pairs == 0: stop recording, keep the dataset (training
 * can continue).  max_pairs < 0: stop and release the dataset. */
int pic_ws_record(pic_ctx* ctx, int64_t max_pairs, double phi_scale, double db_scale,
                  double target_scale);
/* The three scales in use: phi, RHS change times dx^2, target. */
int pic_ws_scales(pic_ctx* ctx, double* scales3);
int pic_ws_pairs(pic_ctx* ctx, int64_t* n);
/* Adam epochs over the recorded pairs (one pair per step); *loss = mean
 * normalised squared error of the last epoch. */
int pic_ws_train(pic_ctx* ctx, int epochs, double lr, double* loss);
/* The same with the step size decaying over the call's steps from lr_max to
 * lr_min along a half cosine.  Each epoch visits the pairs in a new seeded
 * order (both entry points). */
int pic_ws_train_cosine(pic_ctx* ctx, int epochs, double lr_max, double lr_min, double* loss);
int64_t pic_ws_num_params(void);
int pic_ws_get_params(pic_ctx* ctx, float* host, int64_t n);
int pic_ws_set_params(pic_ctx* ctx, const float* host, int64_t n, double phi_scale,
                      double db_scale, double target_scale);
/* Side length P of the network's padded square grid. */
int pic_ws_grid(pic_ctx* ctx, int* P);
/* Training loss: the starting residual of PCG from the network's guess, in
 * scaled units, r = rhs - kappa L(out) on non-electrode nodes, where
 * rhs = (b_n - b_{n-1}) dx^2 / s1, kappa = s2/s1, and
 * L(u) = (2 + 2 dx^2/dy^2) u - (u_w + u_e) - (dx^2/dy^2)(u_s + u_n) with
 * u = 0 on electrodes; loss = sum r^2 / (GX*GY).
 * One forward + backward pass on a given scaled input image x0[P*P*3]
 * (channels phi, RHS change, mask) and rhs[GX*GY]: returns the output image
 * out[P*P], the parameter gradient grad[pic_ws_num_params()] and the loss.
 * For gradient checks. */
int pic_ws_debug_step(pic_ctx* ctx, const float* x0, const float* rhs, float* out,
                      float* grad, double* loss);

/* ---- ensembles (no reference counterpart: the reference runs one
 * simulation per process) ------------------------------------------------
 * N independent instances on one device, advanced together: one step of all
 * of them is one launch per phase -- the charge-deposit conversion of every
 * species, ONE persistent cooperative launch for all the Poisson solves
 * (MG-PCG to each instance's tolerance, then its E field), and per species
 * one push launch and one side-list launch over all instances -- captured
 * in a CUDA graph after the first step.  Instances may differ in grid size,
 * electrodes, Bz, species weights and tolerances; they must share the
 * device, the number of species and the energy-mesh mode, use the MG-PCG
 * solver and no learned warm start.  Each instance is an ordinary context
 * (pic_ensemble_instance) for loading particles and reading results; its
 * step operators must not be called while it belongs to the ensemble. */
typedef struct pic_ensemble pic_ensemble;
int pic_ensemble_create(const pic_config* cfgs, int n, pic_ensemble** out);
void pic_ensemble_destroy(pic_ensemble* ens);
int pic_ensemble_size(pic_ensemble* ens);
pic_ctx* pic_ensemble_instance(pic_ensemble* ens, int i);
/* zero rho, deposit, Poisson + E, push: all instances.  Synchronises once. */
int pic_ensemble_step(pic_ensemble* ens, int iteration);
/* Times the batched push with every tile shape (state left as it was) and
 * keeps the fastest; ms_per_shape may be NULL. */
int pic_ensemble_autotune(pic_ensemble* ens, int* tile_shape, double* ms_per_shape);
/* 0: launch the phases directly instead of replaying the captured graph. */
int pic_ensemble_use_graph(pic_ensemble* ens, int on);
/* Device milliseconds of the last step: deposit conversion, Poisson + E,
 * push (all instances). */
int pic_ensemble_timing(pic_ensemble* ens, double* deposit_ms, double* poisson_ms, double* push_ms);
/* Whether the last step replayed a captured graph, the tile shape in use, and
 * the blocks of the persistent Poisson launch. */
int pic_ensemble_info(pic_ensemble* ens, int* graph_active, int* tile_shape, int* solver_blocks);

/* ---- Poisson controls -------------------------------------------------- */
int pic_set_poisson(pic_ctx* ctx, int solver, int warm_start, double tol, int maxit);
/* (no reference counterpart) enable = 0: run the PCG iterations as direct
 * launches with one host synchronisation per iteration instead of one CUDA
 * graph per solve (same kernels, same results; slower).  For profilers that
 * do not follow the kernels of a graph's conditional node.  Default 1. */
int pic_set_poisson_graph(pic_ctx* ctx, int enable);
/* Iterations, achieved relative residual and device milliseconds of the most
 * recent solve. */
int pic_poisson_stats(pic_ctx* ctx, int* iterations, double* relres, double* ms);
/* (no reference counterpart) Relative residual ||b - A x0|| / ||b|| of the
 * starting guess x0 of the most recent single-context solve (the previous
 * phi, zero, or the learned guess), on the reduced system. */
int pic_poisson_start_relres(pic_ctx* ctx, double* relres0);

#ifdef __cplusplus
}
#endif

#endif /* PIC_CAPI_H */
