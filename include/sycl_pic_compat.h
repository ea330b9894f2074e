/*
 * sycl_pic_compat.h -- the reference's own C ABI names, served by the
 * B200 library on one process-global context.
 *
 * Each function replaces the same-named extern "C" function of
 * SYCL-PIC-poissonsolver/src/sycl_pic_ctypes.cpp (line cited per entry) with
 * the same signature and argument meaning.  Like the reference they are
 * synchronous and return elapsed wall seconds.  Where the reference calls
 * exit() these return -1.0 (doubles), -1 (ints) or NULL (pointers) and leave
 * the reason in pic_last_error() (declared in pic_capi.h).
 *
 * rho and phi pointers are host memory owned by the library, refreshed after
 * every operator that changes them (the reference's malloc_shared arrays are
 * host-visible in the same way).  Writes through the phi pointer reach the
 * device through sycl_pic_update_fields_from_phi(), as in the reference's
 * Python extension.
 */
#ifndef SYCL_PIC_COMPAT_H
#define SYCL_PIC_COMPAT_H

#ifdef __cplusplus
extern "C" {
#endif

/* :49  reads ./M_PICDAT.DAT and ./geometry.conf.  dev_type "gpu" (or "cpu",
 * accepted and served by the GPU: this library has no CPU path).  wg and ps
 * (work-group and probe size of the hashmap) are accepted and ignored: the
 * counting sort has no per-cell capacity.  input1/input2 are ignored as in
 * the reference (readPICDAT initialises particles randomly). */
int sycl_pic_init(const char* dev_type, int wg, int ps, const char* input1, const char* input2);
int sycl_pic_get_grid_size(void);        /* :91  GRID_X*GRID_Y            */
/* sycl_pic_module.cpp:110-118 (Python extension): GRID_X, GRID_Y. */
int sycl_pic_get_grid_x(void);
int sycl_pic_get_grid_y(void);
int sycl_pic_get_timesteps(void);        /* :95  TIMESTEPS                */
int sycl_pic_get_print_interval(void);   /* :99  printInterval            */
int sycl_pic_get_num_species(void);      /* :103 num_type                 */
int sycl_pic_get_particle_count(int species); /* :107 live particles       */
double* sycl_pic_get_rho_ptr(void);      /* :112 host rho, GRID_X*GRID_Y  */
double* sycl_pic_get_phi_ptr(void);      /* :116 host phi, GRID_X*GRID_Y  */
void sycl_pic_zero_rho(void);            /* :121                          */
double sycl_pic_charge_deposition(int species);          /* :127 */
double sycl_pic_poisson_solve(int iteration);            /* :153 */
double sycl_pic_move_particles(int species, int iteration); /* :161 */
double sycl_pic_compact_particles(int species, double* out_alloc_t, double* out_scan_t); /* :179 */
double sycl_pic_cleanup_map(int species);                /* :201 */
/* :212 particle sources: re-injection of left-wall electron exits beyond the
 * ions' and ionisation pairs (pic_generate_new_particles with the reference's
 * constants, temperatures from M_PICDAT.DAT). */
double sycl_pic_generate_new_particles(void);
/* :239 text snapshots into dir/{electronDensity,ionDensity,electronenergy,
 * ionenergy,potential,Ex,Ey}/<iter> (printNumberDensity, printEnergy,
 * printElectricField, printPhi: src/utils.cpp:829-991).  Where the reference
 * exits on a file it cannot create, this returns with the reason in
 * pic_last_error() and the status in sycl_pic_last_status(). */
void sycl_pic_print_diagnostics(const char* dir, int iteration);
void sycl_pic_save_meshes(void);         /* :247 Mesh_<s>.out              */
/* No reference counterpart: PIC_OK or the PIC_ERR_* status of the last
 * sycl_pic_print_diagnostics / sycl_pic_save_meshes call (the reference's
 * signatures return nothing). */
int sycl_pic_last_status(void);
void sycl_pic_finalize(void);            /* :267                          */
/* sycl_pic_module.cpp:216-223 (Python extension): E from host phi. */
void sycl_pic_update_fields_from_phi(void);

#ifdef __cplusplus
}
#endif

#endif /* SYCL_PIC_COMPAT_H */
