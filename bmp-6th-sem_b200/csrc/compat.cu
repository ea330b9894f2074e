// compat.cu -- the reference's sycl_pic_* C ABI on one process-global context
// (SYCL-PIC-poissonsolver/src/sycl_pic_ctypes.cpp:46-272).  Synchronous; each
// operator returns elapsed wall seconds like the reference.  Host copies of
// rho and phi stand in for the reference's malloc_shared arrays and are
// refreshed after every operator that changes them.
#include <sys/stat.h>

#include <cerrno>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "picdat.h"
#include "pic_internal.h"
#include "sycl_pic_compat.h"

namespace picb200 {
namespace {

struct Global {
    pic_ctx* ctx = nullptr;
    PicdatFile file;
    std::vector<double> rho, phi;
    int status = PIC_OK;  // of the last void operator (diagnostics writers)
};
Global g;

double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// initParticlesRandomly (src/particles.cpp:127-173): uniform positions over the
// domain (or the init box when the uniform flag is 0) and an isotropic
// Maxwellian with v = sqrt(2|q/m|T): vx = v*sqrt(-ln u1)*cos(2 pi u2).  The
// reference seeds std::rand with time(); this uses a fixed-seed mt19937_64
// (PIC_SEED overrides it) so runs repeat.
int init_species_points(pic_ctx* c, int s, const PicdatFile& f) {
    const int64_t n = (int64_t)f.species[s].sim;
    uint64_t seed = 0x5EED0000ull + (uint64_t)s;
    if (const char* e = std::getenv("PIC_SEED")) seed = std::strtoull(e, nullptr, 10) + s;
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> U(0.0, 1.0);
    auto ran2 = [&]() {
        double r = U(rng);
        return r < 1e-10 ? 1e-10 : r;  // utils.cpp:51-56
    };
    const double W = f.xmax, H = f.ymax;
    const double ctom = f.species[s].charge / f.species[s].mass;
    double T = 0;
    if (s == 0) T = f.te;
    if (s == 1) T = f.ti;
    const double v = std::sqrt(2 * std::fabs(ctom) * T);
    std::vector<pic_point> pts((size_t)n);
    for (int64_t i = 0; i < n; ++i) {
        pic_point& p = pts[(size_t)i];
        if (f.uniform_init) {
            p.x = W * U(rng);
            p.y = H * U(rng);
        } else {
            p.x = f.frac_left * W + (f.frac_right - f.frac_left) * W * U(rng);
            p.y = f.frac_top * H + (f.frac_bottom - f.frac_top) * H * U(rng);
        }
        p.z = 0;
        double z1 = std::sqrt(-std::log(ran2())), z2 = 6.283185307 * ran2();
        p.vx = v * z1 * std::cos(z2);
        p.vy = v * z1 * std::sin(z2);
        z1 = std::sqrt(-std::log(ran2()));
        z2 = 6.283185307 * ran2();
        p.vz = v * z1 * std::cos(z2);
        p.pointer = 0;
        p.pad_ = 0;
    }
    return pic_import_points(c, s, pts.data(), n);
}

int refresh_host(bool rho, bool phi) {
    if (rho) PIC_TRY(pic_get_rho(g.ctx, g.rho.data()));
    if (phi) PIC_TRY(pic_get_phi(g.ctx, g.phi.data()));
    return PIC_OK;
}

bool ready() {
    if (!g.ctx) {
        set_error("sycl_pic_init has not been called");
        return false;
    }
    return true;
}

// One grid as the reference's print* functions write it: GY lines of GX
// "%lf" values, space separated.  Every write and the close are checked (a
// full disk shows up at fclose at the latest).
int write_grid(const std::string& path, int GX, int GY, const std::vector<double>& v,
               double scale) {
    FILE* fd = std::fopen(path.c_str(), "w");
    if (!fd) return fail(PIC_ERR_IO, "cannot create " + path + ": " + std::strerror(errno));
    bool ok = true;
    for (int i = 0; i < GY && ok; ++i) {
        for (int j = 0; j < GX - 1 && ok; ++j)
            ok = std::fprintf(fd, "%lf ", v[(size_t)i * GX + j] * scale) > 0;
        ok = ok && std::fprintf(fd, "%lf\n", v[(size_t)i * GX + GX - 1] * scale) > 0;
    }
    const int err = ok ? 0 : errno;
    if (std::fclose(fd) != 0 && ok) return fail(PIC_ERR_IO, "cannot write " + path + ": " + std::strerror(errno));
    if (!ok) return fail(PIC_ERR_IO, "cannot write " + path + ": " + std::strerror(err));
    return PIC_OK;
}

// mkdir that accepts an existing folder.
int ensure_dir(const std::string& d) {
    if (mkdir(d.c_str(), 0755) == 0 || errno == EEXIST) {
        struct stat st;
        if (stat(d.c_str(), &st) == 0 && S_ISDIR(st.st_mode)) return PIC_OK;
    }
    return fail(PIC_ERR_IO, "cannot create folder " + d + ": " + std::strerror(errno));
}

}  // namespace
}  // namespace picb200

using namespace picb200;

extern "C" {

int sycl_pic_init(const char* dev_type, int wg, int ps, const char* input1, const char* input2) {
    (void)wg; (void)ps; (void)input1; (void)input2;
    const std::string dt = dev_type ? dev_type : "";
    if (dt != "gpu" && dt != "cpu") {
        set_error("sycl_pic_init: device must be 'cpu' or 'gpu'");
        return -1;
    }
    if (g.ctx) sycl_pic_finalize();
    pic_config cfg;
    if (config_from_files("M_PICDAT.DAT", "geometry.conf", &cfg, &g.file) != PIC_OK) return -1;
    if (pic_create(&cfg, &g.ctx) != PIC_OK) return -1;
    for (int s = 0; s < cfg.num_species; ++s)
        if (init_species_points(g.ctx, s, g.file) != PIC_OK) return -1;
    g.rho.assign((size_t)g.ctx->nodes, 0.0);
    g.phi.assign((size_t)g.ctx->nodes, 0.0);
    if (refresh_host(true, true) != PIC_OK) return -1;
    return 0;
}

int sycl_pic_get_grid_size(void) { return g.ctx ? (int)g.ctx->nodes : -1; }
int sycl_pic_get_grid_x(void) { return g.ctx ? g.ctx->GX : -1; }
int sycl_pic_get_grid_y(void) { return g.ctx ? g.ctx->GY : -1; }
int sycl_pic_get_timesteps(void) { return g.ctx ? g.file.timesteps : -1; }
int sycl_pic_get_print_interval(void) { return g.ctx ? g.file.print_interval : -1; }
int sycl_pic_get_num_species(void) { return g.ctx ? g.ctx->cfg.num_species : -1; }

int sycl_pic_get_particle_count(int species) {
    if (!ready()) return -1;
    int64_t n = 0;
    if (pic_particle_count(g.ctx, species, &n) != PIC_OK) return -1;
    return (int)n;
}

double* sycl_pic_get_rho_ptr(void) { return g.ctx ? g.rho.data() : nullptr; }
double* sycl_pic_get_phi_ptr(void) { return g.ctx ? g.phi.data() : nullptr; }

void sycl_pic_zero_rho(void) {
    if (!ready()) return;
    pic_zero_rho(g.ctx);
    std::fill(g.rho.begin(), g.rho.end(), 0.0);
}

double sycl_pic_charge_deposition(int species) {
    if (!ready()) return -1.0;
    const double t0 = now();
    if (pic_charge_deposition(g.ctx, species) != PIC_OK || refresh_host(true, false) != PIC_OK)
        return -1.0;
    return now() - t0;
}

double sycl_pic_poisson_solve(int iteration) {
    if (!ready()) return -1.0;
    const double t0 = now();
    if (pic_poisson_solve(g.ctx, iteration) != PIC_OK || refresh_host(true, true) != PIC_OK)
        return -1.0;
    return now() - t0;
}

double sycl_pic_move_particles(int species, int iteration) {
    if (!ready()) return -1.0;
    const double t0 = now();
    if (pic_move_particles(g.ctx, species, iteration) != PIC_OK || pic_synchronize(g.ctx) != PIC_OK)
        return -1.0;
    return now() - t0;
}

double sycl_pic_compact_particles(int species, double* out_alloc_t, double* out_scan_t) {
    if (!ready()) return -1.0;
    if (out_alloc_t) *out_alloc_t = 0.0;
    if (out_scan_t) *out_scan_t = 0.0;
    return pic_compact_particles(g.ctx, species) == PIC_OK ? 0.0 : -1.0;
}

double sycl_pic_cleanup_map(int species) {
    if (!ready()) return -1.0;
    return pic_cleanup_map(g.ctx, species) == PIC_OK ? 0.0 : -1.0;
}

double sycl_pic_generate_new_particles(void) {
    if (!ready()) return -1.0;
    const double t0 = now();
    pic_source_desc d;
    pic_source_default(&d);
    d.te_ev = g.file.te;  // electronTemp / ionTemp from M_PICDAT.DAT
    d.ti_ev = g.file.ti;
    if (const char* e = std::getenv("PIC_SEED")) d.seed = std::strtoull(e, nullptr, 10) ^ 0x5A1CE5ull;
    int64_t ne = 0, np = 0;
    if (pic_generate_new_particles(g.ctx, &d, &ne, &np) != PIC_OK) return -1.0;
    return now() - t0;
}

void sycl_pic_update_fields_from_phi(void) {
    if (!ready()) return;
    if (pic_set_phi(g.ctx, g.phi.data()) != PIC_OK) return;
    if (pic_update_fields_from_phi(g.ctx) != PIC_OK) return;
    refresh_host(false, true);  // the electrode potentials, as overwritePhi leaves them
}

// printNumberDensity / printEnergy / printElectricField / printPhi
// (src/utils.cpp:829-1025): one text grid per quantity under
// dir/<quantity>/<iteration>, "%lf" values, space separated.  The reference
// prints a message and exits when a file cannot be created; this returns
// PIC_ERR_IO (or the status of the failing read-back) instead.
int pic_write_diagnostics(pic_ctx* c, const char* dir, int iteration, double scale_factor) {
    if (!c || !dir) return fail(PIC_ERR_ARG, "pic_write_diagnostics: null argument");
    const int GX = c->GX, GY = c->GY;
    const size_t n = (size_t)c->nodes;
    const std::string it = std::to_string(iteration);
    const std::string d = dir;
    std::vector<double> f0(n, 0.0), f1(n, 0.0), e0(n, 0.0), e1(n, 0.0), ex(n), ey(n), phi(n);
    PIC_TRY(pic_get_final_mesh(c, 0, f0.data()));
    PIC_TRY(pic_get_energy_mesh(c, 0, e0.data()));
    if (c->cfg.num_species > 1) {
        PIC_TRY(pic_get_final_mesh(c, 1, f1.data()));
        PIC_TRY(pic_get_energy_mesh(c, 1, e1.data()));
    }
    std::vector<pic_field> ef(n);
    PIC_TRY(pic_get_efield(c, ef.data()));
    for (size_t i = 0; i < n; ++i) {
        ex[i] = ef[i].fx;
        ey[i] = ef[i].fy;
    }
    PIC_TRY(pic_get_phi(c, phi.data()));
    PIC_TRY(ensure_dir(d));  // the output folder itself (an existing one is kept)
    auto put = [&](const char* q, const std::vector<double>& v, double scale) {
        const std::string p = d + "/" + q;
        PIC_TRY(ensure_dir(p));
        return write_grid(p + "/" + it, GX, GY, v, scale);
    };
    PIC_TRY(put("electronDensity", f0, scale_factor));
    PIC_TRY(put("ionDensity", f1, scale_factor));
    // temperature-like energy: 0.66667*E/(n+1); the reference's last electron
    // column divides by (energy+1) (src/utils.cpp printEnergy), kept as is
    std::vector<double> te(n), ti(n);
    for (int i = 0; i < GY; ++i)
        for (int j = 0; j < GX; ++j) {
            const size_t k = (size_t)i * GX + j;
            const double den0 = (j == GX - 1) ? e0[k] + 1.0 : f0[k] + 1.0;
            te[k] = 0.66667 * e0[k] / den0;
            ti[k] = 0.66667 * e1[k] / (f1[k] + 1.0);
        }
    PIC_TRY(put("electronenergy", te, 1.0));
    PIC_TRY(put("ionenergy", ti, 1.0));
    PIC_TRY(put("Ex", ex, 1.0));
    PIC_TRY(put("Ey", ey, 1.0));
    PIC_TRY(put("potential", phi, 1.0));
    return PIC_OK;
}

// The reference's signature returns nothing; a failure leaves its reason in
// pic_last_error() and in sycl_pic_last_status().
void sycl_pic_print_diagnostics(const char* dir, int iteration) {
    if (!ready() || !dir) {
        g.status = PIC_ERR_STATE;
        return;
    }
    g.status = pic_write_diagnostics(g.ctx, dir, iteration, g.file.scale_factor);
}

// Mesh_<s>.out: the final_mesh of each species (src/main.cpp:260-274).
void sycl_pic_save_meshes(void) {
    if (!ready()) {
        g.status = PIC_ERR_STATE;
        return;
    }
    pic_ctx* c = g.ctx;
    std::vector<double> f((size_t)c->nodes);
    g.status = PIC_OK;
    for (int s = 0; s < c->cfg.num_species && g.status == PIC_OK; ++s) {
        g.status = pic_get_final_mesh(c, s, f.data());
        if (g.status != PIC_OK) break;
        const std::string path = "Mesh_" + std::to_string(s) + ".out";
        FILE* fd = std::fopen(path.c_str(), "w");
        if (!fd) {
            g.status = fail(PIC_ERR_IO, "cannot create " + path + ": " + std::strerror(errno));
            break;
        }
        bool ok = true;
        for (int y = 0; y < c->GY && ok; ++y) {
            for (int x = 0; x < c->GX && ok; ++x) ok = std::fprintf(fd, "%g ", f[(size_t)y * c->GX + x]) > 0;
            ok = ok && std::fprintf(fd, "\n") > 0;
        }
        if (std::fclose(fd) != 0 || !ok)
            g.status = fail(PIC_ERR_IO, "cannot write " + path + ": " + std::strerror(errno));
    }
}

int sycl_pic_last_status(void) { return g.status; }

void sycl_pic_finalize(void) {
    if (g.ctx) pic_destroy(g.ctx);
    g.ctx = nullptr;
    g.rho.clear();
    g.phi.clear();
}

}  // extern "C"
