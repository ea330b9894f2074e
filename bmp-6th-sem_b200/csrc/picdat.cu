// picdat.cu -- readers for the reference's input files (host C++).
//
// M_PICDAT.DAT (readPICDAT, SYCL-PIC-poissonsolver/src/particles.cpp:308-633)
// is a sequence of blocks separated by dashed lines; each block holds header
// text and ends with its value line.  geometry.conf (readGeometry,
// src/particles.cpp:636-686) holds a rectangle count and then rows of
// "x1 z1 x2 z2 V" fractions.  The readers below walk the same blocks in the
// same order; they return PIC_ERR_CONFIG / PIC_ERR_IO where the reference
// exits.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <regex>
#include <sstream>
#include <string>
#include <vector>

#include "picdat.h"
#include "pic_internal.h"

namespace picb200 {

namespace {

bool is_separator(const std::string& s) {
    size_t n = 0;
    for (char ch : s) {
        if (ch == '-') ++n;
        else if (!isspace((unsigned char)ch)) return false;
    }
    return n >= 5;
}

std::string trim(const std::string& s) {
    size_t a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return "";
    size_t b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
}

bool starts_numeric(const std::string& s) {
    const std::string t = trim(s);
    if (t.empty()) return false;
    const char c0 = t[0];
    return (c0 >= '0' && c0 <= '9') || c0 == '.' || ((c0 == '-' || c0 == '+') && t.size() > 1);
}

int read_blocks(const char* path, std::vector<std::vector<std::string>>& blocks) {
    std::ifstream in(path);
    if (!in) return fail(PIC_ERR_IO, std::string("cannot open ") + path);
    blocks.assign(1, {});
    std::string line;
    while (std::getline(in, line)) {
        if (is_separator(line)) {
            blocks.push_back({});
            continue;
        }
        if (!trim(line).empty()) blocks.back().push_back(line);
    }
    return PIC_OK;
}

template <typename... T>
bool parse_line(const std::string& s, T&... out) {
    std::istringstream is(s);
    bool ok = true;
    ((ok = ok && static_cast<bool>(is >> out)), ...);
    return ok;
}

}  // namespace

int read_picdat(const char* path, PicdatFile& f) {
    std::vector<std::vector<std::string>> b;
    PIC_TRY(read_blocks(path, b));
    // drop empty blocks (leading/trailing separators)
    std::vector<std::vector<std::string>> blk;
    for (auto& x : b)
        if (!x.empty()) blk.push_back(x);
    // scalar blocks in file order (src/particles.cpp:341-563)
    const int kScalarBlocks = 20;
    if ((int)blk.size() < kScalarBlocks + 1)
        return fail(PIC_ERR_CONFIG, "M_PICDAT.DAT: too few blocks");
    auto val = [&](int i) { return blk[i].back(); };
    bool ok = true;
    ok &= parse_line(val(0), f.timesteps);
    ok &= parse_line(val(1), f.xmax, f.ymax, f.nx, f.ny);
    ok &= parse_line(val(2), f.dt);
    ok &= parse_line(val(3), f.b0_mT, f.b_sigma, f.b_mean);
    ok &= parse_line(val(4), f.te, f.ti, f.tg);
    ok &= parse_line(val(5), f.pressure);
    ok &= parse_line(val(6), f.uniform_init);
    ok &= parse_line(val(7), f.frac_left, f.frac_right, f.frac_top, f.frac_bottom);
    ok &= parse_line(val(8), f.reinjection);
    ok &= parse_line(val(9), f.scale_factor);
    ok &= parse_line(val(10), f.init_particle_flag);
    ok &= parse_line(val(11), f.epsilon);
    ok &= parse_line(val(12), f.periodic);
    f.gas = trim(val(13));
    ok &= parse_line(val(14), f.attachment);
    ok &= parse_line(val(15), f.collision);
    ok &= parse_line(val(16), f.power_mode, f.heat_frequency, f.power);
    ok &= parse_line(val(17), f.print_interval);
    ok &= parse_line(val(18), f.start_avg, f.end_avg);
    ok &= parse_line(val(19), f.num_species);
    if (!ok) return fail(PIC_ERR_CONFIG, "M_PICDAT.DAT: malformed value line");
    if (f.num_species < 1 || f.num_species > PIC_MAX_SPECIES)
        return fail(PIC_ERR_CONFIG, "M_PICDAT.DAT: number of species must be 1..4");
    // species table: the numeric rows of the next block (src/particles.cpp:590-608)
    f.species.clear();
    for (const std::string& row : blk[kScalarBlocks]) {
        if ((int)f.species.size() == f.num_species) break;
        if (!starts_numeric(row)) continue;
        // header lines such as "1-electron,2-positiveIon,..." do not parse
        // as five numbers and are skipped like readPICDAT's two header reads
        PicdatSpecies s{};
        if (!parse_line(row, s.id, s.sim, s.actual, s.charge, s.mass)) continue;
        f.species.push_back(s);
    }
    if ((int)f.species.size() != f.num_species)
        return fail(PIC_ERR_CONFIG, "M_PICDAT.DAT: species table shorter than the species count");
    if (f.nx < 4 || f.ny < 4 || !(f.xmax > 0) || !(f.ymax > 0))
        return fail(PIC_ERR_CONFIG, "M_PICDAT.DAT: bad grid line");
    return PIC_OK;
}

int read_geometry(const char* path, int GX, int GY, int periodic, std::vector<pic_rect>& rects) {
    std::vector<std::vector<std::string>> b;
    PIC_TRY(read_blocks(path, b));
    std::vector<std::vector<std::string>> blk;
    for (auto& x : b)
        if (!x.empty()) blk.push_back(x);
    if (blk.size() < 2) return fail(PIC_ERR_CONFIG, "geometry.conf: too few blocks");
    int count = 0;
    if (!parse_line(blk[0].back(), count) || count < 0 || count > PIC_MAX_RECTS)
        return fail(PIC_ERR_CONFIG, "geometry.conf: bad rectangle count");
    // readGeometry, src/particles.cpp:651-654: a periodic run has the two
    // x walls and at most one more electrode
    if (periodic && count > 3)
        return fail(PIC_ERR_CONFIG, "geometry.conf: a periodic boundary expects at most 3 rectangles");
    rects.clear();
    for (const std::string& row : blk[1]) {
        if ((int)rects.size() == count) break;
        if (!starts_numeric(row)) continue;
        double x1, y1, x2, y2, v;
        if (!parse_line(row, x1, y1, x2, y2, v))
            return fail(PIC_ERR_CONFIG, "geometry.conf: malformed rectangle row");
        // (int)((GRID-1)*fraction), src/particles.cpp:677-681
        pic_rect r;
        r.x1 = (int32_t)((double)(GX - 1) * x1);
        r.y1 = (int32_t)((double)(GY - 1) * y1);
        r.x2 = (int32_t)((double)(GX - 1) * x2);
        r.y2 = (int32_t)((double)(GY - 1) * y2);
        r.potential = v;
        rects.push_back(r);
    }
    if ((int)rects.size() != count)
        return fail(PIC_ERR_CONFIG, "geometry.conf: fewer rectangles than the count");
    return PIC_OK;
}

int config_from_files(const char* picdat_path, const char* geometry_path, pic_config* cfg,
                      PicdatFile* file_out) {
    PicdatFile f;
    PIC_TRY(read_picdat(picdat_path, f));
    std::vector<pic_rect> rects;
    PIC_TRY(read_geometry(geometry_path, f.nx + 1, f.ny + 1, f.periodic != 0, rects));
    pic_config_default(cfg);
    cfg->nx = f.nx;
    cfg->ny = f.ny;
    cfg->xmax = f.xmax;
    cfg->ymax = f.ymax;
    cfg->dt = f.dt;
    cfg->epsilon = f.epsilon;
    cfg->b0 = f.b0_mT / 1000.0;  // src/particles.cpp:389
    // surfArea, src/particles.cpp:431-432
    cfg->surf_area = f.uniform_init ? f.xmax * f.ymax
                                    : (f.frac_right - f.frac_left) * f.xmax *
                                          (f.frac_bottom - f.frac_top) * f.ymax;
    cfg->num_species = f.num_species;
    for (int s = 0; s < f.num_species; ++s) {
        cfg->species[s].charge = f.species[s].charge;
        cfg->species[s].mass = f.species[s].mass;
        cfg->species[s].sim_count = f.species[s].sim;
        cfg->species[s].actual_count = f.species[s].actual;
    }
    cfg->num_rects = (int32_t)rects.size();
    for (size_t r = 0; r < rects.size(); ++r) cfg->rects[r] = rects[r];
    cfg->timesteps = f.timesteps;
    cfg->print_interval = f.print_interval;
    cfg->periodic_y = f.periodic != 0 ? 1 : 0;
    if (file_out) *file_out = f;
    return PIC_OK;
}

}  // namespace picb200

extern "C" int pic_config_from_files(const char* picdat_path, const char* geometry_path,
                                     pic_config* cfg) {
    if (!picdat_path || !geometry_path || !cfg) return picb200::fail(PIC_ERR_ARG, "null argument");
    return picb200::config_from_files(picdat_path, geometry_path, cfg, nullptr);
}
