// picdat.h -- parsed M_PICDAT.DAT / geometry.conf (host only).
#pragma once

#include <string>
#include <vector>

#include "pic_capi.h"

namespace picb200 {

struct PicdatSpecies {
    int id;
    double sim, actual, charge, mass;
};

// Every field readPICDAT reads (SYCL-PIC-poissonsolver/src/particles.cpp:308-633).
struct PicdatFile {
    int timesteps = 0;
    double xmax = 0, ymax = 0;
    int nx = 0, ny = 0;
    double dt = 0;
    double b0_mT = 0, b_sigma = 0, b_mean = 0;
    double te = 0, ti = 0, tg = 0;
    double pressure = 0;
    int uniform_init = 1;
    double frac_left = 0, frac_right = 1, frac_top = 0, frac_bottom = 1;
    int reinjection = 0;
    int scale_factor = 1;
    int init_particle_flag = 1;
    double epsilon = 0;
    int periodic = 0;
    std::string gas;
    double attachment = 0;
    int collision = 0;
    int power_mode = 0;
    double heat_frequency = 0, power = 0;
    int print_interval = 1;
    int start_avg = 0, end_avg = 0;
    int num_species = 0;
    std::vector<PicdatSpecies> species;
};

int read_picdat(const char* path, PicdatFile& f);
int read_geometry(const char* path, int GX, int GY, int periodic, std::vector<pic_rect>& rects);
int config_from_files(const char* picdat_path, const char* geometry_path, pic_config* cfg,
                      PicdatFile* file_out);

}  // namespace picb200
