// io.h -- readers of the reference's input files and writers of its binary
// snapshot files (implementation and citations in io.cpp).
#pragma once
#include <map>
#include <string>
#include <vector>

#include "../../include/nbc.h"

namespace nbc {

// A working directory of the reference: world.par, the ph/ch .bt files and
// Rocks/.  Owns the arrays `desc` points to.
struct Workdir {
    std::string dir;
    int driver = -1;   // NBC_DRIVER_* for a sphere-driver directory, -1 for the clump path
    std::map<std::string, std::string> par;
    nbc_scene_desc desc;
    bool is_intruder = false;
    double intr_quat[4] = {0, 0, 0, 1};
    std::vector<int> cid, type, level, kind;
    std::vector<double> pos, local, mass, radius, cpos, cvel, cquat, cw, cprop, lcell;
};

bool load_workdir(const std::string& dir, Workdir& w, std::string& err);
bool load_sphere_workdir(const std::string& dir, int driver, Workdir& w, std::string& err);
bool make_dirs(const std::string& path);
std::string bin_name(const std::string& dir, const char* prefix, int step);
bool write_ph(const std::string& path, int n, const int* sorted_id, const int* part_fix, const int* clump_id,
              const double* pos, const double* local, const double* mass, const double* radius);
bool write_ch(const std::string& path, int k, const double* pos, const double* vel, const double* quat,
              const double* w, const double* prop, const double* ipos, const double* ivel, const double* iquat,
              const double* iw);
bool write_sphere_ph(const std::string& path, int n, const int* sorted_id, const int* part_fix, const int* type,
                     const double* pos, const double* vel, const double* quat, const double* angvel,
                     const double* prop, const double* radius);
bool write_fc(const std::string& path, int interval, const double* hist6);
bool write_yi(const std::string& path, int n, const int* clump_id, const double* diag);
bool write_cnt(const std::string& dir, int step, int n, int bl, const int* nei, const double* fcn, const double* cpt);

}  // namespace nbc
