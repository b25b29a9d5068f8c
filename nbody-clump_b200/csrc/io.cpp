// io.cpp -- the reference's input files and binary snapshot files.
//
// Readers: world.par (LoadParameters, src/dem_subsphere_io.cu:40-149, exactly
// 38 keys, an unknown or missing key is an error), the ph and ch text files
// (src/dem_subsphere_io.cu:151-193, src/dem_clumpsphere_io.cu:24-62),
// Rocks/CubeWall.bt (src/dem_cube_wall_io.cu:21-53), Rocks/Penetrator.bt
// (src/dem_penetrator_io.cu:21-116) and Rocks/CylindWall.bt
// (src/dem_cylind_wall_io.cu:20-55); the sphere drivers' 21-column ph file
// and grid.bt (src/dem_io.cu:155-248).  Writers: the field-block .bin files
// of src/dem_binary_io.h:17-181 and src/dem_io.cu:313-329.  Errors are
// returned, never exit().
#include "io.h"

#include <sys/stat.h>
#include <sys/types.h>

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <sstream>

namespace nbc {

static bool file_exists(const std::string& p) {
    struct stat st;
    return ::stat(p.c_str(), &st) == 0;
}

static std::string lower(std::string s) {
    std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return (char)std::tolower(c); });
    return s;
}

bool make_dirs(const std::string& path) {
    std::string cur;
    for (size_t i = 0; i <= path.size(); i++) {
        if (i == path.size() || path[i] == '/') {
            if (!cur.empty() && !file_exists(cur) && ::mkdir(cur.c_str(), 0755) != 0 && errno != EEXIST)
                return false;
        }
        if (i < path.size()) cur.push_back(path[i]);
    }
    return true;
}

// LoadParameters (src/dem_subsphere_io.cu:40-149)
static bool load_par(const std::string& path, Workdir& w, std::string& err) {
    std::ifstream in(path);
    if (!in) { err = "cannot open " + path; return false; }
    static const char* keys[] = {
        "NumberBody", "BodyFileDir", "IniConFile", "BranchLmtLen", "StepSize", "EndStep", "StartStep",
        "OutputInterval", "Ymod", "Prat", "Frcoe", "NormRes", "Frvel", "Beta", "MU_T", "MU_R", "Cohesion",
        "ClumpNum", "Thresh", "GridLevels", "Gravity", "Update", "WorldSize_x", "WorldSize_y", "WorldSize_z",
        "WorldOrigin_x", "WorldOrigin_y", "WorldOrigin_z", "BoxLowLmt_x", "BoxLowLmt_y", "BoxLowLmt_z",
        "BoxUpLmt_x", "BoxUpLmt_y", "BoxUpLmt_z", "isIntruder", "isSelfGravity", "isWallForce", "isQuaternion"};
    const int nkeys = (int)(sizeof(keys) / sizeof(keys[0]));
    std::string line;
    int flag = 0;
    while (std::getline(in, line)) {
        std::string core = line.substr(0, line.find('#'));
        core.erase(std::remove(core.begin(), core.end(), '\t'), core.end());
        core.erase(std::remove(core.begin(), core.end(), ' '), core.end());
        core.erase(std::remove(core.begin(), core.end(), '\r'), core.end());
        if (core.empty()) continue;
        size_t eq = core.find('=');
        if (eq == std::string::npos || eq == 0 || eq + 1 >= core.size()) { err = "malformed line in world.par: " + line; return false; }
        std::string name = core.substr(0, eq), value = core.substr(eq + 1);
        bool known = false;
        for (int k = 0; k < nkeys; k++) known |= name == keys[k];
        if (!known) { err = "Unrecoganized item " + name + "!"; return false; }
        w.par[name] = value;
        flag++;
    }
    if (flag != nkeys) { err = "Important parameter setting missing! (" + std::to_string(flag) + " of 38)"; return false; }
    return true;
}

static double pd(const Workdir& w, const char* k) { return std::atof(w.par.at(k).c_str()); }

// the scalars of world.par both paths read
static bool par_scalars(Workdir& w, std::string& err) {
    nbc_scene_desc& D = w.desc;
    memset(&D, 0, sizeof(D));
    D.n_sub = (int)pd(w, "NumberBody");
    D.n_clump = (int)pd(w, "ClumpNum");
    D.branch_len = (int)pd(w, "BranchLmtLen");
    D.dt = pd(w, "StepSize");
    D.end_step = (int)pd(w, "EndStep");
    D.start_step = (int)pd(w, "StartStep");
    D.output_interval = (int)pd(w, "OutputInterval");
    D.ymod = pd(w, "Ymod"); D.prat = pd(w, "Prat"); D.frcoe = pd(w, "Frcoe"); D.normres = pd(w, "NormRes");
    D.beta = pd(w, "Beta"); D.cohesion = pd(w, "Cohesion"); D.gravity = pd(w, "Gravity"); D.thresh = pd(w, "Thresh");
    const char* ax = "xyz";
    for (int a = 0; a < 3; a++) {
        std::string s(1, ax[a]);
        D.world_origin[a] = pd(w, ("WorldOrigin_" + s).c_str());
        D.world_size[a] = pd(w, ("WorldSize_" + s).c_str());
        D.box_lo[a] = pd(w, ("BoxLowLmt_" + s).c_str());
        D.box_hi[a] = pd(w, ("BoxUpLmt_" + s).c_str());
    }
    D.is_wall_force = pd(w, "isWallForce") != 0;
    w.is_intruder = pd(w, "isIntruder") != 0;
    if (D.n_sub <= 0) { err = "NumberBody must be positive"; return false; }
    if (D.output_interval <= 0) { err = "OutputInterval must be positive"; return false; }
    D.levels = 1;
    return true;
}

// Rocks/CubeWall.bt (src/dem_cube_wall_io.cu:21-53)
static bool read_cube(const std::string& path, nbc_scene_desc& D, std::string& err) {
    std::ifstream f(path);
    if (!f) { err = "Error! Cannot open " + path + "!"; return false; }
    double v[16];
    for (int k = 0; k < 16; k++)
        if (!(f >> v[k])) { err = "Rocks/CubeWall.bt: malformed"; return false; }
    D.wall = NBC_WALL_CUBE;
    for (int a = 0; a < 3; a++) {
        D.cube_half[a] = v[a]; D.cube_centre[a] = v[3 + a]; D.cube_vel[a] = v[6 + a]; D.cube_angvel[a] = v[13 + a];
    }
    return true;
}

// Rocks/CylindWall.bt (src/dem_cylind_wall_io.cu:20-55)
static bool read_cyl(const std::string& path, nbc_scene_desc& D, std::string& err) {
    std::ifstream f(path);
    if (!f) { err = "Error! Cannot open " + path + "!"; return false; }
    double v[22];
    for (int k = 0; k < 22; k++)
        if (!(f >> v[k])) { err = "Rocks/CylindWall.bt: malformed"; return false; }
    D.wall = NBC_WALL_CYLINDER;
    D.cyl_radius = v[0]; D.cyl_half_height = v[1];
    for (int a = 0; a < 3; a++) {
        D.cyl_axis[a] = v[2 + a]; D.cyl_centre[a] = v[9 + a]; D.cyl_vel[a] = v[12 + a]; D.cyl_angvel[a] = v[19 + a];
    }
    return true;
}

// Rocks/Penetrator.bt (src/dem_penetrator_io.cu:21-116); `use` sets the
// scene's intruder, otherwise the file is only checked
static bool read_penetrator(const std::string& dir, Workdir& w, bool use, std::string& err) {
    nbc_scene_desc& D = w.desc;
    const std::string pp = dir + "/Rocks/Penetrator.bt";
    std::ifstream f(pp);
    if (!f) { err = "Error! Cannot open " + pp + "!"; return false; }
    nbc_scene_desc T;
    memset(&T, 0, sizeof(T));
    std::string tok;
    f >> tok;
    std::string lt = lower(tok);
    if (lt == "sphere") {
        T.intruder = NBC_INTR_SPHERE;
        f >> T.intr_radius;
        T.intr_half_height = T.intr_radius;
        T.intr_axis[2] = 1.0;
    } else if (lt == "cylinder") {
        T.intruder = NBC_INTR_CYLINDER;
        f >> T.intr_radius >> T.intr_half_height >> T.intr_axis[0] >> T.intr_axis[1] >> T.intr_axis[2];
    } else {
        char* end = nullptr;
        T.intr_radius = std::strtod(tok.c_str(), &end);
        if (end == tok.c_str() || *end != '\0') { err = "Error! Unknown penetrator shape '" + tok + "'"; return false; }
        T.intruder = NBC_INTR_CYLINDER;
        f >> T.intr_half_height >> T.intr_axis[0] >> T.intr_axis[1] >> T.intr_axis[2];
    }
    double q[4];
    f >> T.intr_prop[0] >> T.intr_prop[1] >> T.intr_prop[2] >> T.intr_prop[3];
    f >> T.intr_pos[0] >> T.intr_pos[1] >> T.intr_pos[2];
    f >> T.intr_vel[0] >> T.intr_vel[1] >> T.intr_vel[2];
    f >> q[0] >> q[1] >> q[2] >> q[3];
    f >> T.intr_angvel[0] >> T.intr_angvel[1] >> T.intr_angvel[2];
    if (!f || T.intr_radius <= 0.0 || T.intr_prop[3] <= 0.0) { err = "Error! Invalid penetrator data in " + pp; return false; }
    T.intr_motion = NBC_MOTION_CONSTANT_VELOCITY;
    std::string opt;
    if (f >> opt) {
        if (lower(opt) != "motion") { err = "Error! Unknown penetrator option '" + opt + "'"; return false; }
        std::string m;
        f >> m;
        m = lower(m);
        if (m == "constant_velocity" || m == "constant" || m == "kinematic") T.intr_motion = NBC_MOTION_CONSTANT_VELOCITY;
        else if (m == "gravity" || m == "dynamic") T.intr_motion = NBC_MOTION_GRAVITY;
        else if (m == "gravity_after_contact") T.intr_motion = NBC_MOTION_GRAVITY_AFTER_CONTACT;
        else { err = "Error! Unknown penetrator motion mode '" + m + "'"; return false; }
    }
    if (!use) return true;
    D.intruder = T.intruder;
    D.intr_motion = T.intr_motion;
    D.intr_radius = T.intr_radius;
    D.intr_half_height = T.intr_half_height;
    for (int a = 0; a < 3; a++) {
        D.intr_axis[a] = T.intr_axis[a]; D.intr_pos[a] = T.intr_pos[a]; D.intr_vel[a] = T.intr_vel[a];
        D.intr_angvel[a] = T.intr_angvel[a];
    }
    for (int c = 0; c < 4; c++) { D.intr_prop[c] = T.intr_prop[c]; w.intr_quat[c] = q[c]; }
    return true;
}

static void point_desc(Workdir& w) {
    nbc_scene_desc& D = w.desc;
    D.clump_id = w.cid.data(); D.pos = w.pos.data(); D.local = w.local.data(); D.mass = w.mass.data();
    D.radius = w.radius.data();
    D.clump_pos = w.cpos.data(); D.clump_vel = w.cvel.data(); D.clump_quat = w.cquat.data();
    D.clump_angvel = w.cw.data(); D.clump_prop = w.cprop.data();
    D.level = w.level.empty() ? nullptr : w.level.data();
    D.level_cell = w.lcell.empty() ? nullptr : w.lcell.data();
    D.body_kind = w.kind.empty() ? nullptr : w.kind.data();
}

bool load_workdir(const std::string& dir, Workdir& w, std::string& err) {
    w.dir = dir;
    w.driver = -1;
    if (!load_par(dir + "/world.par", w, err)) return false;
    if (!par_scalars(w, err)) return false;
    nbc_scene_desc& D = w.desc;
    if (D.n_clump <= 0) { err = "NumberBody and ClumpNum must be positive"; return false; }

    // ph (src/dem_subsphere_io.cu:151-193)
    std::string ini = w.par["IniConFile"];
    std::ifstream ph(dir + "/" + ini);
    if (!ph) { err = "Error! Cannot open " + ini + "!"; return false; }
    w.cid.resize(D.n_sub);
    w.pos.resize(3 * (size_t)D.n_sub);
    w.local.resize(3 * (size_t)D.n_sub);
    w.mass.resize(D.n_sub);
    w.radius.resize(D.n_sub);
    for (int i = 0; i < D.n_sub; i++) {
        double t0, t1;
        ph >> t0 >> t1 >> w.cid[i] >> w.pos[3 * i] >> w.pos[3 * i + 1] >> w.pos[3 * i + 2] >> w.local[3 * i] >>
            w.local[3 * i + 1] >> w.local[3 * i + 2] >> w.mass[i] >> w.radius[i];
        if (!ph) { err = ini + ": short or malformed at row " + std::to_string(i); return false; }
    }
    // ch (src/dem_clumpsphere_io.cu:24-62)
    std::ifstream ch(dir + "/ch.00000000.bt");
    if (!ch) { err = "Error! Cannot open ch.00000000.bt!"; return false; }
    const size_t K = D.n_clump;
    w.cpos.resize(3 * K); w.cvel.resize(3 * K); w.cquat.resize(4 * K); w.cw.resize(3 * K); w.cprop.resize(4 * K);
    for (size_t k = 0; k < K; k++) {
        double t;
        ch >> t >> w.cpos[3 * k] >> w.cpos[3 * k + 1] >> w.cpos[3 * k + 2] >> w.cvel[3 * k] >> w.cvel[3 * k + 1] >>
            w.cvel[3 * k + 2] >> w.cquat[4 * k] >> w.cquat[4 * k + 1] >> w.cquat[4 * k + 2] >> w.cquat[4 * k + 3] >>
            w.cw[3 * k] >> w.cw[3 * k + 1] >> w.cw[3 * k + 2] >> w.cprop[4 * k] >> w.cprop[4 * k + 1] >>
            w.cprop[4 * k + 2] >> w.cprop[4 * k + 3];
        if (!ch) { err = "ch.00000000.bt: short or malformed at row " + std::to_string(k); return false; }
    }
    point_desc(w);
    for (int i = 0; i < D.n_sub; i++)
        if (w.cid[i] < 0 || w.cid[i] >= D.n_clump) { err = "clump id out of range in " + ini; return false; }

    // walls: the cube of the clump path (src/dem_cube_wall_io.cu:21-53); a
    // closed cylinder when only Rocks/CylindWall.bt is present
    const std::string cube = dir + "/Rocks/CubeWall.bt", cyl = dir + "/Rocks/CylindWall.bt";
    if (file_exists(cube)) {
        if (!read_cube(cube, D, err)) return false;
    } else if (file_exists(cyl)) {
        if (!read_cyl(cyl, D, err)) return false;
    } else if (D.is_wall_force) {
        err = "isWallForce set but neither Rocks/CubeWall.bt nor Rocks/CylindWall.bt exists";
        return false;
    }
    // intruder (src/dem_penetrator_io.cu:21-116)
    D.intruder = NBC_INTR_NONE;
    if (w.is_intruder && !read_penetrator(dir, w, true, err)) return false;
    return true;
}

// The sphere-only drivers' working directory (class DEMmain): world.par with
// the same 38 keys, the 21-column ph file named by IniConFile
// (DEMSphereIo::LoadPhase, src/dem_io.cu:155-202: id, id, Type, Pos, Vel,
// Quat, AngSpd, Property = Ixx Iyy Izz M, Radius), the driver's wall file (read
// whatever isWallForce says: the drivers apply the wall unconditionally,
// src/dem_simulation_cylind.cu:157), Rocks/Penetrator.bt (always read,
// src/dem_simulation_cylind.cu:54-60) and, for the hgrid driver, grid.bt
// (DEMSphereIo::LoadGridLevels, src/dem_io.cu:204-248: per level "id
// cellSize nx ny nz offset id", GridLevels rows; Type is the sphere's level,
// 0 the coarsest).  Sphere k becomes clump k with one member at its centre.
bool load_sphere_workdir(const std::string& dir, int driver, Workdir& w, std::string& err) {
    w.dir = dir;
    w.driver = driver;
    if (driver < NBC_DRIVER_CYLINDER || driver > NBC_DRIVER_HGRID) { err = "unknown DEMmain driver"; return false; }
    if (!load_par(dir + "/world.par", w, err)) return false;
    if (!par_scalars(w, err)) return false;
    nbc_scene_desc& D = w.desc;
    const int n = D.n_sub;
    D.n_clump = n;
    std::string ini = w.par["IniConFile"];
    std::ifstream ph(dir + "/" + ini);
    if (!ph) { err = "Error! Cannot open " + ini + "!"; return false; }
    w.cid.resize(n); w.type.resize(n);
    w.pos.resize(3 * (size_t)n); w.local.assign(3 * (size_t)n, 0.0);
    w.mass.resize(n); w.radius.resize(n);
    w.cpos.resize(3 * (size_t)n); w.cvel.resize(3 * (size_t)n); w.cquat.resize(4 * (size_t)n);
    w.cw.resize(3 * (size_t)n); w.cprop.resize(4 * (size_t)n);
    for (int i = 0; i < n; i++) {
        double t0, t1;
        double* p = &w.cpos[3 * (size_t)i];
        double* v = &w.cvel[3 * (size_t)i];
        double* q = &w.cquat[4 * (size_t)i];
        double* a = &w.cw[3 * (size_t)i];
        double* pr = &w.cprop[4 * (size_t)i];
        ph >> t0 >> t1 >> w.type[i] >> p[0] >> p[1] >> p[2] >> v[0] >> v[1] >> v[2] >> q[0] >> q[1] >> q[2] >> q[3] >>
            a[0] >> a[1] >> a[2] >> pr[0] >> pr[1] >> pr[2] >> pr[3] >> w.radius[i];
        if (!ph) { err = ini + ": short or malformed at row " + std::to_string(i); return false; }
        w.cid[i] = i;
        for (int c = 0; c < 3; c++) w.pos[3 * (size_t)i + c] = p[c];
        w.mass[i] = pr[3];
    }
    D.is_wall_force = 1;
    D.sphere_mode = NBC_SPHERE_KINEMATICS;
    if (driver == NBC_DRIVER_CUBE) {
        if (!read_cube(dir + "/Rocks/CubeWall.bt", D, err)) return false;
        D.sphere_mode |= NBC_SPHERE_CUBE_WALL;
    } else {
        if (!read_cyl(dir + "/Rocks/CylindWall.bt", D, err)) return false;
        if (driver != NBC_DRIVER_HGRID) D.sphere_mode |= NBC_SPHERE_RESET_HISTORY;
    }
    if (driver == NBC_DRIVER_SPLIT) {
        for (int i = 0; i < n; i++)
            if (w.type[i] < 0 || w.type[i] > 2) { err = ini + ": Type must be 0, 1 or 2 at row " + std::to_string(i); return false; }
        w.kind = w.type;
    }
    if (driver == NBC_DRIVER_HGRID) {
        const int L = (int)pd(w, "GridLevels");
        if (L < 1 || L > 6) { err = "GridLevels must be 1 .. 6"; return false; }
        std::ifstream g(dir + "/grid.bt");
        if (!g) { err = "Error! Cannot open grid.bt!"; return false; }
        std::vector<double> cell(L);
        for (int l = 0; l < L; l++) {
            int id, nx, ny, nz, off, id2;
            g >> id >> cell[l] >> nx >> ny >> nz >> off >> id2;
            if (!g || !(cell[l] > 0)) { err = "grid.bt: short or malformed at level " + std::to_string(l); return false; }
        }
        for (int i = 0; i < n; i++)
            if (w.type[i] < 0 || w.type[i] >= L) { err = ini + ": Type is not a grid level at row " + std::to_string(i); return false; }
        if (L > 1) {
            D.levels = L;
            w.level = w.type;
            w.lcell = cell;
        }
    }
    D.intruder = NBC_INTR_NONE;
    if (!read_penetrator(dir, w, w.is_intruder, err)) return false;
    point_desc(w);
    return true;
}


// ---------------------------------------------------------------------------
// writers (src/dem_binary_io.h)
// ---------------------------------------------------------------------------
std::string bin_name(const std::string& dir, const char* prefix, int step) {
    std::ostringstream s;
    s << dir << '/' << prefix << '.' << std::setw(8) << std::setfill('0') << step << ".bin";
    return s.str();
}

struct BinWriter {
    FILE* f;
    bool ok;
    explicit BinWriter(const std::string& p) : f(std::fopen(p.c_str(), "wb")), ok(f != nullptr) {}
    ~BinWriter() { if (f) std::fclose(f); }
    void raw(const void* p, size_t b) { if (ok && b) ok = std::fwrite(p, 1, b, f) == b; }
    void i32(int v) { raw(&v, 4); }
};

bool write_ph(const std::string& path, int n, const int* sorted_id, const int* part_fix, const int* clump_id,
              const double* pos, const double* local, const double* mass, const double* radius) {
    BinWriter w(path);
    w.i32(n);
    w.raw(sorted_id, 4 * (size_t)n);
    w.raw(part_fix, 4 * (size_t)n);
    w.raw(clump_id, 4 * (size_t)n);
    w.raw(pos, 24 * (size_t)n);
    w.raw(local, 24 * (size_t)n);
    w.raw(mass, 8 * (size_t)n);
    w.raw(radius, 8 * (size_t)n);
    return w.ok;
}

// SaveParticles_Bin of the sphere drivers (src/dem_io.cu:313-329)
bool write_sphere_ph(const std::string& path, int n, const int* sorted_id, const int* part_fix, const int* type,
                     const double* pos, const double* vel, const double* quat, const double* angvel,
                     const double* prop, const double* radius) {
    BinWriter w(path);
    w.i32(n);
    w.raw(sorted_id, 4 * (size_t)n);
    w.raw(part_fix, 4 * (size_t)n);
    w.raw(type, 4 * (size_t)n);
    w.raw(pos, 24 * (size_t)n);
    w.raw(vel, 24 * (size_t)n);
    w.raw(quat, 32 * (size_t)n);
    w.raw(angvel, 24 * (size_t)n);
    w.raw(prop, 32 * (size_t)n);
    w.raw(radius, 8 * (size_t)n);
    return w.ok;
}

bool write_ch(const std::string& path, int k, const double* pos, const double* vel, const double* quat,
              const double* w, const double* prop, const double* ipos, const double* ivel, const double* iquat,
              const double* iw) {
    BinWriter f(path);
    const bool intr = ipos != nullptr;
    const int c = k + (intr ? 1 : 0);
    f.i32(c);
    if (intr) f.i32(-1);
    for (int i = 0; i < k; i++) f.i32(i);
    if (intr) f.raw(ipos, 24);
    f.raw(pos, 24 * (size_t)k);
    if (intr) f.raw(ivel, 24);
    f.raw(vel, 24 * (size_t)k);
    if (intr) f.raw(iquat, 32);
    f.raw(quat, 32 * (size_t)k);
    if (intr) f.raw(iw, 24);
    f.raw(w, 24 * (size_t)k);
    if (intr) { double z[4] = {0, 0, 0, 0}; f.raw(z, 32); }
    f.raw(prop, 32 * (size_t)k);
    return f.ok;
}

// SaveForceHistory (src/dem_binary_io.h:123-144): every 100th step of the interval
bool write_fc(const std::string& path, int interval, const double* hist6) {
    const int skip = 100;
    const int count = interval / skip + (interval % skip != 0 ? 1 : 0);
    BinWriter f(path);
    f.i32(count);
    for (int i = 0; i < count; i++) f.i32(i * skip);
    for (int i = 0; i < count; i++) f.raw(hist6 + 6 * (size_t)(i * skip), 24);
    for (int i = 0; i < count; i++) f.raw(hist6 + 6 * (size_t)(i * skip) + 3, 24);
    return f.ok;
}

// the intruder contact file of SaveParticles_Bin (src/dem_subsphere_io.cu:279-303)
bool write_yi(const std::string& path, int n, const int* clump_id, const double* diag) {
    std::vector<int> idx;
    const double* fn = diag;
    for (int j = 0; j < n; j++)
        if (fn[3 * j] * fn[3 * j] + fn[3 * j + 1] * fn[3 * j + 1] + fn[3 * j + 2] * fn[3 * j + 2] > 1e-28)
            idx.push_back(j);
    BinWriter f(path);
    f.i32((int)idx.size());
    for (int j : idx) f.i32(clump_id[j]);
    for (int c = 0; c < 4; c++)
        for (int j : idx) f.raw(diag + ((size_t)c * n + j) * 3, 24);
    return f.ok;
}

// SaveContacts (src/dem_binary_io.h:100-121)
bool write_cnt(const std::string& dir, int step, int n, int bl, const int* nei, const double* fcn, const double* cpt) {
    const size_t cnt = (size_t)n * bl;
    {
        BinWriter f(bin_name(dir, "Nei", step));
        f.i32(n); f.i32(bl); f.raw(nei, 4 * cnt);
        if (!f.ok) return false;
    }
    {
        BinWriter f(bin_name(dir, "Fcn", step));
        f.i32(n); f.i32(bl); f.raw(fcn, 24 * cnt);
        if (!f.ok) return false;
    }
    BinWriter f(bin_name(dir, "Cpt", step));
    f.i32(n); f.i32(bl); f.raw(cpt, 24 * cnt);
    return f.ok;
}

}  // namespace nbc
