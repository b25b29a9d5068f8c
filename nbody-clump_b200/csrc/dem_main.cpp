// dem_main.cpp -- DEMmain on the C ABI (see dem_main.h).
#include "dem_main.h"

#include <cstdio>
#include <cstdlib>

DEMmain::DEMmain() {}
DEMmain::~DEMmain() {}

void DEMmain::run(int driver) {
    nbc_options opt;
    nbc_default_options(&opt);
    opt.precision = NBC_PREC_F64;  // the reference computes everything in FP64
    if (const char* p = std::getenv("NBC_PRECISION")) opt.precision = p[0] == 'm' ? NBC_PREC_MIXED : NBC_PREC_F64;
    nbc_engine* e = nullptr;
    status_ = nbc_open_sphere(".", driver, &opt, &e);
    if (status_ == NBC_OK) status_ = nbc_run(e);
    if (status_ != NBC_OK) std::fprintf(stderr, "DEMmain: %s (status %d)\n", nbc_last_error(), status_);
    nbc_destroy(e);
}

void DEMmain::RunSimulation() { run(NBC_DRIVER_CYLINDER); }
void DEMmain::RunSimulation2() { run(NBC_DRIVER_CUBE); }
void DEMmain::RunSimulation_Split() { run(NBC_DRIVER_SPLIT); }
void DEMmain::RunSimulation_HGrid() { run(NBC_DRIVER_HGRID); }
