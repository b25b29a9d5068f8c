// dem_clump_main.cpp -- DEMClumpMain on the C ABI (see dem_clump_main.h).
#include "dem_clump_main.h"

#include <cstdio>
#include <cstdlib>

DEMClumpMain::DEMClumpMain() {}
DEMClumpMain::~DEMClumpMain() {}

void DEMClumpMain::RunSimulationClump() {
    nbc_options opt;
    nbc_default_options(&opt);
    opt.precision = NBC_PREC_F64;  // the reference computes everything in FP64
    if (const char* p = std::getenv("NBC_PRECISION")) opt.precision = p[0] == 'm' ? NBC_PREC_MIXED : NBC_PREC_F64;
    nbc_engine* e = nullptr;
    status_ = nbc_open(".", &opt, &e);
    if (status_ == NBC_OK) status_ = nbc_run(e);
    if (status_ != NBC_OK) std::fprintf(stderr, "DEMClumpMain: %s (status %d)\n", nbc_last_error(), status_);
    nbc_destroy(e);
}
