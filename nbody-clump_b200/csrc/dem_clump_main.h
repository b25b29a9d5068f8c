// dem_clump_main.h -- drop-in replacement for the reference's driver class.
//
// The reference's entry point is `DEMClumpMain dem; dem.RunSimulationClump();`
// (src/dem_clump.h:36-96, src/main.cpp:4-16): no arguments, inputs read from
// the working directory, outputs written into it, exit() on any error.  This
// class keeps that call shape on top of the C ABI (include/nbc.h); errors are
// reported on stderr and through LastStatus() instead of exit().
#pragma once
#include "../../include/nbc.h"

class DEMClumpMain {
   public:
    DEMClumpMain();
    ~DEMClumpMain();
    // world.par, IniConFile, ch.00000000.bt and Rocks/ from the current
    // directory; OutPart/OutClump/OutForce/OutCnt written into it
    void RunSimulationClump();
    nbc_status LastStatus() const { return status_; }

   private:
    nbc_status status_ = NBC_OK;
};
