// dem_main.h -- drop-in replacement for the reference's sphere-only driver
// class DEMmain (src/dem.h:31-99).
//
// Its four drivers read their inputs from the working directory and write
// their outputs into it: RunSimulation (closed cylinder wall,
// src/dem_simulation_cylind.cu:3-211), RunSimulation2 (cube wall,
// src/dem_simulation_cube.cu:3-226), RunSimulation_Split (cylinder wall with
// free, driven and fixed spheres, src/dem_simulation_split.cu:3-211) and
// RunSimulation_HGrid (cylinder wall on the level table of grid.bt,
// src/dem_simulation_hgrid.cu:3-201).  The reference's main() has the calls
// commented out (src/main.cpp:10-11); with this class they link against the
// B200 engine unchanged.  Errors go to stderr and LastStatus() instead of
// exit().
#pragma once
#include "../../include/nbc.h"

class DEMmain {
   public:
    DEMmain();
    ~DEMmain();
    void RunSimulation();
    void RunSimulation2();
    void RunSimulation_Split();
    void RunSimulation_HGrid();
    nbc_status LastStatus() const { return status_; }

   private:
    void run(int driver);
    nbc_status status_ = NBC_OK;
};
