// Harness entry point for the reference's sphere-only drivers (parity
// checker only, never linked into the product).  The reference's own main()
// (src/main.cpp:4-16) runs the clump path and has the sphere drivers'
// calls commented out (src/main.cpp:10-11).  This main runs one of them in
// the working directory, chosen by the argument: cylinder (the default,
// DEMmain::RunSimulation, src/dem_simulation_cylind.cu:3-211), cube
// (RunSimulation2), split (RunSimulation_Split) or hgrid
// (RunSimulation_HGrid).  Their inputs are world.par, the 21-column sphere
// ph file named by IniConFile, the driver's Rocks/ wall file,
// Rocks/Penetrator.bt and, for hgrid, grid.bt.
#include <cstdio>
#include <cstring>

#include "dem.h"

int main(int argc, char** argv) {
    const char* which = argc > 1 ? argv[1] : "cylinder";
    DEMmain dem;
    if (!std::strcmp(which, "cylinder")) dem.RunSimulation();
    else if (!std::strcmp(which, "cube")) dem.RunSimulation2();
    else if (!std::strcmp(which, "split")) dem.RunSimulation_Split();
    else if (!std::strcmp(which, "hgrid")) dem.RunSimulation_HGrid();
    else {
        std::fprintf(stderr, "unknown driver %s\n", which);
        return 2;
    }
    return 0;
}
