// Harness entry point for the reference's sphere-only driver (parity checker
// only, never linked into the product).  The reference's own main()
// (src/main.cpp:4-16) runs the clump path, whose walls are a cube only; its
// closed cylinder wall exists on the sphere path, DEMmain::RunSimulation
// (src/dem_simulation_cylind.cu:3-211).  This main runs that driver in the
// working directory (world.par, the 21-column sphere ph file named by
// IniConFile, Rocks/CylindWall.bt, Rocks/Penetrator.bt), so scenes of
// one-sphere clumps with LocalPos = 0 pin the engine's and the oracle's
// cylinder wall with clump kinematics.
#include "dem.h"

int main() {
    DEMmain dem;
    dem.RunSimulation();
    return 0;
}
