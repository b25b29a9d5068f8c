// main.cpp -- the reference's executable (src/main.cpp:4-16) on the B200 engine.
#include <cstdio>

#include "dem_clump_main.h"

int main() {
    DEMClumpMain dem;
    dem.RunSimulationClump();
    std::printf("Final!!\n");
    return dem.LastStatus() == NBC_OK ? 0 : 1;
}
