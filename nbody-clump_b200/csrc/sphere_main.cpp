// sphere_main.cpp -- an executable for the sphere-only drivers: the calls
// the reference's main() has commented out (src/main.cpp:10-11), one of them
// selected by the argument (cylinder = RunSimulation, the default; cube =
// RunSimulation2; split = RunSimulation_Split; hgrid = RunSimulation_HGrid).
#include <cstdio>
#include <cstring>

#include "dem_main.h"

int main(int argc, char** argv) {
    const char* which = argc > 1 ? argv[1] : "cylinder";
    DEMmain dem;
    if (!std::strcmp(which, "cylinder")) dem.RunSimulation();
    else if (!std::strcmp(which, "cube")) dem.RunSimulation2();
    else if (!std::strcmp(which, "split")) dem.RunSimulation_Split();
    else if (!std::strcmp(which, "hgrid")) dem.RunSimulation_HGrid();
    else {
        std::fprintf(stderr, "usage: %s [cylinder|cube|split|hgrid]\n", argv[0]);
        return 2;
    }
    std::printf("Final!!\n");
    return dem.LastStatus() == NBC_OK ? 0 : 1;
}
