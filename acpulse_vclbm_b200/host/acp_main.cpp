// The reference's driver loop (main.cpp:37-271) on the drop-in Control and
// Lattice: construct, initialise, call solve once per coarse step with the
// caller-owned ping-pong flags, toggle the flag, write results every
// WriteInterval.  Prints the throughput in MLUPS at the end.
//
// usage: acp_main <BoundaryConditions.txt> [steps] [--dump-rho file] [--no-vtk]
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sstream>
#include <string>
#include <vector>

#include "Control.h"
#include "Lattice.h"

int main(int argc, char* argv[]) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s <BoundaryConditions.txt> [steps] [--dump-rho file] [--no-vtk]\n", argv[0]);
        return 1;
    }
    std::string dump;
    bool vtk = true;
    int stepsArg = -1;
    for (int a = 2; a < argc; ++a) {
        if (!std::strcmp(argv[a], "--dump-rho") && a + 1 < argc) dump = argv[++a];
        else if (!std::strcmp(argv[a], "--no-vtk")) vtk = false;
        else stepsArg = std::atoi(argv[a]);
    }
    Control boundaryConditions(argv[1]);
    Lattice simulationCase(boundaryConditions);
    const int maxTimeStep = stepsArg >= 0 ? stepsArg : boundaryConditions.getTimeStepMax();
    const int writeInterval = boundaryConditions.getWriteInterval();
    const int maxLevel = boundaryConditions.getLevelMax();
    bool alternatingL0 = true, negAlternatingL0 = false, alternatingL1 = true;
    simulationCase.initialization(boundaryConditions);
    auto t0 = std::chrono::steady_clock::now();
    for (int time = 0; time < maxTimeStep;) {
        if (maxLevel == 0) simulationCase.solve(alternatingL0);
        else simulationCase.solve(alternatingL0, alternatingL1);
        ++time;
        boundaryConditions.setTime_(static_cast<double>(time));
        alternatingL0 = !alternatingL0;
        negAlternatingL0 = !negAlternatingL0;
        if (vtk && writeInterval > 0 && time % writeInterval == 0) {
            std::ostringstream name;
            name << boundaryConditions.getCaseName() << "_" << time;
            simulationCase.writeResultsVTK(name.str(), alternatingL0, alternatingL1);
        }
    }
    long long coarse = 0, fine = 0;
    acp_sync(simulationCase.handle());
    auto t1 = std::chrono::steady_clock::now();
    acp_active_updates(simulationCase.handle(), &coarse, &fine);
    const double sec = std::chrono::duration<double>(t1 - t0).count();
    std::printf("{\"steps\": %d, \"seconds\": %.6f, \"mlups\": %.3f}\n", maxTimeStep, sec,
                sec > 0 ? (coarse + 2.0 * fine) * maxTimeStep / sec / 1e6 : 0.0);
    if (!dump.empty()) {
        // density of every node of level 0, x fastest, through getDistribution
        FILE* f = std::fopen(dump.c_str(), "wb");
        int level = 0;
        for (int k = 0; k < boundaryConditions.getNumberOfNodesZ(); ++k)
            for (int j = 0; j < boundaryConditions.getNumberOfNodesY(); ++j)
                for (int i = 0; i < boundaryConditions.getNumberOfNodesX(); ++i) {
                    double r = 0;
                    for (int d = 0; d < 19; ++d) r += simulationCase.getDistribution(alternatingL0, d, level, i, j, k);
                    std::fwrite(&r, sizeof r, 1, f);
                }
        std::fclose(f);
    }
    return 0;
}
