// The reference's driver loop (main.cpp:37-271) on the drop-in Control and
// Lattice: construct, initialise, call solve once per coarse step with the
// caller-owned ping-pong flags, toggle the flag, write results every
// WriteInterval.  Prints the throughput in MLUPS at the end.
//
// usage: acp_main <BoundaryConditions.txt> [steps] [--dump-rho file] [--no-vtk]
//                 [--dump-nodes file level]
// --dump-nodes writes, for every node of a level (x fastest), the Node view's
// ID, density, velocity and pressure (six doubles), and prints the count of
// each GridCoupling tag of that level.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sstream>
#include <string>
#include <vector>

#include <map>

#include "Control.h"
#include "Lattice.h"
#include "Node.h"

int main(int argc, char* argv[]) {
    if (argc < 2) {
        std::fprintf(stderr,
                     "usage: %s <BoundaryConditions.txt> [steps] [--dump-rho file] [--no-vtk] [--dump-nodes file level]\n",
                     argv[0]);
        return 1;
    }
    std::string dump, dumpNodes;
    int nodesLevel = 0;
    bool vtk = true;
    int stepsArg = -1;
    for (int a = 2; a < argc; ++a) {
        if (!std::strcmp(argv[a], "--dump-rho") && a + 1 < argc) dump = argv[++a];
        else if (!std::strcmp(argv[a], "--no-vtk")) vtk = false;
        else if (!std::strcmp(argv[a], "--dump-nodes") && a + 2 < argc) {
            dumpNodes = argv[++a];
            nodesLevel = std::atoi(argv[++a]);
        }
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
    if (!dumpNodes.empty()) {
        int dims[3], origin[3];
        acp_level_dims(simulationCase.handle(), nodesLevel, dims);
        acp_level_origin(simulationCase.handle(), nodesLevel, origin);
        FILE* f = std::fopen(dumpNodes.c_str(), "wb");
        std::map<std::string, long long> tags;
        for (int k = origin[2]; k < origin[2] + dims[2]; ++k)
            for (int j = origin[1]; j < origin[1] + dims[1]; ++j)
                for (int i = origin[0]; i < origin[0] + dims[0]; ++i) {
                    Node node(simulationCase, nodesLevel, i, j, k);
                    double rec[6] = {(double)node.getNodeID(), 0, 0, 0, 0, 0};
                    if (node.getNodeID() >= 0) {
                        rec[1] = node.calcDensity(boundaryConditions, alternatingL0);
                        node.calcVelocity(boundaryConditions, alternatingL0, rec[1], rec + 2);
                        rec[5] = node.calcPressure(alternatingL0, boundaryConditions);
                    }
                    if (node.getNodeID() == 2) ++tags[GridCoupling(simulationCase, nodesLevel, i, j, k).getGridCouplingTag()];
                    std::fwrite(rec, sizeof rec, 1, f);
                }
        std::fclose(f);
        std::printf("{");
        const char* sep = "";
        for (const auto& t : tags) {
            std::printf("%s\"%s\": %lld", sep, t.first.c_str(), t.second);
            sep = ", ";
        }
        std::printf("}\n");
    }
    return 0;
}
