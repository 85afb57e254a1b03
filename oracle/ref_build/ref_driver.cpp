// Driver for the reference's own Control/Lattice classes (compiled from the
// reference sources where they lie).  It replaces the reference's main.cpp,
// whose input path is hard-coded (main.cpp:44), and follows the same call
// pattern: Control(file) -> Lattice(bc) -> initialization(bc) -> solve(alt)
// once per coarse step with the ping-pong flag toggled by the caller
// (main.cpp:46-47, 98, 121, 155).  Instead of ASCII VTK it dumps the full
// FP64 distribution state through Lattice::getDistribution (Lattice.h:119).
//
// usage: acp_ref <BoundaryConditions.txt> <steps> <out.bin> [probe_every]
// out.bin layout (little endian):
//   int32 nx, ny, nz, steps
//   float64 f[nx][ny][nz][19]   -- state after `steps` steps, array `alt`
// When probe_every > 0 a second file <out.bin>.rho holds the density of every
// node after every probe_every steps (float64 [n_probe][nx][ny][nz]).
//
// usage: acp_ref --vtk <BoundaryConditions.txt> <steps> <prefix>
// writes the reference's ASCII VTK file <prefix>.vtk after `steps` steps.
//
// usage: acp_ref --topo <BoundaryConditions.txt> <out.txt>
// writes, for every boundary node of level 0, the wiring that setConnectivity
// (Lattice.cpp:500-1394) gives it: normal direction, the two normal
// neighbours, the in-plane (tangent) neighbours where they are set, the corner
// flag and the set of directions it pushes into.  The mesh is a private member
// of Lattice, so this translation unit opens the class for reading.
#include "Control.h"
#define private public
#include "Lattice.h"
#undef private
#include <map>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <vector>

static int dumpTopology(const char* bcFile, const char* outPath)
{
    Control bc(bcFile);
    Lattice lat(bc);
    int nx = bc.getNumberOfNodesX(), ny = bc.getNumberOfNodesY(), nz = bc.getNumberOfNodesZ();
    Node**** m = lat.mesh_[0];
    std::map<const Node*, long> id;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) id[m[i][j][k]] = ((long)k * ny + j) * nx + i;
    auto idx = [&](const Node* p) -> long {
        if (p == nullptr) return -1;
        auto it = id.find(p);
        return it == id.end() ? -2 : it->second;
    };
    FILE* f = std::fopen(outPath, "w");
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                Node* n = m[i][j][k];
                if (n->getTag() != "boundary") continue;
                int onB = (i == 0 || i == nx - 1) + (j == 0 || j == ny - 1) + (k == 0 || k == nz - 1);
                long push = 0;
                for (int d = 0; d < 18; ++d) {
                    long t = idx(n->getNeighbor(d));
                    if (t == -2) { std::fprintf(stderr, "stray neighbour pointer\n"); return 3; }
                    if (t >= 0) push |= 1L << d;
                }
                long t1a = -1, t1b = -1, t2a = -1, t2b = -1;
                if (onB == 1) {
                    t1a = idx(n->getTangentNeighbor1(0)); t1b = idx(n->getTangentNeighbor1(1));
                    t2a = idx(n->getTangentNeighbor2(0)); t2b = idx(n->getTangentNeighbor2(1));
                }
                std::fprintf(f, "%d %d %d %d %ld %ld %ld %ld %ld %ld %d %ld\n", i, j, k, n->getNormalDir(),
                             idx(n->getNormalNeighbor()), idx(n->getNormalNeighborSnd()), t1a, t1b, t2a, t2b,
                             onB == 1 ? 0 : (int)n->getIsCorner(), push);
            }
    std::fclose(f);
    return 0;
}

// the reference's own legacy VTK file (Lattice::writeResultsVTK,
// Lattice.cpp:2212-4352) after `steps` coarse steps, flags as main.cpp keeps them
static int writeVtk(const char* bcFile, int steps, const char* prefix)
{
    Control bc(bcFile);
    if (bc.getLevelMax() != 0) return 2;
    Lattice lat(bc);
    lat.initialization(bc);
    bool alt = true, altL1 = true;
    for (int t = 0; t < steps; ++t) {
        lat.solve(alt);
        alt = !alt;
    }
    lat.writeResultsVTK(prefix, alt, altL1);
    return 0;
}

int main(int argc, char** argv)
{
    if (argc == 4 && std::string(argv[1]) == "--topo") return dumpTopology(argv[2], argv[3]);
    if (argc == 5 && std::string(argv[1]) == "--vtk") return writeVtk(argv[2], std::atoi(argv[3]), argv[4]);
    if (argc < 4) {
        std::fprintf(stderr, "usage: %s <bc-file> <steps> <out.bin> [probe_every]\n", argv[0]);
        return 1;
    }
    std::string bcFile = argv[1];
    int steps = std::atoi(argv[2]);
    int probeEvery = argc > 4 ? std::atoi(argv[4]) : 0;
    Control bc(bcFile);
    if (bc.getLevelMax() != 0) {
        std::fprintf(stderr, "only MaxLevel 0 runs: GridCoupling bodies are absent\n");
        return 2;
    }
    Lattice lat(bc);
    lat.initialization(bc);
    int nx = bc.getNumberOfNodesX(), ny = bc.getNumberOfNodesY(), nz = bc.getNumberOfNodesZ();
    bool alt = true;
    int level = 0;
    std::vector<double> rhoTrace;
    auto t0 = std::chrono::steady_clock::now();
    for (int t = 0; t < steps; ++t) {
        lat.solve(alt);
        alt = !alt;
        if (probeEvery > 0 && (t + 1) % probeEvery == 0) {
            for (int i = 0; i < nx; ++i)
                for (int j = 0; j < ny; ++j)
                    for (int k = 0; k < nz; ++k) {
                        double r = 0.;
                        for (int d = 0; d < 19; ++d) r += lat.getDistribution(alt, d, level, i, j, k);
                        rhoTrace.push_back(r);
                    }
        }
    }
    auto t1 = std::chrono::steady_clock::now();
    double sec = std::chrono::duration<double>(t1 - t0).count();
    std::fprintf(stdout, "{\"nodes\": %lld, \"steps\": %d, \"seconds\": %.6f, \"mlups\": %.4f}\n",
                 (long long)nx * ny * nz, steps, sec,
                 sec > 0 ? (double)nx * ny * nz * steps / sec / 1e6 : 0.0);
    FILE* f = std::fopen(argv[3], "wb");
    if (!f) { std::perror("fopen"); return 1; }
    int hdr[4] = {nx, ny, nz, steps};
    std::fwrite(hdr, sizeof(int), 4, f);
    std::vector<double> buf((size_t)nx * ny * nz * 19);
    size_t p = 0;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k)
                for (int d = 0; d < 19; ++d) buf[p++] = lat.getDistribution(alt, d, level, i, j, k);
    std::fwrite(buf.data(), sizeof(double), buf.size(), f);
    std::fclose(f);
    if (probeEvery > 0) {
        std::string tr = std::string(argv[3]) + ".rho";
        FILE* g = std::fopen(tr.c_str(), "wb");
        std::fwrite(rhoTrace.data(), sizeof(double), rhoTrace.size(), g);
        std::fclose(g);
    }
    return 0;
}
