// Lattice over the C ABI (see Lattice.h).
#include "Lattice.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <vector>
#include <string>
#include <sstream>

void Lattice::check(int status, const char* what) {
    if (status != ACP_OK) {
        std::cerr << what << ": " << acp_status_string(status) << ": " << acp_last_error(h_) << std::endl;
        std::exit(1);
    }
}

Lattice::Lattice(Control& bc) : bc_(bc) {
    check(acp_create(&bc.caseDescription(), -1, &h_), "Lattice");
    const acp_case_desc& d = bc.caseDescription();
    for (int l = 0; l <= d.max_level; ++l) {
        check(acp_level_dims(h_, l, dims_[l]), "Lattice");
        check(acp_level_origin(h_, l, origin_[l]), "Lattice");
    }
}

Lattice::~Lattice() {
    if (h_) acp_destroy(h_);
}

void Lattice::initialization(Control&) {
    check(acp_init(h_), "initialization");
    // main.cpp:55-57: both flags start true and the state is in both arrays
    currentFlag_ = true;
    for (auto& w : stepsSeen_) w[0] = w[1] = -1;
}

void Lattice::solve(bool& alternating) {
    check(acp_step(h_, 1), "solve");
    // the reference collides in array `alternating` and streams into the other,
    // which the caller then selects by toggling its flag (main.cpp:155)
    currentFlag_ = !alternating;
}

void Lattice::solve(bool& alternatingL0, bool&) {
    check(acp_step(h_, 1), "solve");
    currentFlag_ = !alternatingL0;
}

void Lattice::refresh(int level, int which) {
    long long steps = 0;
    acp_steps_done(h_, &steps);
    if (stepsSeen_[which][level] == steps) return;
    check(acp_sync(h_), "sync");
    const size_t n = (size_t)dims_[level][0] * dims_[level][1] * dims_[level][2];
    cache_[which][level].resize(n * 19);
    check(which == 0 ? acp_read_populations(h_, level, cache_[which][level].data())
                     : acp_read_populations_other(h_, level, cache_[which][level].data()),
          "getDistribution");
    stepsSeen_[which][level] = steps;
}

double Lattice::getDistribution(bool& alternating, int& dir, int& level, int& i, int& j, int& k) {
    if (dir >= 19 || level < 0 || level > bc_.caseDescription().max_level) return 0.;
    // the flag naming the current state reads it; the other flag reads the
    // other ping-pong array (acp_read_populations_other)
    const int which = alternating == currentFlag_ ? 0 : 1;
    refresh(level, which);
    const int li = i - origin_[level][0], lj = j - origin_[level][1], lk = k - origin_[level][2];
    const int* n = dims_[level];
    if (li < 0 || lj < 0 || lk < 0 || li >= n[0] || lj >= n[1] || lk >= n[2]) return 0.;
    const size_t N = (size_t)n[0] * n[1] * n[2];
    return cache_[which][level][(size_t)dir * N + ((size_t)lk * n[1] + lj) * n[0] + li];
}

// The reference's legacy VTK file (Lattice::writeResultsVTK, Lattice.cpp:2212-
// 4352): one ASCII UNSTRUCTURED_GRID of every live node with voxel cells,
// numbers in scientific notation with 8 digits, the point and cell counts
// patched into fixed-width fields after the data.  Single level: the
// reference's layout exactly (nodes in k, j, i order; Pressure, Density,
// Omega, Velocity).  Two levels: the reference's fields (Omega, NodeID,
// Pressure, Density, Velocity) over the live fine nodes followed by the live
// coarse nodes, each in k, j, i order, with the voxels whose eight corners
// are live on one level (the reference orders the fine shell region by
// region, Lattice.cpp:2244-2400).  With `Non-Reflecting yes` a boundary node
// off the x = 0 face is written from the other ping-pong array, as the
// reference does (Lattice.cpp:4202-4215).  acp_write_vtk writes the binary
// structured-points form of the same fields.
void Lattice::writeResultsVTK(std::string filename, bool& alternatingL0, bool&) {
    filename.append(".vtk");
    std::ofstream out(filename.c_str());
    if (!out) {
        std::cerr << "An error occured while writing paraview file\n";
        return;
    }
    check(acp_sync(h_), "writeResultsVTK");
    const acp_case_desc& d = bc_.caseDescription();
    const int levels = d.max_level + 1;
    const bool reflecting = bc_.getReflectionHandling() != "no";
    struct P {
        int level, i, j, k, id;
    };
    std::vector<P> pts;
    std::vector<std::vector<int>> index(levels);  // local node -> point index (-1: no live node)
    for (int step = 0; step < levels; ++step) {
        const int level = levels - 1 - step;  // the fine level first
        const int* n = dims_[level];
        const int* o = origin_[level];
        index[level].assign((size_t)n[0] * n[1] * n[2], -1);
        for (int k = 0; k < n[2]; ++k)
            for (int j = 0; j < n[1]; ++j)
                for (int i = 0; i < n[0]; ++i) {
                    int id = -1, face = 13;
                    acp_node_kind(h_, level, o[0] + i, o[1] + j, o[2] + k, &id, &face);
                    if (id < 0) continue;
                    index[level][((size_t)k * n[1] + j) * n[0] + i] = (int)pts.size();
                    pts.push_back({level, i, j, k, id});
                }
    }
    for (int level = 0; level < levels; ++level) {
        refresh(level, 0);
        if (reflecting) refresh(level, 1);
    }
    const double cs = bc_.getSpeedOfSound(), cs2 = std::pow(cs, 2.);
    auto f = [&](const P& p, int which, int dir) {
        const int* n = dims_[p.level];
        const size_t N = (size_t)n[0] * n[1] * n[2];
        return cache_[which][p.level][(size_t)dir * N + ((size_t)p.k * n[1] + p.j) * n[0] + p.i];
    };
    auto arrayOf = [&](const P& p) { return reflecting && p.id == 1 && (p.i + origin_[p.level][0]) > 0 ? 1 : 0; };
    auto density = [&](const P& p) {
        const int w = arrayOf(p);
        double dens = 0;
        for (int dir = 0; dir < 19; dir++) dens += f(p, w, dir);
        return dens;
    };
    out << "# vtk DataFile Version 2.0" << "\n";
    out << "LBM results for grid refinement benchmark in channel flow\n";
    out << "ASCII" << "\n";
    out << "DATASET UNSTRUCTURED_GRID" << "\n";
    auto padded = [](const std::string& v, size_t width) { return v + std::string(width > v.size() ? width - v.size() : 0, ' '); };
    out << "POINTS " << padded(std::to_string(pts.size()), 14) << " float" << "\n";
    out << std::setiosflags(std::ios::left | std::ios::showpoint | std::ios::scientific) << std::setprecision(8);
    for (const P& p : pts) {
        const double h = bc_.getSpacing() / std::pow(2., p.level);
        out << (p.i + origin_[p.level][0]) * h << " " << (p.j + origin_[p.level][1]) * h << " "
            << (p.k + origin_[p.level][2]) * h << "\n";
    }
    out << "\n";
    // voxels (VTK type 11) whose eight corners are live nodes of one level
    std::ostringstream cells;
    long long cellCntr = 0;
    for (int step = 0; step < levels; ++step) {
        const int level = levels - 1 - step;
        const int* n = dims_[level];
        auto at = [&](int i, int j, int k) { return index[level][((size_t)k * n[1] + j) * n[0] + i]; };
        for (int k = 0; k + 1 < n[2]; ++k)
            for (int j = 0; j + 1 < n[1]; ++j)
                for (int i = 0; i + 1 < n[0]; ++i) {
                    const int c[8] = {at(i, j, k),         at(i + 1, j, k),         at(i, j + 1, k),
                                      at(i + 1, j + 1, k), at(i, j, k + 1),         at(i + 1, j, k + 1),
                                      at(i, j + 1, k + 1), at(i + 1, j + 1, k + 1)};
                    bool all = true;
                    for (int m = 0; m < 8; ++m) all = all && c[m] >= 0;
                    if (!all) continue;
                    cells << "8 " << c[0] << " " << c[1] << " " << c[2] << " " << c[3] << " " << c[4] << " " << c[5]
                          << " " << c[6] << " " << c[7] << "\n";
                    ++cellCntr;
                }
    }
    out << "CELLS " << padded(std::to_string(cellCntr) + " " + std::to_string(9 * cellCntr), 19) << "\n";
    out << cells.str() << "\n";
    out << "CELL_TYPES " << cellCntr << "\n";
    for (long long c = 0; c < cellCntr; ++c) out << "11" << "\n";
    out << "\n";
    out << "POINT_DATA " << pts.size() << "\n";
    auto omega = [&](int level) {
        const double dt = bc_.getTimeStep() / std::pow(2., level);
        return (cs2 * dt) / (bc_.getKinematicViscosity() + 0.5 * cs2 * dt);
    };
    auto writeOmega = [&]() {
        out << "SCALARS Omega float 1" << "\n" << "LOOKUP_TABLE default" << "\n";
        for (const P& p : pts) out << omega(p.level) << "\n";
    };
    auto writePressure = [&]() {
        out << "SCALARS Pressure float 1" << "\n" << "LOOKUP_TABLE default" << "\n";
        for (const P& p : pts) out << density(p) * cs2 << "\n";
    };
    auto writeDensity = [&]() {
        out << "SCALARS Density float 1" << "\n" << "LOOKUP_TABLE default" << "\n";
        for (const P& p : pts) out << density(p) << "\n";
    };
    if (levels == 1) {
        writePressure();
        writeDensity();
        writeOmega();
    } else {
        writeOmega();
        out << "SCALARS NodeID float 1" << "\n" << "LOOKUP_TABLE default" << "\n";
        for (const P& p : pts) out << (double)p.id << "\n";
        writePressure();
        writeDensity();
    }
    out << "\nVECTORS Velocity float " << "\n";
    const double* xx = bc_.getXsiX();
    const double* xy = bc_.getXsiY();
    const double* xz = bc_.getXsiZ();
    for (const P& p : pts) {
        const int w = arrayOf(p);
        const double dens = density(p);
        double velo[3] = {0., 0., 0.};
        for (int dir = 0; dir < 19; dir++) {
            const double v = f(p, w, dir);
            velo[0] += xx[dir] * v;
            velo[1] += xy[dir] * v;
            velo[2] += xz[dir] * v;
        }
        for (double& v : velo) v /= dens;
        out << velo[0] << " " << velo[1] << " " << velo[2] << " " << "\n";
    }
}
