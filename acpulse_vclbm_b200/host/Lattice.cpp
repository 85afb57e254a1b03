// Lattice over the C ABI (see Lattice.h).
#include "Lattice.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>

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

void Lattice::writeResultsVTK(std::string filename, bool&, bool&) {
    // the reference's ASCII form; acp_write_vtk(h, prefix, 1) writes the binary form of the same files
    check(acp_write_vtk(h_, filename.c_str(), 0), "writeResultsVTK");
}
