// Drop-in replacement of the reference's Lattice class (Lattice.h:9-125):
// the same public members, implemented over the C ABI.  There is no per-node
// object on the host: the state lives on the GPU in the engine's layout, and
// getDistribution reads it back (either ping-pong array, as the reference's
// does) through a host cache refreshed after each solve.  The caller's
// ping-pong flags keep their meaning: after solve(alt) and the caller's
// toggle (main.cpp:121,155), the current state is the array the flag names.
#pragma once

#include <string>
#include <vector>

#include "Control.h"

class Lattice {
public:
    explicit Lattice(Control& bc);  // Lattice.h:23: builds the levels and allocates the device state
    ~Lattice();

    virtual void solve(bool& alternating);                         // one coarse step, single level (Lattice.cpp:2158)
    virtual void solve(bool& alternatingL0, bool& alternatingL1);  // one coarse step, two levels (Lattice.cpp:2185)
    virtual void initialization(Control& bc);                      // Lattice.cpp:1397-1493
    // ASCII legacy VTK (structured points per level) with Pressure, Density and Velocity
    virtual void writeResultsVTK(std::string filename, bool& alternating, bool& alternatingL1);
    // f_dir of node (i, j, k) of a level (level-global node indices), array named by `alternating`
    virtual double getDistribution(bool& alternating, int& dir, int& level, int& i, int& j, int& k);
    virtual double readValue(std::string filename, std::string keyword) { return bc_.readValue(filename, keyword); }

    acp_handle* handle() { return h_; }
    Control& control() { return bc_; }
    bool currentFlag() const { return currentFlag_; }  // the flag value naming the current state

private:
    void check(int status, const char* what);
    void refresh(int level, int which);

    Control& bc_;
    acp_handle* h_ = nullptr;
    bool currentFlag_ = false;  // the flag value naming the current array
    long long stepsSeen_[2][2] = {{-1, -1}, {-1, -1}};  // [current / other array][level]
    std::vector<double> cache_[2][2];
    int dims_[2][3] = {{0, 0, 0}, {0, 0, 0}};
    int origin_[2][3] = {{0, 0, 0}, {0, 0, 0}};
};
