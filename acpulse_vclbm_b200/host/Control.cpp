// Control over the C ABI (see Control.h).
#include "Control.h"

#include <cmath>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <sstream>

namespace {

// first line whose first token equals the keyword (Control.cpp:150-161)
bool findKey(const std::string& file, const std::string& key, std::string& line) {
    std::ifstream in(file.c_str());
    if (!in) {
        std::cerr << "Error reading boundary conditions file " << file;
        std::exit(1);
    }
    std::string s;
    while (std::getline(in, s)) {
        std::istringstream sin(s);
        std::string op;
        if (!(sin >> op)) continue;
        if (op == key) {
            line = s;
            return true;
        }
    }
    return false;
}

}  // namespace

Control::Control(std::string filename) {
    char err[512] = {0};
    if (acp_parse_case_file(filename.c_str(), &desc_, err, sizeof err) != ACP_OK) {
        std::cerr << err;
        std::exit(1);
    }
    timeStepMax_ = static_cast<int>(readValue(filename, "Max-Time-Step"));
    writeInterval_ = static_cast<int>(readValue(filename, "WriteInterval"));
    numberOfThreads_ = static_cast<int>(readValue(filename, "Threads"));
    lodiK2relaxation_ = readValue(filename, "K2-Relaxation");
    caseName_ = readFileName(filename, "Save-as");
    collisionModel_ = readString(filename, "Collision-Model");
    c2f_ = readString(filename, "Coarse-to-Fine");
    f2c_ = readString(filename, "Fine-to-Coarse");
    hanging_ = readString(filename, "Hanging-Node-Reconstruction");
    scalingStyle_ = readString(filename, "Scaling-Style");
    reflecting_ = readString(filename, "Non-Reflecting");
    f2cFilter_ = readString(filename, "F2C-Filter");
    coupling_ = readString(filename, "Coupling-Approach");
    // derived lattice constants (Control.cpp:51-131)
    molecularVelocity_ = desc_.speed_of_sound * std::sqrt(3.);
    timeStep_ = desc_.spacing / molecularVelocity_;
    const double cs2 = std::pow(desc_.speed_of_sound, 2);
    collisionFrequency_ = (cs2 * timeStep_) / (desc_.kinematic_viscosity + 0.5 * cs2 * timeStep_);
    const int ex[19] = {1, 0, -1, 0, 0, 0, 1, 1, 0, 0, -1, -1, 0, 0, -1, 1, 1, -1, 0};
    const int ey[19] = {0, 1, 0, -1, 0, 0, 0, 0, 1, 1, 0, 0, -1, -1, 1, -1, 1, -1, 0};
    const int ez[19] = {0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 0};
    for (int d = 0; d < 19; ++d) {
        xsiX_[d] = ex[d] * molecularVelocity_;
        xsiY_[d] = ey[d] * molecularVelocity_;
        xsiZ_[d] = ez[d] * molecularVelocity_;
        xsi_[d][0] = xsiX_[d];
        xsi_[d][1] = xsiY_[d];
        xsi_[d][2] = xsiZ_[d];
        weightFactors_[d] = d < 6 ? 1. / 18. : (d < 18 ? 1. / 36. : 1. / 3.);
    }
}

double Control::readValue(std::string filename, std::string keyword) {
    std::string line;
    if (!findKey(filename, keyword, line)) {
        std::cerr << "No Value for keyword \"" + keyword + "\" found in " << filename;
        std::exit(1);
    }
    std::istringstream sin(line);
    std::string op;
    double number = 0.;
    sin >> op >> number;
    return number;
}

std::string Control::readString(std::string filename, std::string keyword) {
    std::string line;
    if (!findKey(filename, keyword, line)) {
        std::cerr << "No Value for keyword \"" << keyword << "\" found in " << filename;
        std::exit(1);
    }
    std::istringstream sin(line);
    std::string op, value;
    sin >> op >> value;
    return value;
}

std::string Control::readFileName(std::string filename, std::string keyword) {
    std::string line;
    if (!findKey(filename, keyword, line)) {
        std::cerr << "No Value for keyword \"" << keyword << "\" found in " << filename;
        std::exit(1);
    }
    std::string temp = line.substr(line.find(keyword) + keyword.length());
    const size_t found = temp.find_first_not_of(" ");
    return found == std::string::npos ? std::string() : temp.substr(found);
}

void Control::readVector(std::string filename, std::string keyword, double* vector) {
    std::string line;
    if (!findKey(filename, keyword, line)) {
        std::cerr << "No Value for keyword \"" << keyword << "\" found in " << filename;
        std::exit(1);
    }
    std::istringstream sin(line);
    std::string op;
    sin >> op >> vector[0] >> vector[1] >> vector[2];
}
