// Node and GridCoupling views over the C ABI (see Node.h).
#include "Node.h"

#include <cmath>
#include <cstdlib>
#include <iostream>

#include "Lattice.h"

Node::Node(Lattice& lattice, int level, int i, int j, int k) : lattice_(lattice), level_(level), i_(i), j_(j), k_(k) {
    if (acp_node_kind(lattice.handle(), level, i, j, k, &id_, &faceClass_) != ACP_OK) {
        std::cerr << "\nNode: level " << level << " does not exist" << std::endl;
        std::exit(1);
    }
}

static double levelSpacing(Control& bc, int level) { return bc.getSpacing() / std::pow(2., level); }

double Node::getX() const { return i_ * levelSpacing(lattice_.control(), level_); }
double Node::getY() const { return j_ * levelSpacing(lattice_.control(), level_); }
double Node::getZ() const { return k_ * levelSpacing(lattice_.control(), level_); }
double Node::getTimeStep() const { return lattice_.control().getTimeStep() / std::pow(2., level_); }

std::string Node::getTag() {
    switch (id_) {
        case 0: return "fluid";
        case 1: return "boundary";
        case 2: return "gridcoupling";
        default: return "none";
    }
}

// the interface faces of a coupling node by the reference's face names
// (Lattice.cpp:42-57: bottom/top in z, left/right in y, front/back in x);
// empty where the engine keeps no face class (the coupling nodes of the level
// that lies outside the refined box)
std::string Node::getGridCouplingTag() {
    if (id_ != 2) {
        std::cerr << "\nGetGridCouplinTag() from node invoked." << std::flush;
        std::exit(1);
    }
    const int fx = faceClass_ / 9 - 1, fy = (faceClass_ / 3) % 3 - 1, fz = faceClass_ % 3 - 1;
    std::string t;
    if (fz) t += fz < 0 ? "bottom" : "top";
    if (fy) t += fy < 0 ? "left" : "right";
    if (fx) t += fx < 0 ? "front" : "back";
    return t;
}

double Node::getDistribution(bool& distr, int& dir) {
    if (dir >= 19) return 0.;
    return lattice_.getDistribution(distr, dir, level_, i_, j_, k_);
}

double Node::calcDensity(Control&, bool& alternating) {
    double dens = 0;
    for (int dir = 0; dir < 19; dir++) dens += getDistribution(alternating, dir);
    return dens;
}

double Node::calcPressure(bool& alternating, Control& bc) {
    const double cs = bc.getSpeedOfSound();
    return calcDensity(bc, alternating) * cs * cs;
}

void Node::calcVelocity(Control& bc, bool& alternating, double& dens, double* velo) {
    velo[0] = velo[1] = velo[2] = 0.;
    const double* xx = bc.getXsiX();
    const double* xy = bc.getXsiY();
    const double* xz = bc.getXsiZ();
    for (int dir = 0; dir < 19; dir++) {
        const double f = getDistribution(alternating, dir);
        velo[0] += xx[dir] * f;
        velo[1] += xy[dir] * f;
        velo[2] += xz[dir] * f;
    }
    for (int c = 0; c < 3; ++c) velo[c] /= dens;
}

double Node::getNodeDensity() {
    bool cur = lattice_.currentFlag();
    return calcDensity(lattice_.control(), cur);
}

double Node::getNodeVelocityComponent(int dir) {
    bool cur = lattice_.currentFlag();
    double dens = calcDensity(lattice_.control(), cur), velo[3];
    calcVelocity(lattice_.control(), cur, dens, velo);
    return dir >= 0 && dir < 3 ? velo[dir] : 0.;
}

void Node::levelWide(const char* member) const {
    std::cerr << "\n" << member << " from node invoked: the engine runs it for every node of level " << level_
              << " at once inside Lattice::solve." << std::flush;
    std::exit(1);
}

void Node::collideSRT(Control&, bool&) { levelWide("collideSRT"); }
void Node::collideRR(Control&, bool&) { levelWide("collideRR"); }
void Node::collideMRT_GSbasis(Control&, bool&) { levelWide("collideMRT_GSbasis"); }
void Node::collideMRT_RMbasis(Control&, bool&) { levelWide("collideMRT_RMbasis"); }
void Node::collideHRR(Control&, bool&) { levelWide("collideHRR"); }
void Node::LODIpressureOutlet(Control&, bool&) { levelWide("LODIpressureOutlet"); }
void Node::calcStrainRateTensorFDandCubicMachCorrection(Control&) {
    levelWide("calcStrainRateTensorFDandCubicMachCorrection");
}
void Node::transport(bool&) { levelWide("transport"); }

GridCoupling::GridCoupling(Lattice& lattice, int level, int i, int j, int k) : Node(lattice, level, i, j, k) {
    if (id_ != 2) {
        std::cerr << "\nGridCoupling: node (" << i << ", " << j << ", " << k << ") of level " << level
                  << " is not a coupling node" << std::endl;
        std::exit(1);
    }
}

// the coupling members: the engine's coupling kernels (C2F time and space
// interpolation, F2C restriction, direct coupling) run them for all coupling
// nodes of a step at once
void GridCoupling::interpolTimeDirectCoupling(bool&, bool&, Control&) { levelWide("interpolTimeDirectCoupling"); }
void GridCoupling::directCoupling(bool&, bool&, Control&) { levelWide("directCoupling"); }
void GridCoupling::interpolTimeScalingCoarseToFine(bool&, bool&, int&, int&, int&, int&, Node*****&, Control&) {
    levelWide("interpolTimeScalingCoarseToFine");
}
void GridCoupling::interpolTimeScalingCoarseToFineStrainRates(int&, int&, int&, int&, Node*****&, Control&) {
    levelWide("interpolTimeScalingCoarseToFineStrainRates");
}
void GridCoupling::interpolTimeScalingCoarseToFineMRT_GSbasis(bool&, bool&, int&, int&, int&, int&, Node*****&,
                                                              Control&) {
    levelWide("interpolTimeScalingCoarseToFineMRT_GSbasis");
}
void GridCoupling::scalingCoarseToFine(bool&, bool&, int&, int&, int&, int&, Node*****&, Control&) {
    levelWide("scalingCoarseToFine");
}
void GridCoupling::scalingFineToCoarse(bool&, bool&, int&, int&, int&, int&, Node*****&, Control&) {
    levelWide("scalingFineToCoarse");
}
void GridCoupling::scalingCoarseToFineMRT_GSbasis(bool&, bool&, int&, int&, int&, int&, Node*****&, Control&) {
    levelWide("scalingCoarseToFineMRT_GSbasis");
}
void GridCoupling::scalingFineToCoarseMRT_GSbasis(bool&, bool&, int&, int&, int&, int&, Node*****&, Control&) {
    levelWide("scalingFineToCoarseMRT_GSbasis");
}
void GridCoupling::scalingFineToCoarseMRT_TOU_GSbasis(bool&, bool&, int&, int&, int&, int&, Node*****&, Control&) {
    levelWide("scalingFineToCoarseMRT_TOU_GSbasis");
}
void GridCoupling::scalingFineToCoarseMRT_LAG_GSbasis(bool&, bool&, int&, int&, int&, int&, Node*****&, Control&) {
    levelWide("scalingFineToCoarseMRT_LAG_GSbasis");
}
void GridCoupling::scalingFineToCoarseLAG(bool&, bool&, int&, int&, int&, int&, Node*****&, Control&) {
    levelWide("scalingFineToCoarseLAG");
}
void GridCoupling::scalingFineToCoarseTOU(bool&, bool&, int&, int&, int&, int&, Node*****&, Control&) {
    levelWide("scalingFineToCoarseTOU");
}
void GridCoupling::interpolSpaceMidNode(bool&, int&, int&, int&, int&, int&, Control&, Node*****&) {
    levelWide("interpolSpaceMidNode");
}
void GridCoupling::interpolSpaceCenterNode(bool&, int&, int&, int&, int&, int&, Control&, Node*****&) {
    levelWide("interpolSpaceCenterNode");
}
void GridCoupling::interpolSpaceMidNodeStrainRates(int&, int&, int&, int&, int&, Control&, Node*****&) {
    levelWide("interpolSpaceMidNodeStrainRates");
}
void GridCoupling::interpolSpaceCenterNodeStrainRates(int&, int&, int&, int&, int&, Control&, Node*****&) {
    levelWide("interpolSpaceCenterNodeStrainRates");
}
void GridCoupling::directCouplingCalcDeltaX(double*, double*, double&, double*, std::string&, Control&) {
    levelWide("directCouplingCalcDeltaX");
}
