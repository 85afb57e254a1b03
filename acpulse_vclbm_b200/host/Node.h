// Host-side shims of the reference's Node and GridCoupling classes (Node.h:9-
// 240, GridCoupling.h:7-45).  The engine has no per-node object: a Node here is
// a view of node (i, j, k) (level-global indices) of a level of a Lattice,
// reading the state back through the C ABI (acp_node_kind, and the
// populations behind Lattice::getDistribution).  The reference's per-node
// queries work on it -- identity, coordinates, distributions of either
// ping-pong array, density, pressure and velocity as Node.cpp:11-177 forms
// them.  The per-node update members (collisions, LODI, streaming, the grid
// coupling) keep their declared signatures, but the engine runs them for every
// node of a level at once inside Lattice::solve; called on one node they
// report that and exit, as the reference's own base-class fallbacks do
// (Node.h:149-166).
#pragma once

#include <string>

#include "Control.h"

class Lattice;

class Node {
public:
    Node(Lattice& lattice, int level, int i, int j, int k);
    virtual ~Node() {}

    // identity and coordinates (Node.h:38-47, 65, 67); coordinates are
    // index x level spacing (Lattice.cpp:33-35)
    virtual int getIndexI() const { return i_; }
    virtual int getIndexJ() const { return j_; }
    virtual int getIndexK() const { return k_; }
    virtual int getLevel() const { return level_; }
    virtual int getNodeID() { return id_; }  // 0 fluid, 1 boundary, 2 grid coupling, -1 no live node here
    // a boundary node on two or three domain faces (an edge or a corner)
    virtual bool getIsCorner() {
        const int f = faceClass_;
        return id_ == 1 && (f / 9 != 1) + ((f / 3) % 3 != 1) + (f % 3 != 1) >= 2;
    }
    virtual double getX() const;
    virtual double getY() const;
    virtual double getZ() const;
    virtual double getTimeStep() const;
    virtual std::string getTag();
    virtual std::string getGridCouplingTag();

    // state (Node.h:48-52): f_dir of the array `distr` names, and the
    // density / velocity of the current state
    virtual double getDistribution(bool& distr, int& dir);
    virtual double getNodeDensity();
    virtual double getNodeVelocityComponent(int dir);

    // macroscopic quantities (Node.cpp:11-177).  The cubic-Mach term the
    // reference adds (0.5 dt psi_q) has zero density and momentum moments, so
    // the population sums are the result in both forms.
    virtual double calcDensity(Control& bc, bool& alternating);
    virtual double calcPressure(bool& alternating, Control& bc);
    virtual void calcVelocity(Control& bc, bool& alternating, double& dens, double* velo);

    // per-node updates (Node.h:102-170): run level-wide by Lattice::solve
    virtual void collideSRT(Control& bc, bool& alternating);
    virtual void collideRR(Control& bc, bool& alternating);
    virtual void collideMRT_GSbasis(Control& bc, bool& alternating);
    virtual void collideMRT_RMbasis(Control& bc, bool& alternating);
    virtual void collideHRR(Control& bc, bool& alternating);
    virtual void LODIpressureOutlet(Control& bc, bool& alternating);
    virtual void calcStrainRateTensorFDandCubicMachCorrection(Control& bc);
    virtual void transport(bool& distr);

protected:
    [[noreturn]] void levelWide(const char* member) const;
    Lattice& lattice_;
    int level_, i_, j_, k_;
    int id_ = -1, faceClass_ = 13;
};

// GridCoupling (GridCoupling.h:7-45): the coupling members of a coupling node;
// the engine's coupling kernels run them for every coupling node of a step
class GridCoupling : public Node {
public:
    GridCoupling(Lattice& lattice, int level, int i, int j, int k);

    void interpolTimeDirectCoupling(bool& distrFi, bool& distrCoFut, Control& bc);
    void directCoupling(bool& distrFi, bool& distrCo, Control& bc);
    void interpolTimeScalingCoarseToFine(bool& distrFi, bool& distrCoFut, int& i, int& j, int& k, int& level,
                                         Node*****& mesh, Control& bc);
    void interpolTimeScalingCoarseToFineStrainRates(int& i, int& j, int& k, int& level, Node*****& mesh, Control& bc);
    void interpolTimeScalingCoarseToFineMRT_GSbasis(bool& distrFi, bool& distrCoFut, int& i, int& j, int& k, int& level,
                                                    Node*****& mesh, Control& bc);
    void scalingCoarseToFine(bool& distrFi, bool& distrCo, int& i, int& j, int& k, int& level, Node*****& mesh,
                             Control& bc);
    void scalingFineToCoarse(bool& distrCo, bool& distrFi, int& i, int& j, int& k, int& level, Node*****& mesh,
                             Control& bc);
    void scalingCoarseToFineMRT_GSbasis(bool& distrFi, bool& distrCo, int& i, int& j, int& k, int& level,
                                        Node*****& mesh, Control& bc);
    void scalingFineToCoarseMRT_GSbasis(bool& distrCo, bool& distrFi, int& i, int& j, int& k, int& level,
                                        Node*****& mesh, Control& bc);
    void scalingFineToCoarseMRT_TOU_GSbasis(bool& distrCo, bool& distrFi, int& i, int& j, int& k, int& level,
                                            Node*****& mesh, Control& bc);
    void scalingFineToCoarseMRT_LAG_GSbasis(bool& distrCo, bool& distrFi, int& i, int& j, int& k, int& level,
                                            Node*****& mesh, Control& bc);
    void scalingFineToCoarseLAG(bool& distrCo, bool& distrFi, int& i, int& j, int& k, int& level, Node*****& mesh,
                                Control& bc);
    void scalingFineToCoarseTOU(bool& distrCo, bool& distrFi, int& i, int& j, int& k, int& level, Node*****& mesh,
                                Control& bc);
    void interpolSpaceMidNode(bool& distrFi, int& i, int& j, int& k, int& d1Interpol, int& level, Control& bc,
                              Node*****& mesh);
    void interpolSpaceCenterNode(bool& distrFi, int& i, int& j, int& k, int& d2Interpol, int& level, Control& bc,
                                 Node*****& mesh);
    void interpolSpaceMidNodeStrainRates(int& i, int& j, int& k, int& d1Interpol, int& level, Control& bc,
                                         Node*****& mesh);
    void interpolSpaceCenterNodeStrainRates(int& i, int& j, int& k, int& d2Interpol, int& level, Control& bc,
                                            Node*****& mesh);
    void directCouplingCalcDeltaX(double* X, double* distr, double& rho, double* velo, std::string& interfaceType,
                                  Control& bc);
};
