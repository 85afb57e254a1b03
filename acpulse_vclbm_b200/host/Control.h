// Drop-in replacement of the reference's Control class (Control.h:10-129):
// the same constructor and getters, backed by the C ABI's case parser
// (acp_parse_case_file), which applies the reference's keyword rules.
// Errors keep the reference's behaviour at this level: message on stderr and
// exit(1) (Control.cpp:144-165).
#pragma once

#include <string>

#include "../../include/acp.h"

class Control {
public:
    Control() {}
    explicit Control(std::string filename);
    ~Control() {}

    // same reading helpers as the reference (Control.cpp:135-273)
    double readValue(std::string filename, std::string keyword);
    std::string readString(std::string filename, std::string keyword);
    std::string readFileName(std::string filename, std::string keyword);
    void readVector(std::string filename, std::string keyword, double* vector);

    int getNumberOfNodesX() { return desc_.nx; }
    int getNumberOfNodesY() { return desc_.ny; }
    int getNumberOfNodesZ() { return desc_.nz; }
    int getLevelMax() { return desc_.max_level; }
    int getTimeStepMax() { return timeStepMax_; }
    int getWriteInterval() { return writeInterval_; }
    int getNumberOfThreads() { return numberOfThreads_; }
    int getRefinementLayer() { return desc_.ref_layer_yz; }
    int getRefinementLayerX() { return desc_.ref_layer_x; }
    int getOrderOfEquilibrium() { return desc_.eq_order; }
    void setTime_(double time) { time_ = time; }
    double getSpacing() { return desc_.spacing; }
    double getHybridParameter() { return desc_.hybrid_sigma; }
    double getDensity() { return desc_.density; }
    double getMachNumber() { return desc_.mach; }
    double getMolecularVelocity() { return molecularVelocity_; }
    double getReynoldsNumber() { return 0.; }
    double getSpeedOfSound() { return desc_.speed_of_sound; }
    double getKinematicViscosity() { return desc_.kinematic_viscosity; }
    double getTimeStep() { return timeStep_; }
    double getTime_() { return time_; }
    double getChannelSizeX_() { return desc_.domain_size[0]; }
    double getChannelSizeY_() { return desc_.domain_size[1]; }
    double getChannelSizeZ_() { return desc_.domain_size[2]; }
    double getXsi(int& dir, int& comp) { return xsi_[dir][comp]; }
    double getXsi(unsigned short& dir, unsigned short& comp) { return xsi_[dir][comp]; }
    double* getXsiX() { return xsiX_; }
    double* getXsiY() { return xsiY_; }
    double* getXsiZ() { return xsiZ_; }
    double* getXsi(int& dir) { return xsi_[dir]; }
    double* getXsi(unsigned short& dir) { return xsi_[dir]; }
    double* getWeightFactors() { return weightFactors_; }
    double getLODIK1relaxation() { return desc_.k1; }
    double getLODIK2relaxation() { return lodiK2relaxation_; }
    virtual double getCollisionFrequency() { return collisionFrequency_; }
    virtual double getOverlap() { return desc_.overlap; }
    std::string getCaseName() { return caseName_; }
    std::string getCollisionModel() { return collisionModel_; }
    std::string getCouplingReplacementC2F() { return c2f_; }
    std::string getCouplingReplacementF2C() { return f2c_; }
    std::string getHangingNodeReconstruction() { return hanging_; }
    std::string getScalingStyle() { return scalingStyle_; }
    std::string getReflectionHandling() { return reflecting_; }
    std::string getTransverseInclusion() { return desc_.transverse ? "yes" : "no"; }
    std::string getCubicMachCorrection() { return desc_.cubic_mach ? "yes" : "no"; }
    std::string getF2Cfilter() { return f2cFilter_; }
    std::string getCouplingProcedure() { return coupling_; }

    // the parsed case in the C ABI's form
    const acp_case_desc& caseDescription() const { return desc_; }
    acp_case_desc& caseDescription() { return desc_; }

private:
    acp_case_desc desc_{};
    int timeStepMax_ = 0, writeInterval_ = 1, numberOfThreads_ = 1;
    double time_ = 0, molecularVelocity_ = 0, timeStep_ = 0, collisionFrequency_ = 0, lodiK2relaxation_ = 0;
    double xsiX_[19], xsiY_[19], xsiZ_[19], xsi_[19][3], weightFactors_[19];
    std::string caseName_, collisionModel_, c2f_, f2c_, hanging_, scalingStyle_, reflecting_, f2cFilter_, coupling_;
};
