// GluedForce descriptor: the CV / bias specification a context is built from.
// Same data model and validation as openmmapi/include/GluedForce.h:113-239 and
// openmmapi/src/GluedForce.cpp:11-133, without the OpenMM base class.
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

namespace glued {

// Error with a GLUED_E_* code; the C ABI converts it to a return value.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// Type codes of openmmapi/include/GluedForce.h:27-95.
enum CVType {
    CV_DISTANCE = 1, CV_ANGLE = 2, CV_DIHEDRAL = 3, CV_COM_DISTANCE = 4, CV_GYRATION = 5,
    CV_COORDINATION = 6, CV_RMSD = 7, CV_EXPRESSION = 8, CV_PYTORCH = 9, CV_PATH = 10,
    CV_POSITION = 11, CV_DRMSD = 12, CV_CONTACTMAP = 13, CV_PLANE = 14, CV_PROJECTION = 15,
    CV_PUCKERING = 16, CV_DIPOLE = 17, CV_VOLUME = 18, CV_CELL = 19, CV_SECONDARY_STRUCTURE = 20,
    CV_PCA = 21, CV_ERMSD = 22, CV_ENERGY = 23,
    // Extensions of this library (no reference counterpart):
    // coordination with a hard cutoff (params [r0, n, m, rc]: pairs at r >= rc are left out),
    // and RMSD after optimal superposition (FP64 quaternion eigensolve).
    CV_COORDINATION_CUTOFF = 106, CV_RMSD_KABSCH = 107,
};
enum BiasType {
    BIAS_HARMONIC = 1, BIAS_MOVING_RESTRAINT = 2, BIAS_METAD = 3, BIAS_PBMETAD = 4, BIAS_OPES = 5,
    BIAS_EXTERNAL = 6, BIAS_ABMD = 7, BIAS_UPPER_WALL = 8, BIAS_LOWER_WALL = 9, BIAS_LINEAR = 10,
    BIAS_OPES_EXPANDED = 11, BIAS_EXT_LAGRANGIAN = 12, BIAS_MAXENT = 13, BIAS_EDS = 14,
    BIAS_OPES_MULTITHERMAL = 15,
    // Extension: well-tempered metadynamics as a direct hill sum instead of a grid.
    // params [h0, sigma_0..D-1, gamma, kT, lo_0..D-1, hi_0..D-1]
    // intParams [pace, maxHills, periodic_0..D-1] (period = hi - lo when periodic).
    BIAS_METAD_HILLS = 103,
};

struct CVSpec {
    int type = 0;
    std::vector<int> atoms;
    std::vector<double> params;
    std::string str;  // expression (CV_EXPRESSION) or model path (CV_PYTORCH)
};

struct BiasSpec {
    int type = 0;
    std::vector<int> cvs;
    std::vector<double> params;
    std::vector<int> iparams;
};

class GluedForce {
public:
    int addCollectiveVariable(int type, const std::vector<int>& atoms, const std::vector<double>& params);
    int addExpressionCV(const std::string& expr, const std::vector<int>& inputs);
    int addPyTorchCV(const std::string& path, const std::vector<int>& atoms, const std::vector<double>& params);
    int addBias(int type, const std::vector<int>& cvs, const std::vector<double>& params,
                const std::vector<int>& iparams);

    int numCVValues() const { return numCVValues_; }
    int numCVSpecs() const { return (int)cvs_.size(); }
    int numBiases() const { return (int)biases_.size(); }
    const CVSpec& cv(int i) const;
    const BiasSpec& bias(int i) const;
    const std::vector<CVSpec>& cvs() const { return cvs_; }
    const std::vector<BiasSpec>& biases() const { return biases_; }

    double temperature = -1.0;
    bool usesPBC = false;
    int forceGroup = 0;
    int testForceMode = 0;
    double testForceScale = 0.0;
    std::vector<double> testBiasGradients;

    std::string toXml() const;
    static GluedForce fromXml(const std::string& xml);

private:
    std::vector<CVSpec> cvs_;
    std::vector<BiasSpec> biases_;
    int numCVValues_ = 0;
};

}  // namespace glued
