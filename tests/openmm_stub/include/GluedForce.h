// Test stub: the GluedForce accessors the adapter reads (openmmapi/include/
// GluedForce.h:113-239), over plain storage the test harness fills.
#pragma once
#include <string>
#include <vector>
namespace GluedPlugin {
class GluedForce {
public:
    enum { CV_EXPRESSION = 8, CV_PYTORCH = 9 };
    enum { BIAS_METAD = 3, BIAS_OPES = 5 };
    int getNumCollectiveVariableSpecs() const { return (int)cvType_.size(); }
    void getCollectiveVariableInfo(int idx, int& type, std::vector<int>& atoms, std::vector<double>& params) const {
        type = cvType_[idx]; atoms = cvAtoms_[idx]; params = cvParams_[idx];
    }
    void getExpressionCVInfo(int idx, std::string& expression, std::vector<int>& inputs) const {
        expression = cvString_[idx]; inputs = cvAtoms_[idx];
    }
    std::string getPyTorchCVModelPath(int idx) const { return cvString_[idx]; }
    int getNumBiases() const { return (int)biasType_.size(); }
    void getBiasInfo(int idx, int& type, std::vector<int>& cvs, std::vector<double>& params,
                     std::vector<int>& intParams) const {
        type = biasType_[idx]; cvs = biasCvs_[idx]; params = biasParams_[idx]; intParams = biasInts_[idx];
    }
    double getTemperature() const { return temperature_; }
    bool usesPeriodicBoundaryConditions() const { return pbc_; }
    int getForceGroup() const { return group_; }
    int getTestForceMode() const { return testMode_; }
    double getTestForceScale() const { return testScale_; }
    std::vector<double> getTestBiasGradients() const { return testGrad_; }
    // harness setters
    void addCV(int type, const std::vector<int>& atoms, const std::vector<double>& params, const std::string& s = "") {
        cvType_.push_back(type); cvAtoms_.push_back(atoms); cvParams_.push_back(params); cvString_.push_back(s);
    }
    void addBias(int type, const std::vector<int>& cvs, const std::vector<double>& params, const std::vector<int>& ints) {
        biasType_.push_back(type); biasCvs_.push_back(cvs); biasParams_.push_back(params); biasInts_.push_back(ints);
    }
    double temperature_ = 300.0;
    bool pbc_ = false;
    int group_ = 0, testMode_ = 0;
    double testScale_ = 0.0;
    std::vector<double> testGrad_;
private:
    std::vector<int> cvType_, biasType_;
    std::vector<std::vector<int>> cvAtoms_, biasCvs_, biasInts_;
    std::vector<std::vector<double>> cvParams_, biasParams_;
    std::vector<std::string> cvString_;
};
}  // namespace GluedPlugin
