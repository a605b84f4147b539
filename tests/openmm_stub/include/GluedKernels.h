// Test stub: GLUED's abstract kernel interface (openmmapi/include/GluedKernels.h:23-105),
// the virtual functions the adapter overrides.
#pragma once
#include <string>
#include <vector>
#include "GluedForce.h"
#include "openmm/KernelImpl.h"
#include "openmm/Platform.h"
#include "openmm/System.h"
#include "openmm/internal/ContextImpl.h"
namespace OpenMM { class Context; }
namespace GluedPlugin {
class CalcGluedForceKernel : public OpenMM::KernelImpl {
public:
    static std::string Name() { return "CalcGluedForce"; }
    CalcGluedForceKernel(std::string name, const OpenMM::Platform& platform) : OpenMM::KernelImpl(name, platform) {}
    virtual void initialize(const OpenMM::System& system, const GluedForce& force) = 0;
    virtual void setInnerContext(OpenMM::Context* inner, OpenMM::ContextImpl* innerImpl) {}
    virtual double execute(OpenMM::ContextImpl& context, bool includeForces, bool includeEnergy) = 0;
    virtual void updateState(OpenMM::ContextImpl& context, int step) = 0;
    virtual void getCurrentCVs(OpenMM::ContextImpl& context, std::vector<double>& values) = 0;
    virtual std::vector<char> getBiasStateBytes() = 0;
    virtual void setBiasStateBytes(const std::vector<char>& bytes) = 0;
    virtual std::vector<double> downloadCVValues() = 0;
    virtual double downloadLastBias() { return 0.0; }
    virtual std::vector<double> getOPESMetrics(int biasIndex) = 0;
    virtual std::vector<float> getKernelSigmas(int biasIndex) = 0;
    virtual std::vector<long long> getMultiWalkerPtrs(int biasType, int localIdx) { return {}; }
    virtual void redirectToPrimaryBias(int biasType, int localIdx, const std::vector<long long>& ptrs) {}
};
}  // namespace GluedPlugin
