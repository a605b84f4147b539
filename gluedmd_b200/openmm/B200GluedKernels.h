// OpenMM CUDA-platform adapter: GLUED's CalcGluedForceKernel implemented over
// this library's C ABI (include/glued_b200.h).
//
// It replaces the reference's CudaCalcGluedForceKernel / CommonCalcGluedForceKernel
// (platforms/cuda/src/CudaGluedKernelFactory.cpp:20-72, platforms/common/src/
// CommonGluedKernels.cpp:4608-5288) behind the unchanged GluedForce /
// GluedForceImpl (openmmapi/src/GluedForceImpl.cpp:36-165): the factory is
// registered by registerKernelFactories() (CudaGluedKernelFactory.cpp:77-98),
// the kernel reads OpenMM's posq, atom index array and long force buffer in
// place (zero copy) and rebuilds its user -> GPU slot map when OpenMM reorders
// atoms (CommonCVKernels.cpp:113-124), through a ReorderListener.
//
// Build: compiled with OpenMM's headers (openmm/..., openmm/cuda/...) and GLUED's
// openmmapi headers (GluedForce.h, GluedKernels.h), linked with
// libglued_b200.so and OpenMM's CUDA platform library.
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "GluedForce.h"
#include "GluedKernels.h"
#include "glued_b200.h"
#include "openmm/KernelFactory.h"
#include "openmm/cuda/CudaContext.h"

namespace GluedB200 {

// Throws OpenMM::OpenMMException with the library's message when rc != 0.
void check(int rc, const char* what);

// The descriptor of a GluedForce (its CVs, biases and settings) for the C ABI.
// The caller owns the returned descriptor (glued_force_destroy).
glued_force* describe(const GluedPlugin::GluedForce& force);

class B200CalcGluedForceKernel : public GluedPlugin::CalcGluedForceKernel {
public:
    B200CalcGluedForceKernel(std::string name, const OpenMM::Platform& platform, OpenMM::CudaContext& cu);
    ~B200CalcGluedForceKernel() override;
    void initialize(const OpenMM::System& system, const GluedPlugin::GluedForce& force) override;
    double execute(OpenMM::ContextImpl& context, bool includeForces, bool includeEnergy) override;
    void updateState(OpenMM::ContextImpl& context, int step) override;
    void getCurrentCVs(OpenMM::ContextImpl& context, std::vector<double>& values) override;
    std::vector<char> getBiasStateBytes() override;
    void setBiasStateBytes(const std::vector<char>& bytes) override;
    std::vector<double> downloadCVValues() override;
    double downloadLastBias() override;
    std::vector<double> getOPESMetrics(int biasIndex) override;
    std::vector<float> getKernelSigmas(int biasIndex) override;
    std::vector<long long> getMultiWalkerPtrs(int biasType, int localIdx) override;
    void redirectToPrimaryBias(int biasType, int localIdx, const std::vector<long long>& ptrs) override;

    // The library context (null before initialize) and the descriptor it was built from.
    glued_context* context() const { return ctx_; }
    const glued_force* descriptor() const { return desc_; }

private:
    class Reorder;
    int globalBiasIndex(int biasType, int localIdx) const;
    // binds OpenMM's current stream and buffers (again whenever one of them changed)
    void bindBuffers();
    OpenMM::CudaContext& cu_;
    glued_force* desc_ = nullptr;
    glued_context* ctx_ = nullptr;
    int numCVValues_ = 0;
    std::vector<int> biasTypes_;        // addBias order
    std::shared_ptr<bool> reordered_;   // set by the reorder listener, consumed by execute
    bool bound_ = false;
    void* stream_ = nullptr;
    const void* posq_ = nullptr;
    const int* index_ = nullptr;
    long long* force_ = nullptr;
    int padded_ = 0;
};

class B200GluedKernelFactory : public OpenMM::KernelFactory {
public:
    OpenMM::KernelImpl* createKernelImpl(std::string name, const OpenMM::Platform& platform,
                                         OpenMM::ContextImpl& context) const override;
};

}  // namespace GluedB200

extern "C" void registerKernelFactories();
