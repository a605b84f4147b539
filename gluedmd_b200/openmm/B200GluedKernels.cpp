// OpenMM CUDA-platform adapter over the C ABI; see B200GluedKernels.h.
#include "B200GluedKernels.h"

#include <memory>

#include "openmm/OpenMMException.h"
#include "openmm/Platform.h"
#include "openmm/System.h"
#include "openmm/Vec3.h"
#include "openmm/common/ContextSelector.h"
#include "openmm/cuda/CudaArray.h"
#include "openmm/cuda/CudaPlatform.h"
#include "openmm/internal/ContextImpl.h"

using namespace OpenMM;
using GluedPlugin::GluedForce;

namespace GluedB200 {

void check(int rc, const char* what) {
    if (rc != GLUED_OK) throw OpenMMException(std::string(what) + ": " + glued_last_error());
}

glued_force* describe(const GluedForce& force) {
    glued_force* f = nullptr;
    check(glued_force_create(&f), "GluedForce descriptor");
    try {
        int idx = 0;
        for (int i = 0; i < force.getNumCollectiveVariableSpecs(); i++) {
            int type = 0;
            std::vector<int> atoms;
            std::vector<double> params;
            force.getCollectiveVariableInfo(i, type, atoms, params);
            if (type == GluedForce::CV_EXPRESSION) {
                std::string expr;
                std::vector<int> inputs;
                force.getExpressionCVInfo(i, expr, inputs);
                check(glued_force_add_expression_cv(f, expr.c_str(), inputs.data(), (int)inputs.size(), &idx),
                      "addExpressionCV");
            } else if (type == GluedForce::CV_PYTORCH) {
                const std::string path = force.getPyTorchCVModelPath(i);
                check(glued_force_add_pytorch_cv(f, path.c_str(), atoms.data(), (int)atoms.size(), params.data(),
                                                 (int)params.size(), &idx),
                      "addPyTorchCV");
            } else {
                check(glued_force_add_cv(f, type, atoms.data(), (int)atoms.size(), params.data(), (int)params.size(),
                                         &idx),
                      "addCollectiveVariable");
            }
        }
        for (int i = 0; i < force.getNumBiases(); i++) {
            int type = 0;
            std::vector<int> cvs, ip;
            std::vector<double> p;
            force.getBiasInfo(i, type, cvs, p, ip);
            check(glued_force_add_bias(f, type, cvs.data(), (int)cvs.size(), p.data(), (int)p.size(), ip.data(),
                                       (int)ip.size(), &idx),
                  "addBias");
        }
        check(glued_force_set_temperature(f, force.getTemperature()), "setTemperature");
        check(glued_force_set_pbc(f, force.usesPeriodicBoundaryConditions() ? 1 : 0), "setUsesPeriodicBoundaryConditions");
        check(glued_force_set_force_group(f, force.getForceGroup()), "setForceGroup");
        check(glued_force_set_test_force(f, force.getTestForceMode(), force.getTestForceScale()), "setTestForce");
        const std::vector<double> g = force.getTestBiasGradients();
        if (!g.empty()) check(glued_force_set_test_bias_gradients(f, g.data(), (int)g.size()), "setTestBiasGradients");
    } catch (...) {
        glued_force_destroy(f);
        throw;
    }
    return f;
}

// OpenMM calls execute() on its reorder listeners after it has reordered the
// atoms (the ComputeContext owns and deletes them); the next force evaluation
// then rebuilds the user -> GPU slot map on the device.
class B200CalcGluedForceKernel::Reorder : public ComputeContext::ReorderListener {
public:
    explicit Reorder(std::shared_ptr<bool> flag) : flag_(std::move(flag)) {}
    void execute() override { *flag_ = true; }

private:
    std::shared_ptr<bool> flag_;
};

B200CalcGluedForceKernel::B200CalcGluedForceKernel(std::string name, const Platform& platform, CudaContext& cu)
    : CalcGluedForceKernel(name, platform), cu_(cu), reordered_(std::make_shared<bool>(false)) {}

B200CalcGluedForceKernel::~B200CalcGluedForceKernel() {
    if (ctx_) {
        ContextSelector selector(cu_);
        glued_context_destroy(ctx_);
    }
    if (desc_) glued_force_destroy(desc_);
}

void B200CalcGluedForceKernel::bindBuffers() {
    void* stream = reinterpret_cast<void*>(cu_.getCurrentStream());
    const void* posq = reinterpret_cast<const void*>(cu_.getPosq().getDevicePointer());
    const int* index = reinterpret_cast<const int*>(cu_.getAtomIndexArray().getDevicePointer());
    long long* force = reinterpret_cast<long long*>(cu_.getLongForceBuffer().getDevicePointer());
    const int padded = cu_.getPaddedNumAtoms();
    if (bound_ && stream == stream_ && posq == posq_ && index == index_ && force == force_ && padded == padded_)
        return;
    check(glued_context_bind(ctx_, stream, posq, index, force, padded), "bind OpenMM buffers");
    stream_ = stream; posq_ = posq; index_ = index; force_ = force; padded_ = padded;
    bound_ = true;
}

void B200CalcGluedForceKernel::initialize(const System& system, const GluedForce& force) {
    if (cu_.getUseDoublePrecision())
        throw OpenMMException("GluedForce (B200): double-precision contexts are not supported (posq must be float4)");
    desc_ = describe(force);
    check(glued_force_num_cv_values(desc_, &numCVValues_), "getNumCollectiveVariables");
    biasTypes_.clear();
    for (int i = 0; i < force.getNumBiases(); i++) {
        int type = 0;
        std::vector<int> cvs, ip;
        std::vector<double> p;
        force.getBiasInfo(i, type, cvs, p, ip);
        biasTypes_.push_back(type);
    }
    const int n = system.getNumParticles();
    std::vector<double> masses(n);
    for (int i = 0; i < n; i++) masses[i] = system.getParticleMass(i);
    ContextSelector selector(cu_);
    check(glued_context_create(desc_, n, masses.data(), &ctx_), "GluedForce initialize");
    bindBuffers();
    cu_.addReorderListener(new Reorder(reordered_));
}

double B200CalcGluedForceKernel::execute(ContextImpl& context, bool includeForces, bool includeEnergy) {
    ContextSelector selector(cu_);
    bindBuffers();
    if (*reordered_) {
        check(glued_context_atoms_reordered(ctx_), "atom reorder");
        *reordered_ = false;
    }
    Vec3 a, b, c;
    context.getPeriodicBoxVectors(a, b, c);
    const double box[9] = {a[0], a[1], a[2], b[0], b[1], b[2], c[0], c[1], c[2]};
    check(glued_context_set_box(ctx_, box), "periodic box");
    double energy = 0.0;
    check(glued_context_execute(ctx_, includeForces ? 1 : 0, includeEnergy ? 1 : 0, &energy), "GluedForce execute");
    return includeEnergy ? energy : 0.0;
}

void B200CalcGluedForceKernel::updateState(ContextImpl& context, int step) {
    ContextSelector selector(cu_);
    bindBuffers();
    check(glued_context_update_state(ctx_, step), "GluedForce updateState");
}

void B200CalcGluedForceKernel::getCurrentCVs(ContextImpl& context, std::vector<double>& values) {
    values = downloadCVValues();
}

std::vector<char> B200CalcGluedForceKernel::getBiasStateBytes() {
    ContextSelector selector(cu_);
    size_t n = 0;
    check(glued_context_get_bias_state(ctx_, nullptr, &n), "getBiasStateBytes");
    std::vector<char> out(n);
    check(glued_context_get_bias_state(ctx_, out.data(), &n), "getBiasStateBytes");
    out.resize(n);
    return out;
}

void B200CalcGluedForceKernel::setBiasStateBytes(const std::vector<char>& bytes) {
    ContextSelector selector(cu_);
    check(glued_context_set_bias_state(ctx_, bytes.data(), bytes.size()), "setBiasStateBytes");
}

std::vector<double> B200CalcGluedForceKernel::downloadCVValues() {
    ContextSelector selector(cu_);
    std::vector<double> out(numCVValues_);
    if (numCVValues_ > 0) check(glued_context_get_cv_values(ctx_, out.data(), numCVValues_), "downloadCVValues");
    return out;
}

double B200CalcGluedForceKernel::downloadLastBias() {
    ContextSelector selector(cu_);
    double e = 0.0;
    check(glued_context_get_last_bias(ctx_, &e), "downloadLastBias");
    return e;
}

std::vector<double> B200CalcGluedForceKernel::getOPESMetrics(int biasIndex) {
    ContextSelector selector(cu_);
    std::vector<double> out(4);
    check(glued_context_opes_metrics(ctx_, biasIndex, out.data()), "getOPESMetrics");
    return out;
}

std::vector<float> B200CalcGluedForceKernel::getKernelSigmas(int biasIndex) {
    // an invalid index yields an empty vector (CommonGluedKernels.cpp:5212-5215)
    int nOpes = 0;
    for (int t : biasTypes_) nOpes += t == GluedForce::BIAS_OPES;
    if (biasIndex < 0 || biasIndex >= nOpes) return {};
    ContextSelector selector(cu_);
    int n = 0;
    check(glued_context_kernel_sigmas(ctx_, biasIndex, nullptr, &n), "getKernelSigmas");
    std::vector<float> out(n);
    if (n > 0) check(glued_context_kernel_sigmas(ctx_, biasIndex, out.data(), &n), "getKernelSigmas");
    out.resize(n);
    return out;
}

int B200CalcGluedForceKernel::globalBiasIndex(int biasType, int localIdx) const {
    int k = 0;
    for (int i = 0; i < (int)biasTypes_.size(); i++)
        if (biasTypes_[i] == biasType && k++ == localIdx) return i;
    return -1;
}

std::vector<long long> B200CalcGluedForceKernel::getMultiWalkerPtrs(int biasType, int localIdx) {
    // only METAD grids and OPES tables are shared (CudaGluedKernelFactory.cpp:30-46)
    if (biasType != GluedForce::BIAS_METAD && biasType != GluedForce::BIAS_OPES) return {};
    const int g = globalBiasIndex(biasType, localIdx);
    if (g < 0) return {};
    ContextSelector selector(cu_);
    std::vector<long long> out(8);
    int n = (int)out.size();
    check(glued_context_multiwalker_ptrs(ctx_, g, out.data(), &n), "getMultiWalkerPtrs");
    out.resize(n);
    return out;
}

void B200CalcGluedForceKernel::redirectToPrimaryBias(int biasType, int localIdx, const std::vector<long long>& ptrs) {
    if (biasType != GluedForce::BIAS_METAD && biasType != GluedForce::BIAS_OPES) return;
    const int g = globalBiasIndex(biasType, localIdx);
    if (g < 0) return;
    ContextSelector selector(cu_);
    check(glued_context_set_multiwalker_ptrs(ctx_, g, ptrs.data(), (int)ptrs.size()), "redirectToPrimaryBias");
}

KernelImpl* B200GluedKernelFactory::createKernelImpl(std::string name, const Platform& platform,
                                                    ContextImpl& context) const {
    if (name == GluedPlugin::CalcGluedForceKernel::Name()) {
        CudaPlatform::PlatformData& data = *static_cast<CudaPlatform::PlatformData*>(context.getPlatformData());
        return new B200CalcGluedForceKernel(name, platform, *data.contexts[0]);
    }
    throw OpenMMException("B200GluedKernelFactory: unknown kernel name: " + name);
}

}  // namespace GluedB200

// Called by OpenMM's plugin loader after the CUDA platform library is loaded
// (CudaGluedKernelFactory.cpp:77-86): one factory for every CUDA platform.
extern "C" void registerKernelFactories() {
    for (int i = 0; i < OpenMM::Platform::getNumPlatforms(); i++) {
        OpenMM::Platform& platform = OpenMM::Platform::getPlatform(i);
        if (dynamic_cast<OpenMM::CudaPlatform*>(&platform) != nullptr)
            platform.registerKernelFactory(GluedPlugin::CalcGluedForceKernel::Name(),
                                           new GluedB200::B200GluedKernelFactory());
    }
}
