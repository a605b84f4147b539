// TEST HARNESS (not product code): an in-process stand-in for the OpenMM
// runtime pieces the B200 adapter (gluedmd_b200/openmm/B200GluedKernels.cpp)
// touches, so that the adapter compiles and runs where OpenMM is not
// installed. It provides the platform registry, a CUDA platform whose
// CudaContext hands out device buffers the test allocated, a ContextImpl with
// a box and step count, and a C API the Python tests drive: register the
// plugin's factories, build a GluedForce, create the kernel through the
// registered factory exactly as OpenMM's ContextImpl does, then initialize /
// updateState / execute / read back through the CalcGluedForceKernel interface.
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "B200GluedKernels.h"
#include "openmm/OpenMMException.h"
#include "openmm/cuda/CudaPlatform.h"

using namespace OpenMM;

namespace OpenMM {
static std::vector<Platform*>& platformList() {
    static std::vector<Platform*> p;
    return p;
}
Platform::~Platform() {}
void Platform::registerKernelFactory(const std::string& name, KernelFactory* factory) { factories_[name] = factory; }
KernelFactory* Platform::kernelFactory(const std::string& name) const {
    auto it = factories_.find(name);
    return it == factories_.end() ? nullptr : it->second;
}
int Platform::getNumPlatforms() { return (int)platformList().size(); }
Platform& Platform::getPlatform(int index) { return *platformList()[index]; }
void Platform::registerPlatform(Platform* platform) { platformList().push_back(platform); }
}  // namespace OpenMM

namespace {
// A platform without CUDA: registerKernelFactories must leave it alone.
class ReferencePlatform : public Platform {
public:
    const std::string& getName() const override {
        static const std::string n = "Reference";
        return n;
    }
};

std::string g_error;

struct Harness {
    System system;
    GluedPlugin::GluedForce force;
    CudaContext cu;
    CudaPlatform::PlatformData data;
    std::unique_ptr<ContextImpl> impl;
    std::unique_ptr<GluedPlugin::CalcGluedForceKernel> kernel;
};

CudaPlatform* cudaPlatform() {
    for (int i = 0; i < Platform::getNumPlatforms(); i++)
        if (auto* p = dynamic_cast<CudaPlatform*>(&Platform::getPlatform(i))) return p;
    return nullptr;
}

template <class F>
int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

Harness& H(void* h) { return *static_cast<Harness*>(h); }
}  // namespace

extern "C" {

const char* stub_error() { return g_error.c_str(); }

// Registers a Reference and a CUDA platform (once), runs the plugin's
// registerKernelFactories and returns a bit mask of the platforms that got a
// CalcGluedForce factory (bit 0: Reference, bit 1: CUDA).
int stub_init_platforms() {
    if (Platform::getNumPlatforms() == 0) {
        Platform::registerPlatform(new ReferencePlatform());
        Platform::registerPlatform(new CudaPlatform());
    }
    registerKernelFactories();
    int mask = 0;
    for (int i = 0; i < Platform::getNumPlatforms(); i++)
        if (Platform::getPlatform(i).kernelFactory(GluedPlugin::CalcGluedForceKernel::Name()))
            mask |= dynamic_cast<CudaPlatform*>(&Platform::getPlatform(i)) ? 2 : 1;
    return mask;
}

void* stub_new() { return new Harness(); }
void stub_delete(void* h) { delete static_cast<Harness*>(h); }

void stub_add_particle(void* h, double mass) { H(h).system.addParticle(mass); }

void stub_add_cv(void* h, int type, const int* atoms, int na, const double* p, int np) {
    H(h).force.addCV(type, std::vector<int>(atoms, atoms + na), std::vector<double>(p, p + np));
}

void stub_add_bias(void* h, int type, const int* cvs, int nc, const double* p, int np, const int* ip, int ni) {
    H(h).force.addBias(type, std::vector<int>(cvs, cvs + nc), std::vector<double>(p, p + np),
                       std::vector<int>(ip, ip + ni));
}

void stub_set_config(void* h, double temperature, int pbc, const double* grad, int ng) {
    Harness& x = H(h);
    x.force.temperature_ = temperature;
    x.force.pbc_ = pbc != 0;
    x.force.testGrad_.assign(grad, grad + ng);
}

// The descriptor the adapter builds from the force, as the library's XML.
int stub_describe_xml(void* h, char* buf, size_t* len) {
    return guarded([&] {
        glued_force* f = GluedB200::describe(H(h).force);
        const int rc = glued_force_serialize_xml(f, buf, len);
        glued_force_destroy(f);
        GluedB200::check(rc, "serialize");
    });
}

// Creates the kernel through the CUDA platform's registered factory (as
// ContextImpl does for GluedForceImpl::initialize) and initializes it with the
// given device buffers (CUdeviceptr values) and stream.
int stub_create(void* h, unsigned long long posq, unsigned long long atomIndex, unsigned long long force, int padded,
                unsigned long long stream, int doublePrecision) {
    return guarded([&] {
        Harness& x = H(h);
        CudaPlatform* platform = cudaPlatform();
        if (!platform) throw OpenMMException("no CUDA platform registered");
        KernelFactory* factory = platform->kernelFactory(GluedPlugin::CalcGluedForceKernel::Name());
        if (!factory) throw OpenMMException("no CalcGluedForce factory on the CUDA platform");
        x.cu.setBuffers((CUdeviceptr)posq, (CUdeviceptr)atomIndex, (CUdeviceptr)force, padded);
        x.cu.setStream(reinterpret_cast<CUstream>(stream));
        x.cu.setUseDoublePrecision(doublePrecision != 0);
        x.data.contexts.assign(1, &x.cu);
        x.impl.reset(new ContextImpl(x.system, &x.data));
        KernelImpl* k = factory->createKernelImpl(GluedPlugin::CalcGluedForceKernel::Name(), *platform, *x.impl);
        x.kernel.reset(dynamic_cast<GluedPlugin::CalcGluedForceKernel*>(k));
        if (!x.kernel) throw OpenMMException("factory did not return a CalcGluedForceKernel");
        x.kernel->initialize(x.system, x.force);
    });
}

int stub_set_box(void* h, const double* b) {
    return guarded([&] { H(h).impl->setPeriodicBoxVectors(Vec3(b[0], b[1], b[2]), Vec3(b[3], b[4], b[5]), Vec3(b[6], b[7], b[8])); });
}

int stub_execute(void* h, int forces, int energy, double* e) {
    return guarded([&] { *e = H(h).kernel->execute(*H(h).impl, forces != 0, energy != 0); });
}

int stub_update_state(void* h, int step) {
    return guarded([&] {
        H(h).impl->setStepCount(step);
        H(h).kernel->updateState(*H(h).impl, step);
    });
}

int stub_notify_reordered(void* h) {
    return guarded([&] { H(h).cu.notifyReordered(); });
}

int stub_cv_values(void* h, double* out, int n) {
    return guarded([&] {
        std::vector<double> v;
        H(h).kernel->getCurrentCVs(*H(h).impl, v);
        if ((int)v.size() != n) throw OpenMMException("CV count mismatch");
        std::memcpy(out, v.data(), sizeof(double) * n);
    });
}

int stub_last_bias(void* h, double* e) {
    return guarded([&] { *e = H(h).kernel->downloadLastBias(); });
}

int stub_bias_state(void* h, char* buf, size_t* len) {
    return guarded([&] {
        std::vector<char> b = H(h).kernel->getBiasStateBytes();
        if (buf && *len >= b.size()) std::memcpy(buf, b.data(), b.size());
        *len = b.size();
    });
}

int stub_set_bias_state(void* h, const char* buf, size_t len) {
    return guarded([&] { H(h).kernel->setBiasStateBytes(std::vector<char>(buf, buf + len)); });
}

int stub_opes_metrics(void* h, int i, double* out) {
    return guarded([&] {
        std::vector<double> m = H(h).kernel->getOPESMetrics(i);
        std::memcpy(out, m.data(), sizeof(double) * m.size());
    });
}

int stub_kernel_sigmas(void* h, int i, float* out, int* n) {
    return guarded([&] {
        std::vector<float> s = H(h).kernel->getKernelSigmas(i);
        if (out && *n >= (int)s.size()) std::memcpy(out, s.data(), sizeof(float) * s.size());
        *n = (int)s.size();
    });
}

int stub_multiwalker_ptrs(void* h, int biasType, int localIdx, long long* out, int* n) {
    return guarded([&] {
        std::vector<long long> p = H(h).kernel->getMultiWalkerPtrs(biasType, localIdx);
        if (out && *n >= (int)p.size()) std::memcpy(out, p.data(), sizeof(long long) * p.size());
        *n = (int)p.size();
    });
}

int stub_redirect(void* h, int biasType, int localIdx, const long long* ptrs, int n) {
    return guarded([&] { H(h).kernel->redirectToPrimaryBias(biasType, localIdx, std::vector<long long>(ptrs, ptrs + n)); });
}

}  // extern "C"
