// Test stub: OpenMM's KernelFactory interface.
#pragma once
#include <string>
namespace OpenMM {
class ContextImpl;
class KernelImpl;
class Platform;
class KernelFactory {
public:
    virtual ~KernelFactory() {}
    virtual KernelImpl* createKernelImpl(std::string name, const Platform& platform, ContextImpl& context) const = 0;
};
}  // namespace OpenMM
