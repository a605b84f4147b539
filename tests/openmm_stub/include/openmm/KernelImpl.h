// Test stub: base class of OpenMM kernel implementations.
#pragma once
#include <string>
namespace OpenMM {
class Platform;
class KernelImpl {
public:
    KernelImpl(std::string name, const Platform& platform) : name_(name), platform_(&platform) {}
    virtual ~KernelImpl() {}
    std::string getName() const { return name_; }
    const Platform& getPlatform() { return *platform_; }
private:
    std::string name_;
    const Platform* platform_;
};
}  // namespace OpenMM
