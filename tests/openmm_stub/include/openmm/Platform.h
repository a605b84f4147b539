// Test stub: OpenMM's Platform registry (static list of platforms, kernel
// factories registered by name).
#pragma once
#include <map>
#include <string>
namespace OpenMM {
class KernelFactory;
class Platform {
public:
    virtual ~Platform();
    virtual const std::string& getName() const = 0;
    void registerKernelFactory(const std::string& name, KernelFactory* factory);
    KernelFactory* kernelFactory(const std::string& name) const;   // stub accessor
    static int getNumPlatforms();
    static Platform& getPlatform(int index);
    static void registerPlatform(Platform* platform);
private:
    std::map<std::string, KernelFactory*> factories_;
};
}  // namespace OpenMM
