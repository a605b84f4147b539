// Test stub: the CUDA platform and its per-Context data.
#pragma once
#include <string>
#include <vector>
#include "openmm/Platform.h"
#include "openmm/cuda/CudaContext.h"
namespace OpenMM {
class CudaPlatform : public Platform {
public:
    const std::string& getName() const override { static const std::string n = "CUDA"; return n; }
    class PlatformData {
    public:
        std::vector<CudaContext*> contexts;
    };
};
}  // namespace OpenMM
