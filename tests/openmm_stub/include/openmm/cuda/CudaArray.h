// Test stub: a device array known by its pointer.
#pragma once
#include <cuda.h>
namespace OpenMM {
class CudaArray {
public:
    CUdeviceptr& getDevicePointer() { return ptr_; }
private:
    CUdeviceptr ptr_ = 0;
};
}  // namespace OpenMM
