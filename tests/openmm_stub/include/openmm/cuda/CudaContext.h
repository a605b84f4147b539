// Test stub: the CudaContext accessors the adapter uses (posq, atom index
// array, long force buffer, padding, stream, precision).
#pragma once
#include <cuda.h>
#include "openmm/common/ComputeContext.h"
#include "openmm/cuda/CudaArray.h"
namespace OpenMM {
class CudaContext : public ComputeContext {
public:
    CudaArray& getPosq() { return posq_; }
    CudaArray& getAtomIndexArray() { return atomIndex_; }
    CudaArray& getLongForceBuffer() { return force_; }
    int getPaddedNumAtoms() const { return padded_; }
    CUstream getCurrentStream() { return stream_; }
    bool getUseDoublePrecision() const { return doublePrecision_; }
    // stub setters
    void setBuffers(CUdeviceptr posq, CUdeviceptr atomIndex, CUdeviceptr force, int padded) {
        posq_.getDevicePointer() = posq; atomIndex_.getDevicePointer() = atomIndex;
        force_.getDevicePointer() = force; padded_ = padded;
    }
    void setStream(CUstream s) { stream_ = s; }
    void setUseDoublePrecision(bool yes) { doublePrecision_ = yes; }
private:
    CudaArray posq_, atomIndex_, force_;
    int padded_ = 0;
    CUstream stream_ = nullptr;
    bool doublePrecision_ = false;
};
}  // namespace OpenMM
