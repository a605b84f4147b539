// Test stub: the parts of OpenMM's ContextImpl the adapter reads (system,
// platform data, periodic box, step count).
#pragma once
#include "openmm/System.h"
#include "openmm/Vec3.h"
namespace OpenMM {
class ContextImpl {
public:
    ContextImpl(const System& system, void* platformData) : system_(system), data_(platformData) {}
    const System& getSystem() const { return system_; }
    void* getPlatformData() { return data_; }
    void getPeriodicBoxVectors(Vec3& a, Vec3& b, Vec3& c) { a = box_[0]; b = box_[1]; c = box_[2]; }
    void setPeriodicBoxVectors(const Vec3& a, const Vec3& b, const Vec3& c) { box_[0] = a; box_[1] = b; box_[2] = c; }
    long long getStepCount() const { return step_; }
    void setStepCount(long long s) { step_ = s; }
private:
    const System& system_;
    void* data_;
    Vec3 box_[3];
    long long step_ = 0;
};
}  // namespace OpenMM
