// Test stub: OpenMM's Vec3 (three doubles, indexable).
#pragma once
namespace OpenMM {
class Vec3 {
public:
    Vec3() : d_{0.0, 0.0, 0.0} {}
    Vec3(double x, double y, double z) : d_{x, y, z} {}
    double operator[](int i) const { return d_[i]; }
    double& operator[](int i) { return d_[i]; }
private:
    double d_[3];
};
}  // namespace OpenMM
